// Split-precision (Ozaki-sliced INT8 tensor-core) complex GEMM for the dominant contractions.
#pragma once

#include "context.cuh"
#include "zgemm.cuh"

namespace gg {

// Epilogue that also records the exact row maxima of the product for the next split GEMM: with
// m = mq div_m + mr and n = nq div_n + nr, |Re C|, |Im C| of (m, n) of batch b count towards
// entry ex[b * s_b + mq * s_mq + mr * s_mr + nq * s_nq], which receives (by atomicMax over all
// tiles and batches) the exponent e with max < 2^e - the exponent the slicing pass would compute
// for that row / column of the next GEMM's operand.  ex must start below every exponent (bytes
// 0x80).  No split-K.
struct SplitRowMax {
  int on = 0;
  int div_m = 1, div_n = 1;
  long s_b = 0, s_mq = 0, s_mr = 0, s_nq = 0;
  int* ex = nullptr;
};

// Geometry of a split GEMM's operand planes (as split_zgemm lays them out for descriptor d).
struct SplitPlanes {
  int rows_a_pad = 0, rows_b_pad = 0, ncol_pad = 0;
  long nkb = 0;
  long batch = 0;
  size_t a_bytes = 0, b_bytes = 0;  // planes of every batch
};
SplitPlanes split_planes_for(const ZgemmDesc& d, int S);

struct SplitGemm;
// Per-context engine (workspace for slices); throws if the path is unavailable.
SplitGemm* split_engine(gg_context* c);
// Same contract as zgemm() for descriptors with KB >= 1; FP64 in, FP64 out.
int split_zgemm(SplitGemm* e, const ZgemmDesc& d, int slices, cudaStream_t st);
// Same as split_zgemm, recording the row maxima of C as described by mx (alpha = 1, beta = 0).
int split_zgemm_rowmax(SplitGemm* e, const ZgemmDesc& d, int slices, const SplitRowMax& mx, cudaStream_t st);
// split_zgemm with operand exponents given (ea [batch][rows_a_pad], eb [batch][N], as
// split_zgemm_rowmax records them; NULL: computed by the exponent pass as usual), optionally
// recording the row maxima of its own product (mx may be NULL).
int split_zgemm_exps(SplitGemm* e, const ZgemmDesc& d, int slices, const int* ea, const int* eb, cudaStream_t st,
                     const SplitRowMax* mx = nullptr);
void split_release(SplitGemm* e);
// Make the next launch of this engine run the time-out test (short wait limit, one accumulator
// release withheld by CTA 0), so that its failure path is exercised without any fault.
void split_arm_timeout_test(SplitGemm* e);
// Tile autotuner of the INT8 engine (per engine): the first call of every GEMM shape that
// overwrites its output and is not being captured times each candidate tile width and split-K
// factor with CUDA events and keeps the fastest for every later call of that shape.
void split_set_autotune(SplitGemm* e, bool on);
// One line per tuned shape: "S M N K batch: BN b split-K s (t ms)".
const char* split_autotune_report(const SplitGemm* e);
// Device addresses of the engine's work buffers (appended to `out`): a graph that captured
// split GEMMs stays valid only while none of them was reallocated.
void split_buffers(const SplitGemm* e, std::vector<const void*>& out);
// Raise if any split GEMM enqueued on `st` since the last check timed out (synchronises `st`).
void split_check(SplitGemm* e, cudaStream_t st);

}  // namespace gg
