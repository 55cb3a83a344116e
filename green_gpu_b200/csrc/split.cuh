// Split-precision (Ozaki-sliced INT8 tensor-core) complex GEMM for the dominant contractions.
#pragma once

#include "context.cuh"
#include "zgemm.cuh"

namespace gg {

struct SplitGemm;
// Per-context engine (workspace for slices); throws if the path is unavailable.
SplitGemm* split_engine(gg_context* c);
// Same contract as zgemm() for descriptors with KB >= 1; FP64 in, FP64 out.
int split_zgemm(SplitGemm* e, const ZgemmDesc& d, int slices, cudaStream_t st);
void split_release(SplitGemm* e);
// Make the next launch of this engine run the time-out test (short wait limit, one accumulator
// release withheld by CTA 0), so that its failure path is exercised without any fault.
void split_arm_timeout_test(SplitGemm* e);
// Device addresses of the engine's work buffers (appended to `out`): a graph that captured
// split GEMMs stays valid only while none of them was reallocated.
void split_buffers(const SplitGemm* e, std::vector<const void*>& out);
// Raise if any split GEMM enqueued on `st` since the last check timed out (synchronises `st`).
void split_check(SplitGemm* e, cudaStream_t st);

}  // namespace gg
