// Batched complex FP64 GEMM on the FP64 tensor path (DMMA, mma.sync m8n8k4 f64).
//
// C[b] = alpha * sum_{kb} op(A[b,kb]) op(B[b,kb]) + beta * C[b]
//
// One engine serves every contraction of the FP64 path (P0, Sigma, HF exchange, IR
// transforms, k-symmetry rotations).  Operands are addressed through strides so that no
// transpose/conjugate copies are ever materialised (the reference spends GEAM + RSCAL
// passes on that: src/cugw_qkpt.cu:115-173, src/cuhf_utils.cu:90-106):
//   A(m, k) = A + off_b(A) + kb * a_kb + map(m; a_m_split, a_m_hi, a_m_lo) + k * a_k
//   B(k, n) = B + off_b(B) + kb * b_kb + k * b_k + map(n; b_n_split, b_n_hi, b_n_lo)
//   C(m, n) = C + off_b(C) + map(m; ...) + map(n; ...)
// where map(i; s, hi, lo) = (i / s) * hi + (i % s) * lo for s > 0 and i * lo for s == 0,
// and the batch index decomposes into three levels (b0 fastest) with their own strides.
#pragma once

#include "common.cuh"

namespace gg {

struct IdxMap {
  int split = 0;   // 0: single level
  long hi = 0;
  long lo = 0;
  __host__ __device__ __forceinline__ long operator()(long i) const {
    return split > 0 ? (i / split) * hi + (i % split) * lo : i * lo;
  }
};

struct ZgemmDesc {
  int M = 0, N = 0, K = 0, KB = 1;
  const double2* A = nullptr;
  IdxMap a_m;
  long a_k = 0, a_kb = 0;
  const double2* B = nullptr;
  IdxMap b_n;
  long b_k = 0, b_kb = 0;
  double2* C = nullptr;
  IdxMap c_m, c_n;
  int nb0 = 1, nb1 = 1, nb2 = 1;
  long a_b0 = 0, a_b1 = 0, a_b2 = 0;
  long b_b0 = 0, b_b1 = 0, b_b2 = 0;
  long c_b0 = 0, c_b1 = 0, c_b2 = 0;
  double2 alpha = {1.0, 0.0};
  double2 beta = {0.0, 0.0};
  int conjA = 0, conjB = 0;
  // 1: three real products per complex product, re = ar br - ai bi and
  // im = (ar + ai)(br + bi) - ar br - ai bi (normwise error still O(u K |A||B|), about
  // 1e-16 relative, but not componentwise).  Used only inside the split-precision build, whose
  // error budget is six orders larger; the FP64 path keeps the four-product form.
  int gauss = 0;
  int splits = 1;            // split-K factor (deterministic: partials + ordered reduction)
  double2* work = nullptr;   // [splits][batch][M][N] when splits > 1
  long work_elems = 0;       // capacity of `work` in complex elements
};

// Launches on `stream`; chooses split-K automatically when `d.work` has room and the
// natural grid under-fills the device.  Returns the number of kernel launches issued.
int zgemm(const ZgemmDesc& d, cudaStream_t stream);

}  // namespace gg
