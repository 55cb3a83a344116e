// Fused tail of the GW Sigma contraction of one (k, q) pair (FP64 tensor cores):
//
//   C[t][j][i] += alpha * sum_Q sum_c (sum_l X[t][Q][j][l] G[t][l][c]) conj(V[Q][i][c])
//
// i.e. Z = X G followed by the reduction of Z V^+ over (Q, c), without writing Z.  The
// reference does the same work as GEMM 1 (V G, before the contraction with W) and GEMM 3 (the
// reduction with V) of compute_second_tau_contraction, src/cugw_qkpt.cu:295-332, each a
// batched ZGEMM whose product goes through device memory.
//   X: X + t * x_t + (Q * n + j) * n + l     (the output of the Sigma contraction V^T W~)
//   G: G + (t * n + l) * n + c
//   V: V + (Q * n + i) * n + c
//   C: C + t * c_t + j * n + i
#pragma once

#include "common.cuh"

namespace gg {

// true when the orbital count fits the kernel (five n x n blocks in shared memory) and its
// partial sums fit `work_elems` complex elements
bool sigma_tail_supported(int n, int T, long work_elems);

// Launches the fused kernel and the ordered reduction of its partial sums (deterministic);
// `gauss` selects the three-product complex form.  Returns the number of launches.
int sigma_tail(const double2* X, long x_t, const double2* G, const double2* V, int n, int NQ, int T, double2* C,
               long c_t, double2 alpha, bool gauss, double2* work, long work_elems, cudaStream_t st);

}  // namespace gg
