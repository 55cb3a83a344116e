// Non-GEMM device kernels of the GW / HF path (gathers, symmetry unfolding, the batched
// FP64 Dyson solvers and small reductions).  Host launchers; all run on `stream`.
#pragma once

#include "common.cuh"

namespace gg {

// V(k, k1) gather: out[p][Q][i][j] = op_p(S[pos_p][Q])[i][j], op bit0 = conj, bit1 = transpose.
void launch_gather_pairs(const double2* S, const int64_t* pos_d, const int* op_d, int npairs, int NQ, int n,
                         double2* out, cudaStream_t st);

// Gather full-BZ G from the IBZ input (layout [t][s][ink][i][j]):
// out[k][s][t][i][j] = G[t][s][f2r[k]][i][j] (optionally conjugated later).
void launch_gather_g(const double2* G_tskij, const int* k_f2r_d, int nk, int ns, int nts, int ink, int n,
                     double2* out, cudaStream_t st);

// out[k][...][i][j] = conj(...) for every k with tr[k] != 0; per_k elements per k.
void launch_conj_where(double2* X, const int* tr_d, int nk, long per_k, cudaStream_t st);

// gather blocks: out[p][e] = src[idx[p] * src_stride + e] for e < elems
void launch_gather_blocks(const double2* src, const int* idx_d, int nblocks, long elems, long src_stride,
                          double2* out, cudaStream_t st);
// y += x (n complex numbers)
void launch_axpy(double2* y, const double2* x, long n, cudaStream_t st);
// err[0..2] <- (1, base + i, info[i]) for a failing system i (info != 0), if none is recorded yet
void launch_info_collect(const int* info, int count, int base, int* err, cudaStream_t st);

// Two-component (X2C) spin blocks.  A spinor matrix of order 2n holds the blocks aa (0,0),
// bb (n,n), ab (0,n) and ba (n,0).  Block ss of the pseudo-spin order is (row, col) =
// (ss % 2, ss == 0 ? 0 : ss == 1 ? 1 : ss == 2 ? 1 : 0), i.e. aa, bb, ab, ba (the order of the
// reference's copy_Gk_2c with minus_t = false and copy_Sigma_2c, gw_gpu_kernel.cpp:523-551,
// cugw_qkpt.cu:382-403).
// split: in [nouter][ninner][2n][2n] -> out [nouter][nblk][ninner][n][n] (nblk = 3 or 4)
void launch_x2c_split(const double2* in, long nouter, long ninner, int n, int nblk, double2* out, cudaStream_t st);
// merge: in [nouter][nblk][ninner][n][n] -> out [nouter][ninner][2n][2n]; with nblk = 3 the ba
// block is the adjoint of ab (cuda_common.cu:176-201)
void launch_x2c_merge(const double2* in, long nouter, long ninner, int n, int nblk, double2* out, cudaStream_t st);

// out[b][i][j] = in[b][j][i] for nblocks n x n matrices (32 x 32 tiles through shared memory)
void launch_transpose_blocks(const double2* in, long nblocks, int n, double2* out, cudaStream_t st);

// scale: X *= s
void launch_scale(double2* X, long n, double s, cudaStream_t st);
void launch_fill_zero(double2* X, long n, cudaStream_t st);

// Batched Dyson solve for `nsys` systems of size N x N stored contiguously in P (in place):
// P <- Hermitian-symmetrise(P); A = I - P; Cholesky: P <- (A^{-1} P)^H, LU: P <- sym(A^{-1} P).
// `A` is a workspace of the same size, `info` receives per-system status (0 ok; Cholesky:
// index+1 of the first non-positive pivot; LU: index+1 of the first zero pivot).
void launch_dyson(double2* P, double2* A, int* info, int nsys, int N, int solver, int* piv_ws, cudaStream_t st);

// Hermitian symmetrisation only (cuda_common.cu:249-281), nsys matrices in place.
void launch_hermitian_symmetrize(double2* P, int nsys, int N, cudaStream_t st);

// Hartree coefficients: c[Q] += scale * sum_{ab} V[p][Q][a][b] D[p][b][a] over p (pairs).
void launch_hartree_coeff(const double2* V, const double2* D, int npairs, int NQ, int n, double scale, double2* c,
                          cudaStream_t st);
// J[i][j] = sum_Q c[Q] V[Q][i][j]
void launch_hartree_apply(const double2* V, const double2* c, int NQ, int n, double2* J, cudaStream_t st);

}  // namespace gg
