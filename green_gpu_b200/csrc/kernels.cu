// Non-GEMM device kernels: gathers, symmetry helpers, batched FP64 Dyson solvers.
#include "kernels.cuh"

#include <algorithm>

namespace gg {
namespace {

constexpr int TPB = 256;

__global__ void gather_pairs_kernel(const double2* __restrict__ S, const int64_t* __restrict__ pos,
                                    const int* __restrict__ op, int NQ, int n, double2* __restrict__ out) {
  // one block per (pair, Q); 32x32 tiles through shared memory for the transposed case
  __shared__ double2 tile[32][33];
  const int pq = blockIdx.x;
  const int p = pq / NQ, Q = pq % NQ;
  const double2* src = S + (pos[p] * NQ + Q) * (long)n * n;
  double2* dst = out + ((long)p * NQ + Q) * n * n;
  const int o = op[p];
  const bool cj = o & 1, tr = (o >> 1) & 1;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  for (int i0 = 0; i0 < n; i0 += 32)
    for (int j0 = 0; j0 < n; j0 += 32) {
      if (!tr) {
        for (int r = ty; r < 32; r += 8) {
          int i = i0 + r, j = j0 + tx;
          if (i < n && j < n) {
            double2 v = src[(long)i * n + j];
            dst[(long)i * n + j] = cj ? cconj(v) : v;
          }
        }
      } else {
        // dst[i][j] = src[j][i]: read rows of src (i index = j0..), write rows of dst
        for (int r = ty; r < 32; r += 8) {
          int si = j0 + r, sj = i0 + tx;  // src element (si, sj) -> dst (sj, si)
          tile[r][tx] = (si < n && sj < n) ? src[(long)si * n + sj] : make_double2(0, 0);
        }
        __syncthreads();
        for (int r = ty; r < 32; r += 8) {
          int i = i0 + r, j = j0 + tx;
          if (i < n && j < n) {
            double2 v = tile[tx][r];
            dst[(long)i * n + j] = cj ? cconj(v) : v;
          }
        }
        __syncthreads();
      }
    }
}

__global__ void gather_g_kernel(const double2* __restrict__ G, const int* __restrict__ f2r, int nk, int ns, int nts,
                                int ink, int n, double2* __restrict__ out) {
  const long nn = (long)n * n;
  const long total = (long)nk * ns * nts * nn;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
    long e = idx % nn;
    long r = idx / nn;
    int t = (int)(r % nts);
    r /= nts;
    int s = (int)(r % ns);
    int k = (int)(r / ns);
    out[idx] = G[(((long)t * ns + s) * ink + f2r[k]) * nn + e];
  }
}

__global__ void conj_where_kernel(double2* X, const int* tr, int nk, long per_k) {
  const long total = (long)nk * per_k;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
    if (tr[idx / per_k]) X[idx].y = -X[idx].y;
  }
}

__global__ void gather_blocks_kernel(const double2* __restrict__ src, const int* __restrict__ idx, long elems,
                                     long stride, int nblocks, double2* __restrict__ out) {
  const long total = (long)nblocks * elems;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    long b = i / elems, e = i % elems;
    out[i] = src[(long)idx[b] * stride + e];
  }
}

__global__ void transpose_blocks_kernel(const double2* __restrict__ in, int n, int tiles, double2* __restrict__ out) {
  __shared__ double2 t[32][33];
  const long b = blockIdx.y;
  const int ti = blockIdx.x / tiles, tj = blockIdx.x % tiles;
  const double2* src = in + b * (long)n * n;
  double2* dst = out + b * (long)n * n;
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int i = ti * 32 + r, j = tj * 32 + threadIdx.x;
    if (i < n && j < n) t[r][threadIdx.x] = src[(long)i * n + j];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int j = tj * 32 + r, i = ti * 32 + threadIdx.x;
    if (i < n && j < n) dst[(long)j * n + i] = t[threadIdx.x][r];
  }
}

__global__ void axpy_kernel(double2* y, const double2* x, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    y[i] = cadd(y[i], x[i]);
}

__global__ void scale_kernel(double2* X, long n, double s) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    X[i] = cscale(X[i], s);
}

inline unsigned grid_for(long n, int tpb = TPB) {
  long b = (n + tpb - 1) / tpb;
  return (unsigned)std::max(1L, std::min(b, 148L * 32));
}

// ----------------------------------------------------------------------------------------
// Batched Dyson solve, one CTA per (q, Omega) system.
constexpr int NB = 32;

__device__ __forceinline__ void sync() { __syncthreads(); }

__global__ void __launch_bounds__(TPB) dyson_kernel(double2* Pall, double2* Aall, int* info, int N, int solver,
                                                    int* piv_all) {
  __shared__ double2 s1[NB][NB + 1];
  __shared__ double2 s2[NB][NB + 1];
  __shared__ int s_fail;
  __shared__ int s_piv;
  __shared__ double s_red_v[TPB];
  __shared__ int s_red_i[TPB];
  const int tid = threadIdx.x;
  const long NN = (long)N * N;
  double2* P = Pall + blockIdx.x * NN;
  double2* A = Aall + blockIdx.x * NN;
  int* piv = piv_all ? piv_all + (long)blockIdx.x * N : nullptr;
  if (tid == 0) s_fail = 0;

  // --- Hermitian-symmetrise P and form A = I - P (cuda_common.cu:249-281, cu_compute_Pq.cu:44-63)
  for (long idx = tid; idx < NN; idx += TPB) {
    int i = (int)(idx / N), j = (int)(idx % N);
    if (i > j) {
      double2 lo = P[(long)i * N + j], up = P[(long)j * N + i];
      double re = 0.5 * (lo.x + up.x), im = 0.5 * (lo.y - up.y);
      P[(long)i * N + j] = make_double2(re, im);
      P[(long)j * N + i] = make_double2(re, -im);
      A[(long)i * N + j] = make_double2(-re, -im);
      A[(long)j * N + i] = make_double2(-re, im);
    } else if (i == j) {
      double d = P[(long)i * N + i].x;
      P[(long)i * N + i] = make_double2(d, 0.0);
      A[(long)i * N + i] = make_double2(1.0 - d, 0.0);
    }
  }
  sync();

  if (solver == GG_SOLVER_CHOLESKY) {
    // --- blocked right-looking Cholesky, A = L L^H (lower, in place)
    for (int j0 = 0; j0 < N; j0 += NB) {
      const int jb = min(NB, N - j0);
      for (int e = tid; e < jb * jb; e += TPB) {
        int r = e / jb, c = e % jb;
        s1[r][c] = A[(long)(j0 + r) * N + j0 + c];
      }
      sync();
      if (tid < 32) {
        // warp-level unblocked factorisation of the diagonal block; lane r owns row r
        for (int c = 0; c < jb; ++c) {
          __syncwarp();
          double d = s1[c][c].x;
          bool bad = !(d > 0.0);
          double sq = sqrt(bad ? 1.0 : d);
          __syncwarp();
          if (tid == c) {
            s1[c][c] = make_double2(sq, 0.0);
            if (bad && s_fail == 0) s_fail = j0 + c + 1;
          }
          if (tid > c && tid < jb) s1[tid][c] = cscale(s1[tid][c], 1.0 / sq);
          __syncwarp();
          if (tid > c && tid < jb) {
            double2 lrc = s1[tid][c];
            for (int c2 = c + 1; c2 <= tid; ++c2) s1[tid][c2] = csub(s1[tid][c2], cmulc(lrc, s1[c2][c]));
          }
        }
      }
      sync();
      for (int e = tid; e < jb * jb; e += TPB) {
        int r = e / jb, c = e % jb;
        if (c <= r) A[(long)(j0 + r) * N + j0 + c] = s1[r][c];
      }
      // panel: rows below solve x L_jj^H = a
      for (int i = j0 + jb + tid; i < N; i += TPB) {
        double2 x[NB];
        double2* row = A + (long)i * N + j0;
#pragma unroll
        for (int c = 0; c < NB; ++c) {
          if (c < jb) {
            double2 v = row[c];
#pragma unroll
            for (int c2 = 0; c2 < NB; ++c2)
              if (c2 < c) v = csub(v, cmulc(x[c2], s1[c][c2]));
            x[c] = cscale(v, 1.0 / s1[c][c].x);
            row[c] = x[c];
          }
        }
      }
      sync();
      // trailing update A[i][j] -= sum_c L[i][c] conj(L[j][c]) for the lower trailing part
      const int t0 = j0 + jb;
      const int ntl = (N - t0 + NB - 1) / NB;
      for (int ti = 0; ti < ntl; ++ti)
        for (int tj = 0; tj <= ti; ++tj) {
          const int i0 = t0 + ti * NB, jj0 = t0 + tj * NB;
          for (int e = tid; e < NB * NB; e += TPB) {
            int r = e / NB, c = e % NB;
            s1[r][c] = (i0 + r < N && c < jb) ? A[(long)(i0 + r) * N + j0 + c] : make_double2(0, 0);
            s2[r][c] = (jj0 + r < N && c < jb) ? A[(long)(jj0 + r) * N + j0 + c] : make_double2(0, 0);
          }
          sync();
          const int col = tid & 31, rb = tid >> 5;
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int r = rb + 8 * q;
            double2 acc = make_double2(0, 0);
            for (int c = 0; c < jb; ++c) acc = cadd(acc, cmulc(s1[r][c], s2[col][c]));
            if (i0 + r < N && jj0 + col < N && jj0 + col <= i0 + r) {
              double2* a = A + (long)(i0 + r) * N + jj0 + col;
              *a = csub(*a, acc);
            }
          }
          sync();
        }
    }
  } else {
    // --- unblocked right-looking LU with partial pivoting (row interchanges recorded in piv)
    for (int j = 0; j < N; ++j) {
      double best = -1.0;
      int bi = j;
      for (int i = j + tid; i < N; i += TPB) {
        double2 v = A[(long)i * N + j];
        double m = fabs(v.x) + fabs(v.y);
        if (m > best) { best = m; bi = i; }
      }
      s_red_v[tid] = best;
      s_red_i[tid] = bi;
      sync();
      for (int s = TPB / 2; s > 0; s >>= 1) {
        if (tid < s) {
          if (s_red_v[tid + s] > s_red_v[tid] ||
              (s_red_v[tid + s] == s_red_v[tid] && s_red_i[tid + s] < s_red_i[tid])) {
            s_red_v[tid] = s_red_v[tid + s];
            s_red_i[tid] = s_red_i[tid + s];
          }
        }
        sync();
      }
      if (tid == 0) {
        s_piv = s_red_i[0];
        piv[j] = s_piv;
        if (!(s_red_v[0] > 0.0) && s_fail == 0) s_fail = j + 1;
      }
      sync();
      const int p = s_piv;
      if (p != j)
        for (int c = tid; c < N; c += TPB) {
          double2 t = A[(long)j * N + c];
          A[(long)j * N + c] = A[(long)p * N + c];
          A[(long)p * N + c] = t;
        }
      sync();
      double2 d = A[(long)j * N + j];
      double dn = d.x * d.x + d.y * d.y;
      double2 inv = dn > 0.0 ? make_double2(d.x / dn, -d.y / dn) : make_double2(0.0, 0.0);
      for (int i = j + 1 + tid; i < N; i += TPB) A[(long)i * N + j] = cmul(A[(long)i * N + j], inv);
      sync();
      const int rem = N - j - 1;
      for (long e = tid; e < (long)rem * rem; e += TPB) {
        int i = j + 1 + (int)(e / rem), c = j + 1 + (int)(e % rem);
        A[(long)i * N + c] = csub(A[(long)i * N + c], cmul(A[(long)i * N + j], A[(long)j * N + c]));
      }
      sync();
    }
  }

  // --- solve A Y = P (P holds the Hermitian-symmetrised right-hand side; Y overwrites P)
  if (solver == GG_SOLVER_CHOLESKY) {
    // forward: Z = L^{-1} P by block rows
    for (int i0 = 0; i0 < N; i0 += NB) {
      const int ib = min(NB, N - i0);
      // update P[i0:i0+ib, :] -= L[i0:i0+ib, 0:i0] P[0:i0, :]
      for (int c0 = 0; c0 < N; c0 += NB) {
        const int col = tid & 31, rb = tid >> 5;
        double2 acc[4] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
        for (int k0 = 0; k0 < i0; k0 += NB) {
          for (int e = tid; e < NB * NB; e += TPB) {
            int r = e / NB, c = e % NB;
            s1[r][c] = (r < ib) ? A[(long)(i0 + r) * N + k0 + c] : make_double2(0, 0);
            s2[r][c] = (c0 + c < N) ? P[(long)(k0 + r) * N + c0 + c] : make_double2(0, 0);
          }
          sync();
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int r = rb + 8 * q;
            for (int c = 0; c < NB; ++c) acc[q] = cadd(acc[q], cmul(s1[r][c], s2[c][col]));
          }
          sync();
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int r = rb + 8 * q;
          if (r < ib && c0 + col < N) {
            double2* x = P + (long)(i0 + r) * N + c0 + col;
            *x = csub(*x, acc[q]);
          }
        }
      }
      // diagonal block L_ii into s1, then column-parallel forward substitution
      for (int e = tid; e < NB * NB; e += TPB) {
        int r = e / NB, c = e % NB;
        s1[r][c] = (r < ib && c < ib) ? A[(long)(i0 + r) * N + i0 + c] : make_double2(0, 0);
      }
      sync();
      for (int c = tid; c < N; c += TPB) {
        double2 z[NB];
#pragma unroll
        for (int r = 0; r < NB; ++r) {
          if (r < ib) {
            double2 v = P[(long)(i0 + r) * N + c];
#pragma unroll
            for (int r2 = 0; r2 < NB; ++r2)
              if (r2 < r) v = csub(v, cmul(s1[r][r2], z[r2]));
            z[r] = cscale(v, 1.0 / s1[r][r].x);
            P[(long)(i0 + r) * N + c] = z[r];
          }
        }
      }
      sync();
    }
    // backward: Y = L^{-H} Z by block rows from the bottom
    const int nblk = (N + NB - 1) / NB;
    for (int bi = nblk - 1; bi >= 0; --bi) {
      const int i0 = bi * NB;
      const int ib = min(NB, N - i0);
      for (int c0 = 0; c0 < N; c0 += NB) {
        const int col = tid & 31, rb = tid >> 5;
        double2 acc[4] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
        for (int k0 = i0 + ib; k0 < N; k0 += NB) {
          for (int e = tid; e < NB * NB; e += TPB) {
            int r = e / NB, c = e % NB;
            // s1[r][c] = (L^H)[i0 + r][k0 + c] = conj(L[k0 + c][i0 + r])
            s1[r][c] = (r < ib && k0 + c < N) ? cconj(A[(long)(k0 + c) * N + i0 + r]) : make_double2(0, 0);
            s2[r][c] = (k0 + r < N && c0 + c < N) ? P[(long)(k0 + r) * N + c0 + c] : make_double2(0, 0);
          }
          sync();
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int r = rb + 8 * q;
            for (int c = 0; c < NB; ++c) acc[q] = cadd(acc[q], cmul(s1[r][c], s2[c][col]));
          }
          sync();
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int r = rb + 8 * q;
          if (r < ib && c0 + col < N) {
            double2* x = P + (long)(i0 + r) * N + c0 + col;
            *x = csub(*x, acc[q]);
          }
        }
      }
      for (int e = tid; e < NB * NB; e += TPB) {
        int r = e / NB, c = e % NB;
        s1[r][c] = (r < ib && c < ib) ? A[(long)(i0 + r) * N + i0 + c] : make_double2(0, 0);
      }
      sync();
      for (int c = tid; c < N; c += TPB) {
        double2 y[NB];
#pragma unroll
        for (int rr = NB - 1; rr >= 0; --rr) {
          if (rr < ib) {
            double2 v = P[(long)(i0 + rr) * N + c];
#pragma unroll
            for (int r2 = NB - 1; r2 >= 0; --r2)
              if (r2 > rr && r2 < ib) v = csub(v, cmulc(y[r2], s1[r2][rr]));
            y[rr] = cscale(v, 1.0 / s1[rr][rr].x);
            P[(long)(i0 + rr) * N + c] = y[rr];
          }
        }
      }
      sync();
    }
    // the reference's column-major solve returns (A^{-1} P)^H in row-major terms
    for (long idx = tid; idx < NN; idx += TPB) {
      int i = (int)(idx / N), j = (int)(idx % N);
      if (i > j) {
        double2 a = P[(long)i * N + j], b = P[(long)j * N + i];
        P[(long)i * N + j] = cconj(b);
        P[(long)j * N + i] = cconj(a);
      } else if (i == j) {
        P[(long)i * N + i].y = -P[(long)i * N + i].y;
      }
    }
  } else {
    // apply row interchanges to the right-hand side, then unit-lower and upper solves
    for (int j = 0; j < N; ++j) {
      const int p = piv[j];
      if (p != j)
        for (int c = tid; c < N; c += TPB) {
          double2 t = P[(long)j * N + c];
          P[(long)j * N + c] = P[(long)p * N + c];
          P[(long)p * N + c] = t;
        }
      sync();
    }
    for (int c = tid; c < N; c += TPB) {
      for (int r = 1; r < N; ++r) {
        double2 v = P[(long)r * N + c];
        for (int r2 = 0; r2 < r; ++r2) v = csub(v, cmul(A[(long)r * N + r2], P[(long)r2 * N + c]));
        P[(long)r * N + c] = v;
      }
      for (int r = N - 1; r >= 0; --r) {
        double2 v = P[(long)r * N + c];
        for (int r2 = r + 1; r2 < N; ++r2) v = csub(v, cmul(A[(long)r * N + r2], P[(long)r2 * N + c]));
        double2 d = A[(long)r * N + r];
        double dn = d.x * d.x + d.y * d.y;
        P[(long)r * N + c] = dn > 0.0 ? cmul(v, make_double2(d.x / dn, -d.y / dn)) : make_double2(0, 0);
      }
    }
    sync();
    // Hermitian symmetrisation of the result (cugw_qpt.cu:314-316)
    for (long idx = tid; idx < NN; idx += TPB) {
      int i = (int)(idx / N), j = (int)(idx % N);
      if (i > j) {
        double2 lo = P[(long)i * N + j], up = P[(long)j * N + i];
        double re = 0.5 * (lo.x + up.x), im = 0.5 * (lo.y - up.y);
        P[(long)i * N + j] = make_double2(re, im);
        P[(long)j * N + i] = make_double2(re, -im);
      } else if (i == j) {
        P[(long)i * N + i].y = 0.0;
      }
    }
  }
  sync();
  if (tid == 0) info[blockIdx.x] = s_fail;
}

__global__ void hermitize_kernel(double2* Pall, int N) {
  double2* P = Pall + blockIdx.x * (long)N * N;
  for (long idx = threadIdx.x; idx < (long)N * N; idx += blockDim.x) {
    int i = (int)(idx / N), j = (int)(idx % N);
    if (i > j) {
      double2 lo = P[(long)i * N + j], up = P[(long)j * N + i];
      double re = 0.5 * (lo.x + up.x), im = 0.5 * (lo.y - up.y);
      P[(long)i * N + j] = make_double2(re, im);
      P[(long)j * N + i] = make_double2(re, -im);
    } else if (i == j) {
      P[(long)i * N + i].y = 0.0;
    }
  }
}

__global__ void hartree_coeff_kernel(const double2* __restrict__ V, const double2* __restrict__ D, int npairs, int NQ,
                                     int n, double scale, double2* c) {
  // one block per Q; c[Q] += scale * sum_p sum_ab V[p][Q][a][b] D[p][b][a]
  __shared__ double2 red[TPB];
  const int Q = blockIdx.x;
  const long nn = (long)n * n;
  double2 acc = make_double2(0, 0);
  for (int p = 0; p < npairs; ++p) {
    const double2* v = V + ((long)p * NQ + Q) * nn;
    const double2* d = D + (long)p * nn;
    for (long e = threadIdx.x; e < nn; e += TPB) {
      int a = (int)(e / n), b = (int)(e % n);
      acc = cadd(acc, cmul(v[e], d[(long)b * n + a]));
    }
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = TPB / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = cadd(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) c[Q] = cadd(c[Q], cscale(red[0], scale));
}

__global__ void hartree_apply_kernel(const double2* __restrict__ V, const double2* __restrict__ c, int NQ, int n,
                                     double2* J) {
  const long nn = (long)n * n;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < nn; e += (long)gridDim.x * blockDim.x) {
    double2 acc = make_double2(0, 0);
    for (int Q = 0; Q < NQ; ++Q) acc = cadd(acc, cmul(c[Q], V[(long)Q * nn + e]));
    J[e] = acc;
  }
}

}  // namespace

void launch_gather_pairs(const double2* S, const int64_t* pos_d, const int* op_d, int npairs, int NQ, int n,
                         double2* out, cudaStream_t st) {
  if (npairs <= 0) return;
  gather_pairs_kernel<<<npairs * NQ, 256, 0, st>>>(S, pos_d, op_d, NQ, n, out);
  GG_CHECK_LAUNCH();
}

void launch_gather_g(const double2* G, const int* f2r, int nk, int ns, int nts, int ink, int n, double2* out,
                     cudaStream_t st) {
  long total = (long)nk * ns * nts * n * n;
  gather_g_kernel<<<grid_for(total), TPB, 0, st>>>(G, f2r, nk, ns, nts, ink, n, out);
  GG_CHECK_LAUNCH();
}

void launch_conj_where(double2* X, const int* tr, int nk, long per_k, cudaStream_t st) {
  conj_where_kernel<<<grid_for((long)nk * per_k), TPB, 0, st>>>(X, tr, nk, per_k);
  GG_CHECK_LAUNCH();
}

void launch_gather_blocks(const double2* src, const int* idx, int nblocks, long elems, long stride, double2* out,
                          cudaStream_t st) {
  if (nblocks <= 0) return;
  gather_blocks_kernel<<<grid_for((long)nblocks * elems), TPB, 0, st>>>(src, idx, elems, stride, nblocks, out);
  GG_CHECK_LAUNCH();
}

namespace {
__device__ __forceinline__ void x2c_block(int ss, int& a, int& b) {
  a = ss & 1;
  b = (ss == 1 || ss == 2) ? 1 : 0;
}

__global__ void x2c_split_kernel(const double2* in, long nouter, long ninner, int n, int nblk, double2* out) {
  const long nn = (long)n * n, total = nouter * nblk * ninner * nn;
  const int n2 = 2 * n;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long ij = e % nn;
    long r = e / nn;
    const long kin = r % ninner;
    r /= ninner;
    const int ss = (int)(r % nblk);
    const long o = r / nblk;
    int a, b;
    x2c_block(ss, a, b);
    const int i = (int)(ij / n), j = (int)(ij % n);
    out[e] = in[((o * ninner + kin) * n2 + a * n + i) * n2 + b * n + j];
  }
}

__global__ void x2c_merge_kernel(const double2* in, long nouter, long ninner, int n, int nblk, double2* out) {
  const int n2 = 2 * n;
  const long nn = (long)n * n, mm = (long)n2 * n2, total = nouter * ninner * mm;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const int J = (int)(e % n2), I = (int)((e / n2) % n2);
    const long r = e / mm, kin = r % ninner, o = r / ninner;
    const int a = I >= n, b = J >= n, i = I - a * n, j = J - b * n;
    // block index of (a, b): aa 0, bb 1, ab 2, ba 3
    const int ss = (a == b) ? a : (a == 0 ? 2 : 3);
    double2 v;
    if (ss == 3 && nblk == 3) {
      const double2 u = in[((o * nblk + 2) * ninner + kin) * nn + (long)j * n + i];
      v = make_double2(u.x, -u.y);
    } else {
      v = in[((o * nblk + ss) * ninner + kin) * nn + (long)i * n + j];
    }
    out[e] = v;
  }
}
}  // namespace

void launch_x2c_split(const double2* in, long nouter, long ninner, int n, int nblk, double2* out, cudaStream_t st) {
  x2c_split_kernel<<<grid_for(nouter * nblk * ninner * (long)n * n), TPB, 0, st>>>(in, nouter, ninner, n, nblk, out);
  GG_CHECK_LAUNCH();
}

void launch_x2c_merge(const double2* in, long nouter, long ninner, int n, int nblk, double2* out, cudaStream_t st) {
  x2c_merge_kernel<<<grid_for(nouter * ninner * 4L * n * n), TPB, 0, st>>>(in, nouter, ninner, n, nblk, out);
  GG_CHECK_LAUNCH();
}

namespace {
__global__ void info_collect_kernel(const int* info, int count, int base, int* err) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    if (info[i] != 0 && atomicCAS(&err[0], 0, 1) == 0) {
      err[1] = base + i;
      err[2] = info[i];
    }
}
}  // namespace

void launch_info_collect(const int* info, int count, int base, int* err, cudaStream_t st) {
  info_collect_kernel<<<grid_for(count), TPB, 0, st>>>(info, count, base, err);
  GG_CHECK_LAUNCH();
}

void launch_transpose_blocks(const double2* in, long nblocks, int n, double2* out, cudaStream_t st) {
  if (nblocks <= 0 || n <= 0) return;
  if (nblocks > 65535) throw Error(GG_ERR_ARG, "transpose: too many blocks for one launch");
  const int tiles = (n + 31) / 32;
  transpose_blocks_kernel<<<dim3((unsigned)(tiles * tiles), (unsigned)nblocks), dim3(32, 8), 0, st>>>(in, n, tiles, out);
  GG_CHECK_LAUNCH();
}

void launch_axpy(double2* y, const double2* x, long n, cudaStream_t st) {
  axpy_kernel<<<grid_for(n), TPB, 0, st>>>(y, x, n);
  GG_CHECK_LAUNCH();
}

void launch_scale(double2* X, long n, double s, cudaStream_t st) {
  scale_kernel<<<grid_for(n), TPB, 0, st>>>(X, n, s);
  GG_CHECK_LAUNCH();
}

void launch_fill_zero(double2* X, long n, cudaStream_t st) {
  GG_CUDA(cudaMemsetAsync(X, 0, sizeof(double2) * n, st));
}

void launch_dyson(double2* P, double2* A, int* info, int nsys, int N, int solver, int* piv_ws, cudaStream_t st) {
  if (nsys <= 0) return;
  dyson_kernel<<<nsys, TPB, 0, st>>>(P, A, info, N, solver, piv_ws);
  GG_CHECK_LAUNCH();
}

void launch_hermitian_symmetrize(double2* P, int nsys, int N, cudaStream_t st) {
  if (nsys <= 0) return;
  hermitize_kernel<<<nsys, TPB, 0, st>>>(P, N);
  GG_CHECK_LAUNCH();
}

void launch_hartree_coeff(const double2* V, const double2* D, int npairs, int NQ, int n, double scale, double2* c,
                          cudaStream_t st) {
  hartree_coeff_kernel<<<NQ, TPB, 0, st>>>(V, D, npairs, NQ, n, scale, c);
  GG_CHECK_LAUNCH();
}

void launch_hartree_apply(const double2* V, const double2* c, int NQ, int n, double2* J, cudaStream_t st) {
  hartree_apply_kernel<<<grid_for((long)n * n), TPB, 0, st>>>(V, c, NQ, n, J);
  GG_CHECK_LAUNCH();
}

}  // namespace gg
