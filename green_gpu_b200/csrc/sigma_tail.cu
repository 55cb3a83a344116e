// Fused Sigma tail (see sigma_tail.cuh) on the FP64 tensor path.
//
// One CTA per (tau, range of Q), NT = ceil(n / 8) warps; warp w owns rows j = 8w..8w+7.
// Per Q, with X[t][Q], V[Q] (double-buffered, cp.async) and G[t]^T (staged once) in shared
// memory, each warp
//   1. forms its 8 rows of Z = X G in column chunks of up to four 8-wide tiles (DMMA,
//      accumulators in registers);
//   2. turns each chunk's accumulator fragments into A fragments of the next product by
//      warp shuffles within the lane quad (the accumulator of m8n8k4 holds two adjacent
//      columns per lane, the A operand one column per lane);
//   3. accumulates Z V^+ for its rows over the chunk's columns into the Sigma accumulators,
//      which stay in registers across all Q of the CTA.
// Z never leaves the registers.  The CTA writes its partial Sigma[t] for its Q range;
// a second kernel adds the partials in a fixed order (deterministic) times alpha to C.
//
// Shared memory: five n x S blocks (G^T, 2 x X, 2 x V), row stride S >= n with S = 4 (mod 8),
// so the fragment loads (row = lane / 4, column = lane % 4) hit eight distinct 16-byte bank
// groups per quarter warp.  Columns n..S-1 are zero (the reductions over l and c read up to
// the next multiple of 4); rows are read clamped to n - 1, which touches only output rows and
// columns >= n, and those are never stored.
#include "sigma_tail.cuh"

#include "dmma.cuh"

#include <algorithm>
#include <atomic>

namespace gg {
namespace {

constexpr int CH = 7;  // Z column tiles per chunk

__host__ __device__ __forceinline__ int row_stride(int n) {
  int s = (n + 3) & ~3;
  if ((s & 7) != 4) s += 4;
  return s;
}

struct TailArgs {
  const double2* X;
  long x_t;
  const double2* G;
  const double2* V;
  double2* P;  // partials [t][split][n][n]
  int n, NQ, SQ;
};

template <int NT, bool G3>
__global__ void __launch_bounds__(32 * NT, 1) sigma_tail_kernel(TailArgs a) {
  extern __shared__ __align__(16) double2 sm[];
  constexpr int NTH = 32 * NT;
  const int n = a.n, S = row_stride(n), nn = n * n;
  const int tile = n * S;
  double2* Gs = sm;             // G^T[c][l]
  double2* Xs = sm + tile;      // two stages
  double2* Vs = sm + 3 * tile;  // two stages
  const int t = blockIdx.x / a.SQ, split = blockIdx.x % a.SQ;
  const int q0 = (int)((long)a.NQ * split / a.SQ), q1 = (int)((long)a.NQ * (split + 1) / a.SQ);
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int fr = lane >> 2, fk = lane & 3;

  // zero the pad columns of the five blocks (the copies write columns < n only)
  if (S > n)
    for (int e = tid; e < 5 * n * (S - n); e += NTH) sm[(e / (S - n)) * S + n + e % (S - n)] = make_double2(0.0, 0.0);

  auto issue = [&](int q, int b) {
    const double2* xg = a.X + (long)t * a.x_t + (long)q * nn;
    const double2* vg = a.V + (long)q * nn;
    for (int r = w; r < 2 * n; r += NT) {
      const bool isx = r < n;
      const int rr = isx ? r : r - n;
      const double2* src = (isx ? xg : vg) + rr * n;
      double2* dst = (isx ? Xs : Vs) + b * tile + rr * S;
      for (int c = lane; c < n; c += 32) cp_async16(dst + c, src + c);
    }
    cp_commit();
  };
  if (q0 < q1) issue(q0, 0);

  // G^T, once per CTA (plain loads, coalesced along c)
  const double2* Gt = a.G + (long)t * nn;
  for (int e = tid; e < nn; e += NTH) Gs[(e % n) * S + e / n] = Gt[e];

  // Sigma accumulators: [tile of i][element]; three planes (rr, ii, (r+i)(r+i)) or re / im
  double s0[NT][2], s1[NT][2], s2[NT][2];
#pragma unroll
  for (int u = 0; u < NT; ++u)
#pragma unroll
    for (int e = 0; e < 2; ++e) s0[u][e] = s1[u][e] = s2[u][e] = 0.0;

  const int ks_end = (n + 3) >> 2;
  const int ra = min(8 * w + fr, n - 1) * S + fk;  // this lane's A row (X rows j)
  int rb[NT];                                        // this lane's B rows (G^T rows c, V rows i)
#pragma unroll
  for (int u = 0; u < NT; ++u) rb[u] = min(8 * u + fr, n - 1) * S + fk;
  const int src_lo = (lane & ~3) | (fk >> 1), sel = fk & 1;

  for (int q = q0; q < q1; ++q) {
    const int b = (q - q0) & 1;
    if (q + 1 < q1) {
      issue(q + 1, b ^ 1);
      cp_wait<1>();
    } else {
      cp_wait<0>();
    }
    __syncthreads();
    const double2* xs = Xs + b * tile;
    const double2* vs = Vs + b * tile;
#pragma unroll
    for (int c0 = 0; c0 < NT; c0 += CH) {
      // ---- Z[:, 8 c0 .. 8 (c0 + CH)) = X G for this warp's rows
      double z0[CH][2], z1[CH][2], z2[CH][2];
#pragma unroll
      for (int u = 0; u < CH; ++u)
#pragma unroll
        for (int e = 0; e < 2; ++e) z0[u][e] = z1[u][e] = z2[u][e] = 0.0;
#pragma unroll 2
      for (int ks = 0; ks < ks_end; ++ks) {
        const double2 av = xs[ra + 4 * ks];
        const double ar = av.x, ai = av.y, ax = G3 ? av.x + av.y : -av.y;
        double br[CH], bi[CH];
#pragma unroll
        for (int u = 0; u < CH; ++u) {
          if (c0 + u >= NT) continue;
          const double2 bv = Gs[rb[c0 + u] + 4 * ks];
          br[u] = bv.x;
          bi[u] = bv.y;
        }
        // plane by plane, so that consecutive DMMAs never share an accumulator
#pragma unroll
        for (int u = 0; u < CH; ++u)
          if (c0 + u < NT) dmma(z0[u][0], z0[u][1], ar, br[u]);
#pragma unroll
        for (int u = 0; u < CH; ++u)
          if (c0 + u < NT) dmma(z1[u][0], z1[u][1], G3 ? ai : ar, bi[u]);
#pragma unroll
        for (int u = 0; u < CH; ++u)
          if (c0 + u < NT) {
            if (G3) dmma(z2[u][0], z2[u][1], ax, br[u] + bi[u]);
            else dmma(z0[u][0], z0[u][1], ax, bi[u]);
          }
        if (!G3) {
#pragma unroll
          for (int u = 0; u < CH; ++u)
            if (c0 + u < NT) dmma(z1[u][0], z1[u][1], ai, br[u]);
        }
      }
      // ---- Sigma[rows, :] += Z[:, chunk] V[:, chunk]^+
#pragma unroll
      for (int u = 0; u < CH; ++u) {
        if (c0 + u >= NT) continue;
        double zr[2], zi[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          zr[e] = G3 ? z0[u][e] - z1[u][e] : z0[u][e];
          zi[e] = G3 ? z2[u][e] - z0[u][e] - z1[u][e] : z1[u][e];
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int kc = 8 * (c0 + u) + 4 * h;  // first Z column of this k step
          if (kc >= n) continue;                // warp-uniform: columns past n are all zero in V
          // A fragment: Z[row][kc + fk], held by lane (row, 2h + fk / 2) as element fk % 2
          const int src = src_lo | (2 * h);
          const double r0 = __shfl_sync(0xffffffffu, zr[0], src), r1 = __shfl_sync(0xffffffffu, zr[1], src);
          const double i0 = __shfl_sync(0xffffffffu, zi[0], src), i1 = __shfl_sync(0xffffffffu, zi[1], src);
          const double ar = sel ? r1 : r0, ai = sel ? i1 : i0;
          const double ax = G3 ? ar + ai : -ai;
          // B fragments: conj(V[i][kc + fk]) for i = 8 v + lane / 4
          double br[NT], bi[NT];
#pragma unroll
          for (int v = 0; v < NT; ++v) {
            const double2 bv = vs[rb[v] + kc];
            br[v] = bv.x;
            bi[v] = -bv.y;
          }
#pragma unroll
          for (int v = 0; v < NT; ++v) dmma(s0[v][0], s0[v][1], ar, br[v]);
#pragma unroll
          for (int v = 0; v < NT; ++v) dmma(s1[v][0], s1[v][1], G3 ? ai : ar, bi[v]);
#pragma unroll
          for (int v = 0; v < NT; ++v) {
            if (G3) dmma(s2[v][0], s2[v][1], ax, br[v] + bi[v]);
            else dmma(s0[v][0], s0[v][1], ax, bi[v]);
          }
          if (!G3) {
#pragma unroll
            for (int v = 0; v < NT; ++v) dmma(s1[v][0], s1[v][1], ai, br[v]);
          }
        }
      }
    }
    __syncthreads();  // every warp is done with stage b before the next issue overwrites it
  }

  // partial Sigma of this Q range: rows 8w + lane / 4, columns 8v + 2 (lane % 4) + e
  const int j = 8 * w + fr;
  if (j < n) {
    double2* out = a.P + ((long)blockIdx.x * n + j) * n;
#pragma unroll
    for (int v = 0; v < NT; ++v)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int i = 8 * v + 2 * fk + e;
        if (i < n)
          out[i] = G3 ? make_double2(s0[v][e] - s1[v][e], s2[v][e] - s0[v][e] - s1[v][e])
                      : make_double2(s0[v][e], s1[v][e]);
      }
  }
}

// C[t][r] += alpha * sum_{s < SQ} P[t][s][r] (fixed order)
__global__ void sigma_tail_reduce(const double2* __restrict__ P, int SQ, int nn, int T, double2* C, long c_t,
                                  double2 alpha) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long)T * nn) return;
  const int t = (int)(e / nn), r = (int)(e % nn);
  const double2* p = P + (long)t * SQ * nn + r;
  double2 sum = make_double2(0.0, 0.0);
  for (int s = 0; s < SQ; ++s) sum = cadd(sum, p[(long)s * nn]);
  double2* c = C + (long)t * c_t + r;
  *c = cadd(*c, cmul(alpha, sum));
}

size_t smem_bytes(int n) { return (size_t)5 * n * row_stride(n) * sizeof(double2); }

int optin_smem() {
  static std::atomic<int> cache[kMaxDevices];
  const int dev = current_device();
  int v = cache[dev].load(std::memory_order_relaxed);
  if (v == 0) {
    GG_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cache[dev].store(v, std::memory_order_relaxed);
  }
  return v;
}

// splits of the Q range: the fewest whose T * splits CTAs (one per SM) fill the waves within
// 1 % of the best split count with at least 8 Q per CTA and room for the partials
int choose_splits(int T, int NQ, int nn, long work_elems) {
  const int sms = device_sm_count();
  const long room = work_elems / ((long)T * nn);
  const int smax = (int)std::max(1L, std::min<long>({(long)std::max(1, NQ / 8), 64L, room}));
  auto eff = [&](int s) {
    const long ctas = (long)T * s;
    return (double)ctas / ((double)((ctas + sms - 1) / sms) * sms);
  };
  double best = 0.0;
  for (int s = 1; s <= smax; ++s) best = std::max(best, eff(s));
  for (int s = 1; s <= smax; ++s)
    if (eff(s) >= 0.99 * best) return s;
  return 1;
}

template <int NT, bool G3>
void launch_nt(const TailArgs& a, int T, size_t smem, cudaStream_t st) {
  static std::atomic<int> configured[kMaxDevices];
  const int dev = current_device();
  if (!configured[dev].load(std::memory_order_relaxed)) {
    GG_CUDA(cudaFuncSetAttribute(sigma_tail_kernel<NT, G3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 optin_smem()));
    configured[dev].store(1, std::memory_order_relaxed);
  }
  sigma_tail_kernel<NT, G3><<<T * a.SQ, 32 * NT, smem, st>>>(a);
  GG_CHECK_LAUNCH();
}

template <bool G3>
void launch_g3(const TailArgs& a, int T, size_t smem, cudaStream_t st) {
  switch ((a.n + 7) / 8) {
    case 1: launch_nt<1, G3>(a, T, smem, st); break;
    case 2: launch_nt<2, G3>(a, T, smem, st); break;
    case 3: launch_nt<3, G3>(a, T, smem, st); break;
    case 4: launch_nt<4, G3>(a, T, smem, st); break;
    case 5: launch_nt<5, G3>(a, T, smem, st); break;
    case 6: launch_nt<6, G3>(a, T, smem, st); break;
    case 7: launch_nt<7, G3>(a, T, smem, st); break;
    default: throw Error(GG_ERR_ARG, "sigma_tail: orbital count outside the fused kernel's range");
  }
}

}  // namespace

bool sigma_tail_supported(int n, int T, long work_elems) {
  if (n < 1 || n > 56 || T < 1) return false;
  if (smem_bytes(n) > (size_t)optin_smem()) return false;
  return work_elems >= (long)T * n * n;
}

int sigma_tail(const double2* X, long x_t, const double2* G, const double2* V, int n, int NQ, int T, double2* C,
               long c_t, double2 alpha, bool gauss, double2* work, long work_elems, cudaStream_t st) {
  if (!sigma_tail_supported(n, T, work_elems)) throw Error(GG_ERR_ARG, "sigma_tail: unsupported shape");
  if (NQ < 1) return 0;
  TailArgs a{X, x_t, G, V, work, n, NQ, choose_splits(T, NQ, n * n, work_elems)};
  const size_t smem = smem_bytes(n);
  if (gauss) launch_g3<true>(a, T, smem, st);
  else launch_g3<false>(a, T, smem, st);
  const long total = (long)T * n * n;
  sigma_tail_reduce<<<(int)((total + 255) / 256), 256, 0, st>>>(work, a.SQ, n * n, T, C, c_t, alpha);
  GG_CHECK_LAUNCH();
  return 2;
}

}  // namespace gg
