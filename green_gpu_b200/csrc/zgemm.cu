// Batched complex FP64 GEMM engine (see zgemm.cuh).
//
// CTA tile 64 x 64 complex, K step 8 complex, 4 warps in a 2 x 2 layout, each warp a
// 32 x 32 complex tile = 4 x 4 DMMA 8x8 tiles per real/imag plane.  Complex products use
// four real DMMAs (rr, -ii, ri, ir) on fragments read with one 16-byte shared load each
// (interleaved complex in shared memory).  Global->shared staging uses cp.async (16 B,
// zero-fill at the edges) into a 3-stage ring; the shared layout follows the global
// contiguity of each operand ([row][k] or [k][row]) with an XOR swizzle so both the async
// copies and the fragment loads are bank-conflict free without padding.
#include "zgemm.cuh"

#include <algorithm>

namespace gg {
namespace {

constexpr int BM = 64, BN = 64, BK = 8, NT = 128, STAGES = 3;
constexpr int TILE = BM * BK;  // complex elements per operand stage
static_assert(BM == BN, "square tiles assumed by the staging code");

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// swizzled position of tile element (row r, k) in a stage
template <bool KMAJ>
__device__ __forceinline__ int sidx(int r, int k) {
  return KMAJ ? r * BK + (k ^ ((r & 1) << 2)) : k * BM + (r ^ ((k & 3) << 1));
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// One CTA computes a run of `span` consecutive tiles along M (span_m) or N, so that for short
// reductions the cp.async ring runs on across tile boundaries: the next tile's first stages
// load while the current tile's epilogue stores (span = 1: one tile per CTA).
template <bool A_K, bool B_K, bool SPAN>
__global__ void __launch_bounds__(NT, 2)
    zgemm_kernel(ZgemmDesc d, int tiles_m, int tiles_n, int span, int span_m) {
  if (!SPAN) span = 1;
  __shared__ __align__(16) double2 As[STAGES][TILE];
  __shared__ __align__(16) double2 Bs[STAGES][TILE];

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;

  // grid: groups of `span` tiles along the spanned dimension
  const int groups_m = span_m ? (tiles_m + span - 1) / span : tiles_m;
  const int groups_n = span_m ? tiles_n : (tiles_n + span - 1) / span;
  const long bid = blockIdx.x;
  const int ngroup = groups_m * groups_n;
  const int group = (int)(bid % ngroup);
  const long rest = bid / ngroup;
  const int split = (int)(rest % d.splits);
  const long batch = rest / d.splits;
  const int b0 = (int)(batch % d.nb0);
  const int b1 = (int)((batch / d.nb0) % d.nb1);
  const int b2 = (int)(batch / ((long)d.nb0 * d.nb1));
  const int gm = group % groups_m, gn = group / groups_m;
  const int tm0 = span_m ? gm * span : gm, tn0 = span_m ? gn : gn * span;
  const int ntiles = !SPAN ? 1 : span_m ? min(span, tiles_m - tm0) : min(span, tiles_n - tn0);

  const double2* Ab = d.A + b0 * d.a_b0 + b1 * d.a_b1 + b2 * d.a_b2;
  const double2* Bb = d.B + b0 * d.b_b0 + b1 * d.b_b1 + b2 * d.b_b2;

  // staging assignment: 512 elements per operand stage, 4 per thread
  //   KMAJ : k = tid % 8, rows tid / 8 + 16 i
  //   !KMAJ: row = tid % 64, k = tid / 64 + 2 i
  long a_off[4], b_off[4];
  bool a_ok[4], b_ok[4];
  auto set_a = [&](int m0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int m = m0 + (A_K ? tid / 8 + 16 * i : tid % 64);
      a_ok[i] = m < d.M;
      a_off[i] = a_ok[i] ? d.a_m(m) : 0;
    }
  };
  auto set_b = [&](int n0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int n = n0 + (B_K ? tid / 8 + 16 * i : tid % 64);
      b_ok[i] = n < d.N;
      b_off[i] = b_ok[i] ? d.b_n(n) : 0;
    }
  };
  set_a(tm0 * BM);
  set_b(tn0 * BN);

  const int ktiles = (d.K + BK - 1) / BK;
  const long total = (long)d.KB * ktiles;
  const long t_begin = total * split / d.splits;
  const long t_end = total * (split + 1) / d.splits;
  const long per_tile = t_end - t_begin;

  auto issue = [&](long t, int st) {
    const int kb = (int)(t / ktiles);
    const int k0 = (int)(t % ktiles) * BK;
    const double2* Ak = Ab + kb * d.a_kb;
    const double2* Bk = Bb + kb * d.b_kb;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = A_K ? tid / 8 + 16 * i : tid % 64;
      const int kk = A_K ? tid % 8 : tid / 64 + 2 * i;
      const int k = k0 + kk;
      const bool v = a_ok[i] && k < d.K;
      cp_async16(&As[st][sidx<A_K>(r, kk)], v ? (const void*)(Ak + a_off[i] + k * d.a_k) : (const void*)Ab, v);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = B_K ? tid / 8 + 16 * i : tid % 64;
      const int kk = B_K ? tid % 8 : tid / 64 + 2 * i;
      const int k = k0 + kk;
      const bool v = b_ok[i] && k < d.K;
      cp_async16(&Bs[st][sidx<B_K>(r, kk)], v ? (const void*)(Bk + b_off[i] + k * d.b_k) : (const void*)Bb, v);
    }
  };
  // issue stream over the run of tiles: (itile, it) is the next step to load
  int itile = 0;
  long it = t_begin;
  auto issue_next = [&](int st) {
    if (itile >= ntiles) return;
    issue(it, st);
    if (++it == t_end) {
      it = t_begin;
      if (++itile < ntiles) {
        if (span_m) set_a((tm0 + itile) * BM);
        else set_b((tn0 + itile) * BN);
      }
    }
  };

  double cr[4][4][2], ci[4][4][2];
  auto zero_acc = [&]() {
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        cr[a][b][0] = cr[a][b][1] = 0.0;
        ci[a][b][0] = ci[a][b][1] = 0.0;
      }
  };
  zero_acc();

  const double sa = d.conjA ? -1.0 : 1.0;
  const double sb = d.conjB ? -1.0 : 1.0;
  const int fr = lane >> 2, fk = lane & 3;

  auto epilogue = [&](int m0, int n0) {
    const long batch_count = (long)d.nb0 * d.nb1 * d.nb2;
    const double2* cbase = d.C + b0 * d.c_b0 + b1 * d.c_b1 + b2 * d.c_b2;
    const bool use_beta = d.beta.x != 0.0 || d.beta.y != 0.0;
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) {
      const int m = m0 + wm * 32 + mt * 8 + fr;
      if (m >= d.M) continue;
      const long cm = d.c_m(m);
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int n = n0 + wn * 32 + nt * 8 + 2 * fk + j;
          if (n >= d.N) continue;
          const double2 acc = make_double2(cr[mt][nt][j], ci[mt][nt][j]);
          if (d.splits > 1) {
            d.work[((split * batch_count + batch) * d.M + m) * (long)d.N + n] = acc;
          } else {
            double2* c = const_cast<double2*>(cbase) + cm + d.c_n(n);
            double2 v = cmul(d.alpha, acc);
            if (use_beta) v = cadd(v, cmul(d.beta, *c));
            *c = v;
          }
        }
      }
    }
  };

  int st = 0;
  if constexpr (SPAN) {
    // prologue: STAGES-1 stages in flight (possibly reaching into the next tiles)
#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
      issue_next(s);
      cp_commit();
    }
    int ctile = 0;   // tile being computed
    long cstep = 0;  // its step
    const long steps = (long)ntiles * per_tile;
    for (long s = 0; s < steps; ++s) {
      cp_wait<STAGES - 2>();
      __syncthreads();
      {
        int sn = st + STAGES - 1;
        if (sn >= STAGES) sn -= STAGES;
        issue_next(sn);
        cp_commit();
      }
      const double2* as = As[st];
      const double2* bs = Bs[st];
#pragma unroll
      for (int ks = 0; ks < BK / 4; ++ks) {
        double ar[4], ai[4], an[4], br[4], bi[4];
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) {
          const double2 v = as[sidx<A_K>(wm * 32 + mt * 8 + fr, ks * 4 + fk)];
          ar[mt] = v.x;
          ai[mt] = sa * v.y;
          an[mt] = -ai[mt];
        }
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          const double2 v = bs[sidx<B_K>(wn * 32 + nt * 8 + fr, ks * 4 + fk)];
          br[nt] = v.x;
          bi[nt] = sb * v.y;
        }
#pragma unroll
        // four passes over the 16 accumulator tiles: consecutive DMMAs never share an
        // accumulator, so each waits on a result issued 16 instructions earlier
        for (int mt = 0; mt < 4; ++mt)
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) dmma(cr[mt][nt][0], cr[mt][nt][1], ar[mt], br[nt]);
#pragma unroll
        for (int mt = 0; mt < 4; ++mt)
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) dmma(ci[mt][nt][0], ci[mt][nt][1], ar[mt], bi[nt]);
#pragma unroll
        for (int mt = 0; mt < 4; ++mt)
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) dmma(cr[mt][nt][0], cr[mt][nt][1], an[mt], bi[nt]);
#pragma unroll
        for (int mt = 0; mt < 4; ++mt)
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) dmma(ci[mt][nt][0], ci[mt][nt][1], ai[mt], br[nt]);
      }
      st = (st + 1 == STAGES) ? 0 : st + 1;
      if (++cstep == per_tile) {
        epilogue((tm0 + (span_m ? ctile : 0)) * BM, (tn0 + (span_m ? 0 : ctile)) * BN);
        zero_acc();
        cstep = 0;
        ++ctile;
      }
    }
    cp_wait<0>();
  } else {
    // one tile: prologue of STAGES-1 stages, then refill one stage per step
#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
      if (t_begin + s < t_end) issue(t_begin + s, s);
      cp_commit();
    }
    for (long t = t_begin; t < t_end; ++t) {
      cp_wait<STAGES - 2>();
      __syncthreads();
      {
        const long tn_ = t + STAGES - 1;
        int sn = st + STAGES - 1;
        if (sn >= STAGES) sn -= STAGES;
        if (tn_ < t_end) issue(tn_, sn);
        cp_commit();
      }
      const double2* as = As[st];
      const double2* bs = Bs[st];
#pragma unroll
      for (int ks = 0; ks < BK / 4; ++ks) {
        double ar[4], ai[4], an[4], br[4], bi[4];
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) {
          const double2 v = as[sidx<A_K>(wm * 32 + mt * 8 + fr, ks * 4 + fk)];
          ar[mt] = v.x;
          ai[mt] = sa * v.y;
          an[mt] = -ai[mt];
        }
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          const double2 v = bs[sidx<B_K>(wn * 32 + nt * 8 + fr, ks * 4 + fk)];
          br[nt] = v.x;
          bi[nt] = sb * v.y;
        }
#pragma unroll
        // four passes over the 16 accumulator tiles: consecutive DMMAs never share an
        // accumulator, so each waits on a result issued 16 instructions earlier
        for (int mt = 0; mt < 4; ++mt)
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) dmma(cr[mt][nt][0], cr[mt][nt][1], ar[mt], br[nt]);
#pragma unroll
        for (int mt = 0; mt < 4; ++mt)
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) dmma(ci[mt][nt][0], ci[mt][nt][1], ar[mt], bi[nt]);
#pragma unroll
        for (int mt = 0; mt < 4; ++mt)
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) dmma(cr[mt][nt][0], cr[mt][nt][1], an[mt], bi[nt]);
#pragma unroll
        for (int mt = 0; mt < 4; ++mt)
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) dmma(ci[mt][nt][0], ci[mt][nt][1], ai[mt], br[nt]);
      }
      st = (st + 1 == STAGES) ? 0 : st + 1;
    }
    cp_wait<0>();
    epilogue(tm0 * BM, tn0 * BN);
  }
}

__global__ void zgemm_reduce(ZgemmDesc d) {
  const long batch_count = (long)d.nb0 * d.nb1 * d.nb2;
  const long mn = (long)d.M * d.N;
  const long total = batch_count * mn;
  const bool use_beta = d.beta.x != 0.0 || d.beta.y != 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const long batch = i / mn;
    const long e = i % mn;
    const int m = (int)(e / d.N);
    const int n = (int)(e % d.N);
    double2 acc = make_double2(0.0, 0.0);
    for (int s = 0; s < d.splits; ++s) acc = cadd(acc, d.work[(s * batch_count + batch) * mn + e]);
    const int b0 = (int)(batch % d.nb0);
    const int b1 = (int)((batch / d.nb0) % d.nb1);
    const int b2 = (int)(batch / ((long)d.nb0 * d.nb1));
    double2* c = d.C + b0 * d.c_b0 + b1 * d.c_b1 + b2 * d.c_b2 + d.c_m(m) + d.c_n(n);
    double2 v = cmul(d.alpha, acc);
    if (use_beta) v = cadd(v, cmul(d.beta, *c));
    *c = v;
  }
}

template <bool A_K, bool B_K>
void launch(const ZgemmDesc& d, int tiles_m, int tiles_n, int span, int span_m, long blocks, cudaStream_t stream) {
  if (span > 1)
    zgemm_kernel<A_K, B_K, true><<<(unsigned)blocks, NT, 0, stream>>>(d, tiles_m, tiles_n, span, span_m);
  else
    zgemm_kernel<A_K, B_K, false><<<(unsigned)blocks, NT, 0, stream>>>(d, tiles_m, tiles_n, 1, 0);
  GG_CHECK_LAUNCH();
}

int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    GG_CUDA(cudaGetDevice(&dev));
    GG_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  }
  return n;
}

}  // namespace

int zgemm(const ZgemmDesc& d0, cudaStream_t stream) {
  ZgemmDesc d = d0;
  if (d.M <= 0 || d.N <= 0 || d.nb0 <= 0 || d.nb1 <= 0 || d.nb2 <= 0) return 0;
  if (d.K < 0 || d.KB < 1) throw Error(GG_ERR_ARG, "zgemm: bad K");
  const int tiles_m = ceil_div(d.M, BM), tiles_n = ceil_div(d.N, BN);
  const long batch = (long)d.nb0 * d.nb1 * d.nb2;
  const long base = (long)tiles_m * tiles_n * batch;
  // split-K when the grid leaves resident CTA slots idle and the reduction is long: the
  // split count minimises the waves per unit of work, ceil(base * s / slots) / s (two CTAs
  // per SM are resident), so a grid of 1.3 waves becomes one of 3 full waves at s = 3
  // rather than 2.6 waves at s = 2; ties go to the smaller count
  int splits = 1;
  const long ksteps = (long)d.KB * ceil_div(d.K, BK);
  const long slots = 2L * sm_count();
  if (d.work && base < 8 * slots && ksteps >= 32) {
    const long need = (long)d.M * d.N * batch;
    long smax = std::min<long>(64, ksteps / 16);
    if (need > 0) smax = std::min<long>(smax, d.work_elems / need);
    double best = (double)ceil_div(base, slots);
    for (long s = 2; s <= smax; ++s) {
      const double cost = (double)((base * s + slots - 1) / slots) / (double)s;
      if (cost < best * 0.97) {
        best = cost;
        splits = (int)s;
      }
    }
  }
  d.splits = splits;
  // short reductions: runs of up to 4 tiles per CTA along the longer tile dimension, as long
  // as at least 8 waves of CTAs remain (the ring then overlaps a tile's epilogue with the next
  // tile's first loads)
  int span = 1, span_m = 0;
  if (splits == 1 && ksteps <= 16) {
    span_m = tiles_m >= tiles_n ? 1 : 0;
    const int along = span_m ? tiles_m : tiles_n;
    const long other = base / along;
    for (int sp = 4; sp >= 2; --sp)
      if (along >= sp && other * ((along + sp - 1) / sp) >= 8 * slots) {
        span = sp;
        break;
      }
  }
  const long groups = span_m ? (long)((tiles_m + span - 1) / span) * tiles_n * batch
                             : (long)tiles_m * ((tiles_n + span - 1) / span) * batch;
  const long blocks = groups * splits;
  if (blocks > 0x7fffffffL) throw Error(GG_ERR_ARG, "zgemm: grid too large");
  const bool ak = (d.a_k == 1), bk = (d.b_k == 1);
  if (ak && bk) launch<true, true>(d, tiles_m, tiles_n, span, span_m, blocks, stream);
  else if (ak) launch<true, false>(d, tiles_m, tiles_n, span, span_m, blocks, stream);
  else if (bk) launch<false, true>(d, tiles_m, tiles_n, span, span_m, blocks, stream);
  else launch<false, false>(d, tiles_m, tiles_n, span, span_m, blocks, stream);
  int launches = 1;
  if (splits > 1) {
    const long total = (long)d.M * d.N * batch;
    const int threads = 256;
    const long nblk = std::min<long>((total + threads - 1) / threads, 65535L * 8);
    zgemm_reduce<<<(unsigned)nblk, threads, 0, stream>>>(d);
    GG_CHECK_LAUNCH();
    ++launches;
  }
  return launches;
}

}  // namespace gg
