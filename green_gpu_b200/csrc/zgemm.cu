// Batched complex FP64 GEMM engine (see zgemm.cuh).
//
// Two kernels share the tile, the staging and the grid.  The four-warp kernel: CTA tile
// 64 x 64 complex, K step 8 complex, 4 warps in a 2 x 2 layout, each warp a
// 32 x 32 complex tile = 4 x 4 DMMA 8x8 tiles per real/imag plane.  Complex products use
// four real DMMAs (rr, -ii, ri, ir) on fragments read with one 16-byte shared load each
// (interleaved complex in shared memory).  Global->shared staging uses cp.async (16 B,
// zero-fill at the edges) into a 3-stage ring; the shared layout follows the global
// contiguity of each operand ([row][k] or [k][row]) with an XOR swizzle so both the async
// copies and the fragment loads are bank-conflict free without padding.
#include "zgemm.cuh"

#include "dmma.cuh"

#include <atomic>

#include <algorithm>

namespace gg {
namespace {

constexpr int BM = 64, BN = 64, BK = 8, NT = 128, STAGES = 3;
constexpr int TILE = BM * BK;  // complex elements per operand stage
static_assert(BM == BN, "square tiles assumed by the staging code");

// x with its sign bit XORed with the sign bit of `s` (s = 0 or 0x80000000)
__device__ __forceinline__ double flip(double x, int s) {
  return __hiloint2double(__double2hiint(x) ^ s, __double2loint(x));
}

// swizzled position of tile element (row r, k) in a stage
template <bool KMAJ>
__device__ __forceinline__ int sidx(int r, int k) {
  return KMAJ ? r * BK + (k ^ ((r & 1) << 2)) : k * BM + (r ^ ((k & 3) << 1));
}

// One CTA per (tile, split, batch entry) for reductions of any length.
template <bool A_K, bool B_K>
__global__ void __launch_bounds__(NT, 2)
    zgemm_kernel(ZgemmDesc d, int tiles_m, int tiles_n) {
  __shared__ __align__(16) double2 As[STAGES][TILE];
  __shared__ __align__(16) double2 Bs[STAGES][TILE];

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;

  const long bid = blockIdx.x;
  const int ntile = tiles_m * tiles_n;
  const int tile = (int)(bid % ntile);
  const long rest = bid / ntile;
  const int split = (int)(rest % d.splits);
  const long batch = rest / d.splits;
  const int b0 = (int)(batch % d.nb0);
  const int b1 = (int)((batch / d.nb0) % d.nb1);
  const int b2 = (int)(batch / ((long)d.nb0 * d.nb1));
  const int tm0 = tile % tiles_m, tn0 = tile / tiles_m;

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

  // conjugation flips the sign bit of the imaginary part (an integer XOR, no FP64 multiply)
  const int sa = d.conjA ? (int)0x80000000 : 0;
  const int sb = d.conjB ? (int)0x80000000 : 0;
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
  {
    // prologue of STAGES-1 stages, then refill one stage per step
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
          ai[mt] = flip(v.y, sa);
          an[mt] = -ai[mt];
        }
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          const double2 v = bs[sidx<B_K>(wn * 32 + nt * 8 + fr, ks * 4 + fk)];
          br[nt] = v.x;
          bi[nt] = flip(v.y, sb);
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

// Eight-warp variant: the same 64 x 64 tile and 3-stage ring, 8 warps of 16 x 32 (4 x 2
// layout; half the accumulators per thread, so two CTAs of 256 threads stay resident at 128
// registers).  It wins where the reduction is short (K = nao, runs of tiles per CTA), the
// four-warp kernel where it is long.  G3 selects the three-product complex form.  NARROW (N <=
// 56, a single column tile): 8 warps of 8 x 56, so the MMAs cover columns 0..55 only (N = nao
// = 52 fills 93 % of them instead of 81 % of 64) and every warp has the same work.  The
// reduction position advances by counters (no division per step), and k quarters that lie
// wholly past K are skipped.
constexpr int NT8 = 256;
constexpr int SPT8 = TILE / NT8;
static_assert(SPT8 * NT8 == TILE, "whole staging assignments");

// index map with 32-bit division (indices of one operand are below 2^31)
__device__ __forceinline__ long imap(const IdxMap& f, int i) {
  return f.split > 0 ? (long)(i / f.split) * f.hi + (long)(i % f.split) * f.lo : (long)i * f.lo;
}

template <bool A_K, bool B_K, bool SPAN, bool G3, bool NARROW>
__global__ void __launch_bounds__(NT8, 2)
    zgemm8_kernel(ZgemmDesc d, int tiles_m, int tiles_n, int span, int span_m) {
  if (!SPAN) span = 1;
  __shared__ __align__(16) double2 As[STAGES][TILE];
  __shared__ __align__(16) double2 Bs[STAGES][TILE];

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  constexpr int WARPS_M8 = NARROW ? 8 : 4;
  constexpr int WM8 = NARROW ? 8 : 16, WN8 = NARROW ? 56 : 32;
  constexpr int FM8 = WM8 / 8, FN8 = WN8 / 8;
  const int wm = warp % WARPS_M8, wn = warp / WARPS_M8;

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

  // staging: BM * BK elements per operand stage, SPT8 per thread
  //   KMAJ : k = tid % BK, rows tid / BK + (NT8 / BK) i
  //   !KMAJ: row = tid % BM, k = tid / BM + (NT8 / BM) i
  long a_off[SPT8], b_off[SPT8];
  bool a_ok[SPT8], b_ok[SPT8];
  auto set_a = [&](int m0) {
#pragma unroll
    for (int i = 0; i < SPT8; ++i) {
      const int m = m0 + (A_K ? tid / BK + (NT8 / BK) * i : tid % BM);
      a_ok[i] = m < d.M;
      a_off[i] = a_ok[i] ? imap(d.a_m, m) : 0;
    }
  };
  auto set_b = [&](int n0) {
#pragma unroll
    for (int i = 0; i < SPT8; ++i) {
      const int n = n0 + (B_K ? tid / BK + (NT8 / BK) * i : tid % BM);
      b_ok[i] = n < d.N;
      b_off[i] = b_ok[i] ? imap(d.b_n, n) : 0;
    }
  };
  set_a(tm0 * BM);
  set_b(tn0 * BN);

  const int ktiles = (d.K + BK - 1) / BK;
  const long total = (long)d.KB * ktiles;
  const long t_begin = total * split / d.splits;
  const long t_end = total * (split + 1) / d.splits;
  const long per_tile = t_end - t_begin;
  const int kb_begin = (int)(t_begin / ktiles), kt_begin = (int)(t_begin % ktiles);

  // issue stream position: tile itile, reduction block ikb, k tile ikt (no divisions per step)
  int itile = 0, ikb = kb_begin, ikt = kt_begin;
  long icount = 0;
  auto issue_next = [&](int st) {
    if (itile >= ntiles) return;
    const int k0 = ikt * BK;
    const double2* Ak = Ab + ikb * d.a_kb;
    const double2* Bk = Bb + ikb * d.b_kb;
#pragma unroll
    for (int i = 0; i < SPT8; ++i) {
      const int r = A_K ? tid / BK + (NT8 / BK) * i : tid % BM;
      const int kk = A_K ? tid % BK : tid / BM + (NT8 / BM) * i;
      const int k = k0 + kk;
      const bool v = a_ok[i] && k < d.K;
      cp_async16(&As[st][sidx<A_K>(r, kk)], v ? (const void*)(Ak + a_off[i] + k * d.a_k) : (const void*)Ab, v);
    }
#pragma unroll
    for (int i = 0; i < SPT8; ++i) {
      const int r = B_K ? tid / BK + (NT8 / BK) * i : tid % BM;
      const int kk = B_K ? tid % BK : tid / BM + (NT8 / BM) * i;
      const int k = k0 + kk;
      const bool v = b_ok[i] && k < d.K;
      cp_async16(&Bs[st][sidx<B_K>(r, kk)], v ? (const void*)(Bk + b_off[i] + k * d.b_k) : (const void*)Bb, v);
    }
    if (++ikt == ktiles) {
      ikt = 0;
      ++ikb;
    }
    if (++icount == per_tile) {
      icount = 0;
      ikb = kb_begin;
      ikt = kt_begin;
      if (++itile < ntiles) {
        if (span_m) set_a((tm0 + itile) * BM);
        else set_b((tn0 + itile) * BN);
      }
    }
  };

  // accumulators: c0/c1 = re/im (four products) or c0/c1/c2 = rr, ii, (r+i)(r+i) (three)
  double c0[FM8][FN8][2], c1[FM8][FN8][2], c2[FM8][FN8][2];
  auto zero_acc = [&]() {
#pragma unroll
    for (int a = 0; a < FM8; ++a)
#pragma unroll
      for (int b = 0; b < FN8; ++b)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          c0[a][b][j] = 0.0;
          c1[a][b][j] = 0.0;
          if (G3) c2[a][b][j] = 0.0;
        }
  };
  zero_acc();

  // conjugation flips the sign bit of the imaginary part (an integer XOR, no FP64 multiply)
  const int sa = d.conjA ? (int)0x80000000 : 0;
  const int sb = d.conjB ? (int)0x80000000 : 0;
  const int fr = lane >> 2, fk = lane & 3;

  auto epilogue = [&](int m0, int n0) {
    const long batch_count = (long)d.nb0 * d.nb1 * d.nb2;
    const double2* cbase = d.C + b0 * d.c_b0 + b1 * d.c_b1 + b2 * d.c_b2;
    const bool use_beta = d.beta.x != 0.0 || d.beta.y != 0.0;
#pragma unroll
    for (int mt = 0; mt < FM8; ++mt) {
      const int m = m0 + wm * WM8 + mt * 8 + fr;
      if (m >= d.M) continue;
      const long cm = imap(d.c_m, m);
#pragma unroll
      for (int nt = 0; nt < FN8; ++nt) {
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int n = n0 + wn * WN8 + nt * 8 + 2 * fk + j;
          if (n >= d.N) continue;
          const double2 acc = G3 ? make_double2(c0[mt][nt][j] - c1[mt][nt][j],
                                                c2[mt][nt][j] - c0[mt][nt][j] - c1[mt][nt][j])
                                 : make_double2(c0[mt][nt][j], c1[mt][nt][j]);
          if (d.splits > 1) {
            d.work[((split * batch_count + batch) * d.M + m) * (long)d.N + n] = acc;
          } else {
            double2* c = const_cast<double2*>(cbase) + cm + imap(d.c_n, n);
            double2 v = cmul(d.alpha, acc);
            if (use_beta) v = cadd(v, cmul(d.beta, *c));
            *c = v;
          }
        }
      }
    }
  };

  auto substep = [&](const double2* as, const double2* bs, int ks) {
    double ar[FM8], ai[FM8], ax[FM8], br[FN8], bi[FN8], bx[FN8];
#pragma unroll
    for (int mt = 0; mt < FM8; ++mt) {
      const double2 v = as[sidx<A_K>(wm * WM8 + mt * 8 + fr, ks * 4 + fk)];
      ar[mt] = v.x;
      ai[mt] = flip(v.y, sa);
      ax[mt] = G3 ? ar[mt] + ai[mt] : -ai[mt];
    }
#pragma unroll
    for (int nt = 0; nt < FN8; ++nt) {
      const double2 v = bs[sidx<B_K>(wn * WN8 + nt * 8 + fr, ks * 4 + fk)];
      br[nt] = v.x;
      bi[nt] = flip(v.y, sb);
      bx[nt] = br[nt] + bi[nt];
    }
    if constexpr (G3) {
#pragma unroll
      for (int mt = 0; mt < FM8; ++mt)
#pragma unroll
        for (int nt = 0; nt < FN8; ++nt) dmma(c0[mt][nt][0], c0[mt][nt][1], ar[mt], br[nt]);
#pragma unroll
      for (int mt = 0; mt < FM8; ++mt)
#pragma unroll
        for (int nt = 0; nt < FN8; ++nt) dmma(c1[mt][nt][0], c1[mt][nt][1], ai[mt], bi[nt]);
#pragma unroll
      for (int mt = 0; mt < FM8; ++mt)
#pragma unroll
        for (int nt = 0; nt < FN8; ++nt) dmma(c2[mt][nt][0], c2[mt][nt][1], ax[mt], bx[nt]);
    } else {
#pragma unroll
      for (int mt = 0; mt < FM8; ++mt)
#pragma unroll
        for (int nt = 0; nt < FN8; ++nt) dmma(c0[mt][nt][0], c0[mt][nt][1], ar[mt], br[nt]);
#pragma unroll
      for (int mt = 0; mt < FM8; ++mt)
#pragma unroll
        for (int nt = 0; nt < FN8; ++nt) dmma(c1[mt][nt][0], c1[mt][nt][1], ar[mt], bi[nt]);
#pragma unroll
      for (int mt = 0; mt < FM8; ++mt)
#pragma unroll
        for (int nt = 0; nt < FN8; ++nt) dmma(c0[mt][nt][0], c0[mt][nt][1], ax[mt], bi[nt]);
#pragma unroll
      for (int mt = 0; mt < FM8; ++mt)
#pragma unroll
        for (int nt = 0; nt < FN8; ++nt) dmma(c1[mt][nt][0], c1[mt][nt][1], ai[mt], br[nt]);
    }
  };

  // prologue: STAGES-1 stages in flight (with SPAN possibly reaching into the next tiles)
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    issue_next(s);
    cp_commit();
  }
  int st = 0;
  int ctile = 0, ckt = kt_begin;
  long cstep = 0;
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
    // k quarters wholly past K (zero-filled) are skipped
    {
      const int krem = d.K - ckt * BK;
#pragma unroll
      for (int ks = 0; ks < BK / 4; ++ks)
        if (ks == 0 || krem > 4 * ks) substep(As[st], Bs[st], ks);
    }
    st = (st + 1 == STAGES) ? 0 : st + 1;
    if (++ckt == ktiles) ckt = 0;
    if constexpr (SPAN) {
      if (++cstep == per_tile) {
        epilogue((tm0 + (span_m ? ctile : 0)) * BM, (tn0 + (span_m ? 0 : ctile)) * BN);
        zero_acc();
        cstep = 0;
        ckt = kt_begin;
        ++ctile;
      }
    }
  }
  cp_wait<0>();
  if constexpr (!SPAN) epilogue(tm0 * BM, tn0 * BN);
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
void launch(const ZgemmDesc& d, int tiles_m, int tiles_n, long blocks, cudaStream_t stream) {
  zgemm_kernel<A_K, B_K><<<(unsigned)blocks, NT, 0, stream>>>(d, tiles_m, tiles_n);
  GG_CHECK_LAUNCH();
}

template <bool A_K, bool B_K, bool G3, bool NARROW>
void launch8(const ZgemmDesc& d, int tiles_m, int tiles_n, int span, int span_m, long blocks, cudaStream_t stream) {
  if (span > 1)
    zgemm8_kernel<A_K, B_K, true, G3, NARROW><<<(unsigned)blocks, NT8, 0, stream>>>(d, tiles_m, tiles_n, span, span_m);
  else
    zgemm8_kernel<A_K, B_K, false, G3, NARROW><<<(unsigned)blocks, NT8, 0, stream>>>(d, tiles_m, tiles_n, 1, 0);
  GG_CHECK_LAUNCH();
}

template <bool G3, bool NARROW>
void launch8_layout(const ZgemmDesc& d, int tiles_m, int tiles_n, int span, int span_m, long blocks,
                    cudaStream_t stream) {
  const bool ak = (d.a_k == 1), bk = (d.b_k == 1);
  if (ak && bk) launch8<true, true, G3, NARROW>(d, tiles_m, tiles_n, span, span_m, blocks, stream);
  else if (ak) launch8<true, false, G3, NARROW>(d, tiles_m, tiles_n, span, span_m, blocks, stream);
  else if (bk) launch8<false, true, G3, NARROW>(d, tiles_m, tiles_n, span, span_m, blocks, stream);
  else launch8<false, false, G3, NARROW>(d, tiles_m, tiles_n, span, span_m, blocks, stream);
}

template <bool G3>
void launch8_any(const ZgemmDesc& d, int tiles_m, int tiles_n, int span, int span_m, long blocks,
                 cudaStream_t stream) {
  if (d.N <= 56) launch8_layout<G3, true>(d, tiles_m, tiles_n, span, span_m, blocks, stream);
  else launch8_layout<G3, false>(d, tiles_m, tiles_n, span, span_m, blocks, stream);
}

int sm_count() { return device_sm_count(); }

}  // namespace

int current_device() {
  int dev = 0;
  GG_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) throw Error(GG_ERR_ARG, "device index " + std::to_string(dev) + " out of range");
  return dev;
}

int device_sm_count() {
  static std::atomic<int> counts[kMaxDevices];
  const int dev = current_device();
  int n = counts[dev].load(std::memory_order_relaxed);
  if (!n) {
    GG_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    counts[dev].store(n, std::memory_order_relaxed);
  }
  return n;
}

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
  // kernel choice (both 64 x 64 tiles, same grid): the three-product form always runs on the
  // eight-warp kernel; the four-product form runs there for runs of tiles (short reductions)
  // and on the four-warp kernel otherwise
  const bool ak = (d.a_k == 1), bk = (d.b_k == 1);
  if (d.gauss) launch8_any<true>(d, tiles_m, tiles_n, span, span_m, blocks, stream);
  else if (span > 1) launch8_any<false>(d, tiles_m, tiles_n, span, span_m, blocks, stream);
  else if (ak && bk) launch<true, true>(d, tiles_m, tiles_n, blocks, stream);
  else if (ak) launch<true, false>(d, tiles_m, tiles_n, blocks, stream);
  else if (bk) launch<false, true>(d, tiles_m, tiles_n, blocks, stream);
  else launch<false, false>(d, tiles_m, tiles_n, blocks, stream);
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
