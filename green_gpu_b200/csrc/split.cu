// Split-precision complex GEMM on the 5th-generation tensor cores (tcgen05, kind::i8).
//
// Ozaki scheme with exact INT8 slices:
//   * every row m of A (over the whole reduction K, all K-batches) gets an exponent e_m with
//     max_k |A(m,k)| < 2^e_m; x = A / 2^e_m is cut into S slices of 7 bits by truncation,
//     a_s = trunc(2^7 r_{s-1}), r_s = 2^7 r_{s-1} - a_s (all exact in FP64), so
//     A = 2^e_m sum_s a_s 2^-7s + O(2^(e_m - 7S)).  Columns of B likewise with f_n.
//   * complex arithmetic is one real GEMM of size M x 2N x 2K: A' rows interleave (re, im)
//     along K, B' rows 2n / 2n+1 hold (re, -im) / (im, re), so C'(m, 2n) = Re C(m,n) and
//     C'(m, 2n+1) = Im C(m,n).
//   * the products a_s b_t with s + t = d share the scale 2^-7d and accumulate into one
//     int32 TMEM accumulator per diagonal d = 2..S+1 (pairs with s + t > S + 1 are dropped,
//     the usual triangular truncation).  K is processed in chunks small enough that no
//     int32 sum can overflow (S * Kchunk * 127^2 < 2^31), so every chunk is exact; chunks
//     are drained to FP64 registers and scaled by 2^(e_m + f_n - 7d).
//
// Kernel roles (one CTA per SM, 320 threads): warp 0 issues TMA loads (2D tensor maps,
// 64-byte swizzle, no multicast) of all S slices of an A and a B K-block into a 3-stage
// ring; warp 1 owns TMEM and issues tcgen05.mma from one thread; warps 2..9 drain TMEM
// with tcgen05.ld.  Every mbarrier wait is bounded: on time-out the kernel records an error
// code, stops issuing work, waits (bounded) for what it already issued and frees TMEM.
#include "split.cuh"

#include <cuda.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "kernels.cuh"

namespace gg {

struct SplitGemm {
  DevBuf<int8_t> a8, b8;
  DevBuf<int> ea, eb, err;
  DevBuf<double2> work;
  int err_host = 0;
};

namespace {

constexpr int BM = 128;        // UMMA M (rows of A per tile)
constexpr int KB = 64;         // K bytes per pipeline stage (one 64-byte swizzle row)
constexpr int NTHREADS = 320;  // 10 warps
constexpr long long WAIT_CYCLES = 4000000000LL;  // ~2 s at B200 clocks

// ------------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait; returns false (and records `code`) on time-out or when another role failed
// (abort_on_err = false for the teardown waits that must see in-flight work complete)
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* err, int code,
                                          bool abort_on_err = true) {
  const long long t0 = clock64();
  int n = 0;
  while (!mbar_try(b, parity)) {
    if (++n == 64) {
      n = 0;
      if (abort_on_err && *err) return false;
      if (clock64() - t0 > WAIT_CYCLES) {
        atomicOr((int*)err, code);
        return false;
      }
    }
  }
  return true;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ uint64_t sw64_desc(const void* p) {
  // K-major, 64-byte swizzle: SBO = 512 B (8 rows x 64 B), LBO unused (1), version 1
  const uint64_t a = (smem_u32(p) >> 4) & 0x3FFF;
  return a | (1ull << 16) | (32ull << 32) | (1ull << 46) | (4ull << 61);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void mma_commit(uint64_t* b) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(b))
               : "memory");
}
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, int* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, int* r) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

struct I8Args {
  int S;
  int rows_a_pad, rows_b_pad;  // per (batch, slice)
  int nkb;                     // K blocks of 64 bytes
  int kcb;                     // K blocks per exact int32 chunk
  int M, N;                    // complex output dims
  int tiles_m, tiles_n, splits;
  int nb0, nb1;
  long batch;
  long units;                  // tiles_m * tiles_n * splits * batch work units
  const int* ea;  // [batch][rows_a_pad]
  const int* eb;  // [batch][N]
  // output: workspace [split][batch][M][N] when splits > 1, else C through the maps
  double2* work;
  double2* C;
  IdxMap c_m, c_n;
  long c_b0, c_b1, c_b2;
  double2 alpha, beta;
  int stages;
  int tmem_cols;
  int nbuf;  // accumulator sets in TMEM (1 or 2)
  int* err;
};

struct Unit {
  long batch;
  int split, m0, n0, kb0, kb1;
};

__device__ __forceinline__ Unit unit_of(const I8Args& p, long u, int BN) {
  Unit w;
  const int ntile = p.tiles_m * p.tiles_n;
  const int tile = (int)(u % ntile);
  const long rest = u / ntile;
  w.split = (int)(rest % p.splits);
  w.batch = rest / p.splits;
  w.m0 = (tile % p.tiles_m) * BM;
  w.n0 = (tile / p.tiles_m) * BN;
  w.kb0 = (int)((long)p.nkb * w.split / p.splits);
  w.kb1 = (int)((long)p.nkb * (w.split + 1) / p.splits);
  return w;
}

__device__ __forceinline__ bool seg_last(const Unit& w, int kb, int kcb) {
  return (kb + 1 == w.kb1) || ((kb + 1) % kcb == 0);
}

// Persistent: one CTA per SM walks the work units u = blockIdx.x + i * gridDim.x.  The TMA
// ring runs on across units; TMEM holds nbuf accumulator sets (S diagonals x BN columns
// each).  With two sets, consecutive K segments alternate so that draining one overlaps the
// MMAs of the next; with one set the tile is as wide as 512 / S columns allow, which halves
// the operand bytes per MAC - the better trade when L2 bandwidth is the limit.
template <int BN>
__global__ void __launch_bounds__(NTHREADS, 1)
    i8_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, I8Args p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int S = p.S;
  const int stA = S * BM * KB, stB = S * BN * KB;
  uint8_t* sA = smem;
  uint8_t* sB = smem + p.stages * stA;
  uint64_t* full = (uint64_t*)(sB + p.stages * stB);
  uint64_t* empty = full + p.stages;
  uint64_t* accf = empty + p.stages;   // [2]
  uint64_t* acce = accf + 2;           // [2]
  uint64_t* fin = acce + 2;
  uint32_t* tslot = (uint32_t*)(fin + 1);
  volatile int* err = p.err;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int i = 0; i < p.stages; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 8);
    }
    mbar_init(fin, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(p.tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t buf_cols = (uint32_t)(S * BN);

  if (warp == 0) {
    // ---------------- TMA producer
    if (lane == 0) {
      long it = 0;
      bool ok = true;
      for (long u = blockIdx.x; u < p.units && ok; u += gridDim.x) {
        const Unit w = unit_of(p, u, BN);
        const int rowA = (int)((w.batch * S) * p.rows_a_pad + w.m0);
        const int rowB = (int)((w.batch * S) * p.rows_b_pad + w.n0);
        for (int kb = w.kb0; kb < w.kb1; ++kb, ++it) {
          const int st = (int)(it % p.stages);
          const uint32_t round = (uint32_t)(it / p.stages);
          if (!mbar_wait(&empty[st], (round & 1) ^ 1, err, 1)) { ok = false; break; }
          mbar_expect_tx(&full[st], (uint32_t)(stA + stB));
          for (int s = 0; s < S; ++s) {
            tma_load_2d(sA + st * stA + s * BM * KB, &tmA, kb * KB, rowA + s * p.rows_a_pad, &full[st]);
            tma_load_2d(sB + st * stB + s * BN * KB, &tmB, kb * KB, rowB + s * p.rows_b_pad, &full[st]);
          }
        }
      }
      // on failure, let the copies already issued land before the CTA can exit
      if (!ok)
        for (long j = (it > p.stages ? it - p.stages : 0); j < it; ++j)
          mbar_wait(&full[j % p.stages], (uint32_t)((j / p.stages) & 1), err, 16, false);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer
    if (lane == 0) {
      const uint32_t idesc =
          (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
      long it = 0, g = 0;
      bool ok = true;
      for (long u = blockIdx.x; u < p.units && ok; u += gridDim.x) {
        const Unit w = unit_of(p, u, BN);
        for (int kb = w.kb0; kb < w.kb1 && ok; ++kb, ++it) {
          const int st = (int)(it % p.stages);
          const uint32_t round = (uint32_t)(it / p.stages);
          const bool first_in_seg = (kb == w.kb0) || (kb % p.kcb == 0);
          const int buf = (int)(g % p.nbuf);
          if (first_in_seg && g >= p.nbuf) {
            if (!mbar_wait(&acce[buf], (uint32_t)(((g / p.nbuf) - 1) & 1), err, 2)) { ok = false; break; }
          }
          if (!mbar_wait(&full[st], round & 1, err, 4)) { ok = false; break; }
          tc_fence_after();
          const uint8_t* a = sA + st * stA;
          const uint8_t* b = sB + st * stB;
          for (int d = 2; d <= S + 1; ++d) {
            const uint32_t tacc = tmem + (uint32_t)buf * buf_cols + (uint32_t)((d - 2) * BN);
            const int s_lo = d - S > 1 ? d - S : 1, s_hi = d - 1 < S ? d - 1 : S;
            for (int s = s_lo; s <= s_hi; ++s) {
              const int t = d - s;
              const uint64_t da = sw64_desc(a + (s - 1) * BM * KB);
              const uint64_t db = sw64_desc(b + (t - 1) * BN * KB);
#pragma unroll
              for (int kk = 0; kk < KB / 32; ++kk) {
                const uint32_t accum = (first_in_seg && s == s_lo && kk == 0) ? 0u : 1u;
                mma_i8(tacc, da + (uint64_t)(kk * 2), db + (uint64_t)(kk * 2), idesc, accum);
              }
            }
          }
          mma_commit(&empty[st]);
          if (seg_last(w, kb, p.kcb)) {
            mma_commit(&accf[buf]);
            ++g;
          }
        }
      }
      // all MMAs issued by this thread complete before TMEM can be freed
      mma_commit(fin);
      mbar_wait(fin, 0, err, 32, false);
    }
  } else {
    // ---------------- epilogue: 8 warps, lanes 32*(warp%4).., column half (warp-2)/4
    const int q = warp & 3, h = (warp - 2) >> 2;
    const int row = q * 32 + lane;
    constexpr int HC = BN / 2;  // int32 columns per thread
    double acc[HC];
    long g = 0;
    bool ok = true;
    for (long u = blockIdx.x; u < p.units && ok; u += gridDim.x) {
      const Unit w = unit_of(p, u, BN);
#pragma unroll
      for (int i = 0; i < HC; ++i) acc[i] = 0.0;
      for (int kb = w.kb0; kb < w.kb1; ++kb) {
        if (!seg_last(w, kb, p.kcb)) continue;
        const int buf = (int)(g % p.nbuf);
        if (!mbar_wait(&accf[buf], (uint32_t)((g / p.nbuf) & 1), err, 8)) { ok = false; break; }
        tc_fence_after();
        for (int d = 2; d <= S + 1; ++d) {
          const double scale = ldexp(1.0, -7 * d);
          const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)buf * buf_cols +
                                (uint32_t)((d - 2) * BN + h * HC);
#pragma unroll
          for (int j = 0; j < HC / 16; ++j) {
            int r[16];
            tmem_ld16(base + j * 16, r);
#pragma unroll
            for (int i = 0; i < 16; ++i) acc[j * 16 + i] += (double)r[i] * scale;
          }
          if constexpr (HC % 16 == 8) {
            // BN = 48 / 80: the last 8 columns of the half
            int r[8];
            tmem_ld8(base + (HC / 16) * 16, r);
#pragma unroll
            for (int i = 0; i < 8; ++i) acc[(HC / 16) * 16 + i] += (double)r[i] * scale;
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&acce[buf]);
        ++g;
      }
      if (!ok || *err) break;
      const int m = w.m0 + row;
      if (m < p.M) {
        const int ea = p.ea[w.batch * p.rows_a_pad + m];
        const int b0 = (int)(w.batch % p.nb0);
        const int b1 = (int)((w.batch / p.nb0) % p.nb1);
        const int b2 = (int)(w.batch / ((long)p.nb0 * p.nb1));
        const bool use_beta = p.beta.x != 0.0 || p.beta.y != 0.0;
        const int nbase = (w.n0 + h * HC) / 2;
#pragma unroll
        for (int c = 0; c < HC / 2; ++c) {
          const int n = nbase + c;
          if (n < p.N) {
            const int e = ea + __ldg(&p.eb[w.batch * p.N + n]);
            const double2 v = make_double2(ldexp(acc[2 * c], e), ldexp(acc[2 * c + 1], e));
            if (p.splits > 1) {
              p.work[((w.split * p.batch + w.batch) * p.M + m) * (long)p.N + n] = v;
            } else {
              double2* cp = p.C + b0 * p.c_b0 + b1 * p.c_b1 + b2 * p.c_b2 + p.c_m(m) + p.c_n(n);
              double2 o = cmul(p.alpha, v);
              if (use_beta) o = cadd(o, cmul(p.beta, *cp));
              *cp = o;
            }
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(p.tmem_cols));
  }
}

// ------------------------------------------------------------------ slicing
// Operand view: element (r, kb, k) of batch b = base + b-offset + map(r) + kb * kbs + k * ks
struct OpView {
  const double2* base;
  IdxMap rmap;
  long kbs, ks;
  int KB, K, R;
  int nb0, nb1;
  long b0s, b1s, b2s;
  int conj;
  __device__ __forceinline__ const double2* ptr(long b) const {
    const int b0 = (int)(b % nb0), b1 = (int)((b / nb0) % nb1), b2 = (int)(b / ((long)nb0 * nb1));
    return base + b0 * b0s + b1 * b1s + b2 * b2s;
  }
};

// exponent per (batch, row): e with max |x| < 2^e over all (kb, k); one warp per row
__global__ void row_exponent_kernel(OpView v, int rows_pad, int* out, long nbatch) {
  const long gw = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const long total = nbatch * rows_pad;
  if (gw >= total) return;
  const long b = gw / rows_pad;
  const int r = (int)(gw % rows_pad);
  double mx = 0.0;
  if (r < v.R) {
    const double2* base = v.ptr(b) + v.rmap(r);
    const long n = (long)v.KB * v.K;
    for (long i = lane; i < n; i += 32) {
      const long kb = i / v.K, k = i % v.K;
      const double2 x = base[kb * v.kbs + k * v.ks];
      mx = fmax(mx, fmax(fabs(x.x), fabs(x.y)));
    }
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (lane == 0) out[gw] = mx > 0.0 ? ilogb(mx) + 1 : 0;
}

// same, for operands whose rows are contiguous in memory: one thread per row, loop over k
// (consecutive threads read consecutive addresses)
__global__ void row_exponent_rc_kernel(OpView v, int rows_pad, int* out, long nbatch) {
  const long gt = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (gt >= nbatch * rows_pad) return;
  const long b = gt / rows_pad;
  const int r = (int)(gt % rows_pad);
  double mx = 0.0;
  if (r < v.R) {
    const double2* base = v.ptr(b) + v.rmap(r);
    for (int kb = 0; kb < v.KB; ++kb)
      for (int k = 0; k < v.K; ++k) {
        const double2 x = base[kb * v.kbs + (long)k * v.ks];
        mx = fmax(mx, fmax(fabs(x.x), fabs(x.y)));
      }
  }
  out[gt] = mx > 0.0 ? ilogb(mx) + 1 : 0;
}

// cut x (|x| < 1 after scaling) into S int8 slices by truncation
__device__ __forceinline__ void cut(double x, int S, int8_t* d) {
  for (int s = 0; s < S; ++s) {
    x *= 128.0;
    const double t = trunc(x);
    d[s] = (int8_t)t;
    x -= t;
  }
}

// Slices of a row operand (A side): out[((b*S + s)*rows_pad + r)*kp + 2*kk + {0,1}].
// A 32 x 32 (row, kk) tile goes through shared memory so global reads follow the
// operand's contiguous direction (rows or k) and writes are along k.
template <bool BSIDE>
__global__ void slice_kernel(OpView v, int S, int rows_pad, long kp, const int* ex, int8_t* out, long nbatch) {
  __shared__ double2 tile[32][33];
  const long Ktot = (long)v.KB * v.K;
  const long ktiles = (kp / 2 + 31) / 32;
  const long rtiles = rows_pad / 32;
  long t = blockIdx.x;
  const long kt = t % ktiles;
  t /= ktiles;
  const long rt = t % rtiles;
  const long b = t / rtiles;
  if (b >= nbatch) return;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  const double2* base = v.ptr(b);
  const bool rcontig = (v.rmap.split == 0 && v.rmap.lo == 1) || (v.rmap.split > 0 && v.rmap.lo == 1);
  // load: tile[rr][kk]
  for (int i = ty; i < 32; i += 8) {
    int rr, kk;
    if (rcontig) { rr = tx; kk = i; } else { rr = i; kk = tx; }
    const long r = rt * 32 + rr, k = kt * 32 + kk;
    double2 x = make_double2(0.0, 0.0);
    if (r < v.R && k < Ktot) {
      const long kbi = k / v.K, ki = k % v.K;
      x = base[v.rmap(r) + kbi * v.kbs + ki * v.ks];
      if (v.conj) x.y = -x.y;
    }
    tile[rr][kk] = x;
  }
  __syncthreads();
  // write: thread (ty -> row, tx -> kk)
  for (int i = ty; i < 32; i += 8) {
    const long r = rt * 32 + i, kk = kt * 32 + tx;
    if (r >= rows_pad || 2 * kk >= kp) continue;
    const double2 x = tile[i][tx];
    const int e = (r < v.R) ? ex[b * (BSIDE ? v.R : rows_pad) + r] : 0;
    int8_t dr[8], di[8];
    cut(ldexp(x.x, -e), S, dr);
    cut(ldexp(x.y, -e), S, di);
    if (!BSIDE) {
      for (int s = 0; s < S; ++s) {
        int8_t* o = out + (((b * S + s) * rows_pad + r) * kp + 2 * kk);
        *(char2*)o = make_char2(dr[s], di[s]);
      }
    } else {
      // B' rows 2r: (re, -im); 2r + 1: (im, re); rows_pad here counts complex columns
      for (int s = 0; s < S; ++s) {
        int8_t* o0 = out + (((b * S + s) * (2L * rows_pad) + 2 * r) * kp + 2 * kk);
        int8_t* o1 = o0 + kp;
        *(char2*)o0 = make_char2(dr[s], (int8_t)(-di[s]));
        *(char2*)o1 = make_char2(di[s], dr[s]);
      }
    }
  }
}

__global__ void split_reduce_kernel(const double2* work, int splits, long batch_count, int M, int N, double2* C,
                                    IdxMap c_m, IdxMap c_n, int nb0, int nb1, long c_b0, long c_b1, long c_b2,
                                    double2 alpha, double2 beta) {
  const long mn = (long)M * N;
  const long total = batch_count * mn;
  const bool use_beta = beta.x != 0.0 || beta.y != 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const long b = i / mn, e = i % mn;
    double2 acc = make_double2(0.0, 0.0);
    for (int s = 0; s < splits; ++s) acc = cadd(acc, work[(s * batch_count + b) * mn + e]);
    const int m = (int)(e / N), n = (int)(e % N);
    const int b0 = (int)(b % nb0), b1 = (int)((b / nb0) % nb1), b2 = (int)(b / ((long)nb0 * nb1));
    double2* cp = C + b0 * c_b0 + b1 * c_b1 + b2 * c_b2 + c_m(m) + c_n(n);
    double2 o = cmul(alpha, acc);
    if (use_beta) o = cadd(o, cmul(beta, *cp));
    *cp = o;
  }
}

// ------------------------------------------------------------------ host side
typedef CUresult (*EncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
  static EncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiled)p;
  });
  if (!fn) throw Error(GG_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  return fn;
}

CUtensorMap make_map(const int8_t* base, long kp, long rows, int box_rows) {
  CUtensorMap m;
  std::memset(&m, 0, sizeof(m));
  const cuuint64_t dims[2] = {(cuuint64_t)kp, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)kp};
  const cuuint32_t box[2] = {(cuuint32_t)KB, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void*)base, dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw Error(GG_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return m;
}

int sms() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    GG_CUDA(cudaGetDevice(&dev));
    GG_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  }
  return n;
}

template <int BN>
void launch_i8(const CUtensorMap& ta, const CUtensorMap& tb, const I8Args& a, long blocks, size_t smem,
               cudaStream_t st) {
  static bool cfg = false;
  if (!cfg) {
    GG_CUDA(cudaFuncSetAttribute(i8_gemm_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, 232448));
    cfg = true;
  }
  i8_gemm_kernel<BN><<<(unsigned)blocks, NTHREADS, smem, st>>>(ta, tb, a);
  GG_CHECK_LAUNCH();
}

}  // namespace

SplitGemm* split_engine(gg_context* c) {
  static std::mutex mu;
  std::lock_guard<std::mutex> g(mu);
  if (!c->split) c->split = new SplitGemm();
  encode_fn();
  return c->split;
}

void split_release(SplitGemm* e) { delete e; }

int split_zgemm(SplitGemm* e, const ZgemmDesc& d, int S, cudaStream_t st) {
  if (S < 2 || S > 8) throw Error(GG_ERR_ARG, "split: slices must be in [2, 8]");
  if (d.M <= 0 || d.N <= 0) return 0;
  // nbuf accumulator sets of S diagonals x BN columns must fit the 512 TMEM columns;
  // BN <= 128 keeps the FP64 drain registers (BN / 2 per thread) in budget
  const int nbuf = S <= 2 ? 2 : 1;
  const int BN = S <= 4 ? 128 : S == 5 ? 96 : S == 6 ? 80 : 64;
  const int bn_pad = BN * 64 / std::__gcd(BN, 64);  // keeps rows_b_pad / 2 a multiple of 32
  const long batch = (long)d.nb0 * d.nb1 * d.nb2;
  const long Ktot = (long)d.KB * d.K;
  const long kp = ((2 * Ktot + KB - 1) / KB) * KB;
  const int rows_a_pad = ((d.M + BM - 1) / BM) * BM;
  const int np = 2 * d.N;
  const int rows_b_pad = ((np + bn_pad - 1) / bn_pad) * bn_pad;  // B' rows (2 per complex column)
  const int ncol_pad = rows_b_pad / 2;                // complex columns incl. padding
  // exact int32 chunk: S * Kchunk * 127^2 < 2^31
  const long kchunk = std::max<long>(KB, ((2147483647L / (16129L * S)) / KB) * KB);
  const int kcb = (int)(kchunk / KB);
  const int nkb = (int)(kp / KB);

  int8_t* a8 = e->a8.ensure((size_t)batch * S * rows_a_pad * kp);
  int8_t* b8 = e->b8.ensure((size_t)batch * S * rows_b_pad * kp);
  int* ea = e->ea.ensure((size_t)batch * rows_a_pad);
  int* eb = e->eb.ensure((size_t)batch * d.N);
  int* err = e->err.p;
  if (!err) {
    err = e->err.ensure(1);
    GG_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
  }

  OpView va{d.A, d.a_m, d.a_kb, d.a_k, d.KB, d.K, d.M, d.nb0, d.nb1, d.a_b0, d.a_b1, d.a_b2, d.conjA};
  OpView vb{d.B, d.b_n, d.b_kb, d.b_k, d.KB, d.K, d.N, d.nb0, d.nb1, d.b_b0, d.b_b1, d.b_b2, d.conjB};
  int launches = 0;
  {
    auto exponents = [&](const OpView& v, int rows_pad, int* out) {
      const bool rcontig = v.rmap.lo == 1 && v.ks != 1;
      const long n = batch * rows_pad;
      if (rcontig)
        row_exponent_rc_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(v, rows_pad, out, batch);
      else
        row_exponent_kernel<<<(unsigned)((n * 32 + 255) / 256), 256, 0, st>>>(v, rows_pad, out, batch);
      GG_CHECK_LAUNCH();
    };
    exponents(va, rows_a_pad, ea);
    exponents(vb, d.N, eb);
    const long ktiles = (kp / 2 + 31) / 32;
    slice_kernel<false><<<(unsigned)(ktiles * (rows_a_pad / 32) * batch), 256, 0, st>>>(va, S, rows_a_pad, kp, ea, a8,
                                                                                        batch);
    GG_CHECK_LAUNCH();
    slice_kernel<true><<<(unsigned)(ktiles * (ncol_pad / 32) * batch), 256, 0, st>>>(vb, S, ncol_pad, kp, eb, b8,
                                                                                    batch);
    GG_CHECK_LAUNCH();
    launches += 4;
  }
  const CUtensorMap ta = make_map(a8, kp, (long)batch * S * rows_a_pad, BM);
  const CUtensorMap tb = make_map(b8, kp, (long)batch * S * rows_b_pad, BN);

  I8Args a{};
  a.S = S;
  a.rows_a_pad = rows_a_pad;
  a.rows_b_pad = rows_b_pad;
  a.nkb = nkb;
  a.kcb = kcb;
  a.M = d.M;
  a.N = d.N;
  a.tiles_m = rows_a_pad / BM;
  a.tiles_n = rows_b_pad / BN;
  a.nb0 = d.nb0;
  a.nb1 = d.nb1;
  a.batch = batch;
  a.ea = ea;
  a.eb = eb;
  a.C = d.C;
  a.c_m = d.c_m;
  a.c_n = d.c_n;
  a.c_b0 = d.c_b0;
  a.c_b1 = d.c_b1;
  a.c_b2 = d.c_b2;
  a.alpha = d.alpha;
  a.beta = d.beta;
  a.err = err;
  a.nbuf = nbuf;
  a.tmem_cols = 32;
  while (a.tmem_cols < nbuf * S * BN) a.tmem_cols *= 2;
  const size_t stage_bytes = (size_t)S * (BM + BN) * KB;
  a.stages = (int)std::min<size_t>(4, (220 * 1024 - 2048) / stage_bytes);
  if (a.stages < 2) throw Error(GG_ERR_ARG, "split: stage does not fit shared memory");
  const size_t smem = a.stages * stage_bytes + 1024 + 256;
  const long base = (long)a.tiles_m * a.tiles_n * batch;
  // split-K so that the units fill whole waves of persistent CTAs (each split keeps >= 8 K blocks)
  int splits = 1;
  {
    const int smax = (int)std::max<long>(1, std::min<long>(nkb / 8, 64));
    double best = 0.0;
    for (int sp = 1; sp <= smax; ++sp) {
      const long units = base * sp;
      const long waves = (units + sms() - 1) / sms();
      const double eff = (double)units / (double)(waves * sms());
      // prefer fewer splits unless a larger count fills the machine noticeably better
      if (eff > best + 0.05) {
        best = eff;
        splits = sp;
      }
      if (units >= 4L * sms()) break;
    }
  }
  const long need = (long)d.M * d.N * batch;
  if (splits > 1) {
    e->work.ensure((size_t)splits * need);
  }
  a.splits = splits;
  a.work = e->work.p;
  a.units = base * splits;
  const long grid = std::min<long>(a.units, sms());
  switch (BN) {
    case 128: launch_i8<128>(ta, tb, a, grid, smem, st); break;
    case 96: launch_i8<96>(ta, tb, a, grid, smem, st); break;
    case 80: launch_i8<80>(ta, tb, a, grid, smem, st); break;
    default: launch_i8<64>(ta, tb, a, grid, smem, st); break;
  }
  ++launches;
  if (splits > 1) {
    const long total = need;
    const long nblk = std::min<long>((total + 255) / 256, 65535L * 8);
    split_reduce_kernel<<<(unsigned)nblk, 256, 0, st>>>(e->work.p, splits, batch, d.M, d.N, d.C, d.c_m, d.c_n, d.nb0,
                                                       d.nb1, d.c_b0, d.c_b1, d.c_b2, d.alpha, d.beta);
    GG_CHECK_LAUNCH();
    ++launches;
  }
  return launches;
}

void split_check(SplitGemm* e, cudaStream_t st) {
  if (!e || !e->err.p) return;
  GG_CUDA(cudaMemcpyAsync(&e->err_host, e->err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  GG_CUDA(cudaStreamSynchronize(st));
  const int h = e->err_host;
  if (h) {
    GG_CUDA(cudaMemsetAsync(e->err.p, 0, sizeof(int), st));
    GG_CUDA(cudaStreamSynchronize(st));
    throw Error(GG_ERR_INTERNAL, "split GEMM: pipeline wait timed out (code " + std::to_string(h) + ")");
  }
}

}  // namespace gg
