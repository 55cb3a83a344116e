// Split-precision complex GEMM on the 5th-generation tensor cores (tcgen05, kind::i8).
//
// Ozaki scheme with exact INT8 slices:
//   * every row m of A (over the whole reduction K, all K-batches) gets an exponent e_m with
//     max_k |A(m,k)| < 2^e_m; x = A / 2^e_m is cut into S slices by rounding to nearest,
//     a_1 = rint(2^6 x), a_s = rint(2^7 r_{s-1}) (|a_s| <= 64, all steps exact in FP64), so
//     A = 2^(e_m+1) sum_s a_s 2^-7s + O(2^(e_m - 7S)) with an unbiased residual.  Columns of
//     B likewise with f_n.
//   * complex arithmetic is one real GEMM of size M x 2N x 2K: A' rows interleave (re, im)
//     along K, B' rows 2n / 2n+1 hold (re, -im) / (im, re), so C'(m, 2n) = Re C(m,n) and
//     C'(m, 2n+1) = Im C(m,n).
//   * the products a_s b_t with s + t = d share the scale 2^-7d and accumulate into one
//     int32 TMEM accumulator per diagonal d = 2..S+1 (pairs with s + t > S + 1 are dropped,
//     the usual triangular truncation).  K is processed in chunks small enough that no
//     int32 sum can overflow (S * Kchunk * 64^2 < 2^31), so every chunk is exact; chunks
//     are drained to FP64 registers and scaled by 2^(e_m + f_n + 2 - 7d).
//
// Slice layout in HBM: K-blocked planes, slice[(b * S + s) * nkb + kb][row][64 bytes], so that
// the rows x 64 bytes box of one K block is one contiguous run (a row-major [row][K] layout
// makes every box row a separate 64-byte access strided by the whole K length, which for
// the long reductions of the polarization contraction leaves DRAM pages mostly unused).
//
// Kernel roles (one CTA per SM, 320 threads): warp 0 issues TMA loads (3D tensor maps over
// the planes, 64-byte swizzle, each CTA loading only for itself) of all S slices of an A
// and a B K-block into a
// ring; warp 1 owns TMEM and issues tcgen05.mma from one thread; warps 2..9 drain TMEM
// with tcgen05.ld.  Every mbarrier wait is bounded: on time-out the kernel records an error
// code, stops issuing work, waits (bounded) for what it already issued and frees TMEM.
#include "split.cuh"

#include <cuda.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include "kernels.cuh"

namespace gg {

struct SplitGemm {
  DevBuf<int8_t> a8, b8;
  DevBuf<int> ea, eb, err;
  DevBuf<double2> work;
  int err_host = 0;
  bool timeout_test = false;  // the next launch runs the time-out test (one-shot)
  // tile autotuner: per GEMM shape the (tile width, split-K factor) that measured fastest
  bool autotune = false;
  struct Choice {
    int BN, splits;
    double ms;
  };
  std::map<std::array<long, 8>, Choice> tuned;
  std::string report;
};

namespace {

constexpr int BM = 128;        // UMMA M (rows of A per tile)
constexpr int KB = 64;         // K bytes per pipeline stage (one 64-byte swizzle row)
constexpr int EPI_WARPS = 16;  // epilogue warps: 4 TMEM lane quadrants x 4 column quarters
constexpr int NTHREADS = 32 * (2 + EPI_WARPS);  // + the TMA warp and the MMA warp
constexpr long long WAIT_CYCLES = 4000000000LL;  // ~2 s at B200 clocks

// ------------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes, uint32_t issue) {
  asm volatile(
      "{\n\t.reg .pred q;\n\t"
      "setp.ne.b32 q, %2, 0;\n\t"
      "@q mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n\t}" ::"r"(smem_u32(b)),
      "r"(bytes), "r"(issue)
      : "memory");
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
// try_wait with a suspend-time hint: a warp whose phase is not complete is suspended (it
// issues nothing, so the warps it shares a scheduler with keep their issue slots) until the
// phase completes or about `ns` nanoseconds pass
__device__ __forceinline__ bool mbar_try_sleep(uint64_t* b, uint32_t parity, uint32_t ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity), "r"(ns)
      : "memory");
  return ok != 0;
}
// bounded wait; returns false (and records `code`) on time-out or when another role failed
// (abort_on_err = false for the teardown waits that must see in-flight work complete).  The
// polling loop is a separate function so that the many inlined waits stay small.
__device__ __noinline__ bool mbar_wait_slow(uint64_t* b, uint32_t parity, volatile int* err, int code, long long limit,
                                            bool abort_on_err) {
  const long long t0 = clock64();
  while (!mbar_try_sleep(b, parity, 100000)) {  // <= 0.1 ms per suspension
    if (abort_on_err && *err) return false;
    if (clock64() - t0 > limit) {
      atomicOr((int*)err, code);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* err, int code, long long limit,
                                          bool abort_on_err = true) {
  if (mbar_try(b, parity)) return true;  // fast path: no clock read when the phase is complete
  return mbar_wait_slow(b, parity, err, code, limit, abort_on_err);
}

// box {64 bytes, rows, 1} at (0, row, plane); the innermost coordinate is always 0.
// Issued by the lane with issue != 0.
__device__ __forceinline__ void tma_load_plane(void* dst, const CUtensorMap* map, int row, int plane, uint64_t* bar,
                                               uint32_t issue) {
  asm volatile(
      "{\n\t.reg .pred q;\n\t"
      "setp.ne.b32 q, %6, 0;\n\t"
      "@q cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n\t}" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(0), "r"(row), "r"(plane), "r"(smem_u32(bar)), "r"(issue)
      : "memory");
}

__device__ __forceinline__ uint64_t sw64_desc(const void* p) {
  // K-major, 64-byte swizzle: SBO = 512 B (8 rows x 64 B), LBO unused (1), version 1
  const uint64_t a = (smem_u32(p) >> 4) & 0x3FFF;
  return a | (1ull << 16) | (32ull << 32) | (1ull << 46) | (4ull << 61);
}

// The issuing warps run their loops with all 32 lanes (warp-uniform control flow, so the
// descriptors and coordinates stay warp-uniform values); `issue` (lane 0) predicates the
// single-thread instructions inside the asm.
__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc,
                                       uint32_t issue) {
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "setp.ne.b32 q, %5, 0;\n\t"
      "@q tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(issue));
}
__device__ __forceinline__ void mma_commit(uint64_t* b, uint32_t issue) {
  asm volatile(
      "{\n\t.reg .pred q;\n\t"
      "setp.ne.b32 q, %1, 0;\n\t"
      "@q tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n\t}" ::"r"(smem_u32(b)),
      "r"(issue)
      : "memory");
}
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// TMEM loads without the wait (several loads share one tcgen05.wait::ld); reg_fence makes
// the loaded registers depend on the wait so no use is scheduled before it
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, int* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, int* r) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, int* r) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void reg_fence4(int* r) { asm volatile("" : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3])); }

// 2^e as a double, e clamped to the normal range (operand exponents come from ilogb of
// finite data, so a row factor times a column factor covers every representable result;
// the clamp only matters for results that underflow or overflow anyway)
__device__ __forceinline__ double pow2i(int e) {
  e = max(-1022, min(1023, e));
  return __longlong_as_double((long long)(e + 1023) << 52);
}

// drain `NC` int32 columns (a multiple of 4, at most 32) starting at taddr into acc * scale
template <int NC>
__device__ __forceinline__ void drain_cols(uint32_t taddr, double* acc, double scale) {
  static_assert(NC % 4 == 0 && NC <= 32, "TMEM loads of 4, 8 or 16 columns");
  int r[32];
#pragma unroll
  for (int j = 0; j < NC / 16; ++j) tmem_ld16(taddr + j * 16, r + j * 16);
  if constexpr (NC % 16 >= 8) tmem_ld8(taddr + (NC / 16) * 16, r + (NC / 16) * 16);
  if constexpr (NC % 8 == 4) tmem_ld4(taddr + (NC / 8) * 8, r + (NC / 8) * 8);
  tmem_wait_ld();
#pragma unroll
  for (int j = 0; j < NC / 4; ++j) reg_fence4(r + j * 4);
#pragma unroll
  for (int i = 0; i < NC; ++i) {
    // exact int32 -> double: the bits (0x43380000, r + 2^31) encode 2^52 + 2^51 + r + 2^31
    const double x = __hiloint2double(0x43380000, r[i] ^ (int)0x80000000) - 6755401588539392.0;
    acc[i] = fma(x, scale, acc[i]);
  }
}

// drain two adjacent diagonals d, d + 1 (`NC` int32 columns each, a multiple of 4, at most 16,
// starting at ta and tb) as one value 128 acc_d + acc_{d+1} = 2^7(d+1) (acc_d 2^-7d +
// acc_{d+1} 2^-7(d+1)): one conversion and one FMA per column pair instead of two each.  Exact
// when |128 acc_d| + |acc_{d+1}| < 2^31, which the host checks for the K segments of the launch
// (I8Args::pair).
template <int NC>
__device__ __forceinline__ void drain_pair_cols(uint32_t ta, uint32_t tb, double* acc, double scale) {
  static_assert(NC % 4 == 0 && NC <= 16, "TMEM loads of 4, 8 or 16 columns");
  int r[16], q[16];
  if constexpr (NC == 16) {
    tmem_ld16(ta, r);
    tmem_ld16(tb, q);
  } else {
    if constexpr (NC >= 8) {
      tmem_ld8(ta, r);
      tmem_ld8(tb, q);
    }
    if constexpr (NC % 8 == 4) {
      tmem_ld4(ta + (NC / 8) * 8, r + (NC / 8) * 8);
      tmem_ld4(tb + (NC / 8) * 8, q + (NC / 8) * 8);
    }
  }
  tmem_wait_ld();
#pragma unroll
  for (int j = 0; j < NC / 4; ++j) {
    reg_fence4(r + j * 4);
    reg_fence4(q + j * 4);
  }
#pragma unroll
  for (int i = 0; i < NC; ++i) {
    const int v = r[i] * 128 + q[i];
    const double x = __hiloint2double(0x43380000, v ^ (int)0x80000000) - 6755401588539392.0;
    acc[i] = fma(x, scale, acc[i]);
  }
}

// biased exponent of |x| (0 for x = 0); every nonzero accumulator value is a normal number
__device__ __forceinline__ int biased_exponent(double x) { return (__double2hiint(x) >> 20) & 0x7ff; }

struct I8Args {
  int S;
  int pair;  // the epilogue drains diagonals (2, 3), (4, 5), ... as pairs (exact: see drain_pair_cols)
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
  int a_shared, b_shared;  // operand identical for every batch: sliced once, planes / exponents of batch 0
  int* err;
  SplitRowMax mx;          // mx.on: the epilogue also records the row maxima of C
  long long wait_cycles;   // limit of every barrier wait (WAIT_CYCLES; shorter in the time-out test)
  int skip_arrive;         // time-out test: CTA 0's first epilogue warp never releases the first
                           // drained accumulator, so the MMA warp's wait for it must run out
};

struct Unit {
  long batch;
  int split, m0, n0, kb0, kb1;
};

__device__ __forceinline__ Unit unit_of(const I8Args& p, long u, int BN) {
  // 32-bit arithmetic: the host keeps units, splits * nkb and the batch count below 2^31
  const unsigned uu = (unsigned)u;
  const unsigned ntile = (unsigned)(p.tiles_m * p.tiles_n);
  const unsigned tile = uu % ntile, rest = uu / ntile;
  const unsigned spl = (unsigned)p.splits;
  Unit w;
  w.split = (int)(rest % spl);
  w.batch = (long)(rest / spl);
  w.m0 = (int)(tile % (unsigned)p.tiles_m) * BM;
  w.n0 = (int)(tile / (unsigned)p.tiles_m) * BN;
  w.kb0 = (int)((unsigned)p.nkb * (unsigned)w.split / spl);
  w.kb1 = (int)((unsigned)p.nkb * (unsigned)(w.split + 1) / spl);
  return w;
}

// MMAs of one K block: every slice pair (s, t) with s + t = d into the accumulator of
// diagonal d.  FIRST: the first K block of a segment (the first MMA of each diagonal
// overwrites it, and with `reuse` it first waits until the epilogue has drained that
// diagonal); LAST: the last K block (a commit per diagonal tells the epilogue that the
// diagonal is complete).  Descriptor offsets are compile-time constants.
template <int S, int BN, bool FIRST, bool LAST>
__device__ __forceinline__ bool issue_kblock(uint32_t tacc0, uint64_t da, uint64_t db, uint32_t idesc, uint32_t leader,
                                             bool reuse, uint64_t* acce, uint64_t* accf, uint32_t par_e,
                                             volatile int* err, long long limit) {
#pragma unroll
  for (int d = 2; d <= S + 1; ++d) {
    if (FIRST && reuse) {
      if (!__all_sync(0xffffffffu, mbar_wait(&acce[d - 2], par_e, err, 2, limit))) return false;
      tc_fence_after();
    }
    const uint32_t tacc = tacc0 + (uint32_t)((d - 2) * BN);
    const int s_lo = d - S > 1 ? d - S : 1, s_hi = d - 1 < S ? d - 1 : S;
#pragma unroll
    for (int s = s_lo; s <= s_hi; ++s) {
      const int t = d - s;
      const uint64_t a = da + (uint64_t)(((s - 1) * BM * KB) >> 4);
      const uint64_t b = db + (uint64_t)(((t - 1) * BN * KB) >> 4);
#pragma unroll
      for (int kk = 0; kk < KB / 32; ++kk)
        mma_i8(tacc, a + (uint64_t)(kk * 2), b + (uint64_t)(kk * 2), idesc, (FIRST && s == s_lo && kk == 0) ? 0u : 1u,
               leader);
    }
    if (LAST) mma_commit(&accf[d - 2], leader);
  }
  return true;
}

// A K block that neither starts nor ends an accumulation segment: the S + 1 - s products
// A_s B_t (t = 1..S+1-s) go to the adjacent accumulators of diagonals s+1..S+1, and the B
// slices lie next to each other in the stage, so one MMA with N = w * BN (w slices of B, N <=
// 256) covers w of them.  A_s is then read from shared memory once per group instead of
// once per slice of B (9 instead of 15 A reads per K step at S = 5).  The int32 sums are the
// same as with one MMA per slice pair.
template <int S, int BN>
__device__ __forceinline__ void issue_kblock_grouped(uint32_t tacc0, uint64_t da, uint64_t db, uint32_t idesc_nofield,
                                                     uint32_t leader) {
  constexpr int W = 256 / BN;  // B slices per MMA
  static_assert(W >= 1 && (BN % 16) == 0, "MMA N must be a multiple of 16 up to 256");
#pragma unroll
  for (int s = 1; s <= S; ++s) {
#pragma unroll
    for (int t0 = 1; t0 <= S + 1 - s; t0 += W) {
      const int w = (S + 2 - s - t0) < W ? (S + 2 - s - t0) : W;
      const uint32_t idesc = idesc_nofield | ((uint32_t)((w * BN) >> 3) << 17);
      const uint32_t tacc = tacc0 + (uint32_t)((s + t0 - 2) * BN);
#pragma unroll
      for (int kk = 0; kk < KB / 32; ++kk)
        mma_i8(tacc, da + (uint64_t)(((s - 1) * BM * KB) >> 4) + (uint64_t)(kk * 2),
               db + (uint64_t)(((t0 - 1) * BN * KB) >> 4) + (uint64_t)(kk * 2), idesc, 1u, leader);
    }
  }
}

// Persistent: one CTA per SM walks the work units u = blockIdx.x + i * gridDim.x.  The TMA
// ring runs on across units; TMEM holds nbuf accumulator sets (S diagonals x BN columns
// each).  Every diagonal has its own pair of barriers (MMAs done / drained), so the
// epilogue drains diagonal d while the MMAs of the later diagonals still run, and the next
// segment's MMAs into diagonal d start as soon as it is drained: with one set (S >= 3, the
// tile as wide as 512 / S columns allow) the drain overlaps the next tile's first K block,
// with two sets (S = 2) consecutive segments alternate.  S is a template parameter so the
// MMA issue loop unrolls into one tcgen05.mma per instruction slot with precomputed
// shared-memory descriptors.
template <int S, int BN>
__global__ void __launch_bounds__(NTHREADS, 1)
    i8_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, I8Args p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  constexpr int stA = S * BM * KB, stB = S * BN * KB;
  constexpr int ND = 8;  // barrier slots per accumulator set (one per diagonal, S <= 8)
  uint8_t* sA = smem;
  uint8_t* sB = smem + p.stages * stA;
  uint64_t* full = (uint64_t*)(sB + p.stages * stB);
  uint64_t* empty = full + p.stages;
  uint64_t* accf = empty + p.stages;   // [2][ND]
  uint64_t* acce = accf + 2 * ND;      // [2][ND]
  uint64_t* fin = acce + 2 * ND;
  uint32_t* tslot = (uint32_t*)(fin + 1);
  volatile int* err = p.err;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int i = 0; i < p.stages; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    for (int b = 0; b < 2 * ND; ++b) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], EPI_WARPS);
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
  constexpr uint32_t buf_cols = (uint32_t)(S * BN);

  const uint32_t leader = lane == 0 ? 1u : 0u;
  if (warp == 0) {
    // ---------------- TMA producer (whole warp, lane 0 issues)
    {
      // ring position (stage, phase) kept incrementally: no divisions in the K loop
      long it = 0;
      int st = 0;
      uint32_t ph = 0;
      bool ok = true;
      for (long u = blockIdx.x; u < p.units && ok; u += gridDim.x) {
        const Unit w = unit_of(p, u, BN);
        const int planeA0 = p.a_shared ? 0 : (int)(w.batch * S * p.nkb);
        const int planeB0 = p.b_shared ? 0 : (int)(w.batch * S * p.nkb);
        for (int kb = w.kb0; kb < w.kb1; ++kb, ++it) {
          if (!__all_sync(0xffffffffu, mbar_wait(&empty[st], ph ^ 1, err, 1, p.wait_cycles))) { ok = false; break; }
          mbar_expect_tx(&full[st], (uint32_t)(stA + stB), leader);
#pragma unroll
          for (int s = 0; s < S; ++s) {
            tma_load_plane(sA + st * stA + s * BM * KB, &tmA, w.m0, planeA0 + s * p.nkb + kb, &full[st], leader);
            tma_load_plane(sB + st * stB + s * BN * KB, &tmB, w.n0, planeB0 + s * p.nkb + kb, &full[st], leader);
          }
          if (++st == p.stages) {
            st = 0;
            ph ^= 1;
          }
        }
      }
      // let the copies already issued land before the CTA can exit: after a failure elsewhere
      // (the MMA warp stops consuming, so the last stages may still be in flight) and, at no
      // cost, after a normal run (those phases completed long ago)
      for (long j = (it > p.stages ? it - p.stages : 0); j < it; ++j)
        mbar_wait(&full[j % p.stages], (uint32_t)((j / p.stages) & 1), err, 16, p.wait_cycles, false);
      (void)ok;
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer (whole warp, lane 0 issues)
    {
      const uint32_t idesc_nofield = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BM >> 4) << 24);
      const uint32_t idesc = idesc_nofield | ((uint32_t)(BN >> 3) << 17);
      // descriptors of stage 0; a stage / slice / K offset adds (bytes >> 4) to the address
      // field (all of shared memory stays below 2^18 bytes, so the field never carries)
      const uint64_t dA0 = sw64_desc(sA), dB0 = sw64_desc(sB);
      // ring position (st, ph), accumulator set (buf) and its use count (use), and the
      // position inside the exact-int32 chunk (kin) are all kept incrementally
      int st = 0, buf = 0;
      uint32_t ph = 0;
      long use = 0;
      bool ok = true;
      for (long u = blockIdx.x; u < p.units && ok; u += gridDim.x) {
        const Unit w = unit_of(p, u, BN);
        int kin = w.kb0 % p.kcb;
        for (int kb = w.kb0; kb < w.kb1 && ok; ++kb) {
          const bool first = (kb == w.kb0) || kin == 0;
          const bool last = (kb + 1 == w.kb1) || kin + 1 == p.kcb;
          const bool reuse = first && use > 0;
          const uint32_t par_e = (uint32_t)((use - 1) & 1);
          if (!__all_sync(0xffffffffu, mbar_wait(&full[st], ph, err, 4, p.wait_cycles))) { ok = false; break; }
          tc_fence_after();
          const uint64_t da = dA0 + (uint64_t)((st * stA) >> 4);
          const uint64_t db = dB0 + (uint64_t)((st * stB) >> 4);
          const uint32_t tacc0 = tmem + (uint32_t)buf * buf_cols;
          uint64_t* ae = acce + buf * ND;
          uint64_t* af = accf + buf * ND;
          if (!first && !last)
            issue_kblock_grouped<S, BN>(tacc0, da, db, idesc_nofield, leader);
          else if (first && !last)
            ok = issue_kblock<S, BN, true, false>(tacc0, da, db, idesc, leader, reuse, ae, af, par_e, err, p.wait_cycles);
          else if (!first)
            issue_kblock<S, BN, false, true>(tacc0, da, db, idesc, leader, false, ae, af, 0u, err, p.wait_cycles);
          else
            ok = issue_kblock<S, BN, true, true>(tacc0, da, db, idesc, leader, reuse, ae, af, par_e, err, p.wait_cycles);
          if (!ok) break;
          mma_commit(&empty[st], leader);
          if (++st == p.stages) {
            st = 0;
            ph ^= 1;
          }
          if (++kin == p.kcb) kin = 0;
          if (last && ++buf == p.nbuf) {
            buf = 0;
            ++use;
          }
        }
      }
      // all MMAs issued by lane 0 complete before TMEM can be freed
      mma_commit(fin, leader);
      mbar_wait(fin, 0, err, 32, p.wait_cycles, false);
    }
  } else {
    // ---------------- epilogue: EPI_WARPS warps, lanes 32*(warp%4).. (the TMEM lane quadrant a
    // warp may access), column part (warp-2)/4 of EPI_WARPS/4
    const int q = warp & 3, h = (warp - 2) >> 2;
    const int row = q * 32 + lane;
    constexpr int HC = BN / (EPI_WARPS / 4);  // int32 columns per thread
    static_assert(HC % 4 == 0 && HC / 2 <= 32, "column part: a multiple of 4 int32 columns, at most 32 complex");
    double acc[HC];
    int buf = 0;
    uint32_t par = 0;
    bool ok = true;
    for (long u = blockIdx.x; u < p.units && ok; u += gridDim.x) {
      const Unit w = unit_of(p, u, BN);
      // exponents of this tile, loaded before the drain so that their latency overlaps it:
      // the row exponent per thread (padded rows carry exponent 0), the column exponents of
      // this half-tile one per lane, broadcast by shuffles in the output loop
      const int m = w.m0 + row;
      const int ea = p.ea[(p.a_shared ? 0 : w.batch) * p.rows_a_pad + m];
      const int nbase = (w.n0 + h * HC) / 2;
      const long ebo = (p.b_shared ? 0 : w.batch) * (long)p.N;
      const int eb_lane = (lane < HC / 2 && nbase + lane < p.N) ? p.eb[ebo + nbase + lane] : 0;
#pragma unroll
      for (int i = 0; i < HC; ++i) acc[i] = 0.0;
      // one drain per K segment: segments end at kb1 and at every multiple of kcb
      for (int k0 = w.kb0; k0 < w.kb1 && ok; k0 = min(w.kb1, (k0 / p.kcb + 1) * p.kcb)) {
        // a runtime loop over the diagonals: one copy of the drain code instead of S (the
        // unrolled form made the epilogue larger than the instruction cache, which stalled
        // the short-K GEMMs whose epilogue runs after every two K blocks)
#pragma unroll 1
        for (int d = 2; d <= S + 1;) {
          const bool two = p.pair && d + 1 <= S + 1;
          if (!mbar_wait(&accf[buf * ND + d - 2], par, err, 8, p.wait_cycles)) { ok = false; break; }
          if (two && !mbar_wait(&accf[buf * ND + d - 1], par, err, 8, p.wait_cycles)) { ok = false; break; }
          tc_fence_after();
          const int dl = two ? d + 1 : d;
          const double scale = __longlong_as_double((long long)(1023 - 7 * dl) << 52);  // 2^-7dl
          const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)buf * buf_cols +
                                (uint32_t)((d - 2) * BN + h * HC);
          if (two) {
            // groups of 8 columns of both diagonals, one wait per group (16 loaded registers:
            // wider groups spill at the register budget of 576 threads)
#pragma unroll
            for (int j = 0; j < HC / 8; ++j) drain_pair_cols<8>(base + j * 8, base + BN + j * 8, acc + j * 8, scale);
            if constexpr (HC % 8 != 0)
              drain_pair_cols<HC % 8>(base + (HC / 8) * 8, base + BN + (HC / 8) * 8, acc + (HC / 8) * 8, scale);
          } else {
            // groups of 32 columns, one wait per group
#pragma unroll
            for (int j = 0; j < HC / 32; ++j) drain_cols<32>(base + j * 32, acc + j * 32, scale);
            if constexpr (HC % 32 != 0) drain_cols<HC % 32>(base + (HC / 32) * 32, acc + (HC / 32) * 32, scale);
          }
          tc_fence_before();
          __syncwarp();
          const bool withheld = p.skip_arrive && blockIdx.x == 0 && warp == 2 && u == blockIdx.x && d == 2;
          if (lane == 0) {
            if (!withheld) mbar_arrive(&acce[buf * ND + d - 2]);
            if (two) mbar_arrive(&acce[buf * ND + d - 1]);
          }
          d += two ? 2 : 1;
        }
        if (++buf == p.nbuf) {
          buf = 0;
          par ^= 1;
        }
      }
      if (!ok) break;
      // output: consecutive lanes hold consecutive rows m, so every store instruction is
      // coalesced wherever C (or the split-K workspace, [split][batch][n][m]) is m-contiguous
      const int b0 = (int)(w.batch % p.nb0);
      const int b1 = (int)((w.batch / p.nb0) % p.nb1);
      const int b2 = (int)(w.batch / ((long)p.nb0 * p.nb1));
      const bool use_beta = p.beta.x != 0.0 || p.beta.y != 0.0;
      const bool alpha_one = p.alpha.x == 1.0 && p.alpha.y == 0.0;
      const bool mok = m < p.M;
      const double sa = pow2i(ea);  // row factor; x = 2 sum d_s 2^-7s per operand gives the + 2
      double2* crow = p.C + b0 * p.c_b0 + b1 * p.c_b1 + b2 * p.c_b2 + (mok ? p.c_m(m) : 0);
      double2* wrow = p.work + (w.split * p.batch + w.batch) * (long)p.N * p.M + m;
      if (p.mx.on) {
        // row maxima for the next GEMM (kept out of the store loop below, whose code stays
        // compact): a run of columns with the same column key is reduced per thread, then over
        // the lanes with the same target row (consecutive lanes: a segmented warp reduction;
        // the first lane of a segment does one atomicMax)
        const int xmq = m / p.mx.div_m, xmr = m - xmq * p.mx.div_m;
        const long xrow = w.batch * p.mx.s_b + xmq * p.mx.s_mq + xmr * p.mx.s_mr;
        int xq = nbase / p.mx.div_n, xr = nbase - xq * p.mx.div_n;
        // in exponents: ilogb(|acc| 2^(ea + eb + 2)) = ilogb|acc| + ea + eb + 2, so the largest
        // exponent of a run is found with integer maxima (the result is that of the largest
        // scaled value); kNone marks a run without a nonzero value
        constexpr int kNone = -(1 << 30);
        const int xoff = ea + 2 - 1023;
        int xe = kNone;
        auto xflush = [&](int colkey) {
          const long idx = xrow + colkey * p.mx.s_nq;
#pragma unroll
          for (int off = 1; off < 32; off <<= 1) {
            const int o = __shfl_down_sync(0xffffffffu, xe, off);
            const long oi = __shfl_down_sync(0xffffffffu, idx, off);
            if (lane + off < 32 && oi == idx) xe = max(xe, o);
          }
          const long prev = __shfl_up_sync(0xffffffffu, idx, 1);
          if ((lane == 0 || prev != idx) && xe != kNone) atomicMax(p.mx.ex + idx, xe + 1);
          xe = kNone;
        };
#pragma unroll
        for (int c = 0; c < HC / 2; ++c) {
          const int eb = __shfl_sync(0xffffffffu, eb_lane, c);
          if (mok && nbase + c < p.N) {
            const int be = max(biased_exponent(acc[2 * c]), biased_exponent(acc[2 * c + 1]));
            if (be != 0) xe = max(xe, be + eb + xoff);
          }
          if (++xr == p.mx.div_n) {
            xflush(xq);
            xr = 0;
            ++xq;
          }
        }
        if (xr != 0) xflush(xq);
      }
      // column offset c_n(n) stepped through the tile: (nq, nr) = divmod(n, split)
      const int csp = p.c_n.split > 0 ? p.c_n.split : 1 << 30;
      int nq = nbase / csp, nr = nbase - nq * csp;
#pragma unroll
      for (int c = 0; c < HC / 2; ++c) {
        const int eb = __shfl_sync(0xffffffffu, eb_lane, c);
        const int n = nbase + c;
        if (mok && n < p.N) {
          const double sb = pow2i(eb + 2);
          const double2 v = make_double2(acc[2 * c] * sa * sb, acc[2 * c + 1] * sa * sb);
          if (p.splits > 1) {
            wrow[(long)n * p.M] = v;
          } else {
            double2* cp = crow + (p.c_n.split > 0 ? nq * p.c_n.hi + nr * p.c_n.lo : (long)n * p.c_n.lo);
            double2 o = alpha_one ? v : cmul(p.alpha, v);
            if (use_beta) o = cadd(o, cmul(p.beta, *cp));
            *cp = o;
          }
        }
        if (++nr == csp) {
          nr = 0;
          ++nq;
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

// IdxMap with 32-bit index arithmetic (every row and K index of an operand is below 2^31)
__device__ __forceinline__ long map32(const IdxMap& m, int i) {
  if (m.split > 0) {
    const int q = i / m.split;
    return (long)q * m.hi + (long)(i - q * m.split) * m.lo;
  }
  return (long)i * m.lo;
}

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
    const double2* base = v.ptr(b) + map32(v.rmap, r);
    // (kb, k) stepped without divisions: lane i starts at i and advances by 32
    int kb = lane / v.K, k = lane - kb * v.K;
    const int step_kb = 32 / v.K, step_k = 32 - step_kb * v.K;
    for (; kb < v.KB; ) {
      const double2 x = base[(long)kb * v.kbs + (long)k * v.ks];
      mx = fmax(mx, fmax(fabs(x.x), fabs(x.y)));
      kb += step_kb;
      k += step_k;
      if (k >= v.K) {
        k -= v.K;
        ++kb;
      }
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
    const double2* base = v.ptr(b) + map32(v.rmap, r);
    for (int kb = 0; kb < v.KB; ++kb)
      for (int k = 0; k < v.K; ++k) {
        const double2 x = base[kb * v.kbs + (long)k * v.ks];
        mx = fmax(mx, fmax(fabs(x.x), fabs(x.y)));
      }
  }
  out[gt] = mx > 0.0 ? ilogb(mx) + 1 : 0;
}


// cut x (|x| < 1 after scaling) into S int8 slices by rounding to nearest:
// d_1 = rint(64 x), r_1 = 64 x - d_1 in [-1/2, 1/2]; d_s = rint(128 r_{s-1}), ...
// so x = 2 sum_s d_s 2^-7s + O(2^-7S), every |d_s| <= 64 and the residual is unbiased.
// rint is done by adding 2^52 + 2^51 (the sum is rounded to an integer, round-to-nearest-
// even like rint, and its low word holds that integer in two's complement); every step is
// exact in FP64 and uses only the add / fma pipes (measured faster than one rounding to int64
// followed by integer digit extraction).
template <int S>
__device__ __forceinline__ void cut(double x, int8_t* d) {
  const double RND = 6755399441055744.0;  // 2^52 + 2^51
  x *= 64.0;
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const double y = x + RND;
    d[s] = (int8_t)__double2loint(y);
    const double t = y - RND;
    x = (x - t) * 128.0;
  }
}

// x * 2^-e, exact while the result is a normal number (ldexp outside the directly encodable range)
__device__ __forceinline__ double scale_neg(double x, int e) {
  if (e > -1000 && e < 1000) return x * __longlong_as_double((long long)(1023 - e) << 52);
  return ldexp(x, -e);
}

// Slices of a row operand (A side): out[(((b*S + s)*nkb + kb)*rows_pad + r)*64 + 2*kk' + {0,1}]
// with kk = 32 kb + kk' (one 32-complex k tile is one 64-byte K block).  A 32 x 32 (row, kk)
// tile goes through shared memory so global reads follow the operand's contiguous direction
// (rows or k) and each warp writes 64 contiguous bytes.
template <bool BSIDE, int S>
__global__ void slice_kernel(OpView v, int rows_pad, int ktiles, const int* ex, int8_t* out, long nbatch) {
  __shared__ double2 tile[32][33];
  const int Ktot = v.KB * v.K;
  const int rtiles = (v.R + 31) / 32;  // valid rows only (padding rows are never written)
  long t = blockIdx.x;
  const int kt = (int)(t % ktiles);
  t /= ktiles;
  const int rt = (int)(t % rtiles);
  const long b = t / rtiles;
  if (b >= nbatch) return;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  const double2* base = v.ptr(b);
  const bool rcontig = v.rmap.lo == 1;
  // load: tile[rr][kk]
  if (rcontig) {
    // rr = tx (fixed row per thread), kk = i
    const int r = rt * 32 + tx;
    const bool rok = r < v.R;
    const double2* rowp = base + (rok ? map32(v.rmap, r) : 0);
    for (int i = ty; i < 32; i += 8) {
      const int k = kt * 32 + i;
      double2 x = make_double2(0.0, 0.0);
      if (rok && k < Ktot) {
        const int kbi = k / v.K, ki = k - kbi * v.K;
        x = rowp[kbi * v.kbs + (long)ki * v.ks];
        if (v.conj) x.y = -x.y;
      }
      tile[tx][i] = x;
    }
  } else {
    // kk = tx (fixed k per thread), rr = i
    const int k = kt * 32 + tx;
    const bool kok = k < Ktot;
    const int kbi = kok ? k / v.K : 0, ki = kok ? k - kbi * v.K : 0;
    const long koff = kbi * v.kbs + (long)ki * v.ks;
    for (int i = ty; i < 32; i += 8) {
      const int r = rt * 32 + i;
      double2 x = make_double2(0.0, 0.0);
      if (kok && r < v.R) {
        x = base[map32(v.rmap, r) + koff];
        if (v.conj) x.y = -x.y;
      }
      tile[i][tx] = x;
    }
  }
  __syncthreads();
  // write: thread (ty -> row, tx -> kk).  Plane addresses are formed once per thread and
  // stepped by the row and slice strides (the full index per store made this pass issue-bound).
  const long plane = (BSIDE ? 2L : 1L) * rows_pad * KB;  // bytes of one K-block plane
  const long sstride = (long)ktiles * plane;              // from slice s to s + 1
  const int8_t* const obase = out + (b * S * ktiles + kt) * plane + 2 * tx;
  const int* const exb = ex + b * (BSIDE ? v.R : rows_pad);
  for (int i = ty; i < 32; i += 8) {
    const int r = rt * 32 + i;
    if (r >= v.R) break;  // padding rows are read back as zeros by the tile loads
    const double2 x = tile[i][tx];
    const int e = exb[r];
    int8_t dr[S], di[S];
    cut<S>(scale_neg(x.x, e), dr);
    cut<S>(scale_neg(x.y, e), di);
    int8_t* o = const_cast<int8_t*>(obase) + (BSIDE ? 2L * r : (long)r) * KB;
    if (!BSIDE) {
#pragma unroll
      for (int s = 0; s < S; ++s, o += sstride) *(char2*)o = make_char2(dr[s], di[s]);
    } else {
      // B' rows 2r: (re, -im); 2r + 1: (im, re); rows_pad here counts complex columns
#pragma unroll
      for (int s = 0; s < S; ++s, o += sstride) {
        *(char2*)o = make_char2(dr[s], (int8_t)(-di[s]));
        *(char2*)(o + KB) = make_char2(di[s], dr[s]);
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
    const long b = i / mn, e = i % mn;  // e = n * M + m (the workspace is m-contiguous)
    double2 acc = make_double2(0.0, 0.0);
    for (int s = 0; s < splits; ++s) acc = cadd(acc, work[(s * batch_count + b) * mn + e]);
    const int n = (int)(e / M), m = (int)(e % M);
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

// planes of rows_pad x 64 bytes; box = one K block of box_rows rows
// planes of rows_pad x 64 bytes of which the first `rows` hold data: the map's row extent is
// `rows`, so tile loads over the padding rows read zeros (out-of-bounds fill) and the slicing
// pass need not write them
CUtensorMap make_map(const int8_t* base, long rows, long rows_pad, long planes, int box_rows) {
  if (planes > 0x7fffffffL) throw Error(GG_ERR_ARG, "split: too many K-block planes for a tensor map");
  if (rows < 1 || rows > rows_pad) throw Error(GG_ERR_ARG, "split: bad plane rows");
  CUtensorMap m;
  std::memset(&m, 0, sizeof(m));
  const cuuint64_t dims[3] = {(cuuint64_t)KB, (cuuint64_t)rows, (cuuint64_t)planes};
  const cuuint64_t strides[2] = {(cuuint64_t)KB, (cuuint64_t)(rows_pad * KB)};
  const cuuint32_t box[3] = {(cuuint32_t)KB, (cuuint32_t)box_rows, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, (void*)base, dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw Error(GG_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return m;
}

int sms() { return device_sm_count(); }

template <int S, int BN>
void launch_i8(const CUtensorMap& ta, const CUtensorMap& tb, const I8Args& a, long blocks, size_t smem,
               cudaStream_t st) {
  // the shared-memory attribute is per device: set once on each
  static std::atomic<bool> cfg[kMaxDevices];
  const int dev = current_device();
  if (!cfg[dev].load(std::memory_order_acquire)) {
    GG_CUDA(cudaFuncSetAttribute(i8_gemm_kernel<S, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, 232448));
    cfg[dev].store(true, std::memory_order_release);
  }
  i8_gemm_kernel<S, BN><<<(unsigned)blocks, NTHREADS, smem, st>>>(ta, tb, a);
  GG_CHECK_LAUNCH();
}

template <int S>
void launch_slices_s(const OpView& va, const OpView& vb, int rows_a_pad, int ncol_pad, int nkb, const int* ea,
                     const int* eb, int8_t* a8, int8_t* b8, long batch_a, long batch_b, cudaStream_t st) {
  slice_kernel<false, S><<<(unsigned)((long)nkb * ((va.R + 31) / 32) * batch_a), 256, 0, st>>>(va, rows_a_pad, nkb, ea,
                                                                                             a8, batch_a);
  GG_CHECK_LAUNCH();
  slice_kernel<true, S><<<(unsigned)((long)nkb * ((vb.R + 31) / 32) * batch_b), 256, 0, st>>>(vb, ncol_pad, nkb, eb, b8,
                                                                                          batch_b);
  GG_CHECK_LAUNCH();
}

void launch_slices(int S, const OpView& va, const OpView& vb, int rows_a_pad, int ncol_pad, int nkb, const int* ea,
                   const int* eb, int8_t* a8, int8_t* b8, long batch_a, long batch_b, cudaStream_t st) {
  switch (S) {
    case 2: launch_slices_s<2>(va, vb, rows_a_pad, ncol_pad, nkb, ea, eb, a8, b8, batch_a, batch_b, st); break;
    case 3: launch_slices_s<3>(va, vb, rows_a_pad, ncol_pad, nkb, ea, eb, a8, b8, batch_a, batch_b, st); break;
    case 4: launch_slices_s<4>(va, vb, rows_a_pad, ncol_pad, nkb, ea, eb, a8, b8, batch_a, batch_b, st); break;
    case 5: launch_slices_s<5>(va, vb, rows_a_pad, ncol_pad, nkb, ea, eb, a8, b8, batch_a, batch_b, st); break;
    case 6: launch_slices_s<6>(va, vb, rows_a_pad, ncol_pad, nkb, ea, eb, a8, b8, batch_a, batch_b, st); break;
    case 7: launch_slices_s<7>(va, vb, rows_a_pad, ncol_pad, nkb, ea, eb, a8, b8, batch_a, batch_b, st); break;
    default: launch_slices_s<8>(va, vb, rows_a_pad, ncol_pad, nkb, ea, eb, a8, b8, batch_a, batch_b, st); break;
  }
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

void split_arm_timeout_test(SplitGemm* e) { e->timeout_test = true; }

void split_set_autotune(SplitGemm* e, bool on) {
  e->autotune = on;
  if (!on) {
    e->tuned.clear();
    e->report.clear();
  }
}

const char* split_autotune_report(const SplitGemm* e) { return e ? e->report.c_str() : ""; }

void split_buffers(const SplitGemm* e, std::vector<const void*>& out) {
  if (!e) {
    out.push_back(nullptr);
    return;
  }
  out.insert(out.end(), {e->a8.p, e->b8.p, e->ea.p, e->eb.p, e->err.p, e->work.p});
}

namespace {

// tile geometry of a split GEMM with S slices
struct Geometry {
  int BN, nbuf, rows_a_pad, rows_b_pad, ncol_pad, nkb, kcb;
  long batch, Ktot, kp;
  int rows_b_plane;  // height of a B plane (>= rows_b_pad when planes are shared by several widths)
};

// tile widths of the INT8 kernels instantiated for S slices (accumulators of S x BN columns fit TMEM)
std::vector<int> widths(int S) {
  if (S == 5) return {96, 80, 64, 48};
  if (S == 6) return {80, 64};
  if (S <= 4) return {128};
  return {64};
}

Geometry geometry(const ZgemmDesc& d, int S, int force_bn = 0) {
  if (S < 2 || S > 8) throw Error(GG_ERR_ARG, "split: slices must be in [2, 8]");
  Geometry g;
  // nbuf accumulator sets of S diagonals x BN columns must fit the 512 TMEM columns;
  // BN <= 128 keeps the FP64 drain registers (BN / 2 per thread) in budget
  // tile width: the widest one whose accumulators fit TMEM, or a narrower one that pads the
  // 2N rows of B' less (2N = 800: 80 divides it, 96 pads it to 864)
  g.BN = S <= 4 ? 128 : S == 5 ? 96 : S == 6 ? 80 : 64;
  if (S == 5 || S == 6) {
    const int cands[4] = {96, 80, 64, 48};
    long best = -1;
    for (int bn : cands) {
      if (S == 6 && (bn == 96 || bn == 48)) continue;
      const long pad = ((2L * d.N + bn - 1) / bn) * bn;
      if (best < 0 || pad < best) {
        best = pad;
        g.BN = bn;
      }
    }
  }
  g.batch = (long)d.nb0 * d.nb1 * d.nb2;
  g.Ktot = (long)d.KB * d.K;
  if (2 * g.Ktot + KB >= (1L << 31) || (long)d.M >= (1L << 31) || (long)d.N >= (1L << 30))
    throw Error(GG_ERR_ARG, "split: operand dimensions too large for one launch");
  g.kp = ((2 * g.Ktot + KB - 1) / KB) * KB;
  g.rows_a_pad = ((d.M + BM - 1) / BM) * BM;
  if (force_bn) g.BN = force_bn;
  // two accumulator sets when they fit TMEM: the next tile's MMAs then run while the epilogue
  // drains the previous tile (S <= 2, or 48-wide tiles at 5 slices)
  g.nbuf = 2 * S * g.BN <= 512 ? 2 : 1;
  g.rows_b_pad = ((2 * d.N + g.BN - 1) / g.BN) * g.BN;  // B' rows (2 per complex column), whole tiles
  g.ncol_pad = g.rows_b_pad / 2;                        // complex columns incl. padding
  g.rows_b_plane = g.rows_b_pad;
  // exact int32 chunk: S * Kchunk * 64^2 < 2^31 (slices are rounded, |d| <= 64)
  const long kchunk = std::max<long>(KB, ((2147483647L / (4096L * S)) / KB) * KB);
  g.kcb = (int)(kchunk / KB);
  g.nkb = (int)(g.kp / KB);
  return g;
}

// the persistent INT8 GEMM on operand planes (a8 / b8 of batch_a / batch_b batches)
int run_planes(SplitGemm* e, const ZgemmDesc& d, int S, const Geometry& g, const int8_t* a8, const int8_t* b8,
               const int* ea, const int* eb, bool a_shared, bool b_shared, cudaStream_t st,
               const SplitRowMax* mx = nullptr, int force_splits = 0) {
  int* err = e->err.p;
  if (!err) {
    err = e->err.ensure(1);
    GG_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
  }
  const long batch_a = a_shared ? 1 : g.batch, batch_b = b_shared ? 1 : g.batch;
  const CUtensorMap ta = make_map(a8, d.M, g.rows_a_pad, batch_a * S * g.nkb, BM);
  const CUtensorMap tb = make_map(b8, 2L * d.N, g.rows_b_plane, batch_b * S * g.nkb, g.BN);

  I8Args a{};
  a.S = S;
  a.rows_a_pad = g.rows_a_pad;
  a.rows_b_pad = g.rows_b_pad;
  a.nkb = g.nkb;
  a.kcb = g.kcb;
  a.M = d.M;
  a.N = d.N;
  a.tiles_m = g.rows_a_pad / BM;
  a.tiles_n = g.rows_b_pad / g.BN;
  a.nb0 = d.nb0;
  a.nb1 = d.nb1;
  a.batch = g.batch;
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
  if (mx) a.mx = *mx;
  a.wait_cycles = WAIT_CYCLES;
  a.skip_arrive = 0;
  if (e->timeout_test) {
    // ~0.1 s limit, and CTA 0 withholds one accumulator release (its MMA warp waits for it in
    // its second work unit: the launch needs more units than CTAs)
    a.wait_cycles = 200000000LL;
    a.skip_arrive = 1;
    e->timeout_test = false;
  }
  a.nbuf = g.nbuf;
  a.a_shared = a_shared ? 1 : 0;
  a.b_shared = b_shared ? 1 : 0;
  a.tmem_cols = 32;
  while (a.tmem_cols < g.nbuf * S * g.BN) a.tmem_cols *= 2;
  const size_t stage_bytes = (size_t)S * (BM + g.BN) * KB;
  a.stages = (int)std::min<size_t>(4, (220 * 1024 - 2048) / stage_bytes);
  if (a.stages < 2) throw Error(GG_ERR_ARG, "split: stage does not fit shared memory");
  const size_t smem = a.stages * stage_bytes + 1024 + 512;  // + alignment + barriers and TMEM slot
  const long base = (long)a.tiles_m * a.tiles_n * g.batch;
  // split-K so that the units fill whole waves of persistent CTAs (each split keeps >= 8 K
  // blocks); the row-max epilogue needs whole reductions (no split-K)
  int splits = 1;
  if (force_splits > 0) {
    splits = a.mx.on ? 1 : force_splits;
  } else if (!a.mx.on) {
    const int smax = (int)std::max<long>(1, std::min<long>(g.nkb / 8, 64));
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
  const long need = (long)d.M * d.N * g.batch;
  if (splits > 1) {
    e->work.ensure((size_t)splits * need);
  }
  a.splits = splits;
  // pairs (d, d+1), d = 2, 4, ...: |acc_d| <= (d - 1) Kc 64^2 for a segment of Kc bytes, so the
  // combined value 128 acc_d + acc_{d+1} stays below 2^31 when (128 (d-1) + d) Kc 4096 < 2^31
  // for the largest paired d (the even d <= S)
  {
    const long seg = std::min<long>(g.kcb, (g.nkb + splits - 1) / splits) * KB;
    const long dmax = (S / 2) * 2;
    a.pair = (128 * (dmax - 1) + dmax) * seg * 4096L < (1L << 31) ? 1 : 0;
  }
  a.work = e->work.p;
  a.units = base * splits;
  if (a.units >= (1L << 31) || (long)splits * g.nkb >= (1L << 31))
    throw Error(GG_ERR_ARG, "split: too many work units for one launch");
  const long grid = std::min<long>(a.units, sms());
  switch (S * 1000 + g.BN) {  // the (S, BN) pairs geometry() chooses
    case 2128: launch_i8<2, 128>(ta, tb, a, grid, smem, st); break;
    case 3128: launch_i8<3, 128>(ta, tb, a, grid, smem, st); break;
    case 4128: launch_i8<4, 128>(ta, tb, a, grid, smem, st); break;
    case 5096: launch_i8<5, 96>(ta, tb, a, grid, smem, st); break;
    case 5080: launch_i8<5, 80>(ta, tb, a, grid, smem, st); break;
    case 5064: launch_i8<5, 64>(ta, tb, a, grid, smem, st); break;
    case 5048: launch_i8<5, 48>(ta, tb, a, grid, smem, st); break;
    case 6080: launch_i8<6, 80>(ta, tb, a, grid, smem, st); break;
    case 6064: launch_i8<6, 64>(ta, tb, a, grid, smem, st); break;
    case 7064: launch_i8<7, 64>(ta, tb, a, grid, smem, st); break;
    case 8064: launch_i8<8, 64>(ta, tb, a, grid, smem, st); break;
    default: throw Error(GG_ERR_INTERNAL, "split: no kernel for this slice count and tile width");
  }
  int launches = 1;
  if (splits > 1) {
    const long total = need;
    const long nblk = std::min<long>((total + 255) / 256, 65535L * 8);
    split_reduce_kernel<<<(unsigned)nblk, 256, 0, st>>>(e->work.p, splits, g.batch, d.M, d.N, d.C, d.c_m, d.c_n,
                                                       d.nb0, d.nb1, d.c_b0, d.c_b1, d.c_b2, d.alpha, d.beta);
    GG_CHECK_LAUNCH();
    ++launches;
  }
  return launches;
}

// exponents and slices of both operands into the engine's planes, then the GEMM
int sliced_gemm(SplitGemm* e, const ZgemmDesc& d, int S, cudaStream_t st, const SplitRowMax* mx = nullptr,
                const int* ea_given = nullptr, const int* eb_given = nullptr) {
  if (d.M <= 0 || d.N <= 0) return 0;
  Geometry g = geometry(d, S);
  // an operand with zero batch strides is the same matrix for every batch: slice it once
  const bool a_shared = g.batch > 1 && d.a_b0 == 0 && d.a_b1 == 0 && d.a_b2 == 0;
  const bool b_shared = g.batch > 1 && d.b_b0 == 0 && d.b_b1 == 0 && d.b_b2 == 0;
  const long batch_a = a_shared ? 1 : g.batch, batch_b = b_shared ? 1 : g.batch;
  // autotuner: a shape seen before runs with its measured best (tile width, split-K); a new
  // shape is timed for every candidate when this call may run more than once (it overwrites C,
  // beta = 0) and is not being captured into a graph
  const std::array<long, 8> key{S, d.M, d.N, g.Ktot, g.batch, (a_shared ? 1 : 0) + (b_shared ? 2 : 0),
                                mx ? 1 : 0, g.nkb};
  int force_splits = 0;
  bool tune = false;
  std::vector<int> cand_bn;
  if (e->autotune) {
    auto it = e->tuned.find(key);
    if (it != e->tuned.end()) {
      g = geometry(d, S, it->second.BN);
      force_splits = it->second.splits;
    } else {
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      GG_CUDA(cudaStreamIsCapturing(st, &cs));
      tune = cs == cudaStreamCaptureStatusNone && d.beta.x == 0.0 && d.beta.y == 0.0;
      if (tune) {
        cand_bn = widths(S);
        for (int bn : cand_bn) g.rows_b_plane = std::max(g.rows_b_plane, geometry(d, S, bn).rows_b_pad);
        g.ncol_pad = g.rows_b_plane / 2;  // slice B once, tall enough for every candidate width
      }
    }
  }
  int8_t* a8 = e->a8.ensure((size_t)batch_a * S * g.rows_a_pad * g.kp);
  int8_t* b8 = e->b8.ensure((size_t)batch_b * S * g.rows_b_plane * g.kp);
  int* ea = e->ea.ensure((size_t)batch_a * g.rows_a_pad);
  int* eb = e->eb.ensure((size_t)batch_b * d.N);
  OpView va{d.A, d.a_m, d.a_kb, d.a_k, d.KB, d.K, d.M, d.nb0, d.nb1, d.a_b0, d.a_b1, d.a_b2, d.conjA};
  OpView vb{d.B, d.b_n, d.b_kb, d.b_k, d.KB, d.K, d.N, d.nb0, d.nb1, d.b_b0, d.b_b1, d.b_b2, d.conjB};
  auto exponents = [&](const OpView& v, int rows_pad, int* out, long nb) {
    const bool rcontig = v.rmap.lo == 1 && v.ks != 1;
    const long n = nb * rows_pad;
    if (rcontig)
      row_exponent_rc_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(v, rows_pad, out, nb);
    else
      row_exponent_kernel<<<(unsigned)((n * 32 + 255) / 256), 256, 0, st>>>(v, rows_pad, out, nb);
    GG_CHECK_LAUNCH();
  };
  int launches = 2;
  if ((ea_given && a_shared) || (eb_given && b_shared))
    throw Error(GG_ERR_ARG, "split: given exponents need per-batch operands");
  if (ea_given) {
    ea = const_cast<int*>(ea_given);
  } else {
    exponents(va, g.rows_a_pad, ea, batch_a);
    ++launches;
  }
  if (eb_given) {
    eb = const_cast<int*>(eb_given);
  } else {
    exponents(vb, d.N, eb, batch_b);
    ++launches;
  }
  launch_slices(S, va, vb, g.rows_a_pad, g.ncol_pad, g.nkb, ea, eb, a8, b8, batch_a, batch_b, st);
  if (!tune) return launches + run_planes(e, d, S, g, a8, b8, ea, eb, a_shared, b_shared, st, mx, force_splits);
  // time every (width, split-K) candidate on the sliced planes; the rule's split-K factor, one
  // and twice the rule's bracket the split-K choice
  cudaEvent_t t0, t1;
  GG_CUDA(cudaEventCreate(&t0));
  GG_CUDA(cudaEventCreate(&t1));
  SplitGemm::Choice best{g.BN, 0, 1e30};
  for (int bn : cand_bn) {
    Geometry gc = geometry(d, S, bn);
    gc.rows_b_plane = g.rows_b_plane;
    gc.ncol_pad = g.ncol_pad;
    const long base = (long)(gc.rows_a_pad / BM) * (gc.rows_b_pad / bn) * gc.batch;
    int rule = 1;
    {
      const int smax = (int)std::max<long>(1, std::min<long>(gc.nkb / 8, 64));
      double b = 0.0;
      for (int sp = 1; sp <= smax; ++sp) {
        const long units = base * sp, waves = (units + sms() - 1) / sms();
        const double eff = (double)units / (double)(waves * sms());
        if (eff > b + 0.05) {
          b = eff;
          rule = sp;
        }
        if (units >= 4L * sms()) break;
      }
    }
    const int smax = mx ? 1 : (int)std::max<long>(1, std::min<long>(gc.nkb / 8, 64));
    std::vector<int> sps{rule, 1, std::min(2 * rule, smax)};
    std::sort(sps.begin(), sps.end());
    sps.erase(std::unique(sps.begin(), sps.end()), sps.end());
    for (int sp : sps) {
      if (mx && sp != 1) continue;
      // one untimed run first: the first launch of a kernel loads its module and starts from a
      // cold L2, which would bias the choice against the first candidate
      launches += run_planes(e, d, S, gc, a8, b8, ea, eb, a_shared, b_shared, st, mx, sp);
      GG_CUDA(cudaEventRecord(t0, st));
      launches += run_planes(e, d, S, gc, a8, b8, ea, eb, a_shared, b_shared, st, mx, sp);
      GG_CUDA(cudaEventRecord(t1, st));
      GG_CUDA(cudaEventSynchronize(t1));
      float ms = 0.f;
      GG_CUDA(cudaEventElapsedTime(&ms, t0, t1));
      if (ms < best.ms) best = {bn, sp, ms};
    }
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  e->tuned[key] = best;
  char line[200];
  std::snprintf(line, sizeof(line), "S %ld M %ld N %ld K %ld batch %ld: BN %d split-K %d (%.3f ms)\n", key[0], key[1],
                key[2], key[3], key[4], best.BN, best.splits, best.ms);
  e->report += line;
  // the result of this call comes from the chosen configuration, as every later call's will
  Geometry gb = geometry(d, S, best.BN);
  gb.rows_b_plane = g.rows_b_plane;
  gb.ncol_pad = g.ncol_pad;
  return launches + run_planes(e, d, S, gb, a8, b8, ea, eb, a_shared, b_shared, st, mx, best.splits);
}

}  // namespace

SplitPlanes split_planes_for(const ZgemmDesc& d, int S) {
  const Geometry g = geometry(d, S);
  SplitPlanes p;
  p.rows_a_pad = g.rows_a_pad;
  p.rows_b_pad = g.rows_b_pad;
  p.ncol_pad = g.ncol_pad;
  p.nkb = g.nkb;
  p.batch = g.batch;
  p.a_bytes = (size_t)g.batch * S * g.rows_a_pad * g.kp;
  p.b_bytes = (size_t)g.batch * S * g.rows_b_pad * g.kp;
  return p;
}

int split_zgemm(SplitGemm* e, const ZgemmDesc& d, int S, cudaStream_t st) { return sliced_gemm(e, d, S, st); }

int split_zgemm_rowmax(SplitGemm* e, const ZgemmDesc& d, int S, const SplitRowMax& mx, cudaStream_t st) {
  if (!mx.on || !mx.ex || mx.div_m < 1 || mx.div_n < 1)
    throw Error(GG_ERR_ARG, "split row max: incomplete target description");
  if (d.alpha.x != 1.0 || d.alpha.y != 0.0 || d.beta.x != 0.0 || d.beta.y != 0.0)
    throw Error(GG_ERR_ARG, "split row max: alpha must be 1 and beta 0");
  return sliced_gemm(e, d, S, st, &mx);
}

int split_zgemm_exps(SplitGemm* e, const ZgemmDesc& d, int S, const int* ea, const int* eb, cudaStream_t st,
                     const SplitRowMax* mx) {
  if (mx && (d.alpha.x != 1.0 || d.alpha.y != 0.0 || d.beta.x != 0.0 || d.beta.y != 0.0))
    throw Error(GG_ERR_ARG, "split row max: alpha must be 1 and beta 0");
  return sliced_gemm(e, d, S, st, mx, ea, eb);
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
