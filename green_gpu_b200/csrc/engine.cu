// Host orchestration of the GW self-energy build and the HF exchange on one B200.
//
// Phase-major design: every phase of an iteration runs as a few large launches over
// all (q, k, tau) it owns, with all state resident in HBM (the reference instead
// round-trips each (q,k) pair through the host: src/cugw_utils.cu:104-202).
//
//   unfold   G(k_ibz, tau) -> G(k_full, tau) for all k        (cu_symmetry.cu:183-233)
//   P0       P0_q(tau) = pref/nk sum_k A_k(tau) B_k(tau)^T     (cugw_qkpt.cu:203-234,
//            with A = G^k(beta-tau) V, B = conj(V) G^{k+q}(tau)^T, K index = (k, a, b))
//   IR fwd   P~_q(iW) = Tnt_BF P0_q(tau), mirror folded in      (cugw_qpt.cu:179-191, 329-339)
//   Dyson    W~ = (I - P~)^{-1} P~ per (q, W), FP64             (cugw_qpt.cu:223-322)
//   IR back  W~_q(tau) = Ttn_FB W~_q(iW)                        (cugw_qpt.cu:341-358)
//   Sigma    Sigma_k(tau) -= sum_q' ((V W~_q') G(k-q')) V^+     (cugw_qkpt.cu:248-338,
//            cugw_utils.cu:240-269; the reference forms V G first, here V W~ is formed
//            first so that V is the tau- and spin-independent operand of the main GEMM)
#include "engine.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "kernels.cuh"
#include "sigma_tail.cuh"
#include "split.cuh"
#include "zgemm.cuh"

namespace gg {
namespace {

inline int64_t tri(long k1, long k2) { return k1 >= k2 ? k1 * (k1 + 1) / 2 + k2 : k2 * (k2 + 1) / 2 + k1; }

struct EventTimer {
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> marks;
  cudaStream_t st;
  bool on;
  explicit EventTimer(cudaStream_t s, bool enabled = true) : st(s), on(enabled) {}
  int begin(int id) {
    if (!on) return -1;
    cudaEvent_t a, b;
    GG_CUDA(cudaEventCreate(&a));
    GG_CUDA(cudaEventCreate(&b));
    GG_CUDA(cudaEventRecord(a, st));
    marks.push_back({id, {a, b}});
    return (int)marks.size() - 1;
  }
  void end(int h) {
    if (h >= 0) GG_CUDA(cudaEventRecord(marks[h].second.second, st));
  }
  void collect(double* acc) {
    for (auto& m : marks) {
      float ms = 0;
      GG_CUDA(cudaEventElapsedTime(&ms, m.second.first, m.second.second));
      acc[m.first] += ms * 1e-3;
    }
  }
  ~EventTimer() {
    for (auto& m : marks) {
      cudaEventDestroy(m.second.first);
      cudaEventDestroy(m.second.second);
    }
  }
};

// (pos, op) of every pair in a list, uploaded once; gathers index into it by offset
struct PairTable {
  DevBuf<int64_t> pos;
  DevBuf<int> op;
  void build(const gg_context* c, const std::vector<int>& k1, const std::vector<int>& k2) {
    const size_t np = k1.size();
    std::vector<int64_t> p(np);
    std::vector<int> o(np);
    for (size_t i = 0; i < np; ++i) kpair_op(c, k1[i], k2[i], &p[i], &o[i]);
    pos.ensure(std::max<size_t>(np, 1));
    op.ensure(std::max<size_t>(np, 1));
    if (np) {
      GG_CUDA(cudaMemcpy(pos.p, p.data(), np * sizeof(int64_t), cudaMemcpyHostToDevice));
      GG_CUDA(cudaMemcpy(op.p, o.data(), np * sizeof(int), cudaMemcpyHostToDevice));
    }
  }
  void gather(const gg_context* c, size_t first, int count, double2* dst, cudaStream_t st) const {
    launch_gather_pairs(c->V, pos.p + first, op.p + first, count, c->sh.NQ, c->sh.nao, dst, st);
  }
};

struct IntTable {
  DevBuf<int> d;
  void build(const std::vector<int>& h) {
    d.ensure(std::max<size_t>(h.size(), 1));
    if (!h.empty()) GG_CUDA(cudaMemcpy(d.p, h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice));
  }
};

// tables of one GW build, kept in the context between builds
struct GwTables {
  PairTable p0_pairs, sg_pairs;
  IntTable g1_idx;
};

size_t free_bytes() {
  size_t fr = 0, tot = 0;
  GG_CUDA(cudaMemGetInfo(&fr, &tot));
  return fr;
}

}  // namespace

// V(k1,k2) location in the store: position and op (bit0 conj, bit1 transpose), following
// df_integral_t::symmetrize (df_integral_t.h:153-235): conj-transpose when k1 < k2, then
// conj or transpose from the k-pair symmetry lists.
void kpair_op(const gg_context* c, int k1, int k2, int64_t* pos, int* op) {
  if (k1 < 0 || k2 < 0 || k1 >= c->sh.nk || k2 >= c->sh.nk) throw Error(GG_ERR_ARG, "k index out of range");
  int64_t idx = tri(k1, k2);
  int cj = k1 < k2, tr = k1 < k2;
  if (c->conj_list[idx] != idx) {
    idx = c->conj_list[idx];
    cj ^= 1;
  } else if (c->trans_list[idx] != idx) {
    idx = c->trans_list[idx];
    tr ^= 1;
  }
  const int64_t p = (idx >= 0 && idx < (int64_t)c->irre_pos.size()) ? c->irre_pos[idx] : -1;
  if (p < 0 || p >= c->nstored)
    throw Error(GG_ERR_ARG, "k-pair (" + std::to_string(k1) + "," + std::to_string(k2) +
                                ") maps to a pair that is not stored");
  *pos = p;
  *op = cj | (tr << 1);
}

// X_full[k][s][m] = U_k X_ibz[m][s][f2r[k]] U_k^+ (conj for TR), X_in layout [nouter][ns][ink][n][n]
void unfold_matrices(gg_context* c, const double2* X_in, int nouter, int ns, double2* out, cudaStream_t st) {
  const int nk = c->sh.nk, ink = c->sh.ink, n = c->sh.nao;
  const long nn = (long)n * n;
  launch_gather_g(X_in, c->k_f2r_d.p, nk, ns, nouter, ink, n, out, st);
  ++c->launches;
  if (c->has_Uk) {
    double2* tmp = c->Gtmp.ensure((size_t)nk * ns * nouter * nn);
    ZgemmDesc d;
    d.M = n; d.N = n; d.K = n;
    d.A = c->Uk.p; d.a_m.lo = n; d.a_k = 1;
    d.B = out; d.b_k = n; d.b_n.lo = 1;
    d.C = tmp; d.c_m.lo = n; d.c_n.lo = 1;
    d.nb0 = ns * nouter; d.nb1 = nk;
    d.a_b0 = 0; d.a_b1 = nn;
    d.b_b0 = nn; d.b_b1 = (long)ns * nouter * nn;
    d.c_b0 = nn; d.c_b1 = (long)ns * nouter * nn;
    c->launches += zgemm(d, st);
    ZgemmDesc e = d;
    e.A = tmp; e.a_m.lo = n; e.a_k = 1; e.a_b0 = nn; e.a_b1 = (long)ns * nouter * nn;
    e.B = c->Uk.p; e.b_k = 1; e.b_n.lo = n; e.conjB = 1; e.b_b0 = 0; e.b_b1 = nn;
    e.C = out;
    c->launches += zgemm(e, st);
  }
  launch_conj_where(out, c->k_tr_d.p, nk, (long)ns * nouter * nn, st);
  ++c->launches;
}

std::vector<int> shard_q_points(int inq, int rank, int size) {
  if (size < 1 || rank < 0 || rank >= size || inq < 0) throw Error(GG_ERR_ARG, "q shard: need 0 <= rank < size");
  std::vector<int> q;
  for (int iq = rank; iq < inq; iq += size) q.push_back(iq);
  return q;
}

int gw_spins(const gg_context* c) { return c->x2c ? 4 : c->sh.ns; }
int hf_spins(const gg_context* c) { return c->x2c ? 3 : c->sh.ns; }

void x2c_check(const gg_context* c) {
  if (!c->x2c) return;
  bool tr = false;
  for (auto v : c->k_tr) tr = tr || v != 0;
  for (auto v : c->q_tr) tr = tr || v != 0;
  if (c->has_Uk || c->has_Uq || tr)
    throw Error(GG_ERR_ARG, "x2c: only the identity k/q symmetry is supported (no U_k / U_q rotations or "
                            "time-reversal partners)");
}

Plan plan_gw(gg_context* c, int slices) {
  const auto& s = c->sh;
  const int nspin = gw_spins(c);
  const size_t z = sizeof(double2);
  const size_t nn = (size_t)s.nao * s.nao, NN = (size_t)s.NQ * s.NQ, Nnn = (size_t)s.NQ * nn;
  const int T2 = s.nts / 2;
  const size_t held = c->Gf.n + c->Gtmp.n + c->Vbuf.n + c->G1buf.n + c->scratchA.n + c->scratchB.n + c->P0buf.n +
                      c->Pw.n + c->Afac.n + c->Wt.n + c->Wrot.n + c->gemm_work.n;
  const size_t budget = (size_t)(0.85 * (double)(free_bytes() + held * z));
  Plan p;
  p.dyson_batch = 4 * 148;
  auto need = [&](const Plan& q) {
    size_t b = 0;
    b += 2 * (size_t)s.nk * nspin * s.nts * nn;       // Gf + Gtmp
    b += (size_t)q.kc * Nnn;                           // Vbuf
    b += (size_t)q.kc * T2 * nn;                       // G1buf
    size_t p0s = (size_t)q.kc * q.tb * Nnn;            // A / B build buffers (each)
    size_t sgs = (size_t)s.nts * std::max(Nnn, NN);    // Sigma X / Z, W rotation (each)
    b += 2 * std::max(p0s, sgs);
    b += (size_t)q.qc * T2 * NN;                       // P0
    b += (size_t)q.qc * s.nw_b * NN;                   // Pw
    b += (size_t)std::min<long>(q.dyson_batch, (long)q.qc * s.nw_b) * NN;  // Dyson workspace
    b += (size_t)q.qc * s.nts * NN;                    // Wt
    b += (size_t)s.nts * NN;                           // Wrot
    b += (size_t)1 << 22;                              // split-K partials
    b *= z;
    if (slices > 0) {
      // int8 slices of the P0 contraction operands (rows padded to the tile sizes), K = 2 nn kc bytes
      b += (size_t)q.tb * slices * (size_t)(3 * s.NQ + 320) * 2 * nn * q.kc;
    }
    return b;
  };
  p.qc = s.inq;
  p.kc = s.nk;
  // tau block of the P0 operand builds: rows (tt, a) of tb * nao, chosen to waste the least
  // of the 64-row GEMM tiles over all tau blocks (largest such tb up to 12)
  {
    long best = -1;
    p.tb = 1;
    for (int tb = 1; tb <= std::min(T2, 12); ++tb) {
      long padded = 0;
      for (int t0 = 0; t0 < T2; t0 += tb) padded += 64L * ((std::min(tb, T2 - t0) * (long)s.nao + 63) / 64);
      if (best < 0 || padded <= best) {
        best = padded;
        p.tb = tb;
      }
    }
  }
  while (need(p) > budget) {
    if (p.qc > 1) p.qc = (p.qc + 1) / 2;
    else if (p.tb > 1) p.tb = (p.tb + 1) / 2;
    else if (p.kc > 1) p.kc = (p.kc + 1) / 2;
    else
      throw Error(GG_ERR_MEMORY, "GW build does not fit the device: need " + std::to_string(need(p) >> 20) +
                                     " MiB of work space, budget " + std::to_string(budget >> 20) + " MiB");
  }
  p.bytes = need(p);
  return p;
}

// system index = position of q in this shard's list x nw_b + Omega
void dyson_failure(const gg_context* c, int solver, int system, int info) {
  const auto& s = c->sh;
  const int nw = s.nw_b;
  const int iq = c->shard_rank + (system / nw) * c->shard_size;
  throw Error(solver == GG_SOLVER_CHOLESKY ? GG_ERR_NOT_HPD : GG_ERR_SINGULAR,
              std::string(solver == GG_SOLVER_CHOLESKY ? "Cholesky" : "LU") + " failed for q_ibz " +
                  std::to_string(iq) + ", frequency " + std::to_string(system % nw) + " (info " +
                  std::to_string(info) + "): I - P~ is not " +
                  (solver == GG_SOLVER_CHOLESKY ? "positive definite" : "invertible"));
}

namespace {

// C^T = B^T A^T as a descriptor: the INT8 engine's epilogue gives each lane one row of C, so
// the operand builds (outputs contiguous along n) are computed transposed for coalesced stores
ZgemmDesc transposed(const ZgemmDesc& d) {
  ZgemmDesc t = d;
  t.M = d.N; t.N = d.M;
  t.A = d.B; t.a_m = d.b_n; t.a_k = d.b_k; t.a_kb = d.b_kb; t.conjA = d.conjB;
  t.a_b0 = d.b_b0; t.a_b1 = d.b_b1; t.a_b2 = d.b_b2;
  t.B = d.A; t.b_n = d.a_m; t.b_k = d.a_k; t.b_kb = d.a_kb; t.conjB = d.conjA;
  t.b_b0 = d.a_b0; t.b_b1 = d.a_b1; t.b_b2 = d.a_b2;
  t.c_m = d.c_n; t.c_n = d.c_m;
  return t;
}

// P0 of one k chunk (kn points from k0) and one spin in split precision.  The operand builds
// (INT8 engine, FP64 output SA / SB as in the FP64 path) also record the exact maximum of every
// row of SA and every column of SB that the main contraction slices with (a segmented warp
// reduction and one atomicMax per row segment in their epilogue), so the two exponent scans over
// SA and SB - a full read of both - are not needed; the slicing pass uses those exponents.
template <typename Main>
void p0_split_block(gg_context* c, SplitGemm* split, const double2* Gf, const double2* G1, const double2* Vb,
                    double2* SA, double2* SB, double2* P0q, int k0, int kn, int spa, const Plan& pl, double pref,
                    bool first, cudaStream_t st, Main&& main) {
  const auto& s = c->sh;
  const int n = s.nao, N = s.NQ, T = s.nts, T2 = T / 2, S = c->slices, ns = gw_spins(c);
  const long nn = (long)n * n, Nnn = (long)N * nn, NN = (long)N * N;
  for (int t0 = 0; t0 < T2; t0 += pl.tb) {
    const int tn = std::min(pl.tb, T2 - t0);
    // P0[t] (+)= pref/nk sum_kk sum_x SA[kk][tt][Q'][x] SB[kk][tt][Q][x]
    ZgemmDesc dm;
    dm.M = N; dm.N = N; dm.K = (int)nn; dm.KB = kn;
    dm.A = SA; dm.a_m.lo = nn; dm.a_k = 1; dm.a_kb = (long)tn * Nnn;
    dm.B = SB; dm.b_k = 1; dm.b_n.lo = nn; dm.b_kb = (long)tn * Nnn;
    dm.C = P0q + (long)t0 * NN; dm.c_m.lo = N; dm.c_n.lo = 1;
    dm.nb0 = tn; dm.a_b0 = Nnn; dm.b_b0 = Nnn; dm.c_b0 = NN;
    dm.alpha = make_double2(pref / s.nk, 0.0);
    dm.beta = first ? make_double2(0.0, 0.0) : make_double2(1.0, 0.0);
    const SplitPlanes g = split_planes_for(dm, S);
    int* ea = c->p0_ea.ensure((size_t)pl.tb * g.rows_a_pad);
    int* eb = c->p0_eb.ensure((size_t)pl.tb * N);
    // every exponent starts below any value's (bytes 0x80: -2139062144)
    GG_CUDA(cudaMemsetAsync(ea, 0x80, sizeof(int) * (size_t)tn * g.rows_a_pad, st));
    GG_CUDA(cudaMemsetAsync(eb, 0x80, sizeof(int) * (size_t)tn * N, st));
    // A-build SA[kk][tt][Q'][a][b] = sum_p G^k(tau_{T-1-t})[a][p] V[kk][Q'][p][b], computed
    // transposed: rows m = (Q', b), columns n = (tt, a); main A row Q' of batch tt
    {
      ZgemmDesc d;
      d.M = tn * n; d.N = N * n; d.K = n;
      d.A = Gf + ((long)k0 * ns + spa) * T * nn + (long)(T - 1 - t0) * nn;
      d.a_m.split = n; d.a_m.hi = -nn; d.a_m.lo = n; d.a_k = 1;
      d.B = Vb; d.b_k = n; d.b_n.split = n; d.b_n.hi = nn; d.b_n.lo = 1;
      d.C = SA; d.c_m.split = n; d.c_m.hi = Nnn; d.c_m.lo = n;
      d.c_n.split = n; d.c_n.hi = nn; d.c_n.lo = 1;
      d.nb0 = kn;
      d.a_b0 = (long)ns * T * nn; d.b_b0 = Nnn; d.c_b0 = (long)tn * Nnn;
      SplitRowMax mx;  // row Q' = mq of batch tt = nq: ea[tt rows_a_pad + Q']
      mx.on = 1; mx.div_m = n; mx.div_n = n; mx.s_mq = 1; mx.s_nq = g.rows_a_pad; mx.ex = ea;
      c->launches += split_zgemm_rowmax(split, transposed(d), S, mx, st);
    }
    // B-build SB[kk][tt][Q][a][b] = sum_l conj(V[kk][Q][a][l]) G^{k+q}(tau_t)[b][l], computed
    // transposed: rows m = (tt, b), columns n = (Q, a); main B column Q of batch tt
    {
      ZgemmDesc d;
      d.M = N * n; d.N = tn * n; d.K = n;
      d.A = Vb; d.a_m.lo = n; d.a_k = 1; d.conjA = 1;
      d.B = G1 + (long)t0 * nn; d.b_k = 1; d.b_n.split = n; d.b_n.hi = nn; d.b_n.lo = n;
      d.C = SB; d.c_m.lo = n; d.c_n.split = n; d.c_n.hi = Nnn; d.c_n.lo = 1;
      d.nb0 = kn;
      d.a_b0 = Nnn; d.b_b0 = (long)T2 * nn; d.c_b0 = (long)tn * Nnn;
      SplitRowMax mx;  // column Q = nq of batch tt = mq: eb[tt N + Q]
      mx.on = 1; mx.div_m = n; mx.div_n = n; mx.s_mq = N; mx.s_nq = 1; mx.ex = eb;
      c->launches += split_zgemm_rowmax(split, transposed(d), S, mx, st);
    }
    main(dm, ea, eb);
  }
}

}  // namespace

void gw_build(gg_context* c, const double2* G_dev, double2* Sigma_dev, int solver, int precision, cudaStream_t st) {
  if (!c->has_sym || !c->has_kpairs || !c->V || !c->has_ir || c->sh.nw_b <= 0)
    throw Error(GG_ERR_STATE, "gw: symmetry, k-pairs, integrals and IR transforms (nw_b > 0) must be set first");
  if (precision != GG_PREC_FP64 && precision != GG_PREC_SPLIT) throw Error(GG_ERR_ARG, "gw: unknown precision");
  if (solver != GG_SOLVER_CHOLESKY && solver != GG_SOLVER_LU) throw Error(GG_ERR_ARG, "gw: unknown solver");
  const auto& s = c->sh;
  x2c_check(c);
  const int n = s.nao, N = s.NQ, T = s.nts, T2 = T / 2, nw = s.nw_b, nk = s.nk, ns = gw_spins(c);
  const long nn = (long)n * n, NN = (long)N * N, Nnn = (long)N * nn;
  // G^k(beta - tau) of pseudo-spin sp in the P0 operand build: the X2C pseudo-spins pair the
  // (s1, s2) block of G^{k+q}(tau) with the (s2, s1) block of G^k(-tau), i.e. ab with ba
  // (copy_Gk_2c with minus_t = true, gw_gpu_kernel.cpp:523-536)
  auto spin_a = [&](int sp) { return (c->x2c && sp >= 2) ? 5 - sp : sp; };
  const bool cap = c->capturing;
  Plan pl;
  if (cap) {
    // the captured build replays the eager build's chunking, so every buffer already exists
    pl.qc = c->plan_qc;
    pl.kc = c->plan_kc;
    pl.tb = c->plan_tb;
    pl.dyson_batch = 4 * 148;
  } else {
    pl = plan_gw(c, precision == GG_PREC_SPLIT ? c->slices : 0);
    c->plan_qc = pl.qc;
    c->plan_kc = pl.kc;
    c->plan_tb = pl.tb;
  }
  if (cap && c->profiling) throw Error(GG_ERR_STATE, "gw: profiling is not available while capturing");
  if (cap && (c->cap_P0 || c->cap_Pw || c->cap_Wt)) throw Error(GG_ERR_STATE, "gw: capture of intermediates needs an eager build");
  c->launches = 0;

  // work buffers (sized before the first launch)
  double2* Gf = c->Gf.ensure((size_t)nk * ns * T * nn);
  c->Gtmp.ensure((size_t)nk * ns * T * nn);
  double2* Vb = c->Vbuf.ensure((size_t)pl.kc * Nnn);
  double2* G1 = c->G1buf.ensure((size_t)pl.kc * T2 * nn);
  const size_t scr = std::max((size_t)pl.kc * pl.tb * Nnn, (size_t)T * std::max(Nnn, NN));
  double2* SA = c->scratchA.ensure(scr);
  double2* SB = c->scratchB.ensure(scr);
  double2* P0 = c->P0buf.ensure((size_t)pl.qc * T2 * NN);
  double2* Pw = c->Pw.ensure((size_t)pl.qc * nw * NN);
  const int dys = (int)std::min<long>(pl.dyson_batch, (long)pl.qc * nw);
  double2* Af = c->Afac.ensure((size_t)dys * NN);
  double2* Wt = c->Wt.ensure((size_t)pl.qc * T * NN);
  double2* Wr = c->Wrot.ensure((size_t)T * NN);
  double2* gw_work = c->gemm_work.ensure((size_t)1 << 22);
  int* info = c->info.ensure((size_t)pl.qc * nw);
  int* piv = solver == GG_SOLVER_LU ? c->piv.ensure((size_t)dys * N) : nullptr;
  std::vector<int> info_h((size_t)pl.qc * nw);
  SplitGemm* split = nullptr;
  if (precision == GG_PREC_SPLIT) split = split_engine(c);

  // FP64 contractions of a split-precision build use the three-product complex form
  // (error ~1e-16 relative, far inside that build's budget)
  auto gemm = [&](ZgemmDesc d) {
    d.work = gw_work;
    d.work_elems = (long)c->gemm_work.n;
    d.gauss = split ? 1 : 0;
    c->launches += zgemm(d, st);
  };
  // the dominant contractions go through the split-precision engine when requested;
  // with profiling on, CUDA events bracket every such launch on `st`
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> kev;
  for (int i = 0; i < 3; ++i) {
    c->kstat_launches[i] = 0;
    c->kstat_seconds[i] = 0.0;
    c->kstat_flops[i] = 0.0;
  }
  struct Exps {
    const int* ea;
    const int* eb;
  };
  auto gemm_main = [&](ZgemmDesc d, int which, bool allow_split = true, const Exps* pr = nullptr,
                       const SplitRowMax* mx = nullptr) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (c->profiling) {
      GG_CUDA(cudaEventCreate(&e0));
      GG_CUDA(cudaEventCreate(&e1));
      GG_CUDA(cudaEventRecord(e0, st));
    }
    if (split && pr) {
      d.work = gw_work;
      d.work_elems = (long)c->gemm_work.n;
      c->launches += split_zgemm_exps(split, d, c->slices, pr->ea, pr->eb, st, mx);
    } else if (split && allow_split) {
      d.work = gw_work;
      d.work_elems = (long)c->gemm_work.n;
      c->launches += mx ? split_zgemm_rowmax(split, d, c->slices, *mx, st) : split_zgemm(split, d, c->slices, st);
    } else {
      gemm(d);
    }
    const double batch = (double)d.nb0 * d.nb1 * d.nb2;
    c->kstat_flops[which] += batch * (8.0 * d.M * d.N * ((double)d.K * d.KB) + 12.0 * d.M * d.N);
    c->kstat_launches[which] += 1;
    if (c->profiling) {
      GG_CUDA(cudaEventRecord(e1, st));
      kev.push_back({which, {e0, e1}});
    }
  };

  // the O(nao^3 NQ) operand builds of P0 (G V and V^+ G) also run on the INT8 engine in split
  // precision: their large operand V is sliced once per launch for the whole tau block and
  // the G operand is small, so slicing costs little next to the FP64 GEMM it replaces
  // The INT8 engine's epilogue gives each lane one row of C, so its stores coalesce when C is
  // contiguous along m; the build outputs are contiguous along n, so they are computed as
  // C^T = B^T A^T (the same slices and int32 sums, so the same result).
  auto gemm_build = [&](ZgemmDesc d) {
    if (split) {
      ZgemmDesc t = transposed(d);
      t.work = gw_work;
      t.work_elems = (long)c->gemm_work.n;
      c->launches += split_zgemm(split, t, c->slices, st);
    } else {
      gemm(d);
    }
  };

  // pair tables: P0 pairs (k, k+q) for every irreducible q, Sigma pairs (k_ibz, k_ibz - q');
  // G1 block indices: block (k1 * ns + sp) of Gf, for every (iq, sp, k).  Built once per
  // symmetry / k-pair / spin setting (the uploads synchronise, so never while capturing).
  if (!c->gw_tables) {
    if (cap) throw Error(GG_ERR_STATE, "gw: tables must be built by an eager build before capture");
    auto tab = std::make_shared<GwTables>();
    std::vector<int> a, b;
    for (int iq = 0; iq < s.inq; ++iq)
      for (int k = 0; k < nk; ++k) {
        a.push_back(k);
        b.push_back((int)c->k1_from_k2q[(size_t)k * s.nq + c->q_r2f[iq]]);
      }
    tab->p0_pairs.build(c, a, b);
    a.clear();
    b.clear();
    for (int qd = 0; qd < s.nq; ++qd)
      for (int kr = 0; kr < s.ink; ++kr) {
        const int k = (int)c->k_r2f[kr];
        a.push_back(k);
        b.push_back((int)c->k2_from_k1q[(size_t)k * s.nq + qd]);
      }
    tab->sg_pairs.build(c, a, b);
    std::vector<int> v;
    for (int iq = 0; iq < s.inq; ++iq)
      for (int sp = 0; sp < ns; ++sp)
        for (int k = 0; k < nk; ++k) v.push_back((int)c->k1_from_k2q[(size_t)k * s.nq + c->q_r2f[iq]] * ns + sp);
    tab->g1_idx.build(v);
    c->gw_tables = tab;
  }
  const GwTables& tables = *std::static_pointer_cast<GwTables>(c->gw_tables);
  const PairTable& p0_pairs = tables.p0_pairs;
  const PairTable& sg_pairs = tables.sg_pairs;
  const IntTable& g1_idx = tables.g1_idx;
  int* gw_err = c->gw_err.ensure(4);
  if (cap) GG_CUDA(cudaMemsetAsync(gw_err, 0, 4 * sizeof(int), st));

  EventTimer tm(st, !cap);
  int h_total = tm.begin(0);
  GG_CUDA(cudaMemsetAsync(Sigma_dev, 0, sizeof(double2) * (size_t)T * ns * s.ink * nn, st));

  // --- unfold G to the full BZ: Gf[k][s][t][i][j]
  int h = tm.begin(1);
  unfold_matrices(c, G_dev, T, ns, Gf, st);
  tm.end(h);

  const double pref = ns == 1 ? -2.0 : -1.0;
  // irreducible q points owned by this shard (round-robin, src/cugw_utils.cu:115), in
  // chunks of pl.qc consecutive owned points; qi indexes the chunk, iq = myq[q0 + qi]
  const std::vector<int> myq = shard_q_points(s.inq, c->shard_rank, c->shard_size);
  const int nmy = (int)myq.size();
  for (int q0 = 0; q0 < nmy; q0 += pl.qc) {
    const int qn = std::min(pl.qc, nmy - q0);
    // ---------------- P0 for every q of the chunk
    h = tm.begin(2);
    for (int qi = 0; qi < qn; ++qi) {
      const int iq = myq[q0 + qi];
      for (int k0 = 0; k0 < nk; k0 += pl.kc) {
        const int kn = std::min(pl.kc, nk - k0);
        p0_pairs.gather(c, (size_t)iq * nk + k0, kn, Vb, st);
        ++c->launches;
        for (int sp = 0; sp < ns; ++sp) {
          // G1[kk][t] = G^{k+q}(tau_t), t < T/2
          launch_gather_blocks(Gf, g1_idx.d.p + ((size_t)iq * ns + sp) * nk + k0, kn, (long)T2 * nn, (long)T * nn,
                               G1, st);
          ++c->launches;
          if (split) {
            p0_split_block(c, split, Gf, G1, Vb, SA, SB, P0 + (long)qi * T2 * NN, k0, kn, spin_a(sp), pl, pref,
                           (sp == 0 && k0 == 0), st, [&](const ZgemmDesc& d, const int* ea, const int* eb) {
                             const Exps pr{ea, eb};
                             gemm_main(d, 0, true, &pr);
                           });
            continue;
          }
          for (int t0 = 0; t0 < T2; t0 += pl.tb) {
            const int tn = std::min(pl.tb, T2 - t0);
            // A-build: SA[kk][tt][Q'][a][b] = sum_p G^k(tau_{T-1-t})[a][p] V[kk][Q'][p][b].
            // The tau block is folded into the rows, m = (tt, a), so that V[kk] is one shared
            // operand and the row tiles are full (n alone is below one tile).
            {
              ZgemmDesc d;
              d.M = tn * n; d.N = N * n; d.K = n;
              d.A = Gf + ((long)k0 * ns + spin_a(sp)) * T * nn + (long)(T - 1 - t0) * nn;
              d.a_m.split = n; d.a_m.hi = -nn; d.a_m.lo = n; d.a_k = 1;
              d.B = Vb; d.b_k = n; d.b_n.split = n; d.b_n.hi = nn; d.b_n.lo = 1;
              d.C = SA; d.c_m.split = n; d.c_m.hi = Nnn; d.c_m.lo = n;
              d.c_n.split = n; d.c_n.hi = nn; d.c_n.lo = 1;
              d.nb0 = kn;
              d.a_b0 = (long)ns * T * nn; d.b_b0 = Nnn; d.c_b0 = (long)tn * Nnn;
              gemm_build(d);
            }
            // B-build: SB[kk][tt][Q][a][b] = sum_l conj(V[kk][Q][a][l]) G^{k+q}(tau_t)[b][l],
            // tau folded into the columns, n = (tt, b)
            {
              ZgemmDesc d;
              d.M = N * n; d.N = tn * n; d.K = n;
              d.A = Vb; d.a_m.lo = n; d.a_k = 1; d.conjA = 1;
              d.B = G1 + (long)t0 * nn; d.b_k = 1; d.b_n.split = n; d.b_n.hi = nn; d.b_n.lo = n;
              d.C = SB; d.c_m.lo = n; d.c_n.split = n; d.c_n.hi = Nnn; d.c_n.lo = 1;
              d.nb0 = kn;
              d.a_b0 = Nnn; d.b_b0 = (long)T2 * nn; d.c_b0 = (long)tn * Nnn;
              gemm_build(d);
            }
            // P0[q][t] (+)= pref/nk sum_kk sum_x SA[kk][tt][Q'][x] SB[kk][tt][Q][x]
            {
              ZgemmDesc d;
              d.M = N; d.N = N; d.K = (int)nn; d.KB = kn;
              d.A = SA; d.a_m.lo = nn; d.a_k = 1; d.a_kb = (long)tn * Nnn;
              d.B = SB; d.b_k = 1; d.b_n.lo = nn; d.b_kb = (long)tn * Nnn;
              d.C = P0 + ((long)qi * T2 + t0) * NN; d.c_m.lo = N; d.c_n.lo = 1;
              d.nb0 = tn; d.a_b0 = Nnn; d.b_b0 = Nnn; d.c_b0 = NN;
              d.alpha = make_double2(pref / nk, 0.0);
              d.beta = (sp == 0 && k0 == 0) ? make_double2(0.0, 0.0) : make_double2(1.0, 0.0);
              gemm_main(d, 0);
            }
          }
        }
      }
    }
    tm.end(h);
    if (c->cap_P0) {
      // mirrored copy P0[nts-1-t] = P0[t] (cugw_qpt.cu:187-190) into the host capture
      GG_CUDA(cudaStreamSynchronize(st));
      for (int qi = 0; qi < qn; ++qi)
        for (int t = 0; t < T2; ++t) {
          const long iq = myq[q0 + qi];
          double2* dst = (double2*)c->cap_P0 + (iq * T + t) * NN;
          GG_CUDA(cudaMemcpy(dst, P0 + ((long)qi * T2 + t) * NN, NN * sizeof(double2), cudaMemcpyDeviceToHost));
          std::memcpy((double2*)c->cap_P0 + (iq * T + (T - 1 - t)) * NN, dst, NN * sizeof(double2));
        }
    }
    // ---------------- IR forward with the tau mirror folded into the matrix
    h = tm.begin(3);
    {
      ZgemmDesc d;
      d.M = nw; d.N = (int)NN; d.K = T2 - 1;
      d.A = c->Tnt_fold.p; d.a_m.lo = T2 - 1; d.a_k = 1;
      d.B = P0 + NN; d.b_k = NN; d.b_n.lo = 1;
      d.C = Pw; d.c_m.lo = NN; d.c_n.lo = 1;
      d.nb0 = qn; d.a_b0 = 0; d.b_b0 = (long)T2 * NN; d.c_b0 = (long)nw * NN;
      gemm(d);
    }
    tm.end(h);
    if (c->cap_Pw) {
      launch_hermitian_symmetrize(Pw, qn * nw, N, st);
      for (int qi = 0; qi < qn; ++qi)
        GG_CUDA(cudaMemcpyAsync((double2*)c->cap_Pw + (long)myq[q0 + qi] * nw * NN, Pw + (long)qi * nw * NN,
                                (size_t)nw * NN * sizeof(double2), cudaMemcpyDeviceToHost, st));
    }
    // ---------------- Dyson, FP64, one CTA per (q, W) system
    h = tm.begin(4);
    for (int s0 = 0; s0 < qn * nw; s0 += dys) {
      const int sn = std::min(dys, qn * nw - s0);
      launch_dyson(Pw + (long)s0 * NN, Af, info + s0, sn, N, solver, piv, st);
      ++c->launches;
    }
    tm.end(h);
    if (cap) {
      // no host round trip inside a graph: the first failing system is recorded on the device
      // and reported after the replay (dyson_failure)
      launch_info_collect(info, qn * nw, q0 * nw, gw_err, st);
    } else {
      GG_CUDA(cudaMemcpyAsync(info_h.data(), info, sizeof(int) * qn * nw, cudaMemcpyDeviceToHost, st));
      GG_CUDA(cudaStreamSynchronize(st));
      for (int i = 0; i < qn * nw; ++i)
        if (info_h[i] != 0) dyson_failure(c, solver, q0 * nw + i, info_h[i]);
    }
    // ---------------- IR back: Wt[q][t] = sum_w Ttn[t][w] W[q][w]
    h = tm.begin(5);
    {
      ZgemmDesc d;
      d.M = T; d.N = (int)NN; d.K = nw;
      d.A = c->Ttn.p; d.a_m.lo = nw; d.a_k = 1;
      d.B = Pw; d.b_k = NN; d.b_n.lo = 1;
      d.C = Wt; d.c_m.lo = NN; d.c_n.lo = 1;
      d.nb0 = qn; d.a_b0 = 0; d.b_b0 = (long)nw * NN; d.c_b0 = (long)T * NN;
      gemm(d);
    }
    tm.end(h);
    if (c->cap_Wt)
      for (int qi = 0; qi < qn; ++qi)
        GG_CUDA(cudaMemcpyAsync((double2*)c->cap_Wt + (long)myq[q0 + qi] * T * NN, Wt + (long)qi * T * NN,
                                (size_t)T * NN * sizeof(double2), cudaMemcpyDeviceToHost, st));
    // ---------------- Sigma contributions of the chunk's q stars
    h = tm.begin(6);
    // the fused tail needs n <= 52 (five n x n blocks in shared memory); larger orbital counts
    // run X G and Z V^+ as two GEMMs.  Flops of the pair (8MNK + 12MN per complex GEMM).
    const bool fused_tail = c->fused_tail && sigma_tail_supported(n, T, (long)c->gemm_work.n);
    const double tail_flops = (double)T * (8.0 * N * n * (double)nn + 12.0 * N * (double)nn) +
                              8.0 * T * n * (double)n * N * n + 12.0 * T * (double)nn;
    for (int qi = 0; qi < qn; ++qi) {
      const int iq = myq[q0 + qi];
      for (int qd : c->q_stars[iq]) {
        const bool trq = c->q_tr[qd] != 0;
        const double2* W = Wt + (long)qi * T * NN;
        if (c->has_Uq) {
          // Wr[t] = U_q' W[t] U_q'^+, once per star member (cugw_qkpt.cu:297-318 does it per (k,t))
          ZgemmDesc d;
          d.M = N; d.N = N; d.K = N;
          d.A = c->Uq.p + (long)qd * NN; d.a_m.lo = N; d.a_k = 1;
          d.B = W; d.b_k = N; d.b_n.lo = 1;
          d.C = SA; d.c_m.lo = N; d.c_n.lo = 1;
          d.nb0 = T; d.a_b0 = 0; d.b_b0 = NN; d.c_b0 = NN;
          gemm(d);
          ZgemmDesc e = d;
          e.A = SA; e.a_b0 = NN;
          e.B = c->Uq.p + (long)qd * NN; e.b_k = 1; e.b_n.lo = N; e.conjB = 1; e.b_b0 = 0;
          e.C = Wr;
          gemm(e);
          W = Wr;
        }
        for (int kr = 0; kr < s.ink; ++kr) {
          const int k1 = (int)c->k2_from_k1q[(size_t)c->k_r2f[kr] * s.nq + qd];
          sg_pairs.gather(c, (size_t)qd * s.ink + kr, 1, Vb, st);
          ++c->launches;
          // X[t][Q][j][l] = sum_P V[P][j][l] W'[t][P][Q]; W' = conj(W) for TR partners.  Rows are
          // x = (j, l), columns Q.  V does not depend on tau or spin: it is the shared operand
          // of the tau batch (sliced once in split precision) and X serves every spin.
          {
            ZgemmDesc d;
            d.M = (int)nn; d.N = N; d.K = N;
            d.A = Vb; d.a_m.lo = 1; d.a_k = nn;
            d.B = W; d.b_k = N; d.b_n.lo = 1; d.conjB = trq ? 1 : 0;
            d.C = SA; d.c_m.lo = 1; d.c_n.lo = nn;
            d.nb0 = T; d.a_b0 = 0; d.b_b0 = NN; d.c_b0 = Nnn;
            gemm_main(d, 1);
          }
          for (int sp = 0; sp < ns; ++sp) {
            const double2* Gk = Gf + ((long)k1 * ns + sp) * T * nn;
            double2* Ck = Sigma_dev + ((long)sp * s.ink + kr) * nn;
            if (fused_tail) {
              // Z = X G and Sigma += -1/nk Z V^+ in one kernel (Z stays in registers); FP64 in
              // both precisions, three-product form inside split builds
              cudaEvent_t e0 = nullptr, e1 = nullptr;
              if (c->profiling) {
                GG_CUDA(cudaEventCreate(&e0));
                GG_CUDA(cudaEventCreate(&e1));
                GG_CUDA(cudaEventRecord(e0, st));
              }
              c->launches += sigma_tail(SA, Nnn, Gk, Vb, n, N, T, Ck, (long)ns * s.ink * nn,
                                        make_double2(-1.0 / nk, 0.0), split != nullptr, gw_work,
                                        (long)c->gemm_work.n, st);
              c->kstat_flops[2] += tail_flops;
              c->kstat_launches[2] += 1;
              if (c->profiling) {
                GG_CUDA(cudaEventRecord(e1, st));
                kev.push_back({2, {e0, e1}});
              }
              continue;
            }
            // Z[t][Q][j][c] = sum_l X[t][Q][j][l] G^{k1}(tau_t)[l][c]
            {
              ZgemmDesc d;
              d.M = N * n; d.N = n; d.K = n;
              d.A = SA; d.a_m.lo = n; d.a_k = 1;
              d.B = Gk; d.b_k = n; d.b_n.lo = 1;
              d.C = SB; d.c_m.lo = n; d.c_n.lo = 1;
              d.nb0 = T; d.a_b0 = Nnn; d.b_b0 = nn; d.c_b0 = Nnn;
              gemm(d);
            }
            // Sigma[t][sp][kr][j][i] += -1/nk sum_Q sum_c Z[t][Q][j][c] conj(V[Q][i][c])
            // (one GEMM over all tau: rows m = (t, j), V is the shared operand).  FP64 in both
            // precisions: on the INT8 engine these two steps (and the slicing of X and Z, new
            // for every tau) measured slower than the FP64 tensor cores
            {
              ZgemmDesc d;
              d.M = T * n; d.N = n; d.K = n; d.KB = N;
              d.A = SB; d.a_m.split = n; d.a_m.hi = Nnn; d.a_m.lo = n; d.a_k = 1; d.a_kb = nn;
              d.B = Vb; d.b_k = 1; d.b_n.lo = n; d.b_kb = nn; d.conjB = 1;
              d.C = Ck;
              d.c_m.split = n; d.c_m.hi = (long)ns * s.ink * nn; d.c_m.lo = n; d.c_n.lo = 1;
              d.alpha = make_double2(-1.0 / nk, 0.0);
              d.beta = make_double2(1.0, 0.0);
              gemm_main(d, 2, false);
            }
          }
        }
      }
    }
    tm.end(h);
  }
  tm.end(h_total);
  if (cap) return;  // the caller checks gw_err and the split engine's flag after the replay
  GG_CUDA(cudaStreamSynchronize(st));
  if (split) split_check(split, st);
  for (auto& e : kev) {
    float ms = 0;
    GG_CUDA(cudaEventElapsedTime(&ms, e.second.first, e.second.second));
    c->kstat_seconds[e.first] += ms * 1e-3;
    cudaEventDestroy(e.second.first);
    cudaEventDestroy(e.second.second);
  }
  double acc[8] = {0};
  tm.collect(acc);
  c->last.total = acc[0];
  c->last.unfold = acc[1];
  c->last.p0 = acc[2];
  c->last.ir_fwd = acc[3];
  c->last.dyson = acc[4];
  c->last.ir_back = acc[5];
  c->last.sigma = acc[6];
}

// ---------------------------------------------------------------------------------------
// HF exchange K_s(k) = pref/nk sum_k2 sum_Q V^Q(k,k2) D_s(k2) V^Q(k,k2)^+ (cuhf_utils.cu:108-134)
void hf_exchange(gg_context* c, const double2* dm_dev, double2* K_dev, cudaStream_t st) {
  if (!c->has_sym || !c->has_kpairs || !c->V)
    throw Error(GG_ERR_STATE, "hf: symmetry, k-pairs and integrals must be set first");
  x2c_check(c);
  const auto& s = c->sh;
  const int n = s.nao, N = s.NQ, nk = s.nk, ns = hf_spins(c);
  const long nn = (long)n * n, Nnn = (long)N * nn;
  c->launches = 0;
  // unfolded density D[k][s][i][j]
  double2* D = c->hf_D.ensure((size_t)nk * ns * nn);
  c->Gtmp.ensure((size_t)nk * ns * nn);
  const size_t room = (size_t)(0.4 * (double)free_bytes()) / (2 * Nnn * sizeof(double2));
  const int kc = (int)std::max<size_t>(1, std::min<size_t>(nk, room));
  double2* Vb = c->Vbuf.ensure((size_t)kc * Nnn);
  double2* X = c->scratchA.ensure((size_t)kc * Nnn);
  double2* work = c->gemm_work.ensure((size_t)1 << 22);
  PairTable pairs;
  {
    std::vector<int> a, b;
    for (int kr = 0; kr < s.ink; ++kr)
      for (int k2 = 0; k2 < nk; ++k2) {
        a.push_back((int)c->k_r2f[kr]);
        b.push_back(k2);
      }
    pairs.build(c, a, b);
  }
  unfold_matrices(c, dm_dev, 1, ns, D, st);  // layout [k][s][n][n]
  GG_CUDA(cudaMemsetAsync(K_dev, 0, sizeof(double2) * (size_t)ns * s.ink * nn, st));
  const double pref = ns == 1 ? -0.5 : -1.0;
  for (int kr = 0; kr < s.ink; ++kr) {
    for (int k0 = 0; k0 < nk; k0 += kc) {
      const int kn = std::min(kc, nk - k0);
      pairs.gather(c, (size_t)kr * nk + k0, kn, Vb, st);
      ++c->launches;
      for (int sp = 0; sp < ns; ++sp) {
        // X[kk][Q][j][c] = sum_a V[kk][Q][j][a] D[k2][sp][a][c]   (cuhf_utils.cu:118)
        ZgemmDesc d;
        d.M = N * n; d.N = n; d.K = n;
        d.A = Vb; d.a_m.lo = n; d.a_k = 1;
        d.B = D + ((long)k0 * ns + sp) * nn; d.b_k = n; d.b_n.lo = 1;
        d.C = X; d.c_m.lo = n; d.c_n.lo = 1;
        d.nb0 = kn; d.a_b0 = Nnn; d.b_b0 = (long)ns * nn; d.c_b0 = Nnn;
        d.work = work; d.work_elems = (long)c->gemm_work.n;
        c->launches += zgemm(d, st);
        // K[sp][kr][j][i] += pref/nk sum_{kk,Q} sum_c X[kk][Q][j][c] conj(V[kk][Q][i][c])  (:127-131)
        // (the dominant exchange contraction; split precision when requested)
        ZgemmDesc e;
        e.M = n; e.N = n; e.K = n; e.KB = kn * N;
        e.A = X; e.a_m.lo = n; e.a_k = 1; e.a_kb = nn;
        e.B = Vb; e.b_k = 1; e.b_n.lo = n; e.b_kb = nn; e.conjB = 1;
        e.C = K_dev + ((long)sp * s.ink + kr) * nn; e.c_m.lo = n; e.c_n.lo = 1;
        e.alpha = make_double2(pref / nk, 0.0);
        e.beta = make_double2(1.0, 0.0);
        e.work = work; e.work_elems = (long)c->gemm_work.n;
        if (c->hf_precision == GG_PREC_SPLIT)
          c->launches += split_zgemm(split_engine(c), e, c->slices, st);
        else
          c->launches += zgemm(e, st);
      }
    }
  }
  if (c->hf_precision == GG_PREC_SPLIT) split_check(c->split, st);
}

// Hartree (direct) term J(k) = sum_Q c_Q V^Q(k,k), c_Q = 1/nk sum_{s,k'} Tr(V^Q(k',k') D_s(k'))
// (hf_gpu_kernel.cpp:141-186).  Uses the unfolded density left in c->hf_D by hf_exchange.
void hf_direct(gg_context* c, double2* F_dev, cudaStream_t st) {
  const auto& s = c->sh;
  // X2C: the density of the aa and bb blocks, J added to both (hf_gpu_kernel.cpp:269-309)
  const int n = s.nao, N = s.NQ, nk = s.nk, ns = hf_spins(c), nsj = c->x2c ? 2 : ns;
  const long nn = (long)n * n, Nnn = (long)N * nn;
  double2* cq = c->hf_c.ensure(N);
  GG_CUDA(cudaMemsetAsync(cq, 0, sizeof(double2) * N, st));
  const int kc = (int)std::max<size_t>(1, std::min<size_t>(nk, c->Vbuf.n / Nnn));
  double2* Vb = c->Vbuf.ensure((size_t)kc * Nnn);
  double2* Dk = c->hf_J.ensure((size_t)kc * nn);
  PairTable diag;
  IntTable didx;
  {
    std::vector<int> a(nk), v;
    for (int k = 0; k < nk; ++k) a[k] = k;
    diag.build(c, a, a);
    for (int sp = 0; sp < ns; ++sp)
      for (int k = 0; k < nk; ++k) v.push_back(k * ns + sp);
    didx.build(v);
  }
  for (int k0 = 0; k0 < nk; k0 += kc) {
    const int kn = std::min(kc, nk - k0);
    diag.gather(c, k0, kn, Vb, st);
    for (int sp = 0; sp < nsj; ++sp) {
      launch_gather_blocks(c->hf_D.p, didx.d.p + (size_t)sp * nk + k0, kn, nn, nn, Dk, st);
      launch_hartree_coeff(Vb, Dk, kn, N, n, 1.0 / nk, cq, st);
    }
  }
  double2* J = c->scratchB.ensure((size_t)nn);
  for (int kr = 0; kr < s.ink; ++kr) {
    diag.gather(c, (size_t)c->k_r2f[kr], 1, Vb, st);
    launch_hartree_apply(Vb, cq, N, n, J, st);
    for (int sp = 0; sp < nsj; ++sp) launch_axpy(F_dev + ((long)sp * s.ink + kr) * nn, J, nn, st);
  }
}

}  // namespace gg
