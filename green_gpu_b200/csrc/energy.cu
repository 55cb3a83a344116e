// FP64 energy and chemical-potential reductions over the library's outputs.
//
// green-gpu returns Sigma(tau) and the Fock matrix; its caller (green-mbpt) reduces the
// energies and the chemical potential from them in double precision.  These entry points do
// the same reductions in FP64 next to the data (the GW energy on the device, over the Sigma
// and G that a build leaves there):
//   k weights w_k = |star(k)| / nk over the irreducible k points (the IBZ sums of the symmetry
//   tables of src/gw_gpu_kernel.cpp:34-91); spin factor f = 2 for ns = 1 (matrices per spin),
//   1 for ns = 2 and for two-component (X2C) matrices;
//   E_1b = f sum_{s,k} w_k Re Tr(D H),  E_HF = (f/2) sum_{s,k} w_k Re Tr(D (H + F));
//   E_GW = -(f/2) sum_{s,k} w_k sum_{t,t'} M[t][t'] Re Tr(Sigma(tau_t) G(tau_t')), M the
//   caller's bilinear quadrature of int_0^beta f(tau) g(beta - tau) dtau on the tau grid;
//   mu: root of f sum_{s,k} w_k sum_n 1 / (1 + exp(beta (e_skn - mu))) = n_elec, e_skn the
//   eigenvalues of F x = e S x (Cholesky reduction and cyclic complex Jacobi, FP64, host).
#include <algorithm>
#include <cmath>
#include <vector>

#include "abi.cuh"
#include "engine.cuh"
#include "kernels.cuh"
#include "zgemm.cuh"

using namespace gg;

namespace {

// order of the matrices and number of spin blocks of a context's dm / F / G / Sigma
void matrix_shape(const gg_context* c, int* ns, int* m, double* f) {
  *ns = c->x2c ? 1 : c->sh.ns;
  *m = c->x2c ? 2 * c->sh.nao : c->sh.nao;
  *f = (c->sh.ns == 1 && !c->x2c) ? 2.0 : 1.0;
}

std::vector<double> kweights(const gg_context* c) {
  if (!c->has_sym) throw Error(GG_ERR_STATE, "energy: symmetry not set (the k weights come from the stars)");
  std::vector<double> w(c->sh.ink);
  for (int k = 0; k < c->sh.ink; ++k) w[k] = (double)c->k_stars[k].size() / c->sh.nk;
  return w;
}

// Re Tr(A B) of two n x n row-major complex matrices
double re_trace(const double2* A, const double2* B, int n) {
  double acc = 0.0;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      const double2 a = A[(size_t)i * n + j], b = B[(size_t)j * n + i];
      acc += a.x * b.x - a.y * b.y;
    }
  return acc;
}

// eigenvalues of the Hermitian pencil (F, S), n x n row-major: S = L L^+, A = L^-1 F L^-+,
// cyclic Jacobi on A (rotations zero |a_pq| until the off-diagonal norm is at rounding level)
std::vector<double> pencil_eigenvalues(const double2* F, const double2* S, int n) {
  std::vector<double2> L((size_t)n * n, make_double2(0, 0));
  for (int j = 0; j < n; ++j) {
    double d = S[(size_t)j * n + j].x;
    for (int k = 0; k < j; ++k) d -= L[(size_t)j * n + k].x * L[(size_t)j * n + k].x + L[(size_t)j * n + k].y * L[(size_t)j * n + k].y;
    if (!(d > 0.0)) throw Error(GG_ERR_ARG, "chemical potential: overlap matrix is not positive definite");
    const double ljj = std::sqrt(d);
    L[(size_t)j * n + j] = make_double2(ljj, 0.0);
    for (int i = j + 1; i < n; ++i) {
      double2 v = S[(size_t)i * n + j];
      for (int k = 0; k < j; ++k) v = csub(v, cmulc(L[(size_t)i * n + k], L[(size_t)j * n + k]));
      L[(size_t)i * n + j] = cscale(v, 1.0 / ljj);
    }
  }
  // Y = L^-1 F (forward substitution per column), A = Y L^-+ = (L^-1 Y^+)^+
  auto lsolve = [&](std::vector<double2>& X) {  // X <- L^-1 X, X n x n
    for (int col = 0; col < n; ++col)
      for (int i = 0; i < n; ++i) {
        double2 v = X[(size_t)i * n + col];
        for (int k = 0; k < i; ++k) v = csub(v, cmul(L[(size_t)i * n + k], X[(size_t)k * n + col]));
        X[(size_t)i * n + col] = cscale(v, 1.0 / L[(size_t)i * n + i].x);
      }
  };
  std::vector<double2> Y(F, F + (size_t)n * n);
  lsolve(Y);
  std::vector<double2> A((size_t)n * n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) A[(size_t)i * n + j] = cconj(Y[(size_t)j * n + i]);
  lsolve(A);  // A = L^-1 (L^-1 F)^+ = L^-1 F L^-+ (F Hermitian)
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < i; ++j) {  // symmetrise away rounding
      const double2 a = A[(size_t)i * n + j], b = cconj(A[(size_t)j * n + i]);
      A[(size_t)i * n + j] = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y + b.y));
      A[(size_t)j * n + i] = cconj(A[(size_t)i * n + j]);
    }
  for (int i = 0; i < n; ++i) A[(size_t)i * n + i].y = 0.0;
  double diag = 0.0;
  for (int i = 0; i < n; ++i) diag = std::max(diag, std::fabs(A[(size_t)i * n + i].x));
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) off += A[(size_t)p * n + q].x * A[(size_t)p * n + q].x + A[(size_t)p * n + q].y * A[(size_t)p * n + q].y;
    if (std::sqrt(off) <= 1e-15 * std::max(diag, 1e-300)) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double2 apq = A[(size_t)p * n + q];
        const double g = std::hypot(apq.x, apq.y);
        if (g == 0.0) continue;
        // phase e^{i phi} = apq / |apq|; real rotation on the phase-adjusted pair
        const double2 ph = make_double2(apq.x / g, apq.y / g);
        const double app = A[(size_t)p * n + p].x, aqq = A[(size_t)q * n + q].x;
        const double theta = 0.5 * std::atan2(2.0 * g, aqq - app);
        const double cs = std::cos(theta), sn = std::sin(theta);
        // columns: a_kp' = c a_kp - s conj(ph) a_kq,  a_kq' = s ph a_kp + c a_kq
        for (int k = 0; k < n; ++k) {
          const double2 akp = A[(size_t)k * n + p], akq = A[(size_t)k * n + q];
          A[(size_t)k * n + p] = csub(cscale(akp, cs), cscale(cmul(cconj(ph), akq), sn));
          A[(size_t)k * n + q] = cadd(cscale(cmul(ph, akp), sn), cscale(akq, cs));
        }
        // rows: a_pk' = c a_pk - s ph a_qk,  a_qk' = s conj(ph) a_pk + c a_qk
        for (int k = 0; k < n; ++k) {
          const double2 apk = A[(size_t)p * n + k], aqk = A[(size_t)q * n + k];
          A[(size_t)p * n + k] = csub(cscale(apk, cs), cscale(cmul(ph, aqk), sn));
          A[(size_t)q * n + k] = cadd(cscale(cmul(cconj(ph), apk), sn), cscale(aqk, cs));
        }
        A[(size_t)p * n + q] = make_double2(0, 0);
        A[(size_t)q * n + p] = make_double2(0, 0);
        A[(size_t)p * n + p].y = 0.0;
        A[(size_t)q * n + q].y = 0.0;
      }
  }
  std::vector<double> e(n);
  for (int i = 0; i < n; ++i) e[i] = A[(size_t)i * n + i].x;
  std::sort(e.begin(), e.end());
  return e;
}

// f sum_k w_k sum_n fermi(beta (e - mu)), overflow-free
double particle_number(const std::vector<std::vector<double>>& eps, const std::vector<double>& wk, double mu,
                       double beta, double f) {
  double n = 0.0;
  for (size_t b = 0; b < eps.size(); ++b) {
    double acc = 0.0;
    for (double e : eps[b]) {
      const double x = beta * (e - mu);
      acc += x > 0 ? std::exp(-x) / (1.0 + std::exp(-x)) : 1.0 / (1.0 + std::exp(x));
    }
    n += wk[b] * acc;
  }
  return f * n;
}

}  // namespace

extern "C" {

int gg_energy_hf(gg_context* c, const double* dm, const double* H, const double* F, double* out) {
  return guarded(c, [&] {
    if (!dm || !H || !F || !out) throw Error(GG_ERR_ARG, "energy: NULL buffer");
    int ns, m;
    double f;
    matrix_shape(c, &ns, &m, &f);
    const auto w = kweights(c);
    const size_t mm = (size_t)m * m;
    const double2* D = (const double2*)dm;
    const double2* Hh = (const double2*)H;
    const double2* Fh = (const double2*)F;
    double e1 = 0.0, e2 = 0.0;
    for (int s = 0; s < ns; ++s)
      for (int k = 0; k < c->sh.ink; ++k) {
        const size_t o = ((size_t)s * c->sh.ink + k) * mm;
        const double th = re_trace(D + o, Hh + o, m), tf = re_trace(D + o, Fh + o, m);
        e1 += w[k] * th;
        e2 += w[k] * (th + tf);
      }
    out[0] = f * e1;
    out[1] = 0.5 * f * e2;
  });
}

int gg_energy_gw_device(gg_context* c, const void* G, const void* Sigma, const double* M, double* e_gw, void* stream) {
  return guarded(c, [&] {
    if (!G || !Sigma || !M || !e_gw) throw Error(GG_ERR_ARG, "energy: NULL buffer");
    int ns, m;
    double f;
    matrix_shape(c, &ns, &m, &f);
    const auto w = kweights(c);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    const int T = c->sh.nts, ink = c->sh.ink;
    const long mm = (long)m * m, nb = (long)ns * ink;
    // C_b[t][t'] = sum_{ij} Sigma_b(t)_ij G_b(t')_ji = Sigma_b(t) . G_b(t')^T (flattened), one
    // batched FP64 GEMM over b = (s, k) after transposing every matrix of G
    DevBuf<double2> gt, cb, work;
    double2* Gt = gt.ensure((size_t)T * nb * mm);
    launch_transpose_blocks((const double2*)G, (long)T * nb, m, Gt, st);
    double2* C = cb.ensure((size_t)nb * T * T);
    ZgemmDesc d;
    d.M = T; d.N = T; d.K = (int)mm;
    d.A = (const double2*)Sigma; d.a_m.lo = nb * mm; d.a_k = 1;
    d.B = Gt; d.b_k = 1; d.b_n.lo = nb * mm;
    d.C = C; d.c_m.lo = T; d.c_n.lo = 1;
    d.nb0 = (int)nb; d.a_b0 = mm; d.b_b0 = mm; d.c_b0 = (long)T * T;
    d.work = work.ensure((size_t)1 << 20);
    d.work_elems = 1 << 20;
    zgemm(d, st);
    std::vector<double2> h((size_t)nb * T * T);
    GG_CUDA(cudaMemcpyAsync(h.data(), C, h.size() * sizeof(double2), cudaMemcpyDeviceToHost, st));
    GG_CUDA(cudaStreamSynchronize(st));
    double e = 0.0;
    for (long b = 0; b < nb; ++b) {
      double acc = 0.0;
      for (int t = 0; t < T; ++t)
        for (int u = 0; u < T; ++u) acc += M[(size_t)t * T + u] * h[((size_t)b * T + t) * T + u].x;
      e += w[b % ink] * acc;
    }
    *e_gw = -0.5 * f * e;
  });
}

int gg_energy_gw(gg_context* c, const double* G, const double* Sigma, const double* M, double* e_gw) {
  return guarded(c, [&] {
    if (!G || !Sigma) throw Error(GG_ERR_ARG, "energy: NULL buffer");
    int ns, m;
    double f;
    matrix_shape(c, &ns, &m, &f);
    const size_t count = (size_t)c->sh.nts * ns * c->sh.ink * m * m;
    DevBuf<double2> g, s;
    g.upload((const double2*)G, count, c->stream);
    s.upload((const double2*)Sigma, count, c->stream);
    const int rc = gg_energy_gw_device(c, g.p, s.p, M, e_gw, c->stream);
    if (rc != GG_OK) throw Error(rc, c->err);
  });
}

int gg_chemical_potential(int32_t ns, int32_t ink, int32_t n, const double* weights, const double* F,
                          const double* S, double beta, double spin_factor, double nelec, double* mu,
                          double* n_at_mu) {
  return guarded_global([&] {
    if (ns < 1 || ink < 1 || n < 1 || !weights || !F || !S || !mu || !(beta > 0.0) || !(spin_factor > 0.0))
      throw Error(GG_ERR_ARG, "chemical potential: bad arguments");
    const size_t nn = (size_t)n * n;
    std::vector<std::vector<double>> eps;
    std::vector<double> wk;
    double lo = 1e300, hi = -1e300, states = 0.0;
    for (int s = 0; s < ns; ++s)
      for (int k = 0; k < ink; ++k) {
        const size_t o = ((size_t)s * ink + k) * nn;
        eps.push_back(pencil_eigenvalues((const double2*)F + o, (const double2*)S + o, n));
        wk.push_back(weights[k]);
        lo = std::min(lo, eps.back().front());
        hi = std::max(hi, eps.back().back());
        states += weights[k] * n;
      }
    if (!(nelec > 0.0) || nelec >= spin_factor * states)
      throw Error(GG_ERR_ARG, "chemical potential: n_elec must lie strictly between 0 and the number of states");
    lo -= 50.0 / beta;
    hi += 50.0 / beta;
    // bisection until the bracket cannot shrink in FP64
    for (int it = 0; it < 400; ++it) {
      const double mid = 0.5 * (lo + hi);
      if (mid <= lo || mid >= hi) break;
      if (particle_number(eps, wk, mid, beta, spin_factor) < nelec) lo = mid;
      else hi = mid;
    }
    *mu = 0.5 * (lo + hi);
    if (n_at_mu) *n_at_mu = particle_number(eps, wk, *mu, beta, spin_factor);
  });
}

}  // extern "C"
