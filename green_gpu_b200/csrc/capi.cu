// extern "C" entry points of libgreen_b200.so (declared in include/green_b200.h).
// No C++ exception crosses this boundary: every call returns a GG_* status and keeps
// the message for gg_last_error().
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "abi.cuh"
#include "context.cuh"
#include "engine.cuh"
#include "kernels.cuh"
#include "split.cuh"
#include "zgemm.cuh"

using namespace gg;

namespace {

thread_local std::string g_create_error;


void check_shape(const gg_shape& s) {
  auto bad = [](const std::string& m) { throw Error(GG_ERR_ARG, "shape: " + m); };
  if (s.nk <= 0 || s.ink <= 0 || s.ink > s.nk) bad("need 0 < ink <= nk");
  if (s.nq != s.nk) bad("nq must equal nk");
  if (s.inq <= 0 || s.inq > s.nq) bad("need 0 < inq <= nq");
  if (s.nao <= 0 || s.NQ <= 0) bad("nao and NQ must be positive");
  if (s.ns != 1 && s.ns != 2) bad("ns must be 1 or 2");
  if (s.nts < 4 || s.nts % 2) bad("nts must be even and >= 4 (gw_gpu_kernel.h:67)");
  if (s.nw_b < 0 || s.nw_b > s.nts) bad("need 0 <= nw_b <= nts (cugw_qpt.cu:79; 0 for HF-only contexts)");
}

}  // namespace

void gg::set_thread_error(const std::string& msg) { g_create_error = msg; }


extern "C" {

const char* gg_version(void) { return "green-b200 0.1 (sm_100a; FP64 DMMA engine)"; }

int gg_create(const gg_shape* shape, int device, gg_context** out) {
  if (!shape || !out) return GG_ERR_ARG;
  *out = nullptr;
  gg_context* c = nullptr;
  try {
    check_shape(*shape);
    int ndev = 0;
    GG_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) throw Error(GG_ERR_ARG, "no CUDA device " + std::to_string(device));
    GG_CUDA(cudaSetDevice(device));
    c = new gg_context();
    c->sh = *shape;
    c->device = device;
    GG_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    *out = c;
    g_create_error.clear();
    return GG_OK;
  } catch (const Error& e) {
    g_create_error = e.what();
    delete c;
    return e.code;
  } catch (const std::exception& e) {
    g_create_error = e.what();
    delete c;
    return GG_ERR_INTERNAL;
  }
}

void gg_destroy(gg_context* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  delete c;
}

const char* gg_last_error(const gg_context* c) { return c ? c->err.c_str() : g_create_error.c_str(); }

int gg_set_symmetry(gg_context* c, const int64_t* k_f2r, const int64_t* k_r2f, const int64_t* k_tr,
                    const int64_t* q_f2r, const int64_t* q_r2f, const int64_t* q_tr, const int64_t* k1q,
                    const int64_t* k2q, const double* U_k, const double* U_q) {
  return guarded(c, [&] {
    c->invalidate();  // tables and captured graph depend on this setting
    if (!k_f2r || !k_r2f || !k_tr || !q_f2r || !q_r2f || !q_tr || !k1q || !k2q)
      throw Error(GG_ERR_ARG, "symmetry: index arrays must not be NULL");
    const auto& s = c->sh;
    auto range = [](const int64_t* a, long n, long hi, const char* what) {
      for (long i = 0; i < n; ++i)
        if (a[i] < 0 || a[i] >= hi) throw Error(GG_ERR_ARG, std::string("symmetry: ") + what + " out of range");
    };
    range(k_f2r, s.nk, s.ink, "k_full_to_reduced");
    range(k_r2f, s.ink, s.nk, "k_reduced_to_full");
    range(q_f2r, s.nq, s.inq, "q_full_to_reduced");
    range(q_r2f, s.inq, s.nq, "q_reduced_to_full");
    range(k1q, (long)s.nk * s.nq, s.nk, "k1_from_k2q");
    range(k2q, (long)s.nk * s.nq, s.nk, "k2_from_k1q");
    for (long i = 0; i < s.ink; ++i)
      if (k_f2r[k_r2f[i]] != i) throw Error(GG_ERR_ARG, "symmetry: k maps are inconsistent");
    for (long i = 0; i < s.inq; ++i)
      if (q_f2r[q_r2f[i]] != i) throw Error(GG_ERR_ARG, "symmetry: q maps are inconsistent");
    c->k_f2r.assign(k_f2r, k_f2r + s.nk);
    c->k_r2f.assign(k_r2f, k_r2f + s.ink);
    c->k_tr.assign(k_tr, k_tr + s.nk);
    c->q_f2r.assign(q_f2r, q_f2r + s.nq);
    c->q_r2f.assign(q_r2f, q_r2f + s.inq);
    c->q_tr.assign(q_tr, q_tr + s.nq);
    c->k1_from_k2q.assign(k1q, k1q + (size_t)s.nk * s.nq);
    c->k2_from_k1q.assign(k2q, k2q + (size_t)s.nk * s.nq);
    c->k_stars.assign(s.ink, {});
    c->q_stars.assign(s.inq, {});
    for (int k = 0; k < s.nk; ++k) c->k_stars[k_f2r[k]].push_back(k);
    for (int q = 0; q < s.nq; ++q) c->q_stars[q_f2r[q]].push_back(q);
    std::vector<int> f2r(s.nk), tr(s.nk);
    for (int k = 0; k < s.nk; ++k) {
      f2r[k] = (int)k_f2r[k];
      tr[k] = k_tr[k] != 0;
    }
    c->k_f2r_d.upload(f2r.data(), f2r.size(), c->stream);
    c->k_tr_d.upload(tr.data(), tr.size(), c->stream);
    const long nn = (long)s.nao * s.nao, NN = (long)s.NQ * s.NQ;
    c->has_Uk = U_k != nullptr;
    c->has_Uq = U_q != nullptr;
    if (U_k) c->Uk.upload((const double2*)U_k, (size_t)s.nk * nn, c->stream);
    if (U_q) c->Uq.upload((const double2*)U_q, (size_t)s.nq * NN, c->stream);
    GG_CUDA(cudaStreamSynchronize(c->stream));
    c->has_sym = true;
  });
}

int gg_set_kpairs(gg_context* c, int64_t nstored, const int64_t* conj_list, const int64_t* trans_list,
                  const int64_t* irre_pos) {
  return guarded(c, [&] {
    c->invalidate();  // tables and captured graph depend on this setting
    if (!conj_list || !trans_list || !irre_pos || nstored <= 0) throw Error(GG_ERR_ARG, "kpairs: bad arguments");
    const long npairs = (long)c->sh.nk * (c->sh.nk + 1) / 2;
    for (long i = 0; i < npairs; ++i) {
      if (conj_list[i] < 0 || conj_list[i] >= npairs || trans_list[i] < 0 || trans_list[i] >= npairs ||
          irre_pos[i] < -1 || irre_pos[i] >= nstored)
        throw Error(GG_ERR_ARG, "kpairs: entry " + std::to_string(i) + " out of range");
    }
    c->nstored = nstored;
    c->conj_list.assign(conj_list, conj_list + npairs);
    c->trans_list.assign(trans_list, trans_list + npairs);
    c->irre_pos.assign(irre_pos, irre_pos + npairs);
    c->has_kpairs = true;
  });
}

int gg_set_coulomb(gg_context* c, const double* V) {
  return guarded(c, [&] {
    c->invalidate();  // tables and captured graph depend on this setting
    if (!V) throw Error(GG_ERR_ARG, "coulomb: NULL");
    if (!c->has_kpairs) throw Error(GG_ERR_STATE, "coulomb: call gg_set_kpairs first");
    const size_t count = (size_t)c->nstored * c->sh.NQ * c->sh.nao * c->sh.nao;
    c->V_owned.upload((const double2*)V, count, c->stream);
    GG_CUDA(cudaStreamSynchronize(c->stream));
    c->V = c->V_owned.p;
  });
}

int gg_set_coulomb_device(gg_context* c, const void* V) {
  return guarded(c, [&] {
    c->invalidate();  // tables and captured graph depend on this setting
    if (!V) throw Error(GG_ERR_ARG, "coulomb: NULL");
    if ((reinterpret_cast<uintptr_t>(V) & 15) != 0) throw Error(GG_ERR_ARG, "coulomb: device pointer not 16-byte aligned");
    if (!c->has_kpairs) throw Error(GG_ERR_STATE, "coulomb: call gg_set_kpairs first");
    cudaPointerAttributes attr{};
    GG_CUDA(cudaPointerGetAttributes(&attr, V));
    if (attr.type != cudaMemoryTypeDevice || attr.device != c->device)
      throw Error(GG_ERR_ARG, "coulomb: pointer is not device memory of this context's device");
    c->V_owned.release();
    c->V = (const double2*)V;
  });
}

int gg_set_ir(gg_context* c, const double* Ttn_FB, const double* Tnt_BF) {
  return guarded(c, [&] {
    c->invalidate();  // tables and captured graph depend on this setting
    if (!Ttn_FB || !Tnt_BF) throw Error(GG_ERR_ARG, "ir: NULL");
    if (c->sh.nw_b <= 0) throw Error(GG_ERR_ARG, "ir: the context was created with nw_b = 0");
    const int T = c->sh.nts, T2 = T / 2, nw = c->sh.nw_b;
    c->Ttn.upload((const double2*)Ttn_FB, (size_t)T * nw, c->stream);
    // Tnt_BF acts on tau points 1..T-2; P0(tau_{T-1-t}) = P0(tau_t) lets the columns of the
    // mirrored half be added onto their partners: fold[w][t-1] = Tnt[w][t-1] + Tnt[w][T-2-t]
    // for t = 1..T/2-1 (t = T-1-t never happens for even T).
    const double2* Tn = (const double2*)Tnt_BF;
    std::vector<double2> fold((size_t)nw * (T2 - 1));
    for (int w = 0; w < nw; ++w)
      for (int t = 1; t < T2; ++t) {
        double2 a = Tn[(size_t)w * (T - 2) + (t - 1)];
        double2 b = Tn[(size_t)w * (T - 2) + (T - 2 - t)];
        fold[(size_t)w * (T2 - 1) + (t - 1)] = make_double2(a.x + b.x, a.y + b.y);
      }
    c->Tnt_fold.upload(fold.data(), fold.size(), c->stream);
    GG_CUDA(cudaStreamSynchronize(c->stream));
    c->has_ir = true;
  });
}

int gg_set_hf_precision(gg_context* c, int precision) {
  return guarded(c, [&] {
    if (precision != GG_PREC_FP64 && precision != GG_PREC_SPLIT) throw Error(GG_ERR_ARG, "hf: unknown precision");
    c->hf_precision = precision;
  });
}

int gg_set_q_shard(gg_context* c, int rank, int size) {
  return guarded(c, [&] {
    c->invalidate();  // tables and captured graph depend on this setting
    if (size < 1 || rank < 0 || rank >= size) throw Error(GG_ERR_ARG, "q shard: need 0 <= rank < size");
    c->shard_rank = rank;
    c->shard_size = size;
  });
}

int gg_q_shard_points(int32_t inq, int rank, int size, int32_t* q_out, int32_t capacity, int32_t* count) {
  return guarded_global([&] {
    if (!count || (capacity > 0 && !q_out) || capacity < 0) throw Error(GG_ERR_ARG, "q shard points: bad buffers");
    const std::vector<int> q = shard_q_points(inq, rank, size);
    *count = (int32_t)q.size();
    for (size_t i = 0; i < q.size() && (int32_t)i < capacity; ++i) q_out[i] = q[i];
  });
}

int gg_set_split_slices(gg_context* c, int slices) {
  return guarded(c, [&] {
    c->invalidate();  // tables and captured graph depend on this setting
    if (slices < 2 || slices > 8) throw Error(GG_ERR_ARG, "split slices must be in [2, 8]");
    c->slices = slices;
  });
}

int gg_set_capture(gg_context* c, double* P0_out, double* Pw_out, double* Wt_out) {
  return guarded(c, [&] {
    c->cap_P0 = P0_out;
    c->cap_Pw = Pw_out;
    c->cap_Wt = Wt_out;
  });
}

// GW build on device buffers in the reference layout; in X2C mode the spinor G is split into
// its four spin blocks, the build runs on them as pseudo-spins and Sigma is reassembled
static void gw_sequence(gg_context* c, const double2* G, double2* Sigma, int solver, int precision, cudaStream_t st) {
  if (!c->x2c) {
    gw_build(c, G, Sigma, solver, precision, st);
    return;
  }
  x2c_check(c);
  const auto& s = c->sh;
  const size_t count = (size_t)s.nts * 4 * s.ink * s.nao * s.nao;
  double2* g4 = c->x2c_in.ensure(count);
  double2* s4 = c->x2c_out.ensure(count);
  launch_x2c_split(G, s.nts, s.ink, s.nao, 4, g4, st);
  gw_build(c, g4, s4, solver, precision, st);
  launch_x2c_merge(s4, s.nts, s.ink, s.nao, 4, Sigma, st);
}

}  // extern "C"

// capture f() (work issued on `st`, and on streams joined to it) into an executable graph
template <typename F>
static cudaGraphExec_t capture_graph(const std::vector<gg_context*>& ctxs, cudaStream_t st, F&& f) {
  cudaGraph_t g = nullptr;
  GG_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  for (auto* c : ctxs) c->capturing = true;
  try {
    f();
  } catch (...) {
    for (auto* c : ctxs) c->capturing = false;
    cudaStreamEndCapture(st, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  for (auto* c : ctxs) c->capturing = false;
  GG_CUDA(cudaStreamEndCapture(st, &g));
  cudaGraphExec_t ex = nullptr;
  const cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) throw Error(GG_ERR_CUDA, std::string("graph instantiation: ") + cudaGetErrorString(e));
  return ex;
}

std::vector<const void*> gg_context::buffer_signature() const {
  std::vector<const void*> v = {V,       V_owned.p, Uk.p,      Uq.p,    k_f2r_d.p,   k_tr_d.p,   Ttn.p,
                                Tnt_fold.p, x2c_in.p, x2c_out.p, G_in.p, Sigma_out.p, Gf.p,       Gtmp.p,
                                Vbuf.p,  G1buf.p,   scratchA.p, scratchB.p, P0buf.p, Pw.p,     Afac.p,
                                Wt.p,    Wrot.p,    gemm_work.p, hf_D.p,  hf_F.p,      hf_c.p,     hf_J.p,
                                info.p,  piv.p,     idx_i.p,   pos_d.p,  op_d.p,      gw_err.p,   gw_tables.get(),
                                p0_ea.p, p0_eb.p};
  split_buffers(split, v);
  return v;
}

extern "C" {

// after a replay: the Dyson status recorded on the device and the split engine's flag
static void graph_check(gg_context* c, int solver) {
  int e[3] = {0, 0, 0};
  GG_CUDA(cudaMemcpy(e, c->gw_err.p, sizeof(e), cudaMemcpyDeviceToHost));
  if (c->split) split_check(c->split, c->stream);
  if (e[0]) dyson_failure(c, solver, e[1], e[2]);
}

static void gw_device(gg_context* c, const double2* G, double2* Sigma, int solver, int precision, cudaStream_t st) {
  if (!c->graph_mode || c->profiling || c->cap_P0 || c->cap_Pw || c->cap_Wt || st == nullptr) {
    gw_sequence(c, G, Sigma, solver, precision, st);
    return;
  }
  if (c->graph_exec && c->graph_G == G && c->graph_S == Sigma && c->graph_solver == solver &&
      c->graph_prec == precision && c->graph_stream == st && c->graph_sig == c->buffer_signature()) {
    GG_CUDA(cudaGraphLaunch(c->graph_exec, st));
    GG_CUDA(cudaStreamSynchronize(st));
    graph_check(c, solver);
    return;
  }
  // eager build (allocates, builds the tables, gives this call's result), then capture the
  // same sequence for the following calls
  c->drop_graph();
  gw_sequence(c, G, Sigma, solver, precision, st);
  c->graph_exec = capture_graph({c}, st, [&] { gw_sequence(c, G, Sigma, solver, precision, st); });
  c->graph_sig = c->buffer_signature();
  c->graph_G = G;
  c->graph_S = Sigma;
  c->graph_solver = solver;
  c->graph_prec = precision;
  c->graph_stream = st;
}

// matrices per (outer, spin, k) block of a G / Sigma / dm buffer: nao^2 x ns, or (2 nao)^2 in X2C
static size_t spin_elems(const gg_context* c) {
  const size_t nn = (size_t)c->sh.nao * c->sh.nao;
  return c->x2c ? 4 * nn : (size_t)c->sh.ns * nn;
}

int gg_set_x2c(gg_context* c, int enable) {
  return guarded(c, [&] {
    if (enable && c->sh.ns != 1) throw Error(GG_ERR_ARG, "x2c: the spinor shape has ns = 1 (nso = 2 nao)");
    c->x2c = enable != 0;
    c->invalidate();
  });
}

int gg_set_graph(gg_context* c, int enable) {
  return guarded(c, [&] {
    c->graph_mode = enable != 0;
    c->drop_graph();
  });
}

// several systems' GW builds in one CUDA graph, each on its own context stream
struct gg_batch {
  std::vector<gg_context*> ctx;
  std::vector<const double2*> G;
  std::vector<double2*> S;
  int solver = 0, precision = 0;
  cudaStream_t master = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t exec = nullptr;
  std::vector<std::vector<const void*>> sig;  // each member's buffer addresses at capture
  ~gg_batch() {
    if (exec) cudaGraphExecDestroy(exec);
    for (auto e : join) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    if (master) cudaStreamDestroy(master);
  }
};

}  // extern "C"

extern "C" {

int gg_batch_create(gg_context* const* ctxs, int n, const void* const* G, void* const* Sigma, int solver,
                    int precision, gg_batch** out) {
  return guarded_global([&] {
    if (!ctxs || n <= 0 || !G || !Sigma || !out) throw Error(GG_ERR_ARG, "batch: bad arguments");
    *out = nullptr;
    auto b = std::make_unique<gg_batch>();
    const int dev = ctxs[0]->device;
    GG_CUDA(cudaSetDevice(dev));
    for (int i = 0; i < n; ++i) {
      gg_context* c = ctxs[i];
      if (!c || c->device != dev) throw Error(GG_ERR_ARG, "batch: contexts must exist and share one device");
      if (c->profiling || c->cap_P0 || c->cap_Pw || c->cap_Wt)
        throw Error(GG_ERR_STATE, "batch: profiling and intermediate capture need eager builds");
      for (int j = 0; j < i; ++j)
        if (ctxs[j] == c) throw Error(GG_ERR_ARG, "batch: a context appears twice");
      b->ctx.push_back(c);
      b->G.push_back((const double2*)G[i]);
      b->S.push_back((double2*)Sigma[i]);
    }
    b->solver = solver;
    b->precision = precision;
    // eager builds: allocate every buffer and build every table, then capture all of them
    for (int i = 0; i < n; ++i) {
      try {
        gw_sequence(b->ctx[i], b->G[i], b->S[i], solver, precision, b->ctx[i]->stream);
      } catch (const Error& e) {
        throw Error(e.code, "batch system " + std::to_string(i) + ": " + e.what());
      }
    }
    GG_CUDA(cudaStreamCreateWithFlags(&b->master, cudaStreamNonBlocking));
    GG_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    b->join.resize(n, nullptr);
    for (int i = 0; i < n; ++i) GG_CUDA(cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming));
    b->exec = capture_graph(b->ctx, b->master, [&] {
      GG_CUDA(cudaEventRecord(b->fork, b->master));
      for (int i = 0; i < n; ++i) {
        cudaStream_t st = b->ctx[i]->stream;
        GG_CUDA(cudaStreamWaitEvent(st, b->fork, 0));
        gw_sequence(b->ctx[i], b->G[i], b->S[i], solver, precision, st);
        GG_CUDA(cudaEventRecord(b->join[i], st));
        GG_CUDA(cudaStreamWaitEvent(b->master, b->join[i], 0));
      }
    });
    for (auto* c : b->ctx) b->sig.push_back(c->buffer_signature());
    *out = b.release();
  });
}

int gg_batch_run(gg_batch* b, void* stream) {
  return guarded_global([&] {
    if (!b) throw Error(GG_ERR_ARG, "batch: NULL");
    GG_CUDA(cudaSetDevice(b->ctx[0]->device));
    // a member context whose buffers moved since the capture (another entry point grew them,
    // or a setter replaced its tables) would make the graph touch freed memory: refuse
    for (size_t i = 0; i < b->ctx.size(); ++i)
      if (b->ctx[i]->buffer_signature() != b->sig[i])
        throw Error(GG_ERR_STATE, "batch system " + std::to_string(i) +
                                      ": its context was changed or its buffers reallocated after the batch was "
                                      "captured; destroy the batch and create it again");
    cudaStream_t st = stream ? (cudaStream_t)stream : b->master;
    GG_CUDA(cudaGraphLaunch(b->exec, st));
    GG_CUDA(cudaStreamSynchronize(st));
    for (size_t i = 0; i < b->ctx.size(); ++i) {
      try {
        graph_check(b->ctx[i], b->solver);
      } catch (const Error& e) {
        throw Error(e.code, "batch system " + std::to_string(i) + ": " + e.what());
      }
    }
  });
}

void gg_batch_destroy(gg_batch* b) {
  if (!b) return;
  cudaSetDevice(b->ctx.empty() ? 0 : b->ctx[0]->device);
  delete b;
}

int gg_gw_sigma_device(gg_context* c, const void* G, void* Sigma, int solver, int precision, void* stream) {
  return guarded(c, [&] {
    if (!G || !Sigma) throw Error(GG_ERR_ARG, "gw: NULL buffer");
    if (((reinterpret_cast<uintptr_t>(G) | reinterpret_cast<uintptr_t>(Sigma)) & 15) != 0)
      throw Error(GG_ERR_ARG, "gw: device buffers must be 16-byte aligned");
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    gw_device(c, (const double2*)G, (double2*)Sigma, solver, precision, st);
  });
}

int gg_gw_sigma(gg_context* c, const double* G, double* Sigma, int solver, int precision) {
  return guarded(c, [&] {
    if (!G || !Sigma) throw Error(GG_ERR_ARG, "gw: NULL buffer");
    const auto& s = c->sh;
    const size_t count = (size_t)s.nts * s.ink * spin_elems(c);
    double2* gin = c->G_in.ensure(count);
    double2* sout = c->Sigma_out.ensure(count);
    cudaEvent_t e0, e1;
    GG_CUDA(cudaEventCreate(&e0));
    GG_CUDA(cudaEventCreate(&e1));
    GG_CUDA(cudaEventRecord(e0, c->stream));
    GG_CUDA(cudaMemcpyAsync(gin, G, count * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
    gw_device(c, gin, sout, solver, precision, c->stream);
    GG_CUDA(cudaMemcpyAsync(Sigma, sout, count * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
    GG_CUDA(cudaEventRecord(e1, c->stream));
    GG_CUDA(cudaStreamSynchronize(c->stream));
    float ms = 0;
    GG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    c->last.e2e = ms * 1e-3;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  });
}

// density upload (split into the aa, bb, ab blocks in X2C mode: get_dm_fbz,
// hf_gpu_kernel.cpp:326-336) and the engine's Fock buffer of hf_spins blocks
static double2* hf_upload(gg_context* c, const double* dm, double2** F_blocks) {
  const auto& s = c->sh;
  const size_t count = (size_t)s.ink * spin_elems(c);
  double2* din = c->G_in.ensure(std::max(count, c->G_in.n));
  GG_CUDA(cudaMemcpyAsync(din, dm, count * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
  const size_t nblk = (size_t)hf_spins(c) * s.ink * s.nao * s.nao;
  *F_blocks = c->hf_F.ensure(nblk);
  if (!c->x2c) return din;
  double2* d3 = c->x2c_in.ensure(std::max(nblk, c->x2c_in.n));
  launch_x2c_split(din, 1, s.ink, s.nao, 3, d3, c->stream);
  return d3;
}

// Fock blocks -> host in the caller's layout (X2C: spinor matrices, ba = ab^+,
// copy_2c_Fock_from_device_to_host in cuda_common.cu:176-201)
static void hf_download(gg_context* c, const double2* F_blocks, double* out) {
  const auto& s = c->sh;
  const size_t count = (size_t)s.ink * spin_elems(c);
  const double2* src = F_blocks;
  if (c->x2c) {
    double2* f2 = c->x2c_out.ensure(std::max(count, c->x2c_out.n));
    launch_x2c_merge(F_blocks, 1, s.ink, s.nao, 3, f2, c->stream);
    src = f2;
  }
  GG_CUDA(cudaMemcpyAsync(out, src, count * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
  GG_CUDA(cudaStreamSynchronize(c->stream));
}

int gg_hf_exchange(gg_context* c, const double* dm, double* K_out) {
  return guarded(c, [&] {
    if (!dm || !K_out) throw Error(GG_ERR_ARG, "hf: NULL buffer");
    double2* kout = nullptr;
    double2* din = hf_upload(c, dm, &kout);
    hf_exchange(c, din, kout, c->stream);
    hf_download(c, kout, K_out);
  });
}

int gg_hf_fock(gg_context* c, const double* dm, const double* S_k, double madelung, double* F_out) {
  return guarded(c, [&] {
    if (!dm || !S_k || !F_out) throw Error(GG_ERR_ARG, "hf: NULL buffer");
    const auto& s = c->sh;
    double2* fout = nullptr;
    double2* din = hf_upload(c, dm, &fout);
    hf_exchange(c, din, fout, c->stream);
    hf_direct(c, fout, c->stream);
    const size_t m = c->x2c ? 2 * (size_t)s.nao : (size_t)s.nao, mm = m * m;
    const size_t count = (size_t)s.ink * spin_elems(c);
    std::vector<double2> F(count);
    hf_download(c, fout, reinterpret_cast<double*>(F.data()));
    // Ewald on the host: F -= c * madelung * S D S per (s, IBZ k), c = 0.5 (ns = 1) or 1
    // (hf_gpu_kernel.cpp:188-201).  X2C: per spin block with the AO overlap S_aa on both
    // sides and c = 1; the ba block gets the adjoint of the ab term (hf_gpu_kernel.cpp:311-323)
    const double2* S = (const double2*)S_k;
    const double2* D = (const double2*)dm;
    const int n = s.nao;
    auto sds = [&](const double2* Sb, size_t sld, const double2* Db, size_t dld, double2* out) {
      std::vector<double2> tmp((size_t)n * n);
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
          double2 acc = make_double2(0, 0);
          for (int a = 0; a < n; ++a) acc = cadd(acc, cmul(Sb[i * sld + a], Db[a * dld + j]));
          tmp[(size_t)i * n + j] = acc;
        }
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
          double2 acc = make_double2(0, 0);
          for (int a = 0; a < n; ++a) acc = cadd(acc, cmul(tmp[(size_t)i * n + a], Sb[a * sld + j]));
          out[(size_t)i * n + j] = acc;
        }
    };
    std::vector<double2> E((size_t)n * n);
    if (!c->x2c) {
      const double pre = (s.ns == 2 ? 1.0 : 0.5) * madelung;
      for (size_t b = 0; b < (size_t)s.ns * s.ink; ++b) {
        sds(S + b * mm, m, D + b * mm, m, E.data());
        for (size_t e = 0; e < mm; ++e) F[b * mm + e] = csub(F[b * mm + e], cscale(E[e], pre));
      }
    } else {
      for (size_t k = 0; k < (size_t)s.ink; ++k) {
        const double2* Sk = S + k * mm;  // S_aa block at (0, 0), leading dimension 2 nao
        double2* Fk = F.data() + k * mm;
        const int blocks[3][2] = {{0, 0}, {1, 1}, {0, 1}};
        for (auto& bl : blocks) {
          const int a = bl[0], b = bl[1];
          sds(Sk, m, D + k * mm + (size_t)a * n * m + (size_t)b * n, m, E.data());
          for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
              const double2 v = cscale(E[(size_t)i * n + j], madelung);
              double2& f = Fk[(size_t)(a * n + i) * m + b * n + j];
              f = csub(f, v);
              if (a != b) {
                double2& g = Fk[(size_t)(n + j) * m + i];
                g = csub(g, make_double2(v.x, -v.y));
              }
            }
        }
      }
    }
    std::memcpy(F_out, F.data(), count * sizeof(double2));
  });
}

int gg_symmetry_unfold(gg_context* c, const double* X_ibz, int64_t nmat, double* X_full) {
  return guarded(c, [&] {
    if (!X_ibz || !X_full || nmat <= 0) throw Error(GG_ERR_ARG, "unfold: bad arguments");
    if (!c->has_sym) throw Error(GG_ERR_STATE, "unfold: symmetry not set");
    const auto& s = c->sh;
    const size_t nn = (size_t)s.nao * s.nao;
    const size_t in_count = (size_t)nmat * s.ink * nn, out_count = (size_t)nmat * s.nk * nn;
    DevBuf<double2> xin, xout;
    xin.upload((const double2*)X_ibz, in_count, c->stream);
    xout.ensure(out_count);
    c->Gtmp.ensure(out_count);
    unfold_matrices(c, xin.p, (int)nmat, 1, xout.p, c->stream);  // -> [k][m][n][n]
    std::vector<double2> h(out_count);
    GG_CUDA(cudaMemcpyAsync(h.data(), xout.p, out_count * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
    GG_CUDA(cudaStreamSynchronize(c->stream));
    double2* o = (double2*)X_full;
    for (int k = 0; k < s.nk; ++k)
      for (int64_t m = 0; m < nmat; ++m)
        std::memcpy(o + ((size_t)m * s.nk + k) * nn, h.data() + ((size_t)k * nmat + m) * nn, nn * sizeof(double2));
  });
}

int gg_set_fused_tail(gg_context* c, int enable) {
  return guarded(c, [&] {
    c->fused_tail = enable != 0;
    c->drop_graph();
  });
}

int gg_set_autotune(gg_context* c, int enable) {
  return guarded(c, [&] {
    split_set_autotune(split_engine(c), enable != 0);
    c->drop_graph();  // a captured graph holds the launch configurations of the old setting
  });
}

const char* gg_autotune_report(const gg_context* c) { return c ? split_autotune_report(c->split) : ""; }

int gg_arm_split_timeout_test(gg_context* c) {
  return guarded(c, [&] { split_arm_timeout_test(split_engine(c)); });
}

int gg_set_profiling(gg_context* c, int enable) {
  return guarded(c, [&] { c->profiling = enable != 0; });
}

int gg_kernel_stats(const gg_context* c, int which, int64_t* launches, double* seconds, double* flops) {
  if (!c || which < 0 || which > 2) return GG_ERR_ARG;
  if (launches) *launches = c->kstat_launches[which];
  if (seconds) *seconds = c->kstat_seconds[which];
  if (flops) *flops = c->kstat_flops[which];
  return GG_OK;
}

int64_t gg_last_launch_count(const gg_context* c) { return c ? c->launches : 0; }

int gg_zgemm(gg_context* c, int64_t M, int64_t N, int64_t K, const double* A, const double* B, double* C,
             int precision) {
  return guarded(c, [&] {
    if (!A || !B || !C || M <= 0 || N <= 0 || K <= 0) throw Error(GG_ERR_ARG, "zgemm: bad arguments");
    DevBuf<double2> a, b, o;
    a.upload((const double2*)A, (size_t)(M * K), c->stream);
    b.upload((const double2*)B, (size_t)(K * N), c->stream);
    o.ensure((size_t)(M * N));
    ZgemmDesc d;
    d.M = (int)M; d.N = (int)N; d.K = (int)K;
    d.A = a.p; d.a_m.lo = K; d.a_k = 1;
    d.B = b.p; d.b_k = N; d.b_n.lo = 1;
    d.C = o.p; d.c_m.lo = N; d.c_n.lo = 1;
    c->launches = 0;
    if (precision == GG_PREC_SPLIT) {
      c->launches += split_zgemm(split_engine(c), d, c->slices, c->stream);
      split_check(c->split, c->stream);
    } else if (precision == GG_PREC_FP64) {
      DevBuf<double2> w;
      d.work = w.ensure((size_t)1 << 20);
      d.work_elems = 1 << 20;
      c->launches += zgemm(d, c->stream);
      GG_CUDA(cudaStreamSynchronize(c->stream));
    } else {
      throw Error(GG_ERR_ARG, "zgemm: unknown precision");
    }
    GG_CUDA(cudaMemcpyAsync(C, o.p, (size_t)(M * N) * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
    GG_CUDA(cudaStreamSynchronize(c->stream));
  });
}

int gg_estimate_bytes(const gg_shape* shape, int64_t nstored, int64_t* bytes) {
  if (!shape || !bytes || nstored < 0) return GG_ERR_ARG;
  try {
    check_shape(*shape);
  } catch (const Error& e) {
    g_create_error = e.what();
    return e.code;
  }
  const auto& s = *shape;
  const double z = 16.0;
  const double nn = (double)s.nao * s.nao, NN = (double)s.NQ * s.NQ, Nnn = (double)s.NQ * nn;
  const int T2 = s.nts / 2, tb = std::min(T2, 4);
  double b = (double)nstored * Nnn;                    // V store
  b += 2.0 * s.nk * s.ns * s.nts * nn;                 // G full BZ + rotation scratch
  b += (double)s.nk * Nnn + (double)s.nk * T2 * nn;    // gathered V, G(k+q)
  b += 2.0 * std::max((double)s.nk * tb * Nnn, (double)s.nts * std::max(Nnn, NN));
  b += (double)s.inq * (T2 + s.nw_b + s.nts) * NN;     // P0, P~ / W(iW), W(tau)
  b += std::min(592.0, (double)s.inq * s.nw_b) * NN;   // Dyson work space
  b += (double)s.nts * NN + (double)(1 << 22);         // W rotation, split-K partials
  *bytes = (int64_t)(b * z);
  return GG_OK;
}

int gg_last_timings(const gg_context* c, double* out, int n) {
  if (!c || !out) return 0;
  const double v[8] = {c->last.total, c->last.unfold, c->last.p0,    c->last.ir_fwd,
                       c->last.dyson, c->last.ir_back, c->last.sigma, c->last.e2e};
  int m = std::min(n, 8);
  for (int i = 0; i < m; ++i) out[i] = v[i];
  return m;
}

}  // extern "C"
