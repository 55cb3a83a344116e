// Per-system device state behind the opaque gg_context of the C ABI.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "common.cuh"

namespace gg {

struct SplitGemm;
void split_release(SplitGemm* e);

// grow-only device buffer
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  T* ensure(size_t count) {
    if (count > n) {
      release();
      if (count) GG_CUDA(cudaMalloc((void**)&p, count * sizeof(T)));
      n = count;
    }
    return p;
  }
  void upload(const T* host, size_t count, cudaStream_t st) {
    ensure(count);
    if (count) GG_CUDA(cudaMemcpyAsync(p, host, count * sizeof(T), cudaMemcpyHostToDevice, st));
  }
};

struct Plan {
  int qc = 1;   // irreducible q points per chunk
  int kc = 1;   // k points per P0 chunk
  int tb = 1;   // tau points per P0 batch
  int dyson_batch = 1;  // Dyson systems per launch
  size_t bytes = 0;
};

struct Timings {
  double total = 0, unfold = 0, p0 = 0, ir_fwd = 0, dyson = 0, ir_back = 0, sigma = 0, e2e = 0;
};

}  // namespace gg

struct gg_context {
  gg_shape sh{};
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;

  // symmetry (host copies + device copies of what kernels index)
  bool has_sym = false;
  std::vector<int64_t> k_f2r, k_r2f, k_tr, q_f2r, q_r2f, q_tr, k1_from_k2q, k2_from_k1q;
  std::vector<std::vector<int>> k_stars, q_stars;
  bool has_Uk = false, has_Uq = false;
  gg::DevBuf<double2> Uk, Uq;
  std::vector<double2> Uk_h;
  gg::DevBuf<int> k_f2r_d, k_tr_d;

  // k-pair store
  bool has_kpairs = false;
  int64_t nstored = 0;
  std::vector<int64_t> conj_list, trans_list, irre_pos;
  const double2* V = nullptr;  // device
  gg::DevBuf<double2> V_owned;

  // IR transforms
  bool has_ir = false;
  gg::DevBuf<double2> Ttn, Tnt_fold;

  int slices = GG_DEFAULT_SPLIT_SLICES;
  // Sigma tail X G -> Z V^+ as one kernel (where the orbital count allows) instead of two GEMMs;
  // off by default: on B200 both forms are bound by the DMMA issue rate and the fused kernel
  // measured 4 % slower at nao 52, NQ 400
  int fused_tail = 0;
  int hf_precision = GG_PREC_FP64;
  // two-component (X2C) mode: inputs and outputs are spinor matrices of order 2 nao; GW runs
  // on the four spin blocks as pseudo-spins (aa, bb, ab, ba), HF on three (aa, bb, ab)
  int x2c = 0;
  gg::DevBuf<double2> x2c_in, x2c_out;
  int shard_rank = 0, shard_size = 1;

  // capture of intermediates (host pointers)
  double* cap_P0 = nullptr;
  double* cap_Pw = nullptr;
  double* cap_Wt = nullptr;

  // work buffers
  gg::DevBuf<double2> G_in, Sigma_out, Gf, Gtmp, Vbuf, G1buf, scratchA, scratchB, P0buf, Pw, Afac, Wt, Wrot,
      gemm_work, hf_D, hf_F, hf_c, hf_J;
  gg::DevBuf<int> info, piv, idx_i;
  // split precision: exponents of the P0 main contraction's operand rows / columns, recorded
  // by the operand builds' epilogues
  gg::DevBuf<int> p0_ea, p0_eb;
  gg::DevBuf<int64_t> pos_d;
  gg::DevBuf<int> op_d;

  gg::Timings last{};
  long launches = 0;
  bool profiling = false;
  // per-kernel stats of the last build: [0] P0 contraction, [1] Sigma contraction
  long kstat_launches[3] = {0, 0, 0};
  double kstat_seconds[3] = {0, 0, 0};
  double kstat_flops[3] = {0, 0, 0};

  gg::SplitGemm* split = nullptr;

  // tables of one GW build (pair positions and ops, G block indices), built on the first build
  // after the symmetry, k-pairs or spin layout changed
  std::shared_ptr<void> gw_tables;
  // graph mode: the first build runs eagerly, the second is captured into a CUDA graph that
  // later builds replay while inputs, buffers and settings match (any setter drops it)
  bool graph_mode = false;
  bool capturing = false;  // true while gw_build is being captured: no host syncs, no timers
  cudaGraphExec_t graph_exec = nullptr;
  const void* graph_G = nullptr;
  void* graph_S = nullptr;
  int graph_solver = -1, graph_prec = -1;
  cudaStream_t graph_stream = nullptr;
  // device addresses of every work buffer when the graph was captured: an entry point that
  // grows a shared buffer (HF, unfold, zgemm) reallocates it, and the graph is then rebuilt
  std::vector<const void*> graph_sig;
  gg::DevBuf<int> gw_err;  // [0] failed, [1] system index (q position x nw_b + Omega), [2] info
  int plan_qc = 0, plan_kc = 0, plan_tb = 0;  // plan of the eager build, reused by the capture

  void drop_graph() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    graph_exec = nullptr;
    graph_G = nullptr;
    graph_S = nullptr;
    graph_sig.clear();
  }
  // addresses of all device buffers a GW build reads or writes (capi.cu)
  std::vector<const void*> buffer_signature() const;
  void invalidate() {
    gw_tables.reset();
    drop_graph();
  }

  ~gg_context() {
    drop_graph();
    if (split) gg::split_release(split);
    if (stream) cudaStreamDestroy(stream);
  }
};
