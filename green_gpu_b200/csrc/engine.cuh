// Host orchestration entry points used by the C ABI (capi.cu).
#pragma once

#include "context.cuh"

namespace gg {

Plan plan_gw(gg_context* c, int slices);
// spin blocks the GW / HF engines loop over: ns, or the X2C pseudo-spins (4 for GW, 3 for HF)
int gw_spins(const gg_context* c);
// irreducible q points of shard `rank` of `size`: iq = rank, rank + size, ... (cugw_utils.cu:115)
std::vector<int> shard_q_points(int inq, int rank, int size);
int hf_spins(const gg_context* c);
// X2C needs the identity k/q symmetry (no rotations, no time-reversal partners): the spinor
// transformation of G under a space-group or time-reversal operation is not applied here
void x2c_check(const gg_context* c);
// throws the Dyson failure of `system` (q position in the shard x nw_b + Omega)
void dyson_failure(const gg_context* c, int solver, int system, int info);
void gw_build(gg_context* c, const double2* G_dev, double2* Sigma_dev, int solver, int precision, cudaStream_t st);
void hf_exchange(gg_context* c, const double2* dm_dev, double2* K_dev, cudaStream_t st);
void hf_direct(gg_context* c, double2* F_dev, cudaStream_t st);
void unfold_matrices(gg_context* c, const double2* X_in, int nouter, int ns, double2* out, cudaStream_t st);
void kpair_op(const gg_context* c, int k1, int k2, int64_t* pos, int* op);

}  // namespace gg
