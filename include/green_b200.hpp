// C++17 RAII wrapper over the C ABI of libgreen_b200.so (include/green_b200.h).
// Status codes become green::b200::error exceptions on the C++ side of the boundary.
#ifndef GREEN_B200_HPP
#define GREEN_B200_HPP

#include <complex>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "green_b200.h"

namespace green::b200 {

class error : public std::runtime_error {
public:
  error(int code, const std::string& msg) : std::runtime_error(msg), code_(code) {}
  int code() const noexcept { return code_; }

private:
  int code_;
};

using cplx = std::complex<double>;

class context {
public:
  context(const gg_shape& shape, int device = 0) {
    int rc = gg_create(&shape, device, &h_);
    if (rc != GG_OK) throw error(rc, gg_last_error(nullptr));
  }
  ~context() { gg_destroy(h_); }
  context(const context&) = delete;
  context& operator=(const context&) = delete;
  context(context&& o) noexcept : h_(o.h_) { o.h_ = nullptr; }

  gg_context* handle() const { return h_; }

  void set_symmetry(const std::vector<int64_t>& k_f2r, const std::vector<int64_t>& k_r2f,
                    const std::vector<int64_t>& k_tr, const std::vector<int64_t>& q_f2r,
                    const std::vector<int64_t>& q_r2f, const std::vector<int64_t>& q_tr,
                    const std::vector<int64_t>& k1_from_k2q, const std::vector<int64_t>& k2_from_k1q,
                    const cplx* U_k = nullptr, const cplx* U_q = nullptr) {
    check(gg_set_symmetry(h_, k_f2r.data(), k_r2f.data(), k_tr.data(), q_f2r.data(), q_r2f.data(), q_tr.data(),
                          k1_from_k2q.data(), k2_from_k1q.data(), reinterpret_cast<const double*>(U_k),
                          reinterpret_cast<const double*>(U_q)));
  }
  void set_kpairs(int64_t nstored, const std::vector<int64_t>& conj_list, const std::vector<int64_t>& trans_list,
                  const std::vector<int64_t>& irre_pos) {
    check(gg_set_kpairs(h_, nstored, conj_list.data(), trans_list.data(), irre_pos.data()));
  }
  void set_coulomb(const cplx* V) { check(gg_set_coulomb(h_, reinterpret_cast<const double*>(V))); }
  void set_ir(const cplx* Ttn_FB, const cplx* Tnt_BF) {
    check(gg_set_ir(h_, reinterpret_cast<const double*>(Ttn_FB), reinterpret_cast<const double*>(Tnt_BF)));
  }
  void set_split_slices(int s) { check(gg_set_split_slices(h_, s)); }
  void set_x2c(bool on) { check(gg_set_x2c(h_, on ? 1 : 0)); }
  void set_q_shard(int rank, int size) { check(gg_set_q_shard(h_, rank, size)); }
  void gw_sigma(const cplx* G, cplx* Sigma, int solver = GG_SOLVER_CHOLESKY, int precision = GG_PREC_FP64) {
    check(gg_gw_sigma(h_, reinterpret_cast<const double*>(G), reinterpret_cast<double*>(Sigma), solver, precision));
  }
  void hf_exchange(const cplx* dm, cplx* K) {
    check(gg_hf_exchange(h_, reinterpret_cast<const double*>(dm), reinterpret_cast<double*>(K)));
  }
  void hf_fock(const cplx* dm, const cplx* S_k, double madelung, cplx* F) {
    check(gg_hf_fock(h_, reinterpret_cast<const double*>(dm), reinterpret_cast<const double*>(S_k), madelung,
                     reinterpret_cast<double*>(F)));
  }

private:
  void check(int rc) const {
    if (rc != GG_OK) throw error(rc, gg_last_error(h_));
  }
  gg_context* h_ = nullptr;
};

}  // namespace green::b200

#endif  // GREEN_B200_HPP
