// Stand-in for green-symmetry's brillouin_zone_utils with the uses in green-gpu:
// make_cu_symmetry_data (gw_gpu_kernel.cpp:34-91) and the integral store's k-pair lists
// (df_integral_t.h:74-102), element types as cu_symmetry.h:45-57 stores them.  Declarations only.
#pragma once
#include <Eigen/Dense>
#include <complex>
#include <cstddef>
#include <vector>
namespace green::symmetry {
using row_matrix = Eigen::Matrix<std::complex<double>, Eigen::Dynamic, Eigen::Dynamic, Eigen::RowMajor>;
class k_symmetry_t {
 public:
  const std::vector<size_t>& full_to_reduced() const;
  const std::vector<size_t>& reduced_to_full() const;
  const std::vector<long>& tr_conj_list() const;
  std::vector<long> star(size_t ik) const;
  void k_sym_transform_ao(row_matrix& U, size_t k) const;
  const std::vector<long>& conj_kpair_list() const;
  const std::vector<long>& trans_kpair_list() const;
  long irre_pos_kpair(size_t idx) const;
  size_t num_kpair_stored() const;
};
class q_symmetry_t {
 public:
  const std::vector<size_t>& full_to_reduced() const;
  const std::vector<size_t>& reduced_to_full() const;
  const std::vector<long>& tr_conj_list() const;
  std::vector<long> star(size_t iq) const;
  void q_sym_transform_p0(row_matrix& U, size_t q) const;
};
class k_q_map_t {
 public:
  size_t k1_from_k2q(size_t k2, size_t q) const;
  size_t k2_from_k1q(size_t k1, size_t q) const;
};
class brillouin_zone_utils {
 public:
  size_t nk() const;
  size_t ink() const;
  size_t nq() const;
  size_t inq() const;
  const k_symmetry_t& k_symmetry() const;
  const q_symmetry_t& q_symmetry() const;
  const k_q_map_t& k_q_map() const;
};
}  // namespace green::symmetry
