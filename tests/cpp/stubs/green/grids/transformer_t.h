// Stand-in for green-grids' transformer_t with the uses in green-gpu: ft.sd().repn_fermi().nts(),
// ft.sd().repn_bose().nw() (gw_gpu_kernel.h:62-64) and the row-major IR matrices Ttn_FB / Tnt_BF
// (gw_gpu_kernel.cpp:303, cugw_utils.cu:29-33).  Declarations only.
#pragma once
#include <Eigen/Dense>
#include <complex>
#include <cstddef>
namespace green::grids {
struct ir_representation {
  size_t nts() const;
  size_t nw() const;
  size_t ni() const;
};
struct sparse_data {
  const ir_representation& repn_fermi() const;
  const ir_representation& repn_bose() const;
};
class transformer_t {
 public:
  using matrix = Eigen::Matrix<std::complex<double>, Eigen::Dynamic, Eigen::Dynamic, Eigen::RowMajor>;
  const sparse_data& sd() const;
  const matrix& Ttn_FB() const;
  const matrix& Tnt_BF() const;
};
}  // namespace green::grids
