// Drop-in replacement of green-gpu's plugin header for green-mbpt, backed by
// libgreen_b200.so.  Same namespace (green::gpu), same factory functions and signatures
// as src/green/gpu/gpu_factory.h:47-102 of the reference; the kernel objects forward to
// the C ABI (include/green_b200.h) through the RAII wrapper (include/green_b200.hpp).
//
// Build inside green-mbpt (needs the green-* headers, MPI and HDF5 that green-mbpt uses):
//   init_kernel("GPU" "GREEN::GPU" "<green/gpu/gpu_factory.h>" "green::gpu")
// with include path <this repo>/include and link to libgreen_b200.so.
#ifndef GREEN_GPU_FACTORY_H
#define GREEN_GPU_FACTORY_H

#include <Eigen/Dense>
#include <hdf5.h>
#include <hdf5_hl.h>

#include <complex>
#include <cstring>
#include <functional>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include <green/grids/transformer_t.h>
#include <green/ndarray/ndarray.h>
#include <green/params/params.h>
#include <green/symmetry/symmetry.h>
#include <green/utils/mpi_shared.h>
#include <green/utils/mpi_utils.h>

#include "../../green_b200.hpp"

namespace green::gpu {

  // common_defs.h:137-139
  enum class LinearSolverType { Cholesky, LU };

  template <size_t D>
  using ztensor = green::ndarray::ndarray<std::complex<double>, D>;
  using bz_utils_t = symmetry::brillouin_zone_utils;
  using x_type     = ztensor<4>;
  using G_type     = utils::shared_object<ztensor<5>>;

  namespace detail {
    // symmetry tables exactly as make_cu_symmetry_data builds them (gw_gpu_kernel.cpp:34-91)
    // x2c: the spinor transformations are not applied (gg_set_x2c accepts only the identity
    // symmetry), so no U_k / U_q are uploaded
    inline void set_symmetry(green::b200::context& ctx, const bz_utils_t& bz, size_t nao, size_t NQ, bool with_uq,
                             bool x2c = false) {
      const auto& ks = bz.k_symmetry();
      const auto& qs = bz.q_symmetry();
      const auto& kq = bz.k_q_map();
      const size_t nk = bz.nk(), nq = bz.nq();
      auto to64 = [](const auto& v) { return std::vector<int64_t>(v.begin(), v.end()); };
      std::vector<int64_t> k1(nk * nq), k2(nk * nq);
      for (size_t k = 0; k < nk; ++k)
        for (size_t q = 0; q < nq; ++q) {
          k1[k * nq + q] = kq.k1_from_k2q(k, q);
          k2[k * nq + q] = kq.k2_from_k1q(k, q);
        }
      std::vector<std::complex<double>> Uk(nk * nao * nao), Uq;
      Eigen::Matrix<std::complex<double>, Eigen::Dynamic, Eigen::Dynamic, Eigen::RowMajor> U(nao, nao);
      for (size_t k = 0; k < nk; ++k) {
        ks.k_sym_transform_ao(U, k);
        std::memcpy(Uk.data() + k * nao * nao, U.data(), nao * nao * sizeof(std::complex<double>));
      }
      if (with_uq) {
        Uq.resize(nq * NQ * NQ);
        Eigen::Matrix<std::complex<double>, Eigen::Dynamic, Eigen::Dynamic, Eigen::RowMajor> W(NQ, NQ);
        for (size_t q = 0; q < nq; ++q) {
          qs.q_sym_transform_p0(W, q);
          std::memcpy(Uq.data() + q * NQ * NQ, W.data(), NQ * NQ * sizeof(std::complex<double>));
        }
      }
      ctx.set_symmetry(to64(ks.full_to_reduced()), to64(ks.reduced_to_full()), to64(ks.tr_conj_list()),
                       to64(qs.full_to_reduced()), to64(qs.reduced_to_full()), to64(qs.tr_conj_list()), k1, k2,
                       x2c ? nullptr : Uk.data(), (with_uq && !x2c) ? Uq.data() : nullptr);
      const size_t npairs = nk * (nk + 1) / 2;
      std::vector<int64_t> conj(npairs), trans(npairs), pos(npairs);
      for (size_t i = 0; i < npairs; ++i) {
        conj[i]  = ks.conj_kpair_list()[i];
        trans[i] = ks.trans_kpair_list()[i];
        pos[i]   = (conj[i] == (int64_t)i && trans[i] == (int64_t)i) ? ks.irre_pos_kpair(i) : -1;
      }
      ctx.set_kpairs(ks.num_kpair_stored(), conj, trans, pos);
    }

    // df_integral_t::read_entire (df_integral_t.h:96-129): all VQ_<c>.h5 chunks of `path`
    inline std::vector<std::complex<double>> read_integrals(const std::string& path, size_t nstored, size_t nao,
                                                            size_t NQ) {
      long  chunk = 0;
      hid_t meta  = H5Fopen((path + "/meta.h5").c_str(), H5F_ACC_RDONLY, H5P_DEFAULT);
      if (meta < 0 || H5LTread_dataset_long(meta, "chunk_size", &chunk) < 0)
        throw std::runtime_error("green-b200: cannot read " + path + "/meta.h5:chunk_size");
      H5Fclose(meta);
      const size_t per = NQ * nao * nao;
      std::vector<std::complex<double>> V(nstored * per);
      for (size_t c = 0; c < nstored; c += chunk) {
        const std::string fn = path + "/VQ_" + std::to_string(c) + ".h5";
        hid_t f = H5Fopen(fn.c_str(), H5F_ACC_RDONLY, H5P_DEFAULT);
        if (f < 0) throw std::runtime_error("green-b200: cannot open " + fn);
        const size_t n = std::min<size_t>(chunk, nstored - c);
        std::vector<std::complex<double>> buf(chunk * per);
        if (H5LTread_dataset_double(f, ("/" + std::to_string(c)).c_str(), reinterpret_cast<double*>(buf.data())) < 0)
          throw std::runtime_error("green-b200: failure reading " + fn);
        H5Fclose(f);
        std::memcpy(V.data() + c * per, buf.data(), n * per * sizeof(std::complex<double>));
      }
      return V;
    }

    inline gg_shape shape(const bz_utils_t& bz, size_t nao, size_t NQ, size_t ns, size_t nts, size_t nw_b) {
      gg_shape s{};
      s.nk  = (int32_t)bz.nk();
      s.ink = (int32_t)bz.ink();
      s.nq  = (int32_t)bz.nq();
      s.inq = (int32_t)bz.inq();
      s.nao = (int32_t)nao;
      s.NQ  = (int32_t)NQ;
      s.ns  = (int32_t)ns;
      s.nts = (int32_t)nts;
      s.nw_b = (int32_t)nw_b;
      return s;
    }
  }  // namespace detail

  // hf_gpu_kernel::solve (hf_gpu_kernel.cpp:66-104): returns exchange + direct - Ewald
  class scalar_hf_gpu_kernel {
  public:
    // x2c = true is x2c_hf_gpu_kernel (hf_gpu_kernel.h:68-100): nso = 2 nao, ns = 1
    scalar_hf_gpu_kernel(const params::params& p, size_t nao, size_t nso, size_t ns, size_t NQ, double madelung,
                         const bz_utils_t& bz, const ztensor<4>& S_k, bool x2c = false) :
        _ctx(detail::shape(bz, nao, NQ, ns, 4, 0)), _madelung(madelung), _S_k(S_k), _ns(ns), _ink(bz.ink()), _nso(nso) {
      detail::set_symmetry(_ctx, bz, nao, NQ, false, x2c);
      if (x2c) _ctx.set_x2c(true);
      auto V = detail::read_integrals(p["dfintegral_hf_file"], bz.k_symmetry().num_kpair_stored(), nao, NQ);
      _ctx.set_coulomb(V.data());
    }
    ztensor<4> solve(const ztensor<4>& dm) {
      ztensor<4> F(_ns, _ink, _nso, _nso);
      _ctx.hf_fock(dm.data(), _S_k.data(), _madelung, F.data());
      return F;
    }

  private:
    green::b200::context _ctx;
    double               _madelung;
    const ztensor<4>&    _S_k;
    size_t               _ns, _ink, _nso;
  };

  // gw_gpu_kernel::solve (gw_gpu_kernel.cpp:163-205): overwrites sigma with Sigma(tau)
  class scalar_gw_gpu_kernel {
  public:
    // x2c = true is x2c_gw_gpu_kernel (gw_gpu_kernel.h:131-206): nso = 2 nao, ns = 1
    scalar_gw_gpu_kernel(const params::params& p, size_t nao, [[maybe_unused]] size_t nso, size_t ns, size_t NQ,
                         const grids::transformer_t& ft, const bz_utils_t& bz, LinearSolverType solver,
                         [[maybe_unused]] int verbose = 1, bool x2c = false) :
        _ctx(detail::shape(bz, nao, NQ, ns, ft.sd().repn_fermi().nts(), ft.sd().repn_bose().nw())),
        _solver(solver == LinearSolverType::Cholesky ? GG_SOLVER_CHOLESKY : GG_SOLVER_LU),
        _precision((p["P_sp"].as<bool>() && p["Sigma_sp"].as<bool>()) ? GG_PREC_SPLIT : GG_PREC_FP64) {
      if (ft.sd().repn_fermi().nts() % 2 != 0) throw std::runtime_error("Number of tau points should be even number");
      detail::set_symmetry(_ctx, bz, nao, NQ, true, x2c);
      if (x2c) _ctx.set_x2c(true);
      auto V = detail::read_integrals(p["dfintegral_file"], bz.k_symmetry().num_kpair_stored(), nao, NQ);
      _ctx.set_coulomb(V.data());
      _ctx.set_ir(ft.Ttn_FB().data(), ft.Tnt_BF().data());
      // P_sp && Sigma_sp: five Ozaki slices keep Sigma within 1e-8 of the FP64 path
      _ctx.set_split_slices(GG_DEFAULT_SPLIT_SLICES);
    }
    void solve(G_type& g, G_type& sigma) {
      sigma.fence();
      if (!utils::context().node_rank) _ctx.gw_sigma(g.object().data(), sigma.object().data(), _solver, _precision);
      sigma.fence();
    }

  private:
    green::b200::context _ctx;
    int                  _solver, _precision;
  };

  inline std::tuple<std::shared_ptr<void>, std::function<x_type(const x_type&)>> custom_hf_kernel(
      bool X2C, const params::params& p, size_t nao, size_t nso, size_t ns, size_t NQ, double madelung,
      const bz_utils_t& bz_utils, const ztensor<4>& S_k) {
    std::shared_ptr<void> kernel(new scalar_hf_gpu_kernel(p, nao, nso, ns, NQ, madelung, bz_utils, S_k, X2C));
    std::function<x_type(const x_type&)> callback = [kernel](const x_type& dm) -> x_type {
      return static_cast<scalar_hf_gpu_kernel*>(kernel.get())->solve(dm);
    };
    return std::tuple{kernel, callback};
  }

  inline std::tuple<std::shared_ptr<void>, std::function<void(G_type&, G_type&)>> custom_gw_kernel(
      bool X2C, const params::params& p, size_t nao, size_t nso, size_t ns, size_t NQ, const grids::transformer_t& ft,
      const bz_utils_t& bz_utils, [[maybe_unused]] const ztensor<4>& S_k) {
    std::shared_ptr<void> kernel(
        new scalar_gw_gpu_kernel(p, nao, nso, ns, NQ, ft, bz_utils, p["cuda_linear_solver"], p["verbose"], X2C));
    std::function<void(G_type&, G_type&)> callback = [kernel](G_type& g, G_type& s) {
      static_cast<scalar_gw_gpu_kernel*>(kernel.get())->solve(g, s);
    };
    return std::tuple{kernel, callback};
  }

  // gpu_factory.h:95-102: same names, types and defaults
  inline void custom_kernel_parameters(params::params& p) {
    p.define<int>("verbose", "Print verbose output.", 0);
    p.define<LinearSolverType>("cuda_linear_solver", "Type of linear solver for Bethe-Salpeter equation (LU or Cholesky).",
                               LinearSolverType::LU);
    p.define<bool>("cuda_low_gpu_memory", "GPU Device has small amount of memory");
    p.define<bool>("cuda_low_cpu_memory", "Host has small amount of memory, we will read Coulomb integrals in chunks");
    p.define<size_t>("nt_batch", "Size of tau batch in cuda GW solver; if set to 0; value will be determined to maximize performance", 0);
  }

}  // namespace green::gpu

#endif  // GREEN_GPU_FACTORY_H
