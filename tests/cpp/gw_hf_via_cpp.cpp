// C++17 host program driving one GW and one HF build through include/green_b200.hpp.
// Inputs are raw little-endian files written by tests/test_cpp_host.py; outputs likewise.
#include <complex>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "green_b200.hpp"

template <typename T>
std::vector<T> load(const std::string& dir, const std::string& name) {
  std::ifstream f(dir + "/" + name, std::ios::binary | std::ios::ate);
  if (!f) throw std::runtime_error("missing " + name);
  const size_t bytes = f.tellg();
  f.seekg(0);
  std::vector<T> v(bytes / sizeof(T));
  f.read(reinterpret_cast<char*>(v.data()), bytes);
  return v;
}

template <typename T>
void save(const std::string& dir, const std::string& name, const std::vector<T>& v) {
  std::ofstream f(dir + "/" + name, std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), v.size() * sizeof(T));
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const std::string d = argv[1];
  try {
    auto dims = load<int64_t>(d, "dims.bin");  // nk ink inq nao NQ ns nts nw_b nstored
    gg_shape s{};
    s.nk = (int32_t)dims[0];
    s.ink = (int32_t)dims[1];
    s.nq = s.nk;
    s.inq = (int32_t)dims[2];
    s.nao = (int32_t)dims[3];
    s.NQ = (int32_t)dims[4];
    s.ns = (int32_t)dims[5];
    s.nts = (int32_t)dims[6];
    s.nw_b = (int32_t)dims[7];
    green::b200::context ctx(s, 0);
    ctx.set_symmetry(load<int64_t>(d, "k_f2r.bin"), load<int64_t>(d, "k_r2f.bin"), load<int64_t>(d, "k_tr.bin"),
                     load<int64_t>(d, "q_f2r.bin"), load<int64_t>(d, "q_r2f.bin"), load<int64_t>(d, "q_tr.bin"),
                     load<int64_t>(d, "k1q.bin"), load<int64_t>(d, "k2q.bin"));
    ctx.set_kpairs(dims[8], load<int64_t>(d, "conj.bin"), load<int64_t>(d, "trans.bin"), load<int64_t>(d, "pos.bin"));
    auto V = load<std::complex<double>>(d, "V.bin");
    ctx.set_coulomb(V.data());
    auto Ttn = load<std::complex<double>>(d, "Ttn.bin");
    auto Tnt = load<std::complex<double>>(d, "Tnt.bin");
    ctx.set_ir(Ttn.data(), Tnt.data());
    auto G = load<std::complex<double>>(d, "G.bin");
    std::vector<std::complex<double>> Sigma(G.size());
    ctx.gw_sigma(G.data(), Sigma.data(), GG_SOLVER_CHOLESKY, GG_PREC_FP64);
    save(d, "Sigma.bin", Sigma);
    auto dm = load<std::complex<double>>(d, "dm.bin");
    std::vector<std::complex<double>> K(dm.size());
    ctx.hf_exchange(dm.data(), K.data());
    save(d, "K.bin", K);
    // errors surface as exceptions with the library's status code
    try {
      ctx.set_split_slices(1);
      return 3;
    } catch (const green::b200::error& e) {
      if (e.code() != GG_ERR_ARG) return 4;
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
