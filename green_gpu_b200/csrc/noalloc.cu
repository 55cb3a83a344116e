// gg_zgemm_noalloc: the FP64 complex GEMM with its split-K scratch in a static device array.
//
// Who needs it: programs that are not allowed to allocate device memory at the point where
// they want a contraction - services whose device memory is owned by another allocator (a
// caching pool that must not be bypassed, or a memory budget fixed at start-up), and
// latency-critical loops where cudaMalloc / cudaFree would synchronise the device and stall
// other streams.  They pass device buffers for A, B and C; everything else this entry point
// needs lives in `g_noalloc_scratch`, which every GPU that loads the library keeps until the
// process exits.  The array's device address is looked up once per device, on the first
// call there (cudaGetSymbolAddress with that device current); a cudaDeviceReset discards the
// module and with it that address, so the entry point must not be called again on a device
// that was reset in the same process.
#include <mutex>

#include "common.cuh"
#include "zgemm.cuh"

namespace {

// 16 MiB of split-K partial sums per device: 2^20 complex numbers.
constexpr long kScratchElems = 1L << 20;
static __device__ __align__(256) double2 g_noalloc_scratch[kScratchElems];

std::mutex g_mu;
double2* g_scratch_ptr[gg::kMaxDevices] = {};

// device address of the scratch on the current device, looked up once per device
double2* scratch_for_current_device() {
  const int dev = gg::current_device();
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev]) {
    double2* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      throw gg::Error(GG_ERR_CUDA, std::string("zgemm_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = p;
  }
  return g_scratch_ptr[dev];
}

}  // namespace

extern "C" int gg_zgemm_noalloc(int64_t M, int64_t N, int64_t K, const void* A, const void* B, void* C, void* stream) {
  try {
    if (!A || !B || !C || M <= 0 || N <= 0 || K <= 0)
      throw gg::Error(GG_ERR_ARG, "zgemm_noalloc: NULL buffer or non-positive size");
    if (M > 0x7fffffffL || N > 0x7fffffffL || K > 0x7fffffffL)
      throw gg::Error(GG_ERR_ARG, "zgemm_noalloc: dimension does not fit a 32-bit int");
    if (M * N > kScratchElems / 2)
      throw gg::Error(GG_ERR_ARG, "zgemm_noalloc: M*N = " + std::to_string(M * N) +
                                      " exceeds the limit of " + std::to_string(kScratchElems / 2) +
                                      " (half of the 2^20-element static scratch)");
    if (((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B) | reinterpret_cast<uintptr_t>(C)) & 15) != 0)
      throw gg::Error(GG_ERR_ARG, "zgemm_noalloc: buffers must be 16-byte aligned");
    double2* scratch = scratch_for_current_device();
    gg::ZgemmDesc d;
    d.M = (int)M;
    d.N = (int)N;
    d.K = (int)K;
    d.A = static_cast<const double2*>(A);
    d.a_m.lo = K;
    d.a_k = 1;
    d.B = static_cast<const double2*>(B);
    d.b_k = N;
    d.b_n.lo = 1;
    d.C = static_cast<double2*>(C);
    d.c_m.lo = N;
    d.c_n.lo = 1;
    d.work = scratch;
    d.work_elems = kScratchElems;
    gg::zgemm(d, static_cast<cudaStream_t>(stream));
    gg::set_thread_error("");
    return GG_OK;
  } catch (const gg::Error& e) {
    gg::set_thread_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    gg::set_thread_error(e.what());
    return GG_ERR_INTERNAL;
  }
}
