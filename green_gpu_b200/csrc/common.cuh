// Shared helpers for the green-b200 CUDA sources: complex arithmetic on double2,
// error propagation and the status codes of the C ABI (include/green_b200.h).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <stdexcept>
#include <string>

#include "../../include/green_b200.h"

namespace gg {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define GG_CUDA(call)                                                                          \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess)                                                                     \
      throw ::gg::Error(GG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_) +      \
                                         " (" + __FILE__ + ":" + std::to_string(__LINE__) + ")"); \
  } while (0)

#define GG_CHECK_LAUNCH() GG_CUDA(cudaGetLastError())

__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// a * conj(b)
__host__ __device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

inline int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }

// message returned by gg_last_error(NULL) on this thread (capi.cu)
void set_thread_error(const std::string& msg);

// number of SMs of the current device, looked up once per device (zgemm.cu)
int device_sm_count();
// index of the current device, checked against the per-device caches' capacity (zgemm.cu)
constexpr int kMaxDevices = 64;
int current_device();

}  // namespace gg
