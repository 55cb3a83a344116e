// Compiles the green-mbpt drop-in header (include/green/gpu/gpu_factory.h) against stand-ins
// for the green-* libraries, HDF5 and Eigen (tests/cpp/stubs), which declare what green-gpu's
// own plugin code uses of them.  Taking the factory functions' addresses makes the compiler
// check every call the drop-in makes into the C++ wrapper (include/green_b200.hpp).
#include <green/gpu/gpu_factory.h>

namespace {
[[maybe_unused]] auto hf_factory = &green::gpu::custom_hf_kernel;
[[maybe_unused]] auto gw_factory = &green::gpu::custom_gw_kernel;
[[maybe_unused]] auto parameters = &green::gpu::custom_kernel_parameters;
}  // namespace
