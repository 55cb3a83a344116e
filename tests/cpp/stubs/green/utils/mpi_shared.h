// Stand-in for green-utils' MPI shared-memory object: object() and fence(), as
// gw_gpu_kernel.cpp:168 and :469 use them.  Declarations only.
#pragma once
namespace green::utils {
template <typename T>
class shared_object {
 public:
  T& object();
  const T& object() const;
  void fence();
};
}  // namespace green::utils
