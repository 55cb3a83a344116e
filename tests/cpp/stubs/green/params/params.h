// Stand-in for green-params with the uses of green-gpu's plugin code: p["name"] converts to the
// parameter's type or gives it through as<T>() (gw_gpu_kernel.h:62-65, gpu_kernel.h:45-47),
// and define<T>(name, help[, default]) (gpu_factory.h:95-102).  Declarations only.
#pragma once
#include <string>
namespace green::params {
class params_item {
 public:
  template <typename T>
  T as() const;
  template <typename T>
  operator T() const;
};
class params {
 public:
  params_item operator[](const std::string& name) const;
  template <typename T>
  void define(const std::string& name, const std::string& help);
  template <typename T>
  void define(const std::string& name, const std::string& help, const T& value);
};
}  // namespace green::params
