// Stand-in for green-ndarray: a dense D-dimensional array with data().  Compile check only.
#pragma once
#include <cstddef>
#include <vector>
namespace green::ndarray {
template <typename T, size_t D>
class ndarray {
 public:
  template <typename... I>
  explicit ndarray(I... n) : d_((static_cast<size_t>(n) * ...)) {}
  T* data() { return d_.data(); }
  const T* data() const { return d_.data(); }

 private:
  std::vector<T> d_;
};
}  // namespace green::ndarray
