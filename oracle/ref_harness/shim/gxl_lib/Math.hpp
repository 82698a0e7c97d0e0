// gxl::sgn stand-in (oracle build only): -1, 0 or +1.
#pragma once
#include <cuda_runtime.h>
namespace gxl {
template <typename T>
__host__ __device__ inline int sgn(T a) {
  return (T(0) < a) - (a < T(0));
}
}  // namespace gxl
