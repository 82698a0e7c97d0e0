// Minimal stand-in for gxl_lib matrices (oracle build only), written from the
// reference's usage: Matrix<real,3,3,1> is 1-based (Mesh.cpp:262-270),
// MatrixDyn is 0-based row-major on host and device (DParameter.cu:14-40,
// Transport.cu:82-92).
#pragma once
#include <cuda_runtime.h>
#include <vector>

namespace gxl {
template <typename T, int R, int C, int base = 1>
struct Matrix {
  __host__ __device__ T &operator()(int r, int c) { return v[(r - base) * C + (c - base)]; }
  __host__ __device__ const T &operator()(int r, int c) const { return v[(r - base) * C + (c - base)]; }
  T v[R * C];
};

template <typename T>
class MatrixDyn {
 public:
  MatrixDyn() = default;
  MatrixDyn(int r, int c) { resize(r, c); }
  void resize(int r, int c) {
    r_ = r, c_ = c;
    v_.assign((size_t)r * c, T{});
  }
  T &operator()(int r, int c) { return v_[(size_t)r * c_ + c]; }
  const T &operator()(int r, int c) const { return v_[(size_t)r * c_ + c]; }
  T *data() { return v_.data(); }
  const T *data() const { return v_.data(); }
  size_t size() const { return v_.size(); }

 private:
  int r_ = 0, c_ = 0;
  std::vector<T> v_;
};
}  // namespace gxl

namespace ggxl {
template <typename T>
struct MatrixDyn {
  MatrixDyn() = default;
  __device__ MatrixDyn(int r, int c) : r_(r), c_(c) { p_ = new T[(size_t)r * c]; }
  void init_with_size(int r, int c) {
    r_ = r, c_ = c;
    cudaMalloc(&p_, (size_t)r * c * sizeof(T));
  }
  __device__ void deallocate_matrix() { delete[] p_; }
  __host__ __device__ T &operator()(int r, int c) const { return p_[(size_t)r * c_ + c]; }
  __host__ __device__ T *data() const { return p_; }
  __host__ __device__ size_t size() const { return (size_t)r_ * c_; }
  T *p_ = nullptr;
  int r_ = 0, c_ = 0;
};
}  // namespace ggxl
