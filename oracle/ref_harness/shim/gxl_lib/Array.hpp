// Minimal stand-in for the reference's un-vendored gxl_lib containers, written
// from how the reference uses them (Field.h, Mesh.h, Field.cu:90-148).  Oracle
// build only.  Layout: i fastest with ngg ghost layers; VectorField3D keeps the
// component index l fastest (Driver.cu:341-344 reads bv_last as idx*N+l).
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <vector>

namespace gxl {
template <typename T>
class Array3D {
 public:
  Array3D() = default;
  Array3D(int mx, int my, int mz, int ngg) { resize(mx, my, mz, ngg); }
  void resize(int mx, int my, int mz, int ngg) {
    mx_ = mx, my_ = my, mz_ = mz, ng_ = ngg;
    nx_ = mx + 2 * ngg, ny_ = my + 2 * ngg, nz_ = mz + 2 * ngg;
    v_.assign((size_t)nx_ * ny_ * nz_, T{});
  }
  T &operator()(int i, int j, int k) { return v_[idx(i, j, k)]; }
  const T &operator()(int i, int j, int k) const { return v_[idx(i, j, k)]; }
  T *data() { return v_.data(); }
  const T *data() const { return v_.data(); }
  size_t size() const { return v_.size(); }
  auto begin() { return v_.begin(); }
  auto end() { return v_.end(); }

 private:
  size_t idx(int i, int j, int k) const {
    return (size_t)(i + ng_) + (size_t)nx_ * ((size_t)(j + ng_) + (size_t)ny_ * (size_t)(k + ng_));
  }
  int mx_ = 0, my_ = 0, mz_ = 0, ng_ = 0, nx_ = 0, ny_ = 0, nz_ = 0;
  std::vector<T> v_;
};

template <typename T>
class VectorField3D {
 public:
  VectorField3D() = default;
  void resize(int mx, int my, int mz, int nl, int ngg) {
    ng_ = ngg, nl_ = nl, nx_ = mx + 2 * ngg, ny_ = my + 2 * ngg, nz_ = mz + 2 * ngg;
    sz = (size_t)nx_ * ny_ * nz_ * nl;
    v_.assign(sz, T{});
  }
  T &operator()(int i, int j, int k, int l) { return v_[idx(i, j, k) * nl_ + l]; }
  const T &operator()(int i, int j, int k, int l) const { return v_[idx(i, j, k) * nl_ + l]; }
  T *data() { return v_.data(); }
  const T *data() const { return v_.data(); }
  size_t sz = 0;

 private:
  size_t idx(int i, int j, int k) const {
    return (size_t)(i + ng_) + (size_t)nx_ * ((size_t)(j + ng_) + (size_t)ny_ * (size_t)(k + ng_));
  }
  int ng_ = 0, nl_ = 0, nx_ = 0, ny_ = 0, nz_ = 0;
  std::vector<T> v_;
};
}  // namespace gxl

namespace ggxl {
template <typename T>
struct Array3D {
  void allocate_memory(int mx, int my, int mz, int ngg) {
    ng_ = ngg, nx_ = mx + 2 * ngg, ny_ = my + 2 * ngg, nz_ = mz + 2 * ngg;
    n_ = (size_t)nx_ * ny_ * nz_;
    cudaMalloc(&p_, n_ * sizeof(T));
    cudaMemset(p_, 0, n_ * sizeof(T));
  }
  __host__ __device__ T &operator()(int i, int j, int k) const {
    return p_[(size_t)(i + ng_) + (size_t)nx_ * ((size_t)(j + ng_) + (size_t)ny_ * (size_t)(k + ng_))];
  }
  __host__ __device__ T *data() const { return p_; }
  __host__ __device__ size_t size() const { return n_; }
  T *p_ = nullptr;
  size_t n_ = 0;
  int ng_ = 0, nx_ = 0, ny_ = 0, nz_ = 0;
};

template <typename T>
struct VectorField3D {
  void allocate_memory(int mx, int my, int mz, int nl, int ngg) {
    ng_ = ngg, nl_ = nl, nx_ = mx + 2 * ngg, ny_ = my + 2 * ngg, nz_ = mz + 2 * ngg;
    sz = (size_t)nx_ * ny_ * nz_ * nl;
    cudaMalloc(&p_, sz * sizeof(T));
    cudaMemset(p_, 0, sz * sizeof(T));
  }
  __host__ __device__ T &operator()(int i, int j, int k, int l) const {
    return p_[((size_t)(i + ng_) + (size_t)nx_ * ((size_t)(j + ng_) + (size_t)ny_ * (size_t)(k + ng_))) * nl_ + l];
  }
  __host__ __device__ T *data() const { return p_; }
  T *p_ = nullptr;
  size_t sz = 0;
  int ng_ = 0, nl_ = 0, nx_ = 0, ny_ = 0, nz_ = 0;
};
}  // namespace ggxl
