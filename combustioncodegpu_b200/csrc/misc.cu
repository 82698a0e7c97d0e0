// Small kernels: precision conversion, time-step bookkeeping and the
// convergence residual of Driver::compute_residual (Driver.cu:219-277,
// TimeAdvanceFunc.cu:13-24 and 292-303), reduced deterministically in FP64.
#include <algorithm>

#include "launch.h"

namespace ccb {

__global__ void k_convert_d2f(const double *src, float *dst, int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (float)src[i];
}

__global__ void k_convert_f2d(const float *src, double *dst, int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (double)src[i];
}

cudaError_t launch_convert_d2f(const double *src, float *dst, int64_t n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_convert_d2f<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src, dst, n);
  return cudaGetLastError();
}

cudaError_t launch_convert_f2d(const float *src, double *dst, int64_t n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_convert_f2d<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src, dst, n);
  return cudaGetLastError();
}

__global__ void k_convert_d2f_shift(const double *src, float *dst, int64_t n, double shift) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (float)(src[i] - shift);
}

__global__ void k_convert_f2d_shift(const float *src, double *dst, int64_t n, double shift) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (double)src[i] + shift;
}

cudaError_t launch_convert_d2f_shift(const double *src, float *dst, int64_t n, double shift, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_convert_d2f_shift<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src, dst, n, shift);
  return cudaGetLastError();
}

cudaError_t launch_convert_f2d_shift(const float *src, double *dst, int64_t n, double shift, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_convert_f2d_shift<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src, dst, n, shift);
  return cudaGetLastError();
}

// dt <- dt_next (when a candidate was reduced), dt_next <- +inf; the step's
// dt is appended to the history slot.
__global__ void k_dt_finalize(double *dt, unsigned long long *dt_next, unsigned *status, double *dt_hist) {
  if (dt_hist) *dt_hist = *dt;  // the step just finished used *dt
  const unsigned long long bits = *dt_next;
  const double v = __longlong_as_double((long long)bits);
  if (bits != 0x7ff0000000000000ull) {
    if (v > 0.0 && isfinite(v))
      *dt = v;
    else
      atomicOr(status, kStatusBadDt);
  } else {
    atomicOr(status, kStatusBadDt);
  }
  *dt_next = 0x7ff0000000000000ull;
}

cudaError_t launch_dt_finalize(double *dt, unsigned long long *dt_next, unsigned *status, double *dt_hist,
                               cudaStream_t s) {
  k_dt_finalize<<<1, 1, 0, s>>>(dt, dt_next, status, dt_hist);
  return cudaGetLastError();
}

__global__ void k_zero_points(double *field, const int64_t *points, int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) field[points[i]] = 0.0;
}

cudaError_t launch_zero_points(double *field, const int64_t *points, int64_t n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_zero_points<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(field, points, n);
  return cudaGetLastError();
}

// Interior rows: the (j, k) rows of the listed blocks, in block order, then
// k, then j; a row's points are contiguous both in the arena and in the
// interior-only arrays.  Each warp walks its rows in increasing order, so the
// block of a row is found by advancing from the previous one.
struct RowCursor {
  int b = 0;
  int64_t first = 0;  // first row of block b
  __device__ __forceinline__ void seek(const BlockInfo *blocks, int nblocks, int64_t r) {
    while (b + 1 < nblocks && r >= first + (int64_t)blocks[b].my * blocks[b].mz) {
      first += (int64_t)blocks[b].my * blocks[b].mz;
      ++b;
    }
  }
};

__device__ __forceinline__ int64_t interior_rows(const BlockInfo *blocks, int nblocks) {
  int64_t n = 0;
  for (int b = 0; b < nblocks; ++b) n += (int64_t)blocks[b].my * blocks[b].mz;
  return n;
}

// store_last_step: (rho, |V|, p, T) of every interior point; |V| is DZone::vel
// (written by the update, zeroed by wall conditions, untouched by interface
// exchanges; TimeAdvanceFunc.cu:13-24).  One warp per row, lanes along i.
template <typename T>
__global__ void k_store_last(const BlockInfo *blocks, int nblocks, const T *P, const double *vel, int64_t N,
                             int64_t n_int, double *last) {
  const int lane = threadIdx.x & 31;
  const int64_t n_rows = interior_rows(blocks, nblocks);
  const int64_t w0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  RowCursor cur;
  for (int64_t r = w0; r < n_rows; r += nw) {
    cur.seek(blocks, nblocks, r);
    const BlockInfo &B = blocks[cur.b];
    const int64_t rr = r - cur.first;
    const int j = (int)(rr % B.my), k = (int)(rr / B.my);
    const int64_t g0 = B.interior_off + (int64_t)B.mx * rr;
    const int64_t p0 = B.base + (int64_t)B.nx * j + (int64_t)B.nx * B.ny * k;
    for (int i = lane; i < B.mx; i += 32) {
      const int64_t g = g0 + i, p = p0 + i;
      last[g] = P[p];
      last[n_int + g] = vel[p];
      last[2 * n_int + g] = P[4 * N + p];
      last[3 * n_int + g] = P[5 * N + p];
    }
  }
}

// Sum over a warp by shuffles in a fixed tree (the result does not depend on
// scheduling); lane 0 holds the sum.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// compute_square_of_dbv + per-CTA sums: each warp takes interior rows in a
// fixed order (lanes along i), then the warps' sums are added by the first
// warp in a fixed order, then one warp sums the partials: the result does
// not depend on scheduling.
template <typename T>
__global__ void k_residual_partial(const BlockInfo *blocks, int nblocks, const T *P, const double *vel, int64_t N,
                                   int64_t n_int, const double *last, double *partials) {
  double acc[4] = {0, 0, 0, 0};
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, n_warps = blockDim.x >> 5;
  const int64_t n_rows = interior_rows(blocks, nblocks);
  const int64_t w0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  RowCursor cur;
  for (int64_t r = w0; r < n_rows; r += nw) {
    cur.seek(blocks, nblocks, r);
    const BlockInfo &B = blocks[cur.b];
    const int64_t rr = r - cur.first;
    const int j = (int)(rr % B.my), k = (int)(rr / B.my);
    const int64_t g0 = B.interior_off + (int64_t)B.mx * rr;
    const int64_t p0 = B.base + (int64_t)B.nx * j + (int64_t)B.nx * B.ny * k;
    for (int i = lane; i < B.mx; i += 32) {
      const int64_t g = g0 + i, p = p0 + i;
      const double d0 = (double)P[p] - last[g];
      const double d1 = vel[p] - last[n_int + g];
      const double d2 = (double)P[4 * N + p] - last[2 * n_int + g];
      const double d3 = (double)P[5 * N + p] - last[3 * n_int + g];
      acc[0] += d0 * d0, acc[1] += d1 * d1, acc[2] += d2 * d2, acc[3] += d3 * d3;
    }
  }
  __shared__ double sh[4][32];
#pragma unroll
  for (int l = 0; l < 4; ++l) {
    const double w = warp_sum(acc[l]);
    if (lane == 0) sh[l][warp] = w;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      const double w = warp_sum(lane < n_warps ? sh[l][lane] : 0.0);
      if (lane == 0) partials[4 * blockIdx.x + l] = w;
    }
  }
}

__global__ void k_residual_final(const double *partials, int n_partials, int64_t n_int, double *res) {
  const int lane = threadIdx.x & 31;
  double r[4] = {0, 0, 0, 0};
  for (int b = lane; b < n_partials; b += 32)  // each lane in fixed order, then a fixed tree
    for (int l = 0; l < 4; ++l) r[l] += partials[4 * b + l];
#pragma unroll
  for (int l = 0; l < 4; ++l) {
    const double w = warp_sum(r[l]);
    if (lane == 0) res[l] = sqrt(w / (double)n_int), res[4 + l] = w;  // the norm, and the sum it came from
  }
}

template <typename T>
cudaError_t launch_store_last(const BlockInfo *blocks, int nblocks, const T *P, const double *vel, int64_t N,
                              int64_t n_interior, double *bv_last, cudaStream_t s) {
  k_store_last<T><<<(unsigned)std::max<int64_t>(1, std::min<int64_t>(1184, (n_interior + 255) / 256)), 256, 0, s>>>(
      blocks, nblocks, P, vel, N, n_interior, bv_last);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_residual(const BlockInfo *blocks, int nblocks, const T *P, const double *vel, int64_t N,
                            int64_t n_interior, const double *bv_last, double *partials, int n_partials, double *res,
                            cudaStream_t s) {
  k_residual_partial<T><<<n_partials, 256, 0, s>>>(blocks, nblocks, P, vel, N, n_interior, bv_last, partials);
  k_residual_final<<<1, 32, 0, s>>>(partials, n_partials, n_interior, res);
  return cudaGetLastError();
}

// Multi-process exchange: nf fields (stride N) of the points idx[0..n) into
// FP64 rows of out (stride n), and back; FP32 values round-trip exactly.
template <typename T>
__global__ void k_gather_points(const T *src, int64_t N, int nf, const int64_t *idx, int64_t n, double *out) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= n * nf) return;
  const int64_t f = e / n, i = e % n;
  out[e] = (double)src[f * N + idx[i]];
}

template <typename T>
__global__ void k_scatter_points(T *dst, int64_t N, int nf, const int64_t *idx, int64_t n, const double *in) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= n * nf) return;
  const int64_t f = e / n, i = e % n;
  dst[f * N + idx[i]] = (T)in[e];
}

template <typename T>
cudaError_t launch_gather_points(const T *src, int64_t N, int nf, const int64_t *idx, int64_t n, double *out,
                                 cudaStream_t s) {
  if (n <= 0 || nf <= 0) return cudaSuccess;
  k_gather_points<T><<<(unsigned)((n * nf + 255) / 256), 256, 0, s>>>(src, N, nf, idx, n, out);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_scatter_points(T *dst, int64_t N, int nf, const int64_t *idx, int64_t n, const double *in,
                                  cudaStream_t s) {
  if (n <= 0 || nf <= 0) return cudaSuccess;
  k_scatter_points<T><<<(unsigned)((n * nf + 255) / 256), 256, 0, s>>>(dst, N, nf, idx, n, in);
  return cudaGetLastError();
}

template cudaError_t launch_gather_points<double>(const double *, int64_t, int, const int64_t *, int64_t, double *,
                                                  cudaStream_t);
template cudaError_t launch_gather_points<float>(const float *, int64_t, int, const int64_t *, int64_t, double *,
                                                 cudaStream_t);
template cudaError_t launch_scatter_points<double>(double *, int64_t, int, const int64_t *, int64_t, const double *,
                                                   cudaStream_t);
template cudaError_t launch_scatter_points<float>(float *, int64_t, int, const int64_t *, int64_t, const double *,
                                                  cudaStream_t);

template cudaError_t launch_store_last<double>(const BlockInfo *, int, const double *, const double *, int64_t,
                                               int64_t, double *, cudaStream_t);
template cudaError_t launch_store_last<float>(const BlockInfo *, int, const float *, const double *, int64_t,
                                              int64_t, double *, cudaStream_t);
template cudaError_t launch_residual<double>(const BlockInfo *, int, const double *, const double *, int64_t,
                                             int64_t, const double *, double *, int, double *, cudaStream_t);
template cudaError_t launch_residual<float>(const BlockInfo *, int, const float *, const double *, int64_t, int64_t,
                                            const double *, double *, int, double *, cudaStream_t);

}  // namespace ccb
