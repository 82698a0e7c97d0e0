// Training kernels of the learned transport closure: forward, backward and
// Adam for the 4-layer MLP (n_in -> H -> H -> H -> n_out, SiLU) with the
// inference kernel's rounding points (quantisation-aware training): every
// weight is rounded to BF16 (round to nearest even) in the forward pass and
// the rounding is passed through unchanged in the backward pass
// (straight-through); the network inputs are BF16 (hi, lo) pairs as the
// kernel forms them; the hidden activations stay FP32 (the inference kernel
// carries them as BF16 hi/lo pairs, ~16 significant bits); accumulation,
// biases and the master weights are FP32.  Loss: mean over the batch and the outputs of
// ((o - y) scale_o)^2, i.e. the squared error of the log properties.
//
// Parameters are one FP32 buffer in the order W1 [H][n_in], b1 [H],
// W2 [H][H], b2, W3 [H][H], b3, W4 [n_out][H], b4 [n_out].  All arrays are
// device memory owned by the caller; the workspace size comes from
// cc_mlp_workspace_bytes.  Every sum runs in a fixed order (per-CTA partial
// sums reduced in CTA order), so a gradient is reproducible bit for bit.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <string>

#include "../../include/cc_b200.h"

void ccb_set_last_error(const std::string &msg);  // api.cu

namespace {

constexpr int kRows = 32;     // batch rows per CTA
constexpr int kThreads = 256;
constexpr int kMaxWidth = 64; // widest layer (n_in, H, n_out <= 64)

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float sigm(float z) { return 1.0f / (1.0f + expf(-z)); }

// Z = A r(W)^T + b for kRows rows; H = silu(Z) (hidden) or Z (output).
// Only the weights are rounded (the first layer's inputs are BF16 values).
__global__ void __launch_bounds__(kThreads) k_dense_fwd(const float *__restrict__ A, const float *__restrict__ W,
                                                        const float *__restrict__ b, float *__restrict__ Z,
                                                        float *__restrict__ H, int B, int n_in, int n_out, int act) {
  __shared__ float sW[kMaxWidth * kMaxWidth];
  __shared__ float sA[kRows * kMaxWidth];
  const int r0 = blockIdx.x * kRows;
  for (int e = threadIdx.x; e < n_out * n_in; e += kThreads) sW[e] = bf16r(W[e]);
  for (int e = threadIdx.x; e < kRows * n_in; e += kThreads) {
    const int r = r0 + e / n_in;
    sA[e] = r < B ? A[(size_t)r * n_in + e % n_in] : 0.0f;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < kRows * n_out; e += kThreads) {
    const int rl = e / n_out, o = e % n_out, r = r0 + rl;
    if (r >= B) continue;
    float z = b[o];
    for (int i = 0; i < n_in; ++i) z = fmaf(sA[rl * n_in + i], sW[o * n_in + i], z);
    Z[(size_t)r * n_out + o] = z;
    H[(size_t)r * n_out + o] = act ? z * sigm(z) : z;
  }
}

// G = 2 ((o - y) s)^2' / (B n_out) = 2 (o - y) s^2 / (B n_out); per-CTA
// partial sums of ((o - y) s)^2.
__global__ void __launch_bounds__(kThreads) k_loss(const float *__restrict__ O, const float *__restrict__ Y,
                                                   const float *__restrict__ scale, float *__restrict__ G,
                                                   float *__restrict__ part, int B, int n_out) {
  __shared__ float red[kThreads];
  const int r0 = blockIdx.x * kRows;
  const float inv = 1.0f / ((float)B * (float)n_out);
  float acc = 0.0f;
  for (int e = threadIdx.x; e < kRows * n_out; e += kThreads) {
    const int r = r0 + e / n_out, o = e % n_out;
    if (r >= B) continue;
    const size_t q = (size_t)r * n_out + o;
    const float err = (O[q] - Y[q]) * scale[o];
    acc = fmaf(err, err, acc);
    G[q] = 2.0f * err * scale[o] * inv;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// dZ_prev = (G r(W)) silu'(Z_prev) for kRows rows (the rounding of W is
// passed through).
__global__ void __launch_bounds__(kThreads) k_dense_bwd_in(const float *__restrict__ G, const float *__restrict__ W,
                                                           const float *__restrict__ Zp, float *__restrict__ dZp,
                                                           int B, int n_in, int n_out) {
  __shared__ float sW[kMaxWidth * kMaxWidth];
  __shared__ float sG[kRows * kMaxWidth];
  const int r0 = blockIdx.x * kRows;
  for (int e = threadIdx.x; e < n_out * n_in; e += kThreads) sW[e] = bf16r(W[e]);
  for (int e = threadIdx.x; e < kRows * n_out; e += kThreads) {
    const int r = r0 + e / n_out;
    sG[e] = r < B ? G[(size_t)r * n_out + e % n_out] : 0.0f;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < kRows * n_in; e += kThreads) {
    const int rl = e / n_in, i = e % n_in, r = r0 + rl;
    if (r >= B) continue;
    float g = 0.0f;
    for (int o = 0; o < n_out; ++o) g = fmaf(sG[rl * n_out + o], sW[o * n_in + i], g);
    const float z = Zp[(size_t)r * n_in + i], s = sigm(z);
    dZp[(size_t)r * n_in + i] = g * (s * (1.0f + z * (1.0f - s)));
  }
}

// Per-CTA partial weight and bias gradients over its kRows rows:
// pW[cta][o][i] = sum_r G[r][o] A[r][i], pb[cta][o] = sum_r G[r][o].
__global__ void __launch_bounds__(kThreads) k_dense_bwd_w(const float *__restrict__ G, const float *__restrict__ A,
                                                          float *__restrict__ pW, float *__restrict__ pb, int B,
                                                          int n_in, int n_out) {
  __shared__ float sA[kRows * kMaxWidth];
  __shared__ float sG[kRows * kMaxWidth];
  const int r0 = blockIdx.x * kRows;
  for (int e = threadIdx.x; e < kRows * n_in; e += kThreads) {
    const int r = r0 + e / n_in;
    sA[e] = r < B ? A[(size_t)r * n_in + e % n_in] : 0.0f;
  }
  for (int e = threadIdx.x; e < kRows * n_out; e += kThreads) {
    const int r = r0 + e / n_out;
    sG[e] = r < B ? G[(size_t)r * n_out + e % n_out] : 0.0f;
  }
  __syncthreads();
  float *w = pW + (size_t)blockIdx.x * n_out * n_in;
  for (int e = threadIdx.x; e < n_out * n_in; e += kThreads) {
    const int o = e / n_in, i = e % n_in;
    float acc = 0.0f;
    for (int rl = 0; rl < kRows; ++rl) acc = fmaf(sG[rl * n_out + o], sA[rl * n_in + i], acc);
    w[e] = acc;
  }
  for (int o = threadIdx.x; o < n_out; o += kThreads) {
    float acc = 0.0f;
    for (int rl = 0; rl < kRows; ++rl) acc += sG[rl * n_out + o];
    pb[(size_t)blockIdx.x * n_out + o] = acc;
  }
}

// out[e] = sum over parts of part[p][e], in part order
__global__ void k_reduce_parts(const float *__restrict__ part, int n_parts, int n, float *__restrict__ out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  float acc = 0.0f;
  for (int p = 0; p < n_parts; ++p) acc += part[(size_t)p * n + e];
  out[e] = acc;
}

__global__ void k_loss_final(const float *__restrict__ part, int n_parts, float inv_count, float *__restrict__ loss) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  float acc = 0.0f;
  for (int p = 0; p < n_parts; ++p) acc += part[p];
  *loss = acc * inv_count;
}

// Adam (Kingma & Ba 2015) with bias correction, no weight decay.
__global__ void k_adam(int64_t n, float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const float gi = g[e];
  const float mi = b1 * m[e] + (1.0f - b1) * gi;
  const float vi = b2 * v[e] + (1.0f - b2) * gi * gi;
  m[e] = mi, v[e] = vi;
  p[e] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

struct Shape {
  int n_in, H, n_out, B, n_cta;
  int64_t off_w[4], off_b[4], n_params;
  int width_in[4], width_out[4];
};

Shape shape_of(int n_in, int H, int n_out, int B) {
  Shape s{};
  s.n_in = n_in, s.H = H, s.n_out = n_out, s.B = B, s.n_cta = (B + kRows - 1) / kRows;
  const int wi[4] = {n_in, H, H, H}, wo[4] = {H, H, H, n_out};
  int64_t o = 0;
  for (int l = 0; l < 4; ++l) {
    s.width_in[l] = wi[l], s.width_out[l] = wo[l];
    s.off_w[l] = o, o += (int64_t)wo[l] * wi[l];
    s.off_b[l] = o, o += wo[l];
  }
  s.n_params = o;
  return s;
}

// workspace (floats): Z[4] (B x out), Hr[3] (B x H), G ping-pong 2 x (B x 64),
// weight partials n_cta x 64 x 64, bias partials n_cta x 64, loss partials n_cta
struct Work {
  float *Z[4], *Hr[3], *G[2], *pW, *pb, *pl;
};

int64_t work_floats(const Shape &s) {
  return (int64_t)s.B * (3 * s.H + s.n_out) + (int64_t)3 * s.B * s.H + 2LL * s.B * kMaxWidth +
         (int64_t)s.n_cta * kMaxWidth * kMaxWidth + (int64_t)s.n_cta * kMaxWidth + s.n_cta;
}

Work carve(const Shape &s, float *w) {
  Work k{};
  for (int l = 0; l < 4; ++l) k.Z[l] = w, w += (int64_t)s.B * s.width_out[l];
  for (int l = 0; l < 3; ++l) k.Hr[l] = w, w += (int64_t)s.B * s.H;
  for (int q = 0; q < 2; ++q) k.G[q] = w, w += (int64_t)s.B * kMaxWidth;
  k.pW = w, w += (int64_t)s.n_cta * kMaxWidth * kMaxWidth;
  k.pb = w, w += (int64_t)s.n_cta * kMaxWidth;
  k.pl = w;
  return k;
}

int fail(int code, const std::string &msg) {
  ccb_set_last_error(msg);
  return code;
}

int check_shape(int n_in, int H, int n_out, int B) {
  if (n_in < 1 || H < 1 || n_out < 1 || n_in > kMaxWidth || H > kMaxWidth || n_out > kMaxWidth)
    return fail(CC_ERR_ARG, "cc_mlp: layer widths must lie in [1, 64]");
  if (B < 1) return fail(CC_ERR_ARG, "cc_mlp: batch must be positive");
  return CC_OK;
}

}  // namespace

extern "C" int64_t cc_mlp_param_count(int n_in, int hidden, int n_out) {
  if (check_shape(n_in, hidden, n_out, 1)) return -1;
  return shape_of(n_in, hidden, n_out, 1).n_params;
}

extern "C" int64_t cc_mlp_workspace_bytes(int n_in, int hidden, int n_out, int batch) {
  if (check_shape(n_in, hidden, n_out, batch)) return -1;
  return work_floats(shape_of(n_in, hidden, n_out, batch)) * (int64_t)sizeof(float);
}

extern "C" int cc_mlp_grad(int n_in, int hidden, int n_out, int batch, const float *params, const float *x,
                           const float *y, const float *out_scale, float *grad, float *loss, void *workspace,
                           void *stream) {
  if (int r = check_shape(n_in, hidden, n_out, batch)) return r;
  if (!params || !x || !y || !out_scale || !grad || !loss || !workspace)
    return fail(CC_ERR_ARG, "cc_mlp_grad: null pointer");
  const Shape s = shape_of(n_in, hidden, n_out, batch);
  Work k = carve(s, static_cast<float *>(workspace));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nc = s.n_cta;
  // forward
  const float *a = x;
  for (int l = 0; l < 4; ++l) {
    float *h = l < 3 ? k.Hr[l] : k.Z[3];
    k_dense_fwd<<<nc, kThreads, 0, st>>>(a, params + s.off_w[l], params + s.off_b[l], k.Z[l], h, s.B,
                                          s.width_in[l], s.width_out[l], l < 3 ? 1 : 0);
    a = h;
  }
  k_loss<<<nc, kThreads, 0, st>>>(k.Z[3], y, out_scale, k.G[0], k.pl, s.B, s.n_out);
  k_loss_final<<<1, 32, 0, st>>>(k.pl, nc, 1.0f / ((float)s.B * (float)s.n_out), loss);
  // backward: G holds dL/dZ of layer l
  int cur = 0;
  for (int l = 3; l >= 0; --l) {
    const float *A = l > 0 ? k.Hr[l - 1] : x;
    const int wi = s.width_in[l], wo = s.width_out[l];
    k_dense_bwd_w<<<nc, kThreads, 0, st>>>(k.G[cur], A, k.pW, k.pb, s.B, wi, wo);
    k_reduce_parts<<<(wo * wi + 255) / 256, 256, 0, st>>>(k.pW, nc, wo * wi, grad + s.off_w[l]);
    k_reduce_parts<<<(wo + 255) / 256, 256, 0, st>>>(k.pb, nc, wo, grad + s.off_b[l]);
    if (l > 0) {
      k_dense_bwd_in<<<nc, kThreads, 0, st>>>(k.G[cur], params + s.off_w[l], k.Z[l - 1], k.G[1 - cur], s.B, wi, wo);
      cur = 1 - cur;
    }
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(CC_ERR_CUDA, std::string("cc_mlp_grad: ") + cudaGetErrorString(e));
  return CC_OK;
}

extern "C" int cc_mlp_adam(int64_t n, float *params, const float *grad, float *m, float *v, float lr, float beta1,
                           float beta2, float eps, int step, void *stream) {
  if (n < 1 || step < 1 || !params || !grad || !m || !v) return fail(CC_ERR_ARG, "cc_mlp_adam: bad arguments");
  const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
  k_adam<<<(unsigned)((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(n, params, grad, m, v, lr, beta1,
                                                                                   beta2, eps, c1, c2);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(CC_ERR_CUDA, std::string("cc_mlp_adam: ") + cudaGetErrorString(e));
  return CC_OK;
}
