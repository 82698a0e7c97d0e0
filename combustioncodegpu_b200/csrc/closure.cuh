// Learned transport closure on the 5th-generation tensor cores (sm_100a).
//
// An MLP (T, X_1..X_ns) -> (log mu, log lambda, log rhoD_1..rhoD_ns) with
// three hidden layers of 64 SiLU units replaces the Wilke / constant-Schmidt
// evaluation (Transport.cu:43-96) for points inside its training hull; points
// outside it (T outside [t_min, t_max]) take the exact transport.  The network
// is evaluated 128 points at a time:
//
//   * operands in shared memory, BF16, K-major without swizzle (the canonical
//     layout: 8-row x 16-byte core matrices; element (r, k) of an R-row
//     operand at byte (k/8)*16R + 16r + 2(k%8), so the two core matrices of a
//     K=16 step are LBO = 16R bytes apart and 8-row groups SBO = 128 bytes);
//   * one elected thread issues tcgen05.mma (kind::f16, BF16 x BF16 -> FP32,
//     M = 128) into a 64-column TMEM accumulator and commits to an mbarrier;
//   * the four warps read their 32 TMEM lanes back with tcgen05.ld, add the
//     bias, apply SiLU in FP32 and store the BF16 activations as the next
//     layer's A operand.
//
// Inputs: t = (T - t_center) / t_scale and the mole fractions, each as a BF16
// pair (hi, lo = value - hi) so that BF16 input rounding does not limit the
// fit: 2 + 2 ns features, padded to 32.  The hidden activations are stored
// the same way, as BF16 (hi, lo) pairs, and every layer after the first runs
// two MMAs into the same accumulator (hi x W, then lo x W): the activations
// keep ~16 significant bits instead of BF16's 8, which would otherwise floor
// the closure's error near 1e-3.  Outputs: 2 + ns values, padded to 16,
// mapped back by property = exp(o * out_scale + out_mean).  Points outside
// the training hull in T, or with a mole fraction of at least 0.998, take the
// exact transport in the same kernel.
//
// Run-time error check (err_bound > 0): after every round of up to 32 tiles a
// CTA evaluates the exact transport at 4 fixed sample points of each tile
// (1 in 32 points, one sample per thread, so the warps stay full) and
// compares it with what the network wrote; a tile whose sampled outputs have
// a root-mean-square relative error above the bound, or one of them above ten
// times the bound, is recomputed with the exact transport.
#pragma once
#include <cuda_bf16.h>

#include "stage.cuh"

namespace ccb {

constexpr int kMlpSmem = kMlpWBytes + kMlpXBytes + 2 * kMlpHBytes + kMlpBias * 4 + 64;
constexpr int kMlpRound = 32;  // tiles per run-time check round (4 samples each: one per thread)
constexpr int kMlpTmemCols = 64;
constexpr unsigned kStatusMlpTimeout = 16u;  // an MMA completion wait gave up
constexpr long long kMlpMaxSpins = kDefaultWaitSpins;  // bound of the drain after an abort
constexpr float kMlpPureX = 0.998f;  // mole fraction above which the exact transport is used

__device__ __forceinline__ uint32_t mlp_smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// shared-memory matrix descriptor: start, leading (K) and stride (M/N) byte
// offsets, descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t mlp_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor, kind::f16: FP32 accumulator, BF16 A and B, both K-major
__host__ __device__ constexpr uint32_t mlp_idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kMlpRows >> 4) << 24);
}

__device__ __forceinline__ void mlp_mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, int acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mlp_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ bool mlp_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(mlp_smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// non-blocking check of the same phase
__device__ __forceinline__ bool mlp_test_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(mlp_smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// x * sigmoid(x) with the hardware exponential and division (relative error
// ~1e-7, below the hi/lo BF16 representation of the activations that follows)
__device__ __forceinline__ float mlp_silu(float x) { return __fdividef(x, 1.0f + __expf(-x)); }

__device__ __forceinline__ uint32_t mlp_pack(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t *>(&h);
}

// BF16 (hi, lo) split of a hidden activation with integer operations only
// (the conversion instructions share the transcendental unit with the
// SiLU's exponential and reciprocal, which bound the kernel): adding 0x8000
// to the bits of x rounds its magnitude to the nearest BF16 in the upper 16
// bits (ties away from zero; a carry moves into the exponent correctly), so
// hi = those upper bits; lo = x - hi is exact in FP32 and is rounded the same
// way.  |x - hi - lo| <= 2^-16 |x| for normal x.  The returned words carry
// the BF16 value in their upper halves.
__device__ __forceinline__ void mlp_split(float x, uint32_t &hi_bits, uint32_t &lo_bits) {
  hi_bits = __float_as_uint(x) + 0x8000u;
  const float hi = __uint_as_float(hi_bits & 0xFFFF0000u);
  lo_bits = __float_as_uint(x - hi) + 0x8000u;
}

// BF16x2 word of two split values: a in the low half, b in the high half
// (the layout of __floats2bfloat162_rn(a, b)).
__device__ __forceinline__ uint32_t mlp_pack_hi(uint32_t a_bits, uint32_t b_bits) {
  return __byte_perm(a_bits, b_bits, 0x7632);
}

template <typename T, int NS>
__global__ void __launch_bounds__(kMlpRows) k_props_mlp(const T *__restrict__ P, T *__restrict__ Pr, int64_t N,
                                                        const ClosureDev cl, unsigned *status,
                                                        const __grid_constant__ ChemParams C) {
  constexpr int A = SpecCount<NS>::kArr;
  const int ns = SpecCount<NS>::n(C);
  extern __shared__ __align__(128) unsigned char sm[];
  unsigned char *sW = sm;                                   // weights, operand layout
  unsigned char *sX = sW + kMlpWBytes;                      // A operand of layer 1 [128 x 32]
  unsigned char *sH = sX + kMlpXBytes;                      // A operand of layers 2-4 [128 x 64], hi
  unsigned char *sHl = sH + kMlpHBytes;                     // the same, lo = value - hi
  float *sB = reinterpret_cast<float *>(sHl + kMlpHBytes);  // biases
  uint64_t *bar = reinterpret_cast<uint64_t *>(sB + kMlpBias);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5;

  for (int e = tid; e < kMlpWBytes / 16; e += kMlpRows)
    reinterpret_cast<uint4 *>(sW)[e] = reinterpret_cast<const uint4 *>(cl.w)[e];
  for (int e = tid; e < kMlpBias; e += kMlpRows) sB[e] = cl.b[e];
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mlp_smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(mlp_smem_u32(tslot)),
                 "r"(kMlpTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  const uint32_t t_row = tmem + ((uint32_t)(32 * warp) << 16);  // this warp's 32 lanes

  const uint32_t aX = mlp_smem_u32(sX), aH = mlp_smem_u32(sH), aHl = mlp_smem_u32(sHl), aW = mlp_smem_u32(sW);
  const uint32_t aW1 = aW, aW2 = aW1 + kMlpW1, aW3 = aW2 + kMlpW2, aW4 = aW3 + kMlpW2;
  uint32_t phase = 0;
  bool late = false;
  unsigned long long n_eval = 0, n_fb = 0, n_chk = 0;
  __shared__ int64_t s_round[kMlpRound];  // tile bases of the current check round
  __shared__ unsigned s_fail;             // bit t: tile t of the round failed its samples
  int n_round = 0;
  // exact transport of point q into Pr (the fallback)
  auto exact_at = [&](int64_t q) {
    T Yt[A], mu, lam, rd[A], gam, c;
#pragma unroll
    for (int l = 0; l < A; ++l)
      if (l < ns) Yt[l] = P[(6 + l) * N + q];
    point_props<T, NS>(C, param_rec<T>(C), P[5 * N + q], Yt, mu, lam, rd, gam, c);
    Pr[q] = mu;
    Pr[N + q] = lam;
#pragma unroll
    for (int l = 0; l < A; ++l)
      if (l < ns) Pr[(2 + l) * N + q] = rd[l];
  };

  for (int64_t base = (int64_t)blockIdx.x * kMlpRows; base < N; base += (int64_t)gridDim.x * kMlpRows) {
    const int64_t p = base + tid;
    const bool valid = p < N && P[p] > T(0);  // padding points of the arena have rho = 0
    float tem = 1000.0f, X[A];
    if (valid) {
      tem = (float)P[5 * N + p];
      float s = 0;
#pragma unroll
      for (int l = 0; l < A; ++l)
        if (l < ns) X[l] = (float)P[(6 + l) * N + p] * tab<float>(C).inv_mw[l], s += X[l];
      const float is = 1.0f / s;
#pragma unroll
      for (int l = 0; l < A; ++l)
        if (l < ns) X[l] *= is;
    } else {
#pragma unroll
      for (int l = 0; l < A; ++l) X[l] = 0;
    }
    // exact fallback outside the training hull in T, and near a pure species,
    // where the exact rhoD_k switches branch at |X_k - 1| < 1e-3
    // (Transport.cu:85-92), a step no smooth fit follows
    float x_top = 0.0f;
#pragma unroll
    for (int l = 0; l < A; ++l)
      if (l < ns) x_top = fmaxf(x_top, X[l]);
    const bool fb = valid && (!(tem >= cl.t_min && tem <= cl.t_max) || x_top >= kMlpPureX);
    {  // features: t hi/lo, X hi/lo, zero padding -> row tid of the layer-1 A operand
      float f[kMlpIn];
#pragma unroll
      for (int k = 0; k < kMlpIn; ++k) f[k] = 0.0f;
      const float t = (tem - cl.t_center) * cl.t_inv_scale;
      f[0] = __bfloat162float(__float2bfloat16_rn(t));
      f[1] = t - f[0];
#pragma unroll
      for (int l = 0; l < A; ++l)
        if (l < ns) {
          f[2 + l] = __bfloat162float(__float2bfloat16_rn(X[l]));
          f[2 + ns + l] = X[l] - f[2 + l];
        }
#pragma unroll
      for (int c = 0; c < kMlpIn / 8; ++c) {
        uint4 v;
        v.x = mlp_pack(f[8 * c], f[8 * c + 1]);
        v.y = mlp_pack(f[8 * c + 2], f[8 * c + 3]);
        v.z = mlp_pack(f[8 * c + 4], f[8 * c + 5]);
        v.w = mlp_pack(f[8 * c + 6], f[8 * c + 7]);
        *reinterpret_cast<uint4 *>(sX + mlp_off(kMlpRows, tid, 8 * c)) = v;
      }
    }
    float out[kMlpOut];
#pragma unroll 1
    for (int layer = 0; layer < 4; ++layer) {
      // make this thread's operand stores visible to the tensor cores, then issue
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (tid == 0) {
        const int ksteps = layer == 0 ? kMlpIn / 16 : kMlpH / 16;
        const int n = layer == 3 ? kMlpOut : kMlpH;
        const uint32_t aA = layer == 0 ? aX : aH;
        const uint32_t aB = layer == 0 ? aW1 : (layer == 1 ? aW2 : (layer == 2 ? aW3 : aW4));
        const uint32_t lboA = 16 * kMlpRows, lboB = 16 * n;
        for (int s = 0; s < ksteps; ++s)
          mlp_mma(tmem, mlp_desc(aA + 2 * s * lboA, lboA, 128), mlp_desc(aB + 2 * s * lboB, lboB, 128),
                  mlp_idesc(n), s > 0);
        if (layer > 0)  // the lo half of the hidden activations into the same accumulator
          for (int s = 0; s < ksteps; ++s)
            mlp_mma(tmem, mlp_desc(aHl + 2 * s * lboA, lboA, 128), mlp_desc(aB + 2 * s * lboB, lboB, 128),
                    mlp_idesc(n), 1);
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         mlp_smem_u32(bar))
                     : "memory");
      }
      bool ok = mlp_test_wait(bar, phase);
      for (long long s = 0; !ok && s < C.max_spins; ++s) ok = mlp_try_wait(bar, phase);
      phase ^= 1u;
      if (__syncthreads_or(!ok)) {
        late = true;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (layer < 3) {
        const float *bias = sB + layer * kMlpH;
#pragma unroll
        for (int q = 0; q < kMlpH / 16; ++q) {
          float v[16];
          mlp_ld16(t_row + 16 * q, v);
#pragma unroll
          for (int i = 0; i < 16; ++i) v[i] = mlp_silu(v[i] + bias[16 * q + i]);
          uint32_t hb[16], lb[16];
#pragma unroll
          for (int i = 0; i < 16; ++i) mlp_split(v[i], hb[i], lb[i]);
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            uint4 w;
            w.x = mlp_pack_hi(hb[8 * h], hb[8 * h + 1]);
            w.y = mlp_pack_hi(hb[8 * h + 2], hb[8 * h + 3]);
            w.z = mlp_pack_hi(hb[8 * h + 4], hb[8 * h + 5]);
            w.w = mlp_pack_hi(hb[8 * h + 6], hb[8 * h + 7]);
            *reinterpret_cast<uint4 *>(sH + mlp_off(kMlpRows, tid, 16 * q + 8 * h)) = w;
            w.x = mlp_pack_hi(lb[8 * h], lb[8 * h + 1]);
            w.y = mlp_pack_hi(lb[8 * h + 2], lb[8 * h + 3]);
            w.z = mlp_pack_hi(lb[8 * h + 4], lb[8 * h + 5]);
            w.w = mlp_pack_hi(lb[8 * h + 6], lb[8 * h + 7]);
            *reinterpret_cast<uint4 *>(sHl + mlp_off(kMlpRows, tid, 16 * q + 8 * h)) = w;
          }
        }
      } else {
        mlp_ld16(t_row, out);
#pragma unroll
        for (int i = 0; i < kMlpOut; ++i) out[i] += sB[3 * kMlpH + i];
      }
    }
    if (late) break;
    if (valid) {
      ++n_eval;
      if (!fb) {
        Pr[p] = T(__expf(out[0] * cl.out_scale[0] + cl.out_mean[0]));
        Pr[N + p] = T(__expf(out[1] * cl.out_scale[1] + cl.out_mean[1]));
#pragma unroll
        for (int l = 0; l < A; ++l)
          if (l < ns) Pr[(2 + l) * N + p] = T(__expf(out[2 + l] * cl.out_scale[2 + l] + cl.out_mean[2 + l]));
      } else {
        ++n_fb;
        exact_at(p);
      }
    }
    if (cl.err_bound > 0.0f) {
      // run-time check of the round: 4 fixed samples per tile, one per thread
      if (tid == 0) s_round[n_round] = base;
      ++n_round;
      if (n_round == kMlpRound || base + (int64_t)gridDim.x * kMlpRows >= N) {
        if (tid == 0) s_fail = 0u;
        __syncthreads();  // the round's properties and tile list visible to the whole CTA
        const int t = tid >> 2, smp = tid & 3;
        float se = 0.0f, mx = 0.0f, cnt = 0.0f;  // squared and largest relative error of the sample's outputs
        if (t < n_round) {
          const int64_t b = s_round[t];
          const int64_t q = b + smp * 32 + (int)(((b / kMlpRows) * 7 + smp * 11) & 31);
          if (q < N && P[q] > T(0)) {
            T Yt[A], mu, lam, rd[A], gam, c;
#pragma unroll
            for (int l = 0; l < A; ++l)
              if (l < ns) Yt[l] = P[(6 + l) * N + q];
            point_props<T, NS>(C, param_rec<T>(C), P[5 * N + q], Yt, mu, lam, rd, gam, c);
            auto acc = [&](T got, T want) {
              const float r = fabsf((float)(got / want) - 1.0f);
              se += r * r, mx = fmaxf(mx, r), cnt += 1.0f;
            };
            acc(Pr[q], mu);
            acc(Pr[N + q], lam);
#pragma unroll
            for (int l = 0; l < A; ++l)
              if (l < ns) acc(Pr[(2 + l) * N + q], rd[l]);
          }
        }
        // the tile's 4 samples are 4 consecutive lanes
#pragma unroll
        for (int o = 1; o < 4; o <<= 1) {
          se += __shfl_xor_sync(0xffffffffu, se, o);
          mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
          cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        }
        // fails: root-mean-square sampled error above the bound, or one sampled
        // output above ten times the bound (NaN fails too)
        if (smp == 0 && t < n_round && cnt > 0.0f &&
            !(sqrtf(se / cnt) <= cl.err_bound && mx <= 10.0f * cl.err_bound))
          atomicOr(&s_fail, 1u << t);
        __syncthreads();
        for (unsigned fail = s_fail; fail; fail &= fail - 1u) {  // tiles sent back to the exact transport
          const int64_t q = s_round[__ffs(fail) - 1] + tid;
          if (q < N && P[q] > T(0)) exact_at(q), ++n_chk;
        }
        __syncthreads();  // before the next round reuses the tile list
        n_round = 0;
      }
    }
  }
  if (late) {
    // a completion wait gave up: record it, let the MMAs in flight finish
    // (bounded) before the accumulator columns are released
    if (tid == 0) atomicOr(status, kStatusMlpTimeout);
    long spins = 0;
    while (!mlp_try_wait(bar, phase ^ 1u) && ++spins < kMlpMaxSpins) {
    }
  }
  // per-CTA counts
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    n_eval += __shfl_xor_sync(0xffffffffu, n_eval, o);
    n_fb += __shfl_xor_sync(0xffffffffu, n_fb, o);
    n_chk += __shfl_xor_sync(0xffffffffu, n_chk, o);
  }
  if ((tid & 31) == 0 && cl.counts) {
    atomicAdd(cl.counts, n_eval);
    atomicAdd(cl.counts + 1, n_fb);
    atomicAdd(cl.counts + 2, n_chk);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kMlpTmemCols) : "memory");
}

}  // namespace ccb
