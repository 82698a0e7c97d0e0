// Definitions of the templated launchers (included by inst_*.cu only).
#pragma once
#include <algorithm>
#include <type_traits>

#include "launch.h"
#include "stage.cuh"
#include "stage_tma.cuh"
#include "stage_split.cuh"
#include "stage_dq.cuh"
#include "closure.cuh"
#include "lusgs.cuh"

namespace ccb {

template <typename T, int NS>
size_t Launch<T, NS>::stage_smem() {
  return StageSmem<T, NS>::kBytes;
}

template <typename T, int NS>
size_t Launch<T, NS>::stage_tma_smem() {
  return TmaLayout<T, NS>::kBytes;
}

template <typename T, int NS>
size_t Launch<T, NS>::faces_smem() {
  return sizeof(T) * SpecCount<NS>::kArr * 2 * kRecLen;
}

template <typename T, int NS>
size_t Launch<T, NS>::update_smem() {
  return StageSmem<T, NS>::kRecBytes;
}

template <typename T, int NS>
cudaError_t Launch<T, NS>::faces(const StageArgs<T> &a, const ChemParams &C, int n_regular, int n_edge,
                                 cudaStream_t s) {
  if (n_regular + n_edge <= 0) return cudaSuccess;
  StageArgs<T> b = a;
  b.n_regular = n_regular;
  k_faces<T, NS><<<n_regular + n_edge, dim3(kTX, kTY), faces_smem(), s>>>(b, C);
  return cudaGetLastError();
}

// (ty, tx) -> the instantiated tile shapes of the TMA face kernel: 32 x 4,
// 32 x 8, 32 x 16, 16 x 8 and 16 x 16 points (i x j); f gets both as
// integral constants.
template <typename F>
cudaError_t with_face_shape(int ty, int tx, F &&f) {
  using std::integral_constant;
  if (tx == 32) {
    if (ty == 4) return f(integral_constant<int, 4>{}, integral_constant<int, 32>{});
    if (ty == 8) return f(integral_constant<int, 8>{}, integral_constant<int, 32>{});
    if (ty == 16) return f(integral_constant<int, 16>{}, integral_constant<int, 32>{});
  } else if (tx == 16) {
    if (ty == 8) return f(integral_constant<int, 8>{}, integral_constant<int, 16>{});
    if (ty == 16) return f(integral_constant<int, 16>{}, integral_constant<int, 16>{});
  }
  return cudaErrorInvalidValue;
}

template <typename T, int NS>
size_t Launch<T, NS>::faces_tma_smem(int ty, int tx) {
  size_t b = 0;
  with_face_shape(ty, tx, [&](auto ty_c, auto tx_c) {
    using L = FacesTmaLayout<T, NS, decltype(ty_c)::value, decltype(tx_c)::value>;
    b = L::kOk ? L::kBytes : 0;
    return cudaSuccess;
  });
  return b;
}

template <typename T, int NS>
cudaError_t Launch<T, NS>::faces_tma(const StageArgs<T> &a, const Tile *tiles, int ty, int tx, const void *maps,
                                     const ChemParams &C, int n_tiles, cudaStream_t s) {
  if (n_tiles <= 0) return cudaSuccess;
  const size_t smem = faces_tma_smem(ty, tx);
  if (smem == 0) return cudaErrorInvalidConfiguration;
  const CUtensorMap *m = (const CUtensorMap *)maps;
  return with_face_shape(ty, tx, [&](auto ty_c, auto tx_c) -> cudaError_t {
    constexpr int TY = decltype(ty_c)::value, TX = decltype(tx_c)::value;
    if constexpr (!FacesTmaLayout<T, NS, TY, TX>::kOk) {
      return cudaErrorInvalidConfiguration;  // the ring does not fit (32 x 16, 16 x 16 in FP64)
    } else {
      k_faces_tma<T, NS, TY, TX><<<n_tiles, dim3(TX, TY), smem, s>>>(a, tiles, m, C);
      return cudaGetLastError();
    }
  });
}

// y-exchange rounds of the dq face kernel per tile height (shared memory)
template <int TY>
struct DqChunks {
  static constexpr int value = TY == 4 ? 2 : (TY == 8 ? 3 : 1);
};

template <typename T, int NS>
size_t Launch<T, NS>::faces_dq_smem(int ty) {
  if (ty == 4) return FacesDqLayout<T, NS, 4, DqChunks<4>::value>::kBytes;
  if (ty == 8) return FacesDqLayout<T, NS, 8, DqChunks<8>::value>::kBytes;
  return FacesDqLayout<T, NS, 16, DqChunks<16>::value>::kBytes;
}

template <typename T, int NS>
cudaError_t Launch<T, NS>::faces_dq(const StageArgs<T> &a, const Tile *tiles, const void *maps, const ChemParams &C,
                                    int n_tiles, int ty, cudaStream_t s) {
  if constexpr (sizeof(T) != 4 || NS < 0) {
    return cudaErrorInvalidValue;  // FP32 bulk precision, compiled species counts only
  } else {
    if (n_tiles <= 0) return cudaSuccess;
    if (faces_dq_smem(ty) > 227 * 1024) return cudaErrorInvalidConfiguration;
    const CUtensorMap *m = (const CUtensorMap *)maps;
    if (ty == 4)
      k_faces_dq<T, NS, 4, DqChunks<4>::value><<<n_tiles, dim3(32, 4), faces_dq_smem(4), s>>>(a, tiles, m, C);
    else if (ty == 8)
      k_faces_dq<T, NS, 8, DqChunks<8>::value><<<n_tiles, dim3(32, 8), faces_dq_smem(8), s>>>(a, tiles, m, C);
    else if (ty == 16)
      k_faces_dq<T, NS, 16, DqChunks<16>::value><<<n_tiles, dim3(32, 16), faces_dq_smem(16), s>>>(a, tiles, m, C);
    else
      return cudaErrorInvalidValue;
    return cudaGetLastError();
  }
}

template <typename T, int NS>
cudaError_t Launch<T, NS>::faces_tma_persistent(const StageArgs<T> &a, const Tile *tiles, int ty, int tx,
                                                const void *maps, const ChemParams &C, int n_tiles, unsigned *ticket,
                                                cudaStream_t s) {
  if (n_tiles <= 0) return cudaSuccess;
  const size_t smem = faces_tma_smem(ty, tx);
  if (smem == 0) return cudaErrorInvalidConfiguration;
  const CUtensorMap *m = (const CUtensorMap *)maps;
  return with_face_shape(ty, tx, [&](auto ty_c, auto tx_c) -> cudaError_t {
    constexpr int TY = decltype(ty_c)::value, TX = decltype(tx_c)::value;
    if constexpr (!FacesTmaLayout<T, NS, TY, TX>::kOk) {
      return cudaErrorInvalidConfiguration;
    } else {
      static int per_sm = 0, n_sm = 0;  // CTAs per SM of this shape, SMs
      if (per_sm == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_faces_tma_persistent<T, NS, TY, TX>, TX * TY, smem);
        per_sm = std::max(1, per_sm);
      }
      cudaError_t e = cudaMemsetAsync(ticket, 0, sizeof(unsigned), s);
      if (e != cudaSuccess) return e;
      const int grid = std::min(n_tiles, n_sm * per_sm);
      k_faces_tma_persistent<T, NS, TY, TX><<<grid, dim3(TX, TY), smem, s>>>(a, tiles, m, C, n_tiles, ticket);
      return cudaGetLastError();
    }
  });
}

template <typename T, int NS>
cudaError_t Launch<T, NS>::update(const StageArgs<T> &a, const ChemParams &C, int n_tiles, cudaStream_t s,
                                  int high_occ, int ux) {
  if (n_tiles <= 0) return cudaSuccess;
  if (ux != 32 && ux != 16) return cudaErrorInvalidValue;
  const dim3 block(ux, 256 / ux);
  if constexpr (sizeof(T) == 4) {
    if (high_occ) {
      if (ux == 16)
        k_update<T, NS, 4, 16><<<n_tiles, block, update_smem(), s>>>(a, C);
      else
        k_update<T, NS, 4, 32><<<n_tiles, block, update_smem(), s>>>(a, C);
      return cudaGetLastError();
    }
  }
  constexpr int kMinb = sizeof(T) == 8 ? 2 : 3;
  if (ux == 16)
    k_update<T, NS, kMinb, 16><<<n_tiles, block, update_smem(), s>>>(a, C);
  else
    k_update<T, NS, kMinb, 32><<<n_tiles, block, update_smem(), s>>>(a, C);
  return cudaGetLastError();
}

template <typename T, int NS>
cudaError_t Launch<T, NS>::props_mlp(const T *P, T *Pr, int64_t N, const void *cl, unsigned *status,
                                     const ChemParams &C, cudaStream_t s) {
  if constexpr (NS == 0) {
    return cudaErrorInvalidValue;  // the closure is for mixtures
  } else {
    if (N <= 0) return cudaSuccess;
    static bool attr_set = false;  // the weights, operands and hi/lo activations take more than 48 KB
    if (!attr_set) {
      cudaError_t e = cudaFuncSetAttribute(k_props_mlp<T, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMlpSmem);
      if (e != cudaSuccess) return e;
      attr_set = true;
    }
    int dev = 0, n_sm = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    const int64_t tiles = (N + kMlpRows - 1) / kMlpRows;
    const int grid = (int)std::min<int64_t>(tiles, (int64_t)n_sm * 3);  // 3 CTAs per SM fit (64 KB each)
    k_props_mlp<T, NS><<<grid, kMlpRows, kMlpSmem, s>>>(P, Pr, N, *static_cast<const ClosureDev *>(cl), status, C);
    return cudaGetLastError();
  }
}

template <typename T, int NS>
cudaError_t Launch<T, NS>::gcl(const BlockInfo *blocks, int nblocks, const T *G, int64_t N, int64_t n_interior,
                               double *out, cudaStream_t s) {
  const int tpb = 256;
  int64_t nb = (n_interior + tpb - 1) / tpb;
  if (nb > 148 * 16) nb = 148 * 16;
  if (nb < 1) return cudaSuccess;
  k_gcl<T><<<(unsigned)nb, tpb, 0, s>>>(blocks, nblocks, G, N, n_interior, out);
  return cudaGetLastError();
}

template <typename T, int NS>
cudaError_t Launch<T, NS>::configure() {
  cudaError_t e = cudaFuncSetAttribute(k_stage<T, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage_smem());
  if (e != cudaSuccess) return e;
  if (stage_tma_smem() <= 227 * 1024)
    e = cudaFuncSetAttribute(k_stage_tma<T, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage_tma_smem());
  for (const int sh : {0, 1, 2, 3, 4}) {  // every tile shape of the TMA face kernel whose ring fits
    const int ty = sh == 0 ? 4 : (sh == 1 || sh == 3 ? 8 : 16), tx = sh < 3 ? 32 : 16;
    with_face_shape(ty, tx, [&](auto ty_c, auto tx_c) -> cudaError_t {
      constexpr int TY = decltype(ty_c)::value, TX = decltype(tx_c)::value;
      if constexpr (FacesTmaLayout<T, NS, TY, TX>::kOk) {
        const int bytes = (int)FacesTmaLayout<T, NS, TY, TX>::kBytes;
        if (e == cudaSuccess)
          e = cudaFuncSetAttribute(k_faces_tma<T, NS, TY, TX>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e == cudaSuccess)
          e = cudaFuncSetAttribute(k_faces_tma_persistent<T, NS, TY, TX>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
      }
      return cudaSuccess;
    });
  }
  if constexpr (NS != 0) {  // the closure kernel (set here too, before any stream capture)
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_props_mlp<T, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMlpSmem);
  }
  if constexpr (sizeof(T) == 4 && NS >= 0) {
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_faces_dq<T, NS, 4, DqChunks<4>::value>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)faces_dq_smem(4));
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_faces_dq<T, NS, 8, DqChunks<8>::value>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)faces_dq_smem(8));
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_faces_dq<T, NS, 16, DqChunks<16>::value>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)faces_dq_smem(16));
  }
  return e;
}

template <typename T, int NS>
cudaError_t Launch<T, NS>::stage_tma(const StageArgs<T> &a, const void *maps, const ChemParams &C, int n_tiles,
                                     cudaStream_t s) {
  if (n_tiles <= 0) return cudaSuccess;
  if (stage_tma_smem() > 227 * 1024) return cudaErrorInvalidConfiguration;
  k_stage_tma<T, NS><<<n_tiles, dim3(kTX, kTY), stage_tma_smem(), s>>>(a, (const CUtensorMap *)maps, C);
  return cudaGetLastError();
}

template <typename T, int NS>
cudaError_t Launch<T, NS>::stage(const StageArgs<T> &a, const ChemParams &C, int n_tiles, cudaStream_t s) {
  if (n_tiles <= 0) return cudaSuccess;
  k_stage<T, NS><<<n_tiles, dim3(kTX, kTY), stage_smem(), s>>>(a, C);
  return cudaGetLastError();
}

template <typename T, int NS>
cudaError_t Launch<T, NS>::lusgs_rhs(const StageArgs<T> &a, const LusgsArgs &L, const ChemParams &C, int n_tiles,
                                     cudaStream_t s) {
  if (n_tiles <= 0) return cudaSuccess;
  k_lusgs_rhs<T, NS><<<n_tiles, dim3(kTX, kTY), 0, s>>>(a, L, C);
  return cudaGetLastError();
}

template <typename T, int NS>
cudaError_t Launch<T, NS>::lusgs_sweep(const LusgsArgs &L, const ChemParams &C, int dir, cudaStream_t s) {
  const int64_t n = L.s1 - L.s0;
  if (n <= 0) return cudaSuccess;
  if (L.lp != LusgsLane<NS, 1>::LP) return cudaErrorInvalidValue;  // rows laid out for another lane count
  const int pts = kSweepThreads / LusgsLane<NS, 1>::LP;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)((n + pts - 1) / pts));
  cfg.blockDim = dim3(kSweepThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;  // programmatic dependent launch
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (dir > 0) return cudaLaunchKernelEx(&cfg, k_lusgs_sweep<NS, 1>, L, C);
  return cudaLaunchKernelEx(&cfg, k_lusgs_sweep<NS, -1>, L, C);
}

template <typename T, int NS>
cudaError_t Launch<T, NS>::lusgs_update(const StageArgs<T> &a, const LusgsArgs &L, const ChemParams &C, int n_tiles,
                                        cudaStream_t s) {
  if (n_tiles <= 0) return cudaSuccess;
  k_lusgs_update<T, NS><<<n_tiles, dim3(kTX, kTY), update_smem(), s>>>(a, L, C);
  return cudaGetLastError();
}

template <typename T, int NS>
cudaError_t Launch<T, NS>::halo_nodes(const HaloArgs<T> &a, const ChemParams &C, cudaStream_t s) {
  const int64_t n = a.end - a.begin;
  if (n <= 0) return cudaSuccess;
  const int tpb = 128;
  k_halo_nodes<T, NS><<<(unsigned)((n + tpb - 1) / tpb), tpb, 0, s>>>(a, C);
  return cudaGetLastError();
}

template <typename T, int NS>
cudaError_t Launch<T, NS>::halo_copies(const HaloArgs<T> &a, const ChemParams &C, double *vel,
                                       const int64_t *vel_zero, int64_t n_vel_zero, cudaStream_t s, int q_filter,
                                       bool only_q) {
  const int64_t n = std::max<int64_t>(a.end - a.begin, vel ? n_vel_zero : 0);
  if (n <= 0) return cudaSuccess;
  const int ns = C.ns, np = 6 + ns, npr = 2 + ns, nq = 5 + ns;
  const int tpb = 256;
  k_halo_copy_fields<T, NS><<<dim3((unsigned)((n + tpb - 1) / tpb), only_q ? 1 : 3), tpb, 0, s>>>(
      a, C, np, npr, nq, vel, vel_zero, n_vel_zero, q_filter, only_q ? 2 : 0);
  return cudaGetLastError();
}

template <typename T, int NS>
cudaError_t Launch<T, NS>::halo_levels(const HaloArgs<T> &a, const ChemParams &C, const HaloLevels &lv,
                                       GridBarrier *bar, unsigned *status, cudaStream_t s) {
  const int tpb = 128;
  static int capacity = 0;  // CTAs that fit on the device at once
  if (capacity == 0) {
    int dev = 0, n_sm = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_halo_levels<T, NS>, tpb, 0);
    capacity = std::max(1, n_sm * per_sm);
  }
  int64_t work = 1;
  for (int l = 0; l < lv.n; ++l) work = std::max(work, lv.begin[l + 1] - lv.begin[l]);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(capacity, (work + tpb - 1) / tpb));
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(tpb);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;  // every CTA resident: the grid barriers can complete
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_halo_levels<T, NS>, a, C, lv, bar, status);
}

template <typename T, int NS>
cudaError_t Launch<T, NS>::cv_from_bv(const ChemParams &C, const double *P0, double *Q, int64_t N, double *vel,
                                      cudaStream_t s) {
  const int tpb = 256;
  k_cv_from_bv<NS><<<(unsigned)((N + tpb - 1) / tpb), tpb, 0, s>>>(C, P0, Q, N, vel);
  return cudaGetLastError();
}

template <typename T, int NS>
cudaError_t Launch<T, NS>::props_all(const ChemParams &C, const T *P, T *Pr, int64_t N, cudaStream_t s) {
  const int tpb = 128;
  k_props_all<T, NS><<<(unsigned)((N + tpb - 1) / tpb), tpb, 0, s>>>(C, P, Pr, N);
  return cudaGetLastError();
}

template <typename T, int NS>
cudaError_t Launch<T, NS>::dt_reduce(const ChemParams &C, const BlockInfo *blocks, int nblocks, const T *P,
                                     const T *Pr, const T *G, int64_t N, int64_t n_interior,
                                     unsigned long long *dt_out, cudaStream_t s) {
  const int tpb = 256;
  int64_t nb = (n_interior + tpb - 1) / tpb;
  if (nb > 148 * 16) nb = 148 * 16;
  k_dt_reduce<T, NS><<<(unsigned)nb, tpb, 0, s>>>(C, blocks, nblocks, P, Pr, G, N, n_interior, dt_out);
  return cudaGetLastError();
}

#define CCB_INSTANTIATE(T, NS) template struct Launch<T, NS>;

}  // namespace ccb
