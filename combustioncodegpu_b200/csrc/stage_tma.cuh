// Stage kernel with the primitive planes of each tile staged in shared memory
// by the Tensor Memory Accelerator (sm_100a), used by the mixed-precision path.
//
// Same work decomposition as k_stage (a kTX x kTY column of points swept
// along k, faces exchanged through shared memory, fused RK update), but every
// stencil read of the primitives hits shared memory: a ring of kSlots planes,
// each the tile plus a 2-point halo in i and j (kHX x kHY points) for all
// 6+ns primitive fields, filled by one cp.async.bulk.tensor (4D tensor map:
// i, j, k, field) per plane and completed on an mbarrier.  Plane k+4 is
// requested into the slot of plane k-1 as soon as the faces of plane k are
// done, so copies run two planes ahead of the sweep and overlap the point
// updates.  Transport properties and geometry are read through L1.
//
// Waits are bounded: a CTA whose plane does not arrive within C.max_spins
// polls sets kStatusTmaTimeout in the status word, waits (at most kMaxSpins
// polls each) for the copies it has in flight and leaves the sweep.
#pragma once
#include <cuda.h>

#include "stage.cuh"

namespace ccb {

constexpr int kHX = kTX + 4;               // staged points along i (i0-2 .. i0+kTX+1)
constexpr int kHY = kTY + 4;               // staged points along j
constexpr int kPlaneVals = kHX * kHY;      // values per field and plane
constexpr int kSlots = 5;                  // planes in flight: k-1 .. k+3
constexpr unsigned kStatusTmaTimeout = 8u;
constexpr long long kMaxSpins = kDefaultWaitSpins;  // bound of the drain after an abort

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Non-blocking check of the same phase (no suspension).
__device__ __forceinline__ bool mbar_test_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for a phase: one non-blocking check, then at most max_polls
// potentially suspending polls (a limit of 0 gives up unless the phase has
// already completed).  Returns false when it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity, long long max_polls) {
  bool ok = mbar_test_wait(bar, parity);
  for (long long s = 0; !ok && s < max_polls; ++s) ok = mbar_try_wait(bar, parity);
  return ok;
}

// One plane: box {kHX, kHY, 1, nf} at (x, y, z, 0) of the block's tensor map.
__device__ __forceinline__ void tma_load_plane(void *dst, const CUtensorMap *map, int x, int y, int z,
                                               uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(0), "r"(smem_u32(bar))
      : "memory");
}

// Primitives around one face from the plane ring: planes k-1 .. k+2 at
// pm, p0, p1, p2; the face's first point at in-plane index q of plane k.
// Scalar plane pointers (not an array): a runtime-indexed array would be
// placed in local memory.  t and c are compile-time after unrolling; d is
// the runtime face direction.
template <typename T>
struct SmemStencil {
  const T *pm, *p0, *p1, *p2;
  int q, d;
  __device__ __forceinline__ const T *plane(int r) const {  // r = 0..3 -> k-1 .. k+2
    return r == 0 ? pm : (r == 1 ? p0 : (r == 2 ? p1 : p2));
  }
  __device__ __forceinline__ T at(int f, int t) const {
    if (d == 2) return plane(1 + t)[f * kPlaneVals + q];
    return p0[f * kPlaneVals + q + t * (d == 0 ? 1 : kHX)];
  }
  __device__ __forceinline__ T cross(int f, int c, int sg, int t) const {
    if (c == 2) {  // neighbour plane of the base point (k or k+t along z)
      if (d == 2) return plane(1 + t + sg)[f * kPlaneVals + q];
      return plane(1 + sg)[f * kPlaneVals + q + t * (d == 0 ? 1 : kHX)];
    }
    const int cs = sg * (c == 0 ? 1 : kHX);
    if (d == 2) return plane(1 + t)[f * kPlaneVals + q + cs];
    return p0[f * kPlaneVals + q + t * (d == 0 ? 1 : kHX) + cs];
  }
};

template <typename T, int NS>
struct TmaLayout {
  static constexpr int kNP = 6 + SpecCount<NS>::kArr;  // primitive fields
  static constexpr int kNV = 5 + SpecCount<NS>::kArr;  // conserved / flux components
  static constexpr size_t kPlaneBytes = ((sizeof(T) * kNP * kPlaneVals + 127) / 128) * 128;
  static constexpr int XS = kTY * (kTX + 1), YS = (kTY + 1) * kTX, ZS = kTY * kTX;
  static constexpr size_t kFluxBytes = ((sizeof(T) * kNV * (XS + YS + 2 * ZS) + 15) / 16) * 16;
  static constexpr size_t kRecD = sizeof(double) * SpecCount<NS>::kArr * 2 * kRecLen;
  static constexpr size_t kRecBytes = kRecD + (sizeof(T) == sizeof(double) ? 0 : sizeof(T) * SpecCount<NS>::kArr * 2 * kRecLen);
  // alignment slack + barriers + ring + fluxes + NASA records (FP64, bulk)
  static constexpr size_t kBytes = 128 + 128 + kSlots * kPlaneBytes + kFluxBytes + kRecBytes;
};

template <typename T, int NS>
__global__ void __launch_bounds__(kTX *kTY, 1)
    k_stage_tma(const StageArgs<T> a, const CUtensorMap *__restrict__ maps, const __grid_constant__ ChemParams C) {
  using L = TmaLayout<T, NS>;
  constexpr int A = SpecCount<NS>::kArr;
  constexpr int NV = L::kNV;
  const int ns = SpecCount<NS>::n(C);
  const int nv = 5 + ns;
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  // TMA destinations must be 128-byte aligned: align the carve-up explicitly
  unsigned char *smem_raw = smem_dyn + ((128u - (smem_u32(smem_dyn) & 127u)) & 127u);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
  unsigned char *ring = smem_raw + 128;
  T *sFx = reinterpret_cast<T *>(ring + kSlots * L::kPlaneBytes);
  T *sFy = sFx + NV * L::XS;
  T *sFz0 = sFy + NV * L::YS;
  T *sFz1 = sFz0 + NV * L::ZS;
  double *sRecD = reinterpret_cast<double *>(reinterpret_cast<unsigned char *>(sFx) + L::kFluxBytes);
  T *sRec = reinterpret_cast<T *>(reinterpret_cast<unsigned char *>(sRecD) +
                                  (sizeof(T) == sizeof(double) ? 0 : L::kRecD));
  constexpr int XS = L::XS, YS = L::YS, ZS = L::ZS;

  const Tile t = a.tiles[blockIdx.x];
  const BlockInfo B = a.blocks[t.blk];
  const CUtensorMap *map = maps + t.blk;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * kTX + tx;
  const int i = t.i0 + tx, j = t.j0 + ty;
  const bool act = (i < B.mx) && (j < B.my);
  const int N = (int)a.N;
  const int sj = B.nx, sk = B.nx * B.ny;
  const int col = (int)B.base + i + sj * j;
  const T *__restrict__ P = a.P;
  const T *__restrict__ Pr = a.Pr;
  const T *__restrict__ G = a.G;
  const bool three_d = B.mz > 1;
  const unsigned plane_bytes = (unsigned)(sizeof(T) * (6 + ns) * kPlaneVals);
  // tensor coordinates of plane kp: x = i0 - 2 + g, y = j0 - 2 + g, z = kp + g
  const int tx0 = t.i0 - 2 + B.g, ty0 = t.j0 - 2 + B.g;
  const int kfirst = t.k0 - 2, klast = t.k1 + 1;  // planes the sweep reads

  for (int e = tid, nrec = ns * 2 * kRecLen; e < nrec; e += kTX * kTY) {
    sRecD[e] = param_rec<double>(C)[e];
    if (sizeof(T) != sizeof(double)) sRec[e] = param_rec<T>(C)[e];
  }
  if (tid == 0) {
    for (int b = 0; b < kSlots; ++b) mbar_init(&bars[b], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(map))
                 : "memory");
  }
  __syncthreads();
  // plane kp lives in slot (kp - kfirst) % kSlots; it is that slot's n-th
  // load with n = (kp - kfirst) / kSlots, completed when phase n ends
  auto slot_of = [&](int kp) { return (kp - kfirst) % kSlots; };
  auto parity_of = [&](int kp) { return (unsigned)(((kp - kfirst) / kSlots) & 1); };
  int k_issued = kfirst - 1;
  if (tid == 0) {
    for (int kp = kfirst; kp <= klast && kp < kfirst + kSlots; ++kp) {
      const int sl = slot_of(kp);
      mbar_arrive_expect_tx(&bars[sl], plane_bytes);
      tma_load_plane(ring + sl * L::kPlaneBytes, map, tx0, ty0, kp + B.g, &bars[sl]);
    }
  }
  k_issued = min(klast, kfirst + kSlots - 1);

  const int q = (ty + 2) * kHX + (tx + 2);  // in-plane index of this thread's point
  const bool ex_x = (ty == 1) && (tx < kTY) && (t.j0 + tx < B.my);
  const bool ex_y = (ty == 0) && act;
  unsigned flags = 0;
  double dt_min = 1e300;
  T *zprev = sFz1, *zcur = sFz0;
  T F[NV];
  bool aborted = false;

  for (int k = t.k0 - 1; k < t.k1; ++k) {
    // planes k-1 .. k+2 must be resident
    bool late = false;
    for (int kp = k - 1; kp <= k + 2 && !late; ++kp)
      late = !mbar_wait_bounded(&bars[slot_of(kp)], parity_of(kp), C.max_spins);
    if (__syncthreads_or(late)) {
      if (tid == 0) atomicOr(a.status, kStatusTmaTimeout);
      aborted = true;
      break;
    }
    const T *plm = reinterpret_cast<const T *>(ring + slot_of(k - 1) * L::kPlaneBytes);
    const T *pl0 = reinterpret_cast<const T *>(ring + slot_of(k) * L::kPlaneBytes);
    const T *pl1 = reinterpret_cast<const T *>(ring + slot_of(k + 1) * L::kPlaneBytes);
    const T *pl2 = reinterpret_cast<const T *>(ring + slot_of(k + 2) * L::kPlaneBytes);
    const int p = col + sk * k;
    const bool first = (k < t.k0);
#pragma unroll 1
    for (int it = 0; it < 5; ++it) {
      bool doit;
      int d, sd, qq = q, gp = p;
      T *dst;
      int ds;
      if (it == 0) {
        doit = act && three_d;
        d = 2, sd = sk, dst = zcur + ty * kTX + tx, ds = ZS;
      } else if (it == 1) {
        doit = act && !first;
        d = 0, sd = 1, dst = sFx + ty * (kTX + 1) + tx + 1, ds = XS;
      } else if (it == 2) {
        doit = act && !first;
        d = 1, sd = sj, dst = sFy + (ty + 1) * kTX + tx, ds = YS;
      } else if (it == 3) {
        doit = ex_x && !first;
        d = 0, sd = 1, dst = sFx + tx * (kTX + 1), ds = XS;
        qq = (tx + 2) * kHX + 1;  // row tx of the tile, i = i0 - 1
        gp = (int)B.base + (t.i0 - 1) + sj * (t.j0 + tx) + sk * k;
      } else {
        doit = ex_y && !first;
        d = 1, sd = sj, dst = sFy + tx, ds = YS;
        qq = q - kHX;
        gp = p - sj;
      }
      if (doit) {
        SmemStencil<T> S{plm, pl0, pl1, pl2, qq, d};
        face_flux_gen<T, NS>(C, sRec, S, Pr, G, N, gp, sd, d, F);
#pragma unroll
        for (int l = 0; l < NV; ++l)
          if (l < nv) dst[l * ds] = F[l];
      }
    }
    __syncthreads();  // faces of plane k written; plane k-1 no longer read
    {
      const int kp = k + 4;  // reuses the slot of plane k-1
      if (kp <= klast) {
        if (tid == 0) {
          const int sl = slot_of(kp);
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          mbar_arrive_expect_tx(&bars[sl], plane_bytes);
          tma_load_plane(ring + sl * L::kPlaneBytes, map, tx0, ty0, kp + B.g, &bars[sl]);
        }
        k_issued = kp;
      }
    }
    if (first) {
      T *tmp = zprev;
      zprev = zcur;
      zcur = tmp;
      continue;
    }
    if (act) {
      double dq[NV];
#pragma unroll
      for (int l = 0; l < NV; ++l) {
        if (l < nv) {
          T acc = (sFx[l * XS + ty * (kTX + 1) + tx + 1] - sFx[l * XS + ty * (kTX + 1) + tx]);
          acc += (sFy[l * YS + (ty + 1) * kTX + tx] - sFy[l * YS + ty * kTX + tx]);
          if (three_d) acc += (zcur[l * ZS + ty * kTX + tx] - zprev[l * ZS + ty * kTX + tx]);
          dq[l] = -(double)acc;
        }
      }
      const T *own = pl0;
      double dt;
      if (a.local_dt) {
        T Y[A];
#pragma unroll
        for (int l = 0; l < A; ++l)
          if (l < ns) Y[l] = own[(6 + l) * kPlaneVals + q];
        T gam, c;
        gamma_and_c<T, NS>(C, sRec, own[5 * kPlaneVals + q], Y, gam, c);
        dt = local_time_step<T>(C, G, N, p, (double)own[q], (double)own[kPlaneVals + q],
                                (double)own[2 * kPlaneVals + q], (double)own[3 * kPlaneVals + q], (double)c,
                                (double)gam, (double)Pr[p], three_d);
      } else {
        dt = *a.dt;
      }
      point_update<T, NS>(C, sRec, sRecD, a, p, N, dq, dt, (double)own[5 * kPlaneVals + q], three_d, flags, dt_min);
      (void)P;
    }
    T *tmp = zprev;
    zprev = zcur;
    zcur = tmp;
    __syncthreads();
  }
  if (aborted) {
    // let this CTA's copies in flight land before the CTA exits (bounded)
    if (tid == 0) {
      for (int kp = max(kfirst, k_issued - kSlots + 1); kp <= k_issued; ++kp) {
        long spins = 0;
        while (!mbar_try_wait(&bars[slot_of(kp)], parity_of(kp)) && ++spins < kMaxSpins) {
        }
      }
    }
    __syncthreads();
    return;
  }
  if (a.dt_next) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dt_min = fmin(dt_min, __shfl_xor_sync(0xffffffffu, dt_min, o));
    if (tx == 0) atomic_min_pos_double(a.dt_next, dt_min);
  }
  const unsigned any = __reduce_or_sync(0xffffffffu, flags);
  if (any && tx == 0) atomicOr(a.status, any);
}

}  // namespace ccb

namespace ccb {

// Primitives around one face from a ring of planes HX points wide with PV
// values per field (the same access pattern as SmemStencil, for any tile
// height).
template <typename T, int HX, int PV>
struct SmemStencilT {
  const T *pm, *p0, *p1, *p2;
  int q, d;
  __device__ __forceinline__ const T *plane(int r) const {  // r = 0..3 -> k-1 .. k+2
    return r == 0 ? pm : (r == 1 ? p0 : (r == 2 ? p1 : p2));
  }
  __device__ __forceinline__ T at(int f, int t) const {
    if (d == 2) return plane(1 + t)[f * PV + q];
    return p0[f * PV + q + t * (d == 0 ? 1 : HX)];
  }
  __device__ __forceinline__ T cross(int f, int c, int sg, int t) const {
    if (c == 2) {
      if (d == 2) return plane(1 + t + sg)[f * PV + q];
      return plane(1 + sg)[f * PV + q + t * (d == 0 ? 1 : HX)];
    }
    const int cs = sg * (c == 0 ? 1 : HX);
    if (d == 2) return plane(1 + t)[f * PV + q + cs];
    return p0[f * PV + q + t * (d == 0 ? 1 : HX) + cs];
  }
};

// Face kernel of the split stage with TMA-staged primitive planes: the
// regular tiles of k_faces, each computing the +x, +y, +z faces of its points
// from a ring of 4 planes (k-1 .. k+2) in shared memory; plane k+3 is
// requested into the slot of plane k-1 once the faces of plane k are done.
// The tile is 32 (i, one warp per row) x TY (j) points: TY = 8 fits the ring
// twice per SM in FP32 (once in FP64, 208 KB), TY = 4 three times in FP32,
// TY = 16 (16 warps, FP32 only) once.  Transport and geometry are read
// through L1; the edge tiles stay with k_faces.  Waits are bounded as in
// k_stage_tma.
template <typename T, int NS, int TY = kTY, int TX = kTX>
struct FacesTmaLayout {
  static constexpr int HX = TX + 4, HY = TY + 4, PV = HX * HY;
  static constexpr int kRing = 4;
  static constexpr size_t kPlaneBytes = ((sizeof(T) * (6 + SpecCount<NS>::kArr) * PV + 127) / 128) * 128;
  static constexpr size_t kRec = ((sizeof(T) * SpecCount<NS>::kArr * 2 * kRecLen + 15) / 16) * 16;
  // alignment slack + barriers + ring + NASA records
  static constexpr size_t kBytes = 128 + 128 + kRing * kPlaneBytes + kRec;
  // CTAs per SM that the shared memory allows (228 KB per SM, 1 KB reserved per CTA)
  static constexpr int kFit = (int)((228 * 1024) / (kBytes + 1024));
  static constexpr bool kOk = kBytes <= 227 * 1024;
  static constexpr int kMinBlocks = kFit < 1 ? 1 : (kFit > 3 ? 3 : kFit);
};

// One regular tile of the face kernel: fill the ring with planes k0-1 ..
// k0+2, then per plane k wait for k-1 .. k+2, compute the +z, +x, +y faces
// of the tile's points and request plane k+3 into the slot of k-1.  pc0 is
// the number of planes this CTA loaded before the tile: plane kp is the
// CTA's (pc0 + kp - k0 + 1)-th load, in slot (that count mod 4) with the
// slot's barrier at parity (count / 4) mod 2.  The mbarriers are initialised
// by the caller.  Returns the planes loaded; *aborted is set (uniformly) when
// a wait timed out, after the copies in flight have landed.
// While plane k is processed, bring into L2 the transport and geometry rows
// of plane kp = k + 2 (1-point halo in j, the tile's i span plus one point
// on each side), which the faces of plane k + 1 read for the first time
// through L1.  Rows are spread over the CTA's threads; a hint nothing waits on.
template <typename T, int TY, int TX>
__device__ __forceinline__ void prefetch_props_geometry(const StageArgs<T> &a, const BlockInfo &B, const Tile &t,
                                                        int kp, int npr, int tid) {
  const int N = (int)a.N, sj = B.nx, sk = B.nx * B.ny;
  const int j_lo = max(t.j0 - 1, -B.g), j_hi = min(t.j0 + TY + 1, B.my + B.g), nr = j_hi - j_lo;
  const int n = (npr + 10) * nr;
  for (int e = tid; e < n; e += TX * TY) {
    const int f = e / nr, j = j_lo + e % nr;
    const T *base = f < npr ? a.Pr + (size_t)f * N : a.G + (size_t)(f - npr) * N;
    const int row = (int)B.base + sk * kp + sj * j;
    l2_prefetch(base, N, row + t.i0 - 1, row + t.i0 + TX + 1);
  }
}

template <typename T, int NS, int TY, int TX>
__device__ __forceinline__ int faces_tma_tile(const StageArgs<T> &a, const CUtensorMap *map, const ChemParams &C,
                                              uint64_t *bars, unsigned char *ring, const T *sRec, const Tile &t,
                                              unsigned pc0, bool &aborted) {
  using L = FacesTmaLayout<T, NS, TY, TX>;
  constexpr int NV = 5 + SpecCount<NS>::kArr;
  const int ns = SpecCount<NS>::n(C);
  const int nv = 5 + ns;
  const BlockInfo B = a.blocks[t.blk];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i = t.i0 + tx, j = t.j0 + ty;
  const bool act = (i < B.mx) && (j < B.my);
  const int N = (int)a.N, sj = B.nx, sk = B.nx * B.ny;
  const int col = (int)B.base + i + sj * j;
  const bool three_d = B.mz > 1;
  const unsigned plane_bytes = (unsigned)(sizeof(T) * (6 + ns) * L::PV);
  // tensor coordinates of plane kp: x = i0 - 2 + g, y = j0 - 2 + g, z = kp + g
  const int tx0 = t.i0 - 2 + B.g, ty0 = t.j0 - 2 + B.g;
  const int kfirst = t.k0 - 1, klast = t.k1 + 1;  // planes the sweep reads
  auto slot_of = [&](int kp) { return (int)((pc0 + (unsigned)(kp - kfirst)) & (L::kRing - 1)); };
  auto parity_of = [&](int kp) { return ((pc0 + (unsigned)(kp - kfirst)) / L::kRing) & 1u; };
  const int k_pro = min(klast, kfirst + L::kRing - 1);
  // request plane kp into its slot (thread 0).  Bounds-checked builds verify
  // the tensor coordinates first (x on a 16-byte boundary, z inside the
  // block's ghosted extent) and skip a bad request, whose wait then gives up.
  auto issue = [&](int kp) {
#ifdef CC_BOUNDS_CHECK
    const bool ok = (tx0 * (int)sizeof(T)) % 16 == 0 && tx0 >= 0 && kp + B.g >= 0 && kp + B.g < B.nz;
    CCB_CHECK(C, ok);
    if (!ok) return;
#endif
    const int sl = slot_of(kp);
    mbar_arrive_expect_tx(&bars[sl], plane_bytes);
    tma_load_plane(ring + sl * L::kPlaneBytes, map, tx0, ty0, kp + B.g, &bars[sl]);
  };
  if (tid == 0) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(map))
                 : "memory");
    // a previous tile's threads read these slots through the generic proxy
    if (pc0 != 0) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    for (int kp = kfirst; kp <= k_pro; ++kp) issue(kp);
  }
  int k_issued = k_pro;

  const int q = (ty + 2) * L::HX + (tx + 2);  // in-plane index of this thread's point
  T F[NV];
  aborted = false;
  for (int k = t.k0; k < t.k1; ++k) {
    bool late = false;
    for (int kp = k - 1; kp <= k + 2 && !late; ++kp)
      late = !mbar_wait_bounded(&bars[slot_of(kp)], parity_of(kp), C.max_spins);
    if (__syncthreads_or(late)) {
      if (tid == 0) atomicOr(a.status, kStatusTmaTimeout);
      aborted = true;
      break;
    }
    const T *plm = reinterpret_cast<const T *>(ring + slot_of(k - 1) * L::kPlaneBytes);
    const T *pl0 = reinterpret_cast<const T *>(ring + slot_of(k) * L::kPlaneBytes);
    const T *pl1 = reinterpret_cast<const T *>(ring + slot_of(k + 1) * L::kPlaneBytes);
    const T *pl2 = reinterpret_cast<const T *>(ring + slot_of(k + 2) * L::kPlaneBytes);
    const int p = col + sk * k;
    // (FP64 only: measured faster there, slower in FP32, whose smaller rows
    // stay in L2 without it)
    if (sizeof(T) == 8 && k + 2 <= B.mz - 1 + B.g) prefetch_props_geometry<T, TY, TX>(a, B, t, k + 2, 2 + ns, tid);
    if (act) {
      // two faces interleaved in FP32 (their loads overlap: 0.74 -> 0.71 ms
      // per launch at 128^3 despite the spills); one at a time in FP64, and
      // all three interleaved spill too much (1.04 ms)
      constexpr int kUnroll = sizeof(T) == 4 ? 2 : 1;
#pragma unroll kUnroll
      for (int it = three_d ? 0 : 1; it < 3; ++it) {
        const int d = it == 0 ? 2 : it - 1;
        const int sd = d == 0 ? 1 : (d == 1 ? sj : sk);
        SmemStencilT<T, L::HX, L::PV> S{plm, pl0, pl1, pl2, q, d};
        face_flux_gen<T, NS>(C, sRec, S, a.Pr, a.G, N, p, sd, d, F);
#pragma unroll
        for (int l = 0; l < NV; ++l)
          if (l < nv) a.faces[(d * nv + l) * N + p] = F[l];
      }
    }
    __syncthreads();  // plane k-1 is no longer read
    if (k + 3 <= klast) {
      if (tid == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue(k + 3);
      }
      k_issued = k + 3;
    }
  }
  if (aborted) {
    // let this CTA's copies in flight land before it leaves (bounded)
    if (tid == 0)
      for (int kp = max(kfirst, k_issued - L::kRing + 1); kp <= k_issued; ++kp) {
        long long spins = 0;
        while (!mbar_try_wait(&bars[slot_of(kp)], parity_of(kp)) && ++spins < kMaxSpins) {
        }
      }
    __syncthreads();
  }
  return klast - kfirst + 1;
}

template <typename T, int NS, int TY, int TX = kTX>
__global__ void __launch_bounds__(TX *TY, (FacesTmaLayout<T, NS, TY, TX>::kMinBlocks))
    k_faces_tma(const StageArgs<T> a, const Tile *__restrict__ tiles, const CUtensorMap *__restrict__ maps,
                const __grid_constant__ ChemParams C) {
  using L = FacesTmaLayout<T, NS, TY, TX>;
  const int ns = SpecCount<NS>::n(C);
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char *smem_raw = smem_dyn + ((128u - (smem_u32(smem_dyn) & 127u)) & 127u);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
  unsigned char *ring = smem_raw + 128;
  T *sRec = reinterpret_cast<T *>(ring + L::kRing * L::kPlaneBytes);
  const int tid = threadIdx.y * TX + threadIdx.x;
  const Tile t = tiles[blockIdx.x];
  for (int e = tid, nrec = ns * 2 * kRecLen; e < nrec; e += TX * TY) sRec[e] = param_rec<T>(C)[e];
  if (tid == 0) {
    for (int b = 0; b < L::kRing; ++b) mbar_init(&bars[b], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  bool aborted;
  faces_tma_tile<T, NS, TY, TX>(a, maps + t.blk, C, bars, ring, sRec, t, 0u, aborted);
}

// Persistent form of k_faces_tma: as many CTAs as fit on the GPU take the
// regular tiles in order from a device counter (zeroed before the launch),
// initialising the NASA records and the mbarriers once; the plane count
// carries the mbarrier phases from one tile to the next.
template <typename T, int NS, int TY, int TX = kTX>
__global__ void __launch_bounds__(TX *TY, (FacesTmaLayout<T, NS, TY, TX>::kMinBlocks))
    k_faces_tma_persistent(const StageArgs<T> a, const Tile *__restrict__ tiles, const CUtensorMap *__restrict__ maps,
                           const __grid_constant__ ChemParams C, int n_tiles, unsigned *ticket) {
  using L = FacesTmaLayout<T, NS, TY, TX>;
  const int ns = SpecCount<NS>::n(C);
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char *smem_raw = smem_dyn + ((128u - (smem_u32(smem_dyn) & 127u)) & 127u);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
  unsigned char *ring = smem_raw + 128;
  T *sRec = reinterpret_cast<T *>(ring + L::kRing * L::kPlaneBytes);
  __shared__ int sh_tile;
  const int tid = threadIdx.y * TX + threadIdx.x;
  for (int e = tid, nrec = ns * 2 * kRecLen; e < nrec; e += TX * TY) sRec[e] = param_rec<T>(C)[e];
  if (tid == 0) {
    for (int b = 0; b < L::kRing; ++b) mbar_init(&bars[b], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  unsigned pc = 0;
  for (;;) {
    if (tid == 0) sh_tile = (int)atomicAdd(ticket, 1u);
    __syncthreads();
    const int ti = sh_tile;
    __syncthreads();  // every thread has its tile index before the next ticket
    if (ti >= n_tiles) break;
    bool aborted;
    pc += (unsigned)faces_tma_tile<T, NS, TY, TX>(a, maps + tiles[ti].blk, C, bars, ring, sRec, tiles[ti], pc, aborted);
    if (aborted) break;
  }
}

}  // namespace ccb
