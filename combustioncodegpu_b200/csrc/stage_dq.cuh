// Face kernel that differences the faces inside the tile (sm_100a).
//
// Same plane ring as k_faces_tma (the primitives of planes k-1 .. k+2 of a
// tile, 2-point halo in i and j, staged in shared memory by
// cp.async.bulk.tensor on mbarriers), but instead of writing the three face
// fluxes of every point to a face arena ([3][n_var][N]) for the update kernel
// to difference, the CTA differences them itself and writes the point's
// residual dq = -(F(i+1/2) - F(i-1/2) + F(j+1/2) - F(j-1/2) + F(k+1/2) -
// F(k-1/2)) ([n_var][N]), the reference's dq (TimeAdvanceFunc.cu:61-243).
// Per plane k every thread computes the +x, +y, +z faces of its point; the
// -x face of a point is the +x face of the lane to its left (a warp shuffle;
// warp 1 computes the tile's -x boundary faces, one per row), the -y face is
// the +y face of the row below (exchanged through shared memory in chunks of
// fields; warp 0 computes the tile's -y boundary faces), and the -z face is
// the +z face of the plane below, which the thread stored as a partial sum in
// its own dq slot of plane k+1 one plane earlier.  A tile of k-chunk
// [k0, k1) starts with a prologue plane k0-1 that only computes the +z faces
// (the -z faces of plane k0).  No block needs separate edge tiles.
//
// Every face goes through the single face_flux_gen call site in the loop over
// `it`, so a face computed by two tiles (a k-chunk boundary, a tile boundary
// in i or j) is computed by the same instructions.
//
// The tile is 32 (i, one warp per row) x TY (j) points; the ring, the y
// exchange (chunks of fields, NCH chunks) and the boundary-face buffers fit
// 3 CTAs per SM for TY = 4, 2 for TY = 8 and 1 (16 warps) for TY = 16 in the
// FP32 bulk precision.  Waits are bounded as in k_faces_tma.
#pragma once
#include "stage_tma.cuh"

namespace ccb {

constexpr size_t round_up(size_t x, size_t m) { return (x + m - 1) / m * m; }

template <typename T, int NS, int TY, int NCH>
struct FacesDqLayout {
  static constexpr int TX = 32, HX = TX + 4, HY = TY + 4, PV = HX * HY;
  static constexpr int A = SpecCount<NS>::kArr;
  static constexpr int kNP = 6 + A, kNV = 5 + A;
  static constexpr int kRing = 4;
  static constexpr int kChunk = (kNV + NCH - 1) / NCH;  // fields per y-exchange round
  static constexpr size_t kPlaneBytes = round_up(sizeof(T) * kNP * PV, 128);
  static constexpr size_t kXch = round_up(sizeof(T) * kChunk * (TY - 1) * TX, 16);  // +y faces of rows 0..TY-2
  static constexpr size_t kYm = round_up(sizeof(T) * kNV * TX, 16);                 // -y boundary faces
  static constexpr size_t kXm = round_up(sizeof(T) * kNV * TY, 16);                 // -x boundary faces
  static constexpr size_t kRec = round_up(sizeof(T) * A * 2 * kRecLen, 16);
  // alignment slack + barriers + ring + exchange + boundary faces + NASA records
  static constexpr size_t kBytes = 128 + 128 + kRing * kPlaneBytes + kXch + kYm + kXm + kRec;
  static constexpr int kMinBlocks = TY == 4 ? 3 : (TY == 8 ? 2 : 1);
};

template <typename T, int NS, int TY, int NCH>
__global__ void __launch_bounds__(32 * TY, (FacesDqLayout<T, NS, TY, NCH>::kMinBlocks))
    k_faces_dq(const StageArgs<T> a, const Tile *__restrict__ tiles, const CUtensorMap *__restrict__ maps,
               const __grid_constant__ ChemParams C) {
  using L = FacesDqLayout<T, NS, TY, NCH>;
  constexpr int TX = L::TX, HX = L::HX, PV = L::PV, NV = L::kNV, CH = L::kChunk;
  using Stencil = SmemStencilT<T, HX, PV>;
  const int ns = SpecCount<NS>::n(C);
  const int nv = 5 + ns;
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char *smem_raw = smem_dyn + ((128u - (smem_u32(smem_dyn) & 127u)) & 127u);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
  unsigned char *ring = smem_raw + 128;
  T *sX = reinterpret_cast<T *>(ring + L::kRing * L::kPlaneBytes);           // [CH][TY-1][TX]
  T *sYm = reinterpret_cast<T *>(reinterpret_cast<unsigned char *>(sX) + L::kXch);   // [NV][TX]
  T *sXm = reinterpret_cast<T *>(reinterpret_cast<unsigned char *>(sYm) + L::kYm);   // [NV][TY]
  T *sRec = reinterpret_cast<T *>(reinterpret_cast<unsigned char *>(sXm) + L::kXm);
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  for (int e = tid, nrec = ns * 2 * kRecLen; e < nrec; e += TX * TY) sRec[e] = param_rec<T>(C)[e];
  if (tid == 0) {
    for (int b = 0; b < L::kRing; ++b) mbar_init(&bars[b], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  const Tile t = tiles[blockIdx.x];
  const BlockInfo B = a.blocks[t.blk];
  const CUtensorMap *map = maps + t.blk;
  const int i = t.i0 + tx, j = t.j0 + ty;
  const bool act = (i < B.mx) && (j < B.my);
  const int N = (int)a.N, sj = B.nx, sk = B.nx * B.ny;
  const int col = (int)B.base + i + sj * j;
  const bool three_d = B.mz > 1;
  const unsigned plane_bytes = (unsigned)(sizeof(T) * (6 + ns) * PV);
  // tensor coordinates of plane kp: x = i0 - 2 + g, y = j0 - 2 + g, z = kp + g
  const int tx0 = t.i0 - 2 + B.g, ty0 = t.j0 - 2 + B.g;
  const int kstart = three_d ? t.k0 - 1 : t.k0;  // prologue plane k0 - 1: the -z faces of plane k0
  const int kfirst = kstart - 1, klast = t.k1 + 1;  // planes the sweep reads
  auto slot_of = [&](int kp) { return (kp - kfirst) & (L::kRing - 1); };
  auto parity_of = [&](int kp) { return (unsigned)(((kp - kfirst) / L::kRing) & 1); };
  const int k_pro = min(klast, kfirst + L::kRing - 1);
  if (tid == 0) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(map))
                 : "memory");
    for (int kp = kfirst; kp <= k_pro; ++kp) {
      const int sl = slot_of(kp);
      mbar_arrive_expect_tx(&bars[sl], plane_bytes);
      tma_load_plane(ring + sl * L::kPlaneBytes, map, tx0, ty0, kp + B.g, &bars[sl]);
    }
  }
  int k_issued = k_pro;

  const int q = (ty + 2) * HX + (tx + 2);  // in-plane index of this thread's point
  // boundary faces: warp 1 lane r computes the -x face of row r, warp 0 the -y face of its column
  const bool ex_x = (ty == 1) && (tx < TY) && (t.j0 + tx < B.my);
  const bool ex_y = (ty == 0) && act;
  T *__restrict__ dqa = a.faces;  // [n_var][N]
  T F[NV], acc[NV];
  bool aborted = false;
  for (int k = kstart; k < t.k1; ++k) {
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
    const bool prologue = k < t.k0;
#pragma unroll
    for (int l = 0; l < NV; ++l) acc[l] = T(0);
    // it: 0 = +z, 1 = +x, 2 = -x boundary (warp 1), 3 = -y boundary (warp 0), 4 = +y
#pragma unroll 1
    for (int it = three_d ? 0 : 1; it < (prologue ? 1 : 5); ++it) {
      bool doit;
      int d, sd, qq = q, gp = p;
      if (it == 0) {
        doit = act, d = 2, sd = sk;
      } else if (it == 1) {
        doit = act, d = 0, sd = 1;
      } else if (it == 2) {
        doit = ex_x, d = 0, sd = 1;
        qq = (tx + 2) * HX + 1;  // row tx of the tile, i = i0 - 1
        gp = (int)B.base + (t.i0 - 1) + sj * (t.j0 + tx) + sk * k;
      } else if (it == 3) {
        doit = ex_y, d = 1, sd = sj;
        qq = q - HX;
        gp = p - sj;
      } else {
        doit = act, d = 1, sd = sj;
      }
      if (doit) {
        Stencil S{plm, pl0, pl1, pl2, qq, d};
        face_flux_gen<T, NS>(C, sRec, S, a.Pr, a.G, N, gp, sd, d, F);
      } else {
#pragma unroll
        for (int l = 0; l < NV; ++l) F[l] = T(0);
      }
      if (it == 0) {
        // +z face: -F here, +F in plane k+1 (stored there as its partial sum)
        if (act) {
#pragma unroll
          for (int l = 0; l < NV; ++l)
            if (l < nv) {
              if (k + 1 < t.k1) dqa[l * N + p + sk] = F[l];
              acc[l] = -F[l];
            }
        }
      } else if (it == 1) {
#pragma unroll
        for (int l = 0; l < NV; ++l) {
          const T left = __shfl_up_sync(0xffffffffu, F[l], 1);
          acc[l] -= F[l];
          if (tx > 0) acc[l] += left;
        }
      } else if (it == 2) {
        if (doit) {
#pragma unroll
          for (int l = 0; l < NV; ++l)
            if (l < nv) sXm[l * TY + tx] = F[l];
        }
      } else if (it == 3) {
        if (doit) {
#pragma unroll
          for (int l = 0; l < NV; ++l)
            if (l < nv) sYm[l * TX + tx] = F[l];
        }
      }
    }
    if (!prologue) {
      __syncthreads();  // boundary faces written
      if (tx == 0) {
#pragma unroll
        for (int l = 0; l < NV; ++l)
          if (l < nv) acc[l] += sXm[l * TY + ty];
      }
      // -y faces: the +y faces (F) of the row below, one chunk of fields at a time
#pragma unroll
      for (int c0 = 0; c0 < NV; c0 += CH) {
        if (ty < TY - 1) {
#pragma unroll
          for (int l = c0; l < c0 + CH && l < NV; ++l) sX[((l - c0) * (TY - 1) + ty) * TX + tx] = F[l];
        }
        __syncthreads();
#pragma unroll
        for (int l = c0; l < c0 + CH && l < NV; ++l) {
          const T below = ty == 0 ? sYm[l * TX + tx] : sX[((l - c0) * (TY - 1) + ty - 1) * TX + tx];
          acc[l] += below - F[l];
        }
        __syncthreads();
      }
      if (act) {
#pragma unroll
        for (int l = 0; l < NV; ++l)
          if (l < nv) {
            // the -z face (+z face of plane k-1), stored by this thread one plane earlier
            if (three_d) acc[l] += dqa[l * N + p];
            dqa[l * N + p] = acc[l];
          }
      }
    } else {
      __syncthreads();  // plane k - 1 is no longer read
    }
    if (k + 3 <= klast) {
      if (tid == 0) {
        const int sl = slot_of(k + 3);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive_expect_tx(&bars[sl], plane_bytes);
        tma_load_plane(ring + sl * L::kPlaneBytes, map, tx0, ty0, k + 3 + B.g, &bars[sl]);
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
}

}  // namespace ccb
