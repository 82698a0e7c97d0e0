// Split stage: faces first, then the point update (sm_100a).
//
// k_faces computes every face flux of the stage exactly once and writes it
// to the face arena; k_update differences the six faces of each point and
// applies the same RK update, FP64 Newton, transport and time-step reduction
// as the fused kernel (point_update).  Splitting costs one write and one read
// of the face fluxes (3 n_var values per point) but removes the fused
// kernel's barriers and shared-memory flux planes: k_faces keeps almost the
// whole 256 KB L1 for the stencil reads, and k_update, which needs far fewer
// registers than the face code, runs three CTAs per SM.
//
// Face d of point p is the face between p and p + e_d (the reference's
// F(i+1/2), TimeAdvanceFunc.cu:61-243).  Regular tiles compute the +x, +y, +z
// faces of their interior points; edge tiles compute the faces between the
// ghost layer -1 and the first interior layer of each block, one direction
// per tile (Tile::pad0):
//   d = 0: i = -1, lanes along j, warps along k (k0..k1)
//   d = 1: j = -1, lanes along i, warps along k (k0..k1)
//   d = 2: k = -1, lanes along i, warps along j
#pragma once
#include "stage.cuh"

namespace ccb {

template <typename T, int NS>
__global__ void __launch_bounds__(kTX *kTY, sizeof(T) == 8 ? 1 : 2)
    k_faces(const StageArgs<T> a, const __grid_constant__ ChemParams C) {
  constexpr int A = SpecCount<NS>::kArr;
  constexpr int NV = 5 + A;
  const int ns = SpecCount<NS>::n(C);
  const int nv = 5 + ns;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sRec = reinterpret_cast<T *>(smem_raw);  // [A][2][kRecLen]
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTX + tx;
  for (int e = tid, nrec = ns * 2 * kRecLen; e < nrec; e += kTX * kTY) sRec[e] = param_rec<T>(C)[e];
  __syncthreads();  // the only barrier: threads may leave from here on

  const bool edge = (int)blockIdx.x >= a.n_regular;
  const Tile t = edge ? a.edge_tiles[blockIdx.x - a.n_regular] : a.tiles[blockIdx.x];
  const BlockInfo B = a.blocks[t.blk];
  const int N = (int)a.N, sj = B.nx, sk = B.nx * B.ny;
  const bool three_d = B.mz > 1;
  T F[NV];
  auto put = [&](int d, int p) {
#pragma unroll
    for (int l = 0; l < NV; ++l)
      if (l < nv) a.faces[(d * nv + l) * N + p] = F[l];
  };
  if (!edge) {
    const int i = t.i0 + tx, j = t.j0 + ty;
    if (i >= B.mx || j >= B.my) return;
    const int col = (int)B.base + i + sj * j;
    for (int k = t.k0; k < t.k1; ++k) {
      const int p = col + sk * k;
#pragma unroll 1
      for (int it = three_d ? 0 : 1; it < 3; ++it) {
        const int d = it == 0 ? 2 : it - 1;
        const int sd = d == 0 ? 1 : (d == 1 ? sj : sk);
        face_flux<T, NS>(C, sRec, a.P, a.Pr, a.G, N, p, d, sd, sj, sk, F);
        put(d, p);
      }
    }
    return;
  }
  const int d = t.pad0;
  int i, j, k;
  bool ok;
  if (d == 0) {
    i = -1, j = t.j0 + tx, k = t.k0 + ty;
    ok = j < B.my && k < t.k1;
  } else if (d == 1) {
    i = t.i0 + tx, j = -1, k = t.k0 + ty;
    ok = i < B.mx && k < t.k1;
  } else {
    i = t.i0 + tx, j = t.j0 + ty, k = -1;
    ok = i < B.mx && j < B.my && three_d;
  }
  if (!ok) return;
  const int p = (int)B.base + i + sj * j + sk * k;
  const int sd = d == 0 ? 1 : (d == 1 ? sj : sk);
  face_flux<T, NS>(C, sRec, a.P, a.Pr, a.G, N, p, d, sd, sj, sk, F);
  put(d, p);
}

// MINB: CTAs per SM the registers are sized for (the autotuner tries 4 in
// FP32: 64 registers with some spills against 80 at 3).  Tiles of UX x
// (256 / UX) points: 32 x 8, or 16 x 16 beside the 16-wide face tiles.
template <typename T, int NS, int MINB = (sizeof(T) == 8 ? 2 : 3), int UX = kTX>
__global__ void __launch_bounds__(256, MINB)
    k_update(const StageArgs<T> a, const __grid_constant__ ChemParams C) {
  constexpr int UY = 256 / UX;
  constexpr int A = SpecCount<NS>::kArr;
  constexpr int NV = 5 + A;
  const int ns = SpecCount<NS>::n(C);
  const int nv = 5 + ns;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *sRecD = reinterpret_cast<double *>(smem_raw);  // [A][2][kRecLen]
  T *sRec = reinterpret_cast<T *>(smem_raw + (sizeof(T) == sizeof(double) ? 0 : StageSmem<T, NS>::kRecD));
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * UX + tx;
  for (int e = tid, nrec = ns * 2 * kRecLen; e < nrec; e += UX * UY) {
    sRecD[e] = param_rec<double>(C)[e];
    if (sizeof(T) != sizeof(double)) sRec[e] = param_rec<T>(C)[e];
  }
  __syncthreads();

  const Tile t = a.tiles[blockIdx.x];
  const BlockInfo B = a.blocks[t.blk];
  const int i = t.i0 + tx, j = t.j0 + ty;
  const bool act = (i < B.mx) && (j < B.my);
  const int N = (int)a.N, sj = B.nx, sk = B.nx * B.ny;
  const bool three_d = B.mz > 1;
  const T *__restrict__ P = a.P;
  const T *__restrict__ Fx = a.faces;
  const T *__restrict__ Fy = a.faces + (size_t)nv * N;
  const T *__restrict__ Fz = a.faces + (size_t)2 * nv * N;
  unsigned flags = 0;
  double dt_min = 1e300;
  if (act) {
    const int col = (int)B.base + i + sj * j;
    // the global step, read once (inside the loop it would follow the
    // previous point's stores)
    const double dt_global = a.local_dt ? 0.0 : *a.dt;
    for (int k = t.k0; k < t.k1; ++k) {
      const int p = CCB_IDX(C, col + sk * k, N);
      double dt;
      if (a.local_dt) {
        T Y[A];
#pragma unroll
        for (int l = 0; l < A; ++l)
          if (l < ns) Y[l] = P[(6 + l) * N + p];
        T gam, c;
        gamma_and_c<T, NS>(C, sRec, P[5 * N + p], Y, gam, c);
        dt = local_time_step<T>(C, a.G, N, p, (double)P[p], (double)P[N + p], (double)P[2 * N + p],
                                (double)P[3 * N + p], (double)c, (double)gam, (double)a.Pr[p], three_d);
      } else {
        dt = dt_global;
      }
      const double dtj = dt / (double)a.G[p];
      // whether this point's step enters the next global time step, read with
      // the state rather than behind the stores
      const bool want_dt = a.dt_next && !((a.skip_dt[p >> 5] >> (p & 31)) & 1u);
      // dq = -(sum over directions of F(+1/2) - F(-1/2)), the fused kernel's
      // order, and the new conserved state, each variable's faces and state
      // read together; the stores follow (Qout may alias Qin)
      double q[NV];
      if (a.dq_direct) {  // dq differenced by the face kernel (k_faces_dq)
#pragma unroll
        for (int l = 0; l < NV; ++l)
          if (l < nv) q[l] = conserved_update<T>(C, a, p, N, l, (double)Fx[l * N + p], dtj, three_d);
      } else {
        // the minus-side faces (checked in bounds-checked builds)
        const int px = CCB_IDX(C, p - 1, N), py = CCB_IDX(C, p - sj, N), pz = CCB_IDX(C, p - sk, N);
#pragma unroll
        for (int l = 0; l < NV; ++l) {
          if (l < nv) {
            const int o = l * N + p;
            T acc = Fx[o] - Fx[l * N + px];
            acc += Fy[o] - Fy[l * N + py];
            if (three_d) acc += Fz[o] - Fz[l * N + pz];
            q[l] = conserved_update<T>(C, a, p, N, l, -(double)acc, dtj, three_d);
          }
        }
      }
      point_finish<T, NS>(C, sRec, sRecD, a, p, N, q, (double)P[5 * N + p], three_d, want_dt, flags, dt_min);
    }
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
