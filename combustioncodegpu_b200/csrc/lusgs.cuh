// Implicit steady step: scalar LU-SGS (lower-upper symmetric Gauss-Seidel,
// Yoon & Jameson, AIAA J. 26(9):1025-1026, 1988) with the viscous spectral
// radius on the diagonal.  The reference declares this scheme (struct LUSGS,
// TemporalScheme.cuh:19-21; temporal_scheme 1, Driver.cu:318-321) and
// allocates its spectral-radius arrays (Field.h:60-61, Field.cu:138-141) but
// gives it no body, so its temporal_scheme 1 runs the explicit update.
//
// Per step, with dq the explicit right-hand side of the steady loop
// (J dQ/dt = dq, TimeAdvanceFunc.cu:255-265) and, per point and direction d,
//   sigma_d  = |u . grad xi_d| + c |grad xi_d|                (inviscid)
//   sigv_d   = max(gamma, 4/3) mu / (rho Pr) |grad xi_d|^2    (viscous runs)
//   r_d      = J (sigma_d + 2 sigv_d)
//   D        = J / dt_local + sum_d r_d     (dt_local: TemporalScheme.cu:11-43)
//   A+-_d dQ = (A_d dQ +- r_d dQ) / 2,      A_d = d(J grad xi_d . F)/dQ
// the two sweeps are
//   D dQ*(p) = dq(p) + sum_d A+_d(p - e_d) dQ*(p - e_d)        (lower, i+j+k ascending)
//   dQ(p)    = dQ*(p) - D^-1 sum_d A-_d(p + e_d) dQ(p + e_d)   (upper, descending)
// over the interior points of each block (neighbours outside the block
// contribute nothing: the block interfaces and boundaries stay explicit), and
// Q += dQ.  A_d dQ is the Jacobian-vector product of the J-weighted flux of
// the thermally perfect mixture, p = rho R T with rho e = sum rho Y_k e_k(T):
//   dp = (gamma - 1)(d(rho E) - u . d(rho u) + |u|^2/2 d rho) + sum_k psi_k d(rho Y_k),
//   psi_k = gamma R_k T - (gamma - 1) h_k(T)
// (the last sum is absent for the calorically perfect air model), so that its
// eigenvalues are U and U +- c |k| and r_d bounds them.  The Jacobian only
// shapes the convergence path; the converged state is that of dq = 0.
//
// A point of sweep hyperplane h = i + j + k depends only on hyperplane h - 1
// (h + 1 for the upper sweep), so each hyperplane is one launch over all
// blocks, in order.  The arithmetic of each point is the oracle's
// lexicographic sweep, term for term.
#pragma once
#include "stage.cuh"

namespace ccb {

// dF = A_d(q) dQ for the J-weighted flux along k = J grad xi_d at q; Q is the
// conserved state at q, p its pressure, psi its species pressure derivatives.
template <int NV>
__device__ __forceinline__ void lusgs_jac_vec(int nv, const double (&Q)[NV], double p, double gam,
                                              const double (&psi)[NV], const double k[3], const double (&dQ)[NV],
                                              double (&dF)[NV]) {
  const double rho = Q[0], inv = 1.0 / rho;
  const double u = Q[1] * inv, v = Q[2] * inv, w = Q[3] * inv;
  const double U = k[0] * u + k[1] * v + k[2] * w;
  const double dm = k[0] * dQ[1] + k[1] * dQ[2] + k[2] * dQ[3];
  const double dU = (dm - U * dQ[0]) * inv;
  double dp = (gam - 1.0) * (dQ[4] - (u * dQ[1] + v * dQ[2] + w * dQ[3]) + 0.5 * (u * u + v * v + w * w) * dQ[0]);
#pragma unroll
  for (int l = 5; l < NV; ++l)
    if (l < nv) dp += psi[l] * dQ[l];
  dF[0] = dm;
  dF[1] = dQ[1] * U + Q[1] * dU + k[0] * dp;
  dF[2] = dQ[2] * U + Q[2] * dU + k[1] * dp;
  dF[3] = dQ[3] * U + Q[3] * dU + k[2] * dp;
  dF[4] = (dQ[4] + dp) * U + (Q[4] + p) * dU;
#pragma unroll
  for (int l = 5; l < NV; ++l)
    if (l < nv) dF[l] = dQ[l] * U + Q[l] * dU;
}

// Right-hand side, spectral radii and diagonal of every interior point of
// the tiles (the split variant's face arena holds the current fluxes).
template <typename T, int NS>
__global__ void __launch_bounds__(kTX *kTY) k_lusgs_rhs(const StageArgs<T> a, const LusgsArgs L,
                                                      const __grid_constant__ ChemParams C) {
  constexpr int A = SpecCount<NS>::kArr;
  constexpr int NV = 5 + A;
  const int ns = SpecCount<NS>::n(C);
  const int nv = 5 + ns;
  const Tile t = a.tiles[blockIdx.x];
  const BlockInfo B = a.blocks[t.blk];
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  if (i >= B.mx || j >= B.my) return;
  const int N = (int)a.N, sj = B.nx, sk = B.nx * B.ny;
  const bool three_d = B.mz > 1;
  const T *__restrict__ P = a.P;
  const T *__restrict__ G = a.G;
  const T *__restrict__ Fx = a.faces;
  const T *__restrict__ Fy = a.faces + (size_t)nv * N;
  const T *__restrict__ Fz = a.faces + (size_t)2 * nv * N;
  const T *rec = param_rec<T>(C);
  const int col = (int)B.base + i + sj * j;
  for (int k = t.k0; k < t.k1; ++k) {
    const int p = col + sk * k;
#pragma unroll
    for (int l = 0; l < NV; ++l) {
      if (l < nv) {
        const int o = l * N + p;
        T acc = Fx[o] - Fx[o - 1];
        acc += Fy[o] - Fy[o - sj];
        if (three_d) acc += Fz[o] - Fz[o - sk];
        double dq = -(double)acc;
        if (a.gcl && l >= 1 && l <= 3) dq -= C.p_ref * a.gcl[(l - 1) * N + p];
        L.R[o] = dq;
      }
    }
    T Y[A];
#pragma unroll
    for (int l = 0; l < A; ++l)
      if (l < ns) Y[l] = P[(6 + l) * N + p];
    T gam, c;
    gamma_and_c<T, NS>(C, rec, P[5 * N + p], Y, gam, c);
    const double rho = (double)P[p], u = (double)P[N + p], v = (double)P[2 * N + p], w = (double)P[3 * N + p];
    const double mu = (double)a.Pr[p];
    const double dt = local_time_step<T>(C, G, N, p, rho, u, v, w, (double)c, (double)gam, mu, three_d);
    const double J = (double)G[p];
    const double c1 = fmax((double)gam, 4.0 / 3.0);
    const double c2 = mu / rho / C.Pr;
    double D = J / dt;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      double r = 0;
      if (d < 2 || three_d) {
        const double m0 = (double)G[(1 + 3 * d) * N + p], m1 = (double)G[(2 + 3 * d) * N + p],
                     m2 = (double)G[(3 + 3 * d) * N + p];
        const double g = sqrt(m0 * m0 + m1 * m1 + m2 * m2);
        const double U = u * m0 + v * m1 + w * m2;
        r = fabs(U) + (double)c * g;
        if (C.viscous) r += 2.0 * c1 * c2 * g * g;
        r *= J;
        D += r;
      }
      L.rad[d * N + p] = r;
    }
    L.diag[p] = D;
    L.gam[p] = (double)gam;
    if (ns > 0) {
      const double td = (double)P[5 * N + p], g1 = (double)gam - 1.0;
#pragma unroll
      for (int l = 0; l < A; ++l)
        if (l < ns)
          L.psi[l * N + p] = (double)gam * C.d.cv_shift[l] * td - g1 * nasa_h<double>(C.d, param_rec<double>(C), l, td);
    }
  }
}

// One hyperplane i + j + k = L.h of the lower (DIR = +1) or upper (DIR = -1)
// sweep; blockIdx.y is the block, threads run over its (j, k) columns.
template <typename T, int NS, int DIR>
__global__ void __launch_bounds__(256) k_lusgs_sweep(const StageArgs<T> a, const LusgsArgs L,
                                                     const __grid_constant__ ChemParams C) {
  constexpr int A = SpecCount<NS>::kArr;
  constexpr int NV = 5 + A;
  const int ns = SpecCount<NS>::n(C);
  const int nv = 5 + ns;
  const BlockInfo B = a.blocks[blockIdx.y];
  const int cidx = blockIdx.x * blockDim.x + threadIdx.x;
  if (cidx >= B.my * B.mz) return;
  const int j = cidx % B.my, k = cidx / B.my;
  const int i = L.h - j - k;
  if (i < 0 || i >= B.mx) return;
  const int N = (int)a.N, sj = B.nx, sk = B.nx * B.ny;
  const bool three_d = B.mz > 1;
  const int p = (int)B.base + i + sj * j + sk * k;
  const T *__restrict__ G = a.G;
  double acc[NV];
#pragma unroll
  for (int l = 0; l < NV; ++l)
    if (l < nv) acc[l] = DIR > 0 ? L.R[l * N + p] : 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (d == 2 && !three_d) break;
    const int id = d == 0 ? i : (d == 1 ? j : k);
    const int md = d == 0 ? B.mx : (d == 1 ? B.my : B.mz);
    const int sd = d == 0 ? 1 : (d == 1 ? sj : sk);
    if (DIR > 0 ? id < 1 : id + 1 >= md) continue;
    const int q = DIR > 0 ? p - sd : p + sd;
    double X[NV], Qq[NV], dF[NV], psi[NV];
#pragma unroll
    for (int l = 0; l < NV; ++l)
      if (l < nv) X[l] = L.R[l * N + q], Qq[l] = a.Qin[l * N + q], psi[l] = l >= 5 ? L.psi[(l - 5) * N + q] : 0.0;
    const double Jq = (double)G[q];
    const double kv[3] = {Jq * (double)G[(1 + 3 * d) * N + q], Jq * (double)G[(2 + 3 * d) * N + q],
                          Jq * (double)G[(3 + 3 * d) * N + q]};
    const double pq = (double)a.P[4 * N + q] + C.p_ref;
    lusgs_jac_vec<NV>(nv, Qq, pq, L.gam[q], psi, kv, X, dF);
    const double r = DIR * L.rad[d * N + q];
#pragma unroll
    for (int l = 0; l < NV; ++l)
      if (l < nv) acc[l] += 0.5 * (dF[l] + r * X[l]);
  }
  const double D = L.diag[p];
#pragma unroll
  for (int l = 0; l < NV; ++l) {
    if (l < nv) {
      if (DIR > 0)
        L.R[l * N + p] = acc[l] / D;
      else
        L.R[l * N + p] = L.R[l * N + p] - acc[l] / D;
    }
  }
}

// Q += dQ and the primitive recovery, transport and |V| of the new state
// (point_update with dq = dQ and dt = J, so that dt / J is exactly 1).
template <typename T, int NS>
__global__ void __launch_bounds__(kTX *kTY) k_lusgs_update(const StageArgs<T> a, const LusgsArgs L,
                                                         const __grid_constant__ ChemParams C) {
  constexpr int A = SpecCount<NS>::kArr;
  constexpr int NV = 5 + A;
  const int ns = SpecCount<NS>::n(C);
  const int nv = 5 + ns;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *sRecD = reinterpret_cast<double *>(smem_raw);  // [A][2][kRecLen]
  T *sRec = reinterpret_cast<T *>(smem_raw + (sizeof(T) == sizeof(double) ? 0 : StageSmem<T, NS>::kRecD));
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTX + tx;
  for (int e = tid, nrec = ns * 2 * kRecLen; e < nrec; e += kTX * kTY) {
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
  unsigned flags = 0;
  double dt_min = 1e300;
  if (act) {
    const int col = (int)B.base + i + sj * j;
    for (int k = t.k0; k < t.k1; ++k) {
      const int p = col + sk * k;
      double dq[NV];
#pragma unroll
      for (int l = 0; l < NV; ++l)
        if (l < nv) dq[l] = L.R[l * N + p];
      point_update<T, NS>(C, sRec, sRecD, a, p, N, dq, (double)a.G[p], (double)a.P[5 * N + p], three_d, flags,
                          dt_min);
    }
  }
  const unsigned any = __reduce_or_sync(0xffffffffu, flags);
  if (any && tx == 0) atomicOr(a.status, any);
}

}  // namespace ccb
