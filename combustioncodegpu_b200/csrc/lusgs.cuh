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
// the two sweeps are (with the reciprocal 1/D formed once per point)
//   dQ*(p) = (dq(p) + sum_d A+_d(p - e_d) dQ*(p - e_d)) (1/D)       (lower, i+j+k ascending)
//   dQ(p)  = dQ*(p) - (sum_d A-_d(p + e_d) dQ(p + e_d)) (1/D)       (upper, descending)
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
// blocks, in order, chained by programmatic dependent launch so that a
// launch and its own loads overlap the previous hyperplane.  The sweeps read and write arrays in sweep order (points
// sorted by hyperplane, block, k, j; LusgsArgs): the points of a hyperplane
// are contiguous and the neighbours a warp reads in the adjacent hyperplane
// are too.  The arithmetic of each point is the oracle's lexicographic sweep,
// term for term.
#pragma once
#include "stage.cuh"

namespace ccb {

// dF = A_d(q) dQ for the J-weighted flux along k = J grad xi_d at q; Q is the
// conserved state at q, inv = 1 / rho and u, v, w = Q[1..3] * inv, p its
// pressure, psi its species pressure derivatives.
template <int NV>
__device__ __forceinline__ void lusgs_jac_vec(int nv, const double (&Q)[NV], double inv, double u, double v, double w,
                                              double p, double gam, const double (&psi)[NV], const double k[3],
                                              const double (&dQ)[NV], double (&dF)[NV]) {
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

// Rows of 16 doubles for 32 points, one per lane, written to their sweep-order
// positions: the lanes first put their rows into a per-warp shared-memory
// buffer, then each store instruction writes two whole rows (two 128-byte
// lines) instead of one word of 32 scattered rows.  Row element e of lane r
// goes to dst[pos_r * stride + e]; lanes without a point pass pos = -1.
__device__ __forceinline__ void lusgs_put_rows(double (*buf)[17], const double (&v)[16], int64_t pos, double *dst,
                                               int stride) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int e = 0; e < 16; ++e) buf[lane][e] = v[e];
  __syncwarp();
#pragma unroll
  for (int m = 0; m < 16; ++m) {
    const int r = 2 * m + (lane >> 4), e = lane & 15;
    const int64_t pr = __shfl_sync(0xffffffffu, pos, r);
    if (pr >= 0) dst[pr * stride + e] = buf[r][e];
  }
  __syncwarp();
}

// Right-hand side, spectral radii, diagonal and the Jacobian inputs of every
// interior point of the tiles (the split variant's face arena holds the
// current fluxes), written in sweep order as whole rows (unused lanes zero).
template <typename T, int NS>
__global__ void __launch_bounds__(kTX *kTY, sizeof(T) == 8 ? 1 : 2) k_lusgs_rhs(const StageArgs<T> a, const LusgsArgs L,
                                                                             const __grid_constant__ ChemParams C) {
  constexpr int A = SpecCount<NS>::kArr;
  constexpr int NV = 5 + A;
  static_assert(NV <= 16 || NS < 0, "rows are 16 doubles for the compiled species counts");
  const int ns = SpecCount<NS>::n(C);
  const int nv = 5 + ns;
  __shared__ double sbuf[kTX * kTY / 32][32][17];
  double (*buf)[17] = sbuf[(threadIdx.y * kTX + threadIdx.x) >> 5];
  const Tile t = a.tiles[blockIdx.x];
  const BlockInfo B = a.blocks[t.blk];
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  const bool act = i < B.mx && j < B.my;  // inactive lanes still take part in the row writes
  const int N = (int)a.N, sj = B.nx, sk = B.nx * B.ny;
  const int64_t S = L.S;
  const int lp = L.lp;
  const bool three_d = B.mz > 1;
  const T *__restrict__ P = a.P;
  const T *__restrict__ G = a.G;
  const T *__restrict__ Fx = a.faces;
  const T *__restrict__ Fy = a.faces + (size_t)nv * N;
  const T *__restrict__ Fz = a.faces + (size_t)2 * nv * N;
  const T *rec = param_rec<T>(C);
  const int col = (int)B.base + (act ? i + sj * j : 0);
  for (int k = t.k0; k < t.k1; ++k) {
    const int p = col + sk * k;
    const int64_t sp = act ? (int64_t)L.pos[p] : -1;
    // the point's primitives, viscosity and geometry, read together with the
    // faces below: read after the row stores they would wait for a second
    // round trip, since the compiler cannot move loads above stores that may
    // alias them
    T pv[6 + A], mu_t = T(0), gv[10];
#pragma unroll
    for (int f = 0; f < 6 + A; ++f) pv[f] = (act && f < 6 + ns) ? P[f * N + p] : T(0);
#pragma unroll
    for (int r = 0; r < 10; ++r) gv[r] = act ? G[r * N + p] : T(0);
    if (act) mu_t = a.Pr[p];
    double qc[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) qc[f] = act ? a.Qin[f * N + p] : 0.0;
    if (NV > 16) {  // runtime species count beyond 11: plain stores of the wider rows
      if (act) {
#pragma unroll
        for (int l = 0; l < NV; ++l) {
          if (l < nv) {
            const int o = l * N + p;
            T acc = Fx[o] - Fx[o - 1];
            acc += Fy[o] - Fy[o - sj];
            if (three_d) acc += Fz[o] - Fz[o - sk];
            double dq = -(double)acc;
            if (a.gcl && l >= 1 && l <= 3) dq -= C.p_ref * a.gcl[(l - 1) * N + p];
            L.R[sp * lp + l] = dq;
            L.Qs[sp * lp + l] = a.Qin[o];
          }
        }
      }
    } else {
      double rv[16], qv[16];
#pragma unroll
      for (int l = 0; l < 16; ++l) {
        rv[l] = qv[l] = 0.0;
        if (act && l < nv) {
          const int o = l * N + p;
          T acc = Fx[o] - Fx[o - 1];
          acc += Fy[o] - Fy[o - sj];
          if (three_d) acc += Fz[o] - Fz[o - sk];
          double dq = -(double)acc;
          if (a.gcl && l >= 1 && l <= 3) dq -= C.p_ref * a.gcl[(l - 1) * N + p];
          rv[l] = dq;
          qv[l] = a.Qin[o];
        }
      }
      lusgs_put_rows(buf, rv, lp == 16 ? sp : -1, L.R, 16);
      lusgs_put_rows(buf, qv, lp == 16 ? sp : -1, L.Qs, 16);
      if (lp != 16 && act)  // 8-lane rows (the air model)
#pragma unroll
        for (int l = 0; l < 8; ++l) L.R[sp * lp + l] = rv[l], L.Qs[sp * lp + l] = qv[l];
    }
    double row[32];
#pragma unroll
    for (int e = 0; e < 32; ++e) row[e] = 0.0;
    double psi[16];
#pragma unroll
    for (int l = 0; l < 16; ++l) psi[l] = 0.0;
    if (act) {
      const double inv = 1.0 / qc[0];
      row[kLuInv] = inv;
      row[kLuU] = qc[1] * inv;
      row[kLuU + 1] = qc[2] * inv;
      row[kLuU + 2] = qc[3] * inv;
      row[kLuP] = (double)pv[4] + C.p_ref;
      T Y[A];
#pragma unroll
      for (int l = 0; l < A; ++l)
        if (l < ns) Y[l] = pv[6 + l];
      T gam, c;
      gamma_and_c<T, NS>(C, rec, pv[5], Y, gam, c);
      const double rho = (double)pv[0], u = (double)pv[1], v = (double)pv[2], w = (double)pv[3];
      const double mu = (double)mu_t;
      double mt[9];
#pragma unroll
      for (int r = 0; r < 9; ++r) mt[r] = (double)gv[1 + r];
      const double dt = local_time_step_m(C, mt, rho, u, v, w, (double)c, (double)gam, mu, three_d);
      const double J = (double)gv[0];
      const double c1 = fmax((double)gam, 4.0 / 3.0);
      const double c2 = mu / rho / C.Pr;
      double D = J / dt;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        double r = 0;
        const double m0 = mt[3 * d], m1 = mt[3 * d + 1], m2 = mt[3 * d + 2];
        if (d < 2 || three_d) {
          const double g = sqrt(m0 * m0 + m1 * m1 + m2 * m2);
          const double U = u * m0 + v * m1 + w * m2;
          r = fabs(U) + (double)c * g;
          if (C.viscous) r += 2.0 * c1 * c2 * g * g;
          r *= J;
          D += r;
        }
        row[kLuRad + d] = r;
        row[kLuK + 3 * d] = J * m0;
        row[kLuK + 3 * d + 1] = J * m1;
        row[kLuK + 3 * d + 2] = J * m2;
      }
      row[kLuRD] = 1.0 / D;
      row[kLuGam] = (double)gam;
      const int id[3] = {i, j, k};
#pragma unroll
      for (int d = 0; d < 3; ++d)
        if (id[d] == 0)  // no lower neighbour: nothing arrives in this row during the lower sweep
          for (int l = 0; l < lp; ++l) L.Cn[(d * S + sp) * lp + l] = 0.0;
      if (ns > 0) {
        const double td = (double)pv[5], g1 = (double)gam - 1.0;
#pragma unroll
        for (int l = 0; l < A; ++l) {
          if (l < ns) {
            const double x = (double)gam * C.d.cv_shift[l] * td - g1 * nasa_h<double>(C.d, param_rec<double>(C), l, td);
            if (NV <= 16)
              psi[5 + l] = x;
            else
              L.psi[sp * lp + 5 + l] = x;
          }
        }
      }
    }
    double half[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) half[e] = row[e];
    lusgs_put_rows(buf, half, sp, L.pt, kLuScalars);
#pragma unroll
    for (int e = 0; e < 16; ++e) half[e] = row[16 + e];
    lusgs_put_rows(buf, half, sp, L.pt + 16, kLuScalars);
    if (NV <= 16 && ns > 0) {
      lusgs_put_rows(buf, psi, lp == 16 ? sp : -1, L.psi, 16);
    }
  }
}

// One point of the lower (DIR = +1) or upper (DIR = -1) sweep, held by a
// group of LP = lusgs_lanes(n_var) lanes of a warp, lane l owning variable l.
// load() reads the point's own data (none of it depends on the preceding
// hyperplane); solve() finishes the point.  The neighbour terms
// A+-_d(q) dQ(q) arrive in this point's rows of L.Cn, stored there by the
// neighbour q when it was solved, so the only loads after the wait are these
// rows.  After solving, the group forms its own terms for the neighbours of
// the next hyperplane: the couplings of the Jacobian (rho, momentum, energy,
// and the species pressure terms in ascending order) come from the other
// lanes by shuffles, and every lane evaluates the oracle's expressions in
// its order.  In the lower sweep a point also clears the rows that no
// neighbour fills in the upper sweep.  Every lane of the warp runs the
// shuffles; lanes without a point mask their memory accesses, lanes without
// a variable hold zeros and store them, so that every row is written whole.  Offsets are 32-bit (3 lp S < 2^31 is checked at allocation).
template <int NS, int DIR>
struct LusgsLane {
  static constexpr int A = SpecCount<NS>::kArr;
  static constexpr int NV = 5 + A;
  static constexpr int LP = lusgs_lanes(NV);
  int s, S, l, nb[3];
  bool act, var;  // the group has a point; this lane has a variable
  double R, Q, psi, kv[9], rad[3], rD, ps, gam, inv, u, v, w;

  // All loads go through L2 (ld.global.cg): with programmatic dependent
  // launch they may run while the preceding kernel is still finishing, and
  // an L1 line of an earlier kernel on this SM must not be used.
  __device__ __forceinline__ void load(const LusgsArgs &L, int nv, int s_, int l_, bool act_) {
    s = s_, S = (int)L.S, l = l_, act = act_, var = act_ && l_ < nv;
    const int *__restrict__ next = DIR > 0 ? L.hi : L.lo;  // neighbours of the next hyperplane
    R = Q = psi = 0.0;
    if (var) R = __ldcg(L.R + s * LP + l), Q = __ldcg(L.Qs + s * LP + l), psi = __ldcg(L.psi + s * LP + l);
#pragma unroll
    for (int d = 0; d < 3; ++d) nb[d] = act ? __ldcg(next + d * S + s) : -1;
    const double *row = L.pt + (int64_t)(act ? s : 0) * kLuScalars;
#pragma unroll
    for (int e = 0; e < 9; ++e) kv[e] = act ? __ldcg(row + kLuK + e) : 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) rad[d] = act ? __ldcg(row + kLuRad + d) : 0.0;
    rD = act ? __ldcg(row + kLuRD) : 0.0, ps = act ? __ldcg(row + kLuP) : 0.0, gam = act ? __ldcg(row + kLuGam) : 1.0;
    inv = act ? __ldcg(row + kLuInv) : 0.0, u = act ? __ldcg(row + kLuU) : 0.0;
    v = act ? __ldcg(row + kLuU + 1) : 0.0, w = act ? __ldcg(row + kLuU + 2) : 0.0;
  }

  __device__ __forceinline__ void solve(const LusgsArgs &L, int nv) {
    double *__restrict__ Cn = L.Cn;
    double acc = DIR > 0 ? R : 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double *c = Cn + ((int64_t)d * S + s) * LP + l;
      if (var) acc += __ldcg(c);
    }
    const double X = DIR > 0 ? acc * rD : R - acc * rD;
    if (act) L.R[s * LP + l] = X;  // whole rows: lanes without a variable store 0
    if (DIR > 0 && act) {
#pragma unroll
      for (int d = 0; d < 3; ++d)
        if (nb[d] < 0) Cn[((int64_t)d * S + s) * LP + l] = 0.0;
    }
    // couplings from the other lanes of the group
    const unsigned full = 0xffffffffu;
    const double x0 = __shfl_sync(full, X, 0, LP), x1 = __shfl_sync(full, X, 1, LP);
    const double x2 = __shfl_sync(full, X, 2, LP), x3 = __shfl_sync(full, X, 3, LP);
    const double x4 = __shfl_sync(full, X, 4, LP);
    const double pX = psi * X;
    double dp = (gam - 1.0) * (x4 - (u * x1 + v * x2 + w * x3) + 0.5 * (u * u + v * v + w * w) * x0);
#pragma unroll
    for (int m = 5; m < NV; ++m) {
      const double t = __shfl_sync(full, pX, m, LP);
      if (m < nv) dp += t;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (nb[d] < 0 || !act) continue;
      const double k0 = kv[3 * d], k1 = kv[3 * d + 1], k2 = kv[3 * d + 2];
      const double U = k0 * u + k1 * v + k2 * w;
      const double dm = k0 * x1 + k1 * x2 + k2 * x3;
      const double dU = (dm - U * x0) * inv;
      double dF;
      if (l == 0)
        dF = dm;
      else if (l <= 3)
        dF = X * U + Q * dU + (l == 1 ? k0 : (l == 2 ? k1 : k2)) * dp;
      else if (l == 4)
        dF = (X + dp) * U + (Q + ps) * dU;
      else
        dF = X * U + Q * dU;
      const double r = DIR * rad[d];
      Cn[((int64_t)d * S + nb[d]) * LP + l] = 0.5 * (dF + r * X);
    }
  }
};

// One hyperplane (sweep positions [L.s0, L.s1)) per launch.
template <int NS, int DIR>
__global__ void __launch_bounds__(kSweepThreads) k_lusgs_sweep(const LusgsArgs L,
                                                               const __grid_constant__ ChemParams C) {
  using Lane = LusgsLane<NS, DIR>;
  const int nv = 5 + SpecCount<NS>::n(C);
  const int64_t s = L.s0 + (int64_t)blockIdx.x * (kSweepThreads / Lane::LP) + threadIdx.x / Lane::LP;
  Lane pt;
  // Programmatic dependent launch: this kernel may start while the previous
  // hyperplane's is still running.  The point's own rows were written by the
  // right-hand side kernel or the lower sweep, which completed before the
  // previous launch passed its wait (it only lets this launch start after
  // that), so they are read before waiting, except by the first launch of a
  // sweep (L.early = 0), whose predecessor produced them.  The neighbour
  // rows of L.Cn are written by the previous launch: read after the wait.
  if (L.early) pt.load(L, nv, (int)s, threadIdx.x % Lane::LP, s < L.s1);
  asm volatile("griddepcontrol.wait;" ::: "memory");
  if (!L.early) pt.load(L, nv, (int)s, threadIdx.x % Lane::LP, s < L.s1);
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  pt.solve(L, nv);
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
      const int64_t sp = L.pos[p];
      double dq[NV];
#pragma unroll
      for (int l = 0; l < NV; ++l)
        if (l < nv) dq[l] = L.R[sp * L.lp + l];
      point_update<T, NS>(C, sRec, sRecD, a, p, N, dq, (double)a.G[p], (double)a.P[5 * N + p], three_d, flags,
                          dt_min);
    }
  }
  const unsigned any = __reduce_or_sync(0xffffffffu, flags);
  if (any && tx == 0) atomicOr(a.status, any);
}

}  // namespace ccb
