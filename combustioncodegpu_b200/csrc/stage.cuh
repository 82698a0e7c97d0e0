// Stage, halo and setup kernels of the residual path (sm_100a).
//
// One RK stage is one launch of k_stage over a list of tiles.  A tile is a
// kTX x kTY column of points of one block swept along k: per k-plane every
// thread computes the +x, +y and +z face fluxes of its point (inviscid AUSM+
// minus second-order viscous), the tile's -x / -y boundary faces are computed
// by warps 1 and 0, the -z face is carried from the previous plane, all in
// shared memory; then each thread differences the six faces (the reference's
// dq, TimeAdvanceFunc.cu:61-243), applies the RK update in FP64, recovers the
// primitives (FP64 Newton, Thermo.cu:89-125) and evaluates the transport
// properties of the new state (Field.cu:178-210).  Stage 3 also reduces the
// next global time step (TemporalScheme.cu:11-43) with warp shuffles and a
// 64-bit atomicMin on the bit pattern of the positive double.
//
// Field arenas are structure-of-arrays over all blocks: field f of point p at
// [f * N + p], point p = BlockInfo.base + i + nx*j + nx*ny*k.
//   P   : rho, u, v, w, p, T, Y_0..Y_{ns-1}         (bulk precision T)
//   Pr  : mu, lambda, rhoD_0..rhoD_{ns-1}           (bulk precision T)
//   G   : J, xi_x, xi_y, xi_z, eta_x, ..., zeta_z   (bulk precision T)
//   Q   : rho, rho u, rho v, rho w, rho E, rho Y_k  (FP64 always)
#pragma once
#include "physics.cuh"

namespace ccb {

__device__ __forceinline__ void atomic_min_pos_double(unsigned long long *dst, double v) {
  if (!(v > 0.0) || !(v < 1e300)) return;
  atomicMin(dst, (unsigned long long)__double_as_longlong(v));
}

// TemporalScheme.cu:11-43: CFL / (inviscid + viscous spectral radius), from
// the point's metrics m[3 d + c] = d xi_d / d x_c.
__device__ __forceinline__ double local_time_step_m(const ChemParams &C, const double (&m)[9], double rho, double u,
                                                    double v, double w, double c, double gamma, double mu,
                                                    bool three_d) {
  const double gxi = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
  const double get = sqrt(m[3] * m[3] + m[4] * m[4] + m[5] * m[5]);
  const double gze = sqrt(m[6] * m[6] + m[7] * m[7] + m[8] * m[8]);
  const double U = u * m[0] + v * m[1] + w * m[2];
  const double V = u * m[3] + v * m[4] + w * m[5];
  const double W = u * m[6] + v * m[7] + w * m[8];
  double sri = fabs(U) + fabs(V) + c * (gxi + get);
  if (three_d) sri += fabs(W) + c * gze;
  const double c1 = fmax(gamma, 4.0 / 3.0);
  const double c2 = mu / rho / C.Pr;
  double srv = gxi * gxi + get * get;
  if (three_d) srv += gze * gze;
  srv *= c1 * c2;
  return C.cfl / (sri + srv);
}

// The same with the metrics read from the geometry arena G.
template <typename T>
__device__ __forceinline__ double local_time_step(const ChemParams &C, const T *G, int64_t N, int64_t p, double rho,
                                                  double u, double v, double w, double c, double gamma, double mu,
                                                  bool three_d) {
  double m[9];
#pragma unroll
  for (int r = 0; r < 9; ++r) m[r] = (double)G[(1 + r) * N + p];
  return local_time_step_m(C, m, rho, u, v, w, c, gamma, mu, three_d);
}

// Stencil access of the primitives around one face (point p0 and its
// neighbour p1 = p0 + e_d):  at(f, t) is field f at p0 + t e_d (t = -1..2);
// cross(f, c, sg, t) is field f at p0 + t e_d + sg e_c.
// The strides are scalars, not an array: an array indexed by the runtime
// face direction would live in local memory and put a local load in front of
// every stencil address.  c is a compile-time index after unrolling.
template <typename T>
struct GlobalStencil {
  const T *__restrict__ P;
  int N, p, sd, sj, sk;  // sd: stride along the face normal; sj, sk: strides of j and k
  __device__ __forceinline__ int stride(int c) const { return c == 0 ? 1 : (c == 1 ? sj : sk); }
  __device__ __forceinline__ T at(int f, int t) const { return P[f * N + p + t * sd]; }
  __device__ __forceinline__ T cross(int f, int c, int sg, int t) const {
    return P[f * N + p + t * sd + sg * stride(c)];
  }
};

// Face flux (inviscid minus viscous) of the face between p0 and p0 + e_d;
// transport properties and geometry are read from the arenas at the global
// point gp (and gp + gsd).
// DIR >= 0 fixes the face direction at compile time (d_rt is then ignored).
template <typename T, int NS, typename Stencil, int DIR = -1>
__device__ __forceinline__ void face_flux_gen(const ChemParams &C, const T *rec, const Stencil &S,
                                              const T *__restrict__ Pr, const T *__restrict__ G, int N, int gp, int gsd,
                                              int d_rt, T *F) {
  const int d = DIR >= 0 ? DIR : d_rt;
  constexpr int A = SpecCount<NS>::kArr;
  const int ns = SpecCount<NS>::n(C);
  const int p = CCB_IDX(C, gp, N), p1 = CCB_IDX(C, gp + gsd, N);
  T v[4][5 + A];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
#pragma unroll
    for (int f = 0; f < 5; ++f) v[t][f] = S.at(f, t - 1);
#pragma unroll
    for (int l = 0; l < A; ++l)
      if (l < ns) v[t][5 + l] = S.at(6 + l, t - 1);
  }
  T k[3];
  const T J0 = G[p], J1 = G[p1];
#pragma unroll
  for (int c = 0; c < 3; ++c) k[c] = T(0.5) * (J0 * G[(1 + 3 * d + c) * N + p] + J1 * G[(1 + 3 * d + c) * N + p1]);
  face_inviscid<T, NS>(C, rec, v, k, F);
  if (!C.viscous) return;
  // the face's transport properties first: their loads (through L1, from the
  // arena written by the previous update) then overlap the gradients below
  // instead of stalling the species loop (0.79 -> 0.74 ms per mixed face
  // launch at 128^3); issued before the inviscid flux they raise its
  // register pressure and lose most of that
  const T mu = T(0.5) * (Pr[p] + Pr[p1]);
  const T lam = T(0.5) * (Pr[N + p] + Pr[N + p1]);
  T D[A];
#pragma unroll
  for (int l = 0; l < A; ++l)
    if (l < ns) D[l] = T(0.5) * (Pr[(2 + l) * N + p] + Pr[(2 + l) * N + p1]);

  // ViscousScheme.cu:11-342, metrics averaged over both points (m and m1)
  T met[3][3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) met[r][c] = T(0.5) * (G[(1 + 3 * r + c) * N + p] + G[(1 + 3 * r + c) * N + p1]);
  auto deriv = [&](int f, T out[3]) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (c == d)
        out[c] = S.at(f, 1) - S.at(f, 0);
      else
        out[c] = T(0.25) * (S.cross(f, c, 1, 0) - S.cross(f, c, -1, 0) + S.cross(f, c, 1, 1) - S.cross(f, c, -1, 1));
    }
  };
  auto grad = [&](const T dd[3], T g[3]) {
#pragma unroll
    for (int c = 0; c < 3; ++c) g[c] = dd[0] * met[0][c] + dd[1] * met[1][c] + dd[2] * met[2][c];
  };
  T du[3], dv[3], dw[3], dT[3], gu[3], gv[3], gw[3], gT[3];
  deriv(1, du);
  deriv(2, dv);
  deriv(3, dw);
  deriv(5, dT);
  grad(du, gu);
  grad(dv, gv);
  grad(dw, gw);
  grad(dT, gT);
  const T third = T(1.0 / 3.0);
  const T txx = mu * (T(4) * gu[0] - T(2) * gv[1] - T(2) * gw[2]) * third;
  const T tyy = mu * (T(4) * gv[1] - T(2) * gu[0] - T(2) * gw[2]) * third;
  const T tzz = mu * (T(4) * gw[2] - T(2) * gu[0] - T(2) * gv[1]) * third;
  const T txy = mu * (gu[1] + gv[0]);
  const T txz = mu * (gu[2] + gw[0]);
  const T tyz = mu * (gv[2] + gw[1]);
  const T kx = k[0], ky = k[1], kz = k[2];
  const T f1 = kx * txx + ky * txy + kz * txz;
  const T f2 = kx * txy + ky * tyy + kz * tyz;
  const T f3 = kx * txz + ky * tyz + kz * tzz;
  const T um = T(0.5) * (S.at(1, 0) + S.at(1, 1));
  const T vm = T(0.5) * (S.at(2, 0) + S.at(2, 1));
  const T wm = T(0.5) * (S.at(3, 0) + S.at(3, 1));
  T f4 = um * f1 + vm * f2 + wm * f3 + lam * (kx * gT[0] + ky * gT[1] + kz * gT[2]);
  F[1] -= f1;
  F[2] -= f2;
  F[3] -= f3;
  if (NS == 0 || (NS < 0 && ns == 0)) {
    F[4] -= f4;
    return;
  }
  const SpecTables<T> &ST = tab<T>(C);
  const T tm = T(0.5) * (S.at(5, 0) + S.at(5, 1));
  T gy[A][3];
  T rho_uc = 0, rho_vc = 0, rho_wc = 0;
#pragma unroll
  for (int l = 0; l < A; ++l) {
    if (l < ns) {
      T dy[3];
      deriv(6 + l, dy);
      grad(dy, gy[l]);
      const T DMulH = D[l] * nasa_h<T>(ST, rec, l, tm);
      f4 += kx * DMulH * gy[l][0];
      f4 += ky * DMulH * gy[l][1];
      f4 += kz * DMulH * gy[l][2];
      rho_uc += D[l] * gy[l][0];
      rho_vc += D[l] * gy[l][1];
      rho_wc += D[l] * gy[l][2];
    }
  }
  F[4] -= f4;
  const T corr = kx * rho_uc + ky * rho_vc + kz * rho_wc;
#pragma unroll
  for (int l = 0; l < A; ++l) {
    if (l < ns) {
      const T ym = T(0.5) * (S.at(6 + l, 0) + S.at(6 + l, 1));
      F[5 + l] -= D[l] * (kx * gy[l][0] + ky * gy[l][1] + kz * gy[l][2]) - ym * corr;
    }
  }
}

template <typename T, int NS, int DIR = -1>
__device__ __forceinline__ void face_flux(const ChemParams &C, const T *rec, const T *__restrict__ P,
                                          const T *__restrict__ Pr, const T *__restrict__ G, int N, int p, int d,
                                          int sd, int sj, int sk, T *F) {
  GlobalStencil<T> S{P, N, p, sd, sj, sk};
  face_flux_gen<T, NS, GlobalStencil<T>, DIR>(C, rec, S, Pr, G, N, p, sd, d, F);
}

// gamma and acoustic speed of a point (Field.cu:187-200)
template <typename T, int NS>
__device__ __forceinline__ void gamma_and_c(const ChemParams &C, const T *rec, T temp, const T *Y, T &gamma, T &c) {
  constexpr int A = SpecCount<NS>::kArr;
  const int ns = SpecCount<NS>::n(C);
  if (NS == 0 || (NS < 0 && ns == 0)) {
    gamma = T(kGammaAir);
    c = sqrt(T(kGammaAir * kRu / kMwAir) * temp);
    return;
  }
  const SpecTables<T> &S = tab<T>(C);
  T mwi = 0, cp_tot = 0, cvv = 0;
#pragma unroll
  for (int l = 0; l < A; ++l) {
    if (l < ns) {
      const T cp = nasa_cp<T>(S, rec, l, temp);
      mwi += Y[l] * S.inv_mw[l];
      cp_tot += Y[l] * cp;
      cvv += Y[l] * (cp - S.cv_shift[l]);
    }
  }
  gamma = cp_tot / cvv;
  c = sqrt(gamma * T(kRu) * temp * mwi);
}

// RK update of one interior point (TimeAdvanceFunc.cu:255-290 with the
// Shu-Osher combination), FP64 primitives and Newton, transport properties of
// the new state (Field.cu:178-210), |V| for the residual and the point's
// contribution to the next global time step.
// The conserved variable l of point p after the RK stage, from its residual
// dq (TimeAdvanceFunc.cu:255-265; SSP-RK3 combination).
template <typename T>
__device__ __forceinline__ double conserved_update(const ChemParams &C, const StageArgs<T> &a, int p, int N, int l,
                                                   double dql, double dtj, bool three_d) {
  // momentum fluxes carry p - p_ref: add back -p_ref sum(k+ - k-) (zero on uniform grids)
  if (a.gcl && l >= 1 && l <= 3) dql -= C.p_ref * a.gcl[(l - 1) * N + p];
  double qs = a.Qin[l * N + p] + dql * dtj;
  if (l == 3 && !three_d) qs = 0;
  double q = (a.a != 0.0) ? a.a * a.Qn[l * N + p] + a.b * qs : qs;
  if (a.q32) q = (double)(float)q;  // full-FP32 study: FP32 conserved state
  return q;
}

// Stores the new conserved state q of point p, recovers its primitives (FP64
// Newton), evaluates its transport and, when want_dt, its local time step.
template <typename T, int NS>
__device__ __forceinline__ void point_finish(const ChemParams &C, const T *rec, const double *rec_d,
                                             const StageArgs<T> &a, int p, int N, const double *q, double t_warm,
                                             bool three_d, bool want_dt, unsigned &flags, double &dt_min) {
  constexpr int A = SpecCount<NS>::kArr;
  const int ns = SpecCount<NS>::n(C);
  const int nv = 5 + ns;
  const T *__restrict__ G = a.G;
#pragma unroll
  for (int l = 0; l < 5 + A; ++l)
    if (l < nv) a.Qout[l * N + p] = q[l];
  // primitives (TimeAdvanceFunc.cu:266-289), FP64
  const double rho = q[0];
  const double inv = 1.0 / rho;
  const double u = q[1] * inv, v = q[2] * inv, w = q[3] * inv;
  const double vel2 = u * u + v * v + w * w;
  double pres, temp;
  double Yd[A];
  if (NS == 0 || (NS < 0 && ns == 0)) {
    pres = (kGammaAir - 1) * (q[4] - 0.5 * rho * vel2);
    temp = pres * kMwAir * inv / kRu;
  } else {
    bool capped;
    double gas_const;
    if (!a.q32) {
      double ysum = 0;
#pragma unroll
      for (int l = 0; l < A; ++l)
        if (l < ns) Yd[l] = q[5 + l] * inv, ysum += Yd[l];
      if (a.renorm_y) {
        const double r = 1.0 / ysum;
#pragma unroll
        for (int l = 0; l < A; ++l)
          if (l < ns) Yd[l] *= r;
      }
      double mwi = 0;
#pragma unroll
      for (int l = 0; l < A; ++l)
        if (l < ns) mwi += Yd[l] * C.d.inv_mw[l];
      gas_const = kRu * mwi;
      const double e = q[4] * inv - 0.5 * vel2;
      temp = newton_temperature<NS>(C, rec_d, e, Yd, gas_const, t_warm, capped);
    } else {
      // full-FP32 study: Y, its renormalisation, e and the Newton in FP32
      // (only the FP32 bulk precision runs it; the FP64 instantiation reads
      // the records from the constant bank)
      const float *rec_f32 = sizeof(T) == 4 ? reinterpret_cast<const float *>(rec) : param_rec<float>(C);
      float Yf[A], ysum = 0;
      const float invf = 1.0f / (float)rho;
#pragma unroll
      for (int l = 0; l < A; ++l)
        if (l < ns) Yf[l] = (float)q[5 + l] * invf, ysum += Yf[l];
      if (a.renorm_y) {
        const float r = 1.0f / ysum;
#pragma unroll
        for (int l = 0; l < A; ++l)
          if (l < ns) Yf[l] *= r;
      }
      float mwi = 0;
#pragma unroll
      for (int l = 0; l < A; ++l)
        if (l < ns) mwi += Yf[l] * C.f.inv_mw[l], Yd[l] = Yf[l];
      const float gcf = float(kRu) * mwi;
      const float ef = (float)q[4] * invf - 0.5f * (float)vel2;
      temp = newton_temperature_w<float, NS>(C, rec_f32, ef, Yf, gcf, (float)t_warm, capped);
      gas_const = gcf;
    }
    if (capped) flags |= kStatusNewtonCap;
    pres = rho * temp * gas_const;
  }
  if (!(rho > 0) || !(pres > 0) || !(temp > 0) || !isfinite(q[4])) flags |= kStatusNonFinite;
  if (a.vel) a.vel[p] = sqrt(vel2);
  T* Pn = a.Pn;
  Pn[p] = T(rho);
  Pn[N + p] = T(u);
  Pn[2 * N + p] = T(v);
  Pn[3 * N + p] = T(w);
  Pn[4 * N + p] = T(pres - C.p_ref);  // gauge pressure
  Pn[5 * N + p] = T(temp);
  T Yt[A];
#pragma unroll
  for (int l = 0; l < A; ++l)
    if (l < ns) Yt[l] = T(Yd[l]), Pn[(6 + l) * N + p] = Yt[l];
  if (a.closure) return;  // transport and the time step follow from the closure kernel
  T mu, lam, rd[A], gam, c;
  point_props<T, NS>(C, rec, T(temp), Yt, mu, lam, rd, gam, c);
  T* Prn = a.Prn;
  Prn[p] = mu;
  Prn[N + p] = lam;
#pragma unroll
  for (int l = 0; l < A; ++l)
    if (l < ns) Prn[(2 + l) * N + p] = rd[l];
  if (want_dt) {
    const double dtl = local_time_step<T>(C, G, N, p, rho, u, v, w, (double)c, (double)gam, (double)mu, three_d);
    dt_min = fmin(dt_min, dtl);
  }
    }

template <typename T, int NS>
__device__ __forceinline__ void point_update(const ChemParams &C, const T *rec, const double *rec_d,
                                             const StageArgs<T> &a, int p, int N,
                                             const double *dq, double dt, double t_warm, bool three_d,
                                             unsigned &flags, double &dt_min) {
  constexpr int A = SpecCount<NS>::kArr;
  constexpr int NV = 5 + A;
  const int ns = SpecCount<NS>::n(C);
  const int nv = 5 + ns;
  p = CCB_IDX(C, p, N);
  const T *__restrict__ G = a.G;
  const double dtj = dt / (double)G[p];
  // whether this point's step enters the next global time step, read with
  // the state rather than behind the stores below
  const bool want_dt = a.dt_next && !((a.skip_dt[p >> 5] >> (p & 31)) & 1u);
  double q[NV];
  // all loads first, then the stores: Qout may alias Qin, so a store between
  // two loads would keep the compiler from issuing the loads together
#pragma unroll
  for (int l = 0; l < NV; ++l)
    if (l < nv) q[l] = conserved_update<T>(C, a, p, N, l, dq[l], dtj, three_d);
  point_finish<T, NS>(C, rec, rec_d, a, p, N, q, t_warm, three_d, want_dt, flags, dt_min);
}

// L2 prefetch of elements [s, e) of one field row through the bulk copy
// engine: a hint that nothing waits on.  The range is clamped to the field's
// [0, N) (N is a multiple of 32 points) and widened to 16-byte boundaries.
template <typename E>
__device__ __forceinline__ void l2_prefetch(const E *field, int N, int s, int e) {
  constexpr int kPer16 = 16 / (int)sizeof(E);
  s = max(s, 0) & ~(kPer16 - 1);
  e = (min(e, N) + kPer16 - 1) & ~(kPer16 - 1);
  if (e <= s) return;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(field + s), "r"((unsigned)((e - s) * sizeof(E)))
               : "memory");
}

// While plane k is processed, bring into L2 what plane k+1 will read for
// the first time: primitives of plane k+3 (tile + 2-point halo in i and j),
// transport and geometry of plane k+2 (1-point halo), conserved variables of
// plane k+1 (tile).  Rows are spread over the CTA's threads.
template <typename T>
__device__ __forceinline__ void prefetch_planes(const StageArgs<T> &a, const BlockInfo &B, const Tile &t, int k,
                                                int np, int npr, int nv, int tid) {
  const int N = (int)a.N, sj = B.nx, sk = B.nx * B.ny;
  const int i_lo = t.i0 - 4, i_hi = t.i0 + kTX + 4;
  auto rows = [&](auto *base, int nf, int kp, int j_lo, int j_hi, int ilo, int ihi, int &e0) {
    const int nr = j_hi - j_lo;
    const int n = nf * nr;
    for (int e = tid - e0; e < n; e += kTX * kTY) {
      if (e < 0) continue;
      const int f = e / nr, j = j_lo + e % nr;
      const int row = (int)B.base + sk * kp + sj * j;
      l2_prefetch(base + (size_t)f * N, N, row + ilo, row + ihi);
    }
    e0 = (e0 + n) % (kTX * kTY);  // next group starts on the next free thread
  };
  int e0 = 0;
  const int kmax = B.mz - 1 + B.g;
  if (k + 3 <= kmax)
    rows(a.P, np, k + 3, max(t.j0 - 2, -B.g), min(t.j0 + kTY + 2, B.my + B.g), i_lo, i_hi, e0);
  if (k + 2 <= kmax) {
    rows(a.Pr, npr, k + 2, max(t.j0 - 1, -B.g), min(t.j0 + kTY + 1, B.my + B.g), i_lo, i_hi, e0);
    rows(a.G, 10, k + 2, max(t.j0 - 1, -B.g), min(t.j0 + kTY + 1, B.my + B.g), i_lo, i_hi, e0);
  }
  if (k + 1 < t.k1) {
    rows(a.Qin, nv, k + 1, t.j0, min(t.j0 + kTY, B.my), t.i0, t.i0 + kTX, e0);
    if (a.a != 0.0 && a.Qn != a.Qin) rows(a.Qn, nv, k + 1, t.j0, min(t.j0 + kTY, B.my), t.i0, t.i0 + kTX, e0);
  }
}

// Dynamic shared memory of k_stage: FP64 NASA records, bulk-precision
// records (aliasing the FP64 ones when T is double), face flux planes.
template <typename T, int NS>
struct StageSmem {
  static constexpr int A = SpecCount<NS>::kArr;
  static constexpr int NV = 5 + A;
  static constexpr size_t kRecD = sizeof(double) * A * 2 * kRecLen;
  static constexpr size_t kRecBytes = kRecD + (sizeof(T) == sizeof(double) ? 0 : sizeof(T) * A * 2 * kRecLen);
  static constexpr size_t kBytes =
      kRecBytes + sizeof(T) * NV * (kTY * (kTX + 1) + (kTY + 1) * kTX + 2 * kTY * kTX);
  static_assert(kRecD % 16 == 0 && kRecBytes % 16 == 0, "records must stay 16-byte aligned");
};

template <typename T, int NS>
__global__ void __launch_bounds__(kTX *kTY, sizeof(T) == 8 ? 1 : 2)
    k_stage(const StageArgs<T> a, const __grid_constant__ ChemParams C) {
  constexpr int A = SpecCount<NS>::kArr;
  constexpr int NV = 5 + A;
  const int ns = SpecCount<NS>::n(C);
  const int nv = 5 + ns;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // NASA-7 records of both precisions (the bulk one for the face and point
  // thermodynamics, FP64 for the temperature Newton), then the face fluxes.
  double *sRecD = reinterpret_cast<double *>(smem_raw);  // [A][2][kRecLen]
  T *sRec = reinterpret_cast<T *>(smem_raw + (sizeof(T) == sizeof(double) ? 0 : StageSmem<T, NS>::kRecD));
  T *sFx = reinterpret_cast<T *>(smem_raw + StageSmem<T, NS>::kRecBytes);  // [NV][kTY][kTX+1]
  T *sFy = sFx + NV * kTY * (kTX + 1);                   // [NV][kTY+1][kTX]
  T *sFz0 = sFy + NV * (kTY + 1) * kTX;                  // [NV][kTY][kTX]
  T *sFz1 = sFz0 + NV * kTY * kTX;
  constexpr int XS = kTY * (kTX + 1), YS = (kTY + 1) * kTX, ZS = kTY * kTX;

  const Tile t = a.tiles[blockIdx.x];
  const BlockInfo B = a.blocks[t.blk];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = t.i0 + tx, j = t.j0 + ty;
  const bool act = (i < B.mx) && (j < B.my);
  const int N = (int)a.N;
  const int sj = B.nx, sk = B.nx * B.ny;
  const int col = (int)B.base + i + sj * j;
  const T *__restrict__ P = a.P;
  const T *__restrict__ Pr = a.Pr;
  const T *__restrict__ G = a.G;
  const bool three_d = B.mz > 1;
  T F[NV];

  {
    const int tid = ty * kTX + tx, nrec = ns * 2 * kRecLen;
    const double *gd = param_rec<double>(C);
    const T *gt = param_rec<T>(C);
    for (int e = tid; e < nrec; e += kTX * kTY) {
      sRecD[e] = gd[e];
      if (sizeof(T) != sizeof(double)) sRec[e] = gt[e];
    }
    __syncthreads();
  }
  const bool ex_x = (ty == 1) && (tx < kTY) && (t.j0 + tx < B.my);  // -x boundary face of row tx
  const bool ex_y = (ty == 0) && act;                               // -y boundary face of column tx
  unsigned flags = 0;
  double dt_min = 1e300;
  T *zprev = sFz1, *zcur = sFz0;

  // k = k0-1 only produces the -z face of the first plane.  Every face flux
  // goes through the single call site below, so a face shared by two tiles
  // or two blocks is computed by identical instructions.
  for (int k = t.k0 - 1; k < t.k1; ++k) {
    const int p = col + sk * k;
    const bool first = (k < t.k0);
    prefetch_planes<T>(a, B, t, k, 6 + ns, 2 + ns, nv, ty * kTX + tx);
#pragma unroll 1
    for (int it = 0; it < 5; ++it) {
      bool doit;
      int d, sd;
      int pf = p;
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
        pf = (int)B.base + (t.i0 - 1) + sj * (t.j0 + tx) + sk * k;
      } else {
        doit = ex_y && !first;
        d = 1, sd = sj, dst = sFy + tx, ds = YS;
        pf = p - sj;
      }
      if (doit) {
        face_flux<T, NS>(C, sRec, P, Pr, G, N, pf, d, sd, sj, sk, F);
#pragma unroll
        for (int l = 0; l < NV; ++l)
          if (l < nv) dst[l * ds] = F[l];
      }
    }
    if (first) {
      T *tmp = zprev;
      zprev = zcur;
      zcur = tmp;
      continue;
    }
    __syncthreads();
    if (act) {
      // dq = -(sum over directions of F(+1/2) - F(-1/2))
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
      // time step of this point: global (RK) or local (steady, from the current state)
      double dt;
      if (a.local_dt) {
        T Y[A];
#pragma unroll
        for (int l = 0; l < A; ++l)
          if (l < ns) Y[l] = P[(6 + l) * N + p];
        T gam, c;
        gamma_and_c<T, NS>(C, sRec, P[5 * N + p], Y, gam, c);
        dt = local_time_step<T>(C, G, N, p, (double)P[p], (double)P[N + p], (double)P[2 * N + p],
                                (double)P[3 * N + p], (double)c, (double)gam, (double)Pr[p], three_d);
      } else {
        dt = *a.dt;
      }
      point_update<T, NS>(C, sRec, sRecD, a, p, N, dq, dt, (double)P[5 * N + p], three_d, flags, dt_min);
    }
    T *tmp = zprev;
    zprev = zcur;
    zcur = tmp;
    __syncthreads();
  }
  if (a.dt_next) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dt_min = fmin(dt_min, __shfl_xor_sync(0xffffffffu, dt_min, o));
    if (tx == 0) atomic_min_pos_double(a.dt_next, dt_min);
  }
  const unsigned any = __reduce_or_sync(0xffffffffu, flags);
  if (any && tx == 0) atomicOr(a.status, any);
}

// ---------------------------------------------------------------- halo

template <typename T>
struct RefPtrs {
  const T *P;
  const T *Pr;
  const double *Q;
  int64_t stride;
  int64_t idx;
};

template <typename T>
__device__ __forceinline__ RefPtrs<T> resolve(const HaloArgs<T> &a, const HaloRef &r) {
  if (r.kind == 0) return {a.P, a.Pr, a.Q, a.N, r.idx};
  if (r.kind == 1) return {a.Pprev, a.Prprev, a.Qprev, a.N, r.idx};
  return {a.sP, a.sPr, a.sQ, a.NS_cap, r.idx};
}

// Total energy of a point from primitives (Thermo.cu:66-86), FP64.
template <int NS>
__device__ __forceinline__ double total_energy(const ChemParams &C, double rho, double u, double v, double w, double p,
                                               double t, const double *Y) {
  const double *rec = param_rec<double>(C);
  constexpr int A = SpecCount<NS>::kArr;
  const int ns = SpecCount<NS>::n(C);
  double e = 0.5 * rho * (u * u + v * v + w * w);
  if (NS == 0 || (NS < 0 && ns == 0)) return e + p / (kGammaAir - 1);
#pragma unroll
  for (int l = 0; l < A; ++l)
    if (l < ns) e += nasa_h<double>(C.d, rec, l, t) * (rho * Y[l]);
  return e - p;
}

// Phase A: evaluate halo node e into its scratch slot.
template <typename T, int NS>
__device__ __forceinline__ void halo_node(const HaloArgs<T> &a, const ChemParams &C, int64_t e) {
  constexpr int A = SpecCount<NS>::kArr;
  const int ns = SpecCount<NS>::n(C);
  const int nv = 5 + ns;
  const HaloNode nd = a.nodes[e];
  const int64_t o = CCB_IDX(C, nd.slot, a.NS_cap);
  const int64_t S = a.NS_cap;
  double pr[6];
  double Y[A];
  double q[5 + A];
  bool props_copy = false;
  RefPtrs<T> ra = resolve(a, nd.a);
  ra.idx = CCB_IDX(C, ra.idx, ra.stride);
  // every field is loaded into registers before the first store: the stores
  // may alias the sources as far as the compiler knows, and interleaving them
  // would serialise one memory round trip per field
  if (nd.op == kHaloCopy) {
    T vP[6 + A], vPr[2 + A];
    double vQ[5 + A];
#pragma unroll
    for (int f = 0; f < 6 + A; ++f)
      if (f < 6 + ns) vP[f] = ra.P[f * ra.stride + ra.idx];
#pragma unroll
    for (int f = 0; f < 2 + A; ++f)
      if (f < 2 + ns) vPr[f] = ra.Pr[f * ra.stride + ra.idx];
#pragma unroll
    for (int f = 0; f < 5 + A; ++f)
      if (f < nv) vQ[f] = ra.Q[f * ra.stride + ra.idx];
#pragma unroll
    for (int f = 0; f < 6 + A; ++f)
      if (f < 6 + ns) a.sP[f * S + o] = vP[f];
#pragma unroll
    for (int f = 0; f < 2 + A; ++f)
      if (f < 2 + ns) a.sPr[f * S + o] = vPr[f];
#pragma unroll
    for (int f = 0; f < 5 + A; ++f)
      if (f < nv) a.sQ[f * S + o] = vQ[f];
    return;
  }
  if (nd.op == kHaloAvg) {
    RefPtrs<T> rb = resolve(a, nd.b);
    rb.idx = CCB_IDX(C, rb.idx, rb.stride);
    T xa[6 + A], xb[6 + A], vPr[2 + A];
    double qa[5 + A], qb[5 + A];
#pragma unroll
    for (int f = 0; f < 6 + A; ++f)
      if (f < 6 + ns) xa[f] = ra.P[f * ra.stride + ra.idx], xb[f] = rb.P[f * rb.stride + rb.idx];
#pragma unroll
    for (int f = 0; f < 5 + A; ++f)
      if (f < nv) qa[f] = ra.Q[f * ra.stride + ra.idx], qb[f] = rb.Q[f * rb.stride + rb.idx];
#pragma unroll
    for (int f = 0; f < 2 + A; ++f)
      if (f < 2 + ns) vPr[f] = ra.Pr[f * ra.stride + ra.idx];
    bool same = true;
#pragma unroll
    for (int f = 0; f < 6 + A; ++f)
      if (f < 6 + ns) {
        same = same && (xa[f] == xb[f]);
        a.sP[f * S + o] = T(0.5) * (xb[f] + xa[f]);
      }
#pragma unroll
    for (int f = 0; f < 5 + A; ++f)
      if (f < nv) a.sQ[f * S + o] = 0.5 * (qb[f] + qa[f]);
    if (same) {
#pragma unroll
      for (int f = 0; f < 2 + A; ++f)
        if (f < 2 + ns) a.sPr[f * S + o] = vPr[f];
      return;
    }
    // averaged state: recompute its transport properties below
    for (int f = 0; f < 6; ++f) pr[f] = (double)a.sP[f * S + o];
#pragma unroll
    for (int l = 0; l < A; ++l)
      if (l < ns) Y[l] = (double)a.sP[(6 + l) * S + o];
  } else {
    const BcDevice &bc = a.bcs[nd.bc];
    if (nd.op == kHaloInflow) {
      pr[0] = bc.rho, pr[1] = bc.u, pr[2] = bc.v, pr[3] = bc.w, pr[4] = bc.p, pr[5] = bc.T;
#pragma unroll
      for (int l = 0; l < A; ++l)
        if (l < ns) Y[l] = bc.yk[l];
      for (int f = 0; f < 6; ++f) a.sP[f * S + o] = T(f == 4 ? pr[f] - C.p_ref : pr[f]);
#pragma unroll
      for (int l = 0; l < A; ++l)
        if (l < ns) a.sP[(6 + l) * S + o] = T(Y[l]);
      a.sQ[o] = bc.rho;
      a.sQ[S + o] = bc.rho * bc.u;
      a.sQ[2 * S + o] = bc.rho * bc.v;
      a.sQ[3 * S + o] = bc.rho * bc.w;
      a.sQ[4 * S + o] = bc.rhoE;
#pragma unroll
      for (int l = 0; l < A; ++l)
        if (l < ns) a.sQ[(5 + l) * S + o] = bc.rho * bc.yk[l];
      a.sPr[o] = T(bc.mu);
      a.sPr[S + o] = T(bc.lam);
#pragma unroll
      for (int l = 0; l < A; ++l)
        if (l < ns) a.sPr[(2 + l) * S + o] = T(bc.rho_d[l]);
      props_copy = true;
    } else {
      // BoundCond.cu:529-629 apply_wall
      const double t_in = (double)ra.P[5 * ra.stride + ra.idx];
      const double p_in = (double)ra.P[4 * ra.stride + ra.idx] + C.p_ref;  // stored as gauge pressure
      double mwi = 0;
#pragma unroll
      for (int l = 0; l < A; ++l)
        if (l < ns) Y[l] = (double)ra.P[(6 + l) * ra.stride + ra.idx], mwi += Y[l] * C.d.inv_mw[l];
      const double mw = (NS == 0 || (NS < 0 && ns == 0)) ? kMwAir : 1.0 / mwi;
      if (nd.op == kHaloWallFace) {
        const double tw = bc.thermal_type == 1 ? t_in : bc.t_wall;
        pr[0] = p_in * mw / (tw * kRu);
        pr[1] = pr[2] = pr[3] = 0;
        pr[4] = p_in;
        pr[5] = tw;
      } else {
        RefPtrs<T> rb = resolve(a, nd.b);
        rb.idx = CCB_IDX(C, rb.idx, rb.stride);
        const double tw = bc.thermal_type == 1 ? (double)rb.P[5 * rb.stride + rb.idx] : bc.t_wall;
        double tg = t_in;
        if (bc.thermal_type == 0) {
          tg = 2 * tw - t_in;
          if (tg <= 0.1 * tw) tg = tw;
        }
        pr[0] = p_in * mw / (tg * kRu);
        pr[1] = -(double)ra.P[1 * ra.stride + ra.idx];
        pr[2] = -(double)ra.P[2 * ra.stride + ra.idx];
        pr[3] = -(double)ra.P[3 * ra.stride + ra.idx];
        pr[4] = p_in;
        pr[5] = tg;
      }
      for (int f = 0; f < 6; ++f) a.sP[f * S + o] = T(f == 4 ? pr[f] - C.p_ref : pr[f]);
#pragma unroll
      for (int l = 0; l < A; ++l)
        if (l < ns) a.sP[(6 + l) * S + o] = T(Y[l]);
      q[0] = pr[0];
      q[1] = pr[0] * pr[1];
      q[2] = pr[0] * pr[2];
      q[3] = pr[0] * pr[3];
      q[4] = total_energy<NS>(C, pr[0], pr[1], pr[2], pr[3], pr[4], pr[5], Y);
#pragma unroll
      for (int l = 0; l < A; ++l)
        if (l < ns) q[5 + l] = Y[l] * pr[0];
      for (int f = 0; f < nv; ++f) a.sQ[f * S + o] = q[f];
    }
  }
  if (!props_copy) {
    T Yt[A], mu, lam, rd[A], gam, c;
#pragma unroll
    for (int l = 0; l < A; ++l)
      if (l < ns) Yt[l] = T(Y[l]);
    point_props<T, NS>(C, param_rec<T>(C), T(pr[5]), Yt, mu, lam, rd, gam, c);
    a.sPr[o] = mu;
    a.sPr[S + o] = lam;
#pragma unroll
    for (int l = 0; l < A; ++l)
      if (l < ns) a.sPr[(2 + l) * S + o] = rd[l];
  }
}

// Phase A, one launch per level: the nodes [a.begin, a.end).
template <typename T, int NS>
__global__ void k_halo_nodes(const HaloArgs<T> a, const __grid_constant__ ChemParams C) {
  const int64_t e = a.begin + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= a.end) return;
  halo_node<T, NS>(a, C, e);
}

// Phase B: write every changed point from its resolved source.  One thread
// per (copy, array): grid y selects P, Pr or Q, and the thread moves all
// fields of that array for its copy, loading them all before the first
// store (the stores may alias the sources as far as the compiler knows).
// Consecutive threads take consecutive copies, whose destinations (and
// mostly sources) are consecutive, so every field access is coalesced; the
// copy record is read once per array rather than once per field.
// Interior points rewritten by phase B (coincident interface layers)
// contribute their post-exchange local time step to the next global step,
// as the reference evaluates the step after the exchange (Driver.cu:150-163):
// the thread that copies a flagged copy's primitives evaluates it from the
// values it has just written (and the source's viscosity, which the
// transport copy writes to the same point).
template <typename T, int NS>
__device__ __forceinline__ double halo_copy_dt(const HaloArgs<T> &a, const ChemParams &C, const HaloCopy &c,
                                               const T *v, T mu) {
  constexpr int A = SpecCount<NS>::kArr;
  const int ns = SpecCount<NS>::n(C);
  T Y[A], gam, cs;
#pragma unroll
  for (int l = 0; l < A; ++l)
    if (l < ns) Y[l] = v[6 + l];
  gamma_and_c<T, NS>(C, param_rec<T>(C), v[5], Y, gam, cs);
  return local_time_step<T>(C, a.G, a.N, c.dst, (double)v[0], (double)v[1], (double)v[2], (double)v[3], (double)cs,
                            (double)gam, (double)mu, (c.src.pad & 2) != 0);
}

template <typename T, int NS>
__device__ __forceinline__ double halo_copy(const HaloArgs<T> &a, const ChemParams &C, int64_t e, int which,
                                            int np, int npr, int nq, int q_filter = 0) {
  constexpr int A = SpecCount<NS>::kArr;
  HaloCopy c = a.copies[a.begin + e];
  if (which == 2 && q_filter != 0) {
    // a ghost point's conserved state: no stage kernel reads it (they read Q
    // at interior points only), so steps leave it (q_filter 1) and a later
    // pass writes it before the state is read out (q_filter 2).  Ghost points
    // the halo program itself reads (bit 2) and copies of a previous value
    // keep running every time, so those chains stay exact.
    const bool ghost = (c.src.pad & 5) == 0 && c.src.kind != 1;
    if (ghost == (q_filter == 1)) return 1e300;
  }
  c.dst = CCB_IDX(C, c.dst, a.N);
  RefPtrs<T> r = resolve(a, c.src);
  r.idx = CCB_IDX(C, r.idx, r.stride);
  double dt = 1e300;
  if (which == 0) {
    T v[6 + A];
#pragma unroll
    for (int f = 0; f < 6 + A; ++f)
      if (f < np) v[f] = r.P[f * r.stride + r.idx];
#pragma unroll
    for (int f = 0; f < 6 + A; ++f)
      if (f < np) a.P[f * a.N + c.dst] = v[f];
    if (a.dt_next && ((a.dt_copy_mask[e >> 5] >> (e & 31)) & 1u))
      dt = halo_copy_dt<T, NS>(a, C, c, v, r.Pr[r.idx]);
  } else if (which == 1) {
    T v[2 + A];
#pragma unroll
    for (int f = 0; f < 2 + A; ++f)
      if (f < npr) v[f] = r.Pr[f * r.stride + r.idx];
#pragma unroll
    for (int f = 0; f < 2 + A; ++f)
      if (f < npr) a.Pr[f * a.N + c.dst] = v[f];
  } else {
    double v[5 + A];
#pragma unroll
    for (int f = 0; f < 5 + A; ++f)
      if (f < nq) v[f] = r.Q[f * r.stride + r.idx];
#pragma unroll
    for (int f = 0; f < 5 + A; ++f)
      if (f < nq) a.Q[f * a.N + c.dst] = v[f];
  }
  return dt;
}

// Phase B in one launch: every changed point from its resolved source (grid
// y + y0 selects P, Pr or Q; consecutive threads take consecutive copies;
// q_filter as in halo_copy), the
// post-exchange time step of the rewritten interior points (a.dt_next), and
// the zeroing of |V| at wall-face points (vel).
template <typename T, int NS>
__global__ void k_halo_copy_fields(const HaloArgs<T> a, const __grid_constant__ ChemParams C, int np, int npr,
                                   int nq, double *vel, const int64_t *vel_zero, int64_t n_vel_zero, int q_filter,
                                   int y0) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;  // copy (grid x)
  const int which = (int)blockIdx.y + y0;
  double dt = 1e300;
  if (e < a.end - a.begin) dt = halo_copy<T, NS>(a, C, e, which, np, npr, nq, q_filter);
  if (a.dt_next && which == 0) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dt = fmin(dt, __shfl_xor_sync(0xffffffffu, dt, o));
    if ((threadIdx.x & 31) == 0) atomic_min_pos_double(a.dt_next, dt);
  }
  if (vel && which == 2)
    for (int64_t z = e; z < n_vel_zero; z += (int64_t)gridDim.x * blockDim.x) vel[vel_zero[z]] = 0.0;
}

// Bounded grid-wide barrier of a cooperative launch (every CTA resident):
// thread 0 of each CTA arrives on the counter after the CTA's writes (the
// CTA barrier and its fence make them visible at GPU scope first); the last
// arrival resets the counter and advances the generation, the others poll the
// generation (at most max_polls times, 64 ns apart).  Returns false, in every
// thread of the CTA, when the wait gave up.
__device__ __forceinline__ bool grid_sync_bounded(GridBarrier *bar, long long max_polls) {
  __shared__ int ok_sh;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    volatile unsigned *vgen = &bar->gen;
    const unsigned g = *vgen;
    __threadfence();
    const unsigned arrived = atomicAdd(&bar->count, 1u) + 1u;
    if (arrived == gridDim.x) {
      atomicExch(&bar->count, 0u);
      __threadfence();
      atomicAdd(&bar->gen, 1u);
    } else {
      for (long long polls = 0; *vgen == g;) {
        if (++polls > max_polls) {
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
      __threadfence();
    }
    ok_sh = ok;
  }
  __syncthreads();
  return ok_sh != 0;
}

// Phase A in one cooperative launch: the node levels with a grid-wide
// barrier between levels (every node of a level reads only the state and
// lower levels).  A barrier that gives up sets kStatusHaloTimeout and the
// CTA returns.
template <typename T, int NS>
__global__ void __launch_bounds__(128)
    k_halo_levels(const HaloArgs<T> a, const __grid_constant__ ChemParams C, const HaloLevels lv, GridBarrier *bar,
                  unsigned *status) {
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int l = 0; l < lv.n; ++l) {
    if (l > 0 && !grid_sync_bounded(bar, C.max_spins)) {
      if (threadIdx.x == 0) atomicOr(status, kStatusHaloTimeout);
      return;
    }
    for (int64_t e = lv.begin[l] + tid; e < lv.begin[l + 1]; e += stride) halo_node<T, NS>(a, C, e);
  }
}

// ------------------------------------------------------------ setup / misc

// Field.cu:150-176 compute_cv_from_bv over every arena point (FP64 input).
template <int NS>
__global__ void k_cv_from_bv(const __grid_constant__ ChemParams C, const double *P0, double *Q, int64_t N,
                             double *vel) {
  constexpr int A = SpecCount<NS>::kArr;
  const int ns = SpecCount<NS>::n(C);
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= N) return;
  const double rho = P0[p], u = P0[N + p], v = P0[2 * N + p], w = P0[3 * N + p], pr = P0[4 * N + p], t = P0[5 * N + p];
  if (!(rho > 0)) return;  // padding points of the arena
  double Y[A];
#pragma unroll
  for (int l = 0; l < A; ++l)
    if (l < ns) Y[l] = P0[(6 + l) * N + p];
  Q[p] = rho;
  Q[N + p] = rho * u;
  Q[2 * N + p] = rho * v;
  Q[3 * N + p] = rho * w;
  Q[4 * N + p] = total_energy<NS>(C, rho, u, v, w, pr, t, Y);
  if (vel) vel[p] = sqrt(u * u + v * v + w * w);
#pragma unroll
  for (int l = 0; l < A; ++l)
    if (l < ns) Q[(5 + l) * N + p] = rho * Y[l];
}

// Transport properties at every arena point (Field.cu:178-210).
template <typename T, int NS>
__global__ void k_props_all(const __grid_constant__ ChemParams C, const T *P, T *Pr, int64_t N) {
  constexpr int A = SpecCount<NS>::kArr;
  const int ns = SpecCount<NS>::n(C);
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= N) return;
  if (!(P[p] > T(0))) return;
  T Y[A], mu, lam, rd[A], gam, c;
#pragma unroll
  for (int l = 0; l < A; ++l)
    if (l < ns) Y[l] = P[(6 + l) * N + p];
  point_props<T, NS>(C, param_rec<T>(C), P[5 * N + p], Y, mu, lam, rd, gam, c);
  Pr[p] = mu;
  Pr[N + p] = lam;
#pragma unroll
  for (int l = 0; l < A; ++l)
    if (l < ns) Pr[(2 + l) * N + p] = rd[l];
}

// Geometric part of the momentum flux difference that the gauge pressure
// leaves out: gcl[c][p] = sum over the face directions d of k_c(p, +d) -
// k_c(p, -d), with the face vector k = (J_0 m_0 + J_1 m_1) / 2 formed in the
// bulk precision exactly as the face fluxes form it.  Zero on uniform grids.
template <typename T>
__global__ void k_gcl(const BlockInfo *blocks, int nblocks, const T *G, int64_t N, int64_t n_interior_total,
                      double *gcl) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_interior_total;
       g += (int64_t)gridDim.x * blockDim.x) {
    int b = 0;
    while (b + 1 < nblocks && blocks[b + 1].interior_off <= g) ++b;
    const BlockInfo B = blocks[b];
    const int64_t r = g - B.interior_off;
    const int i = (int)(r % B.mx), j = (int)((r / B.mx) % B.my), k = (int)(r / ((int64_t)B.mx * B.my));
    const int64_t p = B.base + i + (int64_t)B.nx * j + (int64_t)B.nx * B.ny * k;
    const int64_t st[3] = {1, B.nx, (int64_t)B.nx * B.ny};
    double acc[3] = {0, 0, 0};
    for (int d = 0; d < (B.mz > 1 ? 3 : 2); ++d) {
      const int64_t q0 = p - st[d], q1 = p, q2 = p + st[d];
      for (int c = 0; c < 3; ++c) {
        const T *m = G + (1 + 3 * d + c) * N;
        const T kp = T(0.5) * (G[q1] * m[q1] + G[q2] * m[q2]);
        const T km = T(0.5) * (G[q0] * m[q0] + G[q1] * m[q1]);
        acc[c] += (double)kp - (double)km;
      }
    }
    for (int c = 0; c < 3; ++c) gcl[c * N + p] = acc[c];
  }
}

// Global time step of the current state over interior points.// Global time step of the current state over interior points.
template <typename T, int NS>
__global__ void k_dt_reduce(const __grid_constant__ ChemParams C, const BlockInfo *blocks, int nblocks, const T *P,
                            const T *Pr, const T *G, int64_t N, int64_t n_interior_total,
                            unsigned long long *dt_out) {
  constexpr int A = SpecCount<NS>::kArr;
  const int ns = SpecCount<NS>::n(C);
  double m = 1e300;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_interior_total;
       g += (int64_t)gridDim.x * blockDim.x) {
    int b = 0;
    while (b + 1 < nblocks && blocks[b + 1].interior_off <= g) ++b;
    const BlockInfo B = blocks[b];
    const int64_t r = g - B.interior_off;
    const int i = (int)(r % B.mx);
    const int j = (int)((r / B.mx) % B.my);
    const int k = (int)(r / ((int64_t)B.mx * B.my));
    const int64_t p = B.base + i + (int64_t)B.nx * j + (int64_t)B.nx * B.ny * k;
    T Y[A], gam, c;
#pragma unroll
    for (int l = 0; l < A; ++l)
      if (l < ns) Y[l] = P[(6 + l) * N + p];
    gamma_and_c<T, NS>(C, param_rec<T>(C), P[5 * N + p], Y, gam, c);
    const double dtl = local_time_step<T>(C, G, N, p, (double)P[p], (double)P[N + p], (double)P[2 * N + p],
                                          (double)P[3 * N + p], (double)c, (double)gam, (double)Pr[p], B.mz > 1);
    m = fmin(m, dtl);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomic_min_pos_double(dt_out, m);
}

}  // namespace ccb
