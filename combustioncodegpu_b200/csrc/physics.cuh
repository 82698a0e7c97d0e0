// Device physics of the residual path, templated on the bulk precision T
// (double for the plain path, float for the mixed path) and on the species
// count NS (compile-time; -1 = runtime count up to kMaxSpec, 0 = perfect air).
//
// Reference counterparts (file:line in CombustionCodeGPU):
//   NASA-7 h/cp with linear h below T_low ......... Thermo.cu:7-63
//   total energy .................................. Thermo.cu:66-86
//   temperature Newton (FP64 in every precision) .. Thermo.cu:89-125
//   Sutherland ..................................... Transport.cu:7-10
//   Wilke / constant-Schmidt transport ............. Transport.cu:43-96 (X[l])
//   MUSCL + minmod + face thermo ................... Reconstruction.cu:26-89, Limiter.cuh:13-16
//   AUSM+ ........................................... InviscidScheme.cu:24-108
// The polynomials are evaluated in Horner form and sqrt(mu_m/mu_n) as
// sqrt(mu_m)/sqrt(mu_n); both differ from the reference only by rounding.
#pragma once
#include <cuda_runtime.h>

#include "cc_common.h"

namespace ccb {

template <typename T>
__device__ __forceinline__ const SpecTables<T> &tab(const ChemParams &C);
template <>
__device__ __forceinline__ const SpecTables<double> &tab<double>(const ChemParams &C) {
  return C.d;
}
template <>
__device__ __forceinline__ const SpecTables<float> &tab<float>(const ChemParams &C) {
  return C.f;
}

template <int NS>
struct SpecCount {
  static constexpr int kArr = NS > 0 ? NS : (NS == 0 ? 1 : kMaxSpec);
  __device__ __forceinline__ static int n(const ChemParams &C) { return NS >= 0 ? NS : C.ns; }
};

// Division, reciprocal, square root and x^-0.145 of the bulk precision: IEEE
// in FP64 (the plain path), hardware approximations in FP32 (the mixed path;
// relative error of a few ulp, far below the path's 1e-5 error budget).
__device__ __forceinline__ double fdiv(double a, double b) { return a / b; }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double frcp(double a) { return 1.0 / a; }
__device__ __forceinline__ float frcp(float a) { return __fdividef(1.0f, a); }
__device__ __forceinline__ double fsqrt(double a) { return sqrt(a); }
__device__ __forceinline__ float fsqrt(float a) { return a * rsqrtf(a); }

// NASA-7 records (SpecTables::rec) are read through a pointer `rec` to the
// [kMaxSpec][2][kRecLen] array: the stage kernel points it at a copy in
// shared memory, other kernels at the constant bank (param_rec).  The range
// is chosen per thread by the record address, so a warp whose points
// straddle t_mid reads two records in one vector load instead of serialising
// on divergent constant addresses, and the coefficients cannot be hoisted
// out of the surrounding loops into registers.
template <typename T>
__device__ __forceinline__ const T *param_rec(const ChemParams &C) {
  return &tab<T>(C).rec[0][0][0];
}

template <typename T>
__device__ __forceinline__ void load_rec(const T *r, T (&x)[kRecLen]);
template <>
__device__ __forceinline__ void load_rec<float>(const float *r, float (&x)[kRecLen]) {
  const float4 *v = reinterpret_cast<const float4 *>(r);
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const float4 w = v[q];
    x[4 * q] = w.x, x[4 * q + 1] = w.y, x[4 * q + 2] = w.z, x[4 * q + 3] = w.w;
  }
}
template <>
__device__ __forceinline__ void load_rec<double>(const double *r, double (&x)[kRecLen]) {
  const double2 *v = reinterpret_cast<const double2 *>(r);
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const double2 w = v[q];
    x[2 * q] = w.x, x[2 * q + 1] = w.y;
  }
}

// Enthalpy and cp of species k at temperature t (per unit mass); below
// t_low, h continues linearly with cp(t_low) (Thermo.cu:7-63).
template <typename T>
__device__ __forceinline__ void nasa_h_cp(const SpecTables<T> &S, const T *rec, int k, T t, T &h, T &cp) {
  const T tl = S.t_low[k];
  const bool below = t < tl;
  const T te = below ? tl : t;
  const bool lo = below || t < S.t_mid[k];
  T x[kRecLen];
  load_rec<T>(rec + (2 * k + (lo ? 0 : 1)) * kRecLen, x);
  const T c = x[0] + te * (x[1] + te * (x[2] + te * (x[3] + te * x[4])));
  T hh = x[10] + te * (x[5] + te * (x[6] + te * (x[7] + te * (x[8] + te * x[9]))));
  if (below) hh += c * (t - te);
  h = hh * S.r_over_mw[k];
  cp = c * S.r_over_mw[k];
}

template <typename T>
__device__ __forceinline__ T nasa_h(const SpecTables<T> &S, const T *rec, int k, T t) {
  T h, cp;
  nasa_h_cp(S, rec, k, t, h, cp);
  return h;
}

template <typename T>
__device__ __forceinline__ T nasa_cp(const SpecTables<T> &S, const T *rec, int k, T t) {
  const T tl = S.t_low[k];
  const T te = t < tl ? tl : t;
  T x[kRecLen];
  load_rec<T>(rec + (2 * k + (t < S.t_mid[k] ? 0 : 1)) * kRecLen, x);
  return (x[0] + te * (x[1] + te * (x[2] + te * (x[3] + te * x[4])))) * S.r_over_mw[k];
}

template <typename T>
__device__ __forceinline__ T sutherland(T t) {
  // 1.716e-5 (T/273)^1.5 (273+111)/(T+111)
  const T r = t / T(273);
  return T(1.716e-5) * (r * sqrt(r)) * T(384) / (t + T(111));
}

template <typename T>
__device__ __forceinline__ T pow_m0145(T x);
template <>
__device__ __forceinline__ double pow_m0145<double>(double x) {
  return pow(x, -0.145);
}
template <>
__device__ __forceinline__ float pow_m0145<float>(float x) {
  return __powf(x, -0.145f);
}

// Wilke mixture viscosity, modified-Wilke conductivity and constant-Schmidt
// rho*D_k.  cp[k] is the species cp per unit mass at temp.
template <typename T, int NS>
__device__ __forceinline__ void transport(const ChemParams &C, T temp, const T *Y, T mw_total, const T *cp,
                                          T &mu_out, T &lam_out, T *rhod) {
  const SpecTables<T> &S = tab<T>(C);
  constexpr int A = SpecCount<NS>::kArr;
  const int ns = SpecCount<NS>::n(C);
  T X[A], vis[A], svis[A], isvis[A];
  const T sqt = fsqrt(temp);
#pragma unroll
  for (int l = 0; l < A; ++l) {
    if (l < ns) {
      X[l] = Y[l] * mw_total * S.inv_mw[l];
      const T t_dl = temp * S.lj_inv[l];
      const T tp = t_dl + T(0.5);
      const T omega = T(1.147) * pow_m0145<T>(t_dl) + frcp(tp * tp);
      vis[l] = fdiv(S.vis_coeff[l] * sqt, omega);
      svis[l] = fsqrt(vis[l]);
      isvis[l] = frcp(svis[l]);
    }
  }
  T viscosity = 0, conductivity = 0;
#pragma unroll
  for (int m = 0; m < A; ++m) {
    if (m < ns) {
      T vt = 0;
#pragma unroll
      for (int n = 0; n < A; ++n) {
        if (n < ns) {
          T phi;
          if (m == n) {
            phi = T(1);
          } else {
            const T num = T(1) + svis[m] * isvis[n] * S.wj[m * kMaxSpec + n];
            phi = num * num * S.sw[m * kMaxSpec + n];
          }
          vt += phi * X[n];
        }
      }
      const T lam_m = vis[m] * (cp[m] + S.lam_shift[m]);
      viscosity += fdiv(vis[m] * X[m], vt);
      conductivity += fdiv(lam_m * X[m], T(1.065) * vt - T(0.065) * X[m]);
    }
  }
  mu_out = viscosity;
  lam_out = conductivity;
  const T inv_sc = T(1) / T(C.Sc);
#pragma unroll
  for (int l = 0; l < A; ++l) {
    if (l < ns) {
      const T d = X[l] - T(1);
      rhod[l] = (fabs(d) < T(1e-3)) ? viscosity * inv_sc : fdiv((T(1) - Y[l]) * viscosity, (T(1) - X[l]) * T(C.Sc));
    }
  }
}

// Point properties used by the stage update and the time step:
// mu, lambda, rho*D_k (stored) and gamma, acoustic speed (for dt).
template <typename T, int NS>
__device__ __forceinline__ void point_props(const ChemParams &C, const T *rec, T temp, const T *Y, T &mu, T &lam,
                                            T *rhod, T &gamma, T &c) {
  constexpr int A = SpecCount<NS>::kArr;
  const int ns = SpecCount<NS>::n(C);
  if (NS == 0 || (NS < 0 && ns == 0)) {
    const T c_temp = T(kGammaAir * kRu / kMwAir);
    c = sqrt(c_temp * temp);
    mu = sutherland<T>(temp);
    lam = mu * c_temp / T(kGammaAir - 1) / T(C.Pr);
    gamma = T(kGammaAir);
    return;
  }
  const SpecTables<T> &S = tab<T>(C);
  T cp[A];
  T mwi = 0, cp_tot = 0, cvv = 0;
#pragma unroll
  for (int l = 0; l < A; ++l) {
    if (l < ns) {
      cp[l] = nasa_cp<T>(S, rec, l, temp);
      mwi += Y[l] * S.inv_mw[l];
      cp_tot += Y[l] * cp[l];
      cvv += Y[l] * (cp[l] - S.cv_shift[l]);
    }
  }
  const T mw = frcp(mwi);
  gamma = fdiv(cp_tot, cvv);
  c = fsqrt(gamma * T(kRu) * temp * mwi);
  transport<T, NS>(C, temp, Y, mw, cp, mu, lam, rhod);
}

// Temperature from internal energy by Newton iteration (tolerance 1e-3 on
// |1 - T1/T|, at most C.newton_max_iter iterations (1000 by default, as the
// reference), warm start t), in the precision W:
// FP64 for the plain and mixed paths, FP32 for the full-FP32 study.
template <typename W, int NS>
__device__ __forceinline__ W newton_temperature_w(const ChemParams &C, const W *rec, W e, const W *Y, W gas_const,
                                                  W t, bool &capped) {
  const SpecTables<W> &S = tab<W>(C);
  constexpr int A = SpecCount<NS>::kArr;
  const int ns = SpecCount<NS>::n(C);
  W err = 1;
  int iter = 0;
  while (err > W(1e-3) && iter++ < C.newton_max_iter) {
    W cp_tot = 0, h = 0;
#pragma unroll
    for (int l = 0; l < A; ++l) {
      if (l < ns) {
        W hl, cpl;
        nasa_h_cp<W>(S, rec, l, t, hl, cpl);
        cp_tot += cpl * Y[l];
        h += hl * Y[l];
      }
    }
    const W e_t = h - gas_const * t;
    const W cvv = cp_tot - gas_const;
    const W t1 = t - (e_t - e) / cvv;
    err = fabs(W(1) - t1 / t);
    t = t1;
  }
  capped = err > W(1e-3);
  return t;
}

template <int NS>
__device__ __forceinline__ double newton_temperature(const ChemParams &C, const double *rec, double e, const double *Y,
                                                     double gas_const, double t, bool &capped) {
  return newton_temperature_w<double, NS>(C, rec, e, Y, gas_const, t, capped);
}

template <typename T>
__device__ __forceinline__ T sgn1(T a) {
  return T((T(0) < a) - (a < T(0)));
}

// 0.5 (sgn a + sgn b) min(|a|, |b|), written as a sign test
template <typename T>
__device__ __forceinline__ T minmod(T a, T b) {
  const T m = fmin(fabs(a), fabs(b));
  return (a > T(0) && b > T(0)) ? m : ((a < T(0) && b < T(0)) ? -m : T(0));
}

// AUSM+ pressure splitting P+(M) = (M+1)^2 (2-M)/4 + a M (M^2-1)^2 and
// P-(M) = (M-1)^2 (2+M)/4 - a M (M^2-1)^2 for |M| <= 1, 1 / 0 beyond, with
// P+(M) + P-(M) = 1.  Returns P+(ml) + P-(mr) - 1 without the cancellation of
// forming the sum: in the subsonic case it is P+(ml) - P+(mr) = (ml - mr) x
// the divided difference of P+(M) = 1/2 + 3M/4 - M^3/4 + a (M^5 - 2M^3 + M).
template <typename T>
__device__ __forceinline__ T ausm_pressure_defect(T ml, T mr, T a) {
  auto p_plus = [&](T m) {
    const T q = m * m - T(1);
    return (m + T(1)) * (m + T(1)) * (T(2) - m) * T(0.25) + a * m * q * q;
  };
  auto p_minus = [&](T m) {
    const T q = m * m - T(1);
    return (m - T(1)) * (m - T(1)) * (T(2) + m) * T(0.25) - a * m * q * q;
  };
  const bool sl = !(fabs(ml) > T(1)), sr = !(fabs(mr) > T(1));
  if (sl && sr) {
    const T x2 = ml * ml, y2 = mr * mr, xy = ml * mr;
    const T s2 = x2 + xy + y2;
    const T s4 = x2 * x2 + x2 * xy + xy * xy + xy * y2 + y2 * y2;
    return (ml - mr) * (T(0.75) - T(0.25) * s2 + a * (s4 - T(2) * s2 + T(1)));
  }
  if (!sl) {                                        // P+(ml) is 1 or 0
    if (ml > T(0)) return sr ? p_minus(mr) : (mr < T(0) ? T(1) : T(0));
    return sr ? -p_plus(mr) : (mr < T(0) ? T(0) : T(-1));
  }
  return mr < T(0) ? p_plus(ml) : -p_minus(ml);     // P-(mr) is 1 or 0
}

// MUSCL (kappa = 1/3, minmod) or first-order states at the face between
// points 1 and 2 of v[0..3], face thermodynamics, then AUSM+.
// v[t][0..4] = rho,u,v,w,p ; v[t][5+l] = Y_l.  F receives n_var values.
template <typename T, int NS>
__device__ __forceinline__ void face_inviscid(const ChemParams &C, const T *rec, const T (&v)[4][5 + SpecCount<NS>::kArr],
                                              const T k[3], T *F) {
  constexpr int A = SpecCount<NS>::kArr;
  constexpr int NV = 5 + A;
  const int ns = SpecCount<NS>::n(C);
  const int nv = 5 + ns;
  T L[NV], R[NV];
  if (C.reconstruction == 2) {
    const T kappa = T(1.0 / 3.0);
    const T w1 = T(0.25) * (T(1) - kappa), w2 = T(0.25) * (T(1) + kappa);
#pragma unroll
    for (int l = 0; l < NV; ++l) {
      if (l < nv) {
        const T d_i = v[1][l] - v[0][l];
        const T d_i1 = v[2][l] - v[1][l];
        const T d_i2 = v[3][l] - v[2][l];
        const T m1 = minmod(d_i, d_i1);
        const T m2 = minmod(d_i1, d_i2);
        // minmod is symmetric: (1-k) mm(a,b) + (1+k) mm(b,a) = 2 mm(a,b)
        L[l] = v[1][l] + (w1 * m1 + w2 * m1);
        R[l] = v[2][l] - (w1 * m2 + w2 * m2);
      }
    }
  } else {
#pragma unroll
    for (int l = 0; l < NV; ++l)
      if (l < nv) L[l] = v[1][l], R[l] = v[2][l];
  }
  // L[4], R[4] hold the gauge pressure p - p_ref (p_ref = 0 in FP64)
  const T pref = T(C.p_ref);
  const T pl = L[4] + pref, pr = R[4] + pref;
  T el = T(0.5) * (L[1] * L[1] + L[2] * L[2] + L[3] * L[3]);
  T er = T(0.5) * (R[1] * R[1] + R[2] * R[2] + R[3] * R[3]);
  T El, Er, gam_l, gam_r;
  if (NS == 0 || (NS < 0 && ns == 0)) {
    El = el * L[0] + pl / T(kGammaAir - 1);
    Er = er * R[0] + pr / T(kGammaAir - 1);
    gam_l = gam_r = T(kGammaAir);
  } else {
    const SpecTables<T> &S = tab<T>(C);
    T mwl = 0, mwr = 0;
#pragma unroll
    for (int l = 0; l < A; ++l)
      if (l < ns) mwl += L[5 + l] * S.inv_mw[l], mwr += R[5 + l] * S.inv_mw[l];
    const T t_l = fdiv(pl, L[0] * T(kRu) * mwl);
    const T t_r = fdiv(pr, R[0] * T(kRu) * mwr);
    T cpl = 0, cpr = 0, cvl = 0, cvr = 0;
#pragma unroll
    for (int l = 0; l < A; ++l) {
      if (l < ns) {
        T hl, cl, hr, cr;
        nasa_h_cp<T>(S, rec, l, t_l, hl, cl);
        nasa_h_cp<T>(S, rec, l, t_r, hr, cr);
        cpl += cl * L[5 + l];
        cpr += cr * R[5 + l];
        cvl += L[5 + l] * (cl - S.cv_shift[l]);
        cvr += R[5 + l] * (cr - S.cv_shift[l]);
        el += hl * L[5 + l];
        er += hr * R[5 + l];
      }
    }
    El = L[0] * el - pl;
    Er = R[0] * er - pr;
    gam_l = fdiv(cpl, cvl);
    gam_r = fdiv(cpr, cvr);
  }
  const T alpha = T(3.0 / 16.0);
  const T k1 = k[0], k2 = k[1], k3 = k[2];
  const T gk = fsqrt(k1 * k1 + k2 * k2 + k3 * k3);
  const T igk = frcp(gk);
  const T ul = (k1 * L[1] + k2 * L[2] + k3 * L[3]) * igk;
  const T ur = (k1 * R[1] + k2 * R[2] + k3 * R[3]) * igk;
  const T rho_l = L[0], rho_r = R[0];
  const T c = T(0.5) * (fsqrt(fdiv(gam_l * pl, rho_l)) + fsqrt(fdiv(gam_r * pr, rho_r)));
  const T ic = frcp(c);
  const T mach_l = ul * ic, mach_r = ur * ic;
  T mlp, mrn, plp, prn;
  if (fabs(mach_l) > T(1)) {
    mlp = T(0.5) * (mach_l + fabs(mach_l));
    plp = fdiv(mlp, mach_l);
  } else {
    const T a = (mach_l + T(1)) * (mach_l + T(1)) * T(0.25);
    const T b = (mach_l * mach_l - T(1)) * (mach_l * mach_l - T(1));
    mlp = a + T(0.125) * b;
    plp = a * (T(2) - mach_l) + alpha * mach_l * b;
  }
  if (fabs(mach_r) > T(1)) {
    mrn = T(0.5) * (mach_r - fabs(mach_r));
    prn = fdiv(mrn, mach_r);
  } else {
    const T a = (mach_r - T(1)) * (mach_r - T(1)) * T(0.25);
    const T b = (mach_r * mach_r - T(1)) * (mach_r * mach_r - T(1));
    mrn = -a - T(0.125) * b;
    prn = a * (T(2) + mach_r) - alpha * mach_r * b;
  }
  // pressure term of the momentum flux, less p_ref k: plp p'_l + prn p'_r
  // + p_ref (plp + prn - 1), the last factor evaluated without cancellation
  T p_coeff;
  if (C.p_ref == 0.0) {
    p_coeff = plp * pl + prn * pr;
  } else {
    p_coeff = plp * L[4] + prn * R[4] + pref * ausm_pressure_defect(mach_l, mach_r, alpha);
  }
  // interface Mach number M+(ml) + M-(mr); at low Mach both terms are near
  // +-3/8 and their FP32 sum loses ~5 bits, so the FP32 path uses the
  // cancellation-free form (the FP64 path keeps the reference's sum)
  T m_half = mlp + mrn;
  if (sizeof(T) == 4 && !(fabs(mach_l) > T(1)) && !(fabs(mach_r) > T(1))) {
    // M+(M) + M-(M) = M: M+(ml) + M-(mr) = mr + (ml - mr) [1/2 + (ml + mr)(1/4 + (ml^2 + mr^2 - 2)/8)]
    m_half = mach_r + (mach_l - mach_r) *
                          (T(0.5) + (mach_l + mach_r) * (T(0.25) + T(0.125) * (mach_l * mach_l + mach_r * mach_r - T(2))));
  }
  const T mach_pos = T(0.5) * (m_half + fabs(m_half));
  const T mach_neg = T(0.5) * (m_half - fabs(m_half));
  const T mass_flux_half = c * (rho_l * mach_pos + rho_r * mach_neg);
  const T coeff = mass_flux_half * gk;
  const bool up = mass_flux_half >= T(0);
  F[0] = coeff;
  F[1] = coeff * (up ? L[1] : R[1]) + p_coeff * k1;
  F[2] = coeff * (up ? L[2] : R[2]) + p_coeff * k2;
  F[3] = coeff * (up ? L[3] : R[3]) + p_coeff * k3;
  F[4] = up ? fdiv(coeff * (El + pl), rho_l) : fdiv(coeff * (Er + pr), rho_r);
#pragma unroll
  for (int l = 0; l < A; ++l)
    if (l < ns) F[5 + l] = coeff * (up ? L[5 + l] : R[5 + l]);
}

}  // namespace ccb
