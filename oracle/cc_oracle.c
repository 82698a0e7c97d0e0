/*
 * cc_oracle.c -- CPU FP64 restatement of CombustionCodeGPU's per-timestep
 * residual path.  TEST INFRASTRUCTURE ONLY (what the tests compare the CUDA
 * results against, and the timed CPU baseline); the CUDA product never links
 * or calls it.
 *
 * Each routine names the reference file:line it follows.  The arithmetic is
 * written in the reference's evaluation order so that the restatement agrees
 * with the reference's FP64 kernels to rounding.  Three reference defects are
 * restated in their intended form (the same three are patched in the
 * reference build of oracle/ref_harness, see its build script):
 *   - Transport.cu:88 tests X[i] (grid index) -> X[l];
 *   - ViscousScheme.cu:317 averages rho_D(i,j+1,k) on zeta faces -> (i,j,k+1);
 *   - ViscousScheme.cu:17-24/240-246 average m+m instead of m+m1 (inert on
 *     uniform grids) -> m+m1.
 * Field.cu:216 / Driver.cu:204 (inner-face exchange launch) are restated as
 * intended: every point of the face range is visited once.
 */
#include "cc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define R_U 8314.462618   /* Constants.h:19 */
#define GAMMA_AIR 1.4     /* Constants.h:23 */
#define MW_AIR 28.9647    /* Constants.h:28 */
#define MAXS 32
#define MAXV (5 + MAXS)

typedef struct {
  int mx, my, mz, g, nx, ny, nz;
  size_t ng, n;
  double *jac, *metric;                 /* [ng], [9][ng] */
  double *cv, *bv, *yk;                 /* [nv][ng], [6][ng], [ns][ng] */
  double *vel, *acoustic, *mul, *cond, *gamma, *rho_d, *mach;
  double *dq, *dt_local, *bv_last, *qn; /* interior: [nv][n], [n], [4][n], [nv][n] */
  double *lu_rad, *lu_diag, *lu_psi;    /* LU-SGS, interior: r_d [3][n], 1/D [n], psi [ns][n] (on first use) */
  oc_boundary *bnd;
  int n_bnd, cap_bnd;
  oc_inner_face *inf;
  int n_inf, cap_inf;
} oblk;

struct oc_solver {
  oc_params p;
  double *tab;  /* owned copies of the species tables */
  int ns, nv;
  int nb;
  oblk *b;
  oc_bc bcs[64];
  int n_bc;
  double last_dt;
  double res[4];
  long n_grid_total;
  int newton_fail;
};

#define ID(B, i, j, k) \
  ((size_t)((i) + (B)->g) + (size_t)(B)->nx * ((size_t)((j) + (B)->g) + (size_t)(B)->ny * (size_t)((k) + (B)->g)))
#define IN(B, i, j, k) ((size_t)(i) + (size_t)(B)->mx * ((size_t)(j) + (size_t)(B)->my * (size_t)(k)))

int oc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

/* ------------------------------------------------------------------ thermo */

/* Thermo.cu:7-25 compute_enthalpy */
static void th_enthalpy(const oc_solver *s, double t, double *h) {
  const oc_params *P = &s->p;
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
  for (int i = 0; i < s->ns; ++i) {
    if (t < P->t_low[i]) {
      const double tt = P->t_low[i];
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt5 = tt4 * tt;
      const double *c = P->low_coeff + 7 * i;
      h[i] = c[0] * tt + 0.5 * c[1] * tt2 + c[2] * tt3 / 3 + 0.25 * c[3] * tt4 + 0.2 * c[4] * tt5 + c[5];
      const double cp = c[0] + c[1] * tt + c[2] * tt2 + c[3] * tt3 + c[4] * tt4;
      h[i] += cp * (t - tt);
    } else {
      const double *c = (t < P->t_mid[i] ? P->low_coeff : P->high_coeff) + 7 * i;
      h[i] = c[0] * t + 0.5 * c[1] * t2 + c[2] * t3 / 3 + 0.25 * c[3] * t4 + 0.2 * c[4] * t5 + c[5];
    }
    h[i] *= R_U / P->mw[i];
  }
}

/* Thermo.cu:27-47 compute_enthalpy_and_cp */
static void th_enthalpy_cp(const oc_solver *s, double t, double *h, double *cp) {
  const oc_params *P = &s->p;
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
  for (int i = 0; i < s->ns; ++i) {
    if (t < P->t_low[i]) {
      const double tt = P->t_low[i];
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt5 = tt4 * tt;
      const double *c = P->low_coeff + 7 * i;
      h[i] = c[0] * tt + 0.5 * c[1] * tt2 + c[2] * tt3 / 3 + 0.25 * c[3] * tt4 + 0.2 * c[4] * tt5 + c[5];
      cp[i] = c[0] + c[1] * tt + c[2] * tt2 + c[3] * tt3 + c[4] * tt4;
      h[i] += cp[i] * (t - tt);
    } else {
      const double *c = (t < P->t_mid[i] ? P->low_coeff : P->high_coeff) + 7 * i;
      h[i] = c[0] * t + 0.5 * c[1] * t2 + c[2] * t3 / 3 + 0.25 * c[3] * t4 + 0.2 * c[4] * t5 + c[5];
      cp[i] = c[0] + c[1] * t + c[2] * t2 + c[3] * t3 + c[4] * t4;
    }
    h[i] *= R_U / P->mw[i];
    cp[i] *= R_U / P->mw[i];
  }
}

/* Thermo.cu:49-63 compute_cp */
static void th_cp(const oc_solver *s, double t, double *cp) {
  const oc_params *P = &s->p;
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t;
  for (int i = 0; i < s->ns; ++i) {
    if (t < P->t_low[i]) {
      const double tt = P->t_low[i];
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt;
      const double *c = P->low_coeff + 7 * i;
      cp[i] = c[0] + c[1] * tt + c[2] * tt2 + c[3] * tt3 + c[4] * tt4;
    } else {
      const double *c = (t < P->t_mid[i] ? P->low_coeff : P->high_coeff) + 7 * i;
      cp[i] = c[0] + c[1] * t + c[2] * t2 + c[3] * t3 + c[4] * t4;
    }
    cp[i] *= R_U / P->mw[i];
  }
}

/* Thermo.cu:66-86 compute_total_energy at one point */
static void th_total_energy(const oc_solver *s, oblk *B, size_t q) {
  const size_t ng = B->ng;
  const double u = B->bv[1 * ng + q], v = B->bv[2 * ng + q], w = B->bv[3 * ng + q];
  double vel = u * u + v * v + w * w;
  B->vel[q] = vel;
  double e = 0.5 * B->bv[q] * vel;
  if (s->ns > 0) {
    double h[MAXS];
    th_enthalpy(s, B->bv[5 * ng + q], h);
    for (int l = 0; l < s->ns; l++) e += h[l] * B->cv[(5 + l) * ng + q];
    e -= B->bv[4 * ng + q];
  } else {
    e += B->bv[4 * ng + q] / (GAMMA_AIR - 1);
  }
  B->cv[4 * ng + q] = e;
  B->vel[q] = sqrt(vel);
}

/* Transport.cu:7-10 Sutherland */
static double sutherland(double t) { return 1.716e-5 * pow(t / 273, 1.5) * (273 + 111) / (t + 111); }

/* Transport.cu:43-96 compute_transport_property (X[l] in the Schmidt branch) */
static void tr_props(const oc_solver *s, double T, const double *Y, double mw_total, const double *cp, double *mu_out,
                     double *lam_out, double *rhod_out) {
  const oc_params *P = &s->p;
  const int ns = s->ns;
  double X[MAXS], vis[MAXS], lam[MAXS];
  for (int l = 0; l < ns; ++l) {
    X[l] = Y[l] * mw_total / P->mw[l];
    const double t_dl = T * P->LJ_potent_inv[l];
    const double omega = 1.147 * pow(t_dl, -0.145) + pow(t_dl + 0.5, -2);
    vis[l] = P->vis_coeff[l] * sqrt(T) / omega;
  }
  for (int l = 0; l < ns; ++l) lam[l] = vis[l] * (cp[l] + 1.25 * R_U / P->mw[l]);
  double viscosity = 0, conductivity = 0;
  for (int m = 0; m < ns; ++m) {
    double vis_temp = 0;
    for (int n = 0; n < ns; ++n) {
      double phi;
      if (m == n) {
        phi = 1.0;
      } else {
        const double num = 1 + sqrt(vis[m] / vis[n]) * P->WjDivWi_to_One4th[m * ns + n];
        phi = num * num * P->sqrt_WiDivWjPl1Mul8[m * ns + n];
      }
      vis_temp += phi * X[n];
    }
    const double cond_temp = 1.065 * vis_temp - 0.065 * X[m];
    viscosity += vis[m] * X[m] / vis_temp;
    conductivity += lam[m] * X[m] / cond_temp;
  }
  *mu_out = viscosity;
  *lam_out = conductivity;
  const double sc = P->Sc;
  for (int l = 0; l < ns; ++l) {
    if (fabs(X[l] - 1) < 1e-3)
      rhod_out[l] = viscosity / sc;
    else
      rhod_out[l] = (1 - Y[l]) * viscosity / ((1 - X[l]) * sc);
  }
}

/* Field.cu:178-210 update_physical_properties at one point */
static void props_point(const oc_solver *s, oblk *B, size_t q) {
  const size_t ng = B->ng;
  const double T = B->bv[5 * ng + q];
  if (s->ns > 0) {
    const int ns = s->ns;
    double Y[MAXS], cp[MAXS], rd[MAXS];
    double mw = 0, cp_tot = 0, cvv = 0;
    th_cp(s, T, cp);
    for (int l = 0; l < ns; ++l) {
      Y[l] = B->yk[l * ng + q];
      mw += Y[l] / s->p.mw[l];
      cp_tot += Y[l] * cp[l];
      cvv += Y[l] * (cp[l] - R_U / s->p.mw[l]);
    }
    mw = 1 / mw;
    B->gamma[q] = cp_tot / cvv;
    B->acoustic[q] = sqrt(B->gamma[q] * R_U * T / mw);
    double mu, lam;
    tr_props(s, T, Y, mw, cp, &mu, &lam, rd);
    B->mul[q] = mu;
    B->cond[q] = lam;
    for (int l = 0; l < ns; ++l) B->rho_d[l * ng + q] = rd[l];
  } else {
    const double c_temp = GAMMA_AIR * R_U / MW_AIR;
    B->acoustic[q] = sqrt(c_temp * T);
    B->mul[q] = sutherland(T);
    B->cond[q] = B->mul[q] * c_temp / (GAMMA_AIR - 1) / s->p.Pr;
    B->gamma[q] = GAMMA_AIR;
  }
  B->mach[q] = B->vel[q] / B->acoustic[q];
}

static void props_all(oc_solver *s) {
  for (int bi = 0; bi < s->nb; ++bi) {
    oblk *B = &s->b[bi];
#pragma omp parallel for schedule(static)
    for (long q = 0; q < (long)B->ng; ++q) props_point(s, B, (size_t)q);
  }
}

/* Field.cu:150-176 compute_cv_from_bv over every point, ghosts included */
static void cv_from_bv_all(oc_solver *s) {
  for (int bi = 0; bi < s->nb; ++bi) {
    oblk *B = &s->b[bi];
    const size_t ng = B->ng;
#pragma omp parallel for schedule(static)
    for (long qq = 0; qq < (long)ng; ++qq) {
      const size_t q = (size_t)qq;
      const double rho = B->bv[q];
      B->cv[q] = rho;
      B->cv[1 * ng + q] = rho * B->bv[1 * ng + q];
      B->cv[2 * ng + q] = rho * B->bv[2 * ng + q];
      B->cv[3 * ng + q] = rho * B->bv[3 * ng + q];
      for (int l = 0; l < s->ns; ++l) B->cv[(5 + l) * ng + q] = rho * B->yk[l * ng + q];
      th_total_energy(s, B, q);
    }
  }
}

/* Thermo.cu:89-125 compute_temperature (Newton on e(T)); returns 1 when the
 * iteration cap was reached without meeting the tolerance. */
static int th_temperature(const oc_solver *s, oblk *B, size_t q) {
  const size_t ng = B->ng;
  const int ns = s->ns;
  double mw = 0;
  for (int l = 0; l < ns; ++l) mw += B->yk[l * ng + q] / s->p.mw[l];
  mw = 1 / mw;
  const double gas_const = R_U / mw;
  const double u = B->bv[1 * ng + q], v = B->bv[2 * ng + q], w = B->bv[3 * ng + q];
  const double e = B->cv[4 * ng + q] / B->cv[q] - 0.5 * (u * u + v * v + w * w);
  double err = 1, t = B->bv[5 * ng + q];
  const int max_iter = 1000;
  const double eps = 1e-3;
  int iter = 0;
  double h_i[MAXS], cp_i[MAXS];
  while (err > eps && iter++ < max_iter) {
    th_enthalpy_cp(s, t, h_i, cp_i);
    double cp_tot = 0, h = 0;
    for (int l = 0; l < ns; ++l) {
      cp_tot += cp_i[l] * B->yk[l * ng + q];
      h += h_i[l] * B->yk[l * ng + q];
    }
    const double e_t = h - gas_const * t;
    const double cvv = cp_tot - gas_const;
    const double t1 = t - (e_t - e) / cvv;
    err = fabs(1 - t1 / t);
    t = t1;
  }
  B->bv[5 * ng + q] = t;
  B->bv[4 * ng + q] = B->bv[q] * B->bv[5 * ng + q] * gas_const;
  return err > eps;
}

/* TimeAdvanceFunc.cu:262-289 (update_cv_and_bv after the cv increment):
 * primitives from cv, Newton for T (multispecies) or the perfect-gas closure. */
static int bv_from_cv(const oc_solver *s, oblk *B, size_t q, int renorm_y) {
  const size_t ng = B->ng;
  B->bv[q] = B->cv[q];
  const double density_inv = 1.0 / B->cv[q];
  B->bv[1 * ng + q] = B->cv[1 * ng + q] * density_inv;
  B->bv[2 * ng + q] = B->cv[2 * ng + q] * density_inv;
  B->bv[3 * ng + q] = B->cv[3 * ng + q] * density_inv;
  const double u = B->bv[1 * ng + q], v = B->bv[2 * ng + q], w = B->bv[3 * ng + q];
  double velocity = u * u + v * v + w * w;
  int fail = 0;
  if (s->ns > 0) {
    for (int l = 0; l < s->ns; ++l) B->yk[l * ng + q] = B->cv[(5 + l) * ng + q] * density_inv;
    if (renorm_y) {
      double sum = 0;
      for (int l = 0; l < s->ns; ++l) sum += B->yk[l * ng + q];
      const double inv = 1.0 / sum;
      for (int l = 0; l < s->ns; ++l) B->yk[l * ng + q] *= inv;
    }
    fail = th_temperature(s, B, q);
  } else {
    B->bv[4 * ng + q] = (GAMMA_AIR - 1) * (B->cv[4 * ng + q] - 0.5 * B->bv[q] * velocity);
    B->bv[5 * ng + q] = B->bv[4 * ng + q] * MW_AIR * density_inv / R_U;
  }
  B->vel[q] = sqrt(velocity);
  return fail;
}

/* ------------------------------------------------------------- inviscid */

static double sgn(double a) { return (double)((0.0 < a) - (a < 0.0)); }
/* Limiter.cuh:13-16 minmod */
static double minmod(double a, double b) { return 0.5 * (sgn(a) + sgn(b)) * fmin(fabs(a), fabs(b)); }

/* Reconstruction.cu:26-89 (MUSCL / first order + face thermo) and
 * InviscidScheme.cu:24-108 (AUSM+).  pv[0..3] are points i-1,i,i+1,i+2 with
 * n_var primitives (rho,u,v,w,p,Y_k); the face lies between i and i+1. */
static void face_inviscid(const oc_solver *s, const double *pv[4], const double ml[3], double jl, const double mr[3],
                          double jr, double *fc) {
  const int nv = s->nv, ns = s->ns;
  double L[MAXV + 2], R[MAXV + 2];
  if (s->p.reconstruction == 2) {
    const double kappa = 1.0 / 3.0;
    for (int l = 0; l < nv; ++l) {
      const double d_i = pv[1][l] - pv[0][l];
      const double d_i1 = pv[2][l] - pv[1][l];
      const double d_i2 = pv[3][l] - pv[2][l];
      const double dnl = minmod(d_i, d_i1);
      const double dpl = minmod(d_i1, d_i);
      const double dnr = minmod(d_i1, d_i2);
      const double dpr = minmod(d_i2, d_i1);
      L[l] = pv[1][l] + 0.25 * ((1 - kappa) * dnl + (1 + kappa) * dpl);
      R[l] = pv[2][l] - 0.25 * ((1 - kappa) * dpr + (1 + kappa) * dnr);
    }
  } else {
    for (int l = 0; l < nv; ++l) {
      L[l] = pv[1][l];
      R[l] = pv[2][l];
    }
  }
  double el = 0.5 * (L[1] * L[1] + L[2] * L[2] + L[3] * L[3]);
  double er = 0.5 * (R[1] * R[1] + R[2] * R[2] + R[3] * R[3]);
  double gam_l = GAMMA_AIR, gam_r = GAMMA_AIR;
  if (ns > 0) {
    const double *mw = s->p.mw;
    double mwl = 0, mwr = 0;
    for (int l = 0; l < ns; ++l) {
      mwl += L[5 + l] / mw[l];
      mwr += R[5 + l] / mw[l];
    }
    const double t_l = L[4] / (L[0] * R_U * mwl);
    const double t_r = R[4] / (R[0] * R_U * mwr);
    double hl[MAXS], hr[MAXS], cpl_i[MAXS], cpr_i[MAXS];
    th_enthalpy_cp(s, t_l, hl, cpl_i);
    th_enthalpy_cp(s, t_r, hr, cpr_i);
    double cpl = 0, cpr = 0, cvl = 0, cvr = 0;
    for (int l = 0; l < ns; ++l) {
      cpl += cpl_i[l] * L[l + 5];
      cpr += cpr_i[l] * R[l + 5];
      cvl += L[l + 5] * (cpl_i[l] - R_U / mw[l]);
      cvr += R[l + 5] * (cpr_i[l] - R_U / mw[l]);
      el += hl[l] * L[l + 5];
      er += hr[l] * R[l + 5];
    }
    L[5 + ns] = L[0] * el - L[4];
    R[5 + ns] = R[0] * er - R[4];
    gam_l = cpl / cvl;
    gam_r = cpr / cvr;
  } else {
    L[5] = el * L[0] + L[4] / (GAMMA_AIR - 1);
    R[5] = er * R[0] + R[4] / (GAMMA_AIR - 1);
  }
  const double alpha = 3 / 16.0;
  const double k1 = 0.5 * (jl * ml[0] + jr * mr[0]);
  const double k2 = 0.5 * (jl * ml[1] + jr * mr[1]);
  const double k3 = 0.5 * (jl * ml[2] + jr * mr[2]);
  const double grad_k_div_jac = sqrt(k1 * k1 + k2 * k2 + k3 * k3);
  const double ul = (k1 * L[1] + k2 * L[2] + k3 * L[3]) / grad_k_div_jac;
  const double ur = (k1 * R[1] + k2 * R[2] + k3 * R[3]) / grad_k_div_jac;
  const double pl = L[4], pr = R[4], rho_l = L[0], rho_r = R[0];
  const double c = 0.5 * (sqrt(gam_l * pl / rho_l) + sqrt(gam_r * pr / rho_r));
  const double mach_l = ul / c, mach_r = ur / c;
  double mlp, mrn, plp, prn;
  if (fabs(mach_l) > 1) {
    mlp = 0.5 * (mach_l + fabs(mach_l));
    plp = mlp / mach_l;
  } else {
    const double a = (mach_l + 1) * (mach_l + 1) * 0.25;
    const double b = (mach_l * mach_l - 1) * (mach_l * mach_l - 1);
    mlp = a + 0.125 * b;
    plp = a * (2 - mach_l) + alpha * mach_l * b;
  }
  if (fabs(mach_r) > 1) {
    mrn = 0.5 * (mach_r - fabs(mach_r));
    prn = mrn / mach_r;
  } else {
    const double a = (mach_r - 1) * (mach_r - 1) * 0.25;
    const double b = (mach_r * mach_r - 1) * (mach_r * mach_r - 1);
    mrn = -a - 0.125 * b;
    prn = a * (2 + mach_r) - alpha * mach_r * b;
  }
  const double p_coeff = plp * pl + prn * pr;
  const double m_half = mlp + mrn;
  const double mach_pos = 0.5 * (m_half + fabs(m_half));
  const double mach_neg = 0.5 * (m_half - fabs(m_half));
  const double mass_flux_half = c * (rho_l * mach_pos + rho_r * mach_neg);
  const double coeff = mass_flux_half * grad_k_div_jac;
  const double *S = mass_flux_half >= 0 ? L : R;
  fc[0] = coeff;
  fc[1] = coeff * S[1] + p_coeff * k1;
  fc[2] = coeff * S[2] + p_coeff * k2;
  fc[3] = coeff * S[3] + p_coeff * k3;
  fc[4] = coeff * (S[5 + ns] + S[4]) / S[0];
  for (int l = 5; l < nv; ++l) fc[l] = coeff * S[l];
}

/* gather the n_var reconstruction primitives of a point */
static void load_pv(const oc_solver *s, const oblk *B, size_t q, double *pv) {
  const size_t ng = B->ng;
  for (int l = 0; l < 5; ++l) pv[l] = B->bv[l * ng + q];
  for (int l = 0; l < s->ns; ++l) pv[5 + l] = B->yk[l * ng + q];
}

/* TimeAdvanceFunc.cu:38-154: inviscid flux along direction d for every line,
 * dq -= F(i+1/2) - F(i-1/2) at interior points. */
static void inviscid_dir(const oc_solver *s, oblk *B, int d) {
  const int m[3] = {B->mx, B->my, B->mz};
  const int o1 = (d + 1) % 3, o2 = (d + 2) % 3;
  const int nv = s->nv;
  const size_t ng = B->ng;
#pragma omp parallel for collapse(2) schedule(static)
  for (int b2 = 0; b2 < m[o2]; ++b2) {
    for (int b1 = 0; b1 < m[o1]; ++b1) {
      double *F = (double *)malloc(sizeof(double) * (size_t)nv * (size_t)(m[d] + 1));
      double pvs[4][MAXV];
      for (int f = -1; f < m[d]; ++f) { /* face between f and f+1 */
        const double *pp[4];
        for (int t = 0; t < 4; ++t) {
          int c[3];
          c[d] = f - 1 + t;
          c[o1] = b1;
          c[o2] = b2;
          load_pv(s, B, ID(B, c[0], c[1], c[2]), pvs[t]);
          pp[t] = pvs[t];
        }
        int cl[3], cr[3];
        cl[d] = f, cr[d] = f + 1;
        cl[o1] = cr[o1] = b1;
        cl[o2] = cr[o2] = b2;
        const size_t ql = ID(B, cl[0], cl[1], cl[2]), qr = ID(B, cr[0], cr[1], cr[2]);
        double ml[3], mr[3];
        for (int c = 0; c < 3; ++c) {
          ml[c] = B->metric[(size_t)(3 * d + c) * ng + ql];
          mr[c] = B->metric[(size_t)(3 * d + c) * ng + qr];
        }
        face_inviscid(s, pp, ml, B->jac[ql], mr, B->jac[qr], &F[(size_t)(f + 1) * nv]);
      }
      for (int p = 0; p < m[d]; ++p) {
        int c[3];
        c[d] = p, c[o1] = b1, c[o2] = b2;
        const size_t qi = IN(B, c[0], c[1], c[2]);
        for (int l = 0; l < nv; ++l)
          B->dq[(size_t)l * B->n + qi] -= F[(size_t)(p + 1) * nv + l] - F[(size_t)p * nv + l];
      }
      free(F);
    }
  }
}

/* -------------------------------------------------------------- viscous */

/* ViscousScheme.cu:11-342 (compute_fv/gv/hv) for the face between point
 * (i,j,k) and its neighbour along d. */
static void face_viscous(const oc_solver *s, const oblk *B, int d, int i, int j, int k, double *fv) {
  const size_t ng = B->ng;
  const int ns = s->ns;
  int e[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  const size_t p0 = ID(B, i, j, k);
  const size_t p1 = ID(B, i + e[d][0], j + e[d][1], k + e[d][2]);
  double met[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c)
      met[r][c] = 0.5 * (B->metric[(size_t)(3 * r + c) * ng + p0] + B->metric[(size_t)(3 * r + c) * ng + p1]);
  /* computational-space derivatives of a field f (component offset base) */
#define DERIV(arr, out)                                                                            \
  do {                                                                                             \
    for (int cdir = 0; cdir < 3; ++cdir) {                                                         \
      if (cdir == d) {                                                                             \
        out[cdir] = (arr)[p1] - (arr)[p0];                                                         \
      } else {                                                                                     \
        const int *ec = e[cdir];                                                                   \
        const size_t a0 = ID(B, i + ec[0], j + ec[1], k + ec[2]);                                  \
        const size_t b0 = ID(B, i - ec[0], j - ec[1], k - ec[2]);                                  \
        const size_t a1 = ID(B, i + e[d][0] + ec[0], j + e[d][1] + ec[1], k + e[d][2] + ec[2]);    \
        const size_t b1 = ID(B, i + e[d][0] - ec[0], j + e[d][1] - ec[1], k + e[d][2] - ec[2]);    \
        out[cdir] = 0.25 * ((arr)[a0] - (arr)[b0] + (arr)[a1] - (arr)[b1]);                        \
      }                                                                                            \
    }                                                                                              \
  } while (0)
  double du[3], dv[3], dw[3], dt[3];
  DERIV(B->bv + 1 * ng, du);
  DERIV(B->bv + 2 * ng, dv);
  DERIV(B->bv + 3 * ng, dw);
  DERIV(B->bv + 5 * ng, dt);
  const double xi_x = met[0][0], xi_y = met[0][1], xi_z = met[0][2];
  const double eta_x = met[1][0], eta_y = met[1][1], eta_z = met[1][2];
  const double zeta_x = met[2][0], zeta_y = met[2][1], zeta_z = met[2][2];
  const double u_x = du[0] * xi_x + du[1] * eta_x + du[2] * zeta_x;
  const double u_y = du[0] * xi_y + du[1] * eta_y + du[2] * zeta_y;
  const double u_z = du[0] * xi_z + du[1] * eta_z + du[2] * zeta_z;
  const double v_x = dv[0] * xi_x + dv[1] * eta_x + dv[2] * zeta_x;
  const double v_y = dv[0] * xi_y + dv[1] * eta_y + dv[2] * zeta_y;
  const double v_z = dv[0] * xi_z + dv[1] * eta_z + dv[2] * zeta_z;
  const double w_x = dw[0] * xi_x + dw[1] * eta_x + dw[2] * zeta_x;
  const double w_y = dw[0] * xi_y + dw[1] * eta_y + dw[2] * zeta_y;
  const double w_z = dw[0] * xi_z + dw[1] * eta_z + dw[2] * zeta_z;
  const double viscosity = 0.5 * (B->mul[p0] + B->mul[p1]);
  const double tau_xx = viscosity * (4 * u_x - 2 * v_y - 2 * w_z) / 3.0;
  const double tau_yy = viscosity * (4 * v_y - 2 * u_x - 2 * w_z) / 3.0;
  const double tau_zz = viscosity * (4 * w_z - 2 * u_x - 2 * v_y) / 3.0;
  const double tau_xy = viscosity * (u_y + v_x);
  const double tau_xz = viscosity * (u_z + w_x);
  const double tau_yz = viscosity * (v_z + w_y);
  const double kx = 0.5 * (B->metric[(size_t)(3 * d + 0) * ng + p0] * B->jac[p0] +
                           B->metric[(size_t)(3 * d + 0) * ng + p1] * B->jac[p1]);
  const double ky = 0.5 * (B->metric[(size_t)(3 * d + 1) * ng + p0] * B->jac[p0] +
                           B->metric[(size_t)(3 * d + 1) * ng + p1] * B->jac[p1]);
  const double kz = 0.5 * (B->metric[(size_t)(3 * d + 2) * ng + p0] * B->jac[p0] +
                           B->metric[(size_t)(3 * d + 2) * ng + p1] * B->jac[p1]);
  fv[0] = 0;
  fv[1] = kx * tau_xx + ky * tau_xy + kz * tau_xz;
  fv[2] = kx * tau_xy + ky * tau_yy + kz * tau_yz;
  fv[3] = kx * tau_xz + ky * tau_yz + kz * tau_zz;
  const double um = 0.5 * (B->bv[1 * ng + p0] + B->bv[1 * ng + p1]);
  const double vm = 0.5 * (B->bv[2 * ng + p0] + B->bv[2 * ng + p1]);
  const double wm = 0.5 * (B->bv[3 * ng + p0] + B->bv[3 * ng + p1]);
  const double t_x = dt[0] * xi_x + dt[1] * eta_x + dt[2] * zeta_x;
  const double t_y = dt[0] * xi_y + dt[1] * eta_y + dt[2] * zeta_y;
  const double t_z = dt[0] * xi_z + dt[1] * eta_z + dt[2] * zeta_z;
  const double conductivity = 0.5 * (B->cond[p0] + B->cond[p1]);
  fv[4] = um * fv[1] + vm * fv[2] + wm * fv[3] + conductivity * (kx * t_x + ky * t_y + kz * t_z);
  if (ns > 0) {
    double h[MAXS], D[MAXS], yx[MAXS], yy[MAXS], yz[MAXS];
    const double tm = 0.5 * (B->bv[5 * ng + p0] + B->bv[5 * ng + p1]);
    th_enthalpy(s, tm, h);
    double rho_uc = 0, rho_vc = 0, rho_wc = 0;
    for (int l = 0; l < ns; ++l) {
      D[l] = 0.5 * (B->rho_d[(size_t)l * ng + p0] + B->rho_d[(size_t)l * ng + p1]);
      double dy[3];
      DERIV(B->yk + (size_t)l * ng, dy);
      yx[l] = dy[0] * xi_x + dy[1] * eta_x + dy[2] * zeta_x;
      yy[l] = dy[0] * xi_y + dy[1] * eta_y + dy[2] * zeta_y;
      yz[l] = dy[0] * xi_z + dy[1] * eta_z + dy[2] * zeta_z;
      const double DMulH = D[l] * h[l];
      fv[4] += kx * DMulH * yx[l];
      fv[4] += ky * DMulH * yy[l];
      fv[4] += kz * DMulH * yz[l];
      rho_uc += D[l] * yx[l];
      rho_vc += D[l] * yy[l];
      rho_wc += D[l] * yz[l];
    }
    for (int l = 0; l < ns; ++l) {
      fv[5 + l] = D[l] * (kx * yx[l] + ky * yy[l] + kz * yz[l]) -
                  0.5 * (B->yk[(size_t)l * ng + p0] + B->yk[(size_t)l * ng + p1]) *
                      (kx * rho_uc + ky * rho_vc + kz * rho_wc);
    }
  }
#undef DERIV
}

/* TimeAdvanceFunc.cu:156-243: dq += Fv(i+1/2) - Fv(i-1/2) along d */
static void viscous_dir(const oc_solver *s, oblk *B, int d) {
  const int m[3] = {B->mx, B->my, B->mz};
  const int o1 = (d + 1) % 3, o2 = (d + 2) % 3;
  const int nv = s->nv;
#pragma omp parallel for collapse(2) schedule(static)
  for (int b2 = 0; b2 < m[o2]; ++b2) {
    for (int b1 = 0; b1 < m[o1]; ++b1) {
      double *F = (double *)malloc(sizeof(double) * (size_t)nv * (size_t)(m[d] + 1));
      for (int f = -1; f < m[d]; ++f) {
        int c[3];
        c[d] = f, c[o1] = b1, c[o2] = b2;
        face_viscous(s, B, d, c[0], c[1], c[2], &F[(size_t)(f + 1) * nv]);
      }
      for (int p = 0; p < m[d]; ++p) {
        int c[3];
        c[d] = p, c[o1] = b1, c[o2] = b2;
        const size_t qi = IN(B, c[0], c[1], c[2]);
        for (int l = 0; l < nv; ++l) B->dq[(size_t)l * B->n + qi] += F[(size_t)(p + 1) * nv + l] - F[(size_t)p * nv + l];
      }
      free(F);
    }
  }
}

/* set_dq_to_0 + compute_inviscid_flux + compute_viscous_flux (Driver.cu:145-153) */
static void compute_dq_block(oc_solver *s, oblk *B) {
  memset(B->dq, 0, sizeof(double) * (size_t)s->nv * B->n);
  const int dim = B->mz == 1 ? 2 : 3;
  for (int d = 0; d < dim; ++d) inviscid_dir(s, B, d);
  if (s->p.viscous_order == 2)
    for (int d = 0; d < dim; ++d) viscous_dir(s, B, d);
}

/* TemporalScheme.cu:11-43 local time step at every interior point */
static void local_dt_block(const oc_solver *s, oblk *B) {
  const size_t ng = B->ng;
  const int dim = B->mz == 1 ? 2 : 3;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < B->mz; ++k)
    for (int j = 0; j < B->my; ++j)
      for (int i = 0; i < B->mx; ++i) {
        const size_t q = ID(B, i, j, k);
        double m[3][3];
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) m[r][c] = B->metric[(size_t)(3 * r + c) * ng + q];
        const double grad_xi = sqrt(m[0][0] * m[0][0] + m[0][1] * m[0][1] + m[0][2] * m[0][2]);
        const double grad_eta = sqrt(m[1][0] * m[1][0] + m[1][1] * m[1][1] + m[1][2] * m[1][2]);
        const double grad_zeta = sqrt(m[2][0] * m[2][0] + m[2][1] * m[2][1] + m[2][2] * m[2][2]);
        const double u = B->bv[1 * ng + q], v = B->bv[2 * ng + q], w = B->bv[3 * ng + q];
        const double U = u * m[0][0] + v * m[0][1] + w * m[0][2];
        const double V = u * m[1][0] + v * m[1][1] + w * m[1][2];
        const double W = u * m[2][0] + v * m[2][1] + w * m[2][2];
        const double c = B->acoustic[q];
        double sr_inv = fabs(U) + fabs(V) + c * (grad_xi + grad_eta);
        if (dim == 3) sr_inv += fabs(W) + c * grad_zeta;
        const double coeff_1 = fmax(s->ns > 0 ? B->gamma[q] : GAMMA_AIR, 4.0 / 3.0);
        const double coeff_2 = B->mul[q] / B->bv[q] / s->p.Pr;
        double sr_vis = grad_xi * grad_xi + grad_eta * grad_eta;
        if (dim == 3) sr_vis += grad_zeta * grad_zeta;
        sr_vis *= coeff_1 * coeff_2;
        B->dt_local[IN(B, i, j, k)] = s->p.cfl / (sr_inv + sr_vis);
      }
}

/* --------------------------------------------------------- boundaries */

/* BoundCond.cu:455-487 apply_outflow */
static void bc_outflow(const oc_solver *s, oblk *B, const oc_boundary *f) {
  int dir[3] = {0, 0, 0};
  dir[f->face] = f->direction;
  const size_t ng = B->ng;
  for (int k = f->range_start[2]; k <= f->range_end[2]; ++k)
    for (int j = f->range_start[1]; j <= f->range_end[1]; ++j)
      for (int i = f->range_start[0]; i <= f->range_end[0]; ++i) {
        const size_t q = ID(B, i, j, k);
        for (int g = 1; g <= B->g; ++g) {
          const size_t gq = ID(B, i + g * dir[0], j + g * dir[1], k + g * dir[2]);
          for (int l = 0; l < 6; ++l) B->bv[l * ng + gq] = B->bv[l * ng + q];
          for (int l = 0; l < s->nv; ++l) B->cv[l * ng + gq] = B->cv[l * ng + q];
          for (int l = 0; l < s->ns; ++l) B->yk[l * ng + gq] = B->yk[l * ng + q];
        }
      }
}

/* BoundCond.cu:489-527 apply_inflow */
static void bc_inflow(const oc_solver *s, oblk *B, const oc_boundary *f, const oc_bc *bc) {
  int dir[3] = {0, 0, 0};
  dir[f->face] = f->direction;
  const size_t ng = B->ng;
  for (int k = f->range_start[2]; k <= f->range_end[2]; ++k)
    for (int j = f->range_start[1]; j <= f->range_end[1]; ++j)
      for (int i = f->range_start[0]; i <= f->range_end[0]; ++i) {
        for (int g = 1; g <= B->g; ++g) {
          const size_t gq = ID(B, i + g * dir[0], j + g * dir[1], k + g * dir[2]);
          const double density = bc->density;
          B->bv[gq] = density;
          B->bv[1 * ng + gq] = bc->u;
          B->bv[2 * ng + gq] = bc->v;
          B->bv[3 * ng + gq] = bc->w;
          B->bv[4 * ng + gq] = bc->pressure;
          B->bv[5 * ng + gq] = bc->temperature;
          for (int l = 0; l < s->ns; ++l) {
            B->yk[l * ng + gq] = bc->yk[l];
            B->cv[(5 + l) * ng + gq] = density * bc->yk[l];
          }
          B->cv[gq] = density;
          B->cv[1 * ng + gq] = density * bc->u;
          B->cv[2 * ng + gq] = density * bc->v;
          B->cv[3 * ng + gq] = density * bc->w;
          th_total_energy(s, B, gq);
        }
      }
}

/* BoundCond.cu:529-629 apply_wall */
static void bc_wall(const oc_solver *s, oblk *B, const oc_boundary *f, const oc_bc *bc) {
  int dir[3] = {0, 0, 0};
  dir[f->face] = f->direction;
  const size_t ng = B->ng;
  const int ns = s->ns;
  for (int k = f->range_start[2]; k <= f->range_end[2]; ++k)
    for (int j = f->range_start[1]; j <= f->range_end[1]; ++j)
      for (int i = f->range_start[0]; i <= f->range_end[0]; ++i) {
        double t_wall = bc->t_wall;
        const size_t q = ID(B, i, j, k);
        const size_t qi = ID(B, i - dir[0], j - dir[1], k - dir[2]);
        if (bc->thermal_type == 1) t_wall = B->bv[5 * ng + qi];
        const double p = B->bv[4 * ng + qi];
        double mw;
        if (ns > 0) {
          mw = 0;
          for (int l = 0; l < ns; ++l) {
            B->yk[l * ng + q] = B->yk[l * ng + qi];
            mw += B->yk[l * ng + q] / s->p.mw[l];
          }
          mw = 1 / mw;
        } else {
          mw = MW_AIR;
        }
        B->bv[q] = p * mw / (t_wall * R_U);
        B->bv[1 * ng + q] = 0;
        B->bv[2 * ng + q] = 0;
        B->bv[3 * ng + q] = 0;
        B->bv[4 * ng + q] = p;
        B->bv[5 * ng + q] = t_wall;
        B->cv[q] = B->bv[q];
        B->cv[1 * ng + q] = 0;
        B->cv[2 * ng + q] = 0;
        B->cv[3 * ng + q] = 0;
        for (int l = 0; l < ns; ++l) B->cv[(l + 5) * ng + q] = B->yk[l * ng + q] * B->bv[q];
        th_total_energy(s, B, q);
        for (int g = 1; g <= B->g; ++g) {
          const size_t qin = ID(B, i - g * dir[0], j - g * dir[1], k - g * dir[2]);
          const size_t qgh = ID(B, i + g * dir[0], j + g * dir[1], k + g * dir[2]);
          if (ns > 0) {
            mw = 0;
            for (int l = 0; l < ns; ++l) {
              B->yk[l * ng + qgh] = B->yk[l * ng + qin];
              mw += B->yk[l * ng + qgh] / s->p.mw[l];
            }
            mw = 1 / mw;
          }
          const double u_i = B->bv[1 * ng + qin], v_i = B->bv[2 * ng + qin], w_i = B->bv[3 * ng + qin];
          const double p_i = B->bv[4 * ng + qin], t_i = B->bv[5 * ng + qin];
          double t_g = t_i;
          if (bc->thermal_type == 0) {
            t_g = 2 * t_wall - t_i;
            if (t_g <= 0.1 * t_wall) t_g = t_wall;
          }
          const double rho_g = p_i * mw / (t_g * R_U);
          B->bv[qgh] = rho_g;
          B->bv[1 * ng + qgh] = -u_i;
          B->bv[2 * ng + qgh] = -v_i;
          B->bv[3 * ng + qgh] = -w_i;
          B->bv[4 * ng + qgh] = p_i;
          B->bv[5 * ng + qgh] = t_g;
          B->cv[qgh] = rho_g;
          B->cv[1 * ng + qgh] = -rho_g * u_i;
          B->cv[2 * ng + qgh] = -rho_g * v_i;
          B->cv[3 * ng + qgh] = -rho_g * w_i;
          for (int l = 0; l < ns; ++l) B->cv[(l + 5) * ng + qgh] = B->yk[l * ng + qgh] * rho_g;
          th_total_energy(s, B, qgh);
        }
      }
}

/* Field.cu:213-266 inner_communication for one face of block bi (the
 * Driver.cu:204 host-pointer argument and the Field.cu:216 index typo are
 * restated as intended). */
static void inner_comm(oc_solver *s, int bi, const oc_inner_face *f) {
  oblk *Z = &s->b[bi];
  oblk *T = &s->b[f->target_block];
  const size_t ngz = Z->ng, ngt = T->ng;
  int np[3];
  for (int d = 0; d < 3; ++d) np[d] = abs(f->range_start[d] - f->range_end[d]) + 1;
  const int face_dir = f->direction > 0 ? f->range_start[f->face] : f->range_end[f->face];
  for (int n2 = 0; n2 < np[2]; ++n2)
    for (int n1 = 0; n1 < np[1]; ++n1)
      for (int n0 = 0; n0 < np[0]; ++n0) {
        const int n[3] = {n0, n1, n2};
        int idx[3], it[3];
        for (int d = 0; d < 3; ++d) {
          const int d_idx = f->loop_dir[d] * n[d];
          idx[d] = f->range_start[d] + d_idx;
          it[d] = f->target_start[d] + f->target_loop_dir[d] * d_idx;
        }
        const size_t q = ID(Z, idx[0], idx[1], idx[2]);
        const size_t qt = ID(T, it[0], it[1], it[2]);
        if (idx[f->face] == face_dir) {
          for (int l = 0; l < 6; ++l) {
            const double ave = 0.5 * (T->bv[l * ngt + qt] + Z->bv[l * ngz + q]);
            Z->bv[l * ngz + q] = ave;
            T->bv[l * ngt + qt] = ave;
          }
          for (int l = 0; l < s->nv; ++l) {
            const double ave = 0.5 * (T->cv[l * ngt + qt] + Z->cv[l * ngz + q]);
            Z->cv[l * ngz + q] = ave;
            T->cv[l * ngt + qt] = ave;
          }
          for (int l = 0; l < s->ns; ++l) {
            const double ave = 0.5 * (T->yk[l * ngt + qt] + Z->yk[l * ngz + q]);
            Z->yk[l * ngz + q] = ave;
            T->yk[l * ngt + qt] = ave;
          }
        } else {
          for (int l = 0; l < 5; ++l) {
            Z->bv[l * ngz + q] = T->bv[l * ngt + qt];
            Z->cv[l * ngz + q] = T->cv[l * ngt + qt];
          }
          Z->bv[5 * ngz + q] = T->bv[5 * ngt + qt];
          for (int l = 0; l < s->ns; ++l) {
            Z->yk[l * ngz + q] = T->yk[l * ngt + qt];
            Z->cv[(l + 5) * ngz + q] = T->cv[(l + 5) * ngt + qt];
          }
        }
      }
}

/* BoundCond.cu:251-313 apply_boundary_conditions (outflow, inflow, wall; each
 * condition's faces in block order) followed by Driver.cu:194-217
 * data_communication. */
static void apply_bcs_and_exchange(oc_solver *s) {
  const int kinds[3] = {6, 5, 2};
  for (int kk = 0; kk < 3; ++kk)
    for (int c = 0; c < s->n_bc; ++c) {
      const oc_bc *bc = &s->bcs[c];
      if (bc->kind != kinds[kk]) continue;
      for (int bi = 0; bi < s->nb; ++bi) {
        oblk *B = &s->b[bi];
        for (int f = 0; f < B->n_bnd; ++f) {
          if (B->bnd[f].type_label != bc->label) continue;
          if (bc->kind == 6) bc_outflow(s, B, &B->bnd[f]);
          else if (bc->kind == 5) bc_inflow(s, B, &B->bnd[f], bc);
          else bc_wall(s, B, &B->bnd[f], bc);
        }
      }
    }
  for (int bi = 0; bi < s->nb; ++bi)
    for (int f = 0; f < s->b[bi].n_inf; ++f) inner_comm(s, bi, &s->b[bi].inf[f]);
}

/* ------------------------------------------------------------- setup */

oc_solver *oc_create(const oc_params *p, int n_block, const int *dims) {
  oc_solver *s = (oc_solver *)calloc(1, sizeof(oc_solver));
  s->p = *p;
  s->ns = p->n_spec;
  s->nv = 5 + p->n_spec;
  if (s->ns > MAXS) {
    free(s);
    return NULL;
  }
  const int ns = s->ns;
  if (ns > 0) {
    const size_t nt = (size_t)ns * (4 + 14 + 2) + 2 * (size_t)ns * ns;
    s->tab = (double *)malloc(sizeof(double) * nt);
    double *t = s->tab;
#define CP(dst, src, cnt) \
  memcpy(t, src, sizeof(double) * (cnt)); \
  s->p.dst = t;                           \
  t += (cnt);
    CP(mw, p->mw, ns);
    CP(t_low, p->t_low, ns);
    CP(t_mid, p->t_mid, ns);
    CP(t_high, p->t_high, ns);
    CP(low_coeff, p->low_coeff, 7 * ns);
    CP(high_coeff, p->high_coeff, 7 * ns);
    CP(LJ_potent_inv, p->LJ_potent_inv, ns);
    CP(vis_coeff, p->vis_coeff, ns);
    CP(WjDivWi_to_One4th, p->WjDivWi_to_One4th, ns * ns);
    CP(sqrt_WiDivWjPl1Mul8, p->sqrt_WiDivWjPl1Mul8, ns * ns);
#undef CP
  }
  s->nb = n_block;
  s->b = (oblk *)calloc((size_t)n_block, sizeof(oblk));
  s->n_grid_total = 0;
  for (int bi = 0; bi < n_block; ++bi) {
    oblk *B = &s->b[bi];
    B->mx = dims[3 * bi];
    B->my = dims[3 * bi + 1];
    B->mz = dims[3 * bi + 2];
    B->g = p->ngg;
    B->nx = B->mx + 2 * B->g;
    B->ny = B->my + 2 * B->g;
    B->nz = B->mz + 2 * B->g;
    B->ng = (size_t)B->nx * B->ny * B->nz;
    B->n = (size_t)B->mx * B->my * B->mz;
    s->n_grid_total += (long)B->n;
    const size_t ng = B->ng, n = B->n;
    B->jac = (double *)calloc(ng, sizeof(double));
    B->metric = (double *)calloc(9 * ng, sizeof(double));
    B->cv = (double *)calloc((size_t)s->nv * ng, sizeof(double));
    B->bv = (double *)calloc(6 * ng, sizeof(double));
    B->yk = (double *)calloc((size_t)(ns > 0 ? ns : 1) * ng, sizeof(double));
    B->vel = (double *)calloc(ng, sizeof(double));
    B->acoustic = (double *)calloc(ng, sizeof(double));
    B->mul = (double *)calloc(ng, sizeof(double));
    B->cond = (double *)calloc(ng, sizeof(double));
    B->gamma = (double *)calloc(ng, sizeof(double));
    B->mach = (double *)calloc(ng, sizeof(double));
    B->rho_d = (double *)calloc((size_t)(ns > 0 ? ns : 1) * ng, sizeof(double));
    B->dq = (double *)calloc((size_t)s->nv * n, sizeof(double));
    B->qn = (double *)calloc((size_t)s->nv * n, sizeof(double));
    B->dt_local = (double *)calloc(n, sizeof(double));
    B->bv_last = (double *)calloc(4 * n, sizeof(double));
  }
  return s;
}

void oc_destroy(oc_solver *s) {
  if (!s) return;
  for (int bi = 0; bi < s->nb; ++bi) {
    oblk *B = &s->b[bi];
    free(B->jac), free(B->metric), free(B->cv), free(B->bv), free(B->yk), free(B->vel), free(B->acoustic);
    free(B->mul), free(B->cond), free(B->gamma), free(B->mach), free(B->rho_d), free(B->dq), free(B->qn);
    free(B->dt_local), free(B->bv_last), free(B->bnd), free(B->inf), free(B->lu_rad), free(B->lu_diag), free(B->lu_psi);
  }
  free(s->b);
  free(s->tab);
  free(s);
}

/* Mesh.cpp:14-32 Boundary::register_boundary (3D) */
int oc_add_boundary_raw(oc_solver *s, int blk, const int raw[7]) {
  if (blk < 0 || blk >= s->nb) return -1;
  oblk *B = &s->b[blk];
  oc_boundary b;
  memset(&b, 0, sizeof b);
  b.range_start[0] = raw[0], b.range_end[0] = raw[1];
  b.range_start[1] = raw[2], b.range_end[1] = raw[3];
  b.range_start[2] = raw[4], b.range_end[2] = raw[5];
  b.type_label = raw[6];
  b.face = 0;
  b.direction = 1;
  const int dim = 3, ngg = B->g;
  for (int i = 0; i < dim; ++i) {
    if (b.range_start[i] == b.range_end[i]) {
      b.face = i;
      if (b.range_start[i] == 0) b.direction = -1;
      break;
    }
  }
  for (int i = 0; i < dim; ++i) {
    if (i == b.face) continue;
    if (b.range_end[i] < b.range_start[i]) {
      const int t = b.range_end[i];
      b.range_end[i] = b.range_start[i];
      b.range_start[i] = t;
    }
    b.range_start[i] -= ngg;
    b.range_end[i] += ngg;
  }
  if (B->n_bnd == B->cap_bnd) {
    B->cap_bnd = B->cap_bnd ? 2 * B->cap_bnd : 8;
    B->bnd = (oc_boundary *)realloc(B->bnd, sizeof(oc_boundary) * (size_t)B->cap_bnd);
  }
  B->bnd[B->n_bnd++] = b;
  return 0;
}

static int isgn(int a) { return (0 < a) - (a < 0); }

/* Mesh.cpp:35-143 InnerFace ctor + register_boundary (3D branch) */
int oc_add_inner_face_raw(oc_solver *s, int blk, const int raw[13]) {
  if (blk < 0 || blk >= s->nb) return -1;
  oblk *B = &s->b[blk];
  const int ngg = B->g, dim = 3;
  oc_inner_face f;
  memset(&f, 0, sizeof f);
  f.range_start[0] = raw[0], f.range_end[0] = raw[1];
  f.range_start[1] = raw[2], f.range_end[1] = raw[3];
  f.range_start[2] = raw[4], f.range_end[2] = raw[5];
  f.target_start[0] = raw[6], f.target_end[0] = raw[7];
  f.target_start[1] = raw[8], f.target_end[1] = raw[9];
  f.target_start[2] = raw[10], f.target_end[2] = raw[11];
  f.target_block = raw[12] - 1;
  f.face = 0, f.direction = 1, f.target_face = 0, f.target_direction = 1;
  for (int i = 0; i < 3; ++i) f.loop_dir[i] = f.target_loop_dir[i] = 1;
  for (int i = 0; i < dim; ++i) {
    if (f.range_start[i] == f.range_end[i]) {
      f.face = i;
      if (f.range_start[i] == 1) f.direction = -1;
      f.range_start[i] -= 1;
      f.range_end[i] -= 1;
      break;
    }
  }
  for (int i = 0; i < dim; ++i) {
    if (f.target_start[i] == f.target_end[i]) {
      f.target_face = i;
      if (f.target_start[i] == 1) f.target_direction = -1;
      f.target_start[i] -= 1;
      f.target_end[i] -= 1;
      break;
    }
  }
  f.src_tar[f.target_face] = -(f.direction * f.target_direction) * (f.face + 1);
  {
    int next_face = 0, target_next_face = 0;
    for (int i = 0; i < dim; ++i) {
      if (f.range_start[i] < 0) {
        next_face = i;
        f.range_start[i] = -f.range_start[i] - 1;
        f.range_end[i] = -f.range_end[i] - 1;
        break;
      }
    }
    for (int i = 0; i < dim; ++i) {
      if (f.target_start[i] < 0) {
        target_next_face = i;
        f.target_start[i] = -f.target_start[i] - 1;
        f.target_end[i] = -f.target_end[i] - 1;
        break;
      }
    }
    f.src_tar[target_next_face] = isgn((f.target_end[target_next_face] - f.target_start[target_next_face]) *
                                       (f.range_end[next_face] - f.range_start[next_face])) *
                                  (next_face + 1);
    next_face = 3 - f.face - next_face;
    target_next_face = 3 - f.target_face - target_next_face;
    f.range_start[next_face] -= 1;
    f.range_end[next_face] -= 1;
    f.target_start[target_next_face] -= 1;
    f.target_end[target_next_face] -= 1;
    f.src_tar[target_next_face] = isgn((f.target_end[target_next_face] - f.target_start[target_next_face]) *
                                       (f.range_end[next_face] - f.range_start[next_face])) *
                                  (next_face + 1);
  }
  const int rs = f.direction < 0 ? -ngg : f.range_end[f.face];
  const int re = f.direction < 0 ? 0 : f.range_end[f.face] + ngg;
  f.range_start[f.face] = rs;
  f.range_end[f.face] = re;
  const int sgn_tar = isgn(f.src_tar[f.target_face]);
  if (f.target_direction > 0) {
    if (sgn_tar > 0)
      f.target_start[f.target_face] = f.target_end[f.target_face] - ngg;
    else
      f.target_start[f.target_face] = f.target_end[f.target_face];
  } else {
    f.target_start[f.target_face] = (sgn_tar > 0) ? 0 : ngg;
  }
  for (int i = 0; i < dim; ++i) {
    f.loop_dir[i] = f.range_start[i] <= f.range_end[i] ? 1 : -1;
    f.target_loop_dir[i] = isgn(f.src_tar[i]);
    f.src_tar[i] = abs(f.src_tar[i]) - 1;
  }
  for (int i = 0; i < 3; ++i) {
    if (i != f.face) {
      f.range_start[i] -= f.loop_dir[i] * ngg;
      f.range_end[i] += f.loop_dir[i] * ngg;
      f.target_start[i] -= f.target_loop_dir[i] * f.loop_dir[i] * ngg;
      f.target_end[i] += f.target_loop_dir[i] * f.loop_dir[i] * ngg;
    }
  }
  if (B->n_inf == B->cap_inf) {
    B->cap_inf = B->cap_inf ? 2 * B->cap_inf : 8;
    B->inf = (oc_inner_face *)realloc(B->inf, sizeof(oc_inner_face) * (size_t)B->cap_inf);
  }
  B->inf[B->n_inf++] = f;
  return 0;
}

int oc_get_boundary(const oc_solver *s, int blk, int i, oc_boundary *out) {
  if (blk < 0 || blk >= s->nb || i < 0 || i >= s->b[blk].n_bnd) return -1;
  *out = s->b[blk].bnd[i];
  return 0;
}

int oc_get_inner_face(const oc_solver *s, int blk, int i, oc_inner_face *out) {
  if (blk < 0 || blk >= s->nb || i < 0 || i >= s->b[blk].n_inf) return -1;
  *out = s->b[blk].inf[i];
  return 0;
}

/* BoundCond.cu:218-230 link_bc_to_boundaries: wall faces do not cover the
 * tangential ghost layers.  Applied once, when the condition is registered. */
int oc_add_bc(oc_solver *s, const oc_bc *bc) {
  if (s->n_bc >= 64) return -1;
  s->bcs[s->n_bc++] = *bc;
  if (bc->kind == 2) {
    for (int bi = 0; bi < s->nb; ++bi) {
      oblk *B = &s->b[bi];
      for (int f = 0; f < B->n_bnd; ++f) {
        oc_boundary *b = &B->bnd[f];
        if (b->type_label != bc->label) continue;
        for (int q = 0; q < 3; ++q) {
          if (q == b->face) continue;
          b->range_start[q] += B->g;
          b->range_end[q] -= B->g;
        }
      }
    }
  }
  return 0;
}

int oc_set_geometry(oc_solver *s, int blk, const double *jac, const double *metric) {
  if (blk < 0 || blk >= s->nb) return -1;
  oblk *B = &s->b[blk];
  memcpy(B->jac, jac, sizeof(double) * B->ng);
  memcpy(B->metric, metric, sizeof(double) * 9 * B->ng);
  return 0;
}

int oc_set_state(oc_solver *s, int blk, const double *bv, const double *yk) {
  if (blk < 0 || blk >= s->nb) return -1;
  oblk *B = &s->b[blk];
  memcpy(B->bv, bv, sizeof(double) * 6 * B->ng);
  if (s->ns > 0) memcpy(B->yk, yk, sizeof(double) * (size_t)s->ns * B->ng);
  return 0;
}

/* Driver.cu:59-97 initialize_computation */
int oc_init(oc_solver *s) {
  cv_from_bv_all(s);
  apply_bcs_and_exchange(s);
  props_all(s);
  s->newton_fail = 0;
  return 0;
}

/* TimeAdvanceFunc.cu:13-24 store_last_step */
static void store_last(oc_solver *s) {
  for (int bi = 0; bi < s->nb; ++bi) {
    oblk *B = &s->b[bi];
    const size_t ng = B->ng, n = B->n;
    for (int k = 0; k < B->mz; ++k)
      for (int j = 0; j < B->my; ++j)
        for (int i = 0; i < B->mx; ++i) {
          const size_t q = ID(B, i, j, k), qi = IN(B, i, j, k);
          B->bv_last[qi] = B->bv[q];
          B->bv_last[n + qi] = B->vel[q];
          B->bv_last[2 * n + qi] = B->bv[4 * ng + q];
          B->bv_last[3 * n + qi] = B->bv[5 * ng + q];
        }
  }
}

/* TimeAdvanceFunc.cu:292-303 + Driver.cu:219-277 (sum of squares, sqrt(e/N)) */
static void residual(oc_solver *s) {
  double r[4] = {0, 0, 0, 0};
  for (int bi = 0; bi < s->nb; ++bi) {
    oblk *B = &s->b[bi];
    const size_t ng = B->ng, n = B->n;
    for (int k = 0; k < B->mz; ++k)
      for (int j = 0; j < B->my; ++j)
        for (int i = 0; i < B->mx; ++i) {
          const size_t q = ID(B, i, j, k), qi = IN(B, i, j, k);
          const double a = B->bv[q] - B->bv_last[qi];
          const double b = B->vel[q] - B->bv_last[n + qi];
          const double c = B->bv[4 * ng + q] - B->bv_last[2 * n + qi];
          const double d = B->bv[5 * ng + q] - B->bv_last[3 * n + qi];
          r[0] += a * a, r[1] += b * b, r[2] += c * c, r[3] += d * d;
        }
  }
  for (int l = 0; l < 4; ++l) s->res[l] = sqrt(r[l] / (double)s->n_grid_total);
}

/* cv += dq * dt/J (TimeAdvanceFunc.cu:262-265); the RK combination
 * cv = a*qn + b*cv when a != 0; then primitives. */
static void update_block(oc_solver *s, oblk *B, const double *dt_point, double dt_global, double a, double b,
                         int renorm_y) {
  const size_t ng = B->ng, n = B->n;
  const int nv = s->nv;
  int fails = 0;
#pragma omp parallel for collapse(2) schedule(static) reduction(+ : fails)
  for (int k = 0; k < B->mz; ++k)
    for (int j = 0; j < B->my; ++j)
      for (int i = 0; i < B->mx; ++i) {
        const size_t q = ID(B, i, j, k), qi = IN(B, i, j, k);
        const double dt = dt_point ? dt_point[qi] : dt_global;
        const double dt_div_jac = dt / B->jac[q];
        for (int l = 0; l < nv; ++l) B->cv[l * ng + q] += B->dq[l * n + qi] * dt_div_jac;
        if (B->mz == 1) B->cv[3 * ng + q] = 0;
        if (a != 0.0)
          for (int l = 0; l < nv; ++l) B->cv[l * ng + q] = a * B->qn[l * n + qi] + b * B->cv[l * ng + q];
        fails += bv_from_cv(s, B, q, renorm_y);
      }
  s->newton_fail += fails;
}

int oc_steady_step(oc_solver *s, int renorm_y) {
  store_last(s);
  for (int bi = 0; bi < s->nb; ++bi) {
    oblk *B = &s->b[bi];
    compute_dq_block(s, B);
    local_dt_block(s, B);
    update_block(s, B, B->dt_local, 0, 0, 1, renorm_y);
  }
  apply_bcs_and_exchange(s);
  props_all(s);
  residual(s);
  return 0;
}

/* ------------------------------------------------------------- LU-SGS
 * Scalar LU-SGS steady step (Yoon & Jameson, AIAA J. 26(9):1025-1026, 1988),
 * the implicit scheme the reference declares (TemporalScheme.cuh:19-21,
 * Driver.cu:318-321) and allocates spectral-radius arrays for (Field.h:60-61,
 * Field.cu:138-141) but gives no body.  Per interior point and direction d:
 *   r_d = J (|u . grad xi_d| + c |grad xi_d| + 2 max(gamma,4/3) mu/(rho Pr) |grad xi_d|^2)
 *         (the viscous term in viscous runs only),
 *   D   = J / dt_local + sum_d r_d,
 *   A+-_d dQ = (A_d dQ +- r_d dQ) / 2, A_d the Jacobian of J grad xi_d . F
 *         of the thermally perfect mixture:
 *         dp = (gamma-1)(dE - u.dm + |u|^2/2 drho) + sum_k psi_k d(rho Y_k),
 *         psi_k = gamma R_k T - (gamma-1) h_k(T) (no sum for the air model);
 * lower sweep (lexicographic)  dQ*(p) = (dq(p) + sum_d A+_d(p-e_d) dQ*(p-e_d)) (1/D),
 * upper sweep (reversed)       dQ(p) = dQ*(p) - (sum_d A-_d(p+e_d) dQ(p+e_d)) (1/D),
 * neighbours outside the block contribute nothing; then cv += dQ. */
static void lusgs_jac_vec(int nv, const double *Q, double p, double gam, const double *psi, const double k[3],
                          const double *dQ, double *dF) {
  const double inv = 1.0 / Q[0];
  const double u = Q[1] * inv, v = Q[2] * inv, w = Q[3] * inv;
  const double U = k[0] * u + k[1] * v + k[2] * w;
  const double dm = k[0] * dQ[1] + k[1] * dQ[2] + k[2] * dQ[3];
  const double dU = (dm - U * dQ[0]) * inv;
  double dp = (gam - 1.0) * (dQ[4] - (u * dQ[1] + v * dQ[2] + w * dQ[3]) + 0.5 * (u * u + v * v + w * w) * dQ[0]);
  for (int l = 5; l < nv; ++l) dp += psi[l - 5] * dQ[l];
  dF[0] = dm;
  dF[1] = dQ[1] * U + Q[1] * dU + k[0] * dp;
  dF[2] = dQ[2] * U + Q[2] * dU + k[1] * dp;
  dF[3] = dQ[3] * U + Q[3] * dU + k[2] * dp;
  dF[4] = (dQ[4] + dp) * U + (Q[4] + p) * dU;
  for (int l = 5; l < nv; ++l) dF[l] = dQ[l] * U + Q[l] * dU;
}

/* A+_d(q) X(q) / A-_d(q) X(q) of the neighbour (i,j,k) added into acc */
static void lusgs_neighbour(const oc_solver *s, const oblk *B, int i, int j, int k, int d, double sg, double *acc) {
  const int nv = s->nv;
  const size_t ng = B->ng, n = B->n, qg = ID(B, i, j, k), qn = IN(B, i, j, k);
  double X[MAXV], Q[MAXV], dF[MAXV], psi[MAXS];
  for (int l = 0; l < nv; ++l) X[l] = B->dq[(size_t)l * n + qn], Q[l] = B->cv[(size_t)l * ng + qg];
  for (int l = 0; l < s->ns; ++l) psi[l] = B->lu_psi[(size_t)l * n + qn];
  const double J = B->jac[qg];
  const double kv[3] = {J * B->metric[(size_t)(3 * d) * ng + qg], J * B->metric[(size_t)(3 * d + 1) * ng + qg],
                        J * B->metric[(size_t)(3 * d + 2) * ng + qg]};
  const double gam = s->ns > 0 ? B->gamma[qg] : GAMMA_AIR;
  lusgs_jac_vec(nv, Q, B->bv[4 * ng + qg], gam, psi, kv, X, dF);
  const double r = sg * B->lu_rad[(size_t)d * n + qn];
  for (int l = 0; l < nv; ++l) acc[l] += 0.5 * (dF[l] + r * X[l]);
}

/* B->dq (the right-hand side on entry) becomes dQ */
static void lusgs_block(const oc_solver *s, oblk *B) {
  const size_t ng = B->ng, n = B->n;
  const int nv = s->nv, dim = B->mz == 1 ? 2 : 3;
  if (!B->lu_rad)
    B->lu_rad = calloc(3 * n, sizeof(double)), B->lu_diag = calloc(n, sizeof(double)),
    B->lu_psi = calloc((size_t)(s->ns > 0 ? s->ns : 1) * n, sizeof(double));
  for (int k = 0; k < B->mz; ++k)
    for (int j = 0; j < B->my; ++j)
      for (int i = 0; i < B->mx; ++i) {
        const size_t q = ID(B, i, j, k), qi = IN(B, i, j, k);
        const double J = B->jac[q];
        const double u = B->bv[1 * ng + q], v = B->bv[2 * ng + q], w = B->bv[3 * ng + q];
        const double c = B->acoustic[q];
        const double gam = s->ns > 0 ? B->gamma[q] : GAMMA_AIR;
        const double c1 = fmax(gam, 4.0 / 3.0);
        const double c2 = B->mul[q] / B->bv[q] / s->p.Pr;
        double D = J / B->dt_local[qi];
        for (int d = 0; d < 3; ++d) {
          double r = 0;
          if (d < dim) {
            const double m0 = B->metric[(size_t)(3 * d) * ng + q], m1 = B->metric[(size_t)(3 * d + 1) * ng + q],
                         m2 = B->metric[(size_t)(3 * d + 2) * ng + q];
            const double g = sqrt(m0 * m0 + m1 * m1 + m2 * m2);
            const double U = u * m0 + v * m1 + w * m2;
            r = fabs(U) + c * g;
            if (s->p.viscous_order == 2) r += 2.0 * c1 * c2 * g * g;
            r *= J;
            D += r;
          }
          B->lu_rad[(size_t)d * n + qi] = r;
        }
        B->lu_diag[qi] = 1.0 / D;
        if (s->ns > 0) {
          double h[MAXS];
          const double t = B->bv[5 * ng + q];
          th_enthalpy(s, t, h);
          for (int l = 0; l < s->ns; ++l)
            B->lu_psi[(size_t)l * n + qi] = gam * (R_U / s->p.mw[l]) * t - (gam - 1.0) * h[l];
        }
      }
  double acc[MAXV];
  for (int k = 0; k < B->mz; ++k)
    for (int j = 0; j < B->my; ++j)
      for (int i = 0; i < B->mx; ++i) {
        const size_t qi = IN(B, i, j, k);
        for (int l = 0; l < nv; ++l) acc[l] = B->dq[(size_t)l * n + qi];
        if (i > 0) lusgs_neighbour(s, B, i - 1, j, k, 0, 1.0, acc);
        if (j > 0) lusgs_neighbour(s, B, i, j - 1, k, 1, 1.0, acc);
        if (dim == 3 && k > 0) lusgs_neighbour(s, B, i, j, k - 1, 2, 1.0, acc);
        const double rD = B->lu_diag[qi];
        for (int l = 0; l < nv; ++l) B->dq[(size_t)l * n + qi] = acc[l] * rD;
      }
  for (int k = B->mz - 1; k >= 0; --k)
    for (int j = B->my - 1; j >= 0; --j)
      for (int i = B->mx - 1; i >= 0; --i) {
        const size_t qi = IN(B, i, j, k);
        for (int l = 0; l < nv; ++l) acc[l] = 0.0;
        if (i + 1 < B->mx) lusgs_neighbour(s, B, i + 1, j, k, 0, -1.0, acc);
        if (j + 1 < B->my) lusgs_neighbour(s, B, i, j + 1, k, 1, -1.0, acc);
        if (dim == 3 && k + 1 < B->mz) lusgs_neighbour(s, B, i, j, k + 1, 2, -1.0, acc);
        const double rD = B->lu_diag[qi];
        for (int l = 0; l < nv; ++l) B->dq[(size_t)l * n + qi] = B->dq[(size_t)l * n + qi] - acc[l] * rD;
      }
}

/* cv += dQ, then the primitives (TimeAdvanceFunc.cu:266-289) */
static void lusgs_update_block(oc_solver *s, oblk *B, int renorm_y) {
  const size_t ng = B->ng, n = B->n;
  const int nv = s->nv;
  int fails = 0;
#pragma omp parallel for collapse(2) schedule(static) reduction(+ : fails)
  for (int k = 0; k < B->mz; ++k)
    for (int j = 0; j < B->my; ++j)
      for (int i = 0; i < B->mx; ++i) {
        const size_t q = ID(B, i, j, k), qi = IN(B, i, j, k);
        for (int l = 0; l < nv; ++l) B->cv[l * ng + q] += B->dq[l * n + qi];
        if (B->mz == 1) B->cv[3 * ng + q] = 0;
        fails += bv_from_cv(s, B, q, renorm_y);
      }
  s->newton_fail += fails;
}

int oc_lusgs_step(oc_solver *s, int renorm_y) {
  store_last(s);
  for (int bi = 0; bi < s->nb; ++bi) {
    oblk *B = &s->b[bi];
    compute_dq_block(s, B);
    local_dt_block(s, B);
    lusgs_block(s, B);
    lusgs_update_block(s, B, renorm_y);
  }
  apply_bcs_and_exchange(s);
  props_all(s);
  residual(s);
  return 0;
}

/* SSP-RK3 (Shu-Osher): U1 = U + dt L(U); U2 = 3/4 U + 1/4 (U1 + dt L(U1));
 * U^{n+1} = 1/3 U + 2/3 (U2 + dt L(U2)); every stage increment is the
 * reference update (TimeAdvanceFunc.cu:255-290) with a global dt. */
int oc_rk3_step(oc_solver *s, int renorm_y) {
  static const double A[3] = {0.0, 0.75, 1.0 / 3.0};
  static const double Bc[3] = {1.0, 0.25, 2.0 / 3.0};
  store_last(s);
  double dt = 1e300;
  for (int bi = 0; bi < s->nb; ++bi) {
    oblk *B = &s->b[bi];
    local_dt_block(s, B);
    for (size_t q = 0; q < B->n; ++q)
      if (B->dt_local[q] < dt) dt = B->dt_local[q];
    const size_t ng = B->ng, n = B->n;
    for (int l = 0; l < s->nv; ++l)
      for (int k = 0; k < B->mz; ++k)
        for (int j = 0; j < B->my; ++j)
          for (int i = 0; i < B->mx; ++i) B->qn[l * n + IN(B, i, j, k)] = B->cv[l * ng + ID(B, i, j, k)];
  }
  s->last_dt = dt;
  for (int st = 0; st < 3; ++st) {
    for (int bi = 0; bi < s->nb; ++bi) compute_dq_block(s, &s->b[bi]);
    for (int bi = 0; bi < s->nb; ++bi) update_block(s, &s->b[bi], NULL, dt, A[st], Bc[st], renorm_y);
    apply_bcs_and_exchange(s);
    props_all(s);
  }
  residual(s);
  return 0;
}

int oc_compute_dq(oc_solver *s, int blk, double *dq) {
  if (blk < 0 || blk >= s->nb) return -1;
  oblk *B = &s->b[blk];
  compute_dq_block(s, B);
  memcpy(dq, B->dq, sizeof(double) * (size_t)s->nv * B->n);
  return 0;
}

int oc_get_state(const oc_solver *s, int blk, double *bv, double *yk, double *cv) {
  if (blk < 0 || blk >= s->nb) return -1;
  const oblk *B = &s->b[blk];
  if (bv) memcpy(bv, B->bv, sizeof(double) * 6 * B->ng);
  if (yk && s->ns > 0) memcpy(yk, B->yk, sizeof(double) * (size_t)s->ns * B->ng);
  if (cv) memcpy(cv, B->cv, sizeof(double) * (size_t)s->nv * B->ng);
  return 0;
}

int oc_get_props(const oc_solver *s, int blk, double *mul, double *cond, double *rho_d, double *gamma,
                 double *acoustic) {
  if (blk < 0 || blk >= s->nb) return -1;
  const oblk *B = &s->b[blk];
  if (mul) memcpy(mul, B->mul, sizeof(double) * B->ng);
  if (cond) memcpy(cond, B->cond, sizeof(double) * B->ng);
  if (rho_d && s->ns > 0) memcpy(rho_d, B->rho_d, sizeof(double) * (size_t)s->ns * B->ng);
  if (gamma) memcpy(gamma, B->gamma, sizeof(double) * B->ng);
  if (acoustic) memcpy(acoustic, B->acoustic, sizeof(double) * B->ng);
  return 0;
}

int oc_get_dt_local(const oc_solver *s, int blk, double *dt) {
  if (blk < 0 || blk >= s->nb) return -1;
  memcpy(dt, s->b[blk].dt_local, sizeof(double) * s->b[blk].n);
  return 0;
}

double oc_last_dt(const oc_solver *s) { return s->last_dt; }

int oc_residual(const oc_solver *s, double out[4]) {
  for (int l = 0; l < 4; ++l) out[l] = s->res[l];
  return 0;
}

int oc_newton_failures(const oc_solver *s) { return s->newton_fail; }

/* ---------------------------------------------------- known-answer hooks */

static void kat_solver(oc_solver *t, const oc_params *p) {
  memset(t, 0, sizeof *t);
  t->p = *p;
  t->ns = p->n_spec;
  t->nv = 5 + p->n_spec;
}

double oc_kat_minmod(double a, double b) { return minmod(a, b); }

void oc_kat_face_inviscid(const oc_params *p, const double *pv4, const double ml[3], double jl, const double mr[3],
                          double jr, double *fc) {
  oc_solver t;
  kat_solver(&t, p);
  const double *pp[4] = {pv4, pv4 + t.nv, pv4 + 2 * t.nv, pv4 + 3 * t.nv};
  face_inviscid(&t, pp, ml, jl, mr, jr, fc);
}

void oc_kat_h_cp(const oc_params *p, double temp, double *h, double *cp) {
  oc_solver t;
  kat_solver(&t, p);
  th_enthalpy_cp(&t, temp, h, cp);
}

void oc_kat_transport(const oc_params *p, double temp, const double *Y, double *mu, double *lam, double *rhod) {
  oc_solver t;
  kat_solver(&t, p);
  double cp[MAXS], mwi = 0;
  th_cp(&t, temp, cp);
  for (int l = 0; l < t.ns; ++l) mwi += Y[l] / p->mw[l];
  tr_props(&t, temp, Y, 1 / mwi, cp, mu, lam, rhod);
}

/* Newton of Thermo.cu:89-125 on one point given conserved (rho, rho u, rho
 * v, rho w, rho E) and Y, warm start t0. */
void oc_kat_lusgs_jac_vec(int nv, const double *Q, double p, double gam, const double *psi, const double k[3],
                          const double *dQ, double *dF) {
  lusgs_jac_vec(nv, Q, p, gam, psi, k, dQ, dF);
}

double oc_kat_temperature(const oc_params *p, const double *q5, const double *Y, double t0) {
  oc_solver t;
  kat_solver(&t, p);
  oblk B;
  memset(&B, 0, sizeof B);
  double cv[5 + MAXS], bv[6], yk[MAXS];
  B.ng = 1;
  B.cv = cv, B.bv = bv, B.yk = yk;
  for (int l = 0; l < 5; ++l) cv[l] = q5[l];
  bv[0] = q5[0];
  bv[1] = q5[1] / q5[0], bv[2] = q5[2] / q5[0], bv[3] = q5[3] / q5[0];
  bv[5] = t0;
  for (int l = 0; l < t.ns; ++l) yk[l] = Y[l];
  th_temperature(&t, &B, 0);
  return bv[5];
}

int oc_apply_boundaries(oc_solver *s) {
  apply_bcs_and_exchange(s);
  return 0;
}
