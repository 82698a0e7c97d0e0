/*
 * cc_oracle.h -- CPU FP64 restatement of CombustionCodeGPU's per-timestep
 * residual path.  TEST INFRASTRUCTURE ONLY: this is what the tests compare
 * the CUDA product against, and the timed CPU baseline.  Nothing in
 * the product links, loads or calls it.
 *
 * Every function in cc_oracle.c cites the reference file:line it restates.
 * Parity of this restatement is pinned against the reference's own kernels
 * (compiled from the reference sources by oracle/ref_harness, run on a B200)
 * through the fixtures under tests/golden/.
 *
 * Layout: per block, structure-of-arrays over the full ghosted box
 * (mx+2g)(my+2g)(mz+2g), i fastest: idx = (i+g) + NX*((j+g) + NY*(k+g)).
 */
#ifndef CC_ORACLE_H
#define CC_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* Same member order as cfd::Boundary (Mesh.h:9-32). */
typedef struct oc_boundary {
  int range_start[3];
  int range_end[3];
  int type_label;
  int face;
  int direction;
} oc_boundary;

/* Same member order as cfd::InnerFace (Mesh.h:34-60). */
typedef struct oc_inner_face {
  int range_start[3];
  int range_end[3];
  int face;
  int direction;
  int target_start[3];
  int target_end[3];
  int target_block;
  int target_face;
  int target_direction;
  int src_tar[3];
  int loop_dir[3];
  int target_loop_dir[3];
} oc_inner_face;

/* Boundary-condition definition (BoundCond.h:14-64): kind 2 wall, 5 inflow, 6 outflow. */
typedef struct oc_bc {
  int label;
  int kind;
  int thermal_type;      /* wall: 0 isothermal, 1 adiabatic */
  double t_wall;
  double density, u, v, w, pressure, temperature;  /* inflow state */
  double yk[32];                                   /* inflow mass fractions */
} oc_bc;

/* Scalar parameters and species tables (DParameter.h:9-39). n_spec == 0 is
 * the single-species calorically perfect air model (MULTISPECIES=0). */
typedef struct oc_params {
  int n_spec;
  int reconstruction;   /* 2 = MUSCL, other = first order */
  int limiter;          /* 0/1 = minmod */
  int viscous_order;    /* 0 = inviscid, 2 = 2nd-order central */
  int ngg;
  double Pr, cfl, Sc;
  const double *mw, *t_low, *t_mid, *t_high;
  const double *low_coeff, *high_coeff;          /* [n_spec][7] */
  const double *LJ_potent_inv, *vis_coeff;       /* [n_spec] */
  const double *WjDivWi_to_One4th, *sqrt_WiDivWjPl1Mul8;  /* [n_spec][n_spec] */
} oc_params;

typedef struct oc_solver oc_solver;

oc_solver *oc_create(const oc_params *p, int n_block, const int *dims);
void oc_destroy(oc_solver *s);
int oc_set_threads(int n);

/* raw = (x1,x2,y1,y2,z1,z2,type) as read by Mesh::read_boundary. */
int oc_add_boundary_raw(oc_solver *s, int blk, const int raw[7]);
/* raw = 13 ints as read by Mesh::read_inner_interface (1-based, signed). */
int oc_add_inner_face_raw(oc_solver *s, int blk, const int raw[13]);
int oc_get_boundary(const oc_solver *s, int blk, int i, oc_boundary *out);
int oc_get_inner_face(const oc_solver *s, int blk, int i, oc_inner_face *out);
int oc_add_bc(oc_solver *s, const oc_bc *bc);

/* jac [Ng], metric [9][Ng] with row r*3+c holding m(r+1,c+1). */
int oc_set_geometry(oc_solver *s, int blk, const double *jac, const double *metric);
/* bv [6][Ng] (rho,u,v,w,p,T), yk [n_spec][Ng]; values on ghosts included. */
int oc_set_state(oc_solver *s, int blk, const double *bv, const double *yk);

int oc_init(oc_solver *s);
/* One pass of the reference's steady explicit-Euler loop body with the
 * per-point local time step (Driver.cu:189-244); renorm_y as for RK3. */
int oc_steady_step(oc_solver *s, int renorm_y);
/* One implicit steady step: scalar LU-SGS with the per-point local time step
 * (the scheme the reference declares as temporal_scheme 1 without a body). */
int oc_lusgs_step(oc_solver *s, int renorm_y);
/* One SSP-RK3 step with a global time step; renorm_y renormalises the
 * mass fractions to sum 1 after each stage. */
int oc_rk3_step(oc_solver *s, int renorm_y);
/* Only the spatial operator: dq of the current state into dq [n_var][N]. */
int oc_compute_dq(oc_solver *s, int blk, double *dq);

int oc_get_state(const oc_solver *s, int blk, double *bv, double *yk, double *cv);
int oc_get_props(const oc_solver *s, int blk, double *mul, double *cond, double *rho_d,
                 double *gamma, double *acoustic);
int oc_get_dt_local(const oc_solver *s, int blk, double *dt);
double oc_last_dt(const oc_solver *s);
/* Residual of Driver::compute_residual (Driver.cu:219-277): raw RMS of the
 * change of (rho,|V|,p,T) over the last step, before the res_scale division. */
int oc_residual(const oc_solver *s, double out[4]);
int oc_newton_failures(const oc_solver *s);

/* Known-answer hooks: the face, thermo, transport and Newton routines of the
 * restatement on single inputs, and the boundary/interface fill alone. */
double oc_kat_minmod(double a, double b);
void oc_kat_face_inviscid(const oc_params *p, const double *pv4, const double ml[3], double jl, const double mr[3],
                          double jr, double *fc);
void oc_kat_h_cp(const oc_params *p, double t, double *h, double *cp);
void oc_kat_transport(const oc_params *p, double t, const double *Y, double *mu, double *lam, double *rhod);
double oc_kat_temperature(const oc_params *p, const double *q5, const double *Y, double t0);
/* The LU-SGS Jacobian-vector product dF = A dQ of the flux along k. */
void oc_kat_lusgs_jac_vec(int nv, const double *Q, double p, double gam, const double *psi, const double k[3],
                          const double *dQ, double *dF);
int oc_apply_boundaries(oc_solver *s);

#ifdef __cplusplus
}
#endif
#endif
