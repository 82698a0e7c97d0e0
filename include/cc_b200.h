/*
 * cc_b200.h -- C ABI of the B200 (sm_100a) residual path of CombustionCodeGPU.
 *
 * The reference has no FFI; its operator surface is the C++ stack
 *   Driver(Parameter&, Mesh&, ChemData&)      Driver.h:17-26, main.cu:37-45
 *   Driver::initialize_computation()          Driver.cu:59-97
 *   Driver::simulate() / steady_simulation()  Driver.cu:99-192
 *   Field{HZone, DZone*}, DParameter          Field.h:36-82, DParameter.h:9-39
 *   Boundary / InnerFace                      Mesh.h:9-60
 * Every entry point below names the reference interface it replaces.  All
 * functions return 0 on success and a negative code on failure; the message
 * of the last failure on the calling thread is returned by cc_last_error().
 * Plain pointers and sizes only; the library owns all device memory.
 *
 * Array layout of host buffers: per block, structure-of-arrays over the full
 * ghosted box (mx+2g) x (my+2g) x (mz+2g), i fastest, g = ngg ghost layers:
 *   element (i,j,k) of field f at  f*Ng + (i+g) + (mx+2g)*((j+g) + (my+2g)*(k+g)).
 */
#ifndef CC_B200_H
#define CC_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CC_MAX_SPECIES 16

enum cc_status_code {
  CC_OK = 0,
  CC_ERR_ARG = -1,       /* invalid argument */
  CC_ERR_STATE = -2,     /* call out of order (e.g. cc_step before cc_init) */
  CC_ERR_CUDA = -3,      /* a CUDA call failed (message in cc_last_error) */
  CC_ERR_TOPOLOGY = -4,  /* boundary/interface layout the halo program cannot express */
  CC_ERR_NODEVICE = -5   /* no CUDA device */
};

enum cc_precision {
  CC_FP64 = 0,   /* plain: every field and every operation in FP64 */
  CC_MIXED = 1,  /* reconstruction, fluxes, transport, stored primitives in FP32;
                    conserved variables, RK accumulation, Newton, Y renormalisation,
                    dt and residual reductions in FP64 */
  CC_FP32 = 2    /* full FP32, for precision studies: as CC_MIXED, and the
                    conserved variables are rounded to FP32 after every update,
                    the temperature Newton and the Y renormalisation run in FP32
                    (the residual reduction stays FP64) */
};

enum cc_time_scheme {
  CC_RK3 = 0,          /* SSP-RK3 with a global time step (min of the local CFL step) */
  CC_STEADY_EULER = 1, /* the reference's loop: explicit Euler with the per-point local step */
  CC_STEADY_LUSGS = 2  /* implicit steady step: scalar LU-SGS with the per-point local step
                          (the scheme the reference declares as temporal_scheme 1,
                          TemporalScheme.cuh:19-21, Driver.cu:318-321, without a body) */
};

/* Scalar parameters and species tables, as in DParameter (DParameter.h:9-39)
 * and Species (ChemData.h:11-46).  n_spec == 0 selects the calorically
 * perfect air model (the reference's MULTISPECIES=0 build).  Tables are
 * copied by cc_create. */
typedef struct cc_params {
  int n_spec;
  int inviscid_scheme;   /* 3 = AUSM+ (the only scheme of the reference) */
  int reconstruction;    /* 2 = MUSCL, other = first order */
  int limiter;           /* 0/1 = minmod */
  int viscous_order;     /* 0 = inviscid, 2 = second-order central */
  int ngg;               /* ghost layers, 2 (Parameter.cpp:32-36) */
  double prandtl_number, cfl, schmidt_number;
  const double *mw;                  /* [n_spec] molecular weights */
  const double *t_low, *t_mid, *t_high;
  const double *low_temp_coeff;      /* [n_spec][7] NASA-7, T < t_mid */
  const double *high_temp_coeff;     /* [n_spec][7] NASA-7, T >= t_mid */
  const double *LJ_potent_inv;       /* [n_spec] 1/(eps/k) */
  const double *vis_coeff;           /* [n_spec] 2.6693e-6 sqrt(W)/sigma^2 */
  const double *WjDivWi_to_One4th;   /* [n_spec][n_spec] */
  const double *sqrt_WiDivWjPl1Mul8; /* [n_spec][n_spec] */
} cc_params;

/* Byte-compatible with cfd::Boundary after register_boundary (Mesh.h:9-32). */
typedef struct cc_boundary {
  int range_start[3];
  int range_end[3];
  int type_label;
  int face;
  int direction;
} cc_boundary;

/* Byte-compatible with cfd::InnerFace after register_boundary (Mesh.h:34-60). */
typedef struct cc_inner_face {
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
} cc_inner_face;

/* A boundary condition bound to a face label (BoundCond.h:14-64):
 * kind 6 outflow, 5 inflow (Dirichlet state), 2 wall. */
typedef struct cc_bc {
  int label;
  int kind;
  int thermal_type;   /* wall: 0 isothermal, 1 adiabatic */
  int pad;
  double t_wall;
  double density, u, v, w, pressure, temperature;  /* inflow */
  double yk[CC_MAX_SPECIES];                       /* inflow mass fractions */
} cc_bc;

typedef struct cc_ctx cc_ctx;

const char *cc_last_error(void);
int cc_version(void);
int cc_device_count(int *n);

/* Driver::Driver + DParameter::DParameter (Driver.cu:17-57, DParameter.cu:4-45). */
int cc_create(const cc_params *params, cc_ctx **out);
int cc_destroy(cc_ctx *ctx);

/* Mesh/Field setup for one block (Field::setup_device_memory, Field.cu:90-148):
 * jac [Ng] and metric [9][Ng] (row r*3+c = m(r+1,c+1), Mesh.cpp:226-488). */
int cc_add_block(cc_ctx *ctx, int mx, int my, int mz, const double *jac, const double *metric, int *block_id);
/* Boundary::register_boundary (Mesh.cpp:14-32): raw = x1,x2,y1,y2,z1,z2,type. */
int cc_register_boundary(const int raw[7], int ngg, cc_boundary *out);
/* InnerFace::InnerFace + register_boundary (Mesh.cpp:35-143): 13 raw ints. */
int cc_register_inner_face(const int raw[13], int ngg, cc_inner_face *out);
/* Block::boundary / Block::inner_face entries (processed form). */
int cc_add_boundary(cc_ctx *ctx, int block, const cc_boundary *b);
int cc_add_inner_face(cc_ctx *ctx, int block, const cc_inner_face *f);
/* DBoundCond::initialize_bc_on_GPU (BoundCond.cu:315-409); call after all
 * faces are added.  Conditions are applied in the reference's priority order
 * (outflow, inflow, wall; BoundCond.cu:251-313), then the block interfaces. */
int cc_add_bc(cc_ctx *ctx, const cc_bc *bc);

/* Host layout of the state arrays of cc_set_state / cc_get_state:
 * FIELD_MAJOR = one field after another, [n_field][Ng], i fastest within a
 * field; POINT_MAJOR = the reference's VectorField3D order (Field.h:36-63,
 * indexed point * n_field + l as in Driver.cu:341-344), [Ng][n_field], the
 * component fastest.  Ng runs over the ghosted box, i fastest, then j, k. */
#define CC_LAYOUT_FIELD_MAJOR 0
#define CC_LAYOUT_POINT_MAJOR 1
/* HZone::bv / HZone::yk (Field.h:13-32), copied host -> device:
 * bv = rho,u,v,w,p,T (6 fields);  yk = n_spec fields, in `layout`.  Before
 * cc_init it sets the initial field; afterwards it replaces the state
 * (primitives, conserved variables and properties are re-derived as by
 * cc_init). */
int cc_set_state(cc_ctx *ctx, int block, const double *bv, const double *yk, int layout);
/* Driver::initialize_computation (Driver.cu:59-97). */
int cc_init(cc_ctx *ctx, int precision);
/* Driver::simulate: n_steps steps of the chosen scheme (Driver.cu:113-192).
 * want_residual != 0 also evaluates the residual of the last step. */
int cc_step(cc_ctx *ctx, int n_steps, int scheme, int want_residual);
/* Driver::compute_residual (Driver.cu:219-277): RMS change of rho, |V|, p, T
 * over the last step, before the res_scale normalisation. */
int cc_residual(cc_ctx *ctx, double out[4]);
/* The same four values copied into out[4] on the context's stream without
 * waiting (out should be pinned host memory); they are there once the stream
 * has reached the copy (cc_sync, or an event recorded after the call). */
int cc_residual_async(cc_ctx *ctx, double *out);
/* Device -> host: bv (6 fields), yk (n_spec), cv (n_var) in `layout`; null
 * skips an array.  The steps leave the conserved state of ghost points that
 * no kernel reads; when cv is requested, those values are first written on
 * the context's stream (once after a cc_step), so cv matches a halo program
 * that wrote every point. */
int cc_get_state(cc_ctx *ctx, int block, double *bv, double *yk, double *cv, int layout);
/* DZone::mul / conductivity / rho_D (Field.h:52-56): [Ng], [Ng], [n_spec][Ng]. */
int cc_get_props(cc_ctx *ctx, int block, double *mul, double *conductivity, double *rho_d);
/* Time step of the last completed step (RK3). */
int cc_last_dt(cc_ctx *ctx, double *dt);
/* Device status word: bit 0 Newton iteration cap hit, bit 1 non-finite or
 * non-positive rho/p/T, bit 2 invalid time step, bit 3 a TMA plane wait gave
 * up, bit 4 a tensor-core completion wait of the closure gave up.  Cleared by
 * the call.  The reference checks none of these (its Newton, Thermo.cu:103-121,
 * stops silently after 1000 iterations). */
int cc_status(cc_ctx *ctx, unsigned *flags);
/* No counterpart in the reference.  Polls of a device-side wait (a TMA plane,
 * a tensor-core completion) after its first non-blocking check, before the
 * kernel gives up on it, sets its status bit (3 or 4) and returns; the
 * context stays usable.  0 = give up unless the first check finds the data
 * there; spins < 0 restores the default (2^22).  Takes effect at the next
 * cc_step. */
int cc_set_wait_limit(cc_ctx *ctx, int64_t spins);
/* Iteration cap of the temperature Newton (Thermo.cu:103-121: 1000); a point
 * that reaches it sets status bit 0.  n <= 0 restores 1000.  Takes effect at
 * the next cc_step. */
int cc_set_newton_max_iter(cc_ctx *ctx, int n);
/* Stream used by every launch of the context (default: a private stream). */
int cc_set_stream(cc_ctx *ctx, void *cuda_stream);
void *cc_get_stream(cc_ctx *ctx);
/* Renormalise the mass fractions to sum 1 after every update (FP64):
 * 1 on, 0 off, -1 default (on for CC_MIXED, off for CC_FP64, which keeps the
 * reference's update, TimeAdvanceFunc.cu:273-276, unchanged). */
int cc_set_renormalize(cc_ctx *ctx, int enable);
/* 1 = replay whole steps from a captured CUDA graph (default), 0 = launch. */
int cc_use_graph(cc_ctx *ctx, int enable);
/* Points updated per stage (sum of mx*my*mz) and arena bytes on the device. */
int cc_info(cc_ctx *ctx, int64_t *n_points, int64_t *device_bytes, int *n_tiles, int *n_halo_levels);
/* Runs n_steps steps without graph replay, timing every stage-kernel launch
 * and every halo program with CUDA events on the context's stream:
 * out_ms = {mean stage-kernel ms per stage, mean halo ms per stage,
 *           number of stages, mean stage+halo ms per step,
 *           mean face-kernel ms and mean update-kernel ms per stage (split
 *           variant; 0 for the fused variants)}. */
int cc_time_kernels(cc_ctx *ctx, int n_steps, int scheme, double out_ms[6]);
/* The stage-kernel configuration in use (chosen by the autotuner at the
 * first cc_init, or pinned by cc_set_tuning) and its measured time per
 * stage: variant 0 = fused stage kernel with L1 stencil reads, 1 = fused
 * with TMA-staged primitive planes, 2 = split (face kernel, then update
 * kernel), 3 = split with TMA-staged planes in the face kernel, 4 = as 3
 * with the face kernel on persistent CTAs taking tiles from a counter, 5 =
 * face kernel that differences the faces inside its tile and writes dq, then
 * the update kernel; kz = k-planes per tile; tile (may be null) = the face
 * kernel's tile {i, j, k} in points.  CC_AUTOTUNE=0 keeps the heuristic. */
int cc_tuning(cc_ctx *ctx, int *variant, int *kz, double *stage_ms, int tile[3]);
/* No counterpart in the reference (its launch shapes are fixed: 64-point
 * pencils, TimeAdvanceFunc.cu:44-57).  Pins the stage-kernel configuration
 * instead of autotuning it: variant -1 = autotune, 0 = fused with L1 stencil
 * reads, 1 = fused with TMA-staged planes, 2 = split faces / update, 3 =
 * split with TMA-staged face planes, 4 = as 3 on persistent CTAs, 5 = faces
 * differenced in the tile (TMA variants: 0 or 9 species; 1 and 5: FP32 bulk
 * precision); kz = k-planes per tile, 0 = autotune; tile_j = points along j
 * of the TMA face kernel's tile in variants 3-5 (4, 8 or 16, 16 in the FP32
 * bulk precision only; 0 = autotune; the other kernels' tiles are 32 x 8).
 * Before cc_init it applies to the first cc_init; after it, the new
 * configuration is timed and used from the next cc_step on. */
int cc_set_tuning(cc_ctx *ctx, int variant, int kz, int tile_j);
/* Points along i of the TMA face kernel's tile in variants 3 and 4: 32 (one
 * warp per row), 16 (two rows per warp, with tile heights 8 and 16; fewer
 * idle lanes on blocks whose i extent is not a multiple of 32), or 0 =
 * autotune (default).  Applies from the next tuning: cc_init or
 * cc_set_tuning. */
int cc_set_tile_width(cc_ctx *ctx, int tile_i);
/* Launch granularity of the stage kernels: 0 (default) = one launch per
 * kernel over the tiles of every block; 1 = one launch per block per kernel,
 * the reference's granularity (Driver.cu:144-177 launches per block), kept for
 * comparison.  Results are identical; takes effect at the next cc_step. */
int cc_set_launch_mode(cc_ctx *ctx, int per_block);
/* Multi-process runs: the reference's ParallelFace path (Mesh.h:62-102, with
 * its MPI set-up at Driver.cu:80-82, 252-254), which it leaves unfinished.
 * Every process holds the whole grid and advances the blocks it owns
 * (cc_set_owned_blocks; n <= 0 = every block).  Inside cc_step the exchange
 * hook (cc_set_exchange) is called on the host after each stage's kernels and
 * before its halo program (event CC_EXCHANGE_STAGE, stage 0..2 of RK3, 0 of a
 * steady step): the hook moves, between processes, the points its blocks'
 * halo program reads from blocks that other processes own
 * (cc_halo_dependencies), with cc_pack_points / cc_unpack_points.  After the
 * time-step reduction of an RK3 step it is called with event CC_EXCHANGE_DT
 * and *value = this process's next time step, which it replaces by the
 * minimum over processes.  A nonzero return aborts cc_step with
 * CC_ERR_STATE.  While a hook is set, steps are launched, not replayed from a
 * CUDA graph; the LU-SGS step is not available. */
#define CC_EXCHANGE_STAGE 0
#define CC_EXCHANGE_DT 1
typedef int (*cc_exchange_fn)(void *user, int event, int stage, double *value);
int cc_set_owned_blocks(cc_ctx *ctx, const int *blocks, int n);
int cc_set_exchange(cc_ctx *ctx, cc_exchange_fn fn, void *user);
/* Inside a CC_EXCHANGE_STAGE call: all fields of the listed arena points of
 * the state the halo program reads as current (which 0: the stage's new
 * state) or previous (which 1), as [n_fields][n] FP64 host arrays;
 * n_fields = (6+ns) primitives + (2+ns) transport properties (the bulk
 * precision widened exactly) + (5+ns) conserved variables. */
int cc_exchange_fields(cc_ctx *ctx, int *n_fields);
int cc_pack_points(cc_ctx *ctx, int which, const int64_t *idx, int64_t n, double *out);
int cc_unpack_points(cc_ctx *ctx, int which, const int64_t *idx, int64_t n, const double *in);
/* The last residual's sums of squared changes of rho, |V|, p, T over this
 * process's points and their number (cc_residual = sqrt(sums / count)); a
 * multi-process run adds both over processes. */
int cc_residual_sums(cc_ctx *ctx, double sums[4], int64_t *count);
/* Learned transport closure (a22: absent in the reference, which always
 * evaluates Transport.cu:43-96).  An MLP maps (T, X_1..X_n) to
 * (log mu, log lambda, log rhoD_1..rhoD_n): inputs t = (T - t_center)/t_scale
 * and the mole fractions X_k, each fed as a BF16 pair (hi, value - hi), in the
 * order [t_hi, t_lo, X_hi[n], X_lo[n]]; three hidden layers of 64 SiLU units;
 * output o_j gives property_j = exp(o_j * out_scale[j] + out_mean[j]).
 * Weights are row-major (output, input) FP32 and are stored as BF16 on the
 * device; biases stay FP32; the tensor cores accumulate in FP32.  Points with
 * T outside [t_min, t_max] (the training hull) or a mole fraction of at least
 * 0.998 (where the exact rhoD_k switches branch) take the exact transport.
 * Supports 1..14 species. */
typedef struct cc_closure {
  const float *w1, *b1;            /* [64][2 + 2 n_spec], [64] */
  const float *w2, *b2;            /* [64][64], [64] */
  const float *w3, *b3;            /* [64][64], [64] */
  const float *w4, *b4;            /* [2 + n_spec][64], [2 + n_spec] */
  const float *out_mean, *out_scale; /* [2 + n_spec] */
  double t_center, t_scale;
  double t_min, t_max;
} cc_closure;
/* Copies a closure to the device (any time after cc_create). */
int cc_set_closure(cc_ctx *ctx, const cc_closure *closure);
/* Stages take the transport properties of the new state from the closure
 * (1) or from the exact Wilke / constant-Schmidt evaluation (0, default).
 * With the closure on, the global time step is reduced after the halo. */
int cc_use_closure(cc_ctx *ctx, int on);
/* Since cc_set_closure: out[0] points the closure kernel evaluated, out[1]
 * of those that took the exact transport outside the training hull, out[2]
 * points of tiles the run-time error check sent back to the exact
 * transport. */
int cc_closure_stats(cc_ctx *ctx, int64_t out[3]);
/* No counterpart in the reference.  Relative error bound of the closure's
 * run-time check: every 128-point tile is sampled at 4 fixed points (1 in
 * 32) against the exact transport (Transport.cu:43-96, against which
 * the network's error is measured), and a tile whose sampled properties
 * have a root-mean-square relative error above the bound, or one above ten
 * times the bound, takes the exact transport.  Default 1e-3; 0 switches the check off. */
int cc_set_closure_bound(cc_ctx *ctx, double rel_err);
/* Transport properties of n points (host arrays): T [n], Y [n_spec][n] ->
 * out [2 + n_spec][n] = (mu, lambda, rhoD_k), by the exact FP64 evaluation
 * (mode 0) or by the closure kernel (mode 1).  Needs a device, not cc_init. */
int cc_eval_transport(cc_ctx *ctx, int64_t n, const double *T, const double *Y, int mode, double *out);
/* Checkpoint / restart (absent in the reference, Initialize.cu:14-22 only
 * starts from inflow states): the current state as it is on the device
 * (conserved variables, primitives and transport in the bulk precision, |V|,
 * the time step), so that a restart continues bit-identically.  Loading
 * needs a context initialised with the same blocks, species and precision. */
int cc_save_checkpoint(cc_ctx *ctx, const char *path);
int cc_load_checkpoint(cc_ctx *ctx, const char *path);
/* No counterpart in the reference, whose multi-process exchange
 * (ParallelFace, Mesh.h:62-102) is unfinished.  Host-side query for a run in
 * which each process computes some of the blocks: the halo program's
 * dependencies as triples (dst[k], src[k], which[k]), one for every arena
 * point src[k] of the current (which 0) or previous (which 1) state that the
 * final value of the changed point dst[k] is computed from (a copied point,
 * or a source of an interface average, wall or inflow node), so that a
 * process can fetch from their owners the sources of its own blocks' halo
 * before running it.  Needs no device and may be called before cc_init, once
 * the blocks, faces and conditions are added.  Writes at most cap triples
 * (any of dst, src, which may be null) and the total count to *n. */
int cc_halo_dependencies(cc_ctx *ctx, int64_t *dst, int64_t *src, int *which, int64_t cap, int64_t *n);
/* Arena index of the first point of block b's ghosted box and its point
 * count, in the layout of cc_halo_dependencies (no device needed). */
int cc_block_arena(cc_ctx *ctx, int block, int64_t *first, int64_t *count);
/* Synchronises the context's stream. */
int cc_sync(cc_ctx *ctx);

/* Training of the learned transport closure (no counterpart in the
 * reference): the 4-layer MLP n_in -> hidden -> hidden -> hidden -> n_out
 * (SiLU) of cc_closure, trained with the inference kernel's rounding points
 * (layer inputs and weights rounded to BF16 in the forward pass, passed
 * through unchanged in the backward pass; FP32 master weights, biases and
 * accumulation).  Widths at most 64.  params: one FP32 buffer W1 [hidden][n_in],
 * b1, W2 [hidden][hidden], b2, W3, b3, W4 [n_out][hidden], b4 of
 * cc_mlp_param_count floats.  All pointers are device memory owned by the
 * caller; nothing is allocated; work is cc_mlp_workspace_bytes bytes.
 * cc_mlp_grad: loss = mean over batch and outputs of ((mlp(x) - y) scale)^2
 * (x [batch][n_in] holding BF16-representable values, y [batch][n_out],
 * scale [n_out]) into *loss and its gradient into grad, enqueued on stream;
 * sums run in a fixed order, so results are reproducible bit for bit.
 * cc_mlp_adam: one Adam step (bias-corrected, step >= 1, no weight decay). */
int64_t cc_mlp_param_count(int n_in, int hidden, int n_out);
int64_t cc_mlp_workspace_bytes(int n_in, int hidden, int n_out, int batch);
int cc_mlp_grad(int n_in, int hidden, int n_out, int batch, const float *params, const float *x, const float *y,
                const float *out_scale, float *grad, float *loss, void *workspace, void *stream);
int cc_mlp_adam(int64_t n, float *params, const float *grad, float *m, float *v, float lr, float beta1, float beta2,
                float eps, int step, void *stream);

/* No counterpart in the reference.  Residual norms without any allocation,
 * for callers that cannot call cudaMalloc where they need them (an
 * allocation-free loop, a host application that owns the device allocator):
 * out[l] = sqrt(sum_g (cur[l*n+g] - last[l*n+g])^2 / n), l = 0..3, with cur,
 * last ([4][n]) and out ([4]) in device memory, enqueued on `stream`.  Its
 * scratch is a fixed 64 KiB array inside the library (held by every device
 * that loads it), so n is limited to CC_NOALLOC_MAX_POINTS; larger n is
 * rejected with CC_ERR_ARG.  The first call on a device looks up that
 * array's device address, so make it before any stream capture; the address
 * is kept per device and context, and looked up again on the first call in a
 * new context (after a device reset).  Calls share the array: calls that
 * overlap on the GPU race. */
#define CC_NOALLOC_MAX_POINTS 8388608
int cc_residual_rms_noalloc(const double *cur, const double *last, int64_t n, double *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif
