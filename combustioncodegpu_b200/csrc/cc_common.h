// Shared host/device definitions of the sm_100a residual path.
#pragma once
#include <cstdint>
#include <cstddef>

namespace ccb {

constexpr double kRu = 8314.462618;    // Constants.h:19
constexpr double kGammaAir = 1.4;      // Constants.h:23
constexpr double kMwAir = 28.9647;     // Constants.h:28
constexpr int kMaxSpec = 16;           // species supported by one context
constexpr int kTX = 32;                // stage tile: points along i (one warp)
constexpr int kTY = 8;                 // stage tile: points along j (warps)
constexpr int kRecLen = 12;            // values per NASA-7 record (cp, h, pad)
constexpr long long kDefaultWaitSpins = 1LL << 22;  // polls of a device wait before it gives up

// Per-precision species tables, passed to every kernel by value (constant
// bank).  Horner-form NASA-7 coefficients: for T >= t_mid the `hi` set.
template <typename T>
struct SpecTables {
  T mw[kMaxSpec];
  T inv_mw[kMaxSpec];
  T r_over_mw[kMaxSpec];      // R_u / W_k
  T cv_shift[kMaxSpec];       // R_u / W_k (cp - cv per species)
  T t_low[kMaxSpec], t_mid[kMaxSpec];
  // NASA-7 record of species k, range r (0: T < t_mid, 1: T >= t_mid):
  //   [0..4]  cp/R = a0 + a1 T + ... + a4 T^4
  //   [5..10] h/R  = a5 + T(a0 + T(a1/2 + T(a2/3 + T(a3/4 + T a4/5)))) as b0..b4 = a0, a1/2, .., a4/5; b5 = a5
  //   [11]    padding (records are 16-byte aligned for vector loads)
  alignas(16) T rec[kMaxSpec][2][kRecLen];
  T lj_inv[kMaxSpec];
  T vis_coeff[kMaxSpec];
  T lam_shift[kMaxSpec];      // 1.25 R_u / W_k
  T wj[kMaxSpec * kMaxSpec];  // (W_j/W_i)^(1/4)
  T sw[kMaxSpec * kMaxSpec];  // 1/sqrt(8 (1 + W_i/W_j))
};

struct ChemParams {
  int ns;              // 0 = calorically perfect air
  int nv;              // 5 + ns
  int reconstruction;  // 2 = MUSCL, else first order
  int viscous;         // 1 = second-order central viscous fluxes
  double Pr, cfl, Sc;
  // gauge pressure of the FP32 primitives: the arena stores p - p_ref (0 in
  // the FP64 path), and the momentum face fluxes carry p - p_ref, so that
  // FP32 rounding acts on the pressure variations, not on ~1e5 Pa
  double p_ref;
  // polls of a device wait (TMA plane, tensor-core completion) before the
  // kernel gives up on it and sets its status bit (cc_set_wait_limit); the
  // drain of copies in flight after such an abort keeps its own fixed bound
  long long max_spins;
  // iteration cap of the temperature Newton (Thermo.cu:103-121 stops after
  // 1000; cc_set_newton_max_iter)
  int newton_max_iter;
  int pad_;
  // status word of the context (bounds-checked builds report there)
  unsigned *status;
  SpecTables<double> d;
  SpecTables<float> f;
};

#if defined(__CUDACC__)
#define CCB_HD __host__ __device__
#else
#define CCB_HD
#endif

// Learned transport closure (closure.cuh): tile of 128 points, 3 hidden
// layers of 64, inputs padded to 32 (t and X_k as BF16 hi/lo pairs), outputs
// padded to 16; BF16 weights in the MMA operand layout (W1 [64 x 32],
// W2, W3 [64 x 64], W4 [16 x 64]), FP32 biases.
constexpr int kMlpRows = 128, kMlpH = 64, kMlpIn = 32, kMlpOut = 16;
constexpr int kMlpW1 = kMlpH * kMlpIn * 2, kMlpW2 = kMlpH * kMlpH * 2, kMlpW4 = kMlpOut * kMlpH * 2;
constexpr int kMlpWBytes = kMlpW1 + 2 * kMlpW2 + kMlpW4;  // 22528
constexpr int kMlpBias = 3 * kMlpH + kMlpOut;              // 208 floats
constexpr int kMlpXBytes = kMlpRows * kMlpIn * 2, kMlpHBytes = kMlpRows * kMlpH * 2;

// Byte offset of element (r, k) of an R-row, K-major BF16 operand without
// swizzle: 8-row x 16-byte core matrices, 8-row groups 128 bytes apart, the
// core matrices along K 16R bytes apart.
CCB_HD constexpr int mlp_off(int R, int r, int k) { return (k / 8) * 16 * R + 16 * r + 2 * (k % 8); }

struct ClosureDev {
  const void *w;                        // kMlpWBytes of BF16 weights (16-byte aligned)
  const float *b;                       // kMlpBias
  float out_mean[kMlpOut], out_scale[kMlpOut];
  float t_center, t_inv_scale, t_min, t_max;
  float err_bound;                      // run-time check: relative error above which a tile takes the exact
                                        // transport (0: no check)
  unsigned long long *counts;           // [0] points evaluated, [1] exact outside the hull, [2] exact after the
                                        // run-time check (points of the tiles it sent back)
};

// One block of the multiblock grid in the concatenated field arena.
struct BlockInfo {
  int mx, my, mz, g;
  int nx, ny, nz, pad;  // ghosted extents (nx padded)
  int64_t base;         // arena index of interior point (0,0,0)
  int64_t off;          // arena index of ghost corner (-g,-g,-g)
  int64_t ng;           // points in the ghosted box (nx*ny*nz)
  int64_t interior_off; // offset of this block in interior-only arrays
};

// Work unit of the stage kernel: a kTX x kTY column of points swept over k.
struct Tile {
  int blk, i0, j0, k0, k1, pad0, pad1, pad2;
};

// Halo program entry: one destination point filled from resolved sources.
enum HaloOp : int {
  kHaloCopy = 0,       // dst <- src
  kHaloAvg = 1,        // dst <- (src + src2) / 2       (coincident interface layer)
  kHaloInflow = 2,     // dst <- inflow state bc
  kHaloWallFace = 3,   // wall point: p, Y from src (i-dir), T_wall or T(src)
  kHaloWallGhost = 4,  // mirror of src; T reference from src2 (i-dir)
  kHaloKeep = 5,       // reserved (dst <- previous buffer value of dst): never emitted by the builder
};

struct BcDevice {
  int kind;           // 2 wall, 5 inflow, 6 outflow
  int thermal_type;   // wall: 0 isothermal, 1 adiabatic
  double t_wall;
  double rho, u, v, w, p, T;
  double yk[kMaxSpec];
  double rhoE;                     // inflow total energy (compute_total_energy)
  double mu, lam, rho_d[kMaxSpec]; // inflow transport properties
};

// Status bits reported by cc_status.
enum StatusBits : unsigned {
  kStatusNewtonCap = 1u,     // temperature Newton hit its iteration cap
  kStatusNonFinite = 2u,     // NaN/Inf or non-positive rho/p/T after an update
  kStatusBadDt = 4u,         // global time step not positive and finite
  kStatusHaloTimeout = 32u,  // a grid-wide barrier of the single-launch halo program gave up
  kStatusBounds = 64u,       // bounds-checked build: an index outside its array was caught
};

// Bounds-checked build (nvcc -DCC_BOUNDS_CHECK, libcc_b200_bounds.so): the
// arena, scratch and plane indices the kernels compute are checked before
// use; an index outside [0, n) sets kStatusBounds in the context's status
// word and is replaced by 0, so the access stays inside the allocation.  It
// stands in for compute-sanitizer's memory check.  In the normal build the
// macros are the index itself.
#if defined(CC_BOUNDS_CHECK) && defined(__CUDACC__)
__device__ __forceinline__ int64_t ccb_checked_index(unsigned *status, int64_t idx, int64_t n) {
  if (idx >= 0 && idx < n) return idx;
  if (status) atomicOr(status, (unsigned)kStatusBounds);
  return 0;
}
#define CCB_IDX(C, idx, n) ((decltype(idx))ccb_checked_index((C).status, (int64_t)(idx), (int64_t)(n)))
#define CCB_CHECK(C, cond)                                                   \
  do {                                                                       \
    if (!(cond) && (C).status) atomicOr((C).status, (unsigned)kStatusBounds); \
  } while (0)
#else
#define CCB_IDX(C, idx, n) (idx)
#define CCB_CHECK(C, cond) \
  do {                     \
  } while (0)
#endif

// Arrival counter and generation of the bounded grid-wide barrier of the
// single-launch halo program (zeroed at set-up; every completed barrier
// leaves count at 0).
struct GridBarrier {
  unsigned count;
  unsigned gen;
};

// Node levels the single-launch halo program takes (more fall back to one
// launch per level), and their bounds in the node list.
constexpr int kHaloMaxLevels = 8;
struct HaloLevels {
  int64_t begin[kHaloMaxLevels + 1];
  int n;
};

// Arguments of one stage launch (see stage.cuh).
template <typename T>
struct StageArgs {
  const BlockInfo *blocks;
  const Tile *tiles;
  int64_t N;                 // arena stride in points
  const T *P;                // primitives of the current state
  T *Pn;                     // primitives of the new state
  const T *Pr;               // transport properties, current
  T *Prn;                    // transport properties, new
  const T *G;                // geometry
  const double *Qin;         // conserved, current stage
  const double *Qn;          // conserved, step start (read when a != 0)
  double *Qout;              // conserved, new (may alias Qin)
  double a, b;               // Q = a Qn + b (Qin + dt dq / J)
  const double *dt;          // global time step
  unsigned long long *dt_next;  // next global time step (atomicMin), or null
  unsigned *status;
  double *vel;               // |V| of the updated points (DZone::vel), or null
  const uint32_t *skip_dt;   // bitmask of points the halo rewrites (their dt is reduced there)
  int local_dt;              // 1: per-point time step of the current state
  int renorm_y;              // 1: renormalise Y_k to sum 1
  int q32;                   // 1: full-FP32 precision (conserved variables rounded to FP32, FP32 Newton)
  int closure;               // 1: transport of the new state comes from the learned closure kernel (not here)
  const double *gcl;         // [3][N]: sum over directions of k(+) - k(-) per point (p_ref != 0), else null
  // split variant (stage_split.cuh): face fluxes [3][n_var][N] (face d of
  // point p lies between p and p + e_d), the tiles of the minus-side face
  // layers (i, j or k = -1; direction in Tile::pad0), regular tile count
  T *faces;
  const Tile *edge_tiles;
  int n_regular;
  // 1: `faces` holds the residual dq [n_var][N] of every interior point
  // (k_faces_dq), which k_update reads as it is instead of differencing faces
  int dq_direct;
};

// Work arrays of the LU-SGS steady step (lusgs.cuh), in sweep order: the
// interior points sorted by hyperplane h = i + j + k, then block, k and j,
// so that the points of one hyperplane are contiguous and a warp's
// neighbours in the adjacent hyperplane are too.  Per-variable arrays are
// rows of lp doubles per point (lp = lusgs_lanes(n_var), lanes l < n_var
// used), the sweeps' lane-per-variable layout; per-point scalars are plain
// arrays.
struct LusgsArgs {
  int64_t S;         // interior points (sweep positions)
  int lp;            // row length of the per-variable arrays
  const int *pos;    // [N]: sweep position of an interior arena point (-1 elsewhere)
  const int *lo;     // [3][S]: sweep position of p - e_d in the block, or -1
  const int *hi;     // [3][S]: sweep position of p + e_d in the block, or -1
  double *R;         // [S][lp]: dq, then dQ*, then dQ
  double *Qs;        // [S][lp]: conserved state of the step
  double *psi;       // [S][lp]: lanes l >= 5: dp / d(rho Y_{l-5}) at fixed rho e,
                     //          gamma R_k T - (gamma - 1) h_k(T); lanes < 5: 0
  double *Cn;        // [3][S][lp]: A+-_d(q) dQ(q) of the neighbour q in direction d, stored by q
                     //             at this point's row (zero where the block has no such neighbour)
  double *pt;        // [S][kLuScalars]: the point's scalars, at the kLu* offsets
  int64_t s0, s1;    // sweep positions of one launch (one hyperplane)
  int early;         // 1: the launch may read its points' own rows before waiting for its predecessor
};

// Offsets in a point's scalar row (LusgsArgs::pt): 1 / D (D = J / dt_local +
// sum_d r_d), the absolute pressure, gamma, 1 / rho and u, v, w of the
// conserved state (u = (rho u) (1 / rho)), k_d = J grad xi_d (3 x 3) and
// r_d = J (sigma_d + 2 sigv_d) (3); rows are two 128-byte lines.
enum LuScalar : int { kLuRD = 0, kLuP = 1, kLuGam = 2, kLuInv = 3, kLuU = 4, kLuK = 7, kLuRad = 16, kLuScalars = 32 };

// Lanes per point of the LU-SGS sweeps (a power of two >= n_var) and the
// points of one sweep CTA (kSweepThreads threads).
CCB_HD constexpr int lusgs_lanes(int nv) { return nv <= 8 ? 8 : (nv <= 16 ? 16 : 32); }
constexpr int kSweepThreads = 512;

// A source reference of the halo program: kind 0 = point of the new state,
// 1 = point of the previous state, 2 = scratch slot of an evaluated node.
struct HaloRef {
  int64_t idx;
  int kind;
  int pad;
};

struct HaloNode {
  int64_t slot;
  HaloRef a, b;
  int op;
  int bc;
};

// src.pad of a copy: bit 0 = dst is an interior point, bit 1 = its block is
// 3D, bit 2 = dst is itself read by the halo program (a node operand or a
// copy source, as a stage or previous value).
struct HaloCopy {
  int64_t dst;
  HaloRef src;
};

template <typename T>
struct HaloArgs {
  int64_t N;       // arena stride
  int64_t NS_cap;  // scratch stride (slots)
  T *P;            // new state (written by phase B)
  const T *Pprev;
  T *Pr;
  const T *Prprev;
  double *Q;
  const double *Qprev;
  T *sP;           // scratch [6+ns][NS_cap]
  T *sPr;          // scratch [2+ns][NS_cap]
  double *sQ;      // scratch [nv][NS_cap]
  const BcDevice *bcs;
  const HaloNode *nodes;
  const HaloCopy *copies;
  const uint32_t *dt_copy_mask;   // bit per copy: it rewrites an interior point of an owned block, whose
                                  // post-exchange time step enters the next global step
  int64_t begin, end;
  const T *G;                     // geometry (time step of rewritten interior points)
  unsigned long long *dt_next;    // next global time step, or null
};

}  // namespace ccb
