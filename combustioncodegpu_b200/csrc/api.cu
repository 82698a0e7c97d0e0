// C ABI of the sm_100a residual path (include/cc_b200.h).
//
// A context owns: the arena layout of all blocks, the device fields, the
// halo program, the tile list of the stage kernel and one captured CUDA graph
// per (time scheme, parity of the ping-pong buffers).  Everything up to
// cc_init is host-only, so set-up errors surface without a device.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cc_b200.h"
#include "halo_plan.h"
#include "launch.h"

using namespace ccb;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

#define CK(call)                                                                                           \
  do {                                                                                                     \
    cudaError_t e_ = (call);                                                                               \
    if (e_ != cudaSuccess)                                                                                 \
      return fail(CC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_) + " (" + __FILE__ + ":" + \
                                   std::to_string(__LINE__) + ")");                                        \
  } while (0)

template <typename T>
struct Tag {
  using type = T;
};
template <int V>
struct IntC {
  static constexpr int value = V;
};

}  // namespace

void ccb_set_last_error(const std::string &msg) { g_err = msg; }

struct cc_ctx {
  ChemParams chem{};
  int ngg = 2;
  std::vector<HostBlock> blocks;
  std::vector<std::vector<double>> h_geo;  // per block [10][Ng] user layout (jac, metric)
  std::vector<HostBc> bcs;
  std::vector<std::vector<double>> pend_bv, pend_yk;
  std::vector<char> pend;  // block has pending host state

  bool initialized = false;
  bool state_dirty = false;
  int precision = CC_FP64;
  size_t elem = 8;
  int ns_key = -1;  // 0, 9 or -1 (runtime)

  int64_t N = 0, n_int = 0;
  std::vector<BlockInfo> hblocks;
  std::vector<Tile> htiles;
  BlockInfo *d_blocks = nullptr;
  Tile *d_tiles = nullptr;
  void *P[2] = {nullptr, nullptr};
  void *Pr[2] = {nullptr, nullptr};
  void *G = nullptr;
  double *Q[2] = {nullptr, nullptr};
  double *stage64 = nullptr;  // FP64 staging [6+ns][N] of the uploaded state
  double *tmp64 = nullptr;    // [N]
  int cur = 0;                // P/Pr buffer holding the current state
  int qcur = 0;               // Q buffer holding the current state

  HaloPlan plan;
  HaloNode *d_nodes = nullptr;
  HaloCopy *d_copies = nullptr;
  uint32_t *d_dt_copy_mask = nullptr;  // bit per halo copy: its post-exchange time step enters the next step
  void *sP = nullptr, *sPr = nullptr;
  double *sQ = nullptr;
  int64_t ns_cap = 1;
  BcDevice *d_bcs = nullptr;

  double *d_dt = nullptr;
  unsigned long long *d_dt_next = nullptr;
  unsigned *d_status = nullptr;
  double *d_res = nullptr;
  double *d_partials = nullptr;
  double *d_last = nullptr;
  double *d_vel = nullptr;        // DZone::vel: |V| of the last update
  int64_t *d_vel_zero = nullptr;  // wall-face points (vel = 0 after the wall condition)
  uint32_t *d_skip_dt = nullptr;  // bitmask: interior points the halo rewrites
  int renorm = -1;                // Y renormalisation: -1 = by precision (mixed on, FP64 off)
  int variant = 0;                // stage kernels: 0 fused (L1 stencil reads), 1 fused TMA planes, 2 split faces/update,
                                  // 3 split with TMA-staged face planes, 4 the same on persistent CTAs,
                                  // 5 face kernel differencing in the tile (dq) + update
  int face_ty = 8;                // variants 3-5: tile height of the TMA face kernel (face_tx x face_ty x kz points)
  int face_tx = 32;               // variants 3-4: tile width of the TMA face kernel (32 or 16; 32 for variant 5)
  int force_tx = 0;               // cc_set_tile_width: face tile width, 0 = autotune
  int update_occ = 0;             // 1: the FP32 update kernel sized for 4 CTAs per SM (autotuned)
  int force_ty = 0;               // cc_set_tuning: face tile height, 0 = autotune
  std::vector<Tile> hutiles;      // variants 2-5: tiles of the update kernel (upd_tx x 256/upd_tx x kz)
  std::vector<int> ut_begin;      // per block: first update tile, + end
  Tile *d_utiles = nullptr;
  int upd_tx = 32;                // update tile width: the face tile width in variants 3-4, else 32
  std::vector<Tile> hftiles;      // variants 3-5: tiles of the TMA face kernel
  std::vector<int> ft_begin;      // per block: first face tile (block-ordered list), + end
  Tile *d_ftiles = nullptr;
  std::vector<Tile> hedges;       // split variant: tiles of the minus-side face layers
  std::vector<int> tile_begin, edge_begin;  // per block: first tile / edge tile (lists are block-ordered), + end
  bool per_block = false;         // cc_set_launch_mode: one launch per block per kernel instead of one per stage
  Tile *d_edges = nullptr;
  void *faces = nullptr;          // split variant: face fluxes [3][n_var][N] (bulk precision)
  bool tma_ok = false;            // tensor maps built (the TMA variant can run)
  int force_variant = -1;         // cc_set_tuning: -1 autotune, else the variant
  int force_kz = 0;               // cc_set_tuning: k-planes per tile, 0 = autotune
  bool closure_set = false;       // cc_set_closure: learned transport closure uploaded
  bool closure_on = false;        // cc_use_closure: stages take transport from the closure kernel
  ClosureDev cl{};                // device weights, biases, normalisation, counters
  double closure_bound = 1e-3;    // cc_set_closure_bound: relative error of the run-time check (0: none)
  double *d_gcl = nullptr;        // [3][N] geometric term of the gauge-pressure momentum fluxes
  int kz = 1;                     // k-chunk of the stage tiles
  double tuned_ms = 0;            // stage-kernel time of the chosen configuration
  CUtensorMap *d_tmaps = nullptr; // [3][2][n_blocks]: plane boxes of tile height 8, 4, 16 (kTmaRows) for the
                                  // primitive arenas P[0], P[1] per block
  unsigned *d_ticket = nullptr;   // tile counter of the persistent face kernel
  GridBarrier *d_gridbar = nullptr;  // grid-wide barrier of the single-launch halo program
  // multi-process runs (cc_set_owned_blocks, cc_set_exchange): the blocks
  // this process advances, the hook called between a stage's kernels and its
  // halo program and on the local next time step, the owned blocks' BlockInfo
  // (interior offsets renumbered over them) for the time step and residual
  // reductions, and the state buffers the hook's pack / unpack address
  std::vector<char> owned;        // per block (empty: every block)
  cc_exchange_fn hook = nullptr;
  void *hook_user = nullptr;
  std::vector<BlockInfo> hblocks_owned;
  BlockInfo *d_blocks_owned = nullptr;
  int64_t n_int_owned = 0;
  std::vector<uint32_t> dt_copy_mask;   // bit per copy rewriting an owned block's interior point
  int x_pn = 1, x_pp = 0;               // P / Pr buffers of the current and previous state during the hook
  double *x_qn = nullptr, *x_qp = nullptr;
  double *d_xbuf = nullptr;             // pack / unpack staging [n_fields][cap]
  int64_t *d_xidx = nullptr;
  int64_t x_cap = 0;
  bool halo_coop = false;         // the device takes cooperative launches (single-launch halo program)
  // the steps' halo programs leave the conserved state of ghost points,
  // which no stage kernel reads; it is written before the state is read out
  bool q_ghost_stale = false;
  LusgsArgs lu{};                 // LU-SGS work arrays (allocated by the first LU-SGS step)
  std::vector<int64_t> lu_hb;     // sweep positions where each hyperplane begins, + end
  int n_partials = 296;

  cudaStream_t stream = nullptr;
  bool own_stream = false;
  bool use_graph = true;
  cudaGraphExec_t graph[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};
  int64_t device_bytes = 0;
  std::vector<void *> allocs;
  // kernel timing (cc_time_kernels): events around every stage and halo launch
  bool profiling = false;
  std::vector<cudaEvent_t> ev_stage, ev_halo, ev_mid;  // ev_mid: between the split variant's two kernels
  size_t ev_next_stage = 0, ev_next_halo = 0, ev_next_mid = 0;
};

namespace {

int nv_of(const cc_ctx *c) { return 5 + c->chem.ns; }
int np_of(const cc_ctx *c) { return 6 + c->chem.ns; }
int npr_of(const cc_ctx *c) { return 2 + c->chem.ns; }

// Allocation zeroed on the context's stream: every later upload to the
// buffer is issued on the same stream, so it is ordered after the zeroing
// (the context stream is non-blocking: a cudaMemset on the legacy default
// stream could land after such an upload).
int dev_alloc(cc_ctx *c, void **p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  CK(cudaMalloc(p, bytes));
  CK(cudaMemsetAsync(*p, 0, bytes, c->stream));
  c->allocs.push_back(*p);
  c->device_bytes += (int64_t)bytes;
  return 0;
}

template <typename F>
int dispatch(cc_ctx *c, F &&f) {
  const bool dbl = c->precision == CC_FP64;
  switch (c->ns_key) {
    case 0:
      return dbl ? f(Tag<double>{}, IntC<0>{}) : f(Tag<float>{}, IntC<0>{});
    case 9:
      return dbl ? f(Tag<double>{}, IntC<9>{}) : f(Tag<float>{}, IntC<9>{});
    default:
      return dbl ? f(Tag<double>{}, IntC<-1>{}) : f(Tag<float>{}, IntC<-1>{});
  }
}

template <typename T>
void fill_tables(SpecTables<T> &S, const cc_params *p) {
  std::memset(&S, 0, sizeof(S));
  const int ns = p->n_spec;
  for (int k = 0; k < ns; ++k) {
    const double mw = p->mw[k];
    S.mw[k] = (T)mw;
    S.inv_mw[k] = (T)(1.0 / mw);
    S.r_over_mw[k] = (T)(kRu / mw);
    S.cv_shift[k] = (T)(kRu / mw);
    S.t_low[k] = (T)p->t_low[k];
    S.t_mid[k] = (T)p->t_mid[k];
    const double *lo = p->low_temp_coeff + 7 * k, *hi = p->high_temp_coeff + 7 * k;
    const double sc[5] = {1.0, 0.5, 1.0 / 3.0, 0.25, 0.2};
    for (int r = 0; r < 2; ++r) {
      const double *a = r == 0 ? lo : hi;
      T *rec = S.rec[k][r];
      for (int c = 0; c < 5; ++c) rec[c] = (T)a[c], rec[5 + c] = (T)(a[c] * sc[c]);
      rec[7] = (T)(a[2] / 3);
      rec[10] = (T)a[5];
      rec[11] = 0;
    }
    S.lj_inv[k] = (T)p->LJ_potent_inv[k];
    S.vis_coeff[k] = (T)p->vis_coeff[k];
    S.lam_shift[k] = (T)(1.25 * kRu / mw);
    for (int n = 0; n < ns; ++n) {
      S.wj[k * kMaxSpec + n] = (T)p->WjDivWi_to_One4th[k * ns + n];
      S.sw[k * kMaxSpec + n] = (T)p->sqrt_WiDivWjPl1Mul8[k * ns + n];
    }
  }
}

int64_t ng_user(const HostBlock &b) {
  return (int64_t)(b.mx + 2 * b.g) * (b.my + 2 * b.g) * (b.mz + 2 * b.g);
}

// host [nf][Ng] user layout <-> arena rows (pitched copy per field)
int copy_fields_h2d(cc_ctx *c, const HostBlock &b, const double *host, double *dev, int nf) {
  const size_t w = (size_t)(b.mx + 2 * b.g) * sizeof(double);
  const size_t rows = (size_t)(b.my + 2 * b.g) * (b.mz + 2 * b.g);
  const int64_t ng = ng_user(b);
  for (int f = 0; f < nf; ++f)
    CK(cudaMemcpy2DAsync(dev + (int64_t)f * c->N + b.off, (size_t)b.nx * sizeof(double), host + (int64_t)f * ng, w, w,
                         rows, cudaMemcpyHostToDevice, c->stream));
  return 0;
}

int copy_field_d2h(cc_ctx *c, const HostBlock &b, const double *dev_field, double *host_field) {
  const size_t w = (size_t)(b.mx + 2 * b.g) * sizeof(double);
  const size_t rows = (size_t)(b.my + 2 * b.g) * (b.mz + 2 * b.g);
  CK(cudaMemcpy2DAsync(host_field, w, dev_field + b.off, (size_t)b.nx * sizeof(double), w, rows,
                       cudaMemcpyDeviceToHost, c->stream));
  return 0;
}

// T-precision field f of arena `src` -> FP64 tmp64
int field_to64(cc_ctx *c, const void *src, int f, double shift = 0.0) {
  if (c->precision == CC_FP64) {
    CK(cudaMemcpyAsync(c->tmp64, (const double *)src + (int64_t)f * c->N, sizeof(double) * c->N,
                       cudaMemcpyDeviceToDevice, c->stream));
  } else if (shift != 0.0) {
    CK(launch_convert_f2d_shift((const float *)src + (int64_t)f * c->N, c->tmp64, c->N, shift, c->stream));
  } else {
    CK(launch_convert_f2d((const float *)src + (int64_t)f * c->N, c->tmp64, c->N, c->stream));
  }
  return 0;
}

int from64(cc_ctx *c, const double *src, void *dst, int64_t count) {
  if (c->precision == CC_FP64)
    CK(cudaMemcpyAsync(dst, src, sizeof(double) * count, cudaMemcpyDeviceToDevice, c->stream));
  else
    CK(launch_convert_d2f(src, (float *)dst, count, c->stream));
  return 0;
}

// nf fields of ng points between point-major ([ng][nf], from_point_major)
// and field-major ([nf][ng]) host order.
void transpose_fields(const double *src, int64_t ng, int nf, std::vector<double> &dst, bool from_point_major) {
  dst.resize((size_t)(ng * nf));
  for (int64_t p = 0; p < ng; ++p)
    for (int f = 0; f < nf; ++f) {
      if (from_point_major)
        dst[(size_t)(f * ng + p)] = src[p * nf + f];
      else
        dst[(size_t)(p * nf + f)] = src[f * ng + p];
    }
}

// Whether this process advances block b (cc_set_owned_blocks).
bool owns(const cc_ctx *c, int b) { return c->owned.empty() || c->owned[(size_t)b]; }

// Tensor-map plane boxes, each a tile plus the 2-point halo on both sides:
// 32 x 8 (the kTX x kTY tiles of the split and fused kernels), 32 x 4,
// 32 x 16, 16 x 8 and 16 x 16 (the TMA face kernels, i x j).
constexpr int kTmaShapes = 5;
constexpr int kTmaTileRows[kTmaShapes] = {8, 4, 16, 8, 16};
constexpr int kTmaTileCols[kTmaShapes] = {32, 32, 32, 16, 16};
int tma_shape(int ty, int tx = 32) {
  if (tx == 16) return ty == 16 ? 4 : 3;
  return ty == 4 ? 1 : (ty == 16 ? 2 : 0);
}

// Work list of the TMA face kernels: tx x ty columns, k split into chunks of kz.
void build_face_tiles(cc_ctx *c, int ty, int kz, int tx = 32) {
  c->hftiles.clear();
  c->ft_begin.clear();
  for (int bi = 0; bi < (int)c->blocks.size(); ++bi) {
    c->ft_begin.push_back((int)c->hftiles.size());
    const auto &b = c->blocks[bi];
    if (!owns(c, bi)) continue;
    for (int k0 = 0; k0 < b.mz; k0 += kz)
      for (int j0 = 0; j0 < b.my; j0 += ty)
        for (int i0 = 0; i0 < b.mx; i0 += tx) {
          Tile t{};
          t.blk = bi, t.i0 = i0, t.j0 = j0, t.k0 = k0, t.k1 = std::min(b.mz, k0 + kz);
          c->hftiles.push_back(t);
        }
  }
  c->ft_begin.push_back((int)c->hftiles.size());
  c->face_ty = ty;
  c->face_tx = tx;
}

int max_face_tiles(cc_ctx *c) {
  int64_t n = 0;
  for (const auto &b : c->blocks) n += (int64_t)((b.mx + 15) / 16) * ((b.my + 3) / 4) * b.mz;
  return (int)n;
}

// Stage-kernel work list: kTX x kTY columns, k split into chunks of kz.
void build_tiles_kz(cc_ctx *c, int kz) {
  c->htiles.clear();
  c->tile_begin.clear();
  for (int bi = 0; bi < (int)c->blocks.size(); ++bi) {
    c->tile_begin.push_back((int)c->htiles.size());
    const auto &b = c->blocks[bi];
    if (!owns(c, bi)) continue;
    for (int k0 = 0; k0 < b.mz; k0 += kz)
      for (int j0 = 0; j0 < b.my; j0 += kTY)
        for (int i0 = 0; i0 < b.mx; i0 += kTX) {
          Tile t{};
          t.blk = bi, t.i0 = i0, t.j0 = j0, t.k0 = k0, t.k1 = std::min(b.mz, k0 + kz);
          c->htiles.push_back(t);
        }
  }
  c->tile_begin.push_back((int)c->htiles.size());
  c->kz = kz;
}

// Work list of the update kernel of the split variants: ux x (256 / ux)
// columns (32 x 8 or 16 x 16), k split into chunks of kz.
void build_update_tiles(cc_ctx *c, int kz, int ux) {
  const int uy = 256 / ux;
  c->hutiles.clear();
  c->ut_begin.clear();
  for (int bi = 0; bi < (int)c->blocks.size(); ++bi) {
    c->ut_begin.push_back((int)c->hutiles.size());
    const auto &b = c->blocks[bi];
    if (!owns(c, bi)) continue;
    for (int k0 = 0; k0 < b.mz; k0 += kz)
      for (int j0 = 0; j0 < b.my; j0 += uy)
        for (int i0 = 0; i0 < b.mx; i0 += ux) {
          Tile t{};
          t.blk = bi, t.i0 = i0, t.j0 = j0, t.k0 = k0, t.k1 = std::min(b.mz, k0 + kz);
          c->hutiles.push_back(t);
        }
  }
  c->ut_begin.push_back((int)c->hutiles.size());
  c->upd_tx = ux;
}

int upload_update_tiles(cc_ctx *c) {
  if (!c->hutiles.empty())
    CK(cudaMemcpyAsync(c->d_utiles, c->hutiles.data(), sizeof(Tile) * c->hutiles.size(), cudaMemcpyHostToDevice,
                       c->stream));
  return 0;
}

// Tiles of the split variant's minus-side face layers (stage_split.cuh):
// i = -1 faces with lanes along j and warps along k, j = -1 faces with lanes
// along i and warps along k, k = -1 faces with lanes along i, warps along j.
void build_edge_tiles(cc_ctx *c) {
  c->hedges.clear();
  c->edge_begin.clear();
  for (int bi = 0; bi < (int)c->blocks.size(); ++bi) {
    c->edge_begin.push_back((int)c->hedges.size());
    const auto &b = c->blocks[bi];
    if (!owns(c, bi)) continue;
    for (int k0 = 0; k0 < b.mz; k0 += kTY) {
      for (int j0 = 0; j0 < b.my; j0 += kTX) c->hedges.push_back(Tile{bi, -1, j0, k0, std::min(b.mz, k0 + kTY), 0, 0, 0});
      for (int i0 = 0; i0 < b.mx; i0 += kTX) c->hedges.push_back(Tile{bi, i0, -1, k0, std::min(b.mz, k0 + kTY), 1, 0, 0});
    }
    if (b.mz > 1)
      for (int j0 = 0; j0 < b.my; j0 += kTY)
        for (int i0 = 0; i0 < b.mx; i0 += kTX) c->hedges.push_back(Tile{bi, i0, j0, -1, 0, 2, 0, 0});
  }
  c->edge_begin.push_back((int)c->hedges.size());
}

// Initial chunk size (before autotuning): fewest waves times the per-chunk
// cost (kz planes plus the prologue plane).
int heuristic_kz(cc_ctx *c) {
  const int slots_per_sm = c->precision == CC_FP64 ? 1 : 2;
  int n_sm = 148, dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  const int slots = n_sm * slots_per_sm;
  int max_mz = 1;
  for (const auto &b : c->blocks) max_mz = std::max(max_mz, b.mz);
  int best_kz = max_mz;
  double best_cost = 1e300;
  for (int kz = 1; kz <= max_mz; ++kz) {
    int64_t tiles = 0;
    for (const auto &b : c->blocks)
      tiles += (int64_t)((b.mx + kTX - 1) / kTX) * ((b.my + kTY - 1) / kTY) * ((b.mz + kz - 1) / kz);
    const double cost = std::ceil((double)tiles / slots) * (kz + 1.0);
    if (cost < best_cost - 1e-9) best_cost = cost, best_kz = kz;
  }
  return best_kz;
}

int max_tiles(cc_ctx *c) {
  int64_t n = 0;
  for (const auto &b : c->blocks) n += (int64_t)((b.mx + kTX - 1) / kTX) * ((b.my + kTY - 1) / kTY) * b.mz;
  return (int)n;
}

int upload_bcs(cc_ctx *c) {
  std::vector<BcDevice> h(std::max<size_t>(1, c->bcs.size()));
  for (size_t i = 0; i < c->bcs.size(); ++i) {
    const HostBc &b = c->bcs[i];
    BcDevice &d = h[i];
    std::memset(&d, 0, sizeof d);
    d.kind = b.kind, d.thermal_type = b.thermal_type, d.t_wall = b.t_wall;
    d.rho = b.rho, d.u = b.u, d.v = b.v, d.w = b.w, d.p = b.p, d.T = b.T;
    for (int l = 0; l < kMaxSpec; ++l) d.yk[l] = b.yk[l];
  }
  CK(cudaMemcpyAsync(c->d_bcs, h.data(), sizeof(BcDevice) * h.size(), cudaMemcpyHostToDevice, c->stream));
  return 0;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// One 4D tensor map (i, j, k, field) per block and primitive arena; box =
// the tile plane plus its 2-point halo in i and j, all fields.
int build_tensor_maps(cc_ctx *c) {
  void *fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
  if (!fn || q != cudaDriverEntryPointSuccess) return fail(CC_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  auto encode = reinterpret_cast<EncodeTiledFn>(fn);
  const int nb = (int)c->blocks.size();
  std::vector<CUtensorMap> maps(kTmaShapes * 2 * (size_t)nb);
  const size_t E = c->elem;
  for (int shape = 0; shape < kTmaShapes; ++shape)
  for (int buf = 0; buf < 2; ++buf)
    for (int b = 0; b < nb; ++b) {
      const HostBlock &h = c->blocks[b];
      const cuuint64_t dims[4] = {(cuuint64_t)h.nx, (cuuint64_t)h.ny, (cuuint64_t)h.nz, (cuuint64_t)np_of(c)};
      const cuuint64_t strides[3] = {(cuuint64_t)h.nx * E, (cuuint64_t)h.nx * h.ny * E, (cuuint64_t)c->N * E};
      const cuuint32_t box[4] = {(cuuint32_t)(kTmaTileCols[shape] + 4), (cuuint32_t)(kTmaTileRows[shape] + 4), 1u,
                                 (cuuint32_t)np_of(c)};
      const cuuint32_t estr[4] = {1, 1, 1, 1};
      void *base = (char *)c->P[buf] + (size_t)h.off * E;
      CUresult r = encode(&maps[((size_t)shape * 2 + buf) * nb + b],
                          E == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, base, dims,
                          strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r != CUDA_SUCCESS) return fail(CC_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    }
  void *p;
  if (dev_alloc(c, &p, sizeof(CUtensorMap) * maps.size())) return CC_ERR_CUDA;
  c->d_tmaps = (CUtensorMap *)p;
  CK(cudaMemcpyAsync(c->d_tmaps, maps.data(), sizeof(CUtensorMap) * maps.size(), cudaMemcpyHostToDevice,
                     c->stream));
  return 0;
}

// After set-up or a change of the owned blocks: the work lists over the
// owned blocks (stage tiles at the current k-chunk, face tiles at the current
// tile height, edge tiles), the owned blocks' BlockInfo with interior offsets
// renumbered over them (time-step and residual reductions), and the halo
// copies that rewrite an owned interior point (their post-exchange time step).
int apply_ownership(cc_ctx *c) {
  build_tiles_kz(c, c->kz);
  build_face_tiles(c, c->face_ty, c->kz, c->face_tx);
  build_update_tiles(c, c->kz, c->upd_tx);
  if (int r = upload_update_tiles(c)) return r;
  build_edge_tiles(c);
  c->hblocks_owned.clear();
  int64_t off = 0;
  for (size_t b = 0; b < c->hblocks.size(); ++b)
    if (owns(c, (int)b)) {
      BlockInfo B = c->hblocks[b];
      B.interior_off = off;
      off += (int64_t)B.mx * B.my * B.mz;
      c->hblocks_owned.push_back(B);
    }
  c->n_int_owned = off;
  c->dt_copy_mask.assign(c->plan.copies.size() / 32 + 1, 0u);
  for (int64_t ci : c->plan.interior_copies) {
    const int64_t dst = c->plan.copies[(size_t)ci].dst;
    for (size_t b = 0; b < c->hblocks.size(); ++b) {
      const BlockInfo &B = c->hblocks[b];
      if (dst >= B.off && dst < B.off + B.ng) {
        if (owns(c, (int)b)) c->dt_copy_mask[(size_t)(ci >> 5)] |= 1u << (ci & 31);
        break;
      }
    }
  }
  if (!c->htiles.empty())
    CK(cudaMemcpyAsync(c->d_tiles, c->htiles.data(), sizeof(Tile) * c->htiles.size(), cudaMemcpyHostToDevice,
                       c->stream));
  if (!c->hftiles.empty())
    CK(cudaMemcpyAsync(c->d_ftiles, c->hftiles.data(), sizeof(Tile) * c->hftiles.size(), cudaMemcpyHostToDevice,
                       c->stream));
  if (!c->hedges.empty())
    CK(cudaMemcpyAsync(c->d_edges, c->hedges.data(), sizeof(Tile) * c->hedges.size(), cudaMemcpyHostToDevice,
                       c->stream));
  if (!c->hblocks_owned.empty())
    CK(cudaMemcpyAsync(c->d_blocks_owned, c->hblocks_owned.data(), sizeof(BlockInfo) * c->hblocks_owned.size(),
                       cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_dt_copy_mask, c->dt_copy_mask.data(), sizeof(uint32_t) * c->dt_copy_mask.size(),
                     cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

// Arena layout: rows padded to 32 points, every block starting on a
// 32-point boundary.  Fills each block's extents and offsets and its
// BlockInfo; returns the arena size (a multiple of 32 points).
int64_t layout_blocks(std::vector<HostBlock> &blocks, int ngg, std::vector<BlockInfo> &info, int64_t &n_int) {
  int64_t end = 0;
  n_int = 0;
  info.clear();
  for (auto &b : blocks) {
    b.g = ngg;
    b.nx = ((b.mx + 2 * b.g + 31) / 32) * 32;
    b.ny = b.my + 2 * b.g;
    b.nz = b.mz + 2 * b.g;
    int64_t off = ((end + 31) / 32) * 32;  // 128-B aligned block start (TMA tensor-map base)
    b.off = off;
    b.base = off + b.g + (int64_t)b.nx * b.g + (int64_t)b.nx * b.ny * b.g;
    end = off + (int64_t)b.nx * b.ny * b.nz;
    BlockInfo bi{};
    bi.mx = b.mx, bi.my = b.my, bi.mz = b.mz, bi.g = b.g, bi.nx = b.nx, bi.ny = b.ny, bi.nz = b.nz;
    bi.base = b.base, bi.off = b.off, bi.ng = (int64_t)b.nx * b.ny * b.nz, bi.interior_off = n_int;
    n_int += (int64_t)b.mx * b.my * b.mz;
    info.push_back(bi);
  }
  return ((end + 31) / 32) * 32;
}

// Layout, device allocation, halo program, geometry.  Runs once.
int setup_device(cc_ctx *c) {
  const int ns = c->chem.ns;
  c->elem = c->precision == CC_FP64 ? 8 : 4;
  c->ns_key = ns == 0 ? 0 : (ns == 9 ? 9 : -1);
  int64_t n_int = 0;
  c->N = layout_blocks(c->blocks, c->ngg, c->hblocks, n_int);
  c->n_int = n_int;
  if ((double)c->N * (6 + kMaxSpec) >= 2147483647.0)
    return fail(CC_ERR_ARG, "grid too large for one context (32-bit field offsets); split it over contexts");

  std::vector<HostBc> bcs = c->bcs;
  if (!build_halo_plan(c->blocks, bcs, c->plan)) return fail(CC_ERR_TOPOLOGY, "halo program: " + c->plan.error);
  {
    const char *env = std::getenv("CC_KZ");
    build_tiles_kz(c, env && std::atoi(env) > 0 ? std::atoi(env) : heuristic_kz(c));
  }

  const size_t E = c->elem;
  const int64_t N = c->N;
  void *p;
  if (dev_alloc(c, &p, sizeof(BlockInfo) * c->hblocks.size())) return CC_ERR_CUDA;
  c->d_blocks = (BlockInfo *)p;
  if (dev_alloc(c, &p, sizeof(BlockInfo) * c->hblocks.size())) return CC_ERR_CUDA;
  c->d_blocks_owned = (BlockInfo *)p;
  if (dev_alloc(c, &p, sizeof(Tile) * (size_t)std::max(1, max_tiles(c)))) return CC_ERR_CUDA;
  c->d_tiles = (Tile *)p;
  if (dev_alloc(c, &p, sizeof(Tile) * (size_t)std::max(1, max_face_tiles(c)))) return CC_ERR_CUDA;
  c->d_ftiles = (Tile *)p;
  build_face_tiles(c, c->face_ty, c->kz);
  CK(cudaMemcpyAsync(c->d_ftiles, c->hftiles.data(), sizeof(Tile) * c->hftiles.size(), cudaMemcpyHostToDevice, c->stream));
  if (dev_alloc(c, &p, sizeof(Tile) * (size_t)std::max(1, max_face_tiles(c)))) return CC_ERR_CUDA;
  c->d_utiles = (Tile *)p;  // at most as many as 16 x 4 face tiles
  build_update_tiles(c, c->kz, 32);
  if (int r = upload_update_tiles(c)) return r;
  for (int b = 0; b < 2; ++b) {
    if (dev_alloc(c, &c->P[b], E * N * np_of(c))) return CC_ERR_CUDA;
    if (dev_alloc(c, &c->Pr[b], E * N * npr_of(c))) return CC_ERR_CUDA;
    if (dev_alloc(c, &p, sizeof(double) * N * nv_of(c))) return CC_ERR_CUDA;
    c->Q[b] = (double *)p;
  }
  if (dev_alloc(c, &c->G, E * N * 10)) return CC_ERR_CUDA;
  if (dev_alloc(c, &c->faces, E * N * 3 * nv_of(c))) return CC_ERR_CUDA;
  if (dev_alloc(c, &p, sizeof(unsigned))) return CC_ERR_CUDA;
  c->d_ticket = (unsigned *)p;
  if (dev_alloc(c, &p, sizeof(GridBarrier))) return CC_ERR_CUDA;
  c->d_gridbar = (GridBarrier *)p;
  {
    int dev = 0, coop = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    c->halo_coop = coop != 0;
  }
  if (c->precision != CC_FP64) {
    if (dev_alloc(c, &p, sizeof(double) * 3 * N)) return CC_ERR_CUDA;
    c->d_gcl = (double *)p;
  }
  build_edge_tiles(c);
  if (dev_alloc(c, &p, sizeof(Tile) * std::max<size_t>(1, c->hedges.size()))) return CC_ERR_CUDA;
  c->d_edges = (Tile *)p;
  if (!c->hedges.empty())
    CK(cudaMemcpyAsync(c->d_edges, c->hedges.data(), sizeof(Tile) * c->hedges.size(), cudaMemcpyHostToDevice,
                       c->stream));
  {
    const char *no_tma = std::getenv("CC_NO_TMA");
    c->tma_ok = (c->ns_key == 0 || c->ns_key == 9) && !(no_tma && no_tma[0] == '1');
    if (c->tma_ok)
      if (int r = build_tensor_maps(c)) return r;
    c->variant = 0;
  }
  if (dev_alloc(c, &p, sizeof(double) * N * std::max(np_of(c), 10))) return CC_ERR_CUDA;
  c->stage64 = (double *)p;
  if (dev_alloc(c, &p, sizeof(double) * N)) return CC_ERR_CUDA;
  c->tmp64 = (double *)p;
  c->ns_cap = std::max<int64_t>(1, c->plan.n_slots);
  if (dev_alloc(c, &c->sP, E * c->ns_cap * np_of(c))) return CC_ERR_CUDA;
  if (dev_alloc(c, &c->sPr, E * c->ns_cap * npr_of(c))) return CC_ERR_CUDA;
  if (dev_alloc(c, &p, sizeof(double) * c->ns_cap * nv_of(c))) return CC_ERR_CUDA;
  c->sQ = (double *)p;
  if (dev_alloc(c, &p, sizeof(HaloNode) * std::max<size_t>(1, c->plan.nodes.size()))) return CC_ERR_CUDA;
  c->d_nodes = (HaloNode *)p;
  if (dev_alloc(c, &p, sizeof(HaloCopy) * std::max<size_t>(1, c->plan.copies.size()))) return CC_ERR_CUDA;
  c->d_copies = (HaloCopy *)p;
  if (dev_alloc(c, &p, sizeof(uint32_t) * (c->plan.copies.size() / 32 + 1))) return CC_ERR_CUDA;
  c->d_dt_copy_mask = (uint32_t *)p;
  if (dev_alloc(c, &p, sizeof(BcDevice) * std::max<size_t>(1, c->bcs.size()))) return CC_ERR_CUDA;
  c->d_bcs = (BcDevice *)p;
  if (dev_alloc(c, &p, sizeof(double) * 4)) return CC_ERR_CUDA;
  c->d_dt = (double *)p;
  if (dev_alloc(c, &p, sizeof(unsigned long long))) return CC_ERR_CUDA;
  c->d_dt_next = (unsigned long long *)p;
  if (dev_alloc(c, &p, sizeof(unsigned) * 4)) return CC_ERR_CUDA;
  c->d_status = (unsigned *)p;
  c->chem.status = c->d_status;  // bounds-checked builds report there
  if (dev_alloc(c, &p, sizeof(double) * 8)) return CC_ERR_CUDA;  // norms, then their sums of squares
  c->d_res = (double *)p;
  if (dev_alloc(c, &p, sizeof(double) * 4 * c->n_partials)) return CC_ERR_CUDA;
  c->d_partials = (double *)p;
  if (dev_alloc(c, &p, sizeof(double) * 4 * std::max<int64_t>(1, c->n_int))) return CC_ERR_CUDA;
  c->d_last = (double *)p;
  if (dev_alloc(c, &p, sizeof(double) * N)) return CC_ERR_CUDA;
  c->d_vel = (double *)p;
  {
    std::vector<uint32_t> mask((size_t)(N / 32 + 1), 0u);
    for (const auto &cp : c->plan.copies)
      if (cp.src.pad & 1) mask[(size_t)(cp.dst >> 5)] |= 1u << (cp.dst & 31);
    if (dev_alloc(c, &p, sizeof(uint32_t) * mask.size())) return CC_ERR_CUDA;
    c->d_skip_dt = (uint32_t *)p;
    CK(cudaMemcpyAsync(c->d_skip_dt, mask.data(), sizeof(uint32_t) * mask.size(), cudaMemcpyHostToDevice,
                       c->stream));
  }
  if (dev_alloc(c, &p, sizeof(int64_t) * std::max<size_t>(1, c->plan.vel_zero.size()))) return CC_ERR_CUDA;
  c->d_vel_zero = (int64_t *)p;
  if (!c->plan.vel_zero.empty())
    CK(cudaMemcpyAsync(c->d_vel_zero, c->plan.vel_zero.data(), sizeof(int64_t) * c->plan.vel_zero.size(),
                       cudaMemcpyHostToDevice, c->stream));

  CK(cudaMemcpyAsync(c->d_blocks, c->hblocks.data(), sizeof(BlockInfo) * c->hblocks.size(), cudaMemcpyHostToDevice,
                     c->stream));
  if (!c->htiles.empty())
    CK(cudaMemcpyAsync(c->d_tiles, c->htiles.data(), sizeof(Tile) * c->htiles.size(), cudaMemcpyHostToDevice,
                       c->stream));
  if (!c->plan.nodes.empty())
    CK(cudaMemcpyAsync(c->d_nodes, c->plan.nodes.data(), sizeof(HaloNode) * c->plan.nodes.size(),
                       cudaMemcpyHostToDevice, c->stream));
  if (!c->plan.copies.empty())
    CK(cudaMemcpyAsync(c->d_copies, c->plan.copies.data(), sizeof(HaloCopy) * c->plan.copies.size(),
                       cudaMemcpyHostToDevice, c->stream));
  const unsigned long long inf_bits = 0x7ff0000000000000ull;
  CK(cudaMemcpyAsync(c->d_dt_next, &inf_bits, sizeof inf_bits, cudaMemcpyHostToDevice, c->stream));
  if (int r = upload_bcs(c)) return r;
  if (int r = apply_ownership(c)) return r;

  // geometry: user layout -> FP64 staging -> bulk precision
  CK(cudaMemsetAsync(c->stage64, 0, sizeof(double) * N * 10, c->stream));
  for (size_t b = 0; b < c->blocks.size(); ++b)
    if (int r = copy_fields_h2d(c, c->blocks[b], c->h_geo[b].data(), c->stage64, 10)) return r;
  if (int r = from64(c, c->stage64, c->G, N * 10)) return r;
  CK(cudaMemsetAsync(c->stage64, 0, sizeof(double) * N * std::max(np_of(c), 10), c->stream));
  return 0;
}

// Multi-process hooks (cc_set_exchange).  Stage: with the stage's kernels
// done, the hook moves the halo sources between processes (cc_pack_points /
// cc_unpack_points address the buffers recorded here).  Time step: the local
// next time step (the bit pattern the atomicMin reduction keeps) is replaced
// by the hook's minimum over processes.
int exchange_stage(cc_ctx *c, int stage, int pn, int pp, double *qn, double *qp) {
  if (!c->hook) return 0;
  c->x_pn = pn, c->x_pp = pp, c->x_qn = qn, c->x_qp = qp;
  CK(cudaStreamSynchronize(c->stream));
  if (c->hook(c->hook_user, CC_EXCHANGE_STAGE, stage, nullptr) != 0)
    return fail(CC_ERR_STATE, "exchange hook failed at stage " + std::to_string(stage));
  return 0;
}

int exchange_dt(cc_ctx *c) {
  if (!c->hook) return 0;
  unsigned long long bits = 0;
  CK(cudaMemcpyAsync(&bits, c->d_dt_next, sizeof bits, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  double v;
  std::memcpy(&v, &bits, sizeof v);
  if (c->hook(c->hook_user, CC_EXCHANGE_DT, 0, &v) != 0) return fail(CC_ERR_STATE, "exchange hook failed on dt");
  std::memcpy(&bits, &v, sizeof v);
  CK(cudaMemcpyAsync(c->d_dt_next, &bits, sizeof bits, cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));  // bits is a local
  return 0;
}

template <typename T, int NS>
HaloArgs<T> halo_args(cc_ctx *c, int pn, int pp, double *qn, const double *qp) {
  HaloArgs<T> h{};
  h.N = c->N;
  h.NS_cap = c->ns_cap;
  h.P = (T *)c->P[pn];
  h.Pprev = (const T *)c->P[pp];
  h.Pr = (T *)c->Pr[pn];
  h.Prprev = (const T *)c->Pr[pp];
  h.Q = qn;
  h.Qprev = qp;
  h.sP = (T *)c->sP;
  h.sPr = (T *)c->sPr;
  h.sQ = c->sQ;
  h.bcs = c->d_bcs;
  h.nodes = c->d_nodes;
  h.copies = c->d_copies;
  h.dt_copy_mask = c->d_dt_copy_mask;
  return h;
}

// The halo program after a stage: the node levels (one cooperative launch
// with a grid barrier between levels, or, in the per-block launch mode of the
// reference's granularity and for programs of more than kHaloMaxLevels
// levels, one launch per level), then one launch for the copies, the
// post-exchange time step and the zeroing of |V| at wall faces (vel).  Both
// forms run the same device functions: identical results.
template <typename T, int NS>
int run_halo(cc_ctx *c, int pn, int pp, double *qn, const double *qp, unsigned long long *dt_next = nullptr,
             double *vel = nullptr, int q_filter = 0) {
  HaloArgs<T> h = halo_args<T, NS>(c, pn, pp, qn, qp);
  h.G = (const T *)c->G;
  h.dt_next = dt_next;
  const auto &lb = c->plan.level_begin;
  const int n_levels = lb.empty() ? 0 : (int)lb.size() - 1;
  if (n_levels > 0 && !c->per_block && c->halo_coop && n_levels <= kHaloMaxLevels) {
    HaloLevels lv{};
    lv.n = n_levels;
    for (int l = 0; l <= n_levels; ++l) lv.begin[l] = lb[l];
    CK((Launch<T, NS>::halo_levels(h, c->chem, lv, c->d_gridbar, c->d_status, c->stream)));
  } else {
    for (int l = 0; l < n_levels; ++l) {
      h.begin = lb[l], h.end = lb[l + 1];
      CK((Launch<T, NS>::halo_nodes(h, c->chem, c->stream)));
    }
  }
  h.begin = 0, h.end = (int64_t)c->plan.copies.size();
  CK((Launch<T, NS>::halo_copies(h, c->chem, vel, c->d_vel_zero, (int64_t)c->plan.vel_zero.size(), c->stream,
                                 q_filter)));
  return 0;
}

// The conserved state of the ghost points that the steps' halo programs left
// (q_filter 1), from the sources of the last one: the current state and the
// node slots it computed.
template <typename T, int NS>
int refresh_ghost_q(cc_ctx *c) {
  if (!c->q_ghost_stale) return 0;
  HaloArgs<T> h = halo_args<T, NS>(c, c->cur, 1 - c->cur, c->Q[c->qcur], c->Q[1 - c->qcur]);
  h.G = (const T *)c->G;
  h.begin = 0, h.end = (int64_t)c->plan.copies.size();
  CK((Launch<T, NS>::halo_copies(h, c->chem, nullptr, nullptr, 0, c->stream, 2, true)));
  c->q_ghost_stale = false;
  return 0;
}

// Driver::initialize_computation from the FP64 staging arena: conserved
// variables at every point, properties, boundary conditions and interfaces,
// time step.  Afterwards the current state is P[1], Pr[1], Q[0].
template <typename T, int NS>
int derive_state(cc_ctx *c) {
  const int64_t N = c->N;
  c->qcur = 0;
  CK((Launch<T, NS>::configure()));
  CK(cudaMemsetAsync(c->d_gridbar, 0, sizeof(GridBarrier), c->stream));
  CK((Launch<T, NS>::cv_from_bv(c->chem, c->stage64, c->Q[0], N, c->d_vel, c->stream)));
  CK(cudaMemcpyAsync(c->Q[1], c->Q[0], sizeof(double) * N * nv_of(c), cudaMemcpyDeviceToDevice, c->stream));
  if (int r = from64(c, c->stage64, c->P[0], N * np_of(c))) return r;
  if (c->chem.p_ref != 0.0) {  // the pressure field is stored as p - p_ref
    CK(launch_convert_d2f_shift(c->stage64 + 4 * N, (float *)c->P[0] + 4 * N, N, c->chem.p_ref, c->stream));
    CK((Launch<T, NS>::gcl(c->d_blocks, (int)c->hblocks.size(), (const T *)c->G, N, c->n_int, c->d_gcl,
                           c->stream)));
  }
  CK((Launch<T, NS>::props_all(c->chem, (const T *)c->P[0], (T *)c->Pr[0], N, c->stream)));
  CK(cudaMemcpyAsync(c->P[1], c->P[0], c->elem * N * np_of(c), cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(c->Pr[1], c->Pr[0], c->elem * N * npr_of(c), cudaMemcpyDeviceToDevice, c->stream));
  if (int r = run_halo<T, NS>(c, 1, 0, c->Q[0], c->Q[1], nullptr, c->d_vel)) return r;
  c->q_ghost_stale = false;
  c->cur = 1;
  // inflow transport properties: evaluated once by the same point function
  CK((Launch<T, NS>::dt_reduce(c->chem, c->d_blocks_owned, (int)c->hblocks_owned.size(), (const T *)c->P[1],
                               (const T *)c->Pr[1], (const T *)c->G, N, c->n_int_owned, c->d_dt_next, c->stream)));
  if (int r = exchange_dt(c)) return r;
  CK(launch_dt_finalize(c->d_dt, c->d_dt_next, c->d_status, nullptr, c->stream));
  c->state_dirty = false;
  return 0;
}

// Inflow conditions need rho*E and transport properties of their state;
// evaluated on the device through a one-point arena slice of stage64.
template <typename T, int NS>
int prepare_inflow(cc_ctx *c) {
  bool any = false;
  for (const auto &b : c->bcs) any = any || b.kind == 5;
  if (!any) return 0;
  const int ns = c->chem.ns;
  const int np = np_of(c);
  const int64_t M = (int64_t)c->bcs.size();
  // host FP64 primitives [np][M]
  std::vector<double> h((size_t)np * M, 0.0);
  for (int64_t i = 0; i < M; ++i) {
    const HostBc &b = c->bcs[i];
    const double v[6] = {b.rho, b.u, b.v, b.w, b.p, b.T};
    for (int f = 0; f < 6; ++f) h[f * M + i] = b.kind == 5 ? v[f] : 0.0;
    for (int l = 0; l < ns; ++l) h[(6 + l) * M + i] = b.yk[l];
  }
  double *dP = nullptr, *dQ = nullptr;
  void *dPT = nullptr, *dPr = nullptr;
  CK(cudaMalloc(&dP, sizeof(double) * np * M));
  CK(cudaMalloc(&dQ, sizeof(double) * nv_of(c) * M));
  CK(cudaMalloc(&dPT, c->elem * np * M));
  CK(cudaMalloc(&dPr, c->elem * npr_of(c) * M));
  CK(cudaMemcpyAsync(dP, h.data(), sizeof(double) * np * M, cudaMemcpyHostToDevice, c->stream));
  CK((Launch<T, NS>::cv_from_bv(c->chem, dP, dQ, M, nullptr, c->stream)));
  if (int r = from64(c, dP, dPT, np * M)) return r;
  CK((Launch<T, NS>::props_all(c->chem, (const T *)dPT, (T *)dPr, M, c->stream)));
  std::vector<double> q((size_t)nv_of(c) * M);
  std::vector<T> pr((size_t)npr_of(c) * M);
  CK(cudaMemcpyAsync(q.data(), dQ, sizeof(double) * q.size(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(pr.data(), dPr, sizeof(T) * pr.size(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  cudaFree(dP), cudaFree(dQ), cudaFree(dPT), cudaFree(dPr);
  std::vector<BcDevice> hb(M);
  for (int64_t i = 0; i < M; ++i) {
    const HostBc &b = c->bcs[i];
    BcDevice &d = hb[i];
    std::memset(&d, 0, sizeof d);
    d.kind = b.kind, d.thermal_type = b.thermal_type, d.t_wall = b.t_wall;
    d.rho = b.rho, d.u = b.u, d.v = b.v, d.w = b.w, d.p = b.p, d.T = b.T;
    for (int l = 0; l < kMaxSpec; ++l) d.yk[l] = b.yk[l];
    if (b.kind == 5) {
      d.rhoE = q[4 * M + i];
      d.mu = (double)pr[i];
      d.lam = (double)pr[M + i];
      for (int l = 0; l < ns; ++l) d.rho_d[l] = (double)pr[(2 + l) * M + i];
    }
  }
  CK(cudaMemcpyAsync(c->d_bcs, hb.data(), sizeof(BcDevice) * M, cudaMemcpyHostToDevice, c->stream));
  return 0;
}

int prof_event(cc_ctx *c, std::vector<cudaEvent_t> &pool, size_t &next) {
  if (!c->profiling) return 0;
  if (next == pool.size()) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    pool.push_back(e);
  }
  CK(cudaEventRecord(pool[next++], c->stream));
  return 0;
}

const char *const kVariantName[6] = {"fused-l1", "fused-tma", "split", "split-tma", "split-tma-persistent",
                                     "dq-tma"};

// Variants this context can run: the TMA-staged ones need the tensor maps
// (0 or 9 species); the fused TMA kernel's planes and flux planes fit in
// shared memory in the FP32 bulk precision only.
bool variant_ok(const cc_ctx *c, int v) {
  if (v == 3 || v == 4) return c->tma_ok;
  if (v == 1 || v == 5) return c->tma_ok && c->precision != CC_FP64;
  return v == 0 || v == 2;
}

// One stage's kernels of the given variant over the current tile list:
// one launch per kernel over all blocks, or (per_block) one per block.
template <typename T, int NS>
int launch_stage_range(cc_ctx *c, StageArgs<T> a, int pc, int variant, int nt, int n_edge, const Tile *face_tiles,
                       int n_ft, const Tile *upd_tiles, int n_ut);

template <typename T, int NS>
int launch_stage(cc_ctx *c, StageArgs<T> a, int pc, int variant, int nt) {
  if (!c->per_block || c->tile_begin.size() != c->blocks.size() + 1)
    return launch_stage_range<T, NS>(c, a, pc, variant, nt, (int)c->hedges.size(), c->d_ftiles,
                                     (int)c->hftiles.size(), c->d_utiles, (int)c->hutiles.size());
  const Tile *tiles = a.tiles;
  for (size_t b = 0; b < c->blocks.size(); ++b) {
    a.tiles = tiles + c->tile_begin[b];
    a.edge_tiles = c->d_edges + c->edge_begin[b];
    if (int r = launch_stage_range<T, NS>(c, a, pc, variant, c->tile_begin[b + 1] - c->tile_begin[b],
                                          c->edge_begin[b + 1] - c->edge_begin[b], c->d_ftiles + c->ft_begin[b],
                                          c->ft_begin[b + 1] - c->ft_begin[b], c->d_utiles + c->ut_begin[b],
                                          c->ut_begin[b + 1] - c->ut_begin[b]))
      return r;
  }
  return 0;
}

// The update kernel of the split variants over its own tile list.
template <typename T, int NS>
int launch_update(cc_ctx *c, StageArgs<T> a, const Tile *upd_tiles, int n_ut) {
  a.tiles = upd_tiles;
  CK((Launch<T, NS>::update(a, c->chem, n_ut, c->stream, c->update_occ, c->upd_tx)));
  return 0;
}

template <typename T, int NS>
int launch_stage_range(cc_ctx *c, StageArgs<T> a, int pc, int variant, int nt, int n_edge, const Tile *face_tiles,
                       int n_ft, const Tile *upd_tiles, int n_ut) {
  if ((variant == 1 || variant == 3 || variant == 4 || variant == 5) && !c->d_tmaps)
    return fail(CC_ERR_STATE, "TMA variant without tensor maps");
  if (variant == 5) {  // faces differenced in the tile (dq), then the update
    a.faces = (T *)c->faces;
    a.dq_direct = 1;
    const size_t nb = c->blocks.size();
    CK((Launch<T, NS>::faces_dq(a, face_tiles, c->d_tmaps + ((size_t)tma_shape(c->face_ty) * 2 + pc) * nb, c->chem,
                                n_ft, c->face_ty, c->stream)));
    if (int r = prof_event(c, c->ev_mid, c->ev_next_mid)) return r;
    return launch_update<T, NS>(c, a, upd_tiles, n_ut);
  }
  if (variant == 1) {
    CK((Launch<T, NS>::stage_tma(a, c->d_tmaps + (size_t)pc * c->blocks.size(), c->chem, nt, c->stream)));
  } else if (variant == 2 || variant == 3 || variant == 4) {
    a.faces = (T *)c->faces;
    if (!a.edge_tiles) a.edge_tiles = c->d_edges;
    if (variant == 2) {
      CK((Launch<T, NS>::faces(a, c->chem, nt, n_edge, c->stream)));
    } else {  // regular tiles from TMA-staged planes (persistent CTAs for 4), edge tiles through L1
      const CUtensorMap *maps =
          c->d_tmaps + ((size_t)tma_shape(c->face_ty, c->face_tx) * 2 + pc) * c->blocks.size();
      if (variant == 3)
        CK((Launch<T, NS>::faces_tma(a, face_tiles, c->face_ty, c->face_tx, maps, c->chem, n_ft, c->stream)));
      else
        CK((Launch<T, NS>::faces_tma_persistent(a, face_tiles, c->face_ty, c->face_tx, maps, c->chem, n_ft, c->d_ticket,
                                                c->stream)));
      CK((Launch<T, NS>::faces(a, c->chem, 0, n_edge, c->stream)));
    }
    if (int r = prof_event(c, c->ev_mid, c->ev_next_mid)) return r;
    if (int r = launch_update<T, NS>(c, a, upd_tiles, n_ut)) return r;
  } else {
    CK((Launch<T, NS>::stage(a, c->chem, nt, c->stream)));
  }
  return 0;
}

// The closure transport of the new state (when on), the end of the stage's
// timing bracket and the halo program.
template <typename T, int NS>
int after_stage(cc_ctx *c, const StageArgs<T> &a, int pn, int pc, double *qout, const double *qin, int stage = 0) {
  if (c->closure_on) CK((Launch<T, NS>::props_mlp(a.Pn, a.Prn, c->N, &c->cl, c->d_status, c->chem, c->stream)));
  if (int r = prof_event(c, c->ev_stage, c->ev_next_stage)) return r;
  if (int r = exchange_stage(c, stage, pn, pc, qout, const_cast<double *>(qin))) return r;
  if (int r = prof_event(c, c->ev_halo, c->ev_next_halo)) return r;
  if (int r = run_halo<T, NS>(c, pn, pc, qout, qin, a.dt_next, a.vel ? c->d_vel : nullptr, c->hook ? 0 : 1))
    return r;
  if (int r = prof_event(c, c->ev_halo, c->ev_next_halo)) return r;
  return 0;
}

template <typename T, int NS>
int stage_and_halo(cc_ctx *c, const StageArgs<T> &a, int pn, int pc, double *qout, const double *qin,
                   int stage = 0) {
  const int nt = (int)c->htiles.size();
  if (int r = prof_event(c, c->ev_stage, c->ev_next_stage)) return r;
  if (int r = launch_stage<T, NS>(c, a, pc, c->variant, nt)) return r;
  return after_stage<T, NS>(c, a, pn, pc, qout, qin, stage);
}

// LU-SGS steady step (lusgs.cuh): the face fluxes of the current state (the
// split variant's face kernels), the right-hand side and diagonal, the lower
// and upper sweeps one hyperplane per launch, Q += dQ with the primitive
// recovery, then the halo program as after an explicit step.
template <typename T, int NS>
int lusgs_and_halo(cc_ctx *c, StageArgs<T> a, int pn, int pc) {
  const int nt = (int)c->htiles.size(), n_edge = (int)c->hedges.size();
  if (!c->lu.R) return fail(CC_ERR_STATE, "LU-SGS work arrays missing");
  a.faces = (T *)c->faces;
  a.edge_tiles = c->d_edges;
  if (int r = prof_event(c, c->ev_stage, c->ev_next_stage)) return r;
  if (c->tma_ok && c->d_tmaps) {  // the regular 32 x 8 tiles
    CK((Launch<T, NS>::faces_tma(a, c->d_tiles, 8, kTX, c->d_tmaps + (size_t)pc * c->blocks.size(), c->chem, nt,
                                 c->stream)));
    CK((Launch<T, NS>::faces(a, c->chem, 0, n_edge, c->stream)));
  } else {
    CK((Launch<T, NS>::faces(a, c->chem, nt, n_edge, c->stream)));
  }
  if (int r = prof_event(c, c->ev_mid, c->ev_next_mid)) return r;
  LusgsArgs L = c->lu;
  CK((Launch<T, NS>::lusgs_rhs(a, L, c->chem, nt, c->stream)));
  const int H = (int)c->lu_hb.size() - 1;
  for (int h = 0; h < H; ++h) {
    L.s0 = c->lu_hb[h], L.s1 = c->lu_hb[h + 1], L.early = h > 0;
    CK((Launch<T, NS>::lusgs_sweep(L, c->chem, 1, c->stream)));
  }
  for (int h = H - 1; h >= 0; --h) {
    L.s0 = c->lu_hb[h], L.s1 = c->lu_hb[h + 1], L.early = h < H - 1;
    CK((Launch<T, NS>::lusgs_sweep(L, c->chem, -1, c->stream)));
  }
  a.gcl = nullptr;  // the geometric term is part of the right-hand side
  CK((Launch<T, NS>::lusgs_update(a, L, c->chem, nt, c->stream)));
  return after_stage<T, NS>(c, a, pn, pc, c->Q[c->qcur], c->Q[c->qcur]);
}

// Work arrays of the LU-SGS step and its sweep order, built once (outside
// any capture): interior points sorted by hyperplane h = i + j + k, then
// block, k, j; per point the positions of its six neighbours in the block.
int lusgs_alloc(cc_ctx *c) {
  if (c->lu.R) return 0;
  const int64_t N = c->N, S = c->n_int;
  const int lp = lusgs_lanes(nv_of(c));
  if (std::max(3 * lp, (int)kLuScalars) * S >= (int64_t)1 << 31 || N >= (int64_t)1 << 31)
    return fail(CC_ERR_ARG, "LU-SGS: too many points for 32-bit sweep offsets");
  std::vector<int> pos((size_t)N, -1), lo((size_t)(3 * S), -1), hi((size_t)(3 * S), -1);
  std::vector<int64_t> pt((size_t)S);
  int H = 0;
  for (const auto &b : c->blocks) H = std::max(H, b.mx + b.my + b.mz - 2);
  c->lu_hb.assign((size_t)H + 1, 0);
  int64_t sp = 0;
  for (int h = 0; h < H; ++h) {
    c->lu_hb[h] = sp;
    for (size_t bi = 0; bi < c->blocks.size(); ++bi) {
      const HostBlock &b = c->blocks[bi];
      const BlockInfo &B = c->hblocks[bi];
      for (int k = std::max(0, h - (b.mx - 1) - (b.my - 1)); k <= std::min(b.mz - 1, h); ++k)
        for (int j = std::max(0, h - k - (b.mx - 1)); j <= std::min(b.my - 1, h - k); ++j) {
          const int i = h - j - k;
          const int64_t p = B.base + i + (int64_t)B.nx * j + (int64_t)B.nx * B.ny * k;
          pos[(size_t)p] = (int)sp;
          pt[(size_t)sp++] = p;
        }
    }
  }
  c->lu_hb[H] = sp;
  if (sp != S) return fail(CC_ERR_STATE, "LU-SGS: sweep order does not cover the interior");
  for (size_t bi = 0; bi < c->blocks.size(); ++bi) {
    const HostBlock &b = c->blocks[bi];
    const BlockInfo &B = c->hblocks[bi];
    const int64_t st[3] = {1, (int64_t)B.nx, (int64_t)B.nx * B.ny};
    const int m[3] = {b.mx, b.my, b.mz};
    for (int k = 0; k < b.mz; ++k)
      for (int j = 0; j < b.my; ++j)
        for (int i = 0; i < b.mx; ++i) {
          const int64_t p = B.base + i + st[1] * j + st[2] * k;
          const int64_t s = pos[(size_t)p];
          const int id[3] = {i, j, k};
          for (int d = 0; d < 3; ++d) {
            if (id[d] >= 1) lo[(size_t)(d * S + s)] = pos[(size_t)(p - st[d])];
            if (id[d] + 1 < m[d]) hi[(size_t)(d * S + s)] = pos[(size_t)(p + st[d])];
          }
        }
  }
  void *p;
  auto dbl = [&](double **dst, int64_t n) -> int {
    if (dev_alloc(c, &p, sizeof(double) * (size_t)n)) return CC_ERR_CUDA;
    *dst = (double *)p;
    return 0;
  };
  if (dbl(&c->lu.R, lp * S) || dbl(&c->lu.Qs, lp * S) || dbl(&c->lu.pt, kLuScalars * S) ||
      dbl(&c->lu.psi, lp * S) || dbl(&c->lu.Cn, 3 * lp * S))
    return CC_ERR_CUDA;
  int *ip[3];
  const size_t nint[3] = {(size_t)N, (size_t)(3 * S), (size_t)(3 * S)};
  const std::vector<int> *src[3] = {&pos, &lo, &hi};
  for (int q = 0; q < 3; ++q) {
    if (dev_alloc(c, &p, sizeof(int) * nint[q])) return CC_ERR_CUDA;
    ip[q] = (int *)p;
    CK(cudaMemcpyAsync(ip[q], src[q]->data(), sizeof(int) * nint[q], cudaMemcpyHostToDevice, c->stream));
  }
  c->lu.pos = ip[0], c->lu.lo = ip[1], c->lu.hi = ip[2];
  c->lu.S = S, c->lu.lp = lp;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

// Times the stage kernel of each candidate (kernel variant x k-chunk) on the
// actual problem and keeps the fastest.  The candidates write only the
// scratch halves of the ping-pong buffers, so the state is unchanged.
template <typename T, int NS>
int autotune(cc_ctx *c) {
  const char *env = std::getenv("CC_AUTOTUNE");
  if (env && env[0] == '0' && c->force_variant < 0 && c->force_kz <= 0) return 0;
  const char *venv = std::getenv("CC_AUTOTUNE_VERBOSE");  // print every candidate's time to stderr
  const bool verbose = venv && venv[0] == '1';
  StageArgs<T> a{};
  a.blocks = c->d_blocks;
  a.tiles = c->d_tiles;
  a.N = c->N;
  a.G = (const T *)c->G;
  a.dt = c->d_dt;
  a.status = c->d_status;
  a.skip_dt = c->d_skip_dt;
  const int pc = c->cur, pn = 1 - c->cur;
  a.P = (const T *)c->P[pc], a.Pn = (T *)c->P[pn], a.Pr = (const T *)c->Pr[pc], a.Prn = (T *)c->Pr[pn];
  a.Qin = c->Q[c->qcur], a.Qn = c->Q[c->qcur], a.Qout = c->Q[1 - c->qcur];
  a.a = 0.0, a.b = 1.0;
  int max_mz = 1;
  for (const auto &b : c->blocks) max_mz = std::max(max_mz, b.mz);
  std::vector<int> kzs;
  for (int kz : {2, 3, 4, 6, 8, 16, 32, 64, 128})
    if (kz <= max_mz) kzs.push_back(kz);
  kzs.push_back(max_mz);
  kzs.push_back(heuristic_kz(c));
  std::sort(kzs.begin(), kzs.end());
  kzs.erase(std::unique(kzs.begin(), kzs.end()), kzs.end());
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  double best = 1e300;
  int best_kz = c->kz;
  int best_variant = 0;
  int best_ty = c->face_ty, best_tx = c->face_tx;
  if (c->force_kz > 0) kzs.assign(1, c->force_kz);
  std::vector<int> variants;
  if (c->force_variant >= 0 && !variant_ok(c, c->force_variant))
    return fail(CC_ERR_ARG, "the TMA variants need 0 or 9 species, the fused and dq ones also the FP32 bulk "
                            "precision (cc_set_tuning)");
  if (c->force_variant >= 0)
    variants.push_back(c->force_variant);
  else
    for (int v : {0, 1, 2, 3, 4, 5})
      if (variant_ok(c, v)) variants.push_back(v);
  // tile heights of the TMA face kernels (variants 3-5; the other variants'
  // tiles are 32 x 8), those whose plane ring fits in shared memory
  std::vector<int> tys;
  for (int ty : {4, 8, 16})
    if ((c->force_ty <= 0 || ty == c->force_ty) &&
        (Launch<T, NS>::faces_tma_smem(ty, 32) != 0 || Launch<T, NS>::faces_tma_smem(ty, 16) != 0))
      tys.push_back(ty);
  if (tys.empty()) return fail(CC_ERR_ARG, "the face tile height does not fit in shared memory in this precision");
  std::vector<int> occs = c->precision == CC_FP64 ? std::vector<int>{0} : std::vector<int>{0, 1};
  if (const char *oe = std::getenv("CC_UPDATE_OCC"))  // pins it (profiling runs, whose timings are distorted)
    occs.assign(1, c->precision == CC_FP64 ? 0 : (oe[0] == '1' ? 1 : 0));
  int best_occ = 0;
  // tile widths of the TMA face kernels: 32, and 16 (with heights 8 and 16)
  // for variants 3-4, whose narrower tiles waste fewer lanes on blocks whose
  // extent is not a multiple of 32
  auto txs_of = [&](int variant, int ty) {
    std::vector<int> v;
    for (int tx : {32, 16}) {
      if (c->force_tx > 0 && tx != c->force_tx) continue;
      if (tx == 16 && (variant < 3 || variant > 4 || ty == 4)) continue;
      if (Launch<T, NS>::faces_tma_smem(ty, tx) == 0) continue;
      v.push_back(tx);
    }
    if (v.empty() && (variant < 3 || variant > 4)) v.push_back(32);
    return v;
  };
  for (int variant : variants) {
    for (int ty : (variant >= 3 ? tys : std::vector<int>{8})) {
      for (int tx : txs_of(variant, ty)) {
      for (int occ : (variant >= 2 ? occs : std::vector<int>{0})) {
      c->update_occ = occ;
      for (int kz : kzs) {
        build_tiles_kz(c, kz);
        CK(cudaMemcpyAsync(c->d_tiles, c->htiles.data(), sizeof(Tile) * c->htiles.size(), cudaMemcpyHostToDevice,
                           c->stream));
        build_face_tiles(c, ty, kz, tx);
        CK(cudaMemcpyAsync(c->d_ftiles, c->hftiles.data(), sizeof(Tile) * c->hftiles.size(), cudaMemcpyHostToDevice,
                           c->stream));
        build_update_tiles(c, kz, variant == 3 || variant == 4 ? tx : 32);
        if (int r = upload_update_tiles(c)) return r;
        const int nt = (int)c->htiles.size();
        if (int r = launch_stage<T, NS>(c, a, pc, variant, nt)) return r;
        CK(cudaEventRecord(e0, c->stream));
        for (int r = 0; r < 3; ++r)
          if (int rr = launch_stage<T, NS>(c, a, pc, variant, nt)) return rr;
        CK(cudaEventRecord(e1, c->stream));
        CK(cudaEventSynchronize(e1));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        if (verbose)
          std::fprintf(stderr, "cc autotune: %s tile %dx%dx%d update-occ %d tiles=%d %.4f ms\n",
                       kVariantName[variant], variant >= 3 ? tx : kTX, variant >= 3 ? ty : kTY, kz, occ,
                       variant >= 3 ? (int)c->hftiles.size() : nt, ms / 3);
        if (ms / 3 < best)
          best = ms / 3, best_kz = kz, best_variant = variant, best_ty = ty, best_tx = tx, best_occ = occ;
      }
      }
      }
    }
  }
  c->update_occ = best_occ;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (best == 1e300) return fail(CC_ERR_ARG, "the face tile does not fit in shared memory in this precision");
  build_tiles_kz(c, best_kz);
  CK(cudaMemcpyAsync(c->d_tiles, c->htiles.data(), sizeof(Tile) * c->htiles.size(), cudaMemcpyHostToDevice,
                     c->stream));
  build_face_tiles(c, best_variant >= 3 ? best_ty : 8, best_kz, best_variant >= 3 ? best_tx : 32);
  CK(cudaMemcpyAsync(c->d_ftiles, c->hftiles.data(), sizeof(Tile) * c->hftiles.size(), cudaMemcpyHostToDevice,
                     c->stream));
  build_update_tiles(c, best_kz, best_variant == 3 || best_variant == 4 ? best_tx : 32);
  if (int r = upload_update_tiles(c)) return r;
  c->variant = best_variant;
  c->tuned_ms = best;
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(unsigned), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

template <typename T, int NS>
int enqueue_step(cc_ctx *c, int scheme) {
  StageArgs<T> a{};
  a.blocks = c->d_blocks;
  a.tiles = c->d_tiles;
  a.N = c->N;
  a.G = (const T *)c->G;
  a.dt = c->d_dt;
  a.status = c->d_status;
  a.skip_dt = c->d_skip_dt;
  a.renorm_y = c->chem.ns > 0 && (c->renorm < 0 ? c->precision != CC_FP64 : c->renorm != 0);
  a.q32 = c->precision == CC_FP32;
  a.closure = c->closure_on ? 1 : 0;
  a.gcl = c->chem.p_ref != 0.0 ? c->d_gcl : nullptr;
  const bool dt_after = c->plan.has_wall || c->closure_on;  // global dt reduced after the halo
  if (scheme == CC_STEADY_EULER) {
    const int pc = c->cur, pn = 1 - c->cur;
    a.P = (const T *)c->P[pc], a.Pn = (T *)c->P[pn], a.Pr = (const T *)c->Pr[pc], a.Prn = (T *)c->Pr[pn];
    a.Qin = c->Q[c->qcur], a.Qn = nullptr, a.Qout = c->Q[c->qcur];
    a.a = 0.0, a.b = 1.0, a.local_dt = 1, a.dt_next = nullptr, a.vel = c->d_vel;
    if (int r = stage_and_halo<T, NS>(c, a, pn, pc, c->Q[c->qcur], c->Q[c->qcur])) return r;
    c->cur = pn;
    return 0;
  }
  if (scheme == CC_STEADY_LUSGS) {
    const int pc = c->cur, pn = 1 - c->cur;
    a.P = (const T *)c->P[pc], a.Pn = (T *)c->P[pn], a.Pr = (const T *)c->Pr[pc], a.Prn = (T *)c->Pr[pn];
    a.Qin = c->Q[c->qcur], a.Qn = nullptr, a.Qout = c->Q[c->qcur];
    a.a = 0.0, a.b = 1.0, a.local_dt = 1, a.dt_next = nullptr, a.vel = c->d_vel;
    if (int r = lusgs_and_halo<T, NS>(c, a, pn, pc)) return r;
    c->cur = pn;
    return 0;
  }
  static const double A[3] = {0.0, 0.75, 1.0 / 3.0};
  static const double Bc[3] = {1.0, 0.25, 2.0 / 3.0};
  double *qa = c->Q[c->qcur], *qb = c->Q[1 - c->qcur];
  for (int st = 0; st < 3; ++st) {
    const int pc = c->cur, pn = 1 - c->cur;
    a.P = (const T *)c->P[pc], a.Pn = (T *)c->P[pn], a.Pr = (const T *)c->Pr[pc], a.Prn = (T *)c->Pr[pn];
    const double *qin = st == 0 ? qa : qb;
    double *qout = st == 2 ? qa : qb;
    a.Qin = qin, a.Qn = qa, a.Qout = qout;
    a.a = A[st], a.b = Bc[st], a.local_dt = 0;
    a.dt_next = (st == 2 && !dt_after) ? c->d_dt_next : nullptr;
    a.vel = st == 2 ? c->d_vel : nullptr;
    if (int r = stage_and_halo<T, NS>(c, a, pn, pc, qout, qin, st)) return r;
    c->cur = pn;
  }
  if (dt_after)
    CK((Launch<T, NS>::dt_reduce(c->chem, c->d_blocks_owned, (int)c->hblocks_owned.size(),
                                 (const T *)c->P[c->cur], (const T *)c->Pr[c->cur], (const T *)c->G, c->N,
                                 c->n_int_owned, c->d_dt_next,
                                 c->stream)));
  if (int r = exchange_dt(c)) return r;  // minimum over processes (multi-process runs)
  CK(launch_dt_finalize(c->d_dt, c->d_dt_next, c->d_status, c->d_dt + 1, c->stream));
  return 0;
}

void destroy_graphs(cc_ctx *c) {
  for (auto &row : c->graph)
    for (auto &g : row)
      if (g) cudaGraphExecDestroy(g), g = nullptr;
}

template <typename T, int NS>
int step_once(cc_ctx *c, int scheme) {
  c->q_ghost_stale = !c->hook;  // with a hook every halo copy runs
  if (!c->use_graph || c->hook) return enqueue_step<T, NS>(c, scheme);  // the hook runs on the host between launches
  cudaGraphExec_t &ge = c->graph[scheme][c->cur];
  if (!ge) {
    const int cur0 = c->cur;
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int r = enqueue_step<T, NS>(c, scheme);
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    c->cur = cur0;
    if (r) return r;
    if (e != cudaSuccess) return fail(CC_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(CC_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  }
  CK(cudaGraphLaunch(ge, c->stream));
  c->cur = (scheme == CC_RK3) ? 1 - c->cur : 1 - c->cur;  // 3 or 1 buffer swaps: odd either way
  return 0;
}

int validate_params(const cc_params *p) {
  if (!p) return fail(CC_ERR_ARG, "params is null");
  if (p->n_spec < 0 || p->n_spec > CC_MAX_SPECIES) return fail(CC_ERR_ARG, "n_spec out of range [0,16]");
  if (p->ngg != 2) return fail(CC_ERR_ARG, "only ngg = 2 is supported (MUSCL/AUSM+ and 2nd-order viscous)");
  if (p->inviscid_scheme != 3) return fail(CC_ERR_ARG, "only inviscid_scheme 3 (AUSM+) exists in the reference");
  if (p->viscous_order != 0 && p->viscous_order != 2) return fail(CC_ERR_ARG, "viscous_order must be 0 or 2");
  if (p->limiter != 0 && p->limiter != 1) return fail(CC_ERR_ARG, "limiter must be 0 or 1 (minmod)");
  if (!(p->cfl > 0) || !(p->prandtl_number > 0)) return fail(CC_ERR_ARG, "cfl and prandtl_number must be positive");
  if (p->n_spec > 0) {
    if (!p->mw || !p->t_low || !p->t_mid || !p->low_temp_coeff || !p->high_temp_coeff || !p->LJ_potent_inv ||
        !p->vis_coeff || !p->WjDivWi_to_One4th || !p->sqrt_WiDivWjPl1Mul8)
      return fail(CC_ERR_ARG, "species tables missing");
    if (!(p->schmidt_number > 0)) return fail(CC_ERR_ARG, "schmidt_number must be positive");
  }
  return 0;
}

int check_ctx(cc_ctx *c) { return c ? 0 : fail(CC_ERR_ARG, "context is null"); }

// The staging buffers of cc_pack_points / cc_unpack_points, grown to n points
// (host-side exchange calls between launches, outside any capture).
int exchange_staging(cc_ctx *c, int64_t n) {
  if (n <= c->x_cap) return 0;
  const int nf = np_of(c) + npr_of(c) + nv_of(c);
  if (c->d_xbuf) cudaFree(c->d_xbuf), c->d_xbuf = nullptr;
  if (c->d_xidx) cudaFree(c->d_xidx), c->d_xidx = nullptr;
  c->x_cap = 0;
  CK(cudaMalloc((void **)&c->d_xbuf, sizeof(double) * (size_t)(nf * n)));
  CK(cudaMalloc((void **)&c->d_xidx, sizeof(int64_t) * (size_t)n));
  c->x_cap = n;
  return 0;
}

// cc_pack_points / cc_unpack_points: all fields of the listed points of the
// state the halo program reads as current (which 0) or previous (which 1),
// between the device arenas and [n_fields][n] FP64 host rows.
int pack_unpack(cc_ctx *c, int which, const int64_t *idx, int64_t n, double *host, bool pack) {
  if (int r = check_ctx(c)) return r;
  if (!c->initialized) return fail(CC_ERR_STATE, "cc_pack_points / cc_unpack_points before cc_init");
  if (which != 0 && which != 1) return fail(CC_ERR_ARG, "which must be 0 (current) or 1 (previous)");
  if (n < 0 || (n > 0 && (!idx || !host))) return fail(CC_ERR_ARG, "null index or value array");
  if (n == 0) return 0;
  for (int64_t i = 0; i < n; ++i)
    if (idx[i] < 0 || idx[i] >= c->N) return fail(CC_ERR_ARG, "point index outside the arena");
  double *Q = which == 0 ? c->x_qn : c->x_qp;
  if (!Q) return fail(CC_ERR_STATE, "cc_pack_points / cc_unpack_points outside an exchange hook call");
  if (int r = exchange_staging(c, n)) return r;
  const int np = np_of(c), npr = npr_of(c), nv = nv_of(c), nf = np + npr + nv;
  void *P = c->P[which == 0 ? c->x_pn : c->x_pp], *Pr = c->Pr[which == 0 ? c->x_pn : c->x_pp];
  CK(cudaMemcpyAsync(c->d_xidx, idx, sizeof(int64_t) * (size_t)n, cudaMemcpyHostToDevice, c->stream));
  double *bP = c->d_xbuf, *bPr = bP + (size_t)np * n, *bQ = bPr + (size_t)npr * n;
  const bool f32 = c->elem == 4;
  if (pack) {
    CK(f32 ? launch_gather_points<float>((const float *)P, c->N, np, c->d_xidx, n, bP, c->stream)
           : launch_gather_points<double>((const double *)P, c->N, np, c->d_xidx, n, bP, c->stream));
    CK(f32 ? launch_gather_points<float>((const float *)Pr, c->N, npr, c->d_xidx, n, bPr, c->stream)
           : launch_gather_points<double>((const double *)Pr, c->N, npr, c->d_xidx, n, bPr, c->stream));
    CK(launch_gather_points<double>(Q, c->N, nv, c->d_xidx, n, bQ, c->stream));
    CK(cudaMemcpyAsync(host, c->d_xbuf, sizeof(double) * (size_t)(nf * n), cudaMemcpyDeviceToHost, c->stream));
  } else {
    CK(cudaMemcpyAsync(c->d_xbuf, host, sizeof(double) * (size_t)(nf * n), cudaMemcpyHostToDevice, c->stream));
    CK(f32 ? launch_scatter_points<float>((float *)P, c->N, np, c->d_xidx, n, bP, c->stream)
           : launch_scatter_points<double>((double *)P, c->N, np, c->d_xidx, n, bP, c->stream));
    CK(f32 ? launch_scatter_points<float>((float *)Pr, c->N, npr, c->d_xidx, n, bPr, c->stream)
           : launch_scatter_points<double>((double *)Pr, c->N, npr, c->d_xidx, n, bPr, c->stream));
    CK(launch_scatter_points<double>(Q, c->N, nv, c->d_xidx, n, bQ, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

}  // namespace

extern "C" {

const char *cc_last_error(void) { return g_err.c_str(); }

int cc_version(void) { return 10000; }

int cc_device_count(int *n) {
  if (!n) return fail(CC_ERR_ARG, "n is null");
  int k = 0;
  cudaError_t e = cudaGetDeviceCount(&k);
  if (e != cudaSuccess) k = 0, cudaGetLastError();
  *n = k;
  return 0;
}

int cc_create(const cc_params *params, cc_ctx **out) {
  if (!out) return fail(CC_ERR_ARG, "out is null");
  *out = nullptr;
  if (int r = validate_params(params)) return r;
  cc_ctx *c = new cc_ctx;
  c->ngg = params->ngg;
  c->chem.ns = params->n_spec;
  c->chem.nv = 5 + params->n_spec;
  c->chem.reconstruction = params->reconstruction;
  c->chem.viscous = params->viscous_order == 2 ? 1 : 0;
  c->chem.Pr = params->prandtl_number;
  c->chem.cfl = params->cfl;
  c->chem.Sc = params->n_spec > 0 ? params->schmidt_number : 1.0;
  c->chem.p_ref = 0.0;  // set at the first cc_init for the FP32 bulk precisions
  c->chem.max_spins = kDefaultWaitSpins;
  c->chem.newton_max_iter = 1000;
  fill_tables(c->chem.d, params);
  fill_tables(c->chem.f, params);
  *out = c;
  return 0;
}

int cc_destroy(cc_ctx *c) {
  if (!c) return 0;
  if (c->stream) cudaStreamSynchronize(c->stream);
  destroy_graphs(c);
  for (auto e : c->ev_stage) cudaEventDestroy(e);
  for (auto e : c->ev_halo) cudaEventDestroy(e);
  for (auto e : c->ev_mid) cudaEventDestroy(e);
  for (void *p : c->allocs) cudaFree(p);
  if (c->d_xbuf) cudaFree(c->d_xbuf);
  if (c->d_xidx) cudaFree(c->d_xidx);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return 0;
}

int cc_add_block(cc_ctx *c, int mx, int my, int mz, const double *jac, const double *metric, int *block_id) {
  if (int r = check_ctx(c)) return r;
  if (c->initialized) return fail(CC_ERR_STATE, "blocks must be added before cc_init");
  if (mx < 1 || my < 1 || mz < 1) return fail(CC_ERR_ARG, "block extents must be positive");
  if (!jac || !metric) return fail(CC_ERR_ARG, "jac and metric are required");
  HostBlock b{};
  b.mx = mx, b.my = my, b.mz = mz, b.g = c->ngg;
  const int64_t ng = ng_user(b);
  std::vector<double> geo((size_t)ng * 10);
  std::memcpy(geo.data(), jac, sizeof(double) * ng);
  std::memcpy(geo.data() + ng, metric, sizeof(double) * ng * 9);
  c->blocks.push_back(b);
  c->h_geo.push_back(std::move(geo));
  c->pend_bv.emplace_back();
  c->pend_yk.emplace_back();
  c->pend.push_back(0);
  if (block_id) *block_id = (int)c->blocks.size() - 1;
  return 0;
}

int cc_register_boundary(const int raw[7], int ngg, cc_boundary *out) {
  if (!raw || !out) return fail(CC_ERR_ARG, "null argument");
  HostBoundary b;
  register_boundary(raw, ngg, b);
  static_assert(sizeof(HostBoundary) == sizeof(cc_boundary), "layout");
  std::memcpy(out, &b, sizeof b);
  return 0;
}

int cc_register_inner_face(const int raw[13], int ngg, cc_inner_face *out) {
  if (!raw || !out) return fail(CC_ERR_ARG, "null argument");
  HostInnerFace f;
  register_inner_face(raw, ngg, f);
  static_assert(sizeof(HostInnerFace) == sizeof(cc_inner_face), "layout");
  std::memcpy(out, &f, sizeof f);
  return 0;
}

int cc_add_boundary(cc_ctx *c, int block, const cc_boundary *b) {
  if (int r = check_ctx(c)) return r;
  if (c->initialized) return fail(CC_ERR_STATE, "faces must be added before cc_init");
  if (!b || block < 0 || block >= (int)c->blocks.size()) return fail(CC_ERR_ARG, "bad block or boundary");
  if (b->face < 0 || b->face > 2) return fail(CC_ERR_ARG, "boundary face must be 0, 1 or 2");
  HostBoundary h;
  std::memcpy(&h, b, sizeof h);
  c->blocks[block].bnd.push_back(h);
  return 0;
}

int cc_add_inner_face(cc_ctx *c, int block, const cc_inner_face *f) {
  if (int r = check_ctx(c)) return r;
  if (c->initialized) return fail(CC_ERR_STATE, "faces must be added before cc_init");
  if (!f || block < 0 || block >= (int)c->blocks.size()) return fail(CC_ERR_ARG, "bad block or inner face");
  if (f->face < 0 || f->face > 2) return fail(CC_ERR_ARG, "inner face normal must be 0, 1 or 2");
  HostInnerFace h;
  std::memcpy(&h, f, sizeof h);
  c->blocks[block].inf.push_back(h);
  return 0;
}

int cc_add_bc(cc_ctx *c, const cc_bc *bc) {
  if (int r = check_ctx(c)) return r;
  if (c->initialized) return fail(CC_ERR_STATE, "conditions must be added before cc_init");
  if (!bc || (bc->kind != 2 && bc->kind != 5 && bc->kind != 6))
    return fail(CC_ERR_ARG, "bc kind must be 2 (wall), 5 (inflow) or 6 (outflow)");
  HostBc h{};
  h.label = bc->label, h.kind = bc->kind, h.thermal_type = bc->thermal_type, h.t_wall = bc->t_wall;
  h.rho = bc->density, h.u = bc->u, h.v = bc->v, h.w = bc->w, h.p = bc->pressure, h.T = bc->temperature;
  for (int l = 0; l < kMaxSpec; ++l) h.yk[l] = bc->yk[l];
  c->bcs.push_back(h);
  // BoundCond.cu:218-230: wall faces exclude the tangential ghost layers
  if (bc->kind == 2)
    for (auto &b : c->blocks)
      for (auto &f : b.bnd)
        if (f.type_label == bc->label)
          for (int q = 0; q < 3; ++q)
            if (q != f.face) f.range_start[q] += c->ngg, f.range_end[q] -= c->ngg;
  return 0;
}

int cc_set_state(cc_ctx *c, int block, const double *bv, const double *yk, int layout) {
  if (int r = check_ctx(c)) return r;
  if (block < 0 || block >= (int)c->blocks.size()) return fail(CC_ERR_ARG, "bad block");
  if (!bv || (c->chem.ns > 0 && !yk)) return fail(CC_ERR_ARG, "bv (and yk when n_spec > 0) required");
  if (layout != CC_LAYOUT_FIELD_MAJOR && layout != CC_LAYOUT_POINT_MAJOR)
    return fail(CC_ERR_ARG, "layout must be CC_LAYOUT_FIELD_MAJOR or CC_LAYOUT_POINT_MAJOR");
  const HostBlock &b = c->blocks[block];
  const int64_t ng = ng_user(b);
  std::vector<double> bv_fm, yk_fm;  // field-major copies of point-major input
  if (layout == CC_LAYOUT_POINT_MAJOR) {
    transpose_fields(bv, ng, 6, bv_fm, true);
    bv = bv_fm.data();
    if (c->chem.ns > 0) {
      transpose_fields(yk, ng, c->chem.ns, yk_fm, true);
      yk = yk_fm.data();
    }
  }
  if (!c->initialized) {
    c->pend_bv[block].assign(bv, bv + 6 * ng);
    if (c->chem.ns > 0) c->pend_yk[block].assign(yk, yk + c->chem.ns * ng);
    c->pend[block] = 1;
    return 0;
  }
  if (int r = copy_fields_h2d(c, b, bv, c->stage64, 6)) return r;
  if (c->chem.ns > 0)
    if (int r = copy_fields_h2d(c, b, yk, c->stage64 + 6 * c->N, c->chem.ns)) return r;
  c->state_dirty = true;
  return 0;
}

int cc_init(cc_ctx *c, int precision) {
  if (int r = check_ctx(c)) return r;
  if (precision != CC_FP64 && precision != CC_MIXED && precision != CC_FP32)
    return fail(CC_ERR_ARG, "precision must be CC_FP64, CC_MIXED or CC_FP32");
  if (c->blocks.empty()) return fail(CC_ERR_STATE, "no blocks");
  const bool first_init = !c->initialized;
  if (!c->initialized) {
    for (size_t b = 0; b < c->blocks.size(); ++b)
      if (!c->pend[b]) return fail(CC_ERR_STATE, "block " + std::to_string(b) + " has no state (cc_set_state)");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      return fail(CC_ERR_NODEVICE, "no CUDA device");
    }
    if (!c->stream) {
      CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
      c->own_stream = true;
    }
    c->precision = precision;
    // gauge pressure reference of the FP32 primitives: the mean initial
    // pressure of the first block, representable in FP32 (0 for FP64)
    c->chem.p_ref = 0.0;
    if (precision != CC_FP64) {
      const std::vector<double> &bv = c->pend_bv[0];
      const size_t ng = bv.size() / 6;
      double sum = 0;
      for (size_t i = 0; i < ng; ++i) sum += bv[4 * ng + i];
      c->chem.p_ref = (double)(float)(sum / (double)std::max<size_t>(1, ng));
    }
    if (int r = setup_device(c)) return r;
    for (size_t b = 0; b < c->blocks.size(); ++b) {
      if (int r = copy_fields_h2d(c, c->blocks[b], c->pend_bv[b].data(), c->stage64, 6)) return r;
      if (c->chem.ns > 0)
        if (int r = copy_fields_h2d(c, c->blocks[b], c->pend_yk[b].data(), c->stage64 + 6 * c->N, c->chem.ns))
          return r;
    }
    c->initialized = true;
    int r = dispatch(c, [&](auto tt, auto nn) { return prepare_inflow<typename decltype(tt)::type, decltype(nn)::value>(c); });
    if (r) return r;
    CK(cudaStreamSynchronize(c->stream));
    for (auto &v : c->pend_bv) std::vector<double>().swap(v);
    for (auto &v : c->pend_yk) std::vector<double>().swap(v);
  } else if (precision != c->precision) {
    return fail(CC_ERR_STATE, "a context keeps the precision of its first cc_init");
  }
  destroy_graphs(c);
  int r = dispatch(c, [&](auto tt, auto nn) { return derive_state<typename decltype(tt)::type, decltype(nn)::value>(c); });
  if (r) return r;
  if (first_init) {
    r = dispatch(c, [&](auto tt, auto nn) { return autotune<typename decltype(tt)::type, decltype(nn)::value>(c); });
    if (r) return r;
  }
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int cc_step(cc_ctx *c, int n_steps, int scheme, int want_residual) {
  if (int r = check_ctx(c)) return r;
  if (!c->initialized) return fail(CC_ERR_STATE, "cc_step before cc_init");
  if (scheme != CC_RK3 && scheme != CC_STEADY_EULER && scheme != CC_STEADY_LUSGS)
    return fail(CC_ERR_ARG, "unknown time scheme");
  if (n_steps < 0) return fail(CC_ERR_ARG, "n_steps must be >= 0");
  if (scheme == CC_STEADY_LUSGS && (c->hook || !c->owned.empty()))
    return fail(CC_ERR_STATE, "the LU-SGS step sweeps every block in one order: not available in multi-process runs");
  if (scheme == CC_STEADY_LUSGS)
    if (int r = lusgs_alloc(c)) return r;
  if (c->state_dirty) {
    destroy_graphs(c);
    int r = dispatch(c, [&](auto tt, auto nn) { return derive_state<typename decltype(tt)::type, decltype(nn)::value>(c); });
    if (r) return r;
  }
  return dispatch(c, [&](auto tt, auto nn) -> int {
    using T = typename decltype(tt)::type;
    constexpr int NS = decltype(nn)::value;
    for (int s = 0; s < n_steps; ++s) {
      if (want_residual && s == n_steps - 1)
        CK(launch_store_last<T>(c->d_blocks_owned, (int)c->hblocks_owned.size(), (const T *)c->P[c->cur],
                                c->d_vel, c->N, c->n_int_owned, c->d_last, c->stream));
      if (int r = step_once<T, NS>(c, scheme)) return r;
    }
    if (want_residual && n_steps > 0)
      CK(launch_residual<T>(c->d_blocks_owned, (int)c->hblocks_owned.size(), (const T *)c->P[c->cur], c->d_vel,
                            c->N, c->n_int_owned, c->d_last, c->d_partials, c->n_partials, c->d_res, c->stream));
    return 0;
  });
}

int cc_residual(cc_ctx *c, double out[4]) {
  if (int r = check_ctx(c)) return r;
  if (!c->initialized) return fail(CC_ERR_STATE, "cc_residual before cc_init");
  if (!out) return fail(CC_ERR_ARG, "out is null");
  CK(cudaMemcpyAsync(out, c->d_res, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int cc_residual_async(cc_ctx *c, double *out) {
  if (int r = check_ctx(c)) return r;
  if (!c->initialized) return fail(CC_ERR_STATE, "cc_residual_async before cc_init");
  if (!out) return fail(CC_ERR_ARG, "out is null");
  CK(cudaMemcpyAsync(out, c->d_res, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  return 0;
}

int cc_get_state(cc_ctx *c, int block, double *bv, double *yk, double *cv, int layout) {
  if (int r = check_ctx(c)) return r;
  if (!c->initialized) return fail(CC_ERR_STATE, "cc_get_state before cc_init");
  if (block < 0 || block >= (int)c->blocks.size()) return fail(CC_ERR_ARG, "bad block");
  if (layout != CC_LAYOUT_FIELD_MAJOR && layout != CC_LAYOUT_POINT_MAJOR)
    return fail(CC_ERR_ARG, "layout must be CC_LAYOUT_FIELD_MAJOR or CC_LAYOUT_POINT_MAJOR");
  if (layout == CC_LAYOUT_POINT_MAJOR) {  // field-major into scratch, then transposed
    const int64_t ng = ng_user(c->blocks[block]);
    const int ns = c->chem.ns, nv = nv_of(c);
    std::vector<double> fb(bv ? 6 * ng : 0), fy(yk && ns ? ns * ng : 0), fc(cv ? nv * ng : 0);
    if (int r = cc_get_state(c, block, bv ? fb.data() : nullptr, yk && ns ? fy.data() : nullptr,
                             cv ? fc.data() : nullptr, CC_LAYOUT_FIELD_MAJOR))
      return r;
    std::vector<double> t;
    if (bv) transpose_fields(fb.data(), ng, 6, t, false), std::copy(t.begin(), t.end(), bv);
    if (yk && ns) transpose_fields(fy.data(), ng, ns, t, false), std::copy(t.begin(), t.end(), yk);
    if (cv) transpose_fields(fc.data(), ng, nv, t, false), std::copy(t.begin(), t.end(), cv);
    return 0;
  }
  if (c->state_dirty) {
    destroy_graphs(c);
    int r = dispatch(c, [&](auto tt, auto nn) { return derive_state<typename decltype(tt)::type, decltype(nn)::value>(c); });
    if (r) return r;
  }
  const HostBlock &b = c->blocks[block];
  const int64_t ng = ng_user(b);
  for (int f = 0; f < 6 && bv; ++f) {
    if (int r = field_to64(c, c->P[c->cur], f, f == 4 ? c->chem.p_ref : 0.0)) return r;  // gauge pressure
    if (int r = copy_field_d2h(c, b, c->tmp64, bv + f * ng)) return r;
  }
  for (int l = 0; l < c->chem.ns && yk; ++l) {
    if (int r = field_to64(c, c->P[c->cur], 6 + l)) return r;
    if (int r = copy_field_d2h(c, b, c->tmp64, yk + l * ng)) return r;
  }
  if (cv && c->q_ghost_stale)
    if (int r = dispatch(c, [&](auto tt, auto nn) { return refresh_ghost_q<typename decltype(tt)::type, decltype(nn)::value>(c); }))
      return r;
  for (int f = 0; f < nv_of(c) && cv; ++f)
    if (int r = copy_field_d2h(c, b, c->Q[c->qcur] + (int64_t)f * c->N, cv + f * ng)) return r;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int cc_get_props(cc_ctx *c, int block, double *mul, double *conductivity, double *rho_d) {
  if (int r = check_ctx(c)) return r;
  if (!c->initialized) return fail(CC_ERR_STATE, "cc_get_props before cc_init");
  if (block < 0 || block >= (int)c->blocks.size()) return fail(CC_ERR_ARG, "bad block");
  const HostBlock &b = c->blocks[block];
  const int64_t ng = ng_user(b);
  double *outs[2] = {mul, conductivity};
  for (int f = 0; f < 2; ++f) {
    if (!outs[f]) continue;
    if (int r = field_to64(c, c->Pr[c->cur], f)) return r;
    if (int r = copy_field_d2h(c, b, c->tmp64, outs[f])) return r;
  }
  for (int l = 0; l < c->chem.ns && rho_d; ++l) {
    if (int r = field_to64(c, c->Pr[c->cur], 2 + l)) return r;
    if (int r = copy_field_d2h(c, b, c->tmp64, rho_d + l * ng)) return r;
  }
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int cc_last_dt(cc_ctx *c, double *dt) {
  if (int r = check_ctx(c)) return r;
  if (!c->initialized || !dt) return fail(CC_ERR_STATE, "cc_last_dt before cc_init");
  double h[2];
  CK(cudaMemcpyAsync(h, c->d_dt, sizeof h, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *dt = h[1];
  return 0;
}

int cc_status(cc_ctx *c, unsigned *flags) {
  if (int r = check_ctx(c)) return r;
  if (!flags) return fail(CC_ERR_ARG, "flags is null");
  if (!c->initialized) {
    *flags = 0;
    return 0;
  }
  CK(cudaMemcpyAsync(flags, c->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(unsigned), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  // a grid barrier that gave up leaves its arrival count behind: reset it
  if ((*flags & kStatusHaloTimeout) && c->d_gridbar) {
    CK(cudaMemsetAsync(c->d_gridbar, 0, sizeof(GridBarrier), c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  return 0;
}

int cc_set_stream(cc_ctx *c, void *stream) {
  if (int r = check_ctx(c)) return r;
  if (c->stream) cudaStreamSynchronize(c->stream);
  destroy_graphs(c);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  c->stream = (cudaStream_t)stream;
  c->own_stream = false;
  return 0;
}

void *cc_get_stream(cc_ctx *c) { return c ? (void *)c->stream : nullptr; }

int cc_set_renormalize(cc_ctx *c, int enable) {
  if (int r = check_ctx(c)) return r;
  c->renorm = enable < 0 ? -1 : (enable != 0);
  destroy_graphs(c);
  return 0;
}

int cc_set_wait_limit(cc_ctx *c, int64_t spins) {
  if (int r = check_ctx(c)) return r;
  c->chem.max_spins = spins >= 0 ? (long long)spins : kDefaultWaitSpins;
  destroy_graphs(c);  // the captured launches carry the parameters by value
  return 0;
}

int cc_set_newton_max_iter(cc_ctx *c, int n) {
  if (int r = check_ctx(c)) return r;
  c->chem.newton_max_iter = n > 0 ? n : 1000;
  destroy_graphs(c);
  return 0;
}

int cc_use_graph(cc_ctx *c, int enable) {
  if (int r = check_ctx(c)) return r;
  c->use_graph = enable != 0;
  return 0;
}

int cc_info(cc_ctx *c, int64_t *n_points, int64_t *device_bytes, int *n_tiles, int *n_halo_levels) {
  if (int r = check_ctx(c)) return r;
  int64_t n = 0;
  for (const auto &b : c->blocks) n += (int64_t)b.mx * b.my * b.mz;
  if (n_points) *n_points = n;
  if (device_bytes) *device_bytes = c->device_bytes;
  if (n_tiles) *n_tiles = (int)c->htiles.size();
  if (n_halo_levels) *n_halo_levels = (int)c->plan.level_begin.size() - 1;
  return 0;
}

int cc_time_kernels(cc_ctx *c, int n_steps, int scheme, double out_ms[6]) {
  if (int r = check_ctx(c)) return r;
  if (!c->initialized) return fail(CC_ERR_STATE, "cc_time_kernels before cc_init");
  if (!out_ms || n_steps < 1) return fail(CC_ERR_ARG, "bad arguments");
  if (scheme != CC_RK3 && scheme != CC_STEADY_EULER && scheme != CC_STEADY_LUSGS)
    return fail(CC_ERR_ARG, "unknown time scheme");
  if (scheme == CC_STEADY_LUSGS)
    if (int r = lusgs_alloc(c)) return r;
  if (c->state_dirty) {
    destroy_graphs(c);
    int r = dispatch(c, [&](auto tt, auto nn) { return derive_state<typename decltype(tt)::type, decltype(nn)::value>(c); });
    if (r) return r;
  }
  c->profiling = true;
  c->ev_next_stage = c->ev_next_halo = c->ev_next_mid = 0;
  int r = dispatch(c, [&](auto tt, auto nn) -> int {
    for (int s = 0; s < n_steps; ++s) {
      c->q_ghost_stale = !c->hook;
      if (int e = enqueue_step<typename decltype(tt)::type, decltype(nn)::value>(c, scheme)) return e;
    }
    return 0;
  });
  c->profiling = false;
  if (r) return r;
  CK(cudaStreamSynchronize(c->stream));
  double st = 0, ha = 0;
  for (size_t i = 0; i + 1 < c->ev_next_stage; i += 2) {
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, c->ev_stage[i], c->ev_stage[i + 1]));
    st += ms;
  }
  for (size_t i = 0; i + 1 < c->ev_next_halo; i += 2) {
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, c->ev_halo[i], c->ev_halo[i + 1]));
    ha += ms;
  }
  double fa = 0, up = 0;
  if (c->ev_next_mid * 2 == c->ev_next_stage)  // split variant: one mid event per stage
    for (size_t i = 0; i < c->ev_next_mid; ++i) {
      float m1 = 0, m2 = 0;
      CK(cudaEventElapsedTime(&m1, c->ev_stage[2 * i], c->ev_mid[i]));
      CK(cudaEventElapsedTime(&m2, c->ev_mid[i], c->ev_stage[2 * i + 1]));
      fa += m1, up += m2;
    }
  const double n_launch = (double)(c->ev_next_stage / 2);
  out_ms[0] = n_launch > 0 ? st / n_launch : 0;
  out_ms[1] = n_launch > 0 ? ha / n_launch : 0;
  out_ms[2] = n_launch;
  out_ms[3] = (st + ha) / n_steps;
  out_ms[4] = n_launch > 0 ? fa / n_launch : 0;
  out_ms[5] = n_launch > 0 ? up / n_launch : 0;
  return 0;
}

int cc_tuning(cc_ctx *c, int *variant, int *kz, double *stage_ms, int tile[3]) {
  if (int r = check_ctx(c)) return r;
  if (variant) *variant = c->variant;
  if (kz) *kz = c->kz;
  if (stage_ms) *stage_ms = c->tuned_ms;
  if (tile) {
    tile[0] = c->variant >= 3 ? c->face_tx : kTX;
    tile[1] = c->variant >= 3 ? c->face_ty : kTY;
    tile[2] = c->kz;
  }
  return 0;
}

int cc_set_tile_width(cc_ctx *c, int tile_i) {
  if (int r = check_ctx(c)) return r;
  if (tile_i != 0 && tile_i != 16 && tile_i != 32) return fail(CC_ERR_ARG, "tile_i must be 0 (autotune), 16 or 32");
  c->force_tx = tile_i;
  return 0;
}

int cc_set_tuning(cc_ctx *c, int variant, int kz, int tile_j) {
  if (int r = check_ctx(c)) return r;
  if (variant < -1 || variant > 5)
    return fail(CC_ERR_ARG,
                "variant must be -1 (autotune), 0 (fused, L1), 1 (fused, TMA), 2 (split), 3 (split, TMA faces), 4 "
                "(split, TMA faces on persistent CTAs) or 5 (faces differenced in the tile)");
  if (kz < 0) return fail(CC_ERR_ARG, "kz must be >= 0");
  if (tile_j != 0 && tile_j != 4 && tile_j != 8 && tile_j != 16)
    return fail(CC_ERR_ARG, "tile_j must be 0 (autotune), 4, 8 or 16");
  c->force_variant = variant;
  c->force_kz = kz;
  c->force_ty = tile_j;
  if (!c->initialized) return 0;
  if (!variant_ok(c, variant))
    return fail(CC_ERR_ARG, "the TMA variants need 0 or 9 species, the fused and dq ones also the FP32 bulk precision");
  destroy_graphs(c);
  int r = dispatch(c, [&](auto tt, auto nn) { return autotune<typename decltype(tt)::type, decltype(nn)::value>(c); });
  if (r) return r;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

}  // extern "C"

namespace {

uint16_t f2bf(float f) {  // round to nearest even
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7F800000u) == 0x7F800000u) return (uint16_t)(u >> 16);  // inf / nan
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

// rows x cols FP32 row-major matrix -> BF16 operand of R rows x K columns
void pack_operand(std::vector<uint16_t> &blob, int byte0, int R, int K, const float *w, int rows, int cols) {
  for (int r = 0; r < rows; ++r)
    for (int k = 0; k < cols; ++k) blob[(byte0 + mlp_off(R, r, k)) / 2] = f2bf(w[(size_t)r * cols + k]);
  (void)K;
}

template <int NS>
int eval_transport_ns(cc_ctx *c, int64_t n, const double *T, const double *Y, int mode, double *out) {
  const int ns = c->chem.ns, np = 6 + ns, npr = 2 + ns;
  cudaStream_t st = c->stream;
  std::vector<double> h((size_t)np * n, 0.0);
  for (int64_t i = 0; i < n; ++i) {
    h[i] = 1.0;  // rho > 0 marks a point to evaluate
    h[5 * n + i] = T[i];
    for (int l = 0; l < ns; ++l) h[(6 + l) * n + i] = Y[(size_t)l * n + i];
  }
  std::vector<double> o((size_t)npr * n);
  if (mode == 0) {
    double *dP = nullptr, *dPr = nullptr;
    CK(cudaMalloc(&dP, sizeof(double) * np * n));
    CK(cudaMalloc(&dPr, sizeof(double) * npr * n));
    CK(cudaMemcpyAsync(dP, h.data(), sizeof(double) * np * n, cudaMemcpyHostToDevice, st));
    CK((Launch<double, NS>::props_all(c->chem, dP, dPr, n, st)));
    CK(cudaMemcpyAsync(o.data(), dPr, sizeof(double) * npr * n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    cudaFree(dP);
    cudaFree(dPr);
  } else {
    std::vector<float> hf(h.begin(), h.end()), of((size_t)npr * n);
    float *dP = nullptr, *dPr = nullptr;
    unsigned *dst = nullptr;
    CK(cudaMalloc(&dP, sizeof(float) * np * n));
    CK(cudaMalloc(&dPr, sizeof(float) * npr * n));
    CK(cudaMalloc(&dst, sizeof(unsigned)));
    CK(cudaMemsetAsync(dst, 0, sizeof(unsigned), st));
    CK(cudaMemcpyAsync(dP, hf.data(), sizeof(float) * np * n, cudaMemcpyHostToDevice, st));
    CK((Launch<float, NS>::props_mlp(dP, dPr, n, &c->cl, dst, c->chem, st)));
    unsigned flags = 0;
    CK(cudaMemcpyAsync(of.data(), dPr, sizeof(float) * npr * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&flags, dst, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    cudaFree(dP);
    cudaFree(dPr);
    cudaFree(dst);
    if (flags) return fail(CC_ERR_CUDA, "closure kernel reported status " + std::to_string(flags));
    o.assign(of.begin(), of.end());
  }
  std::memcpy(out, o.data(), sizeof(double) * o.size());
  return 0;
}

}  // namespace

extern "C" {

int cc_set_closure(cc_ctx *c, const cc_closure *m) {
  if (int r = check_ctx(c)) return r;
  const int ns = c->chem.ns, n_in = 2 + 2 * ns, n_out = 2 + ns;
  if (!m || !m->w1 || !m->b1 || !m->w2 || !m->b2 || !m->w3 || !m->b3 || !m->w4 || !m->b4 || !m->out_mean ||
      !m->out_scale)
    return fail(CC_ERR_ARG, "cc_set_closure: null pointer");
  if (ns < 1 || n_in > kMlpIn || n_out > kMlpOut)
    return fail(CC_ERR_ARG, "cc_set_closure: the closure supports 1 to 14 species");
  if (!(m->t_scale > 0) || !(m->t_max > m->t_min)) return fail(CC_ERR_ARG, "cc_set_closure: bad normalisation");
  std::vector<uint16_t> blob(kMlpWBytes / 2, 0);
  pack_operand(blob, 0, kMlpH, kMlpIn, m->w1, kMlpH, n_in);
  pack_operand(blob, kMlpW1, kMlpH, kMlpH, m->w2, kMlpH, kMlpH);
  pack_operand(blob, kMlpW1 + kMlpW2, kMlpH, kMlpH, m->w3, kMlpH, kMlpH);
  pack_operand(blob, kMlpW1 + 2 * kMlpW2, kMlpOut, kMlpH, m->w4, n_out, kMlpH);
  std::vector<float> bias(kMlpBias, 0.0f);
  for (int i = 0; i < kMlpH; ++i) bias[i] = m->b1[i], bias[kMlpH + i] = m->b2[i], bias[2 * kMlpH + i] = m->b3[i];
  for (int i = 0; i < n_out; ++i) bias[3 * kMlpH + i] = m->b4[i];
  if (c->stream) CK(cudaStreamSynchronize(c->stream));
  if (!c->cl.w) {
    void *p = nullptr;
    CK(cudaMalloc(&p, kMlpWBytes + sizeof(float) * kMlpBias + 3 * sizeof(unsigned long long)));
    c->allocs.push_back(p);
    c->cl.w = p;
    c->cl.b = reinterpret_cast<const float *>(static_cast<unsigned char *>(p) + kMlpWBytes);
    c->cl.counts = reinterpret_cast<unsigned long long *>(static_cast<unsigned char *>(p) + kMlpWBytes +
                                                          sizeof(float) * kMlpBias);
  }
  CK(cudaMemcpy(const_cast<void *>(c->cl.w), blob.data(), kMlpWBytes, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(const_cast<float *>(c->cl.b), bias.data(), sizeof(float) * kMlpBias, cudaMemcpyHostToDevice));
  CK(cudaMemset(c->cl.counts, 0, 3 * sizeof(unsigned long long)));
  for (int i = 0; i < kMlpOut; ++i) {
    c->cl.out_mean[i] = i < n_out ? m->out_mean[i] : 0.0f;
    c->cl.out_scale[i] = i < n_out ? m->out_scale[i] : 0.0f;
  }
  c->cl.t_center = (float)m->t_center;
  c->cl.t_inv_scale = (float)(1.0 / m->t_scale);
  c->cl.t_min = (float)m->t_min;
  c->cl.t_max = (float)m->t_max;
  c->cl.err_bound = (float)c->closure_bound;
  c->closure_set = true;
  destroy_graphs(c);
  return 0;
}

int cc_use_closure(cc_ctx *c, int on) {
  if (int r = check_ctx(c)) return r;
  if (on && !c->closure_set) return fail(CC_ERR_STATE, "cc_use_closure: no closure set (cc_set_closure)");
  c->closure_on = on != 0;
  destroy_graphs(c);
  return 0;
}

int cc_closure_stats(cc_ctx *c, int64_t out[3]) {
  if (int r = check_ctx(c)) return r;
  if (!out) return fail(CC_ERR_ARG, "null pointer");
  out[0] = out[1] = out[2] = 0;
  if (!c->cl.counts) return 0;
  if (c->stream) CK(cudaStreamSynchronize(c->stream));
  unsigned long long h[3];
  CK(cudaMemcpy(h, c->cl.counts, sizeof h, cudaMemcpyDeviceToHost));
  out[0] = (int64_t)h[0], out[1] = (int64_t)h[1], out[2] = (int64_t)h[2];
  return 0;
}

int cc_set_closure_bound(cc_ctx *c, double rel_err) {
  if (int r = check_ctx(c)) return r;
  if (!(rel_err >= 0.0)) return fail(CC_ERR_ARG, "cc_set_closure_bound: the bound must be >= 0");
  c->closure_bound = rel_err;
  c->cl.err_bound = (float)rel_err;
  destroy_graphs(c);  // the captured launches carry the closure parameters by value
  return 0;
}

int cc_eval_transport(cc_ctx *c, int64_t n, const double *T, const double *Y, int mode, double *out) {
  if (int r = check_ctx(c)) return r;
  if (n <= 0 || !T || !out || (c->chem.ns > 0 && !Y)) return fail(CC_ERR_ARG, "cc_eval_transport: bad arguments");
  if (mode != 0 && mode != 1) return fail(CC_ERR_ARG, "cc_eval_transport: mode must be 0 (exact) or 1 (closure)");
  if (mode == 1 && !c->closure_set) return fail(CC_ERR_STATE, "cc_eval_transport: no closure set");
  if (c->chem.ns == 0) return fail(CC_ERR_ARG, "cc_eval_transport: needs a mixture (n_spec > 0)");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(CC_ERR_NODEVICE, "no CUDA device");
  return c->chem.ns == 9 ? eval_transport_ns<9>(c, n, T, Y, mode, out) : eval_transport_ns<-1>(c, n, T, Y, mode, out);
}

}  // extern "C"

namespace {

// Checkpoint file: header, then the current state's arrays as they are on
// the device (so that a restart continues bit-identically): Q [n_var][N]
// FP64, P [6+ns][N] and Pr [2+ns][N] in the bulk precision, |V| [N] FP64,
// the time step and its history slot [2] FP64.
struct CkptHeader {
  char magic[8];  // "CCB2CKPT"
  int32_t version, precision, n_spec, n_blocks;
  int64_t N;
  double p_ref;
  int32_t dims[3 * 4096];
};

int ckpt_io(cc_ctx *c, const char *path, bool save) {
  if (int r = check_ctx(c)) return r;
  if (!path) return fail(CC_ERR_ARG, "checkpoint: null path");
  if (!c->initialized) return fail(CC_ERR_STATE, "checkpoint: cc_init first");
  if (c->blocks.size() > 4096) return fail(CC_ERR_ARG, "checkpoint: at most 4096 blocks");
  if (c->state_dirty && save) {
    int r = dispatch(c, [&](auto tt, auto nn) { return derive_state<typename decltype(tt)::type, decltype(nn)::value>(c); });
    if (r) return r;
  }
  CkptHeader h;
  std::memset(&h, 0, sizeof h);
  std::memcpy(h.magic, "CCB2CKPT", 8);
  h.version = 1, h.precision = c->precision, h.n_spec = c->chem.ns, h.n_blocks = (int32_t)c->blocks.size();
  h.N = c->N, h.p_ref = c->chem.p_ref;
  for (size_t b = 0; b < c->blocks.size(); ++b)
    h.dims[3 * b] = c->blocks[b].mx, h.dims[3 * b + 1] = c->blocks[b].my, h.dims[3 * b + 2] = c->blocks[b].mz;
  const size_t N = (size_t)c->N;
  struct Part {
    void *dev;
    size_t bytes;
  };
  if (save && c->q_ghost_stale)
    if (int r = dispatch(c, [&](auto tt, auto nn) { return refresh_ghost_q<typename decltype(tt)::type, decltype(nn)::value>(c); }))
      return r;
  if (!save) c->q_ghost_stale = false;  // the file holds every point's conserved state
  const Part parts[] = {{c->Q[c->qcur], sizeof(double) * N * nv_of(c)},
                        {c->P[c->cur], c->elem * N * np_of(c)},
                        {c->Pr[c->cur], c->elem * N * npr_of(c)},
                        {c->d_vel, sizeof(double) * N},
                        {c->d_dt, sizeof(double) * 2}};
  CK(cudaStreamSynchronize(c->stream));
  std::vector<unsigned char> buf;
  FILE *f = std::fopen(path, save ? "wb" : "rb");
  if (!f) return fail(CC_ERR_ARG, std::string("checkpoint: cannot open ") + path);
  int rc = 0;
  if (save) {
    if (std::fwrite(&h, sizeof h, 1, f) != 1) rc = fail(CC_ERR_ARG, "checkpoint: write failed");
    for (const Part &pt : parts) {
      if (rc) break;
      buf.resize(pt.bytes);
      if (cudaMemcpy(buf.data(), pt.dev, pt.bytes, cudaMemcpyDeviceToHost) != cudaSuccess) {
        rc = fail(CC_ERR_CUDA, "checkpoint: device read failed");
        break;
      }
      if (std::fwrite(buf.data(), 1, pt.bytes, f) != pt.bytes) rc = fail(CC_ERR_ARG, "checkpoint: write failed");
    }
  } else {
    CkptHeader g;
    if (std::fread(&g, sizeof g, 1, f) != 1 || std::memcmp(g.magic, "CCB2CKPT", 8) != 0 || g.version != 1)
      rc = fail(CC_ERR_ARG, "checkpoint: not a checkpoint file");
    else if (g.precision != h.precision || g.n_spec != h.n_spec || g.n_blocks != h.n_blocks || g.N != h.N ||
             std::memcmp(g.dims, h.dims, sizeof(int32_t) * 3 * h.n_blocks) != 0)
      rc = fail(CC_ERR_ARG, "checkpoint: written for another layout or precision");
    for (const Part &pt : parts) {
      if (rc) break;
      buf.resize(pt.bytes);
      if (std::fread(buf.data(), 1, pt.bytes, f) != pt.bytes) {
        rc = fail(CC_ERR_ARG, "checkpoint: file too short");
        break;
      }
      if (cudaMemcpy(pt.dev, buf.data(), pt.bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        rc = fail(CC_ERR_CUDA, "checkpoint: device write failed");
    }
    if (!rc) {
      c->chem.p_ref = g.p_ref;
      c->state_dirty = false;
      destroy_graphs(c);
    }
  }
  std::fclose(f);
  return rc;
}

}  // namespace

extern "C" {

int cc_save_checkpoint(cc_ctx *c, const char *path) { return ckpt_io(c, path, true); }
int cc_load_checkpoint(cc_ctx *c, const char *path) { return ckpt_io(c, path, false); }

int cc_set_launch_mode(cc_ctx *c, int per_block) {
  if (int r = check_ctx(c)) return r;
  c->per_block = per_block != 0;
  destroy_graphs(c);
  return 0;
}

int cc_set_owned_blocks(cc_ctx *c, const int *blocks, int n) {
  if (int r = check_ctx(c)) return r;
  std::vector<char> owned;
  if (n > 0) {
    if (!blocks) return fail(CC_ERR_ARG, "cc_set_owned_blocks: blocks is null");
    owned.assign(c->blocks.size(), 0);
    for (int i = 0; i < n; ++i) {
      if (blocks[i] < 0 || blocks[i] >= (int)c->blocks.size())
        return fail(CC_ERR_ARG, "cc_set_owned_blocks: no block " + std::to_string(blocks[i]));
      owned[(size_t)blocks[i]] = 1;
    }
  }
  c->owned = owned;
  if (!c->initialized) return 0;
  destroy_graphs(c);
  return apply_ownership(c);
}

int cc_set_exchange(cc_ctx *c, cc_exchange_fn fn, void *user) {
  if (int r = check_ctx(c)) return r;
  c->hook = fn;
  c->hook_user = user;
  destroy_graphs(c);
  return 0;
}

int cc_exchange_fields(cc_ctx *c, int *n_fields) {
  if (int r = check_ctx(c)) return r;
  if (!n_fields) return fail(CC_ERR_ARG, "n_fields is null");
  *n_fields = np_of(c) + npr_of(c) + nv_of(c);
  return 0;
}

int cc_pack_points(cc_ctx *c, int which, const int64_t *idx, int64_t n, double *out) {
  return pack_unpack(c, which, idx, n, out, true);
}

int cc_unpack_points(cc_ctx *c, int which, const int64_t *idx, int64_t n, const double *in) {
  return pack_unpack(c, which, idx, n, const_cast<double *>(in), false);
}

int cc_residual_sums(cc_ctx *c, double sums[4], int64_t *count) {
  if (int r = check_ctx(c)) return r;
  if (!c->initialized) return fail(CC_ERR_STATE, "cc_residual_sums before cc_init");
  if (!sums || !count) return fail(CC_ERR_ARG, "null output");
  CK(cudaMemcpyAsync(sums, c->d_res + 4, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *count = c->n_int_owned;
  return 0;
}

int cc_halo_dependencies(cc_ctx *c, int64_t *dst, int64_t *src, int *which, int64_t cap, int64_t *n) {
  if (int r = check_ctx(c)) return r;
  if (!n || cap < 0) return fail(CC_ERR_ARG, "cc_halo_dependencies: n is null or cap < 0");
  if (c->blocks.empty()) return fail(CC_ERR_STATE, "no blocks");
  std::vector<HostBlock> blocks = c->blocks;  // the context's own layout is set by cc_init
  std::vector<BlockInfo> info;
  int64_t n_int = 0;
  layout_blocks(blocks, c->ngg, info, n_int);
  HaloPlan plan;
  if (!build_halo_plan(blocks, c->bcs, plan)) return fail(CC_ERR_TOPOLOGY, "halo program: " + plan.error);
  // the points of the current (kind 0) or previous (kind 1) state that a
  // reference resolves to, through the scratch nodes it reads
  std::vector<std::pair<int64_t, int>> found;
  bool unknown_op = false;
  std::function<void(const HaloRef &)> walk = [&](const HaloRef &r) {
    if (r.kind == 0 || r.kind == 1) {
      found.push_back({r.idx, r.kind});
      return;
    }
    const HaloNode &nd = plan.nodes.at((size_t)r.idx);
    if (nd.op == kHaloInflow) return;  // a constant state: no source point
    if (nd.op != kHaloCopy && nd.op != kHaloAvg && nd.op != kHaloWallFace && nd.op != kHaloWallGhost) {
      // an op without a rule here (kHaloKeep is reserved and never emitted):
      // refuse rather than drop its sources silently
      unknown_op = true;
      return;
    }
    walk(nd.a);
    if (nd.op == kHaloAvg || nd.op == kHaloWallGhost) walk(nd.b);
  };
  int64_t k = 0;
  for (const HaloCopy &hc : plan.copies) {
    found.clear();
    walk(hc.src);
    if (unknown_op) return fail(CC_ERR_STATE, "cc_halo_dependencies: halo node op without a dependency rule");
    std::sort(found.begin(), found.end());
    found.erase(std::unique(found.begin(), found.end()), found.end());
    for (const auto &f : found) {
      if (k < cap) {
        if (dst) dst[k] = hc.dst;
        if (src) src[k] = f.first;
        if (which) which[k] = f.second;
      }
      ++k;
    }
  }
  *n = k;
  return 0;
}

int cc_block_arena(cc_ctx *c, int block, int64_t *first, int64_t *count) {
  if (int r = check_ctx(c)) return r;
  if (block < 0 || block >= (int)c->blocks.size()) return fail(CC_ERR_ARG, "cc_block_arena: no such block");
  std::vector<HostBlock> blocks = c->blocks;
  std::vector<BlockInfo> info;
  int64_t n_int = 0;
  layout_blocks(blocks, c->ngg, info, n_int);
  if (first) *first = info[(size_t)block].off;
  if (count) *count = info[(size_t)block].ng;
  return 0;
}

int cc_sync(cc_ctx *c) {
  if (int r = check_ctx(c)) return r;
  if (c->stream) CK(cudaStreamSynchronize(c->stream));
  return 0;
}

}  // extern "C"
