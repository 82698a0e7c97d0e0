// Host launchers of the templated kernels.  Each (precision, species count)
// pair is instantiated in its own translation unit (inst_*.cu) so that the
// large stage kernels compile in parallel.
#pragma once
#include <cuda_runtime.h>

#include "cc_common.h"

namespace ccb {

template <typename T, int NS>
struct Launch {
  static size_t stage_smem();
  static cudaError_t configure();  // kernel attributes; call outside stream capture
  static cudaError_t stage(const StageArgs<T> &a, const ChemParams &C, int n_tiles, cudaStream_t s);
  // TMA-staged variant (stage_tma.cuh); maps = one CUtensorMap per block for a.P
  static size_t stage_tma_smem();
  static cudaError_t stage_tma(const StageArgs<T> &a, const void *maps, const ChemParams &C, int n_tiles,
                               cudaStream_t s);
  // split variant (stage_split.cuh): faces of n_regular tiles + n_edge edge tiles, then the update
  static size_t faces_smem();
  static size_t update_smem();
  static cudaError_t faces(const StageArgs<T> &a, const ChemParams &C, int n_regular, int n_edge, cudaStream_t s);
  // update kernel; high_occ = 1 runs the FP32 form sized for 4 CTAs per SM
  // ux: tile width, 32 (32 x 8 tiles) or 16 (16 x 16)
  static cudaError_t update(const StageArgs<T> &a, const ChemParams &C, int n_tiles, cudaStream_t s,
                            int high_occ = 0, int ux = 32);
  // split variant with TMA-staged planes in the face kernel: tiles of tx x ty
  // points (32 x 4, 32 x 8, 32 x 16, 16 x 8, 16 x 16; the x 16 shapes in FP32
  // only), smem 0 when the ring does not fit
  static size_t faces_tma_smem(int ty = 8, int tx = 32);
  static cudaError_t faces_tma(const StageArgs<T> &a, const Tile *tiles, int ty, int tx, const void *maps,
                               const ChemParams &C, int n_tiles, cudaStream_t s);
  // persistent form: resident CTAs take the n_tiles regular tiles from *ticket (zeroed here)
  static cudaError_t faces_tma_persistent(const StageArgs<T> &a, const Tile *tiles, int ty, int tx, const void *maps,
                                          const ChemParams &C, int n_tiles, unsigned *ticket, cudaStream_t s);
  // face kernel that differences the faces in the tile and writes dq
  // (stage_dq.cuh): tiles of 32 x ty points (ty = 4, 8, 16), FP32 bulk
  // precision with 0 or 9 species only
  static size_t faces_dq_smem(int ty);
  static cudaError_t faces_dq(const StageArgs<T> &a, const Tile *tiles, const void *maps, const ChemParams &C,
                              int n_tiles, int ty, cudaStream_t s);
  // learned transport closure (closure.cuh) over every arena point; cl is a ClosureDev
  static cudaError_t props_mlp(const T *P, T *Pr, int64_t N, const void *cl, unsigned *status, const ChemParams &C,
                               cudaStream_t s);
  // geometric term of the gauge-pressure momentum fluxes (k_gcl)
  static cudaError_t gcl(const BlockInfo *blocks, int nblocks, const T *G, int64_t N, int64_t n_interior,
                         double *out, cudaStream_t s);
  // LU-SGS steady step (lusgs.cuh): right-hand side and diagonal over the
  // tiles, one sweep hyperplane (dir +1 lower, -1 upper) over all blocks, Q += dQ
  static cudaError_t lusgs_rhs(const StageArgs<T> &a, const LusgsArgs &L, const ChemParams &C, int n_tiles,
                               cudaStream_t s);
  static cudaError_t lusgs_sweep(const LusgsArgs &L, const ChemParams &C, int dir, cudaStream_t s);
  static cudaError_t lusgs_update(const StageArgs<T> &a, const LusgsArgs &L, const ChemParams &C, int n_tiles,
                                  cudaStream_t s);
  static cudaError_t halo_nodes(const HaloArgs<T> &a, const ChemParams &C, cudaStream_t s);
  // the copies of the halo program, with the post-exchange time step
  // (a.dt_next) and the zeroing of |V| at wall faces (vel, when not null)
  // q_filter: 0 every copy; 1 not the conserved state of ghost points (steps);
  // 2 only that (before the state is read out); only_q: the Q pass alone
  static cudaError_t halo_copies(const HaloArgs<T> &a, const ChemParams &C, double *vel, const int64_t *vel_zero,
                                 int64_t n_vel_zero, cudaStream_t s, int q_filter = 0, bool only_q = false);
  // every node level of the halo program in one cooperative launch
  static cudaError_t halo_levels(const HaloArgs<T> &a, const ChemParams &C, const HaloLevels &lv, GridBarrier *bar,
                                 unsigned *status, cudaStream_t s);
  static cudaError_t cv_from_bv(const ChemParams &C, const double *P0, double *Q, int64_t N, double *vel,
                                cudaStream_t s);
  static cudaError_t props_all(const ChemParams &C, const T *P, T *Pr, int64_t N, cudaStream_t s);
  static cudaError_t dt_reduce(const ChemParams &C, const BlockInfo *blocks, int nblocks, const T *P, const T *Pr,
                               const T *G, int64_t N, int64_t n_interior, unsigned long long *dt_out,
                               cudaStream_t s);
};

#define CCB_DECLARE(T, NS) extern template struct Launch<T, NS>;
CCB_DECLARE(double, 0)
CCB_DECLARE(double, 9)
CCB_DECLARE(double, -1)
CCB_DECLARE(float, 0)
CCB_DECLARE(float, 9)
CCB_DECLARE(float, -1)
#undef CCB_DECLARE

// Non-templated helpers (misc.cu).
// dst = (float)(src - shift), dst = (double)src + shift (the gauge pressure field)
cudaError_t launch_convert_d2f_shift(const double *src, float *dst, int64_t n, double shift, cudaStream_t s);
cudaError_t launch_convert_f2d_shift(const float *src, double *dst, int64_t n, double shift, cudaStream_t s);
cudaError_t launch_convert_d2f(const double *src, float *dst, int64_t n, cudaStream_t s);
cudaError_t launch_convert_f2d(const float *src, double *dst, int64_t n, cudaStream_t s);
cudaError_t launch_dt_finalize(double *dt, unsigned long long *dt_next, unsigned *status, double *dt_hist,
                               cudaStream_t s);
cudaError_t launch_zero_points(double *field, const int64_t *points, int64_t n, cudaStream_t s);
template <typename T>
cudaError_t launch_gather_points(const T *src, int64_t N, int nf, const int64_t *idx, int64_t n, double *out,
                                 cudaStream_t s);
template <typename T>
cudaError_t launch_scatter_points(T *dst, int64_t N, int nf, const int64_t *idx, int64_t n, const double *in,
                                  cudaStream_t s);
template <typename T>
cudaError_t launch_store_last(const BlockInfo *blocks, int nblocks, const T *P, const double *vel, int64_t N,
                              int64_t n_interior, double *bv_last, cudaStream_t s);
template <typename T>
cudaError_t launch_residual(const BlockInfo *blocks, int nblocks, const T *P, const double *vel, int64_t N,
                            int64_t n_interior, const double *bv_last, double *partials, int n_partials, double *res,
                            cudaStream_t s);

}  // namespace ccb
