// Oracle harness: drives the reference's OWN kernels (compiled from the
// reference sources by build_ref.sh) on one case file and dumps the result.
// Test infrastructure only; the product never links it.
//
// It replaces the file-driven parts of Driver (Driver.cu:17-57, 113-246) that
// cannot run here, and nothing on the numeric path:
//   - setup: Block/Boundary/InnerFace from the reference's own Mesh.cpp
//     constructors and register_boundary, Field::setup_device_memory, a
//     DParameter filled field by field (DParameter.cu needs input files);
//   - scheme objects are created with the reference's device constructors;
//   - each step is the Driver.cu:189-244 loop body; compute_viscous_flux is
//     only launched for viscous cases (Driver.cu:206 launches it for inviscid
//     runs too, which adds never-written shared memory into dq);
//   - the boundary launches follow DBoundCond::apply_boundary_conditions
//     (BoundCond.cu:251-313) for every face of every block, and the
//     inner-face exchange launches inner_communication with its face extent
//     in device memory (Driver.cu:204 passes a host array).
//
// Case file layout (little endian), written by tests/golden/make_golden.py:
//   char[8] "CCCASE01"
//   int32 n_spec n_block ngg viscous_order reconstruction limiter n_steps n_bc
//   f64 Pr cfl Sc
//   if n_spec: f64 mw[n] t_low[n] t_mid[n] t_high[n] low[n*7] high[n*7]
//              LJ_inv[n] vis_coeff[n] WjDivWi[n*n] sqrtW[n*n]
//   n_bc x { int32 label kind thermal_type pad; f64 t_wall rho u v w p T yk[n] }
//   n_block x { int32 mx my mz n_bnd n_inner; int32 bnd[n_bnd][7];
//               int32 inner[n_inner][13]; f64 jac[Ng] metric[9][Ng] bv[6][Ng]
//               yk[n][Ng] }     (Ng = full ghosted box, i fastest)
// With "--time N" after the two paths, the harness also times N further
// explicit steps of the reference's kernels with CUDA events, after the case
// file's steps as warm-up: the per-block kernels of a step (set_dq_to_0,
// compute_inviscid_flux, compute_viscous_flux, local_time_step,
// update_cv_and_bv, update_physical_properties; Driver.cu:144-177) alone, and
// the whole step with the boundary launches and the harness's interface
// fill, and prints one JSON line with the milliseconds per step.
// Output: char[8] "CCOUT001", int32 n_block, then per block the processed
// boundaries (9 ints each) and inner faces (26 ints each), the first step's
// dq[n_var][N] and dt_local[N], the final bv[6][Ng] yk[n][Ng] cv[n_var][Ng]
// mul[Ng] conductivity[Ng] rho_D[n][Ng] and, after all blocks, residual[4].
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "BoundCond.cuh"
#include "BoundCond.h"
#include "Constants.h"
#include "DParameter.h"
#include "Field.h"
#include "InviscidScheme.cuh"
#include "Mesh.h"
#include "Parameter.h"
#include "TemporalScheme.cuh"
#include "TimeAdvanceFunc.cuh"
#include "ViscousScheme.cuh"

#define CK(x)                                                                                \
  do {                                                                                       \
    cudaError_t e_ = (x);                                                                    \
    if (e_ != cudaSuccess) {                                                                 \
      std::fprintf(stderr, "CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
      std::exit(2);                                                                          \
    }                                                                                        \
  } while (0)

struct Reader {
  FILE *f;
  template <typename T>
  T get() {
    T v;
    if (std::fread(&v, sizeof(T), 1, f) != 1) {
      std::fprintf(stderr, "short case file\n");
      std::exit(3);
    }
    return v;
  }
  template <typename T>
  std::vector<T> vec(size_t n) {
    std::vector<T> v(n);
    if (n && std::fread(v.data(), sizeof(T), n, f) != n) {
      std::fprintf(stderr, "short case file\n");
      std::exit(3);
    }
    return v;
  }
};

struct Writer {
  FILE *f;
  template <typename T>
  void put(const T *p, size_t n) {
    std::fwrite(p, sizeof(T), n, f);
  }
};

struct BcDef {
  int label, kind, thermal_type;
  double t_wall, rho, u, v, w, p, T;
  std::vector<double> yk;
};

__global__ void harness_setup_schemes(cfd::InviscidScheme **inv, cfd::ViscousScheme **visc,
                                      cfd::TemporalScheme **temp, cfd::DParameter *param) {
  *inv = new cfd::AUSMP(param);
  if (param->viscous_scheme == 2)
    *visc = new cfd::SecOrdViscScheme;
  else
    *visc = new cfd::ViscousScheme;
  *temp = new cfd::SteadyTemporalScheme;
}

static double *dev_copy(const std::vector<double> &h) {
  double *d = nullptr;
  CK(cudaMalloc(&d, h.size() * sizeof(double)));
  CK(cudaMemcpy(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
  return d;
}

int main(int argc, char **argv) {
  if (argc != 3 && argc != 5) {
    std::fprintf(stderr, "usage: %s case.bin out.bin [--time N]\n", argv[0]);
    return 1;
  }
  const int time_steps = argc == 5 && std::strcmp(argv[3], "--time") == 0 ? std::atoi(argv[4]) : 0;
  // the reference's kernels allocate per-thread work arrays with device new
  // (InviscidScheme.cu:33, Reconstruction.cu:63, Transport.cu:48-61,
  // Field.cu:190, ViscousScheme.cu:84): at most ~1 KB per thread live at once
  // for 9 species, and at most 2048 resident threads per SM, so 2 GiB of
  // device heap covers every resident thread several times over
  CK(cudaDeviceSetLimit(cudaLimitMallocHeapSize, (size_t)2 << 30));
  Reader rd{std::fopen(argv[1], "rb")};
  if (!rd.f) return 4;
  char magic[8];
  if (std::fread(magic, 1, 8, rd.f) != 8 || std::memcmp(magic, "CCCASE01", 8) != 0) return 5;
  const int n_spec = rd.get<int>(), n_block = rd.get<int>(), ngg = rd.get<int>();
  const int viscous_order = rd.get<int>(), reconstruction = rd.get<int>(), limiter = rd.get<int>();
  const int n_steps = rd.get<int>(), n_bc = rd.get<int>();
  const double Pr = rd.get<double>(), cfl = rd.get<double>(), Sc = rd.get<double>();
#if MULTISPECIES == 1
  if (n_spec <= 0) return 6;
#else
  if (n_spec != 0) return 6;
#endif
  const int n_var = 5 + n_spec;
  std::vector<double> mw, t_low, t_mid, t_high, low, high, lj, visc, wj, sw;
  if (n_spec > 0) {
    mw = rd.vec<double>(n_spec), t_low = rd.vec<double>(n_spec), t_mid = rd.vec<double>(n_spec);
    t_high = rd.vec<double>(n_spec), low = rd.vec<double>(7 * n_spec), high = rd.vec<double>(7 * n_spec);
    lj = rd.vec<double>(n_spec), visc = rd.vec<double>(n_spec);
    wj = rd.vec<double>(n_spec * n_spec), sw = rd.vec<double>(n_spec * n_spec);
  }
  std::vector<BcDef> bcs(n_bc);
  for (auto &b : bcs) {
    b.label = rd.get<int>(), b.kind = rd.get<int>(), b.thermal_type = rd.get<int>();
    (void)rd.get<int>();
    b.t_wall = rd.get<double>(), b.rho = rd.get<double>(), b.u = rd.get<double>(), b.v = rd.get<double>();
    b.w = rd.get<double>(), b.p = rd.get<double>(), b.T = rd.get<double>();
    b.yk = rd.vec<double>(n_spec);
  }

  // Parameter object for Field (Parameter.cpp:20-24 reads "type key = value")
  const std::string pfile = std::string(argv[2]) + ".param";
  {
    std::ofstream pf(pfile);
    pf << "int n_var = " << n_var << "\n";
    pf << "int n_spec = " << n_spec << "\n";
    pf << "int temporal_scheme = 0\n";
    pf << "bool steady = 1\n";
  }
  cfd::Parameter parameter(pfile);

  std::vector<cfd::Block> blocks;
  blocks.reserve(n_block);
  std::vector<std::vector<double>> h_bv(n_block), h_yk(n_block);
  for (int b = 0; b < n_block; ++b) {
    const int mx = rd.get<int>(), my = rd.get<int>(), mz = rd.get<int>();
    const int n_bnd = rd.get<int>(), n_inner = rd.get<int>();
    blocks.emplace_back(mx, my, mz, ngg, b);
    cfd::Block &blk = blocks.back();
    for (int f = 0; f < n_bnd; ++f) {
      auto r = rd.vec<int>(7);
      blk.boundary.emplace_back(r[0], r[1], r[2], r[3], r[4], r[5], r[6]);
      blk.boundary.back().register_boundary(ngg, 3);
    }
    for (int f = 0; f < n_inner; ++f) {
      auto r = rd.vec<int>(13);
      blk.inner_face.emplace_back(r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7], r[8], r[9], r[10], r[11], r[12]);
      blk.inner_face.back().register_boundary(ngg, 3);
    }
    const size_t ng = (size_t)(mx + 2 * ngg) * (my + 2 * ngg) * (mz + 2 * ngg);
    auto jac = rd.vec<double>(ng);
    auto met = rd.vec<double>(9 * ng);
    h_bv[b] = rd.vec<double>(6 * ng);
    h_yk[b] = rd.vec<double>((size_t)n_spec * ng);
    for (int k = -ngg; k < mz + ngg; ++k)
      for (int j = -ngg; j < my + ngg; ++j)
        for (int i = -ngg; i < mx + ngg; ++i) {
          const size_t q = (size_t)(i + ngg) + (size_t)(mx + 2 * ngg) * ((size_t)(j + ngg) + (size_t)(my + 2 * ngg) * (k + ngg));
          blk.jacobian(i, j, k) = jac[q];
          for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) blk.metric(i, j, k)(r + 1, c + 1) = met[(size_t)(3 * r + c) * ng + q];
        }
  }
  std::fclose(rd.f);

  // BoundCond.cu:218-230: wall faces exclude the tangential ghost layers.
  for (auto &blk : blocks)
    for (auto &bd : blk.boundary)
      for (const auto &bc : bcs)
        if (bc.kind == 2 && bd.type_label == bc.label)
          for (int q = 0; q < 3; ++q)
            if (q != bd.face) bd.range_start[q] += ngg, bd.range_end[q] -= ngg;

  std::vector<cfd::Field> field;
  field.reserve(n_block);
  for (int b = 0; b < n_block; ++b) {
    field.emplace_back(parameter, blocks[b]);
    auto &hz = field.back().h_zone;
    const cfd::Block &blk = blocks[b];
    const int mx = blk.mx, my = blk.my, mz = blk.mz;
    const size_t ng = (size_t)(mx + 2 * ngg) * (my + 2 * ngg) * (mz + 2 * ngg);
    for (int k = -ngg; k < mz + ngg; ++k)
      for (int j = -ngg; j < my + ngg; ++j)
        for (int i = -ngg; i < mx + ngg; ++i) {
          const size_t q = (size_t)(i + ngg) + (size_t)(mx + 2 * ngg) * ((size_t)(j + ngg) + (size_t)(my + 2 * ngg) * (k + ngg));
          for (int l = 0; l < 6; ++l) hz.bv(i, j, k, l) = h_bv[b][(size_t)l * ng + q];
#if MULTISPECIES == 1
          for (int l = 0; l < n_spec; ++l) hz.yk(i, j, k, l) = h_yk[b][(size_t)l * ng + q];
#endif
        }
    field.back().setup_device_memory(parameter, blocks[b]);
  }

  cfd::DParameter hp;
  hp.dim = 3, hp.n_block = n_block, hp.inviscid_scheme = 3, hp.reconstruction = reconstruction;
  hp.limiter = limiter, hp.viscous_scheme = viscous_order, hp.temporal_scheme = 0, hp.output_screen = 1;
  hp.Pr = Pr, hp.cfl = cfl, hp.n_spec = n_spec;
#if MULTISPECIES == 1
  hp.mw = dev_copy(mw), hp.t_low = dev_copy(t_low), hp.t_mid = dev_copy(t_mid), hp.t_high = dev_copy(t_high);
  hp.high_temp_coeff.init_with_size(n_spec, 7);
  CK(cudaMemcpy(hp.high_temp_coeff.data(), high.data(), high.size() * 8, cudaMemcpyHostToDevice));
  hp.low_temp_coeff.init_with_size(n_spec, 7);
  CK(cudaMemcpy(hp.low_temp_coeff.data(), low.data(), low.size() * 8, cudaMemcpyHostToDevice));
  hp.LJ_potent_inv = dev_copy(lj), hp.vis_coeff = dev_copy(visc);
  hp.WjDivWi_to_One4th.init_with_size(n_spec, n_spec);
  CK(cudaMemcpy(hp.WjDivWi_to_One4th.data(), wj.data(), wj.size() * 8, cudaMemcpyHostToDevice));
  hp.sqrt_WiDivWjPl1Mul8.init_with_size(n_spec, n_spec);
  CK(cudaMemcpy(hp.sqrt_WiDivWjPl1Mul8.data(), sw.data(), sw.size() * 8, cudaMemcpyHostToDevice));
  hp.Sc = Sc;
#else
  (void)Sc;
#endif
  cfd::DParameter *param = nullptr;
  CK(cudaMalloc(&param, sizeof(cfd::DParameter)));
  CK(cudaMemcpy(param, &hp, sizeof(cfd::DParameter), cudaMemcpyHostToDevice));

  // boundary condition objects on the device (BoundCond.h:14-64)
  std::vector<cfd::Inflow *> d_inflow(n_bc, nullptr);
  std::vector<cfd::Wall *> d_wall(n_bc, nullptr);
  for (int c = 0; c < n_bc; ++c) {
    const auto &bc = bcs[c];
    if (bc.kind == 5) {
      cfd::Inflow in(bc.label);
      in.density = bc.rho, in.u = bc.u, in.v = bc.v, in.w = bc.w, in.pressure = bc.p, in.temperature = bc.T;
#if MULTISPECIES == 1
      in.yk = dev_copy(bc.yk);
#endif
      CK(cudaMalloc(&d_inflow[c], sizeof(cfd::Inflow)));
      CK(cudaMemcpy(d_inflow[c], &in, sizeof(cfd::Inflow), cudaMemcpyHostToDevice));
    } else if (bc.kind == 2) {
      const std::string wfile = std::string(argv[2]) + ".wall";
      {
        std::ofstream wf(wfile);
        wf << "double temperature = " << bc.t_wall << "\n";
        wf << "option thermal_type = " << (bc.thermal_type == 0 ? "isothermal" : "adiabatic") << "\n";
        wf << "end\n";
      }
      std::ifstream wf(wfile);
      cfd::Wall w(bc.label, wf);
      CK(cudaMalloc(&d_wall[c], sizeof(cfd::Wall)));
      CK(cudaMemcpy(d_wall[c], &w, sizeof(cfd::Wall), cudaMemcpyHostToDevice));
    }
  }

  cfd::InviscidScheme **inv = nullptr;
  cfd::ViscousScheme **vis = nullptr;
  cfd::TemporalScheme **tmp = nullptr;
  CK(cudaMalloc(&inv, sizeof(void *)));
  CK(cudaMalloc(&vis, sizeof(void *)));
  CK(cudaMalloc(&tmp, sizeof(void *)));
  harness_setup_schemes<<<1, 1>>>(inv, vis, tmp, param);
  CK(cudaDeviceSynchronize());

  auto apply_bcs = [&]() {
    const int kinds[3] = {6, 5, 2};
    for (int kk = 0; kk < 3; ++kk)
      for (int c = 0; c < n_bc; ++c) {
        if (bcs[c].kind != kinds[kk]) continue;
        for (int b = 0; b < n_block; ++b)
          for (size_t f = 0; f < blocks[b].boundary.size(); ++f) {
            const auto &h_f = blocks[b].boundary[f];
            if (h_f.type_label != bcs[c].label) continue;
            unsigned tpb[3], bpg[3];
            for (int j = 0; j < 3; j++) {
              const int n_point = h_f.range_end[j] - h_f.range_start[j] + 1;
              tpb[j] = n_point <= (2 * ngg + 1) ? 1 : 16;
              bpg[j] = (n_point - 1) / tpb[j] + 1;
            }
            dim3 TPB{tpb[0], tpb[1], tpb[2]}, BPG{bpg[0], bpg[1], bpg[2]};
            if (kinds[kk] == 6) cfd::apply_outflow<<<BPG, TPB>>>(field[b].d_ptr, (int)f);
            if (kinds[kk] == 5) cfd::apply_inflow<<<BPG, TPB>>>(field[b].d_ptr, d_inflow[c], param, (int)f);
            if (kinds[kk] == 2) cfd::apply_wall<<<BPG, TPB>>>(field[b].d_ptr, d_wall[c], param, (int)f);
            CK(cudaGetLastError());
          }
      }
  };
  unsigned *d_np = nullptr;
  CK(cudaMalloc(&d_np, 3 * sizeof(unsigned)));
  auto exchange = [&]() {
    for (int b = 0; b < n_block; ++b)
      for (size_t l = 0; l < blocks[b].inner_face.size(); ++l) {
        const auto &fc = blocks[b].inner_face[l];
        unsigned tpb[3], bpg[3], np[3];
        for (int j = 0; j < 3; ++j) {
          np[j] = std::abs(fc.range_start[j] - fc.range_end[j]) + 1;
          tpb[j] = np[j] <= (unsigned)(2 * ngg + 1) ? 1 : 16;
          bpg[j] = (np[j] - 1) / tpb[j] + 1;
        }
        CK(cudaMemcpy(d_np, np, sizeof np, cudaMemcpyHostToDevice));
        dim3 TPB{tpb[0], tpb[1], tpb[2]}, BPG{bpg[0], bpg[1], bpg[2]};
        cfd::inner_communication<<<BPG, TPB>>>(field[b].d_ptr, field[fc.target_block].d_ptr, d_np, (int)l);
        CK(cudaGetLastError());
        CK(cudaDeviceSynchronize());
      }
  };
  auto props = [&]() {
    const dim3 tpb{8, 8, 4};
    const int ng_1 = 2 * ngg - 1;
    for (int b = 0; b < n_block; ++b) {
      const int mx = blocks[b].mx, my = blocks[b].my, mz = blocks[b].mz;
      dim3 BPG((mx + ng_1) / tpb.x + 1, (my + ng_1) / tpb.y + 1, (mz + ng_1) / tpb.z + 1);
      cfd::update_physical_properties<<<BPG, tpb>>>(field[b].d_ptr, param);
      CK(cudaGetLastError());
    }
  };

  // Driver.cu:59-97 initialize_computation
  {
    const dim3 tpb{8, 8, 4};
    const int ng_1 = 2 * ngg - 1;
    for (int b = 0; b < n_block; ++b) {
      const int mx = blocks[b].mx, my = blocks[b].my, mz = blocks[b].mz;
      dim3 BPG((mx + ng_1) / tpb.x + 1, (my + ng_1) / tpb.y + 1, (mz + ng_1) / tpb.z + 1);
      cfd::compute_cv_from_bv<<<BPG, tpb>>>(field[b].d_ptr, param);
    }
    CK(cudaDeviceSynchronize());
    apply_bcs();
    CK(cudaDeviceSynchronize());
    exchange();
    props();
    CK(cudaDeviceSynchronize());
  }

  std::vector<std::vector<double>> dq1(n_block), dt1(n_block);
  double res[4] = {0, 0, 0, 0};
  long n_total = 0;
  for (auto &blk : blocks) n_total += (long)blk.mx * blk.my * blk.mz;
  const dim3 tpb{8, 8, 4};
  for (int step = 1; step <= n_steps; ++step) {
    for (int b = 0; b < n_block; ++b) {
      const int mx = blocks[b].mx, my = blocks[b].my, mz = blocks[b].mz;
      dim3 bpg((mx - 1) / tpb.x + 1, (my - 1) / tpb.y + 1, (mz - 1) / tpb.z + 1);
      cfd::store_last_step<<<bpg, tpb>>>(field[b].d_ptr);
      cfd::set_dq_to_0<<<bpg, tpb>>>(field[b].d_ptr);
    }
    for (int b = 0; b < n_block; ++b) {
      const int mx = blocks[b].mx, my = blocks[b].my, mz = blocks[b].mz;
      dim3 bpg((mx - 1) / tpb.x + 1, (my - 1) / tpb.y + 1, (mz - 1) / tpb.z + 1);
      cfd::compute_inviscid_flux(blocks[b], field[b].d_ptr, inv, param, n_var);
      if (viscous_order == 2) cfd::compute_viscous_flux(blocks[b], field[b].d_ptr, vis, param, n_var);
      cfd::local_time_step<<<bpg, tpb>>>(field[b].d_ptr, param, tmp);
      CK(cudaGetLastError());
      CK(cudaDeviceSynchronize());
      if (step == 1) {
        const size_t n = (size_t)mx * my * mz;
        std::vector<double> aos(n * n_var), d1(n), dq(n * n_var);
        CK(cudaMemcpy(aos.data(), field[b].h_ptr->dq.data(), aos.size() * 8, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(d1.data(), field[b].h_ptr->dt_local.data(), n * 8, cudaMemcpyDeviceToHost));
        for (size_t q = 0; q < n; ++q)
          for (int l = 0; l < n_var; ++l) dq[(size_t)l * n + q] = aos[q * n_var + l];
        dq1[b] = dq, dt1[b] = d1;
      }
      cfd::update_cv_and_bv<<<bpg, tpb>>>(field[b].d_ptr, param);
      CK(cudaGetLastError());
    }
    CK(cudaDeviceSynchronize());
    apply_bcs();
    CK(cudaDeviceSynchronize());
    exchange();
    props();
    CK(cudaDeviceSynchronize());
    // compute_square_of_dbv (TimeAdvanceFunc.cu:292-303); the sum is taken
    // on the host instead of reduction_of_dbv_squared.
    for (int l = 0; l < 4; ++l) res[l] = 0;
    for (int b = 0; b < n_block; ++b) {
      const int mx = blocks[b].mx, my = blocks[b].my, mz = blocks[b].mz;
      dim3 bpg((mx - 1) / tpb.x + 1, (my - 1) / tpb.y + 1, (mz - 1) / tpb.z + 1);
      cfd::compute_square_of_dbv<<<bpg, tpb>>>(field[b].d_ptr);
      CK(cudaDeviceSynchronize());
      const size_t n = (size_t)mx * my * mz;
      std::vector<double> sq(4 * n);
      CK(cudaMemcpy(sq.data(), field[b].h_ptr->bv_last.data(), sq.size() * 8, cudaMemcpyDeviceToHost));
      for (size_t q = 0; q < n; ++q)
        for (int l = 0; l < 4; ++l) res[l] += sq[q * 4 + l];
    }
    for (int l = 0; l < 4; ++l) res[l] = std::sqrt(res[l] / (double)n_total);
  }

  if (time_steps > 0) {
    const int n_dev_threads = [] {
      int dev = 0, n_sm = 0, per_sm = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
      cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
      return n_sm * per_sm;
    }();
    auto step_kernels = [&]() {
      for (int b = 0; b < n_block; ++b) {
        const int mx = blocks[b].mx, my = blocks[b].my, mz = blocks[b].mz;
        dim3 bpg((mx - 1) / tpb.x + 1, (my - 1) / tpb.y + 1, (mz - 1) / tpb.z + 1);
        cfd::set_dq_to_0<<<bpg, tpb>>>(field[b].d_ptr);
        cfd::compute_inviscid_flux(blocks[b], field[b].d_ptr, inv, param, n_var);
        if (viscous_order == 2) cfd::compute_viscous_flux(blocks[b], field[b].d_ptr, vis, param, n_var);
        cfd::local_time_step<<<bpg, tpb>>>(field[b].d_ptr, param, tmp);
        cfd::update_cv_and_bv<<<bpg, tpb>>>(field[b].d_ptr, param);
      }
      props();
      CK(cudaGetLastError());
    };
    cudaEvent_t e0, e1, e2, e3;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventCreate(&e2));
    CK(cudaEventCreate(&e3));
    step_kernels();
    CK(cudaDeviceSynchronize());
    CK(cudaEventRecord(e0));
    for (int s = 0; s < time_steps; ++s) step_kernels();
    CK(cudaEventRecord(e1));
    CK(cudaEventSynchronize(e1));
    CK(cudaEventRecord(e2));
    for (int s = 0; s < time_steps; ++s) {
      step_kernels();
      apply_bcs();
      exchange();
    }
    CK(cudaEventRecord(e3));
    CK(cudaEventSynchronize(e3));
    float ms_k = 0, ms_s = 0;
    CK(cudaEventElapsedTime(&ms_k, e0, e1));
    CK(cudaEventElapsedTime(&ms_s, e2, e3));
    std::printf("{\"points\": %ld, \"steps\": %d, \"kernels_ms_per_step\": %.6f, "
                "\"step_ms_with_halo_fill\": %.6f, \"device_threads\": %d}\n",
                n_total, time_steps, ms_k / time_steps, ms_s / time_steps, n_dev_threads);
  }

  Writer wr{std::fopen(argv[2], "wb")};
  wr.put("CCOUT001", 8);
  wr.put(&n_block, 1);
  for (int b = 0; b < n_block; ++b) {
    const cfd::Block &blk = blocks[b];
    const int mx = blk.mx, my = blk.my, mz = blk.mz;
    const int nb = (int)blk.boundary.size(), ni = (int)blk.inner_face.size();
    wr.put(&nb, 1);
    for (const auto &bd : blk.boundary) {
      int v[9] = {bd.range_start[0], bd.range_start[1], bd.range_start[2], bd.range_end[0], bd.range_end[1],
                  bd.range_end[2], bd.type_label, bd.face, bd.direction};
      wr.put(v, 9);
    }
    wr.put(&ni, 1);
    for (const auto &f : blk.inner_face) {
      int v[26] = {f.range_start[0], f.range_start[1], f.range_start[2], f.range_end[0], f.range_end[1],
                   f.range_end[2], f.face, f.direction, f.target_start[0], f.target_start[1],
                   f.target_start[2], f.target_end[0], f.target_end[1], f.target_end[2], f.target_block,
                   f.target_face, f.target_direction, f.src_tar[0], f.src_tar[1], f.src_tar[2],
                   f.loop_dir[0], f.loop_dir[1], f.loop_dir[2], f.target_loop_dir[0],
                   f.target_loop_dir[1], f.target_loop_dir[2]};
      wr.put(v, 26);
    }
    const size_t ng = (size_t)(mx + 2 * ngg) * (my + 2 * ngg) * (mz + 2 * ngg);
    const size_t n = (size_t)mx * my * mz;
    if (dq1[b].empty()) dq1[b].assign((size_t)n_var * n, 0.0), dt1[b].assign(n, 0.0);
    wr.put(dq1[b].data(), dq1[b].size());
    wr.put(dt1[b].data(), dt1[b].size());
    auto *hz = field[b].h_ptr;
    auto fetch_vf = [&](double *dev, int nl) {
      std::vector<double> aos(ng * nl), soa(ng * nl);
      CK(cudaMemcpy(aos.data(), dev, aos.size() * 8, cudaMemcpyDeviceToHost));
      for (size_t q = 0; q < ng; ++q)
        for (int l = 0; l < nl; ++l) soa[(size_t)l * ng + q] = aos[q * nl + l];
      wr.put(soa.data(), soa.size());
    };
    auto fetch_a = [&](double *dev) {
      std::vector<double> a(ng);
      CK(cudaMemcpy(a.data(), dev, ng * 8, cudaMemcpyDeviceToHost));
      wr.put(a.data(), a.size());
    };
    fetch_vf(hz->bv.data(), 6);
#if MULTISPECIES == 1
    fetch_vf(hz->yk.data(), n_spec);
#endif
    fetch_vf(hz->cv.data(), n_var);
    fetch_a(hz->mul.data());
    fetch_a(hz->conductivity.data());
#if MULTISPECIES == 1
    fetch_vf(hz->rho_D.data(), n_spec);
#endif
  }
  wr.put(res, 4);
  std::fclose(wr.f);
  std::remove(pfile.c_str());
  std::printf("ok %d blocks %d steps res %.6e %.6e %.6e %.6e\n", n_block, n_steps, res[0], res[1], res[2], res[3]);
  return 0;
}
