// Test driver: C++ code written against the reference's classes (cfd::Parameter,
// cfd::Mesh, cfd::ChemData, cfd::Driver, cfd::Field) running a case through the
// library.  The case comes from a dump directory written by the test
// (tests/test_cpp_drop_in.py): params.txt ("int|double key value" lines),
// species.bin (the Species tables in declaration order), block_<b>.txt
// ("mx my mz n_boundary n_inner" and the raw face records), block_<b>.bin
// (jacobian, metric, bv, yk), bcs.bin (cc_bc records).
//
//   driver_drop_in <case_dir> <out.bin> <precision 0|1|2> <scheme 0|1|2> <n_steps> [layout 0|1]
//
// layout 1 hands the state to the library and reads it back in the
// reference's VectorField3D order (component fastest, CC_LAYOUT_POINT_MAJOR):
// the initial state is set again that way before initialize_computation.
// out.bin: per block bv, yk, cv (doubles, field-major), then the residual of
// the last step.
#include <cstdio>
#include <fstream>
#include <iostream>
#include <sstream>

#include "cfd_b200.hpp"

// [nf][ng] <-> [ng][nf]
static std::vector<double> transpose(const std::vector<double> &a, size_t nf, bool to_point_major) {
  const size_t ng = nf ? a.size() / nf : 0;
  std::vector<double> t(a.size());
  for (size_t p = 0; p < ng; ++p)
    for (size_t f = 0; f < nf; ++f) {
      if (to_point_major)
        t[p * nf + f] = a[f * ng + p];
      else
        t[f * ng + p] = a[p * nf + f];
    }
  return t;
}

static std::vector<double> read_doubles(std::ifstream &f, size_t n) {
  std::vector<double> v(n);
  f.read(reinterpret_cast<char *>(v.data()), (std::streamsize)(n * sizeof(double)));
  if (!f) throw std::runtime_error("short read");
  return v;
}

int main(int argc, char **argv) {
  if (argc != 6 && argc != 7) {
    std::fprintf(stderr, "usage: %s case_dir out.bin precision scheme n_steps [layout]\n", argv[0]);
    return 2;
  }
  const int layout = argc == 7 ? std::atoi(argv[6]) : CC_LAYOUT_FIELD_MAJOR;
  const std::string dir = argv[1];
  try {
    cfd::Parameter parameter;
    {
      std::ifstream f(dir + "/params.txt");
      std::string type, key;
      while (f >> type >> key) {
        if (type == "int") {
          int v;
          f >> v;
          parameter.update_parameter(key, v);
        } else {
          double v;
          f >> v;
          parameter.update_parameter(key, v);
        }
      }
    }
    cfd::ChemData chem;
    const int ns = parameter.get_int("n_spec");
    chem.spec.n_spec = ns;
    if (ns > 0) {
      std::ifstream f(dir + "/species.bin", std::ios::binary);
      cfd::Species &s = chem.spec;
      s.mw = read_doubles(f, ns), s.t_low = read_doubles(f, ns), s.t_mid = read_doubles(f, ns);
      s.t_high = read_doubles(f, ns), s.low_temp_coeff = read_doubles(f, 7 * ns);
      s.high_temp_coeff = read_doubles(f, 7 * ns), s.LJ_potent_inv = read_doubles(f, ns);
      s.vis_coeff = read_doubles(f, ns), s.WjDivWi_to_One4th = read_doubles(f, ns * ns);
      s.sqrt_WiDivWjPl1Mul8 = read_doubles(f, ns * ns);
    }
    cfd::Mesh mesh;
    const int nb = parameter.get_int("n_block"), ngg = parameter.get_int("ngg");
    for (int b = 0; b < nb; ++b) {
      cfd::Block blk;
      std::ifstream t(dir + "/block_" + std::to_string(b) + ".txt");
      int n_bnd = 0, n_inner = 0;
      t >> blk.mx >> blk.my >> blk.mz >> n_bnd >> n_inner;
      blk.boundary.resize(n_bnd);
      for (auto &r : blk.boundary)
        for (int &x : r) t >> x;
      blk.inner_face.resize(n_inner);
      for (auto &r : blk.inner_face)
        for (int &x : r) t >> x;
      const size_t ng = (size_t)blk.n_ghosted(ngg);
      std::ifstream f(dir + "/block_" + std::to_string(b) + ".bin", std::ios::binary);
      blk.jacobian = read_doubles(f, ng);
      blk.metric = read_doubles(f, 9 * ng);
      blk.bv = read_doubles(f, 6 * ng);
      if (ns > 0) blk.yk = read_doubles(f, ns * ng);
      mesh.blocks.push_back(std::move(blk));
    }
    {
      std::ifstream f(dir + "/bcs.bin", std::ios::binary);
      cc_bc bc;
      while (f.read(reinterpret_cast<char *>(&bc), sizeof bc)) mesh.conditions.push_back(bc);
    }

    cfd::Driver driver(parameter, mesh, chem, std::atoi(argv[3]));
    if (layout == CC_LAYOUT_POINT_MAJOR)
      for (size_t b = 0; b < mesh.blocks.size(); ++b)
        driver.field[b].set_state(transpose(mesh.blocks[b].bv, 6, true), transpose(mesh.blocks[b].yk, ns, true),
                                  CC_LAYOUT_POINT_MAJOR);
    driver.initialize_computation();
    driver.simulate(std::atoi(argv[5]), std::atoi(argv[4]), true);
    if (driver.status() != 0) throw std::runtime_error("device status word set");

    std::ofstream out(argv[2], std::ios::binary);
    std::vector<double> bv, yk, cv;
    for (auto &fld : driver.field) {
      fld.get_state(bv, yk, cv, layout);
      if (layout == CC_LAYOUT_POINT_MAJOR) {
        bv = transpose(bv, 6, false);
        yk = transpose(yk, ns, false);
        cv = transpose(cv, 5 + ns, false);
      }
      out.write(reinterpret_cast<const char *>(bv.data()), (std::streamsize)(bv.size() * sizeof(double)));
      out.write(reinterpret_cast<const char *>(yk.data()), (std::streamsize)(yk.size() * sizeof(double)));
      out.write(reinterpret_cast<const char *>(cv.data()), (std::streamsize)(cv.size() * sizeof(double)));
    }
    const auto r = driver.residual();
    out.write(reinterpret_cast<const char *>(r.data()), (std::streamsize)(r.size() * sizeof(double)));
  } catch (const std::exception &e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
