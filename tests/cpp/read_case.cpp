// Test program: reads a reference case directory with the C++ readers
// (include/cfd_b200_io.hpp) and dumps what they produced, for comparison
// with the Python readers (tests/test_cpp_drop_in.py).
//
//   read_case <input_dir> <out.bin>
//
// out.bin (doubles): n_block, ngg, n_spec, the seven scheme parameters,
// the species tables, per block (mx, my, mz, n_boundary, n_inner, the raw
// records, jacobian, metric, bv, yk), n_conditions and per condition (label,
// kind, thermal_type, t_wall, density, u, v, w, pressure, temperature, yk).
#include <cstdio>
#include <fstream>

#include "cfd_b200_io.hpp"

static void put(std::ofstream &o, double v) { o.write(reinterpret_cast<const char *>(&v), sizeof v); }
static void put(std::ofstream &o, const std::vector<double> &v) {
  o.write(reinterpret_cast<const char *>(v.data()), (std::streamsize)(v.size() * sizeof(double)));
}

int main(int argc, char **argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s input_dir out.bin\n", argv[0]);
    return 2;
  }
  try {
    const std::string dir = argv[1];
    cfd::Parameter par = cfd::read_parameters(dir + "/setup");
    cfd::ChemData chem = cfd::read_chemdata(dir, par);
    cfd::Mesh mesh = cfd::read_mesh(dir, par, chem);
    std::ofstream o(argv[2], std::ios::binary);
    const cfd::Species &s = chem.spec;
    put(o, mesh.n_block()), put(o, par.get_int("ngg")), put(o, s.n_spec);
    for (const char *k : {"inviscid_scheme", "reconstruction", "limiter", "viscous_order"}) put(o, par.get_int(k));
    for (const char *k : {"cfl", "prandtl_number", "schmidt_number"}) put(o, par.get_real(k));
    for (const auto *v : {&s.mw, &s.t_low, &s.t_mid, &s.t_high, &s.low_temp_coeff, &s.high_temp_coeff,
                          &s.LJ_potent_inv, &s.vis_coeff, &s.WjDivWi_to_One4th, &s.sqrt_WiDivWjPl1Mul8})
      put(o, *v);
    for (const cfd::Block &b : mesh.blocks) {
      put(o, b.mx), put(o, b.my), put(o, b.mz), put(o, (double)b.boundary.size()), put(o, (double)b.inner_face.size());
      for (const auto &r : b.boundary)
        for (int x : r) put(o, x);
      for (const auto &r : b.inner_face)
        for (int x : r) put(o, x);
      put(o, b.jacobian), put(o, b.metric), put(o, b.bv), put(o, b.yk);
    }
    put(o, (double)mesh.conditions.size());
    for (const cc_bc &c : mesh.conditions) {
      put(o, c.label), put(o, c.kind), put(o, c.thermal_type), put(o, c.t_wall);
      for (double v : {c.density, c.u, c.v, c.w, c.pressure, c.temperature}) put(o, v);
      for (int l = 0; l < s.n_spec; ++l) put(o, c.yk[l]);
    }
  } catch (const std::exception &e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
