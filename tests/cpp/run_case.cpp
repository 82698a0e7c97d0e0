// Test program written the way the reference's main.cu drives a case
// (main.cu:37-45): read the input files, construct the Driver, initialise,
// run the steady loop; here through include/cfd_b200_io.hpp and
// include/cfd_b200.hpp.
//
//   run_case <input_dir> <out.bin> <n_steps>
//
// out.bin: per block bv, yk, cv (doubles), then the residual of the last step.
#include <cstdio>
#include <fstream>

#include "cfd_b200_io.hpp"

int main(int argc, char **argv) {
  if (argc != 4) {
    std::fprintf(stderr, "usage: %s input_dir out.bin n_steps\n", argv[0]);
    return 2;
  }
  try {
    const std::string dir = argv[1];
    cfd::Parameter parameter = cfd::read_parameters(dir + "/setup");
    cfd::ChemData chem_data = cfd::read_chemdata(dir, parameter);
    cfd::Mesh mesh = cfd::read_mesh(dir, parameter, chem_data);
    cfd::Driver driver(parameter, mesh, chem_data);
    driver.initialize_computation();
    driver.simulate(std::atoi(argv[3]), CC_STEADY_EULER, true);
    std::ofstream out(argv[2], std::ios::binary);
    std::vector<double> bv, yk, cv;
    for (auto &f : driver.field) {
      f.get_state(bv, yk, cv);
      for (const auto *v : {&bv, &yk, &cv})
        out.write(reinterpret_cast<const char *>(v->data()), (std::streamsize)(v->size() * sizeof(double)));
    }
    const auto r = driver.residual();
    out.write(reinterpret_cast<const char *>(r.data()), (std::streamsize)(r.size() * sizeof(double)));
  } catch (const std::exception &e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
