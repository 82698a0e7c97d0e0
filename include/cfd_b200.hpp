// cfd_b200.hpp -- C++ host mirror of the reference's call surface over the
// C ABI of cc_b200.h, so that C++ code written against CombustionCodeGPU's
// classes drives the B200 residual path with the same calls:
//
//   cfd::Parameter parameter;            // Parameter.h:12-67 (typed key/value store)
//   cfd::Mesh mesh;                      // Mesh.h:163-232 (blocks, faces)
//   cfd::ChemData chem_data;             // ChemData.h:11-46 (species tables)
//   cfd::Driver driver(parameter, mesh, chem_data);   // Driver.h:17-26, main.cu:37-43
//   driver.initialize_computation();     // Driver.cu:59-97
//   driver.simulate();                   // Driver.cu:99-192 (steady loop, total_step steps)
//
// Header-only; link with -lcc_b200.  Every failing library call throws
// std::runtime_error carrying cc_last_error().  The reference reads the
// boundary conditions and the initial state inside its Driver from the setup
// files; here they are members of Mesh (conditions) and Block (bv, yk), filled
// by the caller or a reader.
#ifndef CFD_B200_HPP
#define CFD_B200_HPP

#include <array>
#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "cc_b200.h"

namespace cfd {

inline void check(int rc, const char *call) {
  if (rc != CC_OK) throw std::runtime_error(std::string(call) + ": " + cc_last_error());
}

// Parameter.h:12-67: "int/double/bool/string key = value" entries.
class Parameter {
 public:
  void update_parameter(const std::string &key, int v) { ints_[key] = v; }
  void update_parameter(const std::string &key, double v) { reals_[key] = v; }
  void update_parameter(const std::string &key, bool v) { bools_[key] = v; }
  void update_parameter(const std::string &key, const std::string &v) { strings_[key] = v; }
  int get_int(const std::string &key) const { return find(ints_, key); }
  double get_real(const std::string &key) const { return find(reals_, key); }
  bool get_bool(const std::string &key) const { return find(bools_, key); }
  const std::string &get_string(const std::string &key) const { return find(strings_, key); }
  bool has_int(const std::string &key) const { return ints_.count(key) != 0; }
  bool has_real(const std::string &key) const { return reals_.count(key) != 0; }
  bool has_bool(const std::string &key) const { return bools_.count(key) != 0; }
  bool has_string(const std::string &key) const { return strings_.count(key) != 0; }

 private:
  template <typename M>
  static const typename M::mapped_type &find(const M &m, const std::string &key) {
    auto it = m.find(key);
    if (it == m.end()) throw std::out_of_range("Parameter: no entry " + key);
    return it->second;
  }
  std::map<std::string, int> ints_;
  std::map<std::string, double> reals_;
  std::map<std::string, bool> bools_;
  std::map<std::string, std::string> strings_;
};

// Mesh.h:109-159 Block: extents, geometry over the ghosted box (ngg layers,
// i fastest: jac [Ng], metric [9][Ng] with row r*3+c = m(r+1,c+1)), the raw
// records of the boundary and interface files (Mesh.cpp:616-670), and the
// block's initial state bv [6][Ng] (rho,u,v,w,p,T), yk [n_spec][Ng].
struct Block {
  int mx = 0, my = 0, mz = 0;
  std::vector<double> jacobian, metric;
  std::vector<std::array<int, 7>> boundary;     // x1,x2,y1,y2,z1,z2,type
  std::vector<std::array<int, 13>> inner_face;  // the two lines of an interface record
  std::vector<double> bv, yk;
  int64_t n_ghosted(int ngg) const {
    return (int64_t)(mx + 2 * ngg) * (my + 2 * ngg) * (mz + 2 * ngg);
  }
};

// Mesh.h:163-232: the blocks of one process, plus the boundary conditions
// bound to their face labels (BoundCond.h:14-64, kind 2 wall, 5 inflow, 6 outflow).
struct Mesh {
  std::vector<Block> blocks;
  std::vector<cc_bc> conditions;
  int n_block() const { return (int)blocks.size(); }
  const Block &operator[](int b) const { return blocks.at(b); }
  Block &operator[](int b) { return blocks.at(b); }
};

// ChemData.h:11-46 Species, with the tables DParameter copies to the device
// (DParameter.h:9-39): per species mw, t_low/t_mid/t_high, NASA-7
// coefficients [n][7] below and above t_mid, 1/(eps/k), the viscosity
// coefficient, and the Wilke factors [n][n].  n_spec = 0 selects the air model.
struct Species {
  int n_spec = 0;
  std::vector<std::string> names;  // mechanism order (ChemData.cpp:36-57)
  std::vector<double> mw, t_low, t_mid, t_high, low_temp_coeff, high_temp_coeff, LJ_potent_inv, vis_coeff,
      WjDivWi_to_One4th, sqrt_WiDivWjPl1Mul8;
};
struct ChemData {
  Species spec;
};

class Driver;

// Field.h:67-82: one block's state on the device.
class Field {
 public:
  Field(Driver *d, int id, const Block *b) : driver_(d), id_(id), block_(b) {}
  // bv (6 fields), yk (n_spec), cv (n_var) over the Ng ghosted points
  // (HZone::bv/yk, DZone::cv): field-major [field][Ng] by default, or
  // CC_LAYOUT_POINT_MAJOR, the VectorField3D order [Ng][field]
  void get_state(std::vector<double> &bv, std::vector<double> &yk, std::vector<double> &cv,
                 int layout = CC_LAYOUT_FIELD_MAJOR) const;
  // DZone::mul, conductivity, rho_D
  void get_props(std::vector<double> &mul, std::vector<double> &cond, std::vector<double> &rho_d) const;
  void set_state(const std::vector<double> &bv, const std::vector<double> &yk, int layout = CC_LAYOUT_FIELD_MAJOR);
  int id() const { return id_; }

 private:
  Driver *driver_;
  int id_;
  const Block *block_;
};

// Driver.h:17-48 on the sm_100a path.  precision: CC_FP64 keeps the
// reference's arithmetic, CC_MIXED is the FP32-bulk path.
class Driver {
 public:
  Driver(Parameter &parameter, Mesh &mesh, ChemData &chem_data, int precision = CC_FP64)
      : parameter_(parameter), mesh_(mesh), chem_(chem_data), precision_(precision) {
    ngg_ = parameter.get_int("ngg");
    const Species &s = chem_data.spec;
    cc_params p{};
    p.n_spec = s.n_spec;
    p.inviscid_scheme = parameter.get_int("inviscid_scheme");
    p.reconstruction = parameter.get_int("reconstruction");
    p.limiter = parameter.get_int("limiter");
    p.viscous_order = parameter.get_int("viscous_order");
    p.ngg = ngg_;
    p.prandtl_number = parameter.get_real("prandtl_number");
    p.cfl = parameter.get_real("cfl");
    p.schmidt_number = parameter.get_real("schmidt_number");
    if (s.n_spec > 0) {
      p.mw = s.mw.data(), p.t_low = s.t_low.data(), p.t_mid = s.t_mid.data(), p.t_high = s.t_high.data();
      p.low_temp_coeff = s.low_temp_coeff.data(), p.high_temp_coeff = s.high_temp_coeff.data();
      p.LJ_potent_inv = s.LJ_potent_inv.data(), p.vis_coeff = s.vis_coeff.data();
      p.WjDivWi_to_One4th = s.WjDivWi_to_One4th.data(), p.sqrt_WiDivWjPl1Mul8 = s.sqrt_WiDivWjPl1Mul8.data();
    }
    check(cc_create(&p, &ctx_), "cc_create");
    for (const Block &b : mesh.blocks) {
      int id = -1;
      check(cc_add_block(ctx_, b.mx, b.my, b.mz, b.jacobian.data(), b.metric.data(), &id), "cc_add_block");
      for (const auto &raw : b.boundary) {
        cc_boundary f;
        check(cc_register_boundary(raw.data(), ngg_, &f), "cc_register_boundary");
        check(cc_add_boundary(ctx_, id, &f), "cc_add_boundary");
      }
      for (const auto &raw : b.inner_face) {
        cc_inner_face f;
        check(cc_register_inner_face(raw.data(), ngg_, &f), "cc_register_inner_face");
        check(cc_add_inner_face(ctx_, id, &f), "cc_add_inner_face");
      }
      field.emplace_back(this, id, &b);
    }
    for (const cc_bc &bc : mesh.conditions) check(cc_add_bc(ctx_, &bc), "cc_add_bc");
    for (size_t b = 0; b < mesh.blocks.size(); ++b)
      if (!mesh.blocks[b].bv.empty()) field[b].set_state(mesh.blocks[b].bv, mesh.blocks[b].yk);
  }
  Driver(const Driver &) = delete;
  Driver &operator=(const Driver &) = delete;
  ~Driver() {
    if (ctx_) cc_destroy(ctx_);
  }

  // Driver.cu:59-97
  void initialize_computation() { check(cc_init(ctx_, precision_), "cc_init"); }
  // Driver.cu:113-192: total_step steps of the steady explicit loop with the
  // per-point local time step, the residual of the last step evaluated (the
  // reference's temporal_scheme tags run this loop)
  void simulate() { simulate(parameter_.get_int("total_step"), CC_STEADY_EULER, true); }
  // n steps of CC_RK3, CC_STEADY_EULER or CC_STEADY_LUSGS
  void simulate(int n_steps, int scheme, bool want_residual = false) {
    check(cc_step(ctx_, n_steps, scheme, want_residual ? 1 : 0), "cc_step");
  }
  // Driver.cu:219-277: RMS change of rho, |V|, p, T over the last step
  std::array<double, 4> residual() const {
    std::array<double, 4> r{};
    check(cc_residual(ctx_, r.data()), "cc_residual");
    return r;
  }
  unsigned status() const {
    unsigned f = 0;
    check(cc_status(ctx_, &f), "cc_status");
    return f;
  }
  cc_ctx *context() const { return ctx_; }
  int ngg() const { return ngg_; }
  int n_spec() const { return chem_.spec.n_spec; }

  std::vector<Field> field;

 private:
  Parameter &parameter_;
  Mesh &mesh_;
  ChemData &chem_;
  int precision_;
  int ngg_ = 2;
  cc_ctx *ctx_ = nullptr;
};

inline void Field::get_state(std::vector<double> &bv, std::vector<double> &yk, std::vector<double> &cv,
                             int layout) const {
  const int64_t ng = block_->n_ghosted(driver_->ngg());
  const int ns = driver_->n_spec();
  bv.assign(6 * ng, 0.0);
  yk.assign(ns * ng, 0.0);
  cv.assign((5 + ns) * ng, 0.0);
  check(cc_get_state(driver_->context(), id_, bv.data(), ns ? yk.data() : nullptr, cv.data(), layout),
        "cc_get_state");
}

inline void Field::get_props(std::vector<double> &mul, std::vector<double> &cond, std::vector<double> &rho_d) const {
  const int64_t ng = block_->n_ghosted(driver_->ngg());
  const int ns = driver_->n_spec();
  mul.assign(ng, 0.0);
  cond.assign(ng, 0.0);
  rho_d.assign(ns * ng, 0.0);
  check(cc_get_props(driver_->context(), id_, mul.data(), cond.data(), ns ? rho_d.data() : nullptr),
        "cc_get_props");
}

inline void Field::set_state(const std::vector<double> &bv, const std::vector<double> &yk, int layout) {
  check(cc_set_state(driver_->context(), id_, bv.data(), yk.empty() ? nullptr : yk.data(), layout), "cc_set_state");
}

}  // namespace cfd

#endif
