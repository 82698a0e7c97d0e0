// cfd_b200_io.hpp -- readers of the reference's input files for C++ callers
// of cfd_b200.hpp, so that a reference case directory runs unchanged:
//
//   cfd::Parameter parameter = cfd::read_parameters("input_files/setup");  // Parameter.cpp:44-71
//   cfd::ChemData chem_data = cfd::read_chemdata("input_files", parameter); // ChemData.cpp:10-261
//   cfd::Mesh mesh = cfd::read_mesh("input_files", parameter, chem_data);  // Mesh.cpp:566-923, BoundCond
//   cfd::Driver driver(parameter, mesh, chem_data);
//
// Header-only, C++17.  The same readers exist in Python
// (combustioncodegpu_b200.io); both give the same arrays.  Single-process
// files only (the "   0" suffix).  Differences from the reference, as in the
// Python readers: interface ghosts across a periodic interface are
// translated by the period (reference_ghosts = true keeps the raw copy), and
// only the first group of 8_initialization.txt sets the initial state.
#ifndef CFD_B200_IO_HPP
#define CFD_B200_IO_HPP

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <set>
#include <sstream>

#include "cfd_b200.hpp"

namespace cfd {
namespace io_detail {

constexpr double kRu = 8314.462618;   // Constants.h:19
constexpr double kGammaAir = 1.4;     // Constants.h:23
constexpr double kMwAir = 28.9647;    // Constants.h:28

inline std::vector<std::string> lines_of(const std::string &path, bool must) {
  std::ifstream f(path);
  if (!f) {
    if (must) throw std::runtime_error("cannot open " + path);
    return {};
  }
  std::vector<std::string> out;
  std::string s;
  while (std::getline(f, s)) {
    if (!s.empty() && s.back() == '\r') s.pop_back();
    out.push_back(s);
  }
  return out;
}

inline std::vector<std::string> split(const std::string &s) {
  std::istringstream is(s);
  std::vector<std::string> t;
  std::string w;
  while (is >> w) t.push_back(w);
  return t;
}

inline std::string upper(std::string s) {
  for (char &c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}
inline std::string lower(std::string s) {
  for (char &c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}
inline bool starts_with(const std::string &s, const std::string &p) { return s.compare(0, p.size(), p) == 0; }
inline std::string strip(const std::string &s) {
  size_t a = s.find_first_not_of(" \t"), b = s.find_last_not_of(" \t");
  return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}
inline std::string cols(const std::string &s, size_t a, size_t b) { return a >= s.size() ? "" : s.substr(a, b - a); }
inline std::string join(const std::string &dir, const std::string &name) {
  return dir.empty() || dir.back() == '/' ? dir + name : dir + "/" + name;
}
inline std::string numbered(const char *stem, const char *ext) {  // "grid%4d.grd" % 0
  char buf[64];
  std::snprintf(buf, sizeof buf, "%s%4d%s", stem, 0, ext);
  return buf;
}

// Element.cpp:14-21 atomic weights of the elements the mechanisms use
inline double atomic_weight(const std::string &e) {
  if (e == "H") return 1.008;
  if (e == "N") return 14.007;
  if (e == "O") return 15.999;
  throw std::runtime_error("ChemData: no atomic weight for element " + e);
}

// {label: (double entries, option entries, species entries)} of a per-label
// setup file ("label n" opens a section; "end" closes the file)
struct Section {
  std::map<std::string, double> dbl, spec;
  std::map<std::string, std::string> opt;
};
inline std::map<int, Section> sections(const std::string &path) {
  std::map<int, Section> out;
  Section *cur = nullptr;
  for (const std::string &line : lines_of(path, false)) {
    const auto raw = split(line);
    const auto toks = split(lower(line));
    if (toks.empty() || starts_with(toks[0], "//")) continue;
    if (toks[0] == "end") break;
    if (toks[0] == "label") {
      cur = &out[std::stoi(toks[1])];
      continue;
    }
    if (cur && toks.size() >= 4) {
      if (toks[0] == "double") cur->dbl[toks[1]] = std::stod(toks[3]);
      else if (toks[0] == "option") cur->opt[toks[1]] = toks[3];
      else if (toks[0] == "species") cur->spec[upper(raw[1])] = std::stod(toks[3]);
    }
  }
  return out;
}

inline double get(const std::map<std::string, double> &m, const std::string &k, double dflt) {
  auto it = m.find(k);
  return it == m.end() ? dflt : it->second;
}

// BoundCond.cpp:10-104: primitive state of an inflow section
inline cc_bc inflow_state(const Section &sec, const Species &sp) {
  const std::vector<std::string> &names = sp.names;
  const auto &d = sec.dbl;
  const double mach = get(d, "mach", -1.0), vel0 = get(d, "velocity", -1.0);
  const double p = get(d, "pressure", 101325.0);
  double T = get(d, "temperature", -1.0), rho = get(d, "density", -1.0);
  cc_bc bc{};
  const int ns = sp.n_spec;
  std::vector<double> yk(ns, 0.0);
  double mw = kMwAir, gamma = kGammaAir;
  if (ns > 0) {
    for (const auto &kv : sec.spec) {
      auto it = std::find(names.begin(), names.end(), kv.first);
      if (it != names.end()) yk[it - names.begin()] = kv.second;
    }
    double s = 0;
    for (int k = 0; k < ns; ++k) s += yk[k] / sp.mw[k];
    mw = 1.0 / s;
  }
  if (T < 0) T = p * mw / (rho * kRu);
  if (ns > 0) {
    double cp = 0, cv = 0;
    for (int k = 0; k < ns; ++k) {
      const double *lo = (T < sp.t_mid[k] ? sp.low_temp_coeff.data() : sp.high_temp_coeff.data()) + 7 * k;
      const double te = std::max(T, sp.t_low[k]);
      double c = 0;
      for (int q = 0; q < 5; ++q) c += lo[q] * std::pow(te, q);
      c = c * kRu / sp.mw[k];
      cp += yk[k] * c;
      cv += yk[k] * (c - kRu / sp.mw[k]);
    }
    gamma = cp / cv;
  }
  const double c = std::sqrt(gamma * kRu / mw * T);
  const double vel = mach >= 0 ? mach * c : vel0;
  if (rho < 0) rho = p * mw / (kRu * T);
  bc.density = rho, bc.u = get(d, "u", 1.0) * vel, bc.v = get(d, "v", 0.0) * vel, bc.w = get(d, "w", 0.0) * vel;
  bc.pressure = p, bc.temperature = T;
  for (int k = 0; k < ns && k < CC_MAX_SPECIES; ++k) bc.yk[k] = yk[k];
  return bc;
}

}  // namespace io_detail

// Parameter.cpp:44-71: every "int/double/bool/string key = value" line of the
// setup files (first definition wins), with the library's defaults for the
// scheme keys the Driver reads (AUSM+ 3, MUSCL 2, minmod 0, viscous_order 2,
// cfl 0.5, Pr 0.72, Sc 0.9) and ngg = 2 (3 for the fifth-order schemes).
inline Parameter read_parameters(const std::string &setup_dir) {
  using namespace io_detail;
  Parameter par;
  std::set<std::string> seen;
  for (const char *name : {"0_global_control.txt", "1_grid_information.txt", "2_scheme.txt",
                           "3_species_reactions.txt", "4_laminar_turbulent.txt", "9_transport_property.txt"}) {
    for (const std::string &line : lines_of(join(setup_dir, name), false)) {
      if (starts_with(line, "//") || starts_with(line, "!") || strip(line).empty()) continue;
      const auto t = split(line);
      if (t.size() < 4 || seen.count(t[1])) continue;
      seen.insert(t[1]);
      if (t[0] == "int") par.update_parameter(t[1], std::stoi(t[3]));
      else if (t[0] == "double") par.update_parameter(t[1], std::stod(t[3]));
      else if (t[0] == "bool") {
        const bool digit = !t[3].empty() && std::all_of(t[3].begin(), t[3].end(), ::isdigit);
        par.update_parameter(t[1], digit ? std::stoi(t[3]) != 0 : lower(t[3]) == "true");
      } else if (t[0] == "string") par.update_parameter(t[1], t[3]);
      else seen.erase(t[1]);
    }
  }
  auto dflt_i = [&](const char *k, int v) {
    if (!par.has_int(k)) par.update_parameter(k, v);
  };
  auto dflt_d = [&](const char *k, double v) {
    if (!par.has_real(k)) par.update_parameter(k, v);
  };
  const int inv = par.has_int("inviscid_scheme") ? par.get_int("inviscid_scheme") : 0;
  dflt_i("ngg", inv / 10 == 5 ? 3 : 2);
  dflt_i("inviscid_scheme", 3);
  dflt_i("reconstruction", 2);
  dflt_i("limiter", 0);
  dflt_i("viscous_order", 2);
  dflt_d("cfl", 0.5);
  dflt_d("prandtl_number", 0.72);
  dflt_d("schmidt_number", 0.9);
  return par;
}

// ChemData.cpp:10-261: species order of the mechanism file, fixed-column
// NASA-7 records of the thermo file, Lennard-Jones parameters of the
// transport file, and the derived Wilke constants.  Returns n_spec = 0 (air)
// when the setup names no mechanism file.
inline ChemData read_chemdata(const std::string &input_dir, const Parameter &par) {
  using namespace io_detail;
  ChemData cd;
  if (!par.has_string("mechanism_file")) return cd;
  const auto mech = lines_of(join(input_dir, par.get_string("mechanism_file")), true);
  size_t i = 4;
  std::vector<std::string> elements;
  while (upper(split(mech.at(i)).at(0)) != "SPECIES") {
    for (const auto &e : split(upper(mech[i]))) elements.push_back(e);
    ++i;
  }
  std::set<std::string> elem_set(elements.begin(), elements.end());
  i += 2;
  const int ns = std::stoi(split(mech.at(i))[0]);
  i += 2;
  std::vector<std::string> names;
  for (;; ++i) {
    const auto t = split(upper(mech.at(i)));
    if (!t.empty() && t[0] == "REACTIONS") break;
    names.insert(names.end(), t.begin(), t.end());
  }
  names.resize(ns);
  Species &s = cd.spec;
  s.n_spec = ns;
  const auto th = lines_of(join(input_dir, par.get_string("therm_file")), true);
  size_t j = 0;
  while (!starts_with(upper(th.at(j)), "THERMO")) ++j;
  const auto glob = split(th.at(j + 1));
  s.t_low.assign(ns, std::stod(glob[0]));
  s.t_mid.assign(ns, std::stod(glob[1]));
  s.t_high.assign(ns, std::stod(glob[2]));
  s.low_temp_coeff.assign(7 * ns, 0.0);
  s.high_temp_coeff.assign(7 * ns, 0.0);
  s.mw.assign(ns, 0.0);
  j += 2;
  while (j < th.size() && !starts_with(upper(th[j]), "END")) {
    const std::string &line = th[j];
    if (strip(line).empty() || starts_with(line, "!")) {
      ++j;
      continue;
    }
    const std::string name = upper(split(cols(line, 0, 18)).at(0));
    auto it = std::find(names.begin(), names.end(), name);
    if (it == names.end()) {
      j += 4;
      continue;
    }
    const int k = (int)(it - names.begin());
    s.t_low[k] = std::stod(cols(line, 45, 55));
    s.t_high[k] = std::stod(cols(line, 55, 65));
    const std::string mid = strip(cols(line, 65, 75));
    if (!mid.empty()) s.t_mid[k] = std::stod(split(mid)[0]);
    std::map<std::string, int> comp;
    for (int q = 0; q < 4; ++q) {
      const std::string c = strip(cols(line, 24 + 5 * q, 29 + 5 * q));
      if (c.empty() || c[0] == '0') break;
      const auto t = split(c);
      comp[upper(t[0])] = std::stoi(t[1]);
    }
    double w = 0.0;
    for (const auto &e : elem_set) w += atomic_weight(e) * (comp.count(e) ? comp[e] : 0);
    s.mw[k] = w;
    auto f = [&](const std::string &l, int q) { return std::stod(cols(l, 15 * q, 15 * q + 15)); };
    const std::string &l2 = th.at(j + 1), &l3 = th.at(j + 2), &l4 = th.at(j + 3);
    double *hi = &s.high_temp_coeff[7 * k], *lo = &s.low_temp_coeff[7 * k];
    for (int q = 0; q < 5; ++q) hi[q] = f(l2, q);
    hi[5] = f(l3, 0), hi[6] = f(l3, 1), lo[0] = f(l3, 2), lo[1] = f(l3, 3), lo[2] = f(l3, 4);
    lo[3] = f(l4, 0), lo[4] = f(l4, 1), lo[5] = f(l4, 2), lo[6] = f(l4, 3);
    j += 4;
  }
  s.LJ_potent_inv.assign(ns, 0.0);
  s.vis_coeff.assign(ns, 0.0);
  for (const std::string &line : lines_of(join(input_dir, par.get_string("transport_file")), true)) {
    const auto t = split(upper(line));
    if (t.empty() || starts_with(t[0], "END")) continue;
    auto it = std::find(names.begin(), names.end(), t[0]);
    if (it == names.end()) continue;
    const int k = (int)(it - names.begin());
    const double eps = std::stod(t[2]), sig = std::stod(t[3]);
    s.LJ_potent_inv[k] = 1.0 / eps;
    s.vis_coeff[k] = 2.6693e-6 * std::sqrt(s.mw[k]) / (sig * sig);
  }
  s.WjDivWi_to_One4th.assign(ns * ns, 0.0);
  s.sqrt_WiDivWjPl1Mul8.assign(ns * ns, 0.0);
  for (int a = 0; a < ns; ++a)
    for (int b = 0; b < ns; ++b) {
      s.WjDivWi_to_One4th[a * ns + b] = std::pow(s.mw[b] / s.mw[a], 0.25);
      s.sqrt_WiDivWjPl1Mul8[a * ns + b] = 1.0 / std::sqrt(8 * (1 + s.mw[a] / s.mw[b]));
    }
  s.names = names;
  return cd;
}

// Mesh.cpp:566-923 and the condition files: the blocks of "grid   0.grd" with
// their ghost grid (reflection across the faces, interface ghosts from the
// neighbour, parallelogram edges and corners), Jacobian and metrics by the
// central differences of Mesh.cpp:226-488 over the ngg-ghosted box, the raw
// records of "boundary   0.txt" and "inner   0.txt", the conditions of the
// labels the boundary file uses (5_boundary_condition.txt, 6_inflow.txt,
// 7_wall.txt; BoundCond.cu:315-409, BoundCond.cpp:10-137), and the initial
// state of the first group of 8_initialization.txt on every point.
inline Mesh read_mesh(const std::string &input_dir, const Parameter &par, const ChemData &chem,
                      bool reference_ghosts = false) {
  using namespace io_detail;
  const int ngg = par.get_int("ngg"), g = ngg + 1;
  const Species &sp = chem.spec;
  // grid
  const auto gl = lines_of(join(join(input_dir, "grid"), numbered("grid", ".grd")), true);
  const int nb = std::stoi(split(gl.at(0))[0]);
  std::vector<std::array<int, 3>> dims(nb);
  for (int b = 0; b < nb; ++b) {
    const auto t = split(gl.at(1 + b));
    dims[b] = {std::stoi(t[0]), std::stoi(t[1]), std::stoi(t[2])};
  }
  std::vector<double> vals;
  for (size_t l = 1 + nb; l < gl.size(); ++l)
    for (const auto &w : split(gl[l])) vals.push_back(std::stod(w));
  // coordinates on the g-ghosted box, X[q][(k+g)*(ny)*(nx) + (j+g)*nx + (i+g)]
  struct G3 {
    int mx, my, mz, nx, ny, nz;
    std::vector<double> X[3];
    double &at(int q, int i, int j, int k) { return X[q][((size_t)(k + g_) * ny + (j + g_)) * nx + (i + g_)]; }
    int g_;
  };
  std::vector<G3> blk(nb);
  size_t off = 0;
  for (int b = 0; b < nb; ++b) {
    G3 &B = blk[b];
    B.mx = dims[b][0], B.my = dims[b][1], B.mz = dims[b][2], B.g_ = g;
    B.nx = B.mx + 2 * g, B.ny = B.my + 2 * g, B.nz = B.mz + 2 * g;
    const size_t n = (size_t)B.mx * B.my * B.mz;
    for (int q = 0; q < 3; ++q) {
      B.X[q].assign((size_t)B.nx * B.ny * B.nz, 0.0);
      for (int k = 0; k < B.mz; ++k)
        for (int j = 0; j < B.my; ++j)
          for (int i = 0; i < B.mx; ++i) B.at(q, i, j, k) = vals.at(off + q * n + ((size_t)k * B.my + j) * B.mx + i);
    }
    off += 3 * n;
  }
  const bool dim3 = dims[0][2] > 1;
  // boundary and interface records
  const auto bl = lines_of(join(join(input_dir, "boundary_condition"), numbered("boundary", ".txt")), true);
  Mesh mesh;
  mesh.blocks.resize(nb);
  size_t li = 0;
  for (int b = 0; b < nb; ++b) {
    const int n = std::stoi(split(bl.at(li++))[0]);
    for (int r = 0; r < n; ++r) {
      const auto t = split(bl.at(li++));
      std::array<int, 7> raw{};
      for (int q = 0; q < 7; ++q) raw[q] = std::stoi(t.at(q));
      mesh.blocks[b].boundary.push_back(raw);
    }
  }
  const auto il = lines_of(join(join(input_dir, "boundary_condition"), numbered("inner", ".txt")), false);
  if (!il.empty()) {
    const auto counts = split(il.at(0));
    size_t r = 2;
    for (int b = 0; b < nb; ++b)
      for (int f = 0; f < std::stoi(counts.at(b)); ++f) {
        const auto a = split(il.at(r++)), t = split(il.at(r++));
        std::array<int, 13> raw{};
        for (int q = 0; q < 6; ++q) raw[q] = std::stoi(a.at(q));
        for (int q = 0; q < 7; ++q) raw[6 + q] = std::stoi(t.at(q));
        mesh.blocks[b].inner_face.push_back(raw);
      }
  }
  // ghost layers by reflection across the faces
  for (int b = 0; b < nb; ++b) {
    G3 &B = blk[b];
    const int mx = B.mx, my = B.my, mz = B.mz;
    for (int q = 0; q < 3; ++q) {
      for (int k = 0; k < mz; ++k)
        for (int j = 0; j < my; ++j) {
          for (int i = -1; i >= -g; --i) B.at(q, i, j, k) = 2 * B.at(q, 0, j, k) - B.at(q, -i, j, k);
          for (int i = mx; i < mx + g; ++i) B.at(q, i, j, k) = 2 * B.at(q, mx - 1, j, k) - B.at(q, 2 * (mx - 1) - i, j, k);
        }
      for (int k = 0; k < mz; ++k)
        for (int i = 0; i < mx; ++i) {
          for (int j = -1; j >= -g; --j) B.at(q, i, j, k) = 2 * B.at(q, i, 0, k) - B.at(q, i, -j, k);
          for (int j = my; j < my + g; ++j) B.at(q, i, j, k) = 2 * B.at(q, i, my - 1, k) - B.at(q, i, 2 * (my - 1) - j, k);
        }
      for (int j = 0; j < my; ++j)
        for (int i = 0; i < mx; ++i) {
          for (int k = -1; k >= -g; --k)
            B.at(q, i, j, k) = dim3 ? 2 * B.at(q, i, j, 0) - B.at(q, i, j, -k) : B.at(q, i, j, 0) + (q == 2 ? k : 0);
          for (int k = mz; k < mz + g; ++k)
            B.at(q, i, j, k) = dim3 ? 2 * B.at(q, i, j, mz - 1) - B.at(q, i, j, 2 * (mz - 1) - k)
                                    : B.at(q, i, j, mz - 1) + (q == 2 ? (k - mz + 1) : 0);
        }
    }
  }
  // interface ghosts from the neighbour (Mesh.cpp:874-923)
  for (int b = 0; b < nb; ++b)
    for (const auto &raw : mesh.blocks[b].inner_face) {
      cc_inner_face fc;
      check(cc_register_inner_face(raw.data(), ngg, &fc), "cc_register_inner_face");
      G3 &nbk = blk[fc.target_block];
      int mn[3], mxr[3], mt[3], ld[3], tld[3], st[3];
      for (int a = 0; a < 3; ++a)
        mn[a] = fc.range_start[a], mxr[a] = fc.range_end[a], mt[a] = fc.target_start[a], ld[a] = fc.loop_dir[a],
        tld[a] = fc.target_loop_dir[a], st[a] = fc.src_tar[a];
      const int shift = fc.direction < 0 ? -1 : 1;
      mn[fc.face] += shift, mxr[fc.face] += shift;
      mt[fc.target_face] += fc.target_direction > 0 ? -1 : 1;
      // translation between the coincident face layers, at a point of this
      // block's face layer with interior tangential indices
      int pt[3], dd[3], tp[3];
      for (int a = 0; a < 3; ++a)
        pt[a] = std::min(std::max((fc.range_start[a] + fc.range_end[a]) / 2, 0), dims[b][a] - 1);
      pt[fc.face] = fc.direction < 0 ? fc.range_end[fc.face] : fc.range_start[fc.face];
      for (int a = 0; a < 3; ++a) dd[a] = pt[a] - fc.range_start[a];
      for (int a = 0; a < 3; ++a) tp[a] = fc.target_start[a] + tld[a] * dd[st[a]];
      double shift_xyz[3];
      for (int q = 0; q < 3; ++q)
        shift_xyz[q] = reference_ghosts ? 0.0 : blk[b].at(q, pt[0], pt[1], pt[2]) - nbk.at(q, tp[0], tp[1], tp[2]);
      for (int i1 = mn[0]; ld[0] * (i1 - mxr[0]) != 1; i1 += ld[0])
        for (int j1 = mn[1]; ld[1] * (j1 - mxr[1]) != 1; j1 += ld[1])
          for (int k1 = mn[2]; ld[2] * (k1 - mxr[2]) != 1; k1 += ld[2]) {
            const int di[3] = {i1 - mn[0], j1 - mn[1], k1 - mn[2]};
            const int i2 = mt[0] + tld[0] * di[st[0]], j2 = mt[1] + tld[1] * di[st[1]], k2 = mt[2] + tld[2] * di[st[2]];
            for (int q = 0; q < 3; ++q) blk[b].at(q, i1, j1, k1) = nbk.at(q, i2, j2, k2) + shift_xyz[q];
          }
    }
  // edges and corners by the parallelogram rule
  for (int b = 0; b < nb; ++b) {
    G3 &B = blk[b];
    const int mx = B.mx, my = B.my, mz = B.mz;
    for (int q = 0; q < 3; ++q) {
      auto A = [&](int i, int j, int k) -> double & { return B.at(q, i, j, k); };
      for (int i = 1; i <= g; ++i)
        for (int j = 1; j <= g; ++j)
          for (int k = 0; k < mz; ++k) {
            const int i1 = -i, j1 = -j, i2 = mx - 1 + i, j2 = my - 1 + j;
            A(i1, j1, k) = A(i1, 0, k) + A(0, j1, k) - A(0, 0, k);
            A(i2, j2, k) = A(i2, my - 1, k) + A(mx - 1, j2, k) - A(mx - 1, my - 1, k);
            A(i1, j2, k) = A(i1, my - 1, k) + A(0, j2, k) - A(0, my - 1, k);
            A(i2, j1, k) = A(i2, 0, k) + A(mx - 1, j1, k) - A(mx - 1, 0, k);
          }
      for (int i = 1; i <= g; ++i)
        for (int j = 0; j < my; ++j)
          for (int k = 1; k <= g; ++k) {
            const int i1 = -i, k1 = -k, i2 = mx - 1 + i, k2 = mz - 1 + k;
            A(i1, j, k1) = A(i1, j, 0) + A(0, j, k1) - A(0, j, 0);
            A(i2, j, k2) = A(i2, j, mz - 1) + A(mx - 1, j, k2) - A(mx - 1, j, mz - 1);
            A(i1, j, k2) = A(i1, j, mz - 1) + A(0, j, k2) - A(0, j, mz - 1);
            A(i2, j, k1) = A(i2, j, 0) + A(mx - 1, j, k1) - A(mx - 1, j, 0);
          }
      for (int i = -g; i < mx + g; ++i)
        for (int j = 1; j <= g; ++j)
          for (int k = 1; k <= g; ++k) {
            const int j1 = -j, k1 = -k, j2 = my - 1 + j, k2 = mz - 1 + k;
            A(i, j1, k1) = A(i, j1, 0) + A(i, 0, k1) - A(i, 0, 0);
            A(i, j2, k2) = A(i, j2, mz - 1) + A(i, my - 1, k2) - A(i, my - 1, mz - 1);
            A(i, j1, k2) = A(i, j1, mz - 1) + A(i, 0, k2) - A(i, 0, mz - 1);
            A(i, j2, k1) = A(i, j2, 0) + A(i, my - 1, k1) - A(i, my - 1, 0);
          }
    }
  }
  // conditions of the labels the boundary file uses
  std::set<int> labels;
  for (const auto &blkr : mesh.blocks)
    for (const auto &r : blkr.boundary) labels.insert(r[6]);
  const std::string setup = join(input_dir, "setup");
  std::map<int, int> kinds;
  for (const std::string &line : lines_of(join(setup, "5_boundary_condition.txt"), false)) {
    const auto t = split(lower(line));
    if (t.empty() || starts_with(t[0], "//")) continue;
    if (t[0] == "end") break;
    const int kind = t[0] == "wall" ? 2 : (t[0] == "inflow" ? 5 : (t[0] == "outflow" ? 6 : 0));
    if (kind && t.size() >= 3 && labels.count(std::stoi(t[2])) && !kinds.count(std::stoi(t[2])))
      kinds[std::stoi(t[2])] = kind;
  }
  for (int lab : labels)
    if (!kinds.count(lab) && (lab == 2 || lab == 5 || lab == 6)) kinds[lab] = lab;
  const auto walls = sections(join(setup, "7_wall.txt"));
  const auto inflows = sections(join(setup, "6_inflow.txt"));
  for (const auto &kv : kinds) {
    cc_bc bc{};
    if (kv.second == 5) {
      auto it = inflows.find(kv.first);
      bc = inflow_state(it == inflows.end() ? Section{} : it->second, sp);
    }
    bc.label = kv.first, bc.kind = kv.second;
    if (kv.second == 2) {
      auto it = walls.find(kv.first);
      const Section w = it == walls.end() ? Section{} : it->second;
      auto th = w.opt.find("thermal_type");
      bc.thermal_type = (th == w.opt.end() || th->second == "isothermal") ? 0 : 1;
      bc.t_wall = get(w.dbl, "temperature", 300.0);
    } else {
      bc.t_wall = 300.0;
    }
    mesh.conditions.push_back(bc);
  }
  // initial state: the first group of 8_initialization.txt
  int label = -1;
  for (const std::string &line : lines_of(join(setup, "8_initialization.txt"), false)) {
    const auto t = split(lower(line));
    if (t.size() >= 2 && t[0] == "label") {
      label = std::stoi(t[1]);
      break;
    }
  }
  const Section *sec = nullptr;
  if (label >= 0 && inflows.count(label)) sec = &inflows.at(label);
  if (!sec && !inflows.empty()) sec = &inflows.begin()->second;
  if (!sec) throw std::runtime_error("no initial state: 8_initialization.txt names no label of 6_inflow.txt");
  const cc_bc init = inflow_state(*sec, sp);
  // per block: Jacobian and metrics over the ngg-ghosted box, the uniform initial state
  for (int b = 0; b < nb; ++b) {
    G3 &B = blk[b];
    Block &out = mesh.blocks[b];
    out.mx = B.mx, out.my = B.my, out.mz = B.mz;
    const int ex = B.mx + 2 * ngg, ey = B.my + 2 * ngg, ez = B.mz + 2 * ngg;
    const size_t ng = (size_t)ex * ey * ez;
    out.jacobian.assign(ng, 0.0);
    out.metric.assign(9 * ng, 0.0);
    for (int k = -ngg; k < B.mz + ngg; ++k)
      for (int j = -ngg; j < B.my + ngg; ++j)
        for (int i = -ngg; i < B.mx + ngg; ++i) {
          auto d = [&](int q, int a) {
            const int di = a == 0, dj = a == 1, dk = a == 2;
            return (B.at(q, i + di, j + dj, k + dk) - B.at(q, i - di, j - dj, k - dk)) * 0.5;
          };
          const double dxd1 = d(0, 0), dyd1 = d(1, 0), dzd1 = d(2, 0);
          const double dxd2 = d(0, 1), dyd2 = d(1, 1), dzd2 = d(2, 1);
          const double dxd3 = d(0, 2), dyd3 = d(1, 2), dzd3 = d(2, 2);
          const double jac = dxd1 * dyd2 * dzd3 + dxd2 * dyd3 * dzd1 + dxd3 * dyd1 * dzd2 - dxd1 * dyd3 * dzd2 -
                             dxd2 * dyd1 * dzd3 - dxd3 * dyd2 * dzd1;
          const double m[9] = {(dyd2 * dzd3 - dyd3 * dzd2) / jac, (dxd3 * dzd2 - dxd2 * dzd3) / jac,
                               (dxd2 * dyd3 - dxd3 * dyd2) / jac, (dyd3 * dzd1 - dyd1 * dzd3) / jac,
                               (dxd1 * dzd3 - dxd3 * dzd1) / jac, (dxd3 * dyd1 - dxd1 * dyd3) / jac,
                               (dyd1 * dzd2 - dyd2 * dzd1) / jac, (dxd2 * dzd1 - dxd1 * dzd2) / jac,
                               (dxd1 * dyd2 - dxd2 * dyd1) / jac};
          const size_t e = ((size_t)(k + ngg) * ey + (j + ngg)) * ex + (i + ngg);
          out.jacobian[e] = jac;
          for (int r = 0; r < 9; ++r) out.metric[r * ng + e] = m[r];
        }
    const double bv0[6] = {init.density, init.u, init.v, init.w, init.pressure, init.temperature};
    out.bv.assign(6 * ng, 0.0);
    for (int f = 0; f < 6; ++f) std::fill(out.bv.begin() + f * ng, out.bv.begin() + (f + 1) * ng, bv0[f]);
    out.yk.assign((size_t)sp.n_spec * ng, 0.0);
    for (int l = 0; l < sp.n_spec; ++l) std::fill(out.yk.begin() + l * ng, out.yk.begin() + (l + 1) * ng, init.yk[l]);
  }
  return mesh;
}

}  // namespace cfd

#endif
