// Host-side builder of the halo program.
//
// The reference fills ghost layers with a sequence of launches whose order
// matters: every outflow face, then every inflow face, then every wall face
// (BoundCond.cu:251-313), then every block interface in block order
// (Driver.cu:194-217, Field.cu:213-266), each face overwriting points that
// earlier faces wrote (edges and corners).  The builder replays that sequence
// symbolically once, at set-up, and records for every point that changes
// which value it finally holds:
//   - a plain copy of a point of the new state (outflow, interface copies),
//   - the previous value of a ghost nothing writes,
//   - a node: interface average, inflow state, wall point or wall ghost,
//     whose sources are again resolved values.
// At run time the program is two phases: nodes are evaluated level by level
// into scratch slots (no point is written, so every source is still
// pristine), then all changed points are written in one parallel pass.  The
// result equals the reference's sequential fill for any face order.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "cc_common.h"

namespace ccb {

struct HostBoundary {
  int range_start[3], range_end[3], type_label, face, direction;
};

struct HostInnerFace {
  int range_start[3], range_end[3], face, direction, target_start[3], target_end[3], target_block, target_face,
      target_direction, src_tar[3], loop_dir[3], target_loop_dir[3];
};

struct HostBc {
  int label, kind, thermal_type;
  double t_wall, rho, u, v, w, p, T;
  double yk[kMaxSpec];
};

struct HostBlock {
  int mx, my, mz, g;
  int nx, ny, nz;
  int64_t off, base;  // arena index of (-g,-g,-g) and of (0,0,0)
  std::vector<HostBoundary> bnd;
  std::vector<HostInnerFace> inf;
};

struct HaloPlan {
  std::vector<HaloNode> nodes;          // ordered by level
  std::vector<int64_t> level_begin;     // nodes[level_begin[l] .. level_begin[l+1])
  std::vector<HaloCopy> copies;         // phase B
  std::vector<int64_t> interior_copies; // indices of the copies that rewrite an interior point
  std::vector<int64_t> vel_zero;       // interior points a wall condition writes (DZone::vel = 0)
  int64_t n_slots = 0;
  bool has_wall = false;
  std::string error;
};

bool build_halo_plan(const std::vector<HostBlock> &blocks, const std::vector<HostBc> &bcs, HaloPlan &plan);

// Mesh.cpp:14-32 / 35-143 restated (3D).
void register_boundary(const int raw[7], int ngg, HostBoundary &out);
void register_inner_face(const int raw[13], int ngg, HostInnerFace &out);

}  // namespace ccb
