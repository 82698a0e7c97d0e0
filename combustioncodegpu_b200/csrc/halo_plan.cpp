// Symbolic replay of the reference's boundary / interface sequence (see
// halo_plan.h) and the face-descriptor registration of Mesh.cpp.
#include "halo_plan.h"

#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstdlib>
#include <functional>
#include <unordered_map>
#include <utility>

namespace ccb {

namespace {

int isgn(int a) { return (0 < a) - (a < 0); }

// A resolved value: kind 0 = point of the new state, 1 = previous value of a
// point, 2 = node.
struct Val {
  int kind;
  int64_t idx;
  bool operator==(const Val &o) const { return kind == o.kind && idx == o.idx; }
  bool operator!=(const Val &o) const { return !(*this == o); }
};

struct SymNode {
  int op;
  Val a, b;
  int bc;
};

class Replay {
 public:
  Replay(const std::vector<HostBlock> &blocks, const std::vector<HostBc> &bcs) : B_(blocks), bcs_(bcs) {}

  bool run(HaloPlan &plan);

 private:
  const std::vector<HostBlock> &B_;
  const std::vector<HostBc> &bcs_;
  std::unordered_map<int64_t, Val> desc_;
  std::vector<SymNode> nodes_;
  std::vector<int> inflow_node_;
  std::string err_;

 public:
  std::vector<int64_t> wall_points_;

 private:

  bool in_box(int b, int i, int j, int k) const {
    const HostBlock &h = B_[b];
    return i >= -h.g && i < h.mx + h.g && j >= -h.g && j < h.my + h.g && k >= -h.g && k < h.mz + h.g;
  }
  bool interior(int b, int i, int j, int k) const {
    const HostBlock &h = B_[b];
    return i >= 0 && i < h.mx && j >= 0 && j < h.my && k >= 0 && k < h.mz;
  }
  int64_t pt(int b, int i, int j, int k) const {
    const HostBlock &h = B_[b];
    return h.base + i + (int64_t)h.nx * j + (int64_t)h.nx * h.ny * k;
  }
  Val dflt(int b, int i, int j, int k) const {
    return Val{interior(b, i, j, k) ? 0 : 1, pt(b, i, j, k)};
  }
  bool get(int b, int i, int j, int k, Val &v) {
    if (!in_box(b, i, j, k)) {
      err_ = "face range reaches outside the ghosted box of block " + std::to_string(b);
      return false;
    }
    auto it = desc_.find(pt(b, i, j, k));
    v = it == desc_.end() ? dflt(b, i, j, k) : it->second;
    return true;
  }
  Val node(int op, Val a, Val b, int bc) {
    nodes_.push_back(SymNode{op, a, b, bc});
    return Val{2, (int64_t)nodes_.size() - 1};
  }
  struct Write {
    int b, i, j, k;
    Val v;
  };
  bool apply(const std::vector<Write> &w) {
    for (const auto &x : w) {
      if (!in_box(x.b, x.i, x.j, x.k)) {
        err_ = "face writes outside the ghosted box of block " + std::to_string(x.b);
        return false;
      }
      desc_[pt(x.b, x.i, x.j, x.k)] = x.v;
    }
    return true;
  }
  bool face_bc(int b, const HostBoundary &f, int c);
  bool face_inner(int b, const HostInnerFace &f);
};

// BoundCond.cu:455-487 (outflow), 489-527 (inflow), 529-629 (wall).
bool Replay::face_bc(int b, const HostBoundary &f, int c) {
  const HostBc &bc = bcs_[c];
  int dir[3] = {0, 0, 0};
  dir[f.face] = f.direction;
  std::vector<Write> w;
  const int g = B_[b].g;
  for (int k = f.range_start[2]; k <= f.range_end[2]; ++k)
    for (int j = f.range_start[1]; j <= f.range_end[1]; ++j)
      for (int i = f.range_start[0]; i <= f.range_end[0]; ++i) {
        if (bc.kind == 6) {
          Val v;
          if (!get(b, i, j, k, v)) return false;
          for (int gg = 1; gg <= g; ++gg) w.push_back({b, i + gg * dir[0], j + gg * dir[1], k + gg * dir[2], v});
        } else if (bc.kind == 5) {
          if (inflow_node_[c] < 0) inflow_node_[c] = (int)node(kHaloInflow, Val{0, -1}, Val{0, -1}, c).idx;
          const Val v{2, inflow_node_[c]};
          for (int gg = 1; gg <= g; ++gg) w.push_back({b, i + gg * dir[0], j + gg * dir[1], k + gg * dir[2], v});
        } else if (bc.kind == 2) {
          Val in1;
          if (!get(b, i - dir[0], j - dir[1], k - dir[2], in1)) return false;
          w.push_back({b, i, j, k, node(kHaloWallFace, in1, in1, c)});
          if (interior(b, i, j, k)) wall_points_.push_back(pt(b, i, j, k));
          for (int gg = 1; gg <= g; ++gg) {
            Val mir;
            if (!get(b, i - gg * dir[0], j - gg * dir[1], k - gg * dir[2], mir)) return false;
            w.push_back({b, i + gg * dir[0], j + gg * dir[1], k + gg * dir[2], node(kHaloWallGhost, mir, in1, c)});
          }
        }
      }
  return apply(w);
}

// Field.cu:213-266 inner_communication: average on the coincident layer,
// copy from the target elsewhere (every point of the face range once).
bool Replay::face_inner(int b, const HostInnerFace &f) {
  const int tb = f.target_block;
  if (tb < 0 || tb >= (int)B_.size()) {
    err_ = "inner face of block " + std::to_string(b) + " targets a missing block";
    return false;
  }
  int np[3];
  for (int d = 0; d < 3; ++d) np[d] = std::abs(f.range_start[d] - f.range_end[d]) + 1;
  const int face_dir = f.direction > 0 ? f.range_start[f.face] : f.range_end[f.face];
  std::vector<Write> w;
  for (int n2 = 0; n2 < np[2]; ++n2)
    for (int n1 = 0; n1 < np[1]; ++n1)
      for (int n0 = 0; n0 < np[0]; ++n0) {
        const int n[3] = {n0, n1, n2};
        int idx[3], it[3];
        for (int d = 0; d < 3; ++d) {
          const int d_idx = f.loop_dir[d] * n[d];
          idx[d] = f.range_start[d] + d_idx;
          it[d] = f.target_start[d] + f.target_loop_dir[d] * d_idx;
        }
        Val vt;
        if (!get(tb, it[0], it[1], it[2], vt)) return false;
        if (idx[f.face] == face_dir) {
          Val vz;
          if (!get(b, idx[0], idx[1], idx[2], vz)) return false;
          // 0.5*(x+x) == x exactly, so an average of one value is that value
          const Val v = (vz == vt) ? vz : node(kHaloAvg, vt, vz, -1);
          w.push_back({b, idx[0], idx[1], idx[2], v});
          w.push_back({tb, it[0], it[1], it[2], v});
        } else {
          w.push_back({b, idx[0], idx[1], idx[2], vt});
        }
      }
  return apply(w);
}

bool Replay::run(HaloPlan &plan) {
  inflow_node_.assign(bcs_.size(), -1);
  const int kinds[3] = {6, 5, 2};
  for (int kk = 0; kk < 3; ++kk)
    for (size_t c = 0; c < bcs_.size(); ++c) {
      if (bcs_[c].kind != kinds[kk]) continue;
      if (kinds[kk] == 2) plan.has_wall = true;
      for (size_t b = 0; b < B_.size(); ++b)
        for (const auto &f : B_[b].bnd)
          if (f.type_label == bcs_[c].label && !face_bc((int)b, f, (int)c)) {
            plan.error = err_;
            return false;
          }
    }
  for (size_t b = 0; b < B_.size(); ++b)
    for (const auto &f : B_[b].inf)
      if (!face_inner((int)b, f)) {
        plan.error = err_;
        return false;
      }

  // changed points, in arena order (coalesced phase-B writes)
  std::vector<std::pair<int64_t, Val>> changed;
  changed.reserve(desc_.size());
  std::unordered_map<int64_t, char> overwritten;
  for (const auto &kv : desc_) {
    const Val &v = kv.second;
    const bool same_as_default = (v.kind == 0 || v.kind == 1) && v.idx == kv.first;
    if (!same_as_default) {
      changed.push_back(kv);
      overwritten[kv.first] = 1;
    }
  }
  std::sort(changed.begin(), changed.end(),
            [](const std::pair<int64_t, Val> &a, const std::pair<int64_t, Val> &b) { return a.first < b.first; });

  // copy nodes that capture a point's stage value before phase B overwrites it
  std::unordered_map<int64_t, int> capture;
  auto capture_node = [&](const Val &v) {
    const int64_t key = v.idx * 2 + v.kind;
    auto it = capture.find(key);
    if (it != capture.end()) return (int64_t)it->second;
    nodes_.push_back(SymNode{kHaloCopy, v, v, -1});
    const int id = (int)nodes_.size() - 1;
    capture[key] = id;
    return (int64_t)id;
  };
  // A stage value (kind 0) or previous value (kind 1; the previous conserved
  // state may share storage with the new one) of a point that phase B also
  // writes is captured into scratch first, so phase B never reads a point it
  // writes.
  for (auto &kv : changed) {
    if ((kv.second.kind == 0 || kv.second.kind == 1) && overwritten.count(kv.second.idx))
      kv.second = Val{2, capture_node(kv.second)};
  }

  // live nodes and their levels
  const int nn = (int)nodes_.size();
  std::vector<int> level(nn, -2);  // -2 = not live
  std::function<int(int)> lev = [&](int id) -> int {
    if (level[id] >= 0) return level[id];
    if (level[id] == -3) return 0;  // cycles cannot occur; defensive
    level[id] = -3;
    int L = 0;
    const SymNode &sn = nodes_[id];
    const bool two = sn.op == kHaloAvg || sn.op == kHaloWallGhost;
    const bool one = sn.op != kHaloInflow;
    if (one && sn.a.kind == 2) L = std::max(L, lev((int)sn.a.idx) + 1);
    if (two && sn.b.kind == 2) L = std::max(L, lev((int)sn.b.idx) + 1);
    level[id] = L;
    return L;
  };
  int max_level = -1;
  for (const auto &kv : changed)
    if (kv.second.kind == 2) max_level = std::max(max_level, lev((int)kv.second.idx));
  for (int id = 0; id < nn; ++id)
    if (level[id] >= 0) max_level = std::max(max_level, level[id]);

  // Scratch slots follow the destination order of phase B: each node is
  // placed by the smallest destination index among the copies that read it,
  // handed down to the lower-level nodes it reads, so that consecutive
  // copies read consecutive slots.
  std::vector<int64_t> pos(nn, INT64_MAX);
  for (const auto &kv : changed)
    if (kv.second.kind == 2) pos[kv.second.idx] = std::min(pos[kv.second.idx], kv.first);
  for (int L = max_level; L > 0; --L)
    for (int id = 0; id < nn; ++id) {
      if (level[id] != L) continue;
      const SymNode &sn = nodes_[id];
      const bool two = sn.op == kHaloAvg || sn.op == kHaloWallGhost;
      if (sn.op != kHaloInflow && sn.a.kind == 2) pos[sn.a.idx] = std::min(pos[sn.a.idx], pos[id]);
      if (two && sn.b.kind == 2) pos[sn.b.idx] = std::min(pos[sn.b.idx], pos[id]);
    }
  std::vector<int> order;
  for (int id = 0; id < nn; ++id)
    if (level[id] >= 0) order.push_back(id);
  std::sort(order.begin(), order.end(), [&](int a, int b) {
    if (level[a] != level[b]) return level[a] < level[b];
    if (pos[a] != pos[b]) return pos[a] < pos[b];
    return a < b;
  });
  std::vector<int64_t> slot(nn, -1);
  for (size_t s = 0; s < order.size(); ++s) slot[order[s]] = (int64_t)s;
  plan.n_slots = (int64_t)order.size();

  auto to_ref = [&](const Val &v) {
    HaloRef r;
    r.pad = 0;
    if (v.kind == 2) {
      r.kind = 2;
      r.idx = slot[v.idx];
    } else {
      r.kind = v.kind;
      r.idx = v.idx;
    }
    return r;
  };
  plan.nodes.clear();
  plan.level_begin.assign(1, 0);
  int cur = 0;
  for (size_t s = 0; s < order.size(); ++s) {
    const int id = order[s];
    while (level[id] > cur) {
      plan.level_begin.push_back((int64_t)plan.nodes.size());
      ++cur;
    }
    const SymNode &sn = nodes_[id];
    HaloNode hn;
    hn.slot = (int64_t)s;
    hn.op = sn.op;
    hn.bc = sn.bc;
    hn.a = sn.op == kHaloInflow ? HaloRef{0, 0, 0} : to_ref(sn.a);
    hn.b = (sn.op == kHaloAvg || sn.op == kHaloWallGhost) ? to_ref(sn.b) : hn.a;
    plan.nodes.push_back(hn);
  }
  plan.level_begin.push_back((int64_t)plan.nodes.size());
  if (order.empty()) plan.level_begin.assign(1, 0);
  std::sort(wall_points_.begin(), wall_points_.end());
  wall_points_.erase(std::unique(wall_points_.begin(), wall_points_.end()), wall_points_.end());
  plan.vel_zero = wall_points_;
  plan.copies.clear();
  plan.interior_copies.clear();
  plan.copies.reserve(changed.size());
  for (const auto &kv : changed) {
    HaloCopy hc{kv.first, to_ref(kv.second)};
    // locate the block of the destination (blocks are contiguous in the arena)
    int flags = 0;
    for (size_t b = 0; b < B_.size(); ++b) {
      const HostBlock &h = B_[b];
      const int64_t r = kv.first - h.off;
      if (r < 0 || r >= (int64_t)h.nx * h.ny * h.nz) continue;
      const int i = (int)(r % h.nx) - h.g, j = (int)((r / h.nx) % h.ny) - h.g, k = (int)(r / ((int64_t)h.nx * h.ny)) - h.g;
      if (interior((int)b, i, j, k)) flags |= 1;
      if (h.mz > 1) flags |= 2;
      break;
    }
    hc.src.pad = flags;
    if (flags & 1) plan.interior_copies.push_back((int64_t)plan.copies.size());
    plan.copies.push_back(hc);
  }
  // bit 2: the destination is read by the program itself as a stage or
  // previous value (a node operand or a copy source), so its every value
  // matters, not only the last one
  std::unordered_map<int64_t, char> read;
  for (const auto &hn : plan.nodes) {
    if (hn.a.kind == 0 || hn.a.kind == 1) read[hn.a.idx] = 1;
    if (hn.b.kind == 0 || hn.b.kind == 1) read[hn.b.idx] = 1;
  }
  for (const auto &hc : plan.copies)
    if (hc.src.kind == 0 || hc.src.kind == 1) read[hc.src.idx] = 1;
  for (auto &hc : plan.copies)
    if (read.count(hc.dst)) hc.src.pad |= 4;
  return true;
}

}  // namespace

bool build_halo_plan(const std::vector<HostBlock> &blocks, const std::vector<HostBc> &bcs, HaloPlan &plan) {
  Replay r(blocks, bcs);
  return r.run(plan);
}

void register_boundary(const int raw[7], int ngg, HostBoundary &b) {
  b.range_start[0] = raw[0], b.range_end[0] = raw[1];
  b.range_start[1] = raw[2], b.range_end[1] = raw[3];
  b.range_start[2] = raw[4], b.range_end[2] = raw[5];
  b.type_label = raw[6];
  b.face = 0;
  b.direction = 1;
  for (int i = 0; i < 3; ++i) {
    if (b.range_start[i] == b.range_end[i]) {
      b.face = i;
      if (b.range_start[i] == 0) b.direction = -1;
      break;
    }
  }
  for (int i = 0; i < 3; ++i) {
    if (i == b.face) continue;
    if (b.range_end[i] < b.range_start[i]) std::swap(b.range_end[i], b.range_start[i]);
    b.range_start[i] -= ngg;
    b.range_end[i] += ngg;
  }
}

void register_inner_face(const int raw[13], int ngg, HostInnerFace &f) {
  f.range_start[0] = raw[0], f.range_end[0] = raw[1];
  f.range_start[1] = raw[2], f.range_end[1] = raw[3];
  f.range_start[2] = raw[4], f.range_end[2] = raw[5];
  f.target_start[0] = raw[6], f.target_end[0] = raw[7];
  f.target_start[1] = raw[8], f.target_end[1] = raw[9];
  f.target_start[2] = raw[10], f.target_end[2] = raw[11];
  f.target_block = raw[12] - 1;
  f.face = 0, f.direction = 1, f.target_face = 0, f.target_direction = 1;
  for (int i = 0; i < 3; ++i) f.src_tar[i] = 0, f.loop_dir[i] = 1, f.target_loop_dir[i] = 1;
  for (int i = 0; i < 3; ++i) {
    if (f.range_start[i] == f.range_end[i]) {
      f.face = i;
      if (f.range_start[i] == 1) f.direction = -1;
      f.range_start[i] -= 1;
      f.range_end[i] -= 1;
      break;
    }
  }
  for (int i = 0; i < 3; ++i) {
    if (f.target_start[i] == f.target_end[i]) {
      f.target_face = i;
      if (f.target_start[i] == 1) f.target_direction = -1;
      f.target_start[i] -= 1;
      f.target_end[i] -= 1;
      break;
    }
  }
  f.src_tar[f.target_face] = -(f.direction * f.target_direction) * (f.face + 1);
  int next_face = 0, target_next_face = 0;
  for (int i = 0; i < 3; ++i) {
    if (f.range_start[i] < 0) {
      next_face = i;
      f.range_start[i] = -f.range_start[i] - 1;
      f.range_end[i] = -f.range_end[i] - 1;
      break;
    }
  }
  for (int i = 0; i < 3; ++i) {
    if (f.target_start[i] < 0) {
      target_next_face = i;
      f.target_start[i] = -f.target_start[i] - 1;
      f.target_end[i] = -f.target_end[i] - 1;
      break;
    }
  }
  f.src_tar[target_next_face] =
      isgn((f.target_end[target_next_face] - f.target_start[target_next_face]) *
           (f.range_end[next_face] - f.range_start[next_face])) *
      (next_face + 1);
  next_face = 3 - f.face - next_face;
  target_next_face = 3 - f.target_face - target_next_face;
  f.range_start[next_face] -= 1;
  f.range_end[next_face] -= 1;
  f.target_start[target_next_face] -= 1;
  f.target_end[target_next_face] -= 1;
  f.src_tar[target_next_face] =
      isgn((f.target_end[target_next_face] - f.target_start[target_next_face]) *
           (f.range_end[next_face] - f.range_start[next_face])) *
      (next_face + 1);
  const int rs = f.direction < 0 ? -ngg : f.range_end[f.face];
  const int re = f.direction < 0 ? 0 : f.range_end[f.face] + ngg;
  f.range_start[f.face] = rs;
  f.range_end[f.face] = re;
  const int sgn_tar = isgn(f.src_tar[f.target_face]);
  if (f.target_direction > 0)
    f.target_start[f.target_face] = sgn_tar > 0 ? f.target_end[f.target_face] - ngg : f.target_end[f.target_face];
  else
    f.target_start[f.target_face] = sgn_tar > 0 ? 0 : ngg;
  for (int i = 0; i < 3; ++i) {
    f.loop_dir[i] = f.range_start[i] <= f.range_end[i] ? 1 : -1;
    f.target_loop_dir[i] = isgn(f.src_tar[i]);
    f.src_tar[i] = std::abs(f.src_tar[i]) - 1;
  }
  for (int i = 0; i < 3; ++i) {
    if (i != f.face) {
      f.range_start[i] -= f.loop_dir[i] * ngg;
      f.range_end[i] += f.loop_dir[i] * ngg;
      f.target_start[i] -= f.target_loop_dir[i] * f.loop_dir[i] * ngg;
      f.target_end[i] += f.target_loop_dir[i] * f.loop_dir[i] * ngg;
    }
  }
}

}  // namespace ccb
