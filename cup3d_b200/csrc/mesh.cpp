// Host mesh construction: leaf lists, space-filling-curve order, face tables.
// See mesh.h for the contract and the reference call sites it replaces.
#include "mesh.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <set>
#include <sstream>

namespace cup3d {

void mesh_spec_finalize(MeshSpec& s) {
  // SimulationData::_preprocessArguments (SimulationData.cpp:134-168): the
  // finest-level cell counts fix the aspect ratio, `extent` fixes the largest.
  const int aux = 1 << (s.level_max - 1);
  const double nfe[3] = {double(s.bpd[0]) * aux * 8, double(s.bpd[1]) * aux * 8,
                         double(s.bpd[2]) * aux * 8};
  const double maxbpd = std::max({nfe[0], nfe[1], nfe[2]});
  for (int d = 0; d < 3; ++d) s.extents[d] = (nfe[d] / maxbpd) * s.extent;
  s.hmin = s.extents[0] / nfe[0];
  s.h0 = s.extents[0] * aux / nfe[0];
}

// Hilbert index of a point on a 2^bits cube (J. Skilling, "Programming the
// Hilbert curve", AIP Conf. Proc. 707, 2004: axes -> transposed form, then
// bit interleave).
static uint64_t hilbert3(uint32_t x, uint32_t y, uint32_t z, int bits) {
  if (bits <= 0) return 0;
  uint32_t X[3] = {x, y, z};
  const uint32_t M = 1u << (bits - 1);
  for (uint32_t Q = M; Q > 1; Q >>= 1) {
    const uint32_t P = Q - 1;
    for (int i = 0; i < 3; ++i) {
      if (X[i] & Q) {
        X[0] ^= P;
      } else {
        const uint32_t t = (X[0] ^ X[i]) & P;
        X[0] ^= t;
        X[i] ^= t;
      }
    }
  }
  for (int i = 1; i < 3; ++i) X[i] ^= X[i - 1];
  uint32_t t = 0;
  for (uint32_t Q = M; Q > 1; Q >>= 1)
    if (X[2] & Q) t ^= Q - 1;
  for (int i = 0; i < 3; ++i) X[i] ^= t;
  uint64_t h = 0;
  for (int b = bits - 1; b >= 0; --b)
    for (int i = 0; i < 3; ++i) h = (h << 1) | ((X[i] >> b) & 1u);
  return h;
}

static int ceil_log2(int n) {
  int b = 0;
  while ((1 << b) < n) ++b;
  return b;
}

// Sort key: Hilbert index of the level-0 root, then the Morton digits of the
// octree path below it, padded to the deepest level (leaves never nest, so
// padding with zeros keeps depth-first order).
static uint64_t sfc_key(const MeshSpec& s, int l, int i, int j, int k) {
  const int bits = ceil_log2(std::max({s.bpd[0], s.bpd[1], s.bpd[2]}));
  const uint64_t root = hilbert3(uint32_t(i >> l), uint32_t(j >> l), uint32_t(k >> l), bits);
  uint64_t path = 0;
  const int L = s.level_max - 1;
  for (int m = 1; m <= L; ++m) {
    uint64_t digit = 0;
    if (m <= l) {
      const int sh = l - m;
      digit = uint64_t((i >> sh) & 1) | (uint64_t((j >> sh) & 1) << 1) |
              (uint64_t((k >> sh) & 1) << 2);
    }
    path = (path << 3) | digit;
  }
  return (root << (3 * L)) | path;
}

bool mesh_build(const MeshSpec& spec_in, const std::vector<std::array<int32_t, 4>>& leaves,
                Mesh& m, std::string& err) {
  MeshSpec spec = spec_in;
  mesh_spec_finalize(spec);
  m = Mesh();
  m.spec = spec;
  if (spec.level_max < 1 || spec.level_max > 12) {
    err = "levelMax out of range [1,12]";
    return false;
  }
  for (int d = 0; d < 3; ++d)
    if (spec.bpd[d] < 1 || spec.bpd[d] > (1 << 16)) {
      err = "bpd out of range";
      return false;
    }
  // validate and sort
  std::vector<std::pair<uint64_t, std::array<int32_t, 4>>> keyed;
  keyed.reserve(leaves.size());
  double volume = 0;
  std::unordered_map<uint64_t, int32_t> tmp;
  for (const auto& b : leaves) {
    const int l = b[0];
    if (l < 0 || l >= spec.level_max) {
      err = "block level out of range";
      return false;
    }
    for (int d = 0; d < 3; ++d)
      if (b[1 + d] < 0 || b[1 + d] >= (spec.bpd[d] << l)) {
        err = "block index out of range";
        return false;
      }
    if (!tmp.emplace(Mesh::key(l, b[1], b[2], b[3]), 1).second) {
      err = "duplicate block";
      return false;
    }
    volume += std::ldexp(1.0, -3 * l);
    keyed.push_back({sfc_key(spec, l, b[1], b[2], b[3]), b});
  }
  // no leaf may contain another leaf
  for (const auto& b : leaves)
    for (int l2 = 0; l2 < b[0]; ++l2) {
      const int sh = b[0] - l2;
      if (tmp.count(Mesh::key(l2, b[1] >> sh, b[2] >> sh, b[3] >> sh))) {
        err = "overlapping blocks";
        return false;
      }
    }
  const double want = double(spec.bpd[0]) * spec.bpd[1] * spec.bpd[2];
  if (std::fabs(volume - want) > 1e-9 * want) {
    err = "blocks do not tile the domain";
    return false;
  }
  std::stable_sort(keyed.begin(), keyed.end(),
                   [](const auto& a, const auto& b) { return a.first < b.first; });
  const int nb = int(keyed.size());
  m.nb = nb;
  m.level.resize(nb);
  m.index.resize(3 * nb);
  m.h.resize(nb);
  m.origin.resize(3 * nb);
  for (int b = 0; b < nb; ++b) {
    const auto& e = keyed[b].second;
    m.level[b] = e[0];
    m.max_level_used = std::max(m.max_level_used, int(e[0]));
    for (int d = 0; d < 3; ++d) m.index[3 * b + d] = e[1 + d];
    m.h[b] = std::ldexp(spec.h0, -e[0]);
    for (int d = 0; d < 3; ++d) m.origin[3 * b + d] = e[1 + d] * 8 * m.h[b];
    m.lookup[Mesh::key(e[0], e[1], e[2], e[3])] = b;
    if (e[1] == 0 && e[2] == 0 && e[3] == 0) m.mean_block = b;
  }
  // faces
  m.face_kind.assign(6 * nb, FACE_BOUNDARY);
  m.face_nbr.assign(24 * nb, -1);
  for (int b = 0; b < nb; ++b) {
    const int l = m.level[b];
    for (int d = 0; d < 3; ++d)
      for (int side = 0; side < 2; ++side) {
        const int f = 2 * d + side;
        int n[3] = {m.index[3 * b], m.index[3 * b + 1], m.index[3 * b + 2]};
        n[d] += side ? 1 : -1;
        const int N = spec.bpd[d] << l;
        int32_t* nbr = &m.face_nbr[24 * b + 4 * f];
        if (n[d] < 0 || n[d] >= N) {
          if (spec.bc[d] == BC_PERIODIC) {
            n[d] = (n[d] + N) % N;
          } else {
            m.face_kind[6 * b + f] = FACE_BOUNDARY;
            nbr[0] = spec.bc[d];
            continue;
          }
        }
        const int same = m.find(l, n[0], n[1], n[2]);
        if (same >= 0) {
          m.face_kind[6 * b + f] = FACE_SAME;
          nbr[0] = same;
          continue;
        }
        if (l > 0) {
          const int coarse = m.find(l - 1, n[0] >> 1, n[1] >> 1, n[2] >> 1);
          if (coarse >= 0) {
            m.face_kind[6 * b + f] = FACE_COARSER;
            nbr[0] = coarse;
            continue;
          }
        }
        // finer: the four children of the same-level position touching us
        const int t1 = tan1(d), t2 = tan2(d);
        bool ok = l + 1 < spec.level_max;
        for (int bb = 0; bb < 2 && ok; ++bb)
          for (int aa = 0; aa < 2 && ok; ++aa) {
            int c[3];
            c[d] = 2 * n[d] + (side == 0 ? 1 : 0);
            c[t1] = 2 * n[t1] + aa;
            c[t2] = 2 * n[t2] + bb;
            const int id = m.find(l + 1, c[0], c[1], c[2]);
            if (id < 0) ok = false;
            nbr[aa + 2 * bb] = id;
          }
        if (!ok) {
          std::ostringstream os;
          os << "2:1 balance violated at block (" << l << "," << m.index[3 * b] << ","
             << m.index[3 * b + 1] << "," << m.index[3 * b + 2] << ") face " << f;
          err = os.str();
          return false;
        }
        m.face_kind[6 * b + f] = FACE_FINER;
      }
  }
  return true;
}

namespace {
struct LeafSet {
  MeshSpec spec;
  std::set<std::array<int32_t, 4>> leaves;
  bool has(int l, int i, int j, int k) const { return leaves.count({l, i, j, k}) != 0; }
  void split(const std::array<int32_t, 4>& b) {
    leaves.erase(b);
    for (int c = 0; c < 8; ++c)
      leaves.insert({b[0] + 1, 2 * b[1] + (c & 1), 2 * b[2] + ((c >> 1) & 1),
                     2 * b[3] + ((c >> 2) & 1)});
  }
  // Leaf at level <= l containing the level-l position p, or level -1.
  std::array<int32_t, 4> covering(int l, const int p[3]) const {
    for (int l2 = l; l2 >= 0; --l2) {
      const int sh = l - l2;
      if (has(l2, p[0] >> sh, p[1] >> sh, p[2] >> sh))
        return {l2, p[0] >> sh, p[1] >> sh, p[2] >> sh};
    }
    return {-1, 0, 0, 0};
  }
  void balance() {
    bool changed = true;
    while (changed) {
      changed = false;
      std::vector<std::array<int32_t, 4>> to_split;
      for (const auto& b : leaves) {
        const int l = b[0];
        if (l < 2) continue;
        for (int dz = -1; dz <= 1; ++dz)
          for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
              if (!dx && !dy && !dz) continue;
              int p[3] = {b[1] + dx, b[2] + dy, b[3] + dz};
              bool inside = true;
              for (int d = 0; d < 3; ++d) {
                const int N = spec.bpd[d] << l;
                if (p[d] < 0 || p[d] >= N) {
                  if (spec.bc[d] == BC_PERIODIC)
                    p[d] = (p[d] + N) % N;
                  else
                    inside = false;
                }
              }
              if (!inside) continue;
              const auto c = covering(l, p);
              if (c[0] >= 0 && c[0] < l - 1) to_split.push_back(c);
            }
      }
      std::sort(to_split.begin(), to_split.end());
      to_split.erase(std::unique(to_split.begin(), to_split.end()), to_split.end());
      for (const auto& c : to_split)
        if (leaves.count(c)) {
          split(c);
          changed = true;
        }
    }
  }
};
}  // namespace

std::vector<std::array<int32_t, 4>> mesh_adapt_leaves(const Mesh& m, const std::vector<uint8_t>& refine,
                                                      const std::vector<uint8_t>& compress) {
  LeafSet ls;
  ls.spec = m.spec;
  for (int b = 0; b < m.nb; ++b) ls.leaves.insert({m.level[b], m.index[3 * b], m.index[3 * b + 1], m.index[3 * b + 2]});
  // refinement first, then the 2:1 balance it needs
  std::vector<std::array<int32_t, 4>> split;
  for (int b = 0; b < m.nb; ++b)
    if (refine[b] && m.level[b] + 1 < m.spec.level_max)
      split.push_back({m.level[b], m.index[3 * b], m.index[3 * b + 1], m.index[3 * b + 2]});
  for (const auto& b : split) ls.split(b);
  ls.balance();
  // compression: a parent whose eight children are leaves that all compress,
  // unless a leaf finer than the children touches the parent's region (the
  // merged block would then sit two levels above a neighbour)
  std::map<std::array<int32_t, 4>, int> votes;
  for (int b = 0; b < m.nb; ++b) {
    const int l = m.level[b];
    if (!compress[b] || refine[b] || l == 0) continue;
    const std::array<int32_t, 4> me{l, m.index[3 * b], m.index[3 * b + 1], m.index[3 * b + 2]};
    if (!ls.leaves.count(me)) continue;  // split by the balance
    ++votes[{l - 1, me[1] >> 1, me[2] >> 1, me[3] >> 1}];
  }
  std::vector<std::array<int32_t, 4>> merge;
  for (const auto& [p, n] : votes) {
    if (n != 8) continue;
    const int l = p[0] + 1;  // the children's level
    bool ok = true;
    for (int dz = -1; dz <= 1 && ok; ++dz)
      for (int dy = -1; dy <= 1 && ok; ++dy)
        for (int dx = -1; dx <= 1 && ok; ++dx) {
          if (!dx && !dy && !dz) continue;
          int q[3] = {p[1] + dx, p[2] + dy, p[3] + dz};
          bool inside = true;
          for (int d = 0; d < 3; ++d) {
            const int N = m.spec.bpd[d] << p[0];
            if (q[d] < 0 || q[d] >= N) {
              if (m.spec.bc[d] == BC_PERIODIC)
                q[d] = (q[d] + N) % N;
              else
                inside = false;
            }
          }
          if (!inside) continue;
          // the neighbour position's eight level-l parts must be covered at level <= l
          for (int c = 0; c < 8 && ok; ++c) {
            const int cp[3] = {2 * q[0] + (c & 1), 2 * q[1] + ((c >> 1) & 1), 2 * q[2] + (c >> 2)};
            ok = ls.covering(l, cp)[0] >= 0;
          }
        }
    if (ok) merge.push_back(p);
  }
  for (const auto& p : merge) {
    for (int c = 0; c < 8; ++c)
      ls.leaves.erase({p[0] + 1, 2 * p[1] + (c & 1), 2 * p[2] + ((c >> 1) & 1), 2 * p[3] + (c >> 2)});
    ls.leaves.insert(p);
  }
  return std::vector<std::array<int32_t, 4>>(ls.leaves.begin(), ls.leaves.end());
}

std::vector<std::array<int32_t, 4>> mesh_refine_leaves(
    const MeshSpec& spec_in, const std::function<bool(int, const double*, const double*)>& tag) {
  MeshSpec spec = spec_in;
  mesh_spec_finalize(spec);
  LeafSet ls;
  ls.spec = spec;
  for (int k = 0; k < spec.bpd[2]; ++k)
    for (int j = 0; j < spec.bpd[1]; ++j)
      for (int i = 0; i < spec.bpd[0]; ++i) ls.leaves.insert({0, i, j, k});
  for (int l = 0; l + 1 < spec.level_max; ++l) {
    std::vector<std::array<int32_t, 4>> cur;
    for (const auto& b : ls.leaves)
      if (b[0] == l) cur.push_back(b);
    const double hb = std::ldexp(spec.h0, -l) * 8;
    for (const auto& b : cur) {
      const double lo[3] = {b[1] * hb, b[2] * hb, b[3] * hb};
      const double hi[3] = {lo[0] + hb, lo[1] + hb, lo[2] + hb};
      if (tag(l, lo, hi)) ls.split(b);
    }
    ls.balance();
  }
  ls.balance();
  return std::vector<std::array<int32_t, 4>>(ls.leaves.begin(), ls.leaves.end());
}

static double box_point_dist(const double* lo, const double* hi, const double* p) {
  double s = 0;
  for (int d = 0; d < 3; ++d) {
    const double e = std::max({lo[d] - p[d], 0.0, p[d] - hi[d]});
    s += e * e;
  }
  return std::sqrt(s);
}

std::vector<std::array<int32_t, 4>> mesh_sphere_wake_leaves(
    const MeshSpec& spec, const double c[3], double r, int flow_dir, double near_radius,
    double wake_len, double wake_radius) {
  auto tag = [&](int l, const double* lo, const double* hi) {
    const double scale = std::ldexp(1.0, -l);
    // near field: within near_radius * 2^-l of the body surface
    if (box_point_dist(lo, hi, c) < r + near_radius * scale) return true;
    // wake: distance to the downstream segment
    const double x0 = c[0], x1 = c[0] + flow_dir * wake_len;
    const double xa = std::min(x0, x1), xb = std::max(x0, x1);
    double s = 0;
    const double ex = std::max({xa - hi[0], 0.0, lo[0] - xb});
    s += ex * ex;
    for (int d = 1; d < 3; ++d) {
      const double e = std::max({lo[d] - c[d], 0.0, c[d] - hi[d]});
      s += e * e;
    }
    return std::sqrt(s) < wake_radius * scale;
  };
  return mesh_refine_leaves(spec, tag);
}

std::vector<std::array<int32_t, 4>> mesh_random_leaves(const MeshSpec& spec, uint64_t seed,
                                                       double refine_prob) {
  uint64_t st = seed * 0x9E3779B97F4A7C15ull + 1;
  auto rnd = [&]() {  // splitmix64
    uint64_t z = (st += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return double(z >> 11) * (1.0 / 9007199254740992.0);
  };
  auto tag = [&](int, const double*, const double*) { return rnd() < refine_prob; };
  return mesh_refine_leaves(spec, tag);
}

std::vector<int32_t> mesh_visit_order(const Mesh& m, int groups) {
  const int nb = m.nb;
  std::vector<int32_t> cost(nb, 2), ids(nb), order(nb);
  for (int b = 0; b < nb; ++b) {
    for (int f = 0; f < 6; ++f) {
      const int k = m.face_kind[6 * b + f];
      cost[b] += k == FACE_COARSER ? 1 : (k == FACE_FINER ? 2 : 0);
    }
    ids[b] = b;
  }
  std::stable_sort(ids.begin(), ids.end(), [&](int a, int b) { return cost[a] > cost[b]; });
  groups = std::max(1, groups);
  for (int r = 0; r * groups < nb; ++r) {
    const int base = r * groups, cnt = std::min(groups, nb - base);
    for (int j = 0; j < cnt; ++j) order[base + j] = ids[base + ((r & 1) ? cnt - 1 - j : j)];
  }
  return order;
}

}  // namespace cup3d
