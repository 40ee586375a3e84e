// Host-side block-structured AMR mesh: the block list, its space-filling-curve
// order and the per-face neighbour tables that every device kernel reads.
//
// The reference delegates all of this to Cubism (GridMPI / BlockInfo /
// MeshAdaptation, absent from the reference tree).  The contract restated here
// is the one the hot path relies on:
//   * blocks of 8^3 cells, level l has spacing h_l = h_0 / 2^l
//     (SimulationData.cpp:134-168 for h_0, hmin, hmax);
//   * block (l, i, j, k) covers cells [8i, 8i+8) x ... at level l;
//   * face neighbours are either at the same level, one level coarser or one
//     level finer (2:1 balance, enforced over all 26 neighbours);
//   * periodic directions wrap block indices (Definitions.h:38, BCflag);
//   * Znei / Zparent / Zchild lookups of PoissonSolverExp.cpp:167-217 become
//     the FACE_SAME / FACE_COARSER / FACE_FINER entries below.
#pragma once
#include <array>
#include <cstdint>
#include <functional>
#include <string>
#include <unordered_map>
#include <vector>

namespace cup3d {

enum FaceKind : int32_t {
  FACE_SAME = 0,      // nbr[0] = neighbour block id
  FACE_BOUNDARY = 1,  // nbr[0] = BC kind (BC_FREESPACE or BC_WALL)
  FACE_COARSER = 2,   // nbr[0] = coarse neighbour block id
  FACE_FINER = 3      // nbr[a + 2b] = fine neighbour at tangential halves (a, b)
};

enum BCKind : int32_t { BC_FREESPACE = 0, BC_PERIODIC = 1, BC_WALL = 2 };

// Tangential dimensions of a face normal to `d`, in increasing order.  The
// per-face arrays of the reference (faceXm[y + 8 z], faceYm[x + 8 z],
// faceZm[x + 8 y], AdvectionDiffusion.cpp:154-211) use the same order.
#ifndef CUP3D_TAN_HELPERS
#define CUP3D_TAN_HELPERS
inline int tan1(int d) { return d == 0 ? 1 : 0; }
inline int tan2(int d) { return d == 2 ? 1 : 2; }
#endif

struct MeshSpec {
  int bpd[3] = {1, 1, 1};   // level-0 blocks per dimension (-bpdx/y/z)
  int level_max = 1;        // number of levels (-levelMax)
  int bc[3] = {BC_FREESPACE, BC_FREESPACE, BC_FREESPACE};
  double extent = 1.0;      // largest physical extent (-extent)
  // derived
  double extents[3] = {0, 0, 0};
  double h0 = 0;            // spacing at level 0
  double hmin = 0;          // spacing at level level_max-1
};

// Fills extents/h0/hmin the way SimulationData::_preprocessArguments does.
void mesh_spec_finalize(MeshSpec& s);

struct Mesh {
  MeshSpec spec;
  int nb = 0;
  std::vector<int32_t> level;      // nb
  std::vector<int32_t> index;      // 3*nb
  std::vector<double> h;           // nb
  std::vector<double> origin;      // 3*nb (physical position of cell (0,0,0) corner)
  std::vector<int32_t> face_kind;  // 6*nb, face f = 2*d + side (side 0 = minus)
  std::vector<int32_t> face_nbr;   // 24*nb, 4 entries per face
  int mean_block = -1;             // block with index (0,0,0) (bMeanConstraint row)
  int max_level_used = 0;
  std::unordered_map<uint64_t, int32_t> lookup;

  static uint64_t key(int l, int i, int j, int k) {
    return (uint64_t(l) << 60) | (uint64_t(i) << 40) | (uint64_t(j) << 20) | uint64_t(k);
  }
  int find(int l, int i, int j, int k) const {
    auto it = lookup.find(key(l, i, j, k));
    return it == lookup.end() ? -1 : it->second;
  }
};

// Builds a mesh from an explicit list of leaf blocks.  The blocks are reordered
// along the space-filling curve (Hilbert order of the level-0 roots, Morton
// order of the octree below each root).  Returns false with a message when the
// blocks overlap, leave holes, or violate face 2:1 balance.
bool mesh_build(const MeshSpec& spec, const std::vector<std::array<int32_t, 4>>& leaves,
                Mesh& out, std::string& err);

// Leaf generation: start from the level-0 grid, refine every leaf for which
// `tag(level, lo[3], hi[3])` is true (box in physical coordinates) up to
// level_max-1, then refine further until every leaf's 26 neighbours are within
// one level.  Deterministic.
std::vector<std::array<int32_t, 4>> mesh_refine_leaves(
    const MeshSpec& spec,
    const std::function<bool(int, const double*, const double*)>& tag);

// Deterministic refinement rule standing in for vorticity tagging around a body
// in a uniform stream: refine blocks near a sphere of radius `r` at `c` and
// inside a wake cylinder of length `wake_len` downstream along `flow_dir` (+1
// or -1 along x).  Radii shrink geometrically with level.
std::vector<std::array<int32_t, 4>> mesh_sphere_wake_leaves(
    const MeshSpec& spec, const double c[3], double r, int flow_dir, double near_radius,
    double wake_len, double wake_radius);

// Random 2:1-balanced refinement (seeded) for tests.
std::vector<std::array<int32_t, 4>> mesh_random_leaves(const MeshSpec& spec, uint64_t seed,
                                                       double refine_prob);

// Order in which `groups` workers that each take blocks slot g, g + groups,
// g + 2 groups, ... should visit the blocks so that every worker gets a
// similar share of the Poisson operator's cost: blocks sorted by estimated
// cost (coarse-fine faces cost extra flux work), dealt in snake order (one
// round forward, the next backward).  A permutation of 0..nb-1.
// Leaves after one adaptation of m (the role of Cubism's MeshAdaptation
// Tag/Adapt, absent from the reference tree): leaves with refine[b] split
// (below level_max - 1), then the 2:1 balance over the 26 neighbours splits
// what it must; a parent whose eight children are leaves that all have
// compress[b] (and no refine) replaces them unless a leaf finer than the
// children touches the parent's region.
std::vector<std::array<int32_t, 4>> mesh_adapt_leaves(const Mesh& m, const std::vector<uint8_t>& refine,
                                                      const std::vector<uint8_t>& compress);

std::vector<int32_t> mesh_visit_order(const Mesh& m, int groups);

}  // namespace cup3d
