// Block + ghost-layer staging ("labs") in shared memory for star stencils.
//
// Ghost values (the role of Cubism's BlockLab, absent from the reference tree):
//   * same level / periodic: the neighbour's cells;
//   * domain boundary: BlockLabBC::applyBCfaceOpen / applyBCfaceWall
//     (Definitions.h:67-397) for vector fields -- every ghost layer copies the
//     boundary cell, the normal component (freespace) or all components (wall)
//     change sign -- and zero-gradient copies for scalar fields;
//   * finer neighbour: mean of the 2x2x2 fine cells;
//   * coarser neighbour C: tensor-product quadratic Lagrange interpolation from
//     C's own cells (normal nodes: C's layers 0,1,2; tangential: the three
//     cells around the containing coarse cell, one-sided at C's block edges).
// Edge and corner ghosts are never filled (all stencils here are stars).
#pragma once
#include "common.cuh"

namespace cup3d {

// Star-shaped lab: the 8^3 block followed by its six face slabs of G layers
// (edges and corners are never read by the star stencils, so they are not
// stored).  Slab f (0..5 = -x,+x,-y,+y,-z,+z), layer l (1..G) holds
// face-local cells (a, bb) (tangential coordinates in increasing dimension
// order) at 512 + (f*G + l-1)*64 + a + 8*bb.
template <int G>
struct LabGeom {
  static constexpr int V = BN + 6 * G * BS * BS;
  __device__ static __forceinline__ int at(int x, int y, int z) {
    if (x < 0) return BN + (0 * G - 1 - x) * 64 + y + 8 * z;
    if (x >= BS) return BN + (1 * G + x - BS) * 64 + y + 8 * z;
    if (y < 0) return BN + (2 * G - 1 - y) * 64 + x + 8 * z;
    if (y >= BS) return BN + (3 * G + y - BS) * 64 + x + 8 * z;
    if (z < 0) return BN + (4 * G - 1 - z) * 64 + x + 8 * y;
    if (z >= BS) return BN + (5 * G + z - BS) * 64 + x + 8 * y;
    return x + BS * y + BS * BS * z;
  }
};

__device__ __forceinline__ void lagrange3(double xi, double w[3]) {
  w[0] = 0.5 * (xi - 1.0) * (xi - 2.0);
  w[1] = -xi * (xi - 2.0);
  w[2] = 0.5 * xi * (xi - 1.0);
}

__device__ __forceinline__ void tan_stencil(int t, int half, int& n0, double w[3]) {
  const int c = half * (BS / 2) + (t >> 1);
  const double eta = (t & 1) ? 0.25 : -0.25;
  if (c == 0) {
    n0 = 0;
    lagrange3(eta, w);
  } else if (c == BS - 1) {
    n0 = BS - 3;
    lagrange3(2.0 + eta, w);
  } else {
    n0 = c - 1;
    lagrange3(1.0 + eta, w);
  }
}

// Ghost of a fine block at layer l (1-based) beyond its face (d, s), tangential
// (a, bb), interpolated from the coarse neighbour cb.  get(cell of cb) reads one
// component.  The fine block's tangential halves inside cb are (h1, h2).
template <class Get>
__device__ __forceinline__ double c2f_ghost(Get get, int d, int s, int l, int a, int bb, int h1, int h2) {
  double wn[3], w1[3], w2[3];
  lagrange3((l - 1.5) * 0.5, wn);
  int n1, n2;
  tan_stencil(a, h1, n1, w1);
  tan_stencil(bb, h2, n2, w2);
  double sum = 0.0;
#pragma unroll
  for (int i2 = 0; i2 < 3; ++i2)
#pragma unroll
    for (int i1 = 0; i1 < 3; ++i1)
#pragma unroll
      for (int in = 0; in < 3; ++in)
        sum += wn[in] * w1[i1] * w2[i2] * get(face_cell(d, 1 - s, in, n1 + i1, n2 + i2));
  return sum;
}

// Fills lab (NC components, each LabGeom<G>::V doubles) for block b, with
// threads t0, t0 + nt, ... (lab_fill: the whole CTA).  get(c, blk, cell)
// reads component c of the field.
template <int G, int NC, class Get>
__device__ void lab_fill_part(double* lab, const DevMesh& M, int b, Get get, bool vector_bc, int t0, int nt) {
  using LG = LabGeom<G>;
  for (int i = t0; i < BN; i += nt) {
    const int x = i & 7, y = (i >> 3) & 7, z = i >> 6;
#pragma unroll
    for (int c = 0; c < NC; ++c) lab[c * LG::V + LG::at(x, y, z)] = get(c, b, i);
  }
  for (int g = t0; g < 6 * G * 64; g += nt) {
    const int f = g / (G * 64), rem = g - f * (G * 64);
    const int l = rem / 64 + 1, a = rem & 7, bb = (rem >> 3) & 7;
    const int d = f >> 1, s = f & 1;
    const int kind = M.fkind[b * 6 + f];
    const int* nb = M.fnbr + b * 24 + 4 * f;
    int q[3];
    q[d] = s ? BS - 1 + l : -l;
    q[tan1(d)] = a;
    q[tan2(d)] = bb;
    const int li = LG::at(q[0], q[1], q[2]);
    if (kind == K_SAME) {
      const int n = nb[0], cell = face_cell(d, 1 - s, l - 1, a, bb);
#pragma unroll
      for (int c = 0; c < NC; ++c) lab[c * LG::V + li] = get(c, n, cell);
    } else if (kind == K_BOUNDARY) {
      const int cell = face_cell(d, s, 0, a, bb);
      const bool wall = nb[0] == BCK_WALL;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        double v = get(c, b, cell);
        if (vector_bc && (wall || c == d)) v = -v;
        lab[c * LG::V + li] = v;
      }
    } else if (kind == K_FINER) {
      const int ch = nb[(a >> 2) + 2 * (bb >> 2)];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        double sum = 0.0;
#pragma unroll
        for (int e2 = 0; e2 < 2; ++e2)
#pragma unroll
          for (int e1 = 0; e1 < 2; ++e1)
#pragma unroll
            for (int en = 0; en < 2; ++en)
              sum += get(c, ch, face_cell(d, 1 - s, 2 * (l - 1) + en, 2 * (a & 3) + e1, 2 * (bb & 3) + e2));
        lab[c * LG::V + li] = 0.125 * sum;
      }
    } else {  // K_COARSER
      const int cb = nb[0];
      const int h1 = M.index[b * 3 + tan1(d)] & 1, h2 = M.index[b * 3 + tan2(d)] & 1;
#pragma unroll
      for (int c = 0; c < NC; ++c)
        lab[c * LG::V + li] = c2f_ghost([&](int cell) { return get(c, cb, cell); }, d, s, l, a, bb, h1, h2);
    }
  }
}

template <int G, int NC, class Get>
__device__ __forceinline__ void lab_fill(double* lab, const DevMesh& M, int b, Get get, bool vector_bc) {
  lab_fill_part<G, NC>(lab, M, b, get, vector_bc, int(threadIdx.x), int(blockDim.x));
}

// Value of the child's ghost at layer 1 beyond its face toward the coarse block
// cb (our block), for the child's face cell (fa, fb): the value the child's own
// lab holds there.  Used by the coarse block's flux correction.
template <class Get>
__device__ __forceinline__ double child_ghost1(Get get_coarse, const DevMesh& M, int ch, int d, int s, int fa, int fb) {
  // the child's face toward us is (d, 1 - s)
  const int h1 = M.index[ch * 3 + tan1(d)] & 1, h2 = M.index[ch * 3 + tan2(d)] & 1;
  return c2f_ghost(get_coarse, d, 1 - s, 1, fa, fb, h1, h2);
}

}  // namespace cup3d
