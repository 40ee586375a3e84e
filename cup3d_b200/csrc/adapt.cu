// Mesh adaptation: Simulation::adaptMesh (Simulation.cpp:128-149).
//
// The reference computes the vorticity into tmpV (KernelVorticity,
// ProcessHelpers.h:96-205), marks obstacle interfaces and interiors on it
// (GradChiOnTmp, ProcessHelpers.h:17-69), then lets Cubism's MeshAdaptation
// tag, refine and compress the blocks and move the fields (Tag, TagLike,
// Adapt).  Cubism is not in the reference tree, so the tagging rule and the
// field transfer are this library's definition:
//   * indicator of a block: the largest |omega| over its cells, where
//     GradChiOnTmp's rules hold: on level levelMaxVorticity-1 (when below
//     levelMax) a cell with |omega| >= Rtol counts as (Rtol+Ctol)/2; a cell
//     whose clamped chi is above 0.9 counts as 0; and a chi value strictly
//     between 1e-5 and 0.9 anywhere in the block or its face ghost layers
//     (two layers on level levelMax-1, one below) makes the indicator 1e10;
//   * decision (mesh_adapt_leaves): refine at indicator >= Rtol, compress
//     eight siblings that are all below Ctol, 2:1 balance;
//   * transfer: blocks that stay are copied; a refined block's cells take the
//     parent cell plus its central-difference slopes at +-1/4 cell (exact for
//     linear fields, and the children average back to the parent); a
//     compressed block's cells are the means of their eight children.
// Velocity and pressure move; tmpV and the Poisson right-hand side restart at
// zero, and the body's chi is created again on the new mesh (CreateObstacles
// runs whenever the mesh changed, ObstaclesCreate.cpp:291-292).
#include <algorithm>
#include <cmath>
#include <vector>

#include "context.h"
#include "lab.cuh"

namespace cup3d {
namespace {

__global__ void __launch_bounds__(NT) k_adapt_indicator(DevMesh M, const double* __restrict__ vel,
                                                        const double* __restrict__ chi, const int* __restrict__ level,
                                                        int level_max, int level_max_vort, double rtol, double ctol,
                                                        double* __restrict__ out) {
  using LV = LabGeom<1>;
  using LC = LabGeom<2>;
  __shared__ double ulab[3 * LV::V];
  __shared__ double clab[LC::V];
  __shared__ double red[NT / 32];
  __shared__ int s_iface;
  const size_t n = size_t(M.nb) * BN;
  auto getV = [&](int c, int blk, int cell) { return vel[c * n + size_t(blk) * BN + cell]; };
  auto getC = [&](int, int blk, int cell) { return chi[size_t(blk) * BN + cell]; };
  for (int b = blockIdx.x; b < M.nb; b += gridDim.x) {
    __syncthreads();
    lab_fill<1, 3>(ulab, M, b, getV, true);
    lab_fill<2, 1>(clab, M, b, getC, false);
    if (threadIdx.x == 0) s_iface = 0;
    __syncthreads();
    const int lev = level[b];
    const int offset = lev == level_max - 1 ? 2 : 1;
    for (int i = threadIdx.x; i < LC::V; i += NT) {
      if (i >= BN && offset == 1 && (((i - BN) >> 6) & 1)) continue;  // the second ghost layer
      const double s = fmax(fmin(clab[i], 1.0), 0.0);
      if (s > 0.00001 && s < 0.9) s_iface = 1;
    }
    const double h = M.h[b], inv2h = .5 * h * h, fac = 1.0 / (h * h * h);
    auto U = [&](int c, int x, int y, int z) { return ulab[c * LV::V + LV::at(x, y, z)]; };
    const bool clamp_vort = lev == level_max_vort - 1 && level_max_vort < level_max;
    double vmax = 0.0;
    for (int cell = threadIdx.x; cell < BN; cell += NT) {
      const int x = cell & 7, y = (cell >> 3) & 7, z = cell >> 6;
      double w0 = inv2h * ((U(2, x, y + 1, z) - U(2, x, y - 1, z)) - (U(1, x, y, z + 1) - U(1, x, y, z - 1)));
      double w1 = inv2h * ((U(0, x, y, z + 1) - U(0, x, y, z - 1)) - (U(2, x + 1, y, z) - U(2, x - 1, y, z)));
      double w2 = inv2h * ((U(1, x + 1, y, z) - U(1, x - 1, y, z)) - (U(0, x, y + 1, z) - U(0, x, y - 1, z)));
      w0 *= fac;
      w1 *= fac;
      w2 *= fac;
      double mag = sqrt(w0 * w0 + w1 * w1 + w2 * w2);
      if (clamp_vort && mag >= rtol) {
        const double a = 0.5 * (rtol + ctol);
        mag = sqrt(a * a + 0.0 * 0.0 + 0.0 * 0.0);
      }
      if (fmax(fmin(clab[cell], 1.0), 0.0) > 0.9) mag = 0.0;  // inside the body
      vmax = fmax(vmax, mag);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = vmax;
    __syncthreads();
    if (threadIdx.x == 0) {
      double m = 0.0;
      for (int w = 0; w < NT / 32; ++w) m = fmax(m, red[w]);
      out[b] = s_iface ? 1e10 : m;
    }
  }
}

// plan[9 b1]: 0 = block kept (plan[1]: its old id); 1 = refined (plan[1]:
// the old parent, plan[2]: octant); 2 = compressed (plan[1..8]: the old
// children by octant).  Octant o = ox + 2 oy + 4 oz.
template <int NC>
__global__ void __launch_bounds__(NT) k_adapt_transfer(DevMesh M0, const double* __restrict__ src, int nb1,
                                                       double* __restrict__ dst, const int* __restrict__ plan,
                                                       bool vector_bc) {
  using LG = LabGeom<1>;
  __shared__ double lab[NC * LG::V];
  const size_t n0 = size_t(M0.nb) * BN, n1 = size_t(nb1) * BN;
  auto get0 = [&](int c, int blk, int cell) { return src[c * n0 + size_t(blk) * BN + cell]; };
  for (int b = blockIdx.x; b < nb1; b += gridDim.x) {
    const int* p = plan + 9 * b;
    const int kind = p[0];
    if (kind == 0) {
      for (int i = threadIdx.x; i < NC * BN; i += NT) {
        const int c = i / BN, cell = i - c * BN;
        dst[c * n1 + size_t(b) * BN + cell] = get0(c, p[1], cell);
      }
    } else if (kind == 1) {
      __syncthreads();
      lab_fill<1, NC>(lab, M0, p[1], get0, vector_bc);
      __syncthreads();
      const int o = p[2];
      for (int cell = threadIdx.x; cell < BN; cell += NT) {
        const int x = cell & 7, y = (cell >> 3) & 7, z = cell >> 6;
        const int X = 4 * (o & 1) + (x >> 1), Y = 4 * ((o >> 1) & 1) + (y >> 1), Z = 4 * (o >> 2) + (z >> 1);
        const double sx = (x & 1) ? 0.25 : -0.25, sy = (y & 1) ? 0.25 : -0.25, sz = (z & 1) ? 0.25 : -0.25;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const double* L = lab + c * LG::V;
          const double u = L[LG::at(X, Y, Z)];
          const double gx = 0.5 * (L[LG::at(X + 1, Y, Z)] - L[LG::at(X - 1, Y, Z)]);
          const double gy = 0.5 * (L[LG::at(X, Y + 1, Z)] - L[LG::at(X, Y - 1, Z)]);
          const double gz = 0.5 * (L[LG::at(X, Y, Z + 1)] - L[LG::at(X, Y, Z - 1)]);
          dst[c * n1 + size_t(b) * BN + cell] = u + ((sx * gx + sy * gy) + sz * gz);
        }
      }
    } else {
      for (int cell = threadIdx.x; cell < BN; cell += NT) {
        const int X = cell & 7, Y = (cell >> 3) & 7, Z = cell >> 6;
        const int ch = p[1 + (X >> 2) + 2 * (Y >> 2) + 4 * (Z >> 2)];
        const int fx = 2 * (X & 3), fy = 2 * (Y & 3), fz = 2 * (Z & 3);
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          double s = 0.0;
#pragma unroll
          for (int e = 0; e < 8; ++e)
            s += get0(c, ch, (fx + (e & 1)) + 8 * (fy + ((e >> 1) & 1)) + 64 * (fz + (e >> 2)));
          dst[c * n1 + size_t(b) * BN + cell] = 0.125 * s;
        }
      }
    }
  }
}

int level_max_vort(const cup_config& cfg) {
  return cfg.level_max_vorticity > 0 ? cfg.level_max_vorticity : cfg.level_max;
}

}  // namespace

// Indicator of every block into out (host, nb values).
int adapt_indicator(cup_ctx* c, std::vector<double>& out) {
  const Mesh& m = c->mesh;
  DevArena tmp;
  int* d_level = nullptr;
  double* d_out = nullptr;
  if (int rc = tmp.alloc(&d_level, m.nb)) return rc;
  if (int rc = tmp.alloc(&d_out, m.nb)) return rc;
  CUP_CUDA_TRY(stream_h2d(c->stream, d_level, m.level.data(), m.nb * sizeof(int32_t)));
  {
    ProfScope ps("adapt_indicator", c->stream);
    k_adapt_indicator<<<std::max(1, std::min(m.nb, c->num_sms * 8)), NT, 0, c->stream>>>(
        c->dm, c->F.vel[c->F.vcur], c->F.chi, d_level, c->cfg.level_max, level_max_vort(c->cfg), c->cfg.rtol,
        c->cfg.ctol, d_out);
  }
  CUP_CUDA_TRY(cudaGetLastError());
  out.resize(m.nb);
  CUP_CUDA_TRY(stream_d2h(c->stream, out.data(), d_out, m.nb * sizeof(double)));
  return 0;
}

// One adaptation of the context's mesh; *changed = 0 when no block changes.
int adapt_mesh(cup_ctx* c, int* changed) {
  *changed = 0;
  std::vector<double> ind;
  if (int rc = adapt_indicator(c, ind)) return rc;
  const Mesh& m0 = c->mesh;
  std::vector<uint8_t> refine(m0.nb), compress(m0.nb);
  for (int b = 0; b < m0.nb; ++b) {
    refine[b] = ind[b] >= c->cfg.rtol ? 1 : 0;
    compress[b] = ind[b] < c->cfg.ctol ? 1 : 0;
  }
  const std::vector<std::array<int32_t, 4>> leaves = mesh_adapt_leaves(m0, refine, compress);
  bool same = int(leaves.size()) == m0.nb;
  for (size_t i = 0; i < leaves.size() && same; ++i)
    same = m0.find(leaves[i][0], leaves[i][1], leaves[i][2], leaves[i][3]) >= 0;
  if (same) return 0;
  Mesh m1;
  std::string err;
  if (!mesh_build(m0.spec, leaves, m1, err)) return set_error(CUP_ERR_MESH, ("adapted mesh: " + err).c_str());
  // where each new block's values come from
  std::vector<int32_t> plan(9 * size_t(m1.nb), -1);
  for (int b = 0; b < m1.nb; ++b) {
    const int l = m1.level[b], i = m1.index[3 * b], j = m1.index[3 * b + 1], k = m1.index[3 * b + 2];
    int32_t* p = &plan[9 * size_t(b)];
    if (int o = m0.find(l, i, j, k); o >= 0) {
      p[0] = 0;
      p[1] = o;
    } else if (int par = l > 0 ? m0.find(l - 1, i >> 1, j >> 1, k >> 1) : -1; par >= 0) {
      p[0] = 1;
      p[1] = par;
      p[2] = (i & 1) + 2 * (j & 1) + 4 * (k & 1);
    } else {
      p[0] = 2;
      for (int o = 0; o < 8; ++o) {
        p[1 + o] = m0.find(l + 1, 2 * i + (o & 1), 2 * j + ((o >> 1) & 1), 2 * k + (o >> 2));
        if (p[1 + o] < 0) return set_error(CUP_ERR_MESH, "adapted mesh: a block has no source");
      }
    }
  }
  // The new tables go into the table set not in use, so the transfer can
  // still read the old mesh's; within the field arena's room the values move
  // from each field's current buffer to its other one, otherwise into a new
  // arena (the old one freed after the transfer).
  const DevMesh dm0 = c->dm;
  const Fields F0 = c->F;
  const int nb1 = m1.nb;
  const int set1 = 1 - c->tab_cur;
  c->mesh = std::move(m1);
  int rc = ctx_upload_mesh(c, set1);
  if (rc) return rc;
  std::vector<void*> old_fields;
  const bool grow = nb1 > c->field_cap;
  if (grow) {
    old_fields.swap(c->field_arena.ptrs);  // F0's buffers stay valid until freed below
    c->field_cap = 0;
  }
  auto free_old = [&]() {
    if (old_fields.empty()) return;
    cudaStreamSynchronize(c->stream);
    for (void* q : old_fields) cudaFree(q);
    old_fields.clear();
  };
  graph_reset(c);
  c->obst_arena.release();
  c->ob = DevObstacle();
  c->proj_open = 0;
  if ((rc = fields_reserve(c, nb1))) {
    free_old();
    return rc;
  }
  const int vdst = grow ? 0 : 1 - F0.vcur, pdst = grow ? 0 : 1 - F0.pcur;
  int* d_plan = c->tabs[set1].plan;
  cudaError_t e = cudaMemcpyAsync(d_plan, plan.data(), plan.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                                  c->stream);
  if (e == cudaSuccess) {
    ProfScope ps("adapt_transfer", c->stream);
    const int grid = std::max(1, std::min(nb1, c->num_sms * 8));
    k_adapt_transfer<3><<<grid, NT, 0, c->stream>>>(dm0, F0.vel[F0.vcur], nb1, c->F.vel[vdst], d_plan, true);
    k_adapt_transfer<1><<<grid, NT, 0, c->stream>>>(dm0, F0.pres[F0.pcur], nb1, c->F.pres[pdst], d_plan, false);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    free_old();
    return set_cuda_error(e, "adapt_transfer", __FILE__, __LINE__);
  }
  c->tab_cur = set1;
  c->F.vcur = vdst;
  c->F.pcur = pdst;
  // the other buffers (the old values, after the transfer in stream order) and the rest zeroed
  rc = fields_reset(c, true);
  free_old();
  if (rc) return rc;
  if ((rc = body_recreate(c))) return rc;
  *changed = 1;
  return 0;
}

}  // namespace cup3d

using namespace cup3d;

extern "C" {

int cup_adapt_indicator(cup_ctx* c, double* out) {
  ProfBind pb_(c);
  if (!c || !out || c->mesh.nb == 0 || c->host_only || c->ncase > 1)
    return ctx_fail(c, CUP_ERR_ARG, "cup_adapt_indicator: bad arguments");
  std::vector<double> v;
  if (int rc = adapt_indicator(c, v)) return ctx_fail(c, rc, cup_last_error(nullptr));
  std::copy(v.begin(), v.end(), out);
  return 0;
}

int cup_adapt_mesh(cup_ctx* c, int32_t* changed) {
  ProfBind pb_(c);
  if (!c || c->mesh.nb == 0 || c->host_only) return ctx_fail(c, CUP_ERR_ARG, "cup_adapt_mesh: bad arguments");
  if (c->ncase > 1) return ctx_fail(c, CUP_ERR_STATE, "cup_adapt_mesh: not available on a batch of cases");
  if (c->ob.nslots > 0 && c->body.kind < 0)
    return ctx_fail(c, CUP_ERR_STATE, "cup_adapt_mesh: obstacle data set with cup_set_obstacle cannot be re-created");
  int ch = 0;
  if (int rc = adapt_mesh(c, &ch)) return ctx_fail(c, rc, cup_last_error(nullptr));
  if (changed) *changed = ch;
  return 0;
}

}  // extern "C"
