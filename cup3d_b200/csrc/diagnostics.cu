// ComputeDissipation (ComputeDissipation.cpp:17-140): the 20 volume integrals
// the reference appends to diagnostics.dat -- circulation, linear impulse,
// linear momentum, angular impulse, angular momentum, pressure power, viscous
// power, helicity, kinetic energy, enstrophy -- from one-layer star labs of
// the velocity (vector boundary ghosts) and the pressure (zero-gradient
// ghosts), positions taken from the domain centre.
//
// k_dissipation: one CTA per block (grid-stride), both labs in shared memory,
// two cells per thread, per-thread sums over its cells and blocks, then a
// fixed-order CTA reduction into partial[cta][20]; k_dissipation_sum adds the
// CTA partials in CTA order.  Bound: one pass over velocity, pressure and chi
// (40 B/cell), latency of the lab fill as in the gradient kernel.
#include "context.h"
#include "lab.cuh"

namespace cup3d {
namespace {

constexpr int kDiag = 20;

__global__ void __launch_bounds__(NT) k_dissipation(DevMesh M, const double* __restrict__ vel,
                                                     const double* __restrict__ pres,
                                                     const double* __restrict__ chi, double nu, double cx, double cy,
                                                     double cz, double* __restrict__ partial) {
  using LG = LabGeom<1>;
  __shared__ double ulab[3 * LG::V];
  __shared__ double plab[LG::V];
  __shared__ double red[NT / 32][kDiag];
  const size_t n = size_t(M.nb) * BN;
  auto getV = [&](int c, int blk, int cell) { return vel[c * n + size_t(blk) * BN + cell]; };
  auto getP = [&](int, int blk, int cell) { return pres[size_t(blk) * BN + cell]; };
  double Q[kDiag];
#pragma unroll
  for (int k = 0; k < kDiag; ++k) Q[k] = 0.0;
  for (int b = blockIdx.x; b < M.nb; b += gridDim.x) {
    __syncthreads();
    lab_fill<1, 3>(ulab, M, b, getV, true);
    lab_fill<1, 1>(plab, M, b, getP, false);
    __syncthreads();
    const double h = M.h[b];
    const double hCube = h * h * h, inv2h = .5 / h, invHh = 1 / (h * h);
    for (int i = threadIdx.x; i < BN; i += NT) {
      const int ix = i & 7, iy = (i >> 3) & 7, iz = i >> 6;
      auto U = [&](int c, int dx, int dy, int dz) { return ulab[c * LG::V + LG::at(ix + dx, iy + dy, iz + dz)]; };
      auto P = [&](int dx, int dy, int dz) { return plab[LG::at(ix + dx, iy + dy, iz + dz)]; };
      const double X = chi[size_t(b) * BN + i];
      const double PX = (M.index[3 * b] * BS + ix + 0.5) * h - cx;
      const double PY = (M.index[3 * b + 1] * BS + iy + 0.5) * h - cy;
      const double PZ = (M.index[3 * b + 2] * BS + iz + 0.5) * h - cz;
      const double WX = inv2h * ((U(2, 0, 1, 0) - U(2, 0, -1, 0)) - (U(1, 0, 0, 1) - U(1, 0, 0, -1)));
      const double WY = inv2h * ((U(0, 0, 0, 1) - U(0, 0, 0, -1)) - (U(2, 1, 0, 0) - U(2, -1, 0, 0)));
      const double WZ = inv2h * ((U(1, 1, 0, 0) - U(1, -1, 0, 0)) - (U(0, 0, 1, 0) - U(0, 0, -1, 0)));
      const double dPdx = inv2h * (P(1, 0, 0) - P(-1, 0, 0));
      const double dPdy = inv2h * (P(0, 1, 0) - P(0, -1, 0));
      const double dPdz = inv2h * (P(0, 0, 1) - P(0, 0, -1));
      const double u0 = U(0, 0, 0, 0), u1 = U(1, 0, 0, 0), u2 = U(2, 0, 0, 0);
      double V1 = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double lap = invHh * (U(c, 1, 0, 0) + U(c, -1, 0, 0) + U(c, 0, 1, 0) + U(c, 0, -1, 0) +
                                    U(c, 0, 0, 1) + U(c, 0, 0, -1) - 6 * U(c, 0, 0, 0));
        V1 += lap * U(c, 0, 0, 0);
      }
      const double D11 = inv2h * (U(0, 1, 0, 0) - U(0, -1, 0, 0));
      const double D22 = inv2h * (U(1, 0, 1, 0) - U(1, 0, -1, 0));
      const double D33 = inv2h * (U(2, 0, 0, 1) - U(2, 0, 0, -1));
      const double D12 = inv2h * (U(0, 0, 1, 0) - U(0, 0, -1, 0) + U(1, 1, 0, 0) - U(1, -1, 0, 0)) / 2;
      const double D13 = inv2h * (U(0, 0, 0, 1) - U(0, 0, 0, -1) + U(2, 1, 0, 0) - U(2, -1, 0, 0)) / 2;
      const double D23 = inv2h * (U(2, 0, 1, 0) - U(2, 0, -1, 0) + U(1, 0, 0, 1) - U(1, 0, 0, -1)) / 2;
      const double V2 = D11 * D11 + D22 * D22 + D33 * D33 + 2 * (D12 * D12 + D13 * D13 + D23 * D23);
      Q[0] += hCube * WX;
      Q[1] += hCube * WY;
      Q[2] += hCube * WZ;
      Q[3] += hCube / 2 * (PY * WZ - PZ * WY);
      Q[4] += hCube / 2 * (PZ * WX - PX * WZ);
      Q[5] += hCube / 2 * (PX * WY - PY * WX);
      Q[6] += hCube * u0;
      Q[7] += hCube * u1;
      Q[8] += hCube * u2;
      Q[9] += hCube / 3 * (PX * (PY * WY + PZ * WZ) - WX * (PY * PY + PZ * PZ));
      Q[10] += hCube / 3 * (PY * (PX * WX + PZ * WZ) - WY * (PX * PX + PZ * PZ));
      Q[11] += hCube / 3 * (PZ * (PX * WX + PY * WY) - WZ * (PX * PX + PY * PY));
      Q[12] += hCube * (PY * u2 - PZ * u1);
      Q[13] += hCube * (PZ * u0 - PX * u2);
      Q[14] += hCube * (PX * u1 - PY * u0);
      Q[15] -= (1 - X) * hCube * (dPdx * u0 + dPdy * u1 + dPdz * u2);
      Q[16] += (1 - X) * hCube * nu * (V1 + 2 * V2);
      Q[17] += hCube * (WX * u0 + WY * u1 + WZ * u2);
      Q[18] += hCube * (u0 * u0 + u1 * u1 + u2 * u2) / 2;
      Q[19] += hCube * sqrt(WX * WX + WY * WY + WZ * WZ);
    }
  }
#pragma unroll
  for (int k = 0; k < kDiag; ++k) {
    double v = Q[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < kDiag) {
    double v = 0.0;
    for (int w = 0; w < NT / 32; ++w) v += red[w][threadIdx.x];
    partial[size_t(blockIdx.x) * kDiag + threadIdx.x] = v;
  }
}

__global__ void k_dissipation_sum(const double* __restrict__ partial, int nparts, double* __restrict__ out) {
  const int k = threadIdx.x;
  if (k >= kDiag) return;
  double v = 0.0;
  for (int p = 0; p < nparts; ++p) v += partial[size_t(p) * kDiag + k];
  out[k] = v;
}

}  // namespace
}  // namespace cup3d

using namespace cup3d;

extern "C" int cup_compute_dissipation(cup_ctx* c, double* out20) {
  ProfBind pb_(c);
  if (!c || !out20 || c->mesh.nb == 0 || c->host_only)
    return ctx_fail(c, CUP_ERR_ARG, "cup_compute_dissipation: bad arguments");
  if (c->ncase > 1) return ctx_fail(c, CUP_ERR_STATE, "cup_compute_dissipation: not available on a batch of cases");
  const int grid = std::max(1, std::min(c->mesh.nb, 2 * c->num_sms));
  if (c->diag_cap < grid) {
    if (int rc = c->field_arena.alloc(&c->d_diag, size_t(grid + 1) * kDiag))
      return ctx_fail(c, rc, "cup_compute_dissipation: allocation failed");
    c->diag_cap = grid;
  }
  const double* ext = c->mesh.spec.extents;
  {
    ProfScope ps("dissipation", c->stream);
    k_dissipation<<<grid, NT, 0, c->stream>>>(c->dm, c->F.vel[c->F.vcur], c->F.pres[c->F.pcur], c->F.chi, c->cfg.nu,
                                              0.5 * ext[0], 0.5 * ext[1], 0.5 * ext[2], c->d_diag);
    k_dissipation_sum<<<1, 32, 0, c->stream>>>(c->d_diag, grid, c->d_diag + size_t(grid) * kDiag);
  }
  CUP_CUDA_TRY(cudaGetLastError());
  CUP_CUDA_TRY(stream_d2h(c->stream, out20, c->d_diag + size_t(grid) * kDiag, kDiag * sizeof(double)));
  return 0;
}
