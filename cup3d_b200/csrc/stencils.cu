// Time-step stencil operators (FP64), one CTA per 8^3 block with its ghost
// layers staged in shared memory.  Each kernel names the reference kernel it
// computes; coarse-fine flux correction (Cubism FluxCorrection, absent from the
// reference tree) adds, to a coarse cell next to a finer face, its own face
// value plus the four fine face values, computed by the coarse block's CTA
// from the fine blocks' face cells and their ghosts.
#include <algorithm>
#include <type_traits>

#include "../../include/cup3d_b200.h"
#include "lab.cuh"
#include "staged.cuh"
#include "stencils.cuh"
#include "profiler.h"

namespace cup3d {

struct Vec3 {
  double v[3];
};

// ---------------------------------------------------------------------------
// AdvectionDiffusion: KernelAdvectDiffuse (AdvectionDiffusion.cpp:19-215)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double sq(double a) { return a * a; }

// WENO5 reconstruction biased to the left (weno5_plus of
// AdvectionDiffusion.cpp:34-64): candidate stencils f1..f3 with smoothness
// indicators b1..b3, nonlinear weights w_k = (d_k/q_k) / sum_j d_j/q_j with
// q_k = (b_k + eps)^2 and d = (0.1, 0.6, 0.3).  The weights are evaluated with
// one division instead of four: multiplying numerator and denominator by
// q1 q2 q3 gives  sum_k a_k f_k / sum_k a_k  with  a_1 = 0.1 q2 q3,
// a_2 = 0.6 q1 q3, a_3 = 0.3 q1 q2  (q_k >= eps^2 = 1e-12, so no underflow).
__device__ __forceinline__ double weno5_left(double um2, double um1, double u, double up1, double up2) {
  const double e = 1e-6;
  const double b1 = 13.0 / 12.0 * sq((um2 + u) - 2 * um1) + 0.25 * sq((um2 + 3 * u) - 4 * um1);
  const double b2 = 13.0 / 12.0 * sq((um1 + up1) - 2 * u) + 0.25 * sq(um1 - up1);
  const double b3 = 13.0 / 12.0 * sq((u + up2) - 2 * up1) + 0.25 * sq((3 * u + up2) - 4 * up1);
  const double q1 = sq(b1 + e), q2 = sq(b2 + e), q3 = sq(b3 + e);
  const double a1 = 0.1 * (q2 * q3), a2 = 0.6 * (q1 * q3), a3 = 0.3 * (q1 * q2);
  const double f1 = (11.0 / 6.0) * u + ((1.0 / 3.0) * um2 - (7.0 / 6.0) * um1);
  const double f2 = (5.0 / 6.0) * u + ((-1.0 / 6.0) * um1 + (1.0 / 3.0) * up1);
  const double f3 = (1.0 / 3.0) * u + ((+5.0 / 6.0) * up1 - (1.0 / 6.0) * up2);
  return ((a1 * f1 + a3 * f3) + a2 * f2) / ((a1 + a3) + a2);
}

// Upwind derivative of KernelAdvectDiffuse (AdvectionDiffusion.cpp:66-103).
// WENO5: the right-biased reconstruction (weno5_minus) is the left-biased one
// of the mirrored stencil, weno5_minus(a,b,c,d,e) = weno5_plus(e,d,c,b,a), so
// the upwind choice only selects the five inputs of two left-biased
// evaluations and no warp diverges on the sign of U.
template <int SCHEME>
__device__ __forceinline__ double deriv(double U, double um3, double um2, double um1, double u, double up1,
                                        double up2, double up3) {
  if (SCHEME == 1) {
    const bool pos = U > 0;
    // face i+1/2 and face i-1/2 reconstructions in the upwind direction
    const double fp = weno5_left(pos ? um2 : up3, pos ? um1 : up2, pos ? u : up1, pos ? up1 : u, pos ? up2 : um1);
    const double fm = weno5_left(pos ? um3 : up2, pos ? um2 : up1, pos ? um1 : u, pos ? u : um1, pos ? up1 : um2);
    return fp - fm;
  }
  if (U > 0) return (-2 * um3 + 15 * um2 - 60 * um1 + 20 * u + 30 * up1 - 3 * up2) / 60.;
  return (2 * up3 - 15 * up2 + 60 * up1 - 20 * u - 30 * um1 + 3 * um2) / 60.;
}

__device__ __forceinline__ bool has_finer(const DevMesh& M, int b) {
  bool r = false;
#pragma unroll
  for (int f = 0; f < 6; ++f) r |= M.fkind[b * 6 + f] == K_FINER;
  return r;
}

// lab coordinates of own face cell (layer 0) and the ghost at layer 1
__device__ __forceinline__ void face_lab_pair(int d, int s, int a, int bb, int q[3], int g[3]) {
  q[d] = s ? BS - 1 : 0;
  q[tan1(d)] = a;
  q[tan2(d)] = bb;
  g[0] = q[0];
  g[1] = q[1];
  g[2] = q[2];
  g[d] += s ? 1 : -1;
}

template <int SCHEME>
__global__ void __launch_bounds__(NT, 3)
    k_advect_stage(DevMesh M, const double* __restrict__ vin, double* __restrict__ vout, double* tmpV, double dt,
                   double nu, Vec3 ui, int stage) {
  extern __shared__ double smem[];
  using LG = LabGeom<3>;
  double* lab = smem;
  double* corr = smem + 3 * LG::V;
  const size_t n = size_t(M.nb) * BN;
  const double alpha = stage == 0 ? 1.0 / 3.0 : (stage == 1 ? 15.0 / 16.0 : 8.0 / 15.0);
  const double beta = stage == 0 ? -5.0 / 9.0 : (stage == 1 ? -153.0 / 128.0 : 0.0);
  auto get = [&](int c, int blk, int cell) { return vin[c * n + size_t(blk) * BN + cell]; };
  for (int b = blockIdx.x; b < M.nb; b += gridDim.x) {
    __syncthreads();
    lab_fill<3, 3>(lab, M, b, get, true);
    const bool fix = has_finer(M, b);
    if (fix)
      for (int i = threadIdx.x; i < 3 * BN; i += NT) corr[i] = 0.0;
    __syncthreads();
    const double h = M.h[b], h3 = h * h * h;
    const double dtb = block_dt(M, b, dt);
    const double facA = -dtb / h * h3;
    const double facD = (nu / h) * (dtb / h) * h3;
    if (fix) {
      for (int f = 0; f < 6; ++f) {
        if (M.fkind[b * 6 + f] != K_FINER) continue;
        const int d = f >> 1, s = f & 1;
        if (threadIdx.x < 64) {
          const int a = threadIdx.x & 7, bb = threadIdx.x >> 3;
          int q[3], g[3];
          face_lab_pair(d, s, a, bb, q, g);
          const int ch = M.fnbr[b * 24 + 4 * f + (a >> 2) + 2 * (bb >> 2)];
          const double hf = M.h[ch];
          const double facDf = (nu / hf) * (dtb / hf) * hf * hf * hf;
          const int oc = face_cell(d, s, 0, a, bb);
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            double val = facD * (lab[c * LG::V + LG::at(q[0], q[1], q[2])] - lab[c * LG::V + LG::at(g[0], g[1], g[2])]);
#pragma unroll
            for (int e2 = 0; e2 < 2; ++e2)
#pragma unroll
              for (int e1 = 0; e1 < 2; ++e1) {
                const int fa = 2 * (a & 3) + e1, fb = 2 * (bb & 3) + e2;
                const double uf = vin[c * n + size_t(ch) * BN + face_cell(d, 1 - s, 0, fa, fb)];
                const double gf = child_ghost1([&](int cell) { return vin[c * n + size_t(b) * BN + cell]; }, M,
                                               ch, d, s, fa, fb);
                val += facDf * (uf - gf);
              }
            corr[c * BN + oc] += val;
          }
        }
        __syncthreads();
      }
    }
    if (SCHEME == 1) {
      // WENO5: each face value is reconstructed once where the cells on both
      // sides take the same upwind side.  Per direction: every cell
      // reconstructs its upper face into fbuf; the lower faces of the first
      // cells of the lines go to fstart; a cell then takes its lower face from
      // the cell below, or reconstructs it itself where the upwind sign flips.
      // The face values are those of deriv<1> (the same reconstruction of the
      // same inputs), so the result does not change.
      double* fbuf = corr + 3 * BN;   // 3 x 512: upper faces along the current direction
      double* fstart = fbuf + 3 * BN; // 3 x 64: lower faces of the lines' first cells
      auto L = [&](int c, int xx, int yy, int zz) { return lab[c * LG::V + LG::at(xx, yy, zz)]; };
      double der[2][3][3];  // [cell slot][component][direction]
      auto direction = [&](auto dconst) {
        constexpr int d = decltype(dconst)::value;
        constexpr int stride = d == 0 ? 1 : (d == 1 ? 8 : 64);
        // reconstruction at the upper face of cell (p0, p1, p2) along d with
        // the upwind side pos, as deriv<1>'s fp
        auto face_up = [&](int c, int p0, int p1, int p2, bool pos) {
          auto at = [&](int k) {
            return L(c, p0 + (d == 0 ? k : 0), p1 + (d == 1 ? k : 0), p2 + (d == 2 ? k : 0));
          };
          const double um2 = at(-2), um1 = at(-1), u0 = at(0), up1 = at(1), up2 = at(2), up3 = at(3);
          return weno5_left(pos ? um2 : up3, pos ? um1 : up2, pos ? u0 : up1, pos ? up1 : u0, pos ? up2 : um1);
        };
#pragma unroll 1
        for (int qq = 0; qq < 2; ++qq) {
          const int cell = threadIdx.x + qq * NT;
          const int x = cell & 7, y = (cell >> 3) & 7, z = cell >> 6;
          const bool pos = L(d, x, y, z) + ui.v[d] > 0;
#pragma unroll 1
          for (int c = 0; c < 3; ++c) fbuf[c * BN + cell] = face_up(c, x, y, z, pos);
        }
        if (threadIdx.x < 3 * 64) {
          const int c = threadIdx.x >> 6, line = threadIdx.x & 63;
          const int t1 = line & 7, t2 = line >> 3;
          const int x = d == 0 ? 0 : t1, y = d == 1 ? 0 : (d == 0 ? t1 : t2), z = d == 2 ? 0 : t2;
          const bool pos = L(d, x, y, z) + ui.v[d] > 0;  // the first cell's side
          fstart[c * 64 + line] = face_up(c, x - (d == 0), y - (d == 1), z - (d == 2), pos);
        }
        __syncthreads();
#pragma unroll
        for (int qq = 0; qq < 2; ++qq) {
          const int cell = threadIdx.x + qq * NT;
          const int x = cell & 7, y = (cell >> 3) & 7, z = cell >> 6;
          const int pd = d == 0 ? x : (d == 1 ? y : z);
          const bool pos = L(d, x, y, z) + ui.v[d] > 0;
          double fm[3];
          if (pd == 0) {
            const int line = d == 0 ? y + 8 * z : (d == 1 ? x + 8 * z : x + 8 * y);
#pragma unroll
            for (int c = 0; c < 3; ++c) fm[c] = fstart[c * 64 + line];
          } else {
            const int xm = x - (d == 0), ym = y - (d == 1), zm = z - (d == 2);
            const bool pos_m = L(d, xm, ym, zm) + ui.v[d] > 0;
            if (pos_m == pos) {
#pragma unroll
              for (int c = 0; c < 3; ++c) fm[c] = fbuf[c * BN + cell - stride];
            } else {  // the upwind side flips between the two cells
#pragma unroll
              for (int c = 0; c < 3; ++c) fm[c] = face_up(c, xm, ym, zm, pos);
            }
          }
#pragma unroll
          for (int c = 0; c < 3; ++c) der[qq][c][d] = fbuf[c * BN + cell] - fm[c];
        }
        __syncthreads();
      };
      direction(std::integral_constant<int, 0>{});
      direction(std::integral_constant<int, 1>{});
      direction(std::integral_constant<int, 2>{});
#pragma unroll 1
      for (int qq = 0; qq < 2; ++qq) {
        const int cell = threadIdx.x + qq * NT;
        const int x = cell & 7, y = (cell >> 3) & 7, z = cell >> 6;
        const double uA[3] = {L(0, x, y, z) + ui.v[0], L(1, x, y, z) + ui.v[1], L(2, x, y, z) + ui.v[2]};
        double out[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const double dx = der[qq][c][0], dy = der[qq][c][1], dz = der[qq][c][2];
          const double sx = L(c, x + 1, y, z) + L(c, x - 1, y, z);
          const double sy = L(c, x, y + 1, z) + L(c, x, y - 1, z);
          const double sz = L(c, x, y, z + 1) + L(c, x, y, z - 1);
          double dD, dA;
          if (c == 0) {
            dD = (sx + (sy + sz)) - 6 * L(0, x, y, z);
            dA = uA[0] * dx + (uA[1] * dy + uA[2] * dz);
          } else if (c == 1) {
            dD = (sy + (sz + sx)) - 6 * L(1, x, y, z);
            dA = uA[1] * dy + (uA[2] * dz + uA[0] * dx);
          } else {
            dD = (sz + (sx + sy)) - 6 * L(2, x, y, z);
            dA = uA[2] * dz + (uA[0] * dx + uA[1] * dy);
          }
          out[c] = facA * dA + facD * dD;
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const size_t gi = c * n + size_t(b) * BN + cell;
          double tot = (stage ? tmpV[gi] : 0.0) + out[c];
          if (fix) tot += corr[c * BN + cell];
          vout[gi] = L(c, x, y, z) + tot * (alpha / h3);
          if (stage < 2) tmpV[gi] = tot * beta;
        }
      }
      continue;
    }
    // the cell and component loops stay rolled: the unrolled body (18 WENO
    // reconstructions per cell) overflowed the instruction cache (the top
    // stall was no_instruction); rolled, a stage takes 188 us instead of 204
#pragma unroll 1
    for (int qq = 0; qq < 2; ++qq) {
      const int cell = threadIdx.x + qq * NT;
      const int x = cell & 7, y = (cell >> 3) & 7, z = cell >> 6;
      auto L = [&](int c, int xx, int yy, int zz) { return lab[c * LG::V + LG::at(xx, yy, zz)]; };
      const double uA[3] = {L(0, x, y, z) + ui.v[0], L(1, x, y, z) + ui.v[1], L(2, x, y, z) + ui.v[2]};
      double out[3];
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {
        const double dx = deriv<SCHEME>(uA[0], L(c, x - 3, y, z), L(c, x - 2, y, z), L(c, x - 1, y, z), L(c, x, y, z),
                                        L(c, x + 1, y, z), L(c, x + 2, y, z), L(c, x + 3, y, z));
        const double dy = deriv<SCHEME>(uA[1], L(c, x, y - 3, z), L(c, x, y - 2, z), L(c, x, y - 1, z), L(c, x, y, z),
                                        L(c, x, y + 1, z), L(c, x, y + 2, z), L(c, x, y + 3, z));
        const double dz = deriv<SCHEME>(uA[2], L(c, x, y, z - 3), L(c, x, y, z - 2), L(c, x, y, z - 1), L(c, x, y, z),
                                        L(c, x, y, z + 1), L(c, x, y, z + 2), L(c, x, y, z + 3));
        const double sx = L(c, x + 1, y, z) + L(c, x - 1, y, z);
        const double sy = L(c, x, y + 1, z) + L(c, x, y - 1, z);
        const double sz = L(c, x, y, z + 1) + L(c, x, y, z - 1);
        double dD, dA;
        if (c == 0) {
          dD = (sx + (sy + sz)) - 6 * L(0, x, y, z);
          dA = uA[0] * dx + (uA[1] * dy + uA[2] * dz);
        } else if (c == 1) {
          dD = (sy + (sz + sx)) - 6 * L(1, x, y, z);
          dA = uA[1] * dy + (uA[2] * dz + uA[0] * dx);
        } else {
          dD = (sz + (sx + sy)) - 6 * L(2, x, y, z);
          dA = uA[2] * dz + (uA[0] * dx + uA[1] * dy);
        }
        out[c] = facA * dA + facD * dD;
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const size_t gi = c * n + size_t(b) * BN + cell;
        double tot = (stage ? tmpV[gi] : 0.0) + out[c];
        if (fix) tot += corr[c * BN + cell];
        vout[gi] = L(c, x, y, z) + tot * (alpha / h3);
        if (stage < 2) tmpV[gi] = tot * beta;
      }
    }
  }
}

int launch_advect_stage(const DevMesh& M, const double* vin, double* vout, double* tmpV, double dt, double nu,
                        const double* uinf, int scheme, int stage, int grid, cudaStream_t s) {
  // lab, flux correction; WENO5 adds the face buffers (3 x 512 + 3 x 64)
  const size_t smem = (3 * LabGeom<3>::V + 3 * BN + (scheme == 1 ? 3 * BN + 3 * 64 : 0)) * sizeof(double);
  static unsigned long long attr_set[2] = {0, 0};
  Vec3 ui{{uinf[0], uinf[1], uinf[2]}};
  if (scheme == 1) {
    if (first_on_device(attr_set[1]))
      CUP_CUDA_TRY(cudaFuncSetAttribute(k_advect_stage<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    ProfScope ps("advect_stage_weno5", s);
    k_advect_stage<1><<<grid, NT, smem, s>>>(M, vin, vout, tmpV, dt, nu, ui, stage);
  } else {
    if (first_on_device(attr_set[0]))
      CUP_CUDA_TRY(cudaFuncSetAttribute(k_advect_stage<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    ProfScope ps("advect_stage_upwind5", s);
    k_advect_stage<0><<<grid, NT, smem, s>>>(M, vin, vout, tmpV, dt, nu, ui, stage);
  }
  CUP_CUDA_TRY(cudaGetLastError());
  return 0;
}

// ---------------------------------------------------------------------------
// PressureProjection RHS: KernelPressureRHS (PressureProjection.cpp:96-199),
// kernelUpdateTmpV (:202-242) and KernelDivPressure (:16-94, step > 2).
// ---------------------------------------------------------------------------
struct UdefGet {
  ObstacleView ob;
  const double* chi;
  __device__ __forceinline__ double operator()(int c, int blk, int cell) const {
    const int sl = ob.slot[blk];
    if (sl < 0) return 0.0;
    return chi[size_t(blk) * BN + cell] <= ob.chi[size_t(sl) * BN + cell]
               ? ob.udef[(size_t(c) * ob.nslots + sl) * BN + cell]
               : 0.0;
  }
};

// One CTA walks its blocks through the staged pipeline (staged.cuh): the
// velocity and p_old labs arrive by bulk copies and per-cell async copies
// while the previous block is computed.  Blocks next to the body (rare) add
// the u_def lab with plain loads.
template <int USE_POLD>
__global__ void __launch_bounds__(NT, 2)
    k_pressure_rhs(DevMesh M, const double* __restrict__ vel, const double* __restrict__ pold,
                   const double* __restrict__ chi, ObstacleView ob, double dt, double* __restrict__ lhs,
                   double* __restrict__ phi) {
  extern __shared__ __align__(16) unsigned char stage_smem[];
  constexpr int NCH = 3 + USE_POLD;
  using SS = StagedShape<NCH, 0>;
  using LG = LabGeom<1>;
  double* dlab = reinterpret_cast<double*>(stage_smem + SS::kBytes);
  double* corr = dlab + 3 * LG::V;  // [0,512): RHS flux correction, [512,1024): div p correction
  const size_t n = size_t(M.nb) * BN;
  const double* src[NCH];
#pragma unroll
  for (int c = 0; c < NCH; ++c) src[c] = c < 3 ? vel + c * n : pold;
  auto getV = [&](int c, int blk, int cell) { return vel[c * n + size_t(blk) * BN + cell]; };
  auto getP = [&](int, int blk, int cell) { return pold[size_t(blk) * BN + cell]; };
  UdefGet getD{ob, chi};
  staged_blocks<NCH, 0>(M, src, ob.near, stage_smem, M.kerr, [&](int, int b, const StageMeta& m, double* ulab) {
    double* plab = ulab + 3 * LG::V;
    stage_fixup<3>(ulab, M, m, getV, true);
    if (USE_POLD) stage_fixup<1>(plab, M, m, getP, false);
    const bool near = m.flag != 0;
    if (near) lab_fill<1, 3>(dlab, M, b, getD, true);
    const bool fix = meta_has_finer(m);
    if (fix)
      for (int i = threadIdx.x; i < 2 * BN; i += NT) corr[i] = 0.0;
    __syncthreads();
    const double dtb = block_dt(M, b, dt);
    const double h = m.h, fac = 0.5 * h * h / dtb;
    auto U = [&](int c, int x, int y, int z) { return ulab[c * LG::V + LG::at(x, y, z)]; };
    auto D = [&](int c, int x, int y, int z) { return near ? dlab[c * LG::V + LG::at(x, y, z)] : 0.0; };
    auto P = [&](int x, int y, int z) { return plab[LG::at(x, y, z)]; };
    if (fix) {
      for (int f = 0; f < 6; ++f) {
        if (m.kind[f] != K_FINER) continue;
        const int d = f >> 1, s = f & 1;
        if (threadIdx.x < 64) {
          const int a = threadIdx.x & 7, bb = threadIdx.x >> 3;
          int q[3], g[3];
          face_lab_pair(d, s, a, bb, q, g);
          const int ch = m.nbr[4 * f + (a >> 2) + 2 * (bb >> 2)];
          const double hf = M.h[ch], facf = 0.5 * hf * hf / dtb;
          const int oc = face_cell(d, s, 0, a, bb);
          const double sg = s ? -1.0 : 1.0, sgc = -sg;
          const double cq = chi[size_t(b) * BN + oc];
          double vr = sg * fac * (U(d, g[0], g[1], g[2]) + U(d, q[0], q[1], q[2])) -
                      sg * cq * fac * (D(d, g[0], g[1], g[2]) + D(d, q[0], q[1], q[2]));
          double vp = USE_POLD ? h * (P(q[0], q[1], q[2]) - P(g[0], g[1], g[2])) : 0.0;
#pragma unroll
          for (int e2 = 0; e2 < 2; ++e2)
#pragma unroll
            for (int e1 = 0; e1 < 2; ++e1) {
              const int fa = 2 * (a & 3) + e1, fb = 2 * (bb & 3) + e2;
              const int cf = face_cell(d, 1 - s, 0, fa, fb);
              const double uf = getV(d, ch, cf);
              const double gu = child_ghost1([&](int cell) { return getV(d, b, cell); }, M, ch, d, s, fa, fb);
              const double cf_chi = chi[size_t(ch) * BN + cf];
              double df = 0.0, gd = 0.0;
              if (near) {
                df = getD(d, ch, cf);
                gd = child_ghost1([&](int cell) { return getD(d, b, cell); }, M, ch, d, s, fa, fb);
              }
              vr += sgc * facf * (gu + uf) - sgc * cf_chi * facf * (gd + df);
              if (USE_POLD) {
                const double pf = getP(0, ch, cf);
                const double gp = child_ghost1([&](int cell) { return getP(0, b, cell); }, M, ch, d, s, fa, fb);
                vp += hf * (pf - gp);
              }
            }
          corr[oc] += vr;
          corr[BN + oc] += vp;
        }
        __syncthreads();
      }
    }
    for (int qq = 0; qq < 2; ++qq) {
      const int cell = threadIdx.x + qq * NT;
      const int x = cell & 7, y = (cell >> 3) & 7, z = cell >> 6;
      const size_t gi = size_t(b) * BN + cell;
      double p = fac * (U(0, x + 1, y, z) - U(0, x - 1, y, z) + U(1, x, y + 1, z) - U(1, x, y - 1, z) +
                        U(2, x, y, z + 1) - U(2, x, y, z - 1));
      if (near) {
        const double divUs = D(0, x + 1, y, z) - D(0, x - 1, y, z) + D(1, x, y + 1, z) - D(1, x, y - 1, z) +
                             D(2, x, y, z + 1) - D(2, x, y, z - 1);
        p += -chi[gi] * fac * divUs;
      }
      if (fix) p += corr[cell];
      if (USE_POLD) {
        double dp = h * (P(x + 1, y, z) + P(x - 1, y, z) + P(x, y + 1, z) + P(x, y - 1, z) + P(x, y, z + 1) +
                         P(x, y, z - 1) - 6.0 * P(x, y, z));
        if (fix) dp += corr[BN + cell];
        p -= dp;
      }
      lhs[gi] = p;
      phi[gi] = 0.0;
    }
    __syncthreads();
  });
}

// CTAs of a staged kernel that fit on the device at once: the pipeline wants
// one resident wave of CTAs, each walking several blocks.
template <class K>
static int resident_ctas(K kern, size_t smem, unsigned long long& cached_mask, int* cache) {
  int dev = 0;
  CUP_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev > 63) return set_error(CUP_ERR_ARG, "device ordinal above 63");
  if (first_on_device(cached_mask)) {
    int per_sm = 0, sms = 0;
    CUP_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    CUP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem));
    CUP_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (per_sm < 1) return set_error(CUP_ERR_CUDA, "staged stencil kernel does not fit on an SM");
    cache[dev] = per_sm * sms;
  }
  return 0;
}

template <int USE_POLD>
constexpr size_t rhs_smem() {
  return StagedShape<3 + USE_POLD, 0>::kBytes + (3 * LabGeom<1>::V + 2 * BN) * sizeof(double);
}

int launch_pressure_rhs(const DevMesh& M, const double* vel, const double* pold, const double* chi,
                        const ObstacleView& ob, double dt, int step, int step_2nd_start, double* lhs, double* phi,
                        int grid, cudaStream_t s) {
  static unsigned long long attr[2] = {0, 0};
  static int resident[2][64];
  int dev = 0;
  CUP_CUDA_TRY(cudaGetDevice(&dev));
  ProfScope ps("pressure_rhs", s);
  // with udef = 0 in every slot the near-body terms (chi times the
  // divergence of udef, with its flux correction) are exact zeros: no block
  // needs the udef lab
  ObstacleView o = ob;
  if (o.udef_zero) o.near = nullptr;
  if (step > step_2nd_start) {
    if (int rc = resident_ctas(k_pressure_rhs<1>, rhs_smem<1>(), attr[1], resident[1])) return rc;
    grid = std::max(1, std::min({grid, resident[1][dev], M.nb}));
    k_pressure_rhs<1><<<grid, NT, rhs_smem<1>(), s>>>(M, vel, pold, chi, o, dt, lhs, phi);
  } else {
    if (int rc = resident_ctas(k_pressure_rhs<0>, rhs_smem<0>(), attr[0], resident[0])) return rc;
    grid = std::max(1, std::min({grid, resident[0][dev], M.nb}));
    k_pressure_rhs<0><<<grid, NT, rhs_smem<0>(), s>>>(M, vel, pold, chi, o, dt, lhs, phi);
  }
  CUP_CUDA_TRY(cudaGetLastError());
  return 0;
}

// ---------------------------------------------------------------------------
// Mean removal + incremental pressure (PressureProjection.cpp:404-446) fused
// with KernelGradP (:244-323) and the velocity update (:451-467).  The
// pressure p = phi - avg (+ p_old) is formed at the point of use from the
// staged phi and p_old labs; the velocity comes in with them as interiors.
// ---------------------------------------------------------------------------
template <int USE_POLD>
__global__ void __launch_bounds__(NT, 3)
    k_grad_update(DevMesh M, double* vel, const double* __restrict__ phi, const double* __restrict__ pold,
                  double* __restrict__ pnew, const double* sums, double dt) {
  extern __shared__ __align__(16) unsigned char stage_smem[];
  constexpr int NCH = 1 + USE_POLD;
  using SS = StagedShape<NCH, 3>;
  using LG = LabGeom<1>;
  double* corr = reinterpret_cast<double*>(stage_smem + SS::kBytes);  // 3 BN
  const size_t n = size_t(M.nb) * BN;
  const double* src[NCH + 3];
#pragma unroll
  for (int c = 0; c < NCH; ++c) src[c] = c == 0 ? phi : pold;
#pragma unroll
  for (int c = 0; c < 3; ++c) src[NCH + c] = vel + c * n;
  auto getPhi = [&](int, int blk, int cell) { return phi[size_t(blk) * BN + cell]; };
  auto getPold = [&](int, int blk, int cell) { return pold[size_t(blk) * BN + cell]; };
  staged_blocks<NCH, 3>(M, src, nullptr, stage_smem, M.kerr, [&](int, int b, const StageMeta& m, double* st) {
    double* flab = st;
    double* olab = st + LG::V;
    const double* vin = st + NCH * LG::V;
    const double avg = M.case_sums ? M.case_sums[2 * M.bcase[b]] / M.case_sums[2 * M.bcase[b] + 1]
                                   : (sums ? sums[0] / sums[1] : 0.0);
    // the pressure of any cell of the mesh (coarse-fine flux correction)
    auto getP = [&](int, int blk, int cell) {
      const size_t i = size_t(blk) * BN + cell;
      const double p = phi[i] - avg;
      return USE_POLD ? p + pold[i] : p;
    };
    stage_fixup<1>(flab, M, m, getPhi, false);
    if (USE_POLD) stage_fixup<1>(olab, M, m, getPold, false);
    const bool fix = meta_has_finer(m);
    if (fix)
      for (int i = threadIdx.x; i < 3 * BN; i += NT) corr[i] = 0.0;
    __syncthreads();
    const double dtb = block_dt(M, b, dt);
    const double h = m.h, fac = -0.5 * dtb * h * h;
    auto P = [&](int x, int y, int z) {
      const int i = LG::at(x, y, z);
      const double p = flab[i] - avg;
      return USE_POLD ? p + olab[i] : p;
    };
    if (fix) {
      for (int f = 0; f < 6; ++f) {
        if (m.kind[f] != K_FINER) continue;
        const int d = f >> 1, s = f & 1;
        if (threadIdx.x < 64) {
          const int a = threadIdx.x & 7, bb = threadIdx.x >> 3;
          int q[3], g[3];
          face_lab_pair(d, s, a, bb, q, g);
          const int ch = m.nbr[4 * f + (a >> 2) + 2 * (bb >> 2)];
          const double hf = M.h[ch], facf = -0.5 * dtb * hf * hf;
          const double sg = s ? -1.0 : 1.0, sgc = -sg;
          double v = sg * fac * (P(g[0], g[1], g[2]) + P(q[0], q[1], q[2]));
#pragma unroll
          for (int e2 = 0; e2 < 2; ++e2)
#pragma unroll
            for (int e1 = 0; e1 < 2; ++e1) {
              const int fa = 2 * (a & 3) + e1, fb = 2 * (bb & 3) + e2;
              const int cf = face_cell(d, 1 - s, 0, fa, fb);
              const double pf = getP(0, ch, cf);
              const double gp = child_ghost1([&](int cell) { return getP(0, b, cell); }, M, ch, d, s, fa, fb);
              v += sgc * facf * (gp + pf);
            }
          corr[d * BN + face_cell(d, s, 0, a, bb)] += v;
        }
        __syncthreads();
      }
    }
    const double ih3 = 1.0 / (h * h * h);
    for (int qq = 0; qq < 2; ++qq) {
      const int cell = threadIdx.x + qq * NT;
      const int x = cell & 7, y = (cell >> 3) & 7, z = cell >> 6;
      const size_t gi = size_t(b) * BN + cell;
      double g0 = fac * (P(x + 1, y, z) - P(x - 1, y, z));
      double g1 = fac * (P(x, y + 1, z) - P(x, y - 1, z));
      double g2 = fac * (P(x, y, z + 1) - P(x, y, z - 1));
      if (fix) {
        g0 += corr[cell];
        g1 += corr[BN + cell];
        g2 += corr[2 * BN + cell];
      }
      vel[gi] = vin[cell] + ih3 * g0;
      vel[n + gi] = vin[BN + cell] + ih3 * g1;
      vel[2 * n + gi] = vin[2 * BN + cell] + ih3 * g2;
      pnew[gi] = P(x, y, z);
    }
    __syncthreads();
  });
}

template <int USE_POLD>
constexpr size_t grad_smem() {
  return StagedShape<1 + USE_POLD, 3>::kBytes + 3 * BN * sizeof(double);
}

int launch_grad_update(const DevMesh& M, double* vel, const double* phi, const double* pold, double* pnew,
                       const double* sums, double dt, int step, int step_2nd_start, int grid, cudaStream_t s) {
  static unsigned long long attr[2] = {0, 0};
  static int resident[2][64];
  int dev = 0;
  CUP_CUDA_TRY(cudaGetDevice(&dev));
  ProfScope ps("grad_update", s);
  if (step > step_2nd_start) {
    if (int rc = resident_ctas(k_grad_update<1>, grad_smem<1>(), attr[1], resident[1])) return rc;
    grid = std::max(1, std::min({grid, resident[1][dev], M.nb}));
    k_grad_update<1><<<grid, NT, grad_smem<1>(), s>>>(M, vel, phi, pold, pnew, sums, dt);
  } else {
    if (int rc = resident_ctas(k_grad_update<0>, grad_smem<0>(), attr[0], resident[0])) return rc;
    grid = std::max(1, std::min({grid, resident[0][dev], M.nb}));
    k_grad_update<0><<<grid, NT, grad_smem<0>(), s>>>(M, vel, phi, pold, pnew, sums, dt);
  }
  CUP_CUDA_TRY(cudaGetLastError());
  return 0;
}

// ---------------------------------------------------------------------------
// Penalization: KernelPenalization (Penalization.cpp:56-89) on obstacle blocks
// and the force/torque sums of kernelFinalizePenalizationForce (:91-109).
// ---------------------------------------------------------------------------
// In a batch (M.bcase set) each slot takes its case's kinematics and time
// step, and the force/torque sums go per slot into slot_force[6 * slot].
__global__ void __launch_bounds__(NT)
    k_penalize(DevMesh M, double* vel, const double* __restrict__ chi, ObstacleView ob, const double* __restrict__ kin,
               double dt, double lambda, int implicit, GridReduce G, double* force, double* slot_force) {
  __shared__ double red[8 * 6];
  const size_t n = size_t(M.nb) * BN;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int sl = blockIdx.x; sl < ob.nslots; sl += gridDim.x) {
    const int b = ob.blk[sl];
    const double* kn = M.case_kin ? M.case_kin + 9 * M.bcase[b] : kin;
    const double CM[3] = {kn[0], kn[1], kn[2]};
    const double V[3] = {kn[3], kn[4], kn[5]};
    const double O[3] = {kn[6], kn[7], kn[8]};
    const double dtb = block_dt(M, b, dt);
    const double lambdaFac = implicit ? lambda : 1.0 / dtb;
    const double h = M.h[b], dv = h * h * h;
    for (int cell = threadIdx.x; cell < BN; cell += NT) {
      const size_t gi = size_t(b) * BN + cell;
      const double CHI = ob.chi[size_t(sl) * BN + cell];
      if (chi[gi] > CHI) continue;
      if (CHI <= 0) continue;
      const int x = cell & 7, y = (cell >> 3) & 7, z = cell >> 6;
      double p[3] = {(M.index[3 * b] * BS + x + 0.5) * h, (M.index[3 * b + 1] * BS + y + 0.5) * h,
                     (M.index[3 * b + 2] * BS + z + 0.5) * h};
      p[0] -= CM[0];
      p[1] -= CM[1];
      p[2] -= CM[2];
      const double* ud = ob.udef;
      const size_t ns = ob.nslots;
      const double U0 = V[0] + O[1] * p[2] - O[2] * p[1] + ud[(0 * ns + sl) * BN + cell];
      const double U1 = V[1] + O[2] * p[0] - O[0] * p[2] + ud[(1 * ns + sl) * BN + cell];
      const double U2 = V[2] + O[0] * p[1] - O[1] * p[0] + ud[(2 * ns + sl) * BN + cell];
      const double X = implicit ? (CHI > 0.5 ? 1.0 : 0.0) : CHI;
      const double penalFac = implicit ? X * lambdaFac / (1 + X * lambdaFac * dtb) : X * lambdaFac;
      const double FPX = penalFac * (U0 - vel[gi]);
      const double FPY = penalFac * (U1 - vel[n + gi]);
      const double FPZ = penalFac * (U2 - vel[2 * n + gi]);
      vel[gi] = vel[gi] + dtb * FPX;
      vel[n + gi] = vel[n + gi] + dtb * FPY;
      vel[2 * n + gi] = vel[2 * n + gi] + dtb * FPZ;
      acc[0] += dv * FPX;
      acc[1] += dv * FPY;
      acc[2] += dv * FPZ;
      acc[3] += dv * (p[1] * FPZ - p[2] * FPY);
      acc[4] += dv * (p[2] * FPX - p[0] * FPZ);
      acc[5] += dv * (p[0] * FPY - p[1] * FPX);
    }
    if (slot_force) {  // uniform over the CTA
      block_reduce<6>(acc, red);
      if (threadIdx.x == 0)
        for (int q = 0; q < 6; ++q) slot_force[6 * sl + q] = acc[q];
      for (int q = 0; q < 6; ++q) acc[q] = 0.0;
    }
  }
  if (!slot_force && grid_reduce<6>(acc, G, red) && threadIdx.x == 0)
    for (int q = 0; q < 6; ++q) force[q] = acc[q];
}

int launch_penalize(const DevMesh& M, double* vel, const double* chi, const ObstacleView& ob, const double* kin,
                    double dt, double lambda, int implicit, double* force, double* partial, unsigned* counter,
                    cudaStream_t s, double* slot_force) {
  if (ob.nslots <= 0) {
    if (slot_force) return 0;
    CUP_CUDA_TRY(cudaMemsetAsync(force, 0, 6 * sizeof(double), s));
    return 0;
  }
  const int grid = std::min(ob.nslots, 1184);
  GridReduce G{partial, counter};
  ProfScope ps("penalize", s);
  k_penalize<<<grid, NT, 0, s>>>(M, vel, chi, ob, kin, dt, lambda, implicit, G, force, slot_force);
  CUP_CUDA_TRY(cudaGetLastError());
  return 0;
}

// ---------------------------------------------------------------------------
// findMaxU (ProcessHelpers.h:71-94)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(NT) k_max_u(size_t n, const double* __restrict__ vel, Vec3 ui, GridReduce G,
                                              double* out) {
  __shared__ double red[8];
  double m = 0.0;
  for (size_t i = size_t(blockIdx.x) * NT + threadIdx.x; i < n; i += size_t(gridDim.x) * NT) {
    const double a = fabs(vel[i] + ui.v[0]);
    const double b = fabs(vel[n + i] + ui.v[1]);
    const double c = fabs(vel[2 * n + i] + ui.v[2]);
    m = fmax(m, fmax(a, fmax(b, c)));
  }
  if (grid_reduce_max(m, G, red) && threadIdx.x == 0) *out = m;
}

int launch_max_u(const DevMesh& M, const double* vel, const double* uinf, double* out, double* partial,
                 unsigned* counter, int grid, cudaStream_t s) {
  GridReduce G{partial, counter};
  Vec3 ui{{uinf[0], uinf[1], uinf[2]}};
  ProfScope ps("max_u", s);
  k_max_u<<<grid, NT, 0, s>>>(size_t(M.nb) * BN, vel, ui, G, out);
  CUP_CUDA_TRY(cudaGetLastError());
  return 0;
}

// ---------------------------------------------------------------------------
// Per-case reductions of a batch: per-item values (blocks or obstacle slots),
// then one CTA per case over the case's item range, in a fixed order.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(NT) k_block_max_u(DevMesh M, const double* __restrict__ vel, Vec3 ui,
                                                    double* bmax) {
  __shared__ double red[NT / 32];
  const size_t n = size_t(M.nb) * BN;
  for (int b = blockIdx.x; b < M.nb; b += gridDim.x) {
    double m = 0.0;
    for (int c = threadIdx.x; c < BN; c += NT) {
      const size_t i = size_t(b) * BN + c;
      m = fmax(m, fmax(fabs(vel[i] + ui.v[0]), fmax(fabs(vel[n + i] + ui.v[1]), fabs(vel[2 * n + i] + ui.v[2]))));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
      double mm = 0.0;
      for (int w = 0; w < NT / 32; ++w) mm = fmax(mm, red[w]);
      bmax[b] = mm;
    }
  }
}

// (sum phi h^3, sum h^3) of each block
__global__ void __launch_bounds__(NT) k_block_sums(DevMesh M, const double* __restrict__ phi, double* bsum) {
  __shared__ double red[64];
  for (int b = blockIdx.x; b < M.nb; b += gridDim.x) {
    const double h = M.h[b], h3 = h * h * h;
    double v[1] = {0.0};
    for (int c = threadIdx.x; c < BN; c += NT) v[0] += phi[size_t(b) * BN + c];
    block_reduce<1>(v, red);
    if (threadIdx.x == 0) {
      bsum[2 * b] = v[0] * h3;
      bsum[2 * b + 1] = BN * h3;
    }
  }
}

// out[NR c + r] = sum (MAX = 0) or max (MAX = 1) of in[NR i + r], i in [first[c], first[c+1])
template <int NR, int MAX>
__global__ void __launch_bounds__(NT) k_case_reduce(const double* __restrict__ in, const int* __restrict__ first,
                                                    double* out) {
  __shared__ double red[8 * NR];
  const int c = blockIdx.x;
  double v[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) v[r] = 0.0;
  for (int i = first[c] + threadIdx.x; i < first[c + 1]; i += NT)
#pragma unroll
    for (int r = 0; r < NR; ++r) v[r] = MAX ? fmax(v[r], in[size_t(NR) * i + r]) : v[r] + in[size_t(NR) * i + r];
  if (MAX) {
#pragma unroll
    for (int r = 0; r < NR; ++r) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v[r] = fmax(v[r], __shfl_xor_sync(0xffffffffu, v[r], o));
      if ((threadIdx.x & 31) == 0) red[(threadIdx.x >> 5) * NR + r] = v[r];
    }
    __syncthreads();
    if (threadIdx.x == 0)
      for (int r = 0; r < NR; ++r) {
        double m = 0.0;
        for (int w = 0; w < NT / 32; ++w) m = fmax(m, red[w * NR + r]);
        out[NR * c + r] = m;
      }
  } else {
    block_reduce<NR>(v, red);
    if (threadIdx.x == 0)
      for (int r = 0; r < NR; ++r) out[NR * c + r] = v[r];
  }
}

int launch_case_max_u(const DevMesh& M, const double* vel, const double* uinf, double* bmax, const int* first,
                      int ncase, double* out, int grid, cudaStream_t s) {
  Vec3 ui{{uinf[0], uinf[1], uinf[2]}};
  ProfScope ps("case_max_u", s);
  k_block_max_u<<<grid, NT, 0, s>>>(M, vel, ui, bmax);
  k_case_reduce<1, 1><<<ncase, NT, 0, s>>>(bmax, first, out);
  CUP_CUDA_TRY(cudaGetLastError());
  return 0;
}

int launch_case_sums(const DevMesh& M, const double* phi, double* bsum, const int* first, int ncase, double* out,
                     int grid, cudaStream_t s) {
  ProfScope ps("case_sums", s);
  k_block_sums<<<grid, NT, 0, s>>>(M, phi, bsum);
  k_case_reduce<2, 0><<<ncase, NT, 0, s>>>(bsum, first, out);
  CUP_CUDA_TRY(cudaGetLastError());
  return 0;
}

int launch_case_forces(const double* slot_force, const int* slot_first, int ncase, double* out, cudaStream_t s) {
  ProfScope ps("case_forces", s);
  k_case_reduce<6, 0><<<ncase, NT, 0, s>>>(slot_force, slot_first, out);
  CUP_CUDA_TRY(cudaGetLastError());
  return 0;
}

// ---------------------------------------------------------------------------
// Simulation::calcMaxTimestep on the device, for captured steps: the same
// operations in the same order as the host version (no contraction), with
// the CFL factor (ramped or not) computed on the host: bit-identical dt.
// ---------------------------------------------------------------------------
__global__ void k_calc_dt(const double* __restrict__ umax, const double* __restrict__ cfl_fac, double nu,
                          double hmin, double* dt) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double u = *umax;
  const double t = __dmul_rn(1.0 / 6.0, hmin);
  const double dtDiffusion = __ddiv_rn(__dmul_rn(t, hmin), __dadd_rn(nu, __dmul_rn(t, u)));
  const double dtAdvection = __ddiv_rn(hmin, __dadd_rn(u, 1e-8));
  const double cand = __dmul_rn(*cfl_fac, dtAdvection);
  *dt = cand < dtDiffusion ? cand : dtDiffusion;
}

int launch_calc_dt(const double* umax, const double* cfl_fac, double nu, double hmin, double* dt, cudaStream_t s) {
  k_calc_dt<<<1, 32, 0, s>>>(umax, cfl_fac, nu, hmin, dt);
  CUP_CUDA_TRY(cudaGetLastError());
  return 0;
}

// The same per case of a batch: dt[c] from umax[c] and hmin[c].
__global__ void k_case_calc_dt(const double* __restrict__ umax, const double* __restrict__ cfl_fac, double nu,
                               const double* __restrict__ hmin, int ncase, double* dt) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncase) return;
  const double u = umax[c], hm = hmin[c];
  const double t = __dmul_rn(1.0 / 6.0, hm);
  const double dtDiffusion = __ddiv_rn(__dmul_rn(t, hm), __dadd_rn(nu, __dmul_rn(t, u)));
  const double dtAdvection = __ddiv_rn(hm, __dadd_rn(u, 1e-8));
  const double cand = __dmul_rn(*cfl_fac, dtAdvection);
  dt[c] = cand < dtDiffusion ? cand : dtDiffusion;
}

int launch_case_calc_dt(const double* umax, const double* cfl_fac, double nu, const double* hmin, int ncase,
                        double* dt, cudaStream_t s) {
  k_case_calc_dt<<<(ncase + 127) / 128, 128, 0, s>>>(umax, cfl_fac, nu, hmin, ncase, dt);
  CUP_CUDA_TRY(cudaGetLastError());
  return 0;
}

}  // namespace cup3d
