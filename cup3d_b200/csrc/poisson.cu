// Poisson operator, exact block preconditioner and fused BiCGSTAB (FP64).
//
// Reference behaviour restated here:
//   * operator rows: PoissonSolverExp::getMat / makeFlux / interpolate
//     (PoissonSolverExp.cpp:112-373; D1/D2/Dmixed in PoissonSolverExp.h:384-478),
//     evaluated matrix-free instead of assembled into COO;
//   * mean constraint: hd_cusparseSpMV (BiCGSTAB.cu:392-413) and ComputeLHS
//     (PoissonSolverAMR.h:108-172);
//   * preconditioner: z = (1/h) P_inv p with P_inv = -(L_D)^-1 of the 8^3
//     Dirichlet Laplacian (PoissonSolverExp.cpp:17-111, BiCGSTAB.cu:526-527),
//     applied by fast diagonalization (three DST-I mode products each way)
//     rather than a 512x512 DGEMM: the same matrix, 96 instead of 1024 flop/cell;
//   * solver: BiCGSTABSolver::main (BiCGSTAB.cu:416-628) with the same
//     scalars, restart rule and best-iterate return, all iterations in one
//     cooperative launch with three grid barriers per iteration (five fused
//     kernels per iteration where a network preconditioner runs between
//     them) and no host round trip inside a solve.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "fd.cuh"
#include "group.cuh"
#include "lmap.cuh"
#include "poisson.cuh"
#include "profiler.h"
#include "cup3d_b200.h"

namespace cup3d {

static_assert(GROUPS == GROUPS_PER_CTA, "group layout");

void poisson_init_constants() { fd_init_constants(); }

// ---------------------------------------------------------------------------
// Coarse-fine interpolation of PoissonSolverExp::interpolate: the Taylor part
// p_c + s1 D1 + s2 D2' + D2(ds1) + D2(ds2) + s1 s2 Dmixed of one face layer
// L(u, v) at coarse face cell (u, v) (PoissonSolverExp.h:159-371, D1/D2/Dmixed
// at :384-478).  Faces normal to y use u = tan2 (z), v = tan1 (x); the others
// u = tan1, v = tan2.  The one-sided forms apply at u, v = 0, 4 (forward) and
// 3, 7 (backward), so every stencil stays inside the 4x4 quarter of the face
// that holds (u, v).  The terms are evaluated without branches, Dmixed
// included: all candidate forms from clamped in-quarter loads, then selects
// (a divergent branch per case serialises a warp up to nine times).
// ---------------------------------------------------------------------------
struct TaylorTerms {
  double c, d1u, d1v, d2u, d2v, dm;
  __device__ __forceinline__ double at(double su, double sv) const {
    return c + su * d1u + sv * d1v + d2u + d2v + su * sv * dm;
  }
};

__device__ __forceinline__ int quarter_clamp(int w, int o) {
  const int lo = w & 4, t = w + o;
  return t < lo ? lo : (t > lo + 3 ? lo + 3 : t);
}

// L(u, v): the face layer in (u, v) order
template <class Layer>
__device__ __forceinline__ TaylorTerms cf_terms(Layer L, int u, int v) {
  const bool bdu = (u & 3) == 3, fdu = (u & 3) == 0;
  const bool bdv = (v & 3) == 3, fdv = (v & 3) == 0;
  const int um1 = quarter_clamp(u, -1), up1 = quarter_clamp(u, 1), um2 = quarter_clamp(u, -2), up2 = quarter_clamp(u, 2);
  const int vm1 = quarter_clamp(v, -1), vp1 = quarter_clamp(v, 1), vm2 = quarter_clamp(v, -2), vp2 = quarter_clamp(v, 2);
  TaylorTerms T;
  const double c = L(u, v);
  const double Lum1 = L(um1, v), Lup1 = L(up1, v), Lum2 = L(um2, v), Lup2 = L(up2, v);
  const double Lvm1 = L(u, vm1), Lvp1 = L(u, vp1), Lvm2 = L(u, vm2), Lvp2 = L(u, vp2);
  const double Nmm = L(um1, vm1), Npp = L(up1, vp1), Npm = L(up1, vm1), Nmp = L(um1, vp1);
  T.c = c;
  T.d1u = bdu ? 1. / 8. * Lum2 - 1. / 2. * Lum1 + 3. / 8. * c
        : fdu ? -1. / 8. * Lup2 + 1. / 2. * Lup1 - 3. / 8. * c
              : -1. / 8. * Lum1 + 1. / 8. * Lup1;
  T.d2u = bdu ? 1. / 32. * Lum2 - 1. / 16. * Lum1 + 1. / 32. * c
        : fdu ? 1. / 32. * Lup2 - 1. / 16. * Lup1 + 1. / 32. * c
              : 1. / 32. * Lum1 + 1. / 32. * Lup1 - 1. / 16. * c;
  T.d1v = bdv ? 1. / 8. * Lvm2 - 1. / 2. * Lvm1 + 3. / 8. * c
        : fdv ? -1. / 8. * Lvp2 + 1. / 2. * Lvp1 - 3. / 8. * c
              : -1. / 8. * Lvm1 + 1. / 8. * Lvp1;
  T.d2v = bdv ? 1. / 32. * Lvm2 - 1. / 16. * Lvm1 + 1. / 32. * c
        : fdv ? 1. / 32. * Lvp2 - 1. / 16. * Lvp1 + 1. / 32. * c
              : 1. / 32. * Lvm1 + 1. / 32. * Lvp1 - 1. / 16. * c;
  // Dmixed: (N(u1,v1) + N(u0,v0)) - N(u0,v1) - N(u1,v0), N(i,j) = L(u+i, v+j),
  // with the pair (u0,u1) = (-1,0) at a backward edge, (0,+1) at a forward
  // edge and (-1,+1) at half weight in the middle (likewise for v): the nine
  // cases of PoissonSolverExp.h:442-478 in one branch-free form
  auto Nsel = [&](int i, int j) {
    const double rm = j < 0 ? Nmm : (j > 0 ? Nmp : Lum1);
    const double r0 = j < 0 ? Lvm1 : (j > 0 ? Lvp1 : c);
    const double rp = j < 0 ? Npm : (j > 0 ? Npp : Lup1);
    return i < 0 ? rm : (i > 0 ? rp : r0);
  };
  const int u1 = bdu ? 0 : 1, u0 = fdu ? 0 : -1, v1 = bdv ? 0 : 1, v0 = fdv ? 0 : -1;
  const double wu = (bdu || fdu) ? 1.0 : 0.5, wv = (bdv || fdv) ? 1.0 : 0.5;
  const double dm = (1. / 16.) * (wu * wv) * (((Nsel(u1, v1) + Nsel(u0, v0)) - Nsel(u0, v1)) - Nsel(u1, v0));
  T.dm = dm;
  return T;
}

// ---------------------------------------------------------------------------
// Vector accessors for the operator: x(i) gives the input vector's value at
// global cell index i.  VecAt reads a stored vector through L2; an accessor
// may also combine stored vectors at the point of use.
// ---------------------------------------------------------------------------
template <class T>
struct VecAt {
  const T* v;
  __device__ __forceinline__ double operator()(size_t i) const { return double(ld_stream(v + i)); }
};

// Group-cooperative copy of block b's table entries into bi (the caller
// synchronises the group before reading it).
__device__ __forceinline__ void fill_block_info(const DevMesh& M, int b, BlockInfo& bi, int lane) {
  if (lane < 6) {
    bi.kind[lane] = M.fkind[b * 6 + lane];
  } else if (lane < 30) {
    bi.nbr[lane - 6] = M.fnbr[b * 24 + lane - 6];
  } else if (lane == 30) {
    bi.h = M.h[b];
    bi.id = b;
    bi.mean = b == (M.bcase ? M.case_mean[M.bcase[b]] : M.mean_block) ? 1 : 0;
  } else if (lane == 31) {
    bi.par = (M.index[b * 3] & 1) | ((M.index[b * 3 + 1] & 1) << 1) | ((M.index[b * 3 + 2] & 1) << 2);
  }
}

// Flux across coarse-fine face f into face cell (a, bb) of block b
// (PoissonSolverExp::makeFlux, PoissonSolverExp.cpp:157-219): the fine side
// of a coarser face (coarse layer staged in tile.cl[f]), or the four fine
// fluxes of a finer face (Taylor terms from the block's own layer).  Reads
// the tile after the group barrier that follows its filling.
template <class X>
__device__ __forceinline__ double cf_flux(const BlockInfo& bi, const X& x, const GroupTile& tile, int f, int kind,
                                          int a, int bb) {
  const int d = f >> 1, s = f & 1;
  auto own = [&](int cell) { return tile.v[cell >> 6][((cell >> 3) & 7) + 1][(cell & 7) + 1]; };
  const double h = bi.h;
  if (kind == K_COARSER) {
    const double* cl = tile.cl[f];
    auto L = [&](int u, int v) { return d == 1 ? cl[v + 8 * u] : cl[u + 8 * v]; };
    const int h1 = (bi.par >> tan1(d)) & 1, h2 = (bi.par >> tan2(d)) & 1;
    const int c1 = h1 * 4 + (a >> 1), c2 = h2 * 4 + (bb >> 1);
    const double sa = (a & 1) ? 1.0 : -1.0, sb = (bb & 1) ? 1.0 : -1.0;
    const TaylorTerms Tt = d == 1 ? cf_terms(L, c2, c1) : cf_terms(L, c1, c2);
    const double tay = d == 1 ? Tt.at(sb, sa) : Tt.at(sa, sb);
    const double xs = own(face_cell(d, s, 0, a, bb)), xi = own(face_cell(d, s, 1, a, bb));
    return h * (2. / 3. * xs - 1. / 5. * xi + 8. / 15. * tay - xs);
  }
  auto L = [&](int u, int v) { return d == 1 ? own(face_cell(d, s, 0, v, u)) : own(face_cell(d, s, 0, u, v)); };
  const TaylorTerms Tt = d == 1 ? cf_terms(L, bb, a) : cf_terms(L, a, bb);
  const int ch = bi.nbr[4 * f + (a >> 2) + 2 * (bb >> 2)];
  const double hf = 0.5 * h;  // h = h0 2^-level: exact
  const size_t xc = size_t(ch) * BN;
  double close[4], far[4];
#pragma unroll
  for (int q4 = 0; q4 < 4; ++q4) {
    const int fa = 2 * (a & 3) + (q4 & 1), fb = 2 * (bb & 3) + (q4 >> 1);
    close[q4] = x(xc + face_cell(d, 1 - s, 0, fa, fb));
    far[q4] = x(xc + face_cell(d, 1 - s, 1, fa, fb));
  }
  double acc = 0.0;
#pragma unroll
  for (int q4 = 0; q4 < 4; ++q4) {
    const double sa = (q4 & 1) ? 1.0 : -1.0, sb = (q4 >> 1) ? 1.0 : -1.0;
    const double tay = d == 1 ? Tt.at(sb, sa) : Tt.at(sa, sb);
    acc += hf * (close[q4] - (2. / 3. * close[q4] - 1. / 5. * far[q4] + 8. / 15. * tay));
  }
  return acc;
}

template <class T>
__device__ __forceinline__ void load_col(const T* __restrict__ v, int b, const GroupIdx& G, double c[8]) {
  const T* p = v + size_t(b) * BN + G.gy * 8 + G.gx;
#pragma unroll
  for (int z = 0; z < 8; ++z) c[z] = double(ld_stream(p + z * 64));
}

// y = A x on the thread's column of block b (col = x there, already loaded).
// Same-level and boundary faces from the tile and halos; coarse-fine faces:
// each thread computes the flux of one face cell per face, owners add them.
// Ends with a group barrier (tile free for reuse).
template <class X>
__device__ __forceinline__ void spmv_group(const BlockInfo& bi, const X& x, const double col[8], double ms,
                                           int mean_mode, GroupTile& tile, const GroupIdx& G, double y[8]) {
  const int* fn = bi.nbr;
  const int cxy = G.gy * 8 + G.gx;
  int kind[6];
#pragma unroll
  for (int f = 0; f < 6; ++f) kind[f] = bi.kind[f];
  // z halo: same-level neighbour values, zero flux (own value) otherwise
  double zm = col[0], zp = col[7];
  if (kind[4] == K_SAME) zm = x(size_t(fn[16]) * BN + 7 * 64 + cxy);
  if (kind[5] == K_SAME) zp = x(size_t(fn[20]) * BN + cxy);
  // x / y ghost layers and coarser faces' coarse layers: the thread loads
  // face-local cell (gx, gy) of each.  The ghost of a same-level face is the
  // neighbour's face cell; on any other face it is the block's own face cell
  // (zero flux; coarse-fine faces get their flux below).
  bool cf = false;
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    const int d = f >> 1, s = f & 1;
    if (f < 4) {
      const size_t src = kind[f] == K_SAME ? size_t(fn[4 * f]) * BN + face_cell(d, 1 - s, 0, G.gx, G.gy)
                                           : size_t(bi.id) * BN + face_cell(d, s, 0, G.gx, G.gy);
      // face-local (a, b) = (gx, gy): (y, z) on x faces, (x, z) on y faces
      double* ghost = d == 0 ? &tile.v[G.gy][G.gx + 1][s ? BS + 1 : 0] : &tile.v[G.gy][s ? BS + 1 : 0][G.gx + 1];
      *ghost = x(src);
    }
    if (kind[f] == K_COARSER)
      tile.cl[f][G.lane] = x(size_t(fn[4 * f]) * BN + face_cell(d, 1 - s, 0, G.gx, G.gy));
    cf |= kind[f] >= K_COARSER;
  }
#pragma unroll
  for (int z = 0; z < 8; ++z) tile.v[z][G.gy + 1][G.gx + 1] = col[z];
  group_sync(G.g);
  double zf0 = 0.0, zf1 = 0.0;  // z-face fluxes of the own column (cells z = 0, 7)
  if (cf) {                      // uniform per block
#pragma unroll 1
    for (int f = 0; f < 6; ++f) {
      const int kf = bi.kind[f];
      if (kf < K_COARSER) continue;
      const double fl = cf_flux(bi, x, tile, f, kf, G.gx, G.gy);
      if (f < 4)
        tile.flx[f][G.lane] = fl;
      else if (f == 4)
        zf0 = fl;
      else
        zf1 = fl;
    }
    group_sync(G.g);
  }
  const double h = bi.h;
  // x/y neighbours: fixed offsets from the own cell in the padded tile
  constexpr int RS = BS + 2, ZS = RS * RS;
  const double* own_cell = &tile.v[0][G.gy + 1][G.gx + 1];
#pragma unroll
  for (int z = 0; z < 8; ++z) {
    const double xm = own_cell[z * ZS - 1], xp = own_cell[z * ZS + 1];
    const double ym = own_cell[z * ZS - RS], yp = own_cell[z * ZS + RS];
    const double zmv = z > 0 ? col[z - 1] : zm;
    const double zpv = z < 7 ? col[z + 1] : zp;
    y[z] = h * (xm + xp + ym + yp + zmv + zpv - 6.0 * col[z]);
  }
  if (cf) {
    // owners add the fluxes in face order
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      if (kind[f] < K_COARSER) continue;
      const int s = f & 1;
      if (f >= 4) {
        y[s ? 7 : 0] += s ? zf1 : zf0;
      } else if (f < 2) {
        if (G.gx == (s ? 7 : 0))
#pragma unroll
          for (int z = 0; z < 8; ++z) y[z] += tile.flx[f][G.gy + 8 * z];
      } else {
        if (G.gy == (s ? 7 : 0))
#pragma unroll
          for (int z = 0; z < 8; ++z) y[z] += tile.flx[f][G.gx + 8 * z];
      }
    }
  }
  if (bi.mean && G.lane == 0) {
    if (mean_mode == 1) y[0] = ms;
    if (mean_mode == 3) y[0] = h * col[0];
  }
  if (mean_mode == 2) {
    const double h3 = h * h * h;
#pragma unroll
    for (int z = 0; z < 8; ++z) y[z] += ms * h3;
  }
  group_sync(G.g);
}

__device__ __forceinline__ void block_inverse_group(double col[8], FdTile& tile, const GroupIdx& G, double h,
                                                    const double* inv) {
  fd_group(col, tile, G, -1.0 / h, inv);
  group_sync(G.g);
}

// Loops a group over its blocks: visit slots g, g + groups, ... of the
// mesh's visit order (a cost-balanced permutation, see mesh_visit_order).
#define GROUP_BLOCKS(b)                                                              \
  for (int slot_ = blockIdx.x * GROUPS + G.g, b = 0;                                \
       slot_ < M.nb && ((b = M.order ? M.order[slot_] : slot_), true); slot_ += gridDim.x * GROUPS)

// ---------------------------------------------------------------------------
// Standalone kernels
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(NT) k_weighted_sum(DevMesh M, const double* __restrict__ v,
                                                     GridReduce G, double* out, double* tgt) {
  __shared__ double red[64];
  double acc[2] = {0.0, 0.0};
  for (int b = blockIdx.x; b < M.nb; b += gridDim.x) {
    const double h = M.h[b], h3 = h * h * h;
    double s = 0.0;
    for (int c = threadIdx.x; c < BN; c += NT) s += v[size_t(b) * BN + c];
    acc[0] += s * h3;
    if (threadIdx.x == 0) acc[1] += 512.0 * h3;
  }
  if (grid_reduce<2>(acc, G, red) && threadIdx.x == 0) {
    if (out) { out[0] = acc[0]; out[1] = acc[1]; }
    if (tgt) *tgt = acc[0];
  }
}

__global__ void __launch_bounds__(NT) k_spmv(DevMesh M, const double* __restrict__ x,
                                             double* __restrict__ y, const double* mean_sum,
                                             int mean_mode) {
  __shared__ GroupTile tiles[GROUPS];
  const GroupIdx G;
  const double ms = mean_sum ? *mean_sum : 0.0;
  GROUP_BLOCKS(b) {
    double col[8], out[8];
    load_col(x, b, G, col);
    fill_block_info(M, b, tiles[G.g].bi, G.lane);
    group_sync(G.g);
    spmv_group(tiles[G.g].bi, VecAt<double>{x}, col, ms, mean_mode, tiles[G.g], G, out);
    double* yb = y + size_t(b) * BN + G.gy * 8 + G.gx;
#pragma unroll
    for (int z = 0; z < 8; ++z) yb[z * 64] = out[z];
  }
}

__global__ void __launch_bounds__(NT) k_block_inverse(DevMesh M, const double* __restrict__ in,
                                                      double* __restrict__ out) {
  __shared__ FdTile tiles[GROUPS];
  __shared__ double inv_eig[BN];
  const GroupIdx G;
  fd_fill_inverse_eigen(inv_eig, c_lam);
  __syncthreads();
  GROUP_BLOCKS(b) {
    double col[8];
    load_col(in, b, G, col);
    block_inverse_group(col, tiles[G.g], G, M.h[b], inv_eig);
    double* ob = out + size_t(b) * BN + G.gy * 8 + G.gx;
#pragma unroll
    for (int z = 0; z < 8; ++z) ob[z * 64] = col[z];
  }
}

// ---------------------------------------------------------------------------
// BiCGSTAB kernels, templated on the vector storage type T (double for the
// FP64 solver, float for the inner solves of the mixed-precision solver).
// Arithmetic, dot products and scalars are FP64 in both cases.
// ---------------------------------------------------------------------------
template <class T>
struct KArgs {
  DevMesh M;
  const T* b;
  T* r;
  T* rhat;
  T* p;
  T* nu;
  T* t;
  T* z1;
  T* z2;
  T* xs0;
  T* xs1;
  T* xs2;
  KrylovState* st;
  GridReduce g;
  int mean_mode;
  int zero_mean_row;  // b and x0 are zero at the mean row (getVec, modes 1 and 3)
  int ncache;         // persistent solver: block entries staged per group at launch (<= KB_CACHE)
  // two-level preconditioner (persistent solver): A_c^-1 (cnb x cnb, cnb = 0:
  // none), the restricted vectors of zv and zr and the blocks' 512 h^3
  int cnb;           // single case: blocks of A_c; batch: 1 when the cases carry coarse spaces
  const long long* coff;  // batch: offset of each case's A_c^-1 (nb_c x nb_c) in cinv; null: one case
  const float* cinv;
  double* crc_v;
  double* crc_r;
  const double* cw;
  // learned local map (persistent solver, lmap.cuh): W in fragment order
  // (null: none) and the [nb][896] BF16 lab buffer
  const uint4* lw;
  uint16_t* llab;
};

template <class T>
struct Vec2;
template <>
struct Vec2<double> {
  using type = double2;
};
template <>
struct Vec2<float> {
  using type = float2;
};

template <class T>
__device__ __forceinline__ T* xslot(const KArgs<T>& A, int i) {
  return i == 0 ? A.xs0 : (i == 1 ? A.xs1 : A.xs2);
}

template <class T>
__device__ __forceinline__ void store_col(T* v, int b, const GroupIdx& G, const double c[8]) {
  T* p = v + size_t(b) * BN + G.gy * 8 + G.gx;
#pragma unroll
  for (int z = 0; z < 8; ++z) p[z * 64] = T(c[z]);
}

// x0[mean row] = 0 (getVec, PoissonSolverExp.cpp:402-410) and sum(x0 h^3)
template <class T>
__global__ void __launch_bounds__(NT) k_bicg_prepare(KArgs<T> A) {
  __shared__ double red[64];
  pdl_wait();
  pdl_launch_dependents();
  const DevMesh& M = A.M;
  if (A.zero_mean_row && M.mean_block >= 0 && blockIdx.x == 0 && threadIdx.x == 0)
    A.xs0[size_t(M.mean_block) * BN] = T(0);
  double acc[1] = {0.0};
  for (int b = blockIdx.x; b < M.nb; b += gridDim.x) {
    const double h = M.h[b], h3 = h * h * h;
    double s = 0.0;
    for (int c = threadIdx.x; c < BN; c += NT) {
      const size_t i = size_t(b) * BN + c;
      s += (A.zero_mean_row && b == M.mean_block && c == 0) ? 0.0 : double(A.xs0[i]);
    }
    acc[0] += s * h3;
  }
  if (grid_reduce<1>(acc, A.g, red) && threadIdx.x == 0) A.st->mean_sum = acc[0];
}

// Scalars of iteration 0 from rr = (r0, r0) (BiCGSTAB.cu:416-470)
__device__ __forceinline__ void fin_init(KrylovState& S, double rr) {
  const double e = sqrt(rr);
  S.err = S.err_init = S.err_opt = e;
  S.rr = S.rr_hat = rr;
  S.rho = rr;  // (rhat, r) of iteration 0
  S.rho_prev = 1.0;
  S.alpha = 1.0;
  S.omega = 1.0;
  S.beta = (S.rho / (S.rho_prev + S.eps)) * (S.alpha / (S.omega + S.eps));
  S.k = 0;
  S.restarts = 0;
  S.cur = 0;
  S.best = 0;
  S.nxt = 1;
  S.restart_pending = 0;
  S.converged = 0;
  S.done = 0;
  S.status = SOLVE_RUNNING;
  S.last_improve_k = 0;
  S.stall_ref = e;
  if (!(e == e)) {
    S.done = 1;
    S.status = SOLVE_NAN;
  } else if (e <= S.tol_abs) {  // nothing to do (also covers b = A x0)
    S.done = 1;
    S.converged = 1;
    S.status = SOLVE_CONVERGED;
  }
}

// r = b - A x0, rhat = r, p = nu = 0; err_init = ||r||
template <class T>
__global__ void __launch_bounds__(NT) k_bicg_init(KArgs<T> A) {
  __shared__ GroupTile tiles[GROUPS];
  __shared__ double red[64];
  const GroupIdx G;
  pdl_wait();
  pdl_launch_dependents();
  const DevMesh& M = A.M;
  const double ms = A.st->mean_sum;
  double acc[1] = {0.0};
  GROUP_BLOCKS(b) {
    double col[8], y[8], bc[8];
    load_col(A.xs0, b, G, col);
    fill_block_info(M, b, tiles[G.g].bi, G.lane);
    group_sync(G.g);
    spmv_group(tiles[G.g].bi, VecAt<T>{A.xs0}, col, ms, A.mean_mode, tiles[G.g], G, y);
    load_col(A.b, b, G, bc);
    if (A.zero_mean_row && b == M.mean_block && G.lane == 0) bc[0] = 0.0;
    double r[8], zero[8];
#pragma unroll
    for (int z = 0; z < 8; ++z) {
      r[z] = bc[z] - y[z];
      zero[z] = 0.0;
      acc[0] += r[z] * r[z];
    }
    store_col(A.r, b, G, r);
    store_col(A.rhat, b, G, r);
    store_col(A.p, b, G, zero);
    store_col(A.nu, b, G, zero);
  }
  if (grid_reduce<1>(acc, A.g, red) && threadIdx.x == 0) fin_init(*A.st, acc[0]);
}

// ---------------------------------------------------------------------------
// The five phases of one BiCGSTAB iteration (BiCGSTAB.cu:416-628).  Each body
// is one pass of the CTA over its blocks (or cells) and returns the CTA's
// partial sums; each finalizer turns the grid totals into the scalars of the
// next phase.  The per-phase kernels run one body per launch with a last-CTA
// finalizer (the flexible solver of the learned preconditioner, whose network
// runs between phases); the finalizers are shared with the three-phase
// persistent solver below.
// ---------------------------------------------------------------------------
// A: p = r + beta (p - omega nu) (or p = r, rhat = r after a restart);
//    z1 = M^-1 p; sum(z1 h^3)
template <class T>
__device__ __forceinline__ double phase_a(const KArgs<T>& A, const GroupIdx& G, FdTile& tile, const double* inv,
                                          double beta, double omega, bool restart) {
  const DevMesh& M = A.M;
  double acc = 0.0;
  GROUP_BLOCKS(b) {
    double r[8], p[8];
    load_col(A.r, b, G, r);
    if (restart) {
#pragma unroll
      for (int z = 0; z < 8; ++z) p[z] = r[z];
      store_col(A.rhat, b, G, r);
    } else {
      double pp[8], nu[8];
      load_col(A.p, b, G, pp);
      load_col(A.nu, b, G, nu);
#pragma unroll
      for (int z = 0; z < 8; ++z) p[z] = double(T(r[z] + beta * (pp[z] - omega * nu[z])));
    }
    store_col(A.p, b, G, p);
    const double h = M.h[b];
    block_inverse_group(p, tile, G, h, inv);
    double s = 0.0;
#pragma unroll
    for (int z = 0; z < 8; ++z) {
      p[z] = double(T(p[z]));
      s += p[z];
    }
    store_col(A.z1, b, G, p);
    acc += s * h * h * h;
  }
  return acc;
}

__device__ __forceinline__ void fin_a(KrylovState& W, double sum, bool restart) {
  W.mean_sum = sum;
  if (restart) {
    W.rho = W.rr;
    W.rr_hat = W.rr;
    W.restart_pending = 0;
  }
}

// B: nu = A z1; (rhat, nu)
template <class T>
__device__ __forceinline__ double phase_b(const KArgs<T>& A, const GroupIdx& G, GroupTile& tile, double ms) {
  const DevMesh& M = A.M;
  double acc = 0.0;
  GROUP_BLOCKS(b) {
    double col[8], y[8], rh[8];
    load_col(A.z1, b, G, col);
    fill_block_info(M, b, tile.bi, G.lane);
    group_sync(G.g);
    spmv_group(tile.bi, VecAt<T>{A.z1}, col, ms, A.mean_mode, tile, G, y);
    load_col(A.rhat, b, G, rh);
#pragma unroll
    for (int z = 0; z < 8; ++z) {
      y[z] = double(T(y[z]));
      acc += rh[z] * y[z];
    }
    store_col(A.nu, b, G, y);
  }
  return acc;
}

__device__ __forceinline__ void fin_b(KrylovState& W, double rhat_nu) { W.alpha = W.rho / (rhat_nu + W.eps); }

// C: s = r - alpha nu (in place in r); z2 = M^-1 s; sum(z2 h^3)
template <class T>
__device__ __forceinline__ double phase_c(const KArgs<T>& A, const GroupIdx& G, FdTile& tile, const double* inv,
                                          double alpha) {
  const DevMesh& M = A.M;
  double acc = 0.0;
  GROUP_BLOCKS(b) {
    double r[8], nu[8];
    load_col(A.r, b, G, r);
    load_col(A.nu, b, G, nu);
#pragma unroll
    for (int z = 0; z < 8; ++z) r[z] = double(T(r[z] - alpha * nu[z]));
    store_col(A.r, b, G, r);
    const double h = M.h[b];
    block_inverse_group(r, tile, G, h, inv);
    double s = 0.0;
#pragma unroll
    for (int z = 0; z < 8; ++z) {
      r[z] = double(T(r[z]));
      s += r[z];
    }
    store_col(A.z2, b, G, r);
    acc += s * h * h * h;
  }
  return acc;
}

__device__ __forceinline__ void fin_c(KrylovState& W, double sum) { W.mean_sum = sum; }

// D: t = A z2; (t, s), (t, t)
template <class T>
__device__ __forceinline__ void phase_d(const KArgs<T>& A, const GroupIdx& G, GroupTile& tile, double ms,
                                        double (&acc)[2]) {
  const DevMesh& M = A.M;
  GROUP_BLOCKS(b) {
    double col[8], y[8], sv[8];
    load_col(A.z2, b, G, col);
    fill_block_info(M, b, tile.bi, G.lane);
    group_sync(G.g);
    spmv_group(tile.bi, VecAt<T>{A.z2}, col, ms, A.mean_mode, tile, G, y);
    load_col(A.r, b, G, sv);
#pragma unroll
    for (int z = 0; z < 8; ++z) {
      y[z] = double(T(y[z]));
      acc[0] += y[z] * sv[z];
      acc[1] += y[z] * y[z];
    }
    store_col(A.t, b, G, y);
  }
}

__device__ __forceinline__ void fin_d(KrylovState& W, const double (&acc)[2]) {
  W.omega = acc[0] / (acc[1] + W.eps);
}

// E: x_new = x + alpha z1 + omega z2; r = s - omega t; (rhat, r), (r, r).
// Two cells per thread per pass with 2-wide vector accesses (nb*512 is even
// and every vector starts on a 16-byte boundary).
template <class T>
__device__ __forceinline__ void phase_e(const KArgs<T>& A, const T* xc, T* xn, double alpha, double omega,
                                        double (&acc)[2]) {
  using V2 = typename Vec2<T>::type;
  const size_t n2 = size_t(A.M.nb) * (BN / 2);
  const V2* xc2 = reinterpret_cast<const V2*>(xc);
  const V2* z12 = reinterpret_cast<const V2*>(A.z1);
  const V2* z22 = reinterpret_cast<const V2*>(A.z2);
  const V2* t2 = reinterpret_cast<const V2*>(A.t);
  const V2* rh2 = reinterpret_cast<const V2*>(A.rhat);
  V2* r2 = reinterpret_cast<V2*>(A.r);
  V2* xn2 = reinterpret_cast<V2*>(xn);
  for (size_t i = size_t(blockIdx.x) * NT + threadIdx.x; i < n2; i += size_t(gridDim.x) * NT) {
    const V2 x = ld_stream(xc2 + i), z1 = ld_stream(z12 + i), z2 = ld_stream(z22 + i), t = ld_stream(t2 + i),
             r = ld_stream(r2 + i), rh = ld_stream(rh2 + i);
    V2 xo, ro;
    xo.x = T((double(x.x) + alpha * double(z1.x)) + omega * double(z2.x));
    xo.y = T((double(x.y) + alpha * double(z1.y)) + omega * double(z2.y));
    ro.x = T(double(r.x) - omega * double(t.x));
    ro.y = T(double(r.y) - omega * double(t.y));
    xn2[i] = xo;
    r2[i] = ro;
    acc[0] += double(rh.x) * double(ro.x);
    acc[0] += double(rh.y) * double(ro.y);
    acc[1] += double(ro.x) * double(ro.x);
    acc[1] += double(ro.y) * double(ro.y);
  }
}

// convergence, best iterate, stall and restart decisions, beta for the next A
__device__ __forceinline__ void fin_e(KrylovState& W, const double (&acc)[2]) {
  const double err = sqrt(acc[1]);
  W.err = err;
  W.rr = acc[1];
  W.k += 1;
  W.cur = W.nxt;
  if (!(err == err)) {
    W.done = 1;
    W.status = SOLVE_NAN;
  } else if (err < W.err_opt) {
    W.err_opt = err;
    W.best = W.cur;
    if (err <= W.tol_abs || err / W.err_init <= W.tol_rel) {
      W.done = 1;
      W.converged = 1;
      W.status = SOLVE_CONVERGED;
    }
  }
  // next free slot: neither the current nor the best iterate
  int nx = 0;
  while (nx == W.cur || nx == W.best) ++nx;
  W.nxt = nx;
  if (!W.done && W.k >= W.max_iter) {
    W.done = 1;
    W.status = SOLVE_MAXITER;
  }
  if (err < 0.9 * W.stall_ref) {
    W.stall_ref = err;
    W.last_improve_k = W.k;
  } else if (!W.done && W.stall_window > 0 && W.k - W.last_improve_k >= W.stall_window) {
    W.done = 1;
    W.status = SOLVE_STALL;
  }
  W.rho_prev = W.rho;
  W.rho = acc[0];
  if (!W.done) {
    const bool breakdown = W.rho * W.rho < 1e-16 * W.rr * W.rr_hat;
    if (breakdown && W.max_restarts > 0) {
      W.restarts += 1;
      if (W.restarts >= W.max_restarts) {
        W.done = 1;
        W.status = SOLVE_RESTARTS;
      } else {
        W.restart_pending = 1;
      }
    }
    W.beta = (W.rho / (W.rho_prev + W.eps)) * (W.alpha / (W.omega + W.eps));
  }
}

// ---- per-phase kernels (one launch per phase, last-CTA finalizer) ----------
template <class T>
__global__ void __launch_bounds__(NT) k_bicg_a(KArgs<T> A) {
  __shared__ FdTile tiles[GROUPS];
  __shared__ double red[64];
  __shared__ double inv_eig[BN];
  const GroupIdx G;
  fd_fill_inverse_eigen(inv_eig, c_lam);  // independent of the previous kernel: overlaps its tail
  __syncthreads();
  pdl_wait();
  pdl_launch_dependents();
  const KrylovState& S = *A.st;
  if (S.done) return;
  const bool restart = S.restart_pending != 0;
  double acc[1] = {phase_a<T>(A, G, tiles[G.g], inv_eig, S.beta, S.omega, restart)};
  if (grid_reduce<1>(acc, A.g, red) && threadIdx.x == 0) fin_a(*A.st, acc[0], restart);
}

template <class T>
__global__ void __launch_bounds__(NT) k_bicg_b(KArgs<T> A) {
  __shared__ GroupTile tiles[GROUPS];
  __shared__ double red[64];
  pdl_wait();
  pdl_launch_dependents();
  const KrylovState& S = *A.st;
  if (S.done) return;
  const GroupIdx G;
  double acc[1] = {phase_b<T>(A, G, tiles[G.g], S.mean_sum)};
  if (grid_reduce<1>(acc, A.g, red) && threadIdx.x == 0) fin_b(*A.st, acc[0]);
}

template <class T>
__global__ void __launch_bounds__(NT) k_bicg_c(KArgs<T> A) {
  __shared__ FdTile tiles[GROUPS];
  __shared__ double red[64];
  __shared__ double inv_eig[BN];
  const GroupIdx G;
  fd_fill_inverse_eigen(inv_eig, c_lam);  // independent of the previous kernel: overlaps its tail
  __syncthreads();
  pdl_wait();
  pdl_launch_dependents();
  const KrylovState& S = *A.st;
  if (S.done) return;
  double acc[1] = {phase_c<T>(A, G, tiles[G.g], inv_eig, S.alpha)};
  if (grid_reduce<1>(acc, A.g, red) && threadIdx.x == 0) fin_c(*A.st, acc[0]);
}

template <class T>
__global__ void __launch_bounds__(NT) k_bicg_d(KArgs<T> A) {
  __shared__ GroupTile tiles[GROUPS];
  __shared__ double red[64];
  pdl_wait();
  pdl_launch_dependents();
  const KrylovState& S = *A.st;
  if (S.done) return;
  const GroupIdx G;
  double acc[2] = {0.0, 0.0};
  phase_d<T>(A, G, tiles[G.g], S.mean_sum, acc);
  if (grid_reduce<2>(acc, A.g, red) && threadIdx.x == 0) fin_d(*A.st, acc);
}

template <class T>
__global__ void __launch_bounds__(NT) k_bicg_e(KArgs<T> A) {
  __shared__ double red[64];
  pdl_wait();
  pdl_launch_dependents();
  const KrylovState& S = *A.st;
  if (S.done) return;
  double acc[2] = {0.0, 0.0};
  phase_e<T>(A, xslot(A, S.cur), xslot(A, S.nxt), S.alpha, S.omega, acc);
  if (grid_reduce<2>(acc, A.g, red) && threadIdx.x == 0) fin_e(*A.st, acc);
}

// ---- persistent solver: three grid barriers per iteration -----------------
// The same iteration as the five phases above, reorganised by the linearity
// of the block preconditioner M^-1 so that the two halo exchanges coincide
// with reductions.  With zr = M^-1 r, zv = M^-1 nu and q = z1 - omega zv:
//   z1 = M^-1 p  = zr + beta q     (p = r + beta (p - omega nu))
//   z2 = M^-1 s  = zr - alpha zv   (s = r - alpha nu)
// so the operator's inputs z1 and z2 are formed at the point of use from
// vectors that the previous phase finished before its barrier.  Per
// iteration:
//   P1: nu = A (zr + beta q); zv = M^-1 nu; (rhat, nu), sum(zv h^3)
//   P2: t = A (zr - alpha zv); s = r - alpha nu; (t, s), (t, t)
//   P3: x += alpha z1 + omega z2; r = s - omega t; q = z1 - omega zv;
//       zr = M^-1 r; (rhat, r), (r, r), sum(zr h^3), sum(q h^3)
// p and s are never stored.  Buffers: zr in z1, zv in z2, q in p.  Every
// vector a phase reads from other blocks (zr, q in P1; zr, zv in P2) is
// written only in another phase, so no phase needs a second buffer.  The
// scalars, the restart rule and the stopping tests are fin_a..fin_e's.
// ---------------------------------------------------------------------------
template <class T>
struct Comb2At {  // a + c b
  const T* a;
  const T* b;
  double c;
  __device__ __forceinline__ double operator()(size_t i) const {
    return double(ld_stream(a + i)) + c * double(ld_stream(b + i));
  }
};

// Blocks of group g in the persistent solver: visit slots g + k G_total of
// the mesh's visit order (G_total groups in the grid), the same in every
// phase.  Their table entries for k < ncache (at most KB_CACHE) are staged in
// shared memory at launch; later ones are staged in the group's tile on the
// way.
constexpr int KB_CACHE = 4;

// Block groups per CTA of the persistent solver, two CTAs per SM.  (One
// 512-thread CTA per SM halves the CTAs in every grid barrier but measured
// 6% slower per iteration on the sphere mesh.)
constexpr int PGROUPS = PERSISTENT_GROUPS_PER_CTA;
constexpr int PNT = PGROUPS * GROUP;

__device__ __forceinline__ const BlockInfo& persistent_block(const DevMesh& M, const BlockInfo* cache, int ncache,
                                                             GroupTile& tile, int k, int slot, const GroupIdx& G) {
  if (k < ncache) return cache[G.g * KB_CACHE + k];
  group_sync(G.g);  // the group is done with the previous staged entry
  fill_block_info(M, M.order ? M.order[slot] : slot, tile.bi, G.lane);
  group_sync(G.g);
  return tile.bi;
}

#define PERSISTENT_BLOCKS(bi)                                                                   \
  for (int k_ = 0, slot_ = blockIdx.x * PGROUPS + G.g; slot_ < M.nb; ++k_, slot_ += gridDim.x * PGROUPS) \
    if (const BlockInfo& bi = persistent_block(M, cache, A.ncache, tile, k_, slot_, G); true)

// PREP: x0 = 0 on the (case's) mean row (modes 1 and 3); sum(x0 h^3)
template <class T>
__device__ __forceinline__ double prep_block(const KArgs<T>& A, const GroupIdx& G, const BlockInfo& bi) {
  const int b = bi.id;
  double c[8];
  load_col(A.xs0, b, G, c);
  if (A.zero_mean_row && bi.mean && G.lane == 0) {
    A.xs0[size_t(b) * BN] = T(0);
    c[0] = 0.0;
  }
  double s = 0.0;
#pragma unroll
  for (int z = 0; z < 8; ++z) s += c[z];
  return s * bi.h * bi.h * bi.h;
}

// INIT: r = b - A x0 (b = 0 on the mean row for modes 1 and 3), rhat = r,
// p = 0; (r, r)
template <class T>
__device__ __forceinline__ double init_block(const KArgs<T>& A, const GroupIdx& G, GroupTile& tile,
                                             const BlockInfo& bi, double ms) {
  const int b = bi.id;
  double col[8], y[8], bc[8];
  load_col(A.xs0, b, G, col);
  spmv_group(bi, VecAt<T>{A.xs0}, col, ms, A.mean_mode, tile, G, y);
  load_col(A.b, b, G, bc);
  if (A.zero_mean_row && bi.mean && G.lane == 0) bc[0] = 0.0;
  double r[8], zero[8], acc = 0.0;
#pragma unroll
  for (int z = 0; z < 8; ++z) {
    r[z] = bc[z] - y[z];  // stored as T; (r, r) from the unrounded values, as k_bicg_init
    zero[z] = 0.0;
    acc += r[z] * r[z];
  }
  store_col(A.r, b, G, r);
  store_col(A.rhat, b, G, r);
  store_col(A.p, b, G, zero);
  return acc;
}

// Phase bodies for one block (bi) of a group; the persistent solvers loop
// them over the group's blocks.
// Sum of v over the 64 threads of a group, in a fixed order; every thread of
// the group gets the totals.  gsm: 2 * NR doubles of the group.
template <int NR>
__device__ __forceinline__ void group_reduce(double (&v)[NR], double* gsm, const GroupIdx& G) {
#pragma unroll
  for (int r = 0; r < NR; ++r)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[r] += __shfl_xor_sync(0xffffffffu, v[r], o);
  if ((G.lane & 31) == 0)
#pragma unroll
    for (int r = 0; r < NR; ++r) gsm[(G.lane >> 5) * NR + r] = v[r];
  group_sync(G.g);
#pragma unroll
  for (int r = 0; r < NR; ++r) v[r] = gsm[r] + gsm[NR + r];
  group_sync(G.g);
}

// Two-level preconditioner in the persistent solver: the restriction of a
// vector is its block sums (lane 0 of the group writes rc[b]); the coarse
// correction of block b is yc = row b of A_c^-1 times rc, added to every cell
// of the block (the group reads its row, 8 * nb bytes, coalesced).  Returns
// yc 512 h^3, the correction's part of sum(v h^3), in lane 0 (0 elsewhere).
__device__ __forceinline__ void coarse_restrict(const double c[8], double* rc, int b, double* gsm, const GroupIdx& G) {
  double s[1] = {((c[0] + c[1]) + (c[2] + c[3])) + ((c[4] + c[5]) + (c[6] + c[7]))};
  group_reduce<1>(s, gsm, G);
  if (G.lane == 0) rc[b] = s[0];
}

// row: block b's row of A_c^-1 (n entries), rc: the restriction of the
// blocks that row spans.
template <class T>
__device__ __forceinline__ double coarse_block_row(const KArgs<T>& A, const GroupIdx& G, int b, const float* row,
                                                   const double* rc, int n, T* v, double* gsm) {
  double s[1] = {0.0};
  for (int j = G.lane; j < n; j += GROUP) s[0] += double(row[j]) * __ldcg(rc + j);
  group_reduce<1>(s, gsm, G);
  const double yc = s[0];
  double c[8];
  load_col(v, b, G, c);
#pragma unroll
  for (int z = 0; z < 8; ++z) c[z] = double(T(c[z] + yc));
  store_col(v, b, G, c);
  return G.lane == 0 ? yc * A.cw[b] : 0.0;  // summed over the CTA's threads by the grid reduction
}

template <class T>
__device__ __forceinline__ double coarse_block(const KArgs<T>& A, const GroupIdx& G, int b, const double* rc, T* v,
                                               double* gsm) {
  return coarse_block_row(A, G, b, A.cinv + size_t(b) * A.cnb, rc, A.cnb, v, gsm);
}

// The same in a batch: block b of case c (blocks cf .. cf + n - 1), whose
// A_c^-1 starts at coff[c] of the packed, block-diagonal cinv.
template <class T>
__device__ __forceinline__ double coarse_block_case(const KArgs<T>& A, const GroupIdx& G, int b, int cf, int n,
                                                    long long off, const double* rc, T* v, double* gsm) {
  return coarse_block_row(A, G, b, A.cinv + off + size_t(b - cf) * n, rc + cf, n, v, gsm);
}

// P0 (once): zr = M^-1 r for the initial residual; sum(zr h^3)
template <class T>
__device__ __forceinline__ double p0_block(const KArgs<T>& A, const GroupIdx& G, GroupTile& tile,
                                           const BlockInfo& bi, const double* inv) {
  FdTile& ftile = reinterpret_cast<FdTile&>(tile);
  const int b = bi.id;
  const double h = bi.h;
  double c[8];
  load_col(A.r, b, G, c);
  if (A.cnb) coarse_restrict(c, A.crc_r, b, ftile.v[0][0] + 0, G);
  block_inverse_group(c, ftile, G, h, inv);
  double s = 0.0;
#pragma unroll
  for (int z = 0; z < 8; ++z) {
    c[z] = double(T(c[z]));
    s += c[z];
  }
  store_col(A.z1, b, G, c);
  return s * h * h * h;
}

// P1: z1 = zr + beta q (beta = 0 after a restart, which also sets rhat = r);
//     nu = A z1; zv = M^-1 nu; (rhat, nu), sum(zv h^3)
template <class T>
__device__ __forceinline__ void p1_block(const KArgs<T>& A, const GroupIdx& G, GroupTile& tile, const BlockInfo& bi,
                                         const double* inv, double beta, double ms, bool restart,
                                         double (&acc)[2]) {
  FdTile& ftile = reinterpret_cast<FdTile&>(tile);
  const Comb2At<T> z1{A.z1, A.p, beta};
  const int b = bi.id;
  const double h = bi.h;
  double col[8], y[8], rh[8];
  {
    const size_t o = size_t(b) * BN + G.gy * 8 + G.gx;
#pragma unroll
    for (int z = 0; z < 8; ++z) col[z] = z1(o + z * 64);  // the accessor the ghosts use: the same values
  }
  spmv_group(bi, z1, col, ms, A.mean_mode, tile, G, y);
  if (restart) {
    load_col(A.r, b, G, rh);
    store_col(A.rhat, b, G, rh);
  } else {
    load_col(A.rhat, b, G, rh);
  }
#pragma unroll
  for (int z = 0; z < 8; ++z) {
    y[z] = double(T(y[z]));
    acc[0] += rh[z] * y[z];
  }
  store_col(A.nu, b, G, y);
  if (A.cnb) coarse_restrict(y, A.crc_v, b, ftile.v[0][0] + 0, G);
  block_inverse_group(y, ftile, G, h, inv);
  double s = 0.0;
#pragma unroll
  for (int z = 0; z < 8; ++z) {
    y[z] = double(T(y[z]));
    s += y[z];
  }
  store_col(A.z2, b, G, y);
  acc[1] += s * h * h * h;
}

// P2: t = A (zr - alpha zv); s = r - alpha nu; (t, s), (t, t)
template <class T>
__device__ __forceinline__ void p2_block(const KArgs<T>& A, const GroupIdx& G, GroupTile& tile, const BlockInfo& bi,
                                         double alpha, double ms, double (&acc)[2]) {
  const Comb2At<T> z2{A.z1, A.z2, -alpha};
  const int b = bi.id;
  double col[8], y[8];
  {
    const size_t o = size_t(b) * BN + G.gy * 8 + G.gx;
#pragma unroll
    for (int z = 0; z < 8; ++z) col[z] = z2(o + z * 64);  // the accessor the ghosts use: the same values
  }
  spmv_group(bi, z2, col, ms, A.mean_mode, tile, G, y);
  double r[8], nu[8];
  load_col(A.r, b, G, r);
  load_col(A.nu, b, G, nu);
#pragma unroll
  for (int z = 0; z < 8; ++z) {
    y[z] = double(T(y[z]));
    const double sv = double(T(r[z] - alpha * nu[z]));
    acc[0] += y[z] * sv;
    acc[1] += y[z] * y[z];
  }
  store_col(A.t, b, G, y);
}

// P3: x_new = x + alpha z1 + omega z2; r = s - omega t; q = z1 - omega zv;
//     zr = M^-1 r; (rhat, r), (r, r), sum(zr h^3), sum(q h^3)
template <class T>
__device__ __forceinline__ void p3_block(const KArgs<T>& A, const GroupIdx& G, GroupTile& tile, const BlockInfo& bi,
                                         const double* inv, const T* xc, T* xn, double alpha, double beta,
                                         double omega, double (&acc)[4]) {
  FdTile& ftile = reinterpret_cast<FdTile&>(tile);
  const int b = bi.id;
  const double h = bi.h, h3 = h * h * h;
  double rn[8], sq = 0.0;
  {
    double r[8], nu[8], t[8], rh[8];
    load_col(A.r, b, G, r);
    load_col(A.nu, b, G, nu);
    load_col(A.t, b, G, t);
    load_col(A.rhat, b, G, rh);
#pragma unroll
    for (int z = 0; z < 8; ++z) {
      const double sv = double(T(r[z] - alpha * nu[z]));
      rn[z] = double(T(sv - omega * t[z]));
      acc[0] += rh[z] * rn[z];
      acc[1] += rn[z] * rn[z];
    }
    store_col(A.r, b, G, rn);
  }
  {
    double zr[8], q[8], zv[8], x[8];
    load_col(A.z1, b, G, zr);
    load_col(A.p, b, G, q);
    load_col(A.z2, b, G, zv);
    load_col(xc, b, G, x);
#pragma unroll
    for (int z = 0; z < 8; ++z) {
      const double z1 = zr[z] + beta * q[z], z2 = zr[z] - alpha * zv[z];
      x[z] = double(T((x[z] + alpha * z1) + omega * z2));
      q[z] = double(T(z1 - omega * zv[z]));
      sq += q[z];
    }
    store_col(xn, b, G, x);
    store_col(A.p, b, G, q);
  }
  if (A.cnb) coarse_restrict(rn, A.crc_r, b, ftile.v[0][0] + 0, G);
  block_inverse_group(rn, ftile, G, h, inv);
  double s = 0.0;
#pragma unroll
  for (int z = 0; z < 8; ++z) {
    rn[z] = double(T(rn[z]));
    s += rn[z];
  }
  store_col(A.z1, b, G, rn);
  acc[2] += s * h3;
  acc[3] += sq * h3;
}

// Every CTA keeps a copy of the Krylov state in shared memory and applies
// the finalizers to the grid totals of each phase, so all copies stay equal;
// CTA 0 writes the state back at the end.  Data written by other CTAs is read
// after the grid barrier's acquire.
// Dynamic shared memory: the inverse eigenvalues (BN doubles), PGROUPS *
// KB_CACHE block entries, PGROUPS tiles.  The learned map's phases use the
// tiles' space as scratch (the lab of the gather, the staged labs of a GEMM
// tile), which is longer than the tiles: kLearnedSmem.
constexpr size_t kSmemCache = BN * sizeof(double);
constexpr size_t kSmemTiles = kSmemCache + PGROUPS * KB_CACHE * sizeof(BlockInfo);
constexpr size_t kPersistentSmem = kSmemTiles + PGROUPS * sizeof(GroupTile);
constexpr size_t kLearnedSmem = std::max(kPersistentSmem, kSmemTiles + LMAP_TILE_BYTES);
static_assert(kSmemTiles % 16 == 0, "tiles and staged labs start 16-byte aligned");
static_assert(LMAP_GATHER * sizeof(LabMeta) <= PGROUPS * sizeof(GroupTile), "the gather's table entries fit in the tiles");
static_assert(PNT == 256, "the learned map's phases run on 8 warps (4 groups of 64 threads)");

template <class T>
__global__ void __launch_bounds__(PNT, 8 / PGROUPS) k_bicg_persistent(KArgs<T> A, GridSync Gs) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* inv_eig = reinterpret_cast<double*>(smem_raw);
  BlockInfo* cache = reinterpret_cast<BlockInfo*>(smem_raw + kSmemCache);
  GroupTile* tiles = reinterpret_cast<GroupTile*>(smem_raw + kSmemTiles);
  __shared__ double red[64];
  __shared__ KrylovState S;
  __shared__ double ms_zr;  // sum(zr h^3) of the current zr
  __shared__ unsigned int epoch;
  __shared__ double gred[2 * PGROUPS];  // per-group reduction scratch of the coarse phases
  const GroupIdx G;
  const DevMesh& M = A.M;
  GroupTile& tile = tiles[G.g];
  fd_fill_inverse_eigen(inv_eig, c_lam);
  for (int i = threadIdx.x; i < PGROUPS * KB_CACHE * 32; i += PNT) {  // 32 lanes fill one entry
    const int e = i >> 5, g = e / KB_CACHE, k = e % KB_CACHE;
    const int slot = blockIdx.x * PGROUPS + g + k * gridDim.x * PGROUPS;
    if (k < A.ncache && slot < M.nb) fill_block_info(M, M.order ? M.order[slot] : slot, cache[e], i & 31);
  }
  if (threadIdx.x == 0) {
    S = *A.st;
    epoch = 0u;
  }
  __syncthreads();
  bool ok = true;
  // PREP and INIT: x0's mean row and sum(x0 h^3); r = b - A x0, rhat = r,
  // p = 0 and the scalars of iteration 0
  {
    double a[1] = {0.0};
    PERSISTENT_BLOCKS(bi) a[0] += prep_block<T>(A, G, bi);
    ok = grid_allreduce<1>(a, Gs, epoch, red);
    if (threadIdx.x == 0) S.mean_sum = a[0];
    __syncthreads();
  }
  if (ok) {
    double a[1] = {0.0};
    PERSISTENT_BLOCKS(bi) a[0] += init_block<T>(A, G, tile, bi, S.mean_sum);
    ok = grid_allreduce<1>(a, Gs, epoch, red);
    if (threadIdx.x == 0) fin_init(S, a[0]);
    __syncthreads();
  }
  // the mean-constraint row (modes 1 and 3 replace cell 0 of the mean block)
  const int mean_blk = (A.mean_mode == 1 || A.mean_mode == 3) ? M.mean_block : -1;
  // The parts of the preconditioner that need the whole vector v (nu or r)
  // in place, added to its block part z (zv or zr):
  //   * the coarse correction of the two-level preconditioner, from v's
  //     restriction rc: every group adds it on its blocks;
  //   * the learned local map (lmap.cuh): the CTAs gather v's labs, then,
  //     after a grid barrier, the GEMM adds W lab / h.
  // The grid sum of the added sum(z h^3) comes back in every CTA.  One grid
  // barrier, two with the learned map.
  auto extra_phases = [&](const double* rc, const T* v, T* z, double& added) -> bool {
    double a[1] = {0.0};
    if (A.cnb) PERSISTENT_BLOCKS(bi) a[0] += coarse_block<T>(A, G, bi.id, rc, z, &gred[2 * G.g]);
    if (A.lw) {
      __syncthreads();  // the groups are done with their tiles
      lmap_gather<T>(M, v, A.llab, reinterpret_cast<LabMeta*>(smem_raw + kSmemTiles), mean_blk);
    }
    if (!grid_allreduce<1>(a, Gs, epoch, red)) return false;
    added = a[0];
    if (A.lw) {
      double l[1] = {lmap_gemm<T>(M, A.lw, A.llab, z, reinterpret_cast<uint16_t*>(smem_raw + kSmemTiles))};
      if (!grid_allreduce<1>(l, Gs, epoch, red)) return false;
      added += l[0];
    }
    return true;
  };
  const bool extra = A.cnb || A.lw;
  if (ok && !S.done) {
    double a[1] = {0.0};
    PERSISTENT_BLOCKS(bi) a[0] += p0_block<T>(A, G, tile, bi, inv_eig);
    ok = grid_allreduce<1>(a, Gs, epoch, red);
    double cz = 0.0;
    if (ok && extra) ok = extra_phases(A.crc_r, A.r, A.z1, cz);
    // q = 0 at the start (init_block), so z1 = zr
    if (threadIdx.x == 0) ms_zr = S.mean_sum = a[0] + cz;
    __syncthreads();
  }
  while (ok && !S.done) {
    const bool restart = S.restart_pending != 0;
    const double beta = restart ? 0.0 : S.beta;
    double a[2] = {0.0, 0.0};
    PERSISTENT_BLOCKS(bi) p1_block<T>(A, G, tile, bi, inv_eig, beta, S.mean_sum, restart, a);
    if (!(ok = grid_allreduce<2>(a, Gs, epoch, red))) break;
    if (threadIdx.x == 0) {
      fin_a(S, S.mean_sum, restart);
      fin_b(S, a[0]);
      S.beta = beta;                        // the beta that formed z1, for P3
      S.mean_sum = ms_zr - S.alpha * a[1];  // sum(z2 h^3)
    }
    __syncthreads();
    if (extra) {  // zv += the rest of M^-1 nu; sum(z2 h^3) with it
      double cv = 0.0;
      if (!(ok = extra_phases(A.crc_v, A.nu, A.z2, cv))) break;
      if (threadIdx.x == 0) S.mean_sum = ms_zr - S.alpha * (a[1] + cv);
      __syncthreads();
    }
    double d[2] = {0.0, 0.0};
    PERSISTENT_BLOCKS(bi) p2_block<T>(A, G, tile, bi, S.alpha, S.mean_sum, d);
    if (!(ok = grid_allreduce<2>(d, Gs, epoch, red))) break;
    if (threadIdx.x == 0) fin_d(S, d);
    __syncthreads();
    double e[4] = {0.0, 0.0, 0.0, 0.0};
    PERSISTENT_BLOCKS(bi)
        p3_block<T>(A, G, tile, bi, inv_eig, xslot(A, S.cur), xslot(A, S.nxt), S.alpha, S.beta, S.omega, e);
    if (!(ok = grid_allreduce<4>(e, Gs, epoch, red))) break;
    if (threadIdx.x == 0) {
      const double re[2] = {e[0], e[1]};
      fin_e(S, re);
      ms_zr = e[2];
      // sum(z1 h^3) of the next P1
      S.mean_sum = S.restart_pending ? e[2] : e[2] + S.beta * e[3];
    }
    __syncthreads();
    if (extra && !S.done) {  // zr += the rest of M^-1 r; the sums with it
      double cr = 0.0;
      if (!(ok = extra_phases(A.crc_r, A.r, A.z1, cr))) break;
      if (threadIdx.x == 0) {
        ms_zr = e[2] + cr;
        S.mean_sum = S.restart_pending ? ms_zr : ms_zr + S.beta * e[3];
      }
      __syncthreads();
    }
  }
  // every CTA holds the final state: its groups move the best iterate into
  // x (slot 0) block by block
  if (ok && S.best != 0) {
    const T* src = xslot(A, S.best);
    PERSISTENT_BLOCKS(bi) {
      double v[8];
      load_col(src, bi.id, G, v);
      store_col(A.xs0, bi.id, G, v);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (!ok) {
      S.done = 1;
      S.status = SOLVE_BARRIER_TIMEOUT;
    }
    *A.st = S;
  }
}

// ---- batched persistent solver: independent cases in one launch ----------
// The mesh holds several independent cases (no face joins two cases).  Every
// block group works for one case and holds that case's Krylov state in
// shared memory; the groups of a case sum only their own partials, in group
// order, so each case runs its own BiCGSTAB (scalars, restarts, stopping
// test, best iterate) while all cases share the grid barriers.  A case that
// has stopped leaves its vectors alone; the launch ends when every case has
// stopped.  Preparation (x0's mean row, sum(x0 h^3)), the initial residual
// and zr = M^-1 r run in the same launch.

struct BatchArgs {
  const int* cfirst;
  const int* cblocks;
  double* part;
  int* case_done;
  int ncase;
  int groups;
};

// Dynamic shared memory of the batched solver: the persistent solver's, then
// the deal of the groups: gfirst and the previous gfirst (ncase + 1 ints
// each) and the running flags (ncase ints).
__host__ __device__ constexpr size_t batch_smem(int ncase) {
  return kPersistentSmem + size_t(3 * ncase + 2) * sizeof(int);
}

// Deals the G block groups of the grid to the running cases, in case order,
// in proportion to their blocks (at least one, at most one per block): the
// groups of case c are gfirst[c] .. gfirst[c+1]-1 (none for a stopped case).
// Integer arithmetic only, so every CTA computes the same deal.  One thread.
__device__ void batch_deal(const int* cfirst, const int* running, int ncase, int G, int* gfirst) {
  long long nba = 0;
  for (int c = 0; c < ncase; ++c)
    if (running[c]) nba += cfirst[c + 1] - cfirst[c];
  int used = 0;
  // first pass: floor of the proportional share, in gfirst[c+1] as a count
  for (int c = 0; c < ncase; ++c) {
    const int nb = cfirst[c + 1] - cfirst[c];
    int q = 0;
    if (running[c] && nba > 0) q = max(1, min(nb, int((long long)G * nb / nba)));
    gfirst[c + 1] = q;
    used += q;
  }
  // over (shares of one): take back round-robin from cases with more than one
  for (int c = 0; used > G; c = (c + 1) % ncase)
    if (gfirst[c + 1] > 1) {
      --gfirst[c + 1];
      --used;
    }
  // spare groups: round-robin to running cases with blocks left to share
  bool any = true;
  while (used < G && any) {
    any = false;
    for (int c = 0; c < ncase && used < G; ++c)
      if (running[c] && gfirst[c + 1] < cfirst[c + 1] - cfirst[c]) {
        ++gfirst[c + 1];
        ++used;
        any = true;
      }
  }
  gfirst[0] = 0;
  for (int c = 0; c < ncase; ++c) gfirst[c + 1] += gfirst[c];
}

// A group's place in the deal: case (-1: none), index within the case's
// groups, the case's group count and the group's block count.
struct GroupPlace {
  int c, j, ng, nblk;
};

__device__ __forceinline__ GroupPlace group_place(const int* gfirst, const int* cfirst, int ncase, int gidx) {
  GroupPlace p{-1, 0, 0, 0};
  for (int c = 0; c < ncase; ++c)
    if (gidx >= gfirst[c] && gidx < gfirst[c + 1]) {
      p.c = c;
      p.j = gidx - gfirst[c];
      p.ng = gfirst[c + 1] - gfirst[c];
      const int nb = cfirst[c + 1] - cfirst[c];
      p.nblk = nb > p.j ? (nb - p.j + p.ng - 1) / p.ng : 0;
    }
  return p;
}

// Grid barrier with per-case sums: each group's partials, then every group
// of case c sums the partials of the groups [g0, g1) that worked for c in
// this phase.  With RUN, also loads the cases' running flags (case_done as
// written before the barrier) into running[] in every CTA.
template <int NR, bool RUN>
__device__ bool batch_allreduce(double (&v)[NR], const BatchArgs& B, const GridSync& Gs, unsigned int& epoch,
                                double* gsm, const GroupIdx& G, int gidx, int c, int g0, int g1, int* running) {
  const unsigned int k = epoch;
  double* part = B.part + size_t(k & 1u) * B.groups * 8;
  group_reduce<NR>(v, gsm, G);
  if (G.lane == 0)
#pragma unroll
    for (int r = 0; r < NR; ++r) part[gidx * 8 + r] = v[r];
  __shared__ int s_ok;
  __syncthreads();  // the CTA's partials and phase stores precede the arrival
  if (threadIdx.x == 0) {
    red_add_release(Gs.arrive, 1u);
    const unsigned int target = (k + 1u) * gridDim.x;
    const long long t0 = clock64();
    int ok = 1;
    while (ld_acquire(Gs.arrive) < target) {
      if (clock64() - t0 > Gs.limit) {
        ok = 0;
        break;
      }
    }
    if (!ok) atomicExch(Gs.error, 1);
    s_ok = ok;
    epoch = k + 1u;
  }
  __syncthreads();
  if (!s_ok) return false;
  if (RUN) {
    for (int i = threadIdx.x; i < B.ncase; i += blockDim.x) running[i] = B.case_done[i] == 0;
    __syncthreads();
  }
  if (c >= 0) {
    double acc[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] = 0.0;
    for (int g = g0 + G.lane; g < g1; g += GROUP)
#pragma unroll
      for (int r = 0; r < NR; ++r) acc[r] += part[g * 8 + r];
    group_reduce<NR>(acc, gsm, G);
#pragma unroll
    for (int r = 0; r < NR; ++r) v[r] = acc[r];
  }
  return true;
}

// A group's k-th block: blocks j, j + ng, j + 2 ng, ... of its case's list
// (decreasing cost, so the groups' shares balance); the entries of the first
// KB_CACHE are staged when the group is placed, later ones on the way.
__device__ __forceinline__ const BlockInfo& batch_block(const DevMesh& M, const BatchArgs& B, const BlockInfo* cache,
                                                        GroupTile& tile, const GroupPlace& P, int k,
                                                        const GroupIdx& G) {
  if (k < KB_CACHE) return cache[G.g * KB_CACHE + k];
  group_sync(G.g);
  fill_block_info(M, B.cblocks[B.cfirst[P.c] + P.j + k * P.ng], tile.bi, G.lane);
  group_sync(G.g);
  return tile.bi;
}

// Stages the table entries of the group's first KB_CACHE blocks (the caller
// synchronises the CTA before they are read).
__device__ __forceinline__ void batch_fill_cache(const DevMesh& M, const BatchArgs& B, BlockInfo* cache,
                                                 const GroupPlace& P, const GroupIdx& G) {
  for (int k = 0; k < KB_CACHE && k < P.nblk; ++k)
    if (G.lane < 32) fill_block_info(M, B.cblocks[B.cfirst[P.c] + P.j + k * P.ng], cache[G.g * KB_CACHE + k], G.lane);
}

#define BATCH_BLOCKS(bi) \
  for (int k_ = 0; k_ < P.nblk; ++k_) if (const BlockInfo& bi = batch_block(M, B, cache, tile, P, k_, G); true)

template <class T>
__global__ void __launch_bounds__(PNT, 8 / PGROUPS) k_bicg_batched(KArgs<T> A, GridSync Gs, BatchArgs B) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* inv_eig = reinterpret_cast<double*>(smem_raw);
  BlockInfo* cache = reinterpret_cast<BlockInfo*>(smem_raw + kSmemCache);
  GroupTile* tiles = reinterpret_cast<GroupTile*>(smem_raw + kSmemTiles);
  int* gfirst = reinterpret_cast<int*>(smem_raw + kPersistentSmem);
  int* gfirst_prev = gfirst + B.ncase + 1;
  int* running = gfirst_prev + B.ncase + 1;
  __shared__ KrylovState Sg[PGROUPS];
  __shared__ double gsm_all[PGROUPS][16];
  __shared__ unsigned int epoch;
  __shared__ int s_changed;
  const GroupIdx G;
  const DevMesh& M = A.M;
  GroupTile& tile = tiles[G.g];
  double* gsm = gsm_all[G.g];
  KrylovState& S = Sg[G.g];
  const int gidx = blockIdx.x * PGROUPS + G.g;
  const int Gtot = gridDim.x * PGROUPS;
  fd_fill_inverse_eigen(inv_eig, c_lam);
  for (int i = threadIdx.x; i < B.ncase; i += blockDim.x) running[i] = 1;
  if (threadIdx.x == 0) epoch = 0u;
  __syncthreads();
  if (threadIdx.x == 0) batch_deal(B.cfirst, running, B.ncase, Gtot, gfirst);
  __syncthreads();
  GroupPlace P = group_place(gfirst, B.cfirst, B.ncase, gidx);
  batch_fill_cache(M, B, cache, P, G);
  if (G.lane == 0 && P.c >= 0) S = A.st[P.c];
  __syncthreads();
  // the case's first group writes its state and done flag
  auto lead = [&]() { return P.c >= 0 && gidx == gfirst[P.c] && G.lane == 0; };
  // two-level preconditioner: the coarse correction of each running case on
  // v (zr or zv) from its restriction rc, added by the case's groups; the
  // case's added sum(v h^3) comes back to its groups (one more barrier)
  auto coarse_phase = [&](const double* rc, T* v, bool active, double& added) -> bool {
    double a[1] = {0.0};
    if (active) {
      const int cf = B.cfirst[P.c], n = B.cfirst[P.c + 1] - cf;
      const long long off = A.coff[P.c];
      BATCH_BLOCKS(bi) a[0] += coarse_block_case<T>(A, G, bi.id, cf, n, off, rc, v, gsm);
    }
    const bool okc = batch_allreduce<1, false>(a, B, Gs, epoch, gsm, G, gidx, P.c, gfirst[max(P.c, 0)],
                                               gfirst[max(P.c, 0) + 1], nullptr);
    added = a[0];
    return okc;
  };
  bool ok = true;
  // PREP, INIT, P0: one barrier each
  {
    double a[1] = {0.0};
    BATCH_BLOCKS(bi) a[0] += prep_block<T>(A, G, bi);
    ok = batch_allreduce<1, false>(a, B, Gs, epoch, gsm, G, gidx, P.c, gfirst[max(P.c, 0)], gfirst[max(P.c, 0) + 1],
                                   nullptr);
    if (ok && P.c >= 0 && G.lane == 0) S.mean_sum = a[0];
    __syncthreads();
  }
  if (ok) {
    double a[1] = {0.0};
    BATCH_BLOCKS(bi) a[0] += init_block<T>(A, G, tile, bi, S.mean_sum);
    ok = batch_allreduce<1, false>(a, B, Gs, epoch, gsm, G, gidx, P.c, gfirst[max(P.c, 0)], gfirst[max(P.c, 0) + 1],
                                   nullptr);
    if (ok && P.c >= 0 && G.lane == 0) fin_init(S, a[0]);
    __syncthreads();
  }
  if (ok) {
    double a[1] = {0.0};
    if (P.c >= 0 && !S.done) BATCH_BLOCKS(bi) a[0] += p0_block<T>(A, G, tile, bi, inv_eig);
    ok = batch_allreduce<1, false>(a, B, Gs, epoch, gsm, G, gidx, P.c, gfirst[max(P.c, 0)], gfirst[max(P.c, 0) + 1],
                                   nullptr);
    double cz = 0.0;
    if (ok && A.cnb) ok = coarse_phase(A.crc_r, A.z1, P.c >= 0 && !S.done, cz);
    // q = 0 at the start, so z1 = zr
    if (ok && P.c >= 0 && G.lane == 0) S.ms_zr = S.mean_sum = a[0] + cz;
    if (ok && lead()) {
      A.st[P.c] = S;
      B.case_done[P.c] = S.done;
    }
    __syncthreads();
  }
  while (ok) {
    bool active = P.c >= 0 && !S.done;
    bool restart = active && S.restart_pending != 0;
    double beta = restart ? 0.0 : S.beta;
    double a[2] = {0.0, 0.0};
    if (active) BATCH_BLOCKS(bi) p1_block<T>(A, G, tile, bi, inv_eig, beta, S.mean_sum, restart, a);
    // the groups that did P1 for case c: this pass's deal
    for (int i = threadIdx.x; i <= B.ncase; i += blockDim.x) gfirst_prev[i] = gfirst[i];
    __syncthreads();
    if (!(ok = batch_allreduce<2, true>(a, B, Gs, epoch, gsm, G, gidx, P.c, gfirst[max(P.c, 0)],
                                        gfirst[max(P.c, 0) + 1], running)))
      break;
    // cases that stopped in the last iteration give their groups to the
    // running ones: deal again, take up the new case's state (written by its
    // first group after the last iteration) and its P1 sums over the groups
    // that did its P1
    if (threadIdx.x == 0) {
      int any = 0, changed = 0;
      for (int cc = 0; cc < B.ncase; ++cc) {
        any |= running[cc];
        changed |= (!running[cc]) && gfirst[cc + 1] > gfirst[cc];
      }
      s_changed = any ? changed : -1;
      if (any && changed) batch_deal(B.cfirst, running, B.ncase, Gtot, gfirst);
    }
    __syncthreads();
    if (s_changed < 0) break;  // every case has stopped
    if (s_changed) {
      const int old_c = P.c;
      P = group_place(gfirst, B.cfirst, B.ncase, gidx);
      batch_fill_cache(M, B, cache, P, G);
      if (G.lane == 0 && P.c >= 0) S = A.st[P.c];
      __syncthreads();
      if (P.c >= 0 && P.c != old_c) {  // P1 sums of the new case, from the groups that did them
        double acc[2] = {0.0, 0.0};
        for (int g = gfirst_prev[P.c] + G.lane; g < gfirst_prev[P.c + 1]; g += GROUP) {
          const double* part = B.part + size_t((epoch - 1u) & 1u) * B.groups * 8;
          acc[0] += part[g * 8];
          acc[1] += part[g * 8 + 1];
        }
        group_reduce<2>(acc, gsm, G);
        a[0] = acc[0];
        a[1] = acc[1];
      }
      active = P.c >= 0 && !S.done;
      restart = active && S.restart_pending != 0;
      beta = restart ? 0.0 : S.beta;
    }
    if (active && G.lane == 0) {
      fin_a(S, S.mean_sum, restart);
      fin_b(S, a[0]);
      S.beta = beta;                          // the beta that formed z1, for P3
      S.mean_sum = S.ms_zr - S.alpha * a[1];  // sum(z2 h^3)
    }
    __syncthreads();
    if (A.cnb) {  // zv += the coarse correction of nu; sum(z2 h^3) with it
      double cv = 0.0;
      if (!(ok = coarse_phase(A.crc_v, A.z2, active, cv))) break;
      if (active && G.lane == 0) S.mean_sum = S.ms_zr - S.alpha * (a[1] + cv);
      __syncthreads();
    }
    const int g0 = gfirst[max(P.c, 0)], g1 = gfirst[max(P.c, 0) + 1];
    double d[2] = {0.0, 0.0};
    if (active) BATCH_BLOCKS(bi) p2_block<T>(A, G, tile, bi, S.alpha, S.mean_sum, d);
    if (!(ok = batch_allreduce<2, false>(d, B, Gs, epoch, gsm, G, gidx, P.c, g0, g1, nullptr))) break;
    if (active && G.lane == 0) fin_d(S, d);
    __syncthreads();
    double e[4] = {0.0, 0.0, 0.0, 0.0};
    if (active)
      BATCH_BLOCKS(bi) p3_block<T>(A, G, tile, bi, inv_eig, xslot(A, S.cur), xslot(A, S.nxt), S.alpha, S.beta,
                                   S.omega, e);
    if (!(ok = batch_allreduce<4, false>(e, B, Gs, epoch, gsm, G, gidx, P.c, g0, g1, nullptr))) break;
    if (active && G.lane == 0) {
      const double re[2] = {e[0], e[1]};
      fin_e(S, re);
      S.ms_zr = e[2];
      S.mean_sum = S.restart_pending ? e[2] : e[2] + S.beta * e[3];  // sum(z1 h^3) of the next P1
    }
    __syncthreads();
    if (A.cnb) {  // zr += the coarse correction of r; the sums with it
      double cr = 0.0;
      if (!(ok = coarse_phase(A.crc_r, A.z1, active && !S.done, cr))) break;
      if (active && !S.done && G.lane == 0) {
        S.ms_zr = e[2] + cr;
        S.mean_sum = S.restart_pending ? S.ms_zr : S.ms_zr + S.beta * e[3];
      }
      __syncthreads();
    }
    if (active && lead()) {
      A.st[P.c] = S;
      B.case_done[P.c] = S.done;
    }
    __syncthreads();
  }
  if (!ok) {  // a barrier timed out: every case reports it
    if (threadIdx.x == 0 && blockIdx.x == 0)
      for (int cc = 0; cc < B.ncase; ++cc) {
        A.st[cc].done = 1;
        A.st[cc].status = SOLVE_BARRIER_TIMEOUT;
      }
    return;
  }
  // every case has stopped: deal all cases again and move each case's best
  // iterate into x (slot 0), block by block
  for (int i = threadIdx.x; i < B.ncase; i += blockDim.x) running[i] = 1;
  __syncthreads();
  if (threadIdx.x == 0) batch_deal(B.cfirst, running, B.ncase, Gtot, gfirst);
  __syncthreads();
  P = group_place(gfirst, B.cfirst, B.ncase, gidx);
  batch_fill_cache(M, B, cache, P, G);
  if (G.lane == 0 && P.c >= 0) S = A.st[P.c];
  __syncthreads();
  if (P.c >= 0 && S.best != 0) {
    const T* src = xslot(A, S.best);
    BATCH_BLOCKS(bi) {
      double v[8];
      load_col(src, bi.id, G, v);
      store_col(A.xs0, bi.id, G, v);
    }
  }
}

// ---------------------------------------------------------------------------
// Iterative refinement (mixed precision): FP64 true residual and update.
// ---------------------------------------------------------------------------
// x += e (e may be null: only the mean-row zeroing and sum); sum(x h^3)
__global__ void __launch_bounds__(NT) k_refine_update(DevMesh M, double* x, const float* __restrict__ e,
                                                      int zero_mean_row, KrylovState* st, GridReduce g) {
  __shared__ double red[64];
  double acc[1] = {0.0};
  for (int b = blockIdx.x; b < M.nb; b += gridDim.x) {
    const double h = M.h[b], h3 = h * h * h;
    double s = 0.0;
    for (int c = threadIdx.x; c < BN; c += NT) {
      const size_t i = size_t(b) * BN + c;
      double v = x[i];
      if (zero_mean_row && b == M.mean_block && c == 0) v = 0.0;
      if (e) v += double(e[i]);
      x[i] = v;
      s += v;
    }
    acc[0] += s * h3;
  }
  if (grid_reduce<1>(acc, g, red) && threadIdx.x == 0) st->mean_sum = acc[0];
}

// r32 = b' - A x in FP64 arithmetic (b' = b with the mean row zeroed for modes
// 1 and 3), ||b' - A x||_2 into st->err (the FP64-checked residual).
__global__ void __launch_bounds__(NT) k_true_residual(DevMesh M, const double* __restrict__ b,
                                                      const double* __restrict__ x, float* __restrict__ r32,
                                                      int mean_mode, int zero_mean_row, KrylovState* st,
                                                      GridReduce g) {
  __shared__ GroupTile tiles[GROUPS];
  __shared__ double red[64];
  const GroupIdx G;
  const double ms = st->mean_sum;
  double acc[1] = {0.0};
  GROUP_BLOCKS(blk) {
    double col[8], y[8], bc[8];
    load_col(x, blk, G, col);
    fill_block_info(M, blk, tiles[G.g].bi, G.lane);
    group_sync(G.g);
    spmv_group(tiles[G.g].bi, VecAt<double>{x}, col, ms, mean_mode, tiles[G.g], G, y);
    load_col(b, blk, G, bc);
    if (zero_mean_row && blk == M.mean_block && G.lane == 0) bc[0] = 0.0;
    float* rb = r32 ? r32 + size_t(blk) * BN + G.gy * 8 + G.gx : nullptr;
#pragma unroll
    for (int z = 0; z < 8; ++z) {
      const double ri = bc[z] - y[z];
      if (rb) rb[z * 64] = float(ri);
      acc[0] += ri * ri;
    }
  }
  if (grid_reduce<1>(acc, g, red) && threadIdx.x == 0) {
    st->rr = acc[0];
    st->err = sqrt(acc[0]);
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
template <class T>
static KArgs<T> make_args(const DevMesh& M, const T* b, T* x, T* const v[9], PoissonWork& W, KrylovState* st,
                          int mean_mode, int zero_mean_row, int site) {
  KArgs<T> A;
  A.M = M;
  A.b = b;
  A.r = v[0];
  A.rhat = v[1];
  A.p = v[2];
  A.nu = v[3];
  A.t = v[4];
  A.z1 = v[5];
  A.z2 = v[6];
  A.xs0 = x;
  A.xs1 = v[7];
  A.xs2 = v[8];
  A.st = st;
  A.g.partial = W.partial;
  A.g.counter = W.counters + site;
  A.mean_mode = mean_mode;
  A.zero_mean_row = zero_mean_row;
  A.ncache = 0;
  A.cnb = 0;
  A.cinv = nullptr;
  A.coff = nullptr;
  A.crc_v = A.crc_r = nullptr;
  A.cw = nullptr;
  A.lw = nullptr;
  A.llab = nullptr;
  return A;
}

int launch_weighted_sum(const DevMesh& M, const double* v, double* d_out, PoissonWork& W,
                        cudaStream_t s) {
  GridReduce g{W.partial, W.counters + 8};
  { ProfScope ps("weighted_sum", s); k_weighted_sum<<<W.grid, NT, 0, s>>>(M, v, g, d_out, nullptr); }
  CUP_CUDA_TRY(cudaGetLastError());
  return 0;
}

int launch_poisson_apply(const DevMesh& M, const double* x, double* y, int mean_mode,
                         PoissonWork& W, cudaStream_t s) {
  poisson_init_constants();
  GridReduce g{W.partial, W.counters + 9};
  double* ms = &W.st->mean_sum;
  if (mean_mode == 1 || mean_mode == 2) {
    { ProfScope ps("weighted_sum", s); k_weighted_sum<<<W.grid, NT, 0, s>>>(M, x, g, nullptr, ms); }
    CUP_CUDA_TRY(cudaGetLastError());
  }
  { ProfScope ps("spmv", s); k_spmv<<<W.ggrid, NT, 0, s>>>(M, x, y, ms, mean_mode); }
  CUP_CUDA_TRY(cudaGetLastError());
  return 0;
}

int launch_block_inverse(const DevMesh& M, const double* in, double* out, PoissonWork& W,
                         cudaStream_t s) {
  poisson_init_constants();
  { ProfScope ps("block_inverse", s); k_block_inverse<<<W.ggrid, NT, 0, s>>>(M, in, out); }
  CUP_CUDA_TRY(cudaGetLastError());
  return 0;
}

// Programmatic dependent launch for this thread's solver launches (off while
// a step is captured into a CUDA graph).
static thread_local bool t_pdl = true;
void solver_pdl(bool on) { t_pdl = on; }

// Launches a solver kernel with programmatic stream serialization: its CTAs
// may be scheduled while the previous kernel drains and wait in pdl_wait().
template <class T>
static cudaError_t launch_pdl(void (*kern)(KArgs<T>), int grid, cudaStream_t s, const KArgs<T>& A,
                              size_t dyn_smem = 0) {
  if (dyn_smem > 0) {
    const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn_smem));
    if (e != cudaSuccess) return e;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(NT);
  cfg.dynamicSmemBytes = dyn_smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = t_pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, A);
}

// CTAs of the persistent solver for a mesh of nb blocks: all co-resident,
// at most one per PGROUPS blocks, two partial slots of 8 doubles per CTA in the
// reduction buffer.
template <class T>
static int persistent_grid(int nb, const PoissonWork& W, int* grid, size_t dyn = kPersistentSmem) {
  void (*kern)(KArgs<T>, GridSync) = k_bicg_persistent<T>;
  CUP_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn)));
  int per_sm = 0, dev = 0, sms = 0;
  CUP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, PNT, dyn));
  CUP_CUDA_TRY(cudaGetDevice(&dev));
  CUP_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (per_sm < 1) return set_error(CUP_ERR_CUDA, "persistent BiCGSTAB: kernel does not fit on an SM");
  *grid = std::max(1, std::min({per_sm * sms, (nb + PGROUPS - 1) / PGROUPS, std::max(W.grid, W.ggrid) / 2}));
  return 0;
}

int persistent_grid_max(int nb, const PoissonWork& W, int* grid) {
  int g1 = 0, g2 = 0;
  if (int rc = persistent_grid<double>(nb, W, &g1)) return rc;
  if (int rc = persistent_grid<float>(nb, W, &g2)) return rc;
  *grid = std::min(g1, g2);
  return 0;
}

int persistent_solver_groups(int nb, PoissonWork& W, int* groups) {
  int g1 = 0, g2 = 0;
  if (int rc = persistent_grid<double>(nb, W, &g1)) return rc;
  if (int rc = persistent_grid<float>(nb, W, &g2)) return rc;
  if (g1 != g2) return set_error(CUP_ERR_CUDA, "persistent BiCGSTAB: FP64 and FP32 grids differ");
  W.pgrid = g1;  // the launches use it (nothing to query while a graph is captured)
  *groups = g1 * PGROUPS;
  return 0;
}

// Launches the persistent solver: one cooperative grid (every CTA resident)
// that runs iterations until the state says done.
template <class T>
static int launch_persistent(const KArgs<T>& A, PoissonWork& W, cudaStream_t s, const char* name) {
  const size_t dyn = A.lw ? kLearnedSmem : kPersistentSmem;
  void (*kern)(KArgs<T>, GridSync) = k_bicg_persistent<T>;
  int grid = W.pgrid;
  if (grid <= 0 || A.lw)
    if (int rc = persistent_grid<T>(A.M.nb, W, &grid, dyn)) return rc;
  // the arrival counter and the error flag start at zero
  CUP_CUDA_TRY(cudaMemsetAsync(W.bar, 0, sizeof(unsigned int), s));
  CUP_CUDA_TRY(cudaMemsetAsync(W.bar_error, 0, sizeof(int), s));
  GridSync Gs{W.bar, W.partial, W.bar_error, W.barrier_cycles > 0 ? W.barrier_cycles : kBarrierClockLimit};
  KArgs<T> Aa = A;
  void* args[] = {(void*)&Aa, (void*)&Gs};
  ProfScope ps(name, s);
  CUP_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3(PNT), args, dyn, s));
  return 0;
}

// CTAs and block groups of the batched solver: every CTA resident (one
// group per block at most), the same shape as the single-case solver.
int batch_solver_shape(int nb, int ncase, int* grid, int* groups) {
  const size_t dyn = batch_smem(ncase);
  // every CTA resident for the FP64 solver and the FP32 inner solves alike
  void (*kern)(KArgs<double>, GridSync, BatchArgs) = k_bicg_batched<double>;
  void (*kernf)(KArgs<float>, GridSync, BatchArgs) = k_bicg_batched<float>;
  CUP_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn)));
  CUP_CUDA_TRY(cudaFuncSetAttribute(kernf, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn)));
  int per_sm = 0, per_sm_f = 0, dev = 0, sms = 0;
  CUP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, PNT, dyn));
  CUP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_f, kernf, PNT, dyn));
  per_sm = std::min(per_sm, per_sm_f);
  CUP_CUDA_TRY(cudaGetDevice(&dev));
  CUP_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (per_sm < 1) return set_error(CUP_ERR_CUDA, "batched BiCGSTAB: kernel does not fit on an SM");
  *grid = std::max(1, std::min(per_sm * sms, (nb + PGROUPS - 1) / PGROUPS));
  *groups = *grid * PGROUPS;
  return 0;
}

// The batched launch on vectors of type T: FP64 for the solver, FP32 for the
// inner solves of the mixed-precision batch.
// zero_mean_row: the mean-constraint row's right-hand side taken as zero
// (the solver), or as given (the inner solves: it holds the row's residual).
// case_tol_rel (launched path only): each case's own relative tolerance in
// place of P.tol_rel (each case's Krylov state carries its stopping test).
template <class T>
static int batched_launch(const DevMesh& M, const T* b, T* x, T* const v[9], const SolveParams& P, PoissonWork& W,
                          BatchWork& B, SolveStats* out, cudaStream_t s, const BatchCoarse* coarse,
                          int zero_mean_row, const double* case_tol_rel = nullptr) {
  poisson_init_constants();
  if (B.ncase < 1 || !B.st) return set_error(CUP_ERR_STATE, "batched BiCGSTAB: not a batch");
  const int zmr = zero_mean_row;
  if (P.graph) {  // captured: the initial states come from the device template
    CUP_CUDA_TRY(cudaMemcpyAsync(B.st, B.st_init, sizeof(KrylovState) * B.ncase, cudaMemcpyDeviceToDevice, s));
  } else {
    std::vector<KrylovState> init(B.ncase);
    for (int c = 0; c < B.ncase; ++c) {
      krylov_init_state(P, init[c]);
      if (case_tol_rel) init[c].tol_rel = case_tol_rel[c];
    }
    CUP_CUDA_TRY(cudaMemcpyAsync(B.st, init.data(), sizeof(KrylovState) * B.ncase, cudaMemcpyHostToDevice, s));
  }
  CUP_CUDA_TRY(cudaMemsetAsync(B.case_done, 0, sizeof(int) * B.ncase, s));
  CUP_CUDA_TRY(cudaMemsetAsync(W.bar, 0, sizeof(unsigned int), s));
  CUP_CUDA_TRY(cudaMemsetAsync(W.bar_error, 0, sizeof(int), s));
  KArgs<T> A = make_args<T>(M, b, x, v, W, B.st, P.mean_mode, zmr, 0);
  A.ncache = KB_CACHE;
  if (coarse && coarse->inv) {  // the cases' two-level preconditioners
    A.cnb = 1;
    A.cinv = coarse->inv;
    A.coff = coarse->off;
    A.crc_v = coarse->rc;
    A.crc_r = coarse->rc2;
    A.cw = coarse->w;
  }
  GridSync Gs{W.bar, W.partial, W.bar_error, W.barrier_cycles > 0 ? W.barrier_cycles : kBarrierClockLimit};
  BatchArgs Ba{B.cfirst, B.cblocks, B.part, B.case_done, B.ncase, B.groups};
  void* args[] = {(void*)&A, (void*)&Gs, (void*)&Ba};
  const size_t dyn = batch_smem(B.ncase);
  void (*kern)(KArgs<T>, GridSync, BatchArgs) = k_bicg_batched<T>;
  if (!P.graph) CUP_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn)));
  {
    ProfScope ps("bicg_batched", s);
    CUP_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)kern, dim3(B.grid), dim3(PNT), args, dyn, s));
  }
  if (P.graph) return 0;  // the caller reads the states after the graph runs
  int h_err = 0;
  std::vector<KrylovState> fin(B.ncase);
  CUP_CUDA_TRY(cudaMemcpyAsync(&h_err, W.bar_error, sizeof(int), cudaMemcpyDeviceToHost, s));
  CUP_CUDA_TRY(cudaMemcpyAsync(fin.data(), B.st, sizeof(KrylovState) * B.ncase, cudaMemcpyDeviceToHost, s));
  CUP_CUDA_TRY(cudaStreamSynchronize(s));
  if (h_err) return set_error(CUP_ERR_CUDA, "batched BiCGSTAB: a grid barrier wait timed out");
  for (int c = 0; c < B.ncase; ++c) {
    out[c].iterations = fin[c].k;
    out[c].restarts = fin[c].restarts;
    out[c].status = fin[c].done ? fin[c].status : SOLVE_MAXITER;
    out[c].outer = 0;
    out[c].err_init = fin[c].err_init;
    out[c].err_opt = fin[c].err_opt;
  }
  return 0;
}

int poisson_bicgstab_batched(const DevMesh& M, const double* b, double* x, const SolveParams& P,
                             PoissonWork& W, BatchWork& B, SolveStats* out, cudaStream_t s,
                             const BatchCoarse* coarse) {
  double* const v[9] = {W.r, W.rhat, W.p, W.nu, W.t, W.z1, W.z2, W.xs[1], W.xs[2]};
  const int zmr = (P.mean_mode == 1 || P.mean_mode == 3) ? 1 : 0;
  return batched_launch<double>(M, b, x, v, P, W, B, out, s, coarse, zmr);
}

// ---- mixed precision in a batch of cases ----------------------------------
// FP32 batched inner solves (every case in one launch, with the batch's
// coarse spaces when they are built) inside FP64 iterative refinement per
// case, as poisson_mixed does for one case.  A case that has reached its
// tolerance (or stopped) gets a zero inner right-hand side, which stops it
// at once in the inner solve, so its x stays as it is.

// Per block: x's mean-row entry zeroed (first call), e added, the block's
// sum(x h^3) into bpart[b].
__global__ void __launch_bounds__(NT) k_refine_update_batch(DevMesh M, double* x, const float* __restrict__ e,
                                                            int zero_mean_row, double* __restrict__ bpart) {
  __shared__ double red[64];
  for (int b = blockIdx.x; b < M.nb; b += gridDim.x) {
    const double h = M.h[b], h3 = h * h * h;
    const int mb = M.case_mean[M.bcase[b]];
    double s[1] = {0.0};
    for (int c = threadIdx.x; c < BN; c += NT) {
      const size_t i = size_t(b) * BN + c;
      double v = x[i];
      if (zero_mean_row && b == mb && c == 0) v = 0.0;
      if (e) v += double(e[i]);
      x[i] = v;
      s[0] += v;
    }
    block_reduce<1>(s, red);
    if (threadIdx.x == 0) bpart[b] = s[0] * h3;
  }
}

// Per block: r = b - A x in FP32 into r32 (each case's operator with its own
// mean row, case_ms[c] = sum(x h^3) of case c), |r|^2 of the block into bpart.
__global__ void __launch_bounds__(NT) k_true_residual_batch(DevMesh M, const double* __restrict__ b,
                                                            const double* __restrict__ x, float* __restrict__ r32,
                                                            int mean_mode, int zero_mean_row,
                                                            const double* __restrict__ case_ms,
                                                            double* __restrict__ bpart) {
  __shared__ GroupTile tiles[GROUPS];
  __shared__ double gsm[2 * GROUPS];
  const GroupIdx G;
  GROUP_BLOCKS(blk) {
    double col[8], y[8], bc[8];
    load_col(x, blk, G, col);
    fill_block_info(M, blk, tiles[G.g].bi, G.lane);
    group_sync(G.g);
    const int c = M.bcase[blk];
    spmv_group(tiles[G.g].bi, VecAt<double>{x}, col, case_ms[c], mean_mode, tiles[G.g], G, y);
    load_col(b, blk, G, bc);
    if (zero_mean_row && blk == M.case_mean[c] && G.lane == 0) bc[0] = 0.0;
    float* rb = r32 + size_t(blk) * BN + G.gy * 8 + G.gx;
    double a[1] = {0.0};
#pragma unroll
    for (int z = 0; z < 8; ++z) {
      const double ri = bc[z] - y[z];
      rb[z * 64] = float(ri);
      a[0] += ri * ri;
    }
    group_reduce<1>(a, &gsm[2 * G.g], G);
    if (G.lane == 0) bpart[blk] = a[0];
  }
}

// out[c] = the sum of part over case c's blocks (one CTA per case, fixed order)
__global__ void __launch_bounds__(NT) k_case_total(const double* __restrict__ part, const int* __restrict__ first,
                                                   double* __restrict__ out) {
  __shared__ double red[64];
  const int c = blockIdx.x;
  double s[1] = {0.0};
  for (int b = first[c] + threadIdx.x; b < first[c + 1]; b += NT) s[0] += part[b];
  block_reduce<1>(s, red);
  if (threadIdx.x == 0) out[c] = s[0];
}

int poisson_mixed_batched(const DevMesh& M, const double* b, double* x, const SolveParams& P, PoissonWork& W,
                          BatchWork& B, SolveStats* out, cudaStream_t s, const BatchCoarse* coarse,
                          const int* d_first, const int* first, double* bpart, double* d_case) {
  const int K = B.ncase;
  const int zmr = (P.mean_mode == 1 || P.mean_mode == 3) ? 1 : 0;
  float* const v[9] = {W.fr, W.frhat, W.fp, W.fnu, W.ft, W.fz1, W.fz2, W.fxs[1], W.fxs[2]};
  float* e = W.fxs[0];
  double* ms = d_case;     // K: each case's sum(x h^3)
  double* rr = d_case + K; // K: each case's |b - A x|^2
  const size_t n = size_t(M.nb) * BN;
  std::vector<double> h_rr(K);
  auto update = [&](const float* ee) -> int {
    k_refine_update_batch<<<W.grid, NT, 0, s>>>(M, x, ee, ee ? 0 : zmr, bpart);
    k_case_total<<<K, NT, 0, s>>>(bpart, d_first, ms);
    CUP_CUDA_TRY(cudaGetLastError());
    return 0;
  };
  auto residual = [&]() -> int {
    {
      ProfScope ps("refine_true_residual_fp64", s);
      k_true_residual_batch<<<W.ggrid, NT, 0, s>>>(M, b, x, W.r32, P.mean_mode, zmr, ms, bpart);
      k_case_total<<<K, NT, 0, s>>>(bpart, d_first, rr);
    }
    CUP_CUDA_TRY(cudaGetLastError());
    CUP_CUDA_TRY(cudaMemcpyAsync(h_rr.data(), rr, K * sizeof(double), cudaMemcpyDeviceToHost, s));
    CUP_CUDA_TRY(cudaStreamSynchronize(s));
    return 0;
  };
  if (int rc = update(nullptr)) return rc;
  if (int rc = residual()) return rc;
  std::vector<double> err0(K), err(K);
  std::vector<int> active(K, 1), total(K, 0), restarts(K, 0), outer_n(K, 0);
  auto converged = [&](int k) { return err[k] <= P.tol_abs || err[k] / err0[k] <= P.tol_rel; };
  for (int k = 0; k < K; ++k) {
    err0[k] = err[k] = std::sqrt(h_rr[k]);
    out[k] = SolveStats{};
    out[k].err_init = err0[k];
    out[k].status = SOLVE_MAXITER;
    if (!(err0[k] == err0[k])) {
      out[k].status = SOLVE_NAN;
      active[k] = 0;
    } else if (err0[k] <= P.tol_abs) {
      out[k].status = SOLVE_CONVERGED;
      active[k] = 0;
    }
  }
  std::vector<SolveStats> in(K);
  std::vector<double> q(K, 0.5);
  for (int outer = 0; outer < 40; ++outer) {
    int min_total = P.max_iter, nact = 0;
    for (int k = 0; k < K; ++k) {
      if (active[k] && converged(k)) {
        out[k].status = SOLVE_CONVERGED;
        active[k] = 0;
      }
      if (!active[k]) continue;
      ++nact;
      // each case's inner tolerance: the reduction it still needs, within
      // FP32 reach, as for one case
      const double want = std::max(P.tol_abs, P.tol_rel * err0[k]);
      q[k] = std::min(0.5, std::max(2e-5, 0.5 * want / err[k]));
      min_total = std::min(min_total, total[k]);
    }
    if (nact == 0) break;
    for (int k = 0; k < K; ++k)
      if (!active[k])
        CUP_CUDA_TRY(cudaMemsetAsync(W.r32 + size_t(first[k]) * BN, 0,
                                     size_t(first[k + 1] - first[k]) * BN * sizeof(float), s));
    SolveParams Q = P;
    Q.tol_abs = 0.0;
    Q.tol_rel = 0.5;
    Q.max_iter = std::max(1, P.max_iter - min_total);
    CUP_CUDA_TRY(cudaMemsetAsync(e, 0, n * sizeof(float), s));
    if (int rc = batched_launch<float>(M, W.r32, e, v, Q, W, B, in.data(), s, coarse, 0, q.data())) return rc;
    if (int rc = update(e)) return rc;
    if (int rc = residual()) return rc;
    for (int k = 0; k < K; ++k) {
      if (!active[k]) continue;
      total[k] += in[k].iterations;
      restarts[k] += in[k].restarts;
      outer_n[k] = outer + 1;
      const double prev = err[k];
      err[k] = std::sqrt(h_rr[k]);
      if (!(err[k] == err[k]) || in[k].status == SOLVE_NAN) {
        out[k].status = SOLVE_NAN;
        active[k] = 0;
      } else if (converged(k)) {
        out[k].status = SOLVE_CONVERGED;
        active[k] = 0;
      } else if ((err[k] > 0.9 * prev && in[k].iterations > 0) || total[k] >= P.max_iter) {
        active[k] = 0;  // refinement stagnated, or the iteration budget is spent
      }
    }
  }
  for (int k = 0; k < K; ++k) {
    out[k].iterations = total[k];
    out[k].restarts = restarts[k];
    out[k].outer = outer_n[k];
    out[k].err_opt = err[k];
  }
  return 0;
}

void krylov_init_state(const SolveParams& P, KrylovState& init) {
  init = KrylovState{};
  init.tol_abs = P.tol_abs;
  init.tol_rel = P.tol_rel;
  init.max_iter = P.max_iter;
  init.max_restarts = P.max_restarts;
  init.stall_window = P.stall_window;
  init.eps = 1e-21;
}

// Runs BiCGSTAB on vectors of type T; x holds x0 on entry, x_opt on exit.
template <class T>
static int run_bicgstab(const DevMesh& M, const T* b, T* x, T* const v[9], const SolveParams& P, int zero_mean_row,
                        PoissonWork& W, SolveStats& out, cudaStream_t s, int* h_done,
                        const LocalMap* lmap = nullptr, const CoarseView* coarse = nullptr,
                        int sms = 148) {
  const bool f32 = sizeof(T) == 4;
  KrylovState init;
  krylov_init_state(P, init);
  const bool persistent = P.persistent;
  if (P.graph && !persistent) return set_error(CUP_ERR_STATE, "captured solves need the persistent solver");
  if (lmap && !persistent) return set_error(CUP_ERR_STATE, "the learned preconditioner needs the persistent solver");
  if (P.graph)
    CUP_CUDA_TRY(cudaMemcpyAsync(W.st, W.st_init, sizeof(init), cudaMemcpyDeviceToDevice, s));
  else
    CUP_CUDA_TRY(cudaMemcpyAsync(W.st, &init, sizeof(init), cudaMemcpyHostToDevice, s));
  KArgs<T> A = make_args<T>(M, b, x, v, W, W.st, P.mean_mode, zero_mean_row, 0);
  A.ncache = std::max(0, std::min(P.block_cache, KB_CACHE));
  if (coarse && coarse->nb > 0 && persistent) {  // the persistent solver adds it itself
    A.cnb = coarse->nb;
    A.cinv = coarse->inv;
    A.crc_v = coarse->rc;
    A.crc_r = coarse->rc2;
    A.cw = coarse->w;
  }
  if (lmap) {
    A.lw = lmap->w;
    A.llab = lmap->lab;
  }
  if (!persistent) {  // the persistent kernel prepares and initialises itself
    { ProfScope ps(f32 ? "bicg32_prepare" : "bicg_prepare", s); CUP_CUDA_TRY(launch_pdl<T>(k_bicg_prepare<T>, W.grid, s, A)); }
    { ProfScope ps(f32 ? "bicg32_init" : "bicg_init", s); CUP_CUDA_TRY(launch_pdl<T>(k_bicg_init<T>, W.ggrid, s, A)); }
  }
  CUP_CUDA_TRY(cudaGetLastError());
  if (persistent) {
    if (int rc = launch_persistent<T>(A, W, s, f32 ? "bicg32_persistent" : "bicg_persistent")) return rc;
    if (P.graph) return 0;  // the caller reads the state after the graph runs
    int h_err = 0;
    CUP_CUDA_TRY(cudaMemcpyAsync(&h_err, W.bar_error, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUP_CUDA_TRY(cudaStreamSynchronize(s));
    if (h_err) return set_error(CUP_ERR_CUDA, "persistent BiCGSTAB: a grid barrier wait timed out");
  }
  const int chunk = P.check_every > 0 ? P.check_every : 8;
  for (int it = 0; it < P.max_iter && !persistent; it += chunk) {
    for (int j = 0; j < chunk; ++j) {
      { ProfScope ps(f32 ? "bicg32_a_pupdate_precond" : "bicg_a_pupdate_precond", s); CUP_CUDA_TRY(launch_pdl<T>(k_bicg_a<T>, W.ggrid, s, A)); }
      if (coarse && coarse->nb > 0)
        if (int rc = coarse_apply<T>(*coarse, A.p, A.z1, &W.st->mean_sum, sms, s)) return rc;
      { ProfScope ps(f32 ? "bicg32_b_spmv_dot" : "bicg_b_spmv_dot", s); CUP_CUDA_TRY(launch_pdl<T>(k_bicg_b<T>, W.ggrid, s, A)); }
      { ProfScope ps(f32 ? "bicg32_c_supdate_precond" : "bicg_c_supdate_precond", s); CUP_CUDA_TRY(launch_pdl<T>(k_bicg_c<T>, W.ggrid, s, A)); }
      if (coarse && coarse->nb > 0)
        if (int rc = coarse_apply<T>(*coarse, A.r, A.z2, &W.st->mean_sum, sms, s)) return rc;
      { ProfScope ps(f32 ? "bicg32_d_spmv_dots" : "bicg_d_spmv_dots", s); CUP_CUDA_TRY(launch_pdl<T>(k_bicg_d<T>, W.ggrid, s, A)); }
      { ProfScope ps(f32 ? "bicg32_e_xr_update_dots" : "bicg_e_xr_update_dots", s); CUP_CUDA_TRY(launch_pdl<T>(k_bicg_e<T>, W.grid, s, A)); }
    }
    CUP_CUDA_TRY(cudaGetLastError());
    CUP_CUDA_TRY(cudaMemcpyAsync(h_done, &W.st->done, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUP_CUDA_TRY(cudaStreamSynchronize(s));
    if (*h_done) break;
  }
  KrylovState fin;
  CUP_CUDA_TRY(cudaMemcpyAsync(&fin, W.st, sizeof(fin), cudaMemcpyDeviceToHost, s));
  CUP_CUDA_TRY(cudaStreamSynchronize(s));
  if (fin.best != 0 && !persistent) {  // the persistent kernel moves it itself
    T* src = fin.best == 1 ? v[7] : v[8];
    CUP_CUDA_TRY(cudaMemcpyAsync(x, src, size_t(M.nb) * BN * sizeof(T), cudaMemcpyDeviceToDevice, s));
  }
  out.iterations = fin.k;
  out.restarts = fin.restarts;
  out.status = fin.done ? fin.status : SOLVE_MAXITER;
  out.err_init = fin.err_init;
  out.err_opt = fin.err_opt;
  return 0;
}

int poisson_bicgstab(const DevMesh& M, const double* b, double* x, const SolveParams& P,
                     PoissonWork& W, SolveStats& out, cudaStream_t s, int* h_done, const LocalMap* lmap,
                     const CoarseView* coarse, int sms) {
  poisson_init_constants();
  double* const v[9] = {W.r, W.rhat, W.p, W.nu, W.t, W.z1, W.z2, W.xs[1], W.xs[2]};
  const int zmr = (P.mean_mode == 1 || P.mean_mode == 3) ? 1 : 0;
  return run_bicgstab<double>(M, b, x, v, P, zmr, W, out, s, h_done, lmap, coarse, sms);
}

// Mixed precision: FP64 iterative refinement around FP32 BiCGSTAB inner solves.
// Every outer step recomputes the true residual b - A x in FP64 (the
// convergence test is on it), solves A e = r with FP32 vectors (FP64 dots and
// scalars) to a relative tolerance tied to the remaining reduction, and adds e
// to x in FP64.
int poisson_mixed(const DevMesh& M, const double* b, double* x, const SolveParams& P, PoissonWork& W,
                  SolveStats& out, cudaStream_t s, int* h_done, const LocalMap* lmap, const CoarseView* coarse,
                  int sms) {
  poisson_init_constants();
  const int zmr = (P.mean_mode == 1 || P.mean_mode == 3) ? 1 : 0;
  const size_t n = size_t(M.nb) * BN;
  GridReduce g{W.partial, W.counters + 12};
  KrylovState* so = W.st2;
  float* const v[9] = {W.fr, W.frhat, W.fp, W.fnu, W.ft, W.fz1, W.fz2, W.fxs[1], W.fxs[2]};
  float* e = W.fxs[0];
  auto residual = [&](double* err) -> int {
    {
      ProfScope ps("refine_true_residual_fp64", s);
      k_true_residual<<<W.ggrid, NT, 0, s>>>(M, b, x, W.r32, P.mean_mode, zmr, so, g);
    }
    CUP_CUDA_TRY(cudaGetLastError());
    CUP_CUDA_TRY(cudaMemcpyAsync(err, &so->err, sizeof(double), cudaMemcpyDeviceToHost, s));
    CUP_CUDA_TRY(cudaStreamSynchronize(s));
    return 0;
  };
  {
    ProfScope ps("refine_update", s);
    k_refine_update<<<W.grid, NT, 0, s>>>(M, x, nullptr, zmr, so, g);
  }
  CUP_CUDA_TRY(cudaGetLastError());
  double err0 = 0, err = 0;
  if (int rc = residual(&err0)) return rc;
  err = err0;
  out = SolveStats{};
  out.err_init = err0;
  out.err_opt = err0;
  out.status = SOLVE_MAXITER;
  if (!(err0 == err0)) {
    out.status = SOLVE_NAN;
    return 0;
  }
  if (err0 <= P.tol_abs) {
    out.status = SOLVE_CONVERGED;
    return 0;
  }
  int inner_total = 0, restarts = 0;
  for (int outer = 0; outer < 40; ++outer) {
    if (err <= P.tol_abs || err / err0 <= P.tol_rel) {
      out.status = SOLVE_CONVERGED;
      break;
    }
    // reduce the residual by what remains to be done, within FP32 reach
    const double want = std::max(P.tol_abs, P.tol_rel * err0);
    SolveParams Q = P;
    Q.tol_abs = 0.0;
    Q.tol_rel = std::min(0.5, std::max(2e-5, 0.5 * want / err));
    Q.max_iter = std::max(1, P.max_iter - inner_total);
    CUP_CUDA_TRY(cudaMemsetAsync(e, 0, n * sizeof(float), s));
    SolveStats in{};
    if (int rc = run_bicgstab<float>(M, W.r32, e, v, Q, 0, W, in, s, h_done, lmap, coarse, sms)) return rc;
    inner_total += in.iterations;
    restarts += in.restarts;
    if (in.status == SOLVE_NAN) {
      out.status = SOLVE_NAN;
      break;
    }
    {
      ProfScope ps("refine_update", s);
      k_refine_update<<<W.grid, NT, 0, s>>>(M, x, e, 0, so, g);
    }
    CUP_CUDA_TRY(cudaGetLastError());
    const double prev = err;
    if (int rc = residual(&err)) return rc;
    out.err_opt = std::min(out.err_opt, err);
    if (!(err == err)) {
      out.status = SOLVE_NAN;
      break;
    }
    if (err > 0.9 * prev && in.iterations > 0 && !(err <= P.tol_abs || err / err0 <= P.tol_rel)) {
      out.status = SOLVE_MAXITER;  // refinement stagnated
      break;
    }
    if (inner_total >= P.max_iter) {
      if (err <= P.tol_abs || err / err0 <= P.tol_rel) out.status = SOLVE_CONVERGED;
      break;
    }
    out.outer = outer + 1;
  }
  if (err <= P.tol_abs || err / err0 <= P.tol_rel) out.status = SOLVE_CONVERGED;
  out.iterations = inner_total;
  out.restarts = restarts;
  out.err_opt = err;
  return 0;
}

// FP64 ||b - A x||_2 (mean row of b zeroed as the solvers do); result in *err_host.
int true_residual_norm(const DevMesh& M, const double* b, const double* x, int mean_mode, PoissonWork& W,
                       double* err_host, cudaStream_t s) {
  const int zmr = (mean_mode == 1 || mean_mode == 3) ? 1 : 0;
  GridReduce g{W.partial, W.counters + 13};
  KrylovState* so = W.st2;
  {
    ProfScope ps("true_residual_fp64", s);
    k_weighted_sum<<<W.grid, NT, 0, s>>>(M, x, g, nullptr, &so->mean_sum);
    k_true_residual<<<W.ggrid, NT, 0, s>>>(M, b, x, nullptr, mean_mode, zmr, so, g);
  }
  CUP_CUDA_TRY(cudaGetLastError());
  CUP_CUDA_TRY(cudaMemcpyAsync(err_host, &so->err, sizeof(double), cudaMemcpyDeviceToHost, s));
  CUP_CUDA_TRY(cudaStreamSynchronize(s));
  return 0;
}


// ---- pipelined BiCGSTAB (PoissonSolverAMR::solve, PoissonSolverAMR.cpp:13-358) --
// The reference's CPU solver: preconditioned pipelined BiCGSTAB (Cools and
// Vanroose) with the exact block inverse, an explicit residual replacement
// every 50 iterations, restarts on a serious breakdown of (r0, r) and the
// best iterate kept.  One cooperative launch: every iteration is two phases
// of the block groups and two grid barriers,
//   1: t = A what; phat, s, shat, z, q, qhat, y; zhat = M z; (q,y), (y,y)
//   2: v = A zhat; omega; x, r, rhat, w; what = M w; the six dot products,
// with the sums sum(v h^3) that the next SpMV's mean-constraint row needs in
// the same reductions.  Replacement iterations compute s, z, r and w from
// their definitions (six phases), as the reference does.
struct PState {
  double alpha, beta, omega, r0r_prev, norm, init_norm, min_norm, eps, tol_abs, tol_rel;
  double qy, yy, ms;  // last dots of phase 1, sum(v h^3) of the vector the next SpMV reads
  int k, restarts, max_restarts, max_iter, converged, done, status, best_pending, use_xopt;
};

struct PArgs {
  DevMesh M;
  const double* b;
  double* x;
  double *xopt, *r0, *r, *rhat, *w, *what, *t, *phat, *s, *shat, *z, *zhat, *v, *q, *qhat, *y;
  PState* st;
  int mean_mode, zero_mean_row, ncache;
};

__global__ void __launch_bounds__(PNT, 8 / PGROUPS) k_pbicg_persistent(PArgs A, GridSync Gs) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* inv_eig = reinterpret_cast<double*>(smem_raw);
  BlockInfo* cache = reinterpret_cast<BlockInfo*>(smem_raw + kSmemCache);
  GroupTile* tiles = reinterpret_cast<GroupTile*>(smem_raw + kSmemTiles);
  __shared__ double red[64];
  __shared__ PState S;
  __shared__ unsigned int epoch;
  const GroupIdx G;
  const DevMesh& M = A.M;
  GroupTile& tile = tiles[G.g];
  FdTile& ftile = reinterpret_cast<FdTile&>(tile);
  fd_fill_inverse_eigen(inv_eig, c_lam);
  for (int i = threadIdx.x; i < PGROUPS * KB_CACHE * 32; i += PNT) {
    const int e = i >> 5, g = e / KB_CACHE, k = e % KB_CACHE;
    const int slot = blockIdx.x * PGROUPS + g + k * gridDim.x * PGROUPS;
    if (k < A.ncache && slot < M.nb) fill_block_info(M, M.order ? M.order[slot] : slot, cache[e], i & 31);
  }
  if (threadIdx.x == 0) {
    S = *A.st;
    epoch = 0u;
  }
  __syncthreads();
  const double eps = S.eps;
  // y = A v for the group's column of block bi (ms = sum(v h^3))
  auto spmv = [&](const BlockInfo& bi, const double* vv, double ms, double out[8]) {
    double col[8];
    load_col(vv, bi.id, G, col);
    spmv_group(bi, VecAt<double>{vv}, col, ms, A.mean_mode, tile, G, out);
  };
  auto precond = [&](const BlockInfo& bi, double c[8]) { block_inverse_group(c, ftile, G, bi.h, inv_eig); };
  auto hsum = [&](const BlockInfo& bi, const double c[8]) {
    double s = 0.0;
#pragma unroll
    for (int zz = 0; zz < 8; ++zz) s += c[zz];
    return s * bi.h * bi.h * bi.h;
  };
  // the best iterate noted by the last reduction is x as it stands: copy it
  // before x changes again
  auto copy_best = [&](const BlockInfo& bi) {
    if (!S.best_pending) return;
    double c[8];
    load_col(A.x, bi.id, G, c);
    store_col(A.xopt, bi.id, G, c);
  };
  auto reduce = [&](auto& a) -> bool { return grid_allreduce(a, Gs, epoch, red); };
  auto sync_state = [&]() { __syncthreads(); };
  // w = A rhat, what = M w; (r0, r0), (r0, w), sum(what h^3): the scalars of a start or restart
  auto start_phase = [&]() -> bool {
    double a[3] = {0.0, 0.0, 0.0};
    PERSISTENT_BLOCKS(bi) {
      double w[8], r0[8];
      spmv(bi, A.rhat, S.ms, w);
      load_col(A.r0, bi.id, G, r0);
      store_col(A.w, bi.id, G, w);
#pragma unroll
      for (int zz = 0; zz < 8; ++zz) {
        a[0] += r0[zz] * r0[zz];
        a[1] += r0[zz] * w[zz];
      }
      precond(bi, w);
      store_col(A.what, bi.id, G, w);
      a[2] += hsum(bi, w);
    }
    if (!reduce(a)) return false;
    if (threadIdx.x == 0) {
      S.alpha = a[0] / (a[1] + eps);
      S.r0r_prev = a[0];
      S.beta = 0.0;
      S.omega = 0.0;
      S.ms = a[2];
    }
    sync_state();
    return true;
  };
  bool ok = true;
  // ---- start: sum(x h^3); r0 = r = b - A x, rhat = M r0; then start_phase
  {
    double a[1] = {0.0};
    PERSISTENT_BLOCKS(bi) {
      double c[8];
      load_col(A.x, bi.id, G, c);
      a[0] += hsum(bi, c);
    }
    ok = reduce(a);
    if (threadIdx.x == 0) S.ms = a[0];
    sync_state();
  }
  if (ok) {
    double a[1] = {0.0};
    PERSISTENT_BLOCKS(bi) {
      double ax[8], bc[8];
      spmv(bi, A.x, S.ms, ax);
      load_col(A.b, bi.id, G, bc);
      if (A.zero_mean_row && bi.mean && G.lane == 0) bc[0] = 0.0;
#pragma unroll
      for (int zz = 0; zz < 8; ++zz) bc[zz] -= ax[zz];
      store_col(A.r0, bi.id, G, bc);
      store_col(A.r, bi.id, G, bc);
      precond(bi, bc);
      store_col(A.rhat, bi.id, G, bc);
      a[0] += hsum(bi, bc);
    }
    ok = reduce(a);
    if (threadIdx.x == 0) S.ms = a[0];
    sync_state();
  }
  if (ok) {
    double a[1] = {0.0};  // (r0, r0) again for the initial norm
    ok = start_phase();
    if (ok && threadIdx.x == 0) {
      S.norm = S.init_norm = sqrt(S.r0r_prev);
      S.min_norm = 1e50;
      if (!(S.norm == S.norm)) {
        S.done = 1;
        S.status = SOLVE_NAN;
      }
    }
    (void)a;
    sync_state();
  }
  // ---- iterations
  while (ok && !S.done && S.k < S.max_iter) {
    const bool replace = S.k % 50 == 0;
    const double al = S.alpha, be = S.beta, om = S.omega;
    if (!replace) {
      // phase 1
      double a[3] = {0.0, 0.0, 0.0};
      PERSISTENT_BLOCKS(bi) {
        copy_best(bi);
        double t[8], z[8];
        spmv(bi, A.what, S.ms, t);
        const size_t o0 = size_t(bi.id) * BN + G.gy * 8 + G.gx;
#pragma unroll
        for (int zz = 0; zz < 8; ++zz) {
          const size_t o = o0 + zz * 64;
          const double rh = A.rhat[o], sho = A.shat[o], w = A.w[o];
          const double ph = rh + be * (A.phat[o] - om * sho);
          const double sv = w + be * (A.s[o] - om * A.z[o]);
          const double sh = A.what[o] + be * (sho - om * A.zhat[o]);
          const double zn = t[zz] + be * (A.z[o] - om * A.v[o]);
          const double q = A.r[o] - al * sv, qh = rh - al * sh, y = w - al * zn;
          A.t[o] = t[zz];
          A.phat[o] = ph;
          A.s[o] = sv;
          A.shat[o] = sh;
          A.z[o] = zn;
          A.q[o] = q;
          A.qhat[o] = qh;
          A.y[o] = y;
          z[zz] = zn;
          a[0] += q * y;
          a[1] += y * y;
        }
        precond(bi, z);
        store_col(A.zhat, bi.id, G, z);
        a[2] += hsum(bi, z);
      }
      if (!(ok = reduce(a))) break;
      if (threadIdx.x == 0) {
        S.qy = a[0];
        S.yy = a[1];
        S.ms = a[2];
        S.best_pending = 0;
      }
      sync_state();
      // phase 2
      const double omn = S.qy / (S.yy + eps);
      double d[7] = {0, 0, 0, 0, 0, 0, 0};
      PERSISTENT_BLOCKS(bi) {
        double v[8], w[8];
        spmv(bi, A.zhat, S.ms, v);
        const size_t o0 = size_t(bi.id) * BN + G.gy * 8 + G.gx;
#pragma unroll
        for (int zz = 0; zz < 8; ++zz) {
          const size_t o = o0 + zz * 64;
          const double qh = A.qhat[o], y = A.y[o], r0 = A.r0[o];
          const double x = A.x[o] + al * A.phat[o] + omn * qh;
          const double r = A.q[o] - omn * y;
          const double rh = qh - omn * (A.what[o] - al * A.zhat[o]);
          const double wn = y - omn * (A.t[o] - al * v[zz]);
          A.v[o] = v[zz];
          A.x[o] = x;
          A.r[o] = r;
          A.rhat[o] = rh;
          A.w[o] = wn;
          w[zz] = wn;
          d[0] += r0 * r;
          d[1] += r0 * wn;
          d[2] += r0 * A.s[o];
          d[3] += r0 * A.z[o];
          d[4] += r * r;
          d[5] += r0 * r0;
        }
        precond(bi, w);
        store_col(A.what, bi.id, G, w);
        d[6] += hsum(bi, w);
      }
      if (!(ok = reduce(d))) break;
      if (threadIdx.x == 0) {
        S.omega = omn;
        S.ms = d[6];
        for (int i = 0; i < 6; ++i) red[32 + i] = d[i];
      }
      sync_state();
    } else {
      // replacement iteration: phat; s = A phat, shat = M s; z = A shat, ...
      double a[1] = {0.0};
      PERSISTENT_BLOCKS(bi) {
        copy_best(bi);
        double ph[8], rh[8], sh[8];
        load_col(A.phat, bi.id, G, ph);
        load_col(A.rhat, bi.id, G, rh);
        load_col(A.shat, bi.id, G, sh);
#pragma unroll
        for (int zz = 0; zz < 8; ++zz) ph[zz] = rh[zz] + be * (ph[zz] - om * sh[zz]);
        store_col(A.phat, bi.id, G, ph);
        a[0] += hsum(bi, ph);
      }
      if (!(ok = reduce(a))) break;
      if (threadIdx.x == 0) {
        S.ms = a[0];
        S.best_pending = 0;
      }
      sync_state();
      a[0] = 0.0;
      PERSISTENT_BLOCKS(bi) {
        double s[8];
        spmv(bi, A.phat, S.ms, s);
        store_col(A.s, bi.id, G, s);
        precond(bi, s);
        store_col(A.shat, bi.id, G, s);
        a[0] += hsum(bi, s);
      }
      if (!(ok = reduce(a))) break;
      if (threadIdx.x == 0) S.ms = a[0];
      sync_state();
      double b3[3] = {0.0, 0.0, 0.0};
      PERSISTENT_BLOCKS(bi) {
        double z[8], r[8], s[8], rh[8], sh[8], w[8];
        spmv(bi, A.shat, S.ms, z);
        store_col(A.z, bi.id, G, z);
        load_col(A.r, bi.id, G, r);
        load_col(A.s, bi.id, G, s);
        load_col(A.rhat, bi.id, G, rh);
        load_col(A.shat, bi.id, G, sh);
        load_col(A.w, bi.id, G, w);
        double q[8], qh[8], y[8];
#pragma unroll
        for (int zz = 0; zz < 8; ++zz) {
          q[zz] = r[zz] - al * s[zz];
          qh[zz] = rh[zz] - al * sh[zz];
          y[zz] = w[zz] - al * z[zz];
          b3[0] += q[zz] * y[zz];
          b3[1] += y[zz] * y[zz];
        }
        store_col(A.q, bi.id, G, q);
        store_col(A.qhat, bi.id, G, qh);
        store_col(A.y, bi.id, G, y);
        precond(bi, z);
        store_col(A.zhat, bi.id, G, z);
        b3[2] += hsum(bi, z);
      }
      if (!(ok = reduce(b3))) break;
      if (threadIdx.x == 0) S.ms = b3[2];
      sync_state();
      const double omn = b3[0] / (b3[1] + eps);
      a[0] = 0.0;
      PERSISTENT_BLOCKS(bi) {
        double v[8], x[8], ph[8], qh[8];
        spmv(bi, A.zhat, S.ms, v);
        store_col(A.v, bi.id, G, v);
        load_col(A.x, bi.id, G, x);
        load_col(A.phat, bi.id, G, ph);
        load_col(A.qhat, bi.id, G, qh);
#pragma unroll
        for (int zz = 0; zz < 8; ++zz) x[zz] = x[zz] + al * ph[zz] + omn * qh[zz];
        store_col(A.x, bi.id, G, x);
        a[0] += hsum(bi, x);
      }
      if (!(ok = reduce(a))) break;
      if (threadIdx.x == 0) S.ms = a[0];
      sync_state();
      a[0] = 0.0;
      PERSISTENT_BLOCKS(bi) {  // r = b - A x, rhat = M r
        double ax[8], bc[8];
        spmv(bi, A.x, S.ms, ax);
        load_col(A.b, bi.id, G, bc);
        if (A.zero_mean_row && bi.mean && G.lane == 0) bc[0] = 0.0;
#pragma unroll
        for (int zz = 0; zz < 8; ++zz) bc[zz] -= ax[zz];
        store_col(A.r, bi.id, G, bc);
        precond(bi, bc);
        store_col(A.rhat, bi.id, G, bc);
        a[0] += hsum(bi, bc);
      }
      if (!(ok = reduce(a))) break;
      if (threadIdx.x == 0) S.ms = a[0];
      sync_state();
      double d[7] = {0, 0, 0, 0, 0, 0, 0};
      PERSISTENT_BLOCKS(bi) {  // w = A rhat, what = M w; the dots
        double w[8], r0[8], r[8], s[8], z[8];
        spmv(bi, A.rhat, S.ms, w);
        store_col(A.w, bi.id, G, w);
        load_col(A.r0, bi.id, G, r0);
        load_col(A.r, bi.id, G, r);
        load_col(A.s, bi.id, G, s);
        load_col(A.z, bi.id, G, z);
#pragma unroll
        for (int zz = 0; zz < 8; ++zz) {
          d[0] += r0[zz] * r[zz];
          d[1] += r0[zz] * w[zz];
          d[2] += r0[zz] * s[zz];
          d[3] += r0[zz] * z[zz];
          d[4] += r[zz] * r[zz];
          d[5] += r0[zz] * r0[zz];
        }
        precond(bi, w);
        store_col(A.what, bi.id, G, w);
        d[6] += hsum(bi, w);
      }
      if (!(ok = reduce(d))) break;
      if (threadIdx.x == 0) {
        S.omega = omn;
        S.ms = d[6];
        for (int i = 0; i < 6; ++i) red[32 + i] = d[i];
      }
      sync_state();
    }
    // scalars, restart, best iterate, stopping test (every CTA, its own copy)
    if (threadIdx.x == 0) {
      const double r0r = red[32], r0w = red[33], r0s = red[34], r0z = red[35], n1 = red[36], n2 = red[37];
      const double omn = S.omega;
      S.norm = sqrt(n1);
      S.beta = S.alpha / (omn + eps) * r0r / (S.r0r_prev + eps);
      double alpha = r0r / (r0w + S.beta * r0s - S.beta * omn * r0z);
      double alphat = 1.0 / (omn + eps) + r0w / (r0r + eps) - S.beta * omn * r0z / (r0r + eps);
      alphat = 1.0 / (alphat + eps);
      if (fabs(alphat) < 10 * fabs(alpha)) alpha = alphat;
      S.alpha = alpha;
      S.r0r_prev = r0r;
      S.best_pending = 0;
      // restart on a serious breakdown (decided here, done below by all threads)
      S.status = (r0r * r0r < 1e-16 * n1 * n2 && S.restarts < S.max_restarts) ? -1 : S.status;
      if (S.norm < S.min_norm) {
        S.use_xopt = 1;
        S.min_norm = S.norm;
        S.best_pending = 1;
      }
      if (!(S.norm == S.norm)) {
        S.done = 1;
        S.status = SOLVE_NAN;
      } else if (S.norm < S.tol_abs || S.norm / (S.init_norm + eps) < S.tol_rel) {
        S.done = 1;
        S.converged = 1;
        S.status = SOLVE_CONVERGED;
      }
      S.k += 1;
    }
    sync_state();
    // every thread reads the decision before thread 0 changes the state
    const bool do_restart = S.status == -1 && !S.done;
    const bool restart_at_end = S.status == -1 && S.done;
    sync_state();
    if (do_restart) {  // r0 = r; rhat = M r0; then as at the start
      if (threadIdx.x == 0) {
        S.status = SOLVE_RUNNING;
        S.restarts += 1;
      }
      double a[1] = {0.0};
      PERSISTENT_BLOCKS(bi) {
        copy_best(bi);
        double r[8];
        load_col(A.r, bi.id, G, r);
        store_col(A.r0, bi.id, G, r);
        precond(bi, r);
        store_col(A.rhat, bi.id, G, r);
        a[0] += hsum(bi, r);
      }
      if (!(ok = reduce(a))) break;
      if (threadIdx.x == 0) {
        S.ms = a[0];
        S.best_pending = 0;
      }
      sync_state();
      if (!(ok = start_phase())) break;
    } else if (restart_at_end && threadIdx.x == 0) {
      S.status = SOLVE_CONVERGED;
    }
    sync_state();
  }
  // the best iterate into x: x itself when the last reduction found it best
  if (ok && S.use_xopt && !S.best_pending)
    PERSISTENT_BLOCKS(bi) {
      double c[8];
      load_col(A.xopt, bi.id, G, c);
      store_col(A.x, bi.id, G, c);
    }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (!ok) {
      S.done = 1;
      S.status = SOLVE_BARRIER_TIMEOUT;
    } else if (!S.done) {
      S.status = SOLVE_MAXITER;
    }
    *A.st = S;
  }
}

int poisson_pipelined(const DevMesh& M, const double* b, double* x, const SolveParams& P, PoissonWork& W,
                      double* const vec[16], SolveStats& out, cudaStream_t s) {
  poisson_init_constants();
  PState init{};
  init.eps = 1e-100;
  init.tol_abs = P.tol_abs;
  init.tol_rel = P.tol_rel;
  init.max_iter = P.max_iter;
  init.max_restarts = 100;
  init.status = SOLVE_RUNNING;
  PState* st = reinterpret_cast<PState*>(W.st2);  // the refinement state's slot: unused by this solver
  static_assert(sizeof(PState) <= sizeof(KrylovState), "PState fits the state slot");
  CUP_CUDA_TRY(cudaMemcpyAsync(st, &init, sizeof(init), cudaMemcpyHostToDevice, s));
  PArgs A{};
  A.M = M;
  A.b = b;
  A.x = x;
  double** dst[16] = {&A.xopt, &A.r0, &A.r, &A.rhat, &A.w, &A.what, &A.t, &A.phat,
                      &A.s, &A.shat, &A.z, &A.zhat, &A.v, &A.q, &A.qhat, &A.y};
  for (int i = 0; i < 16; ++i) *dst[i] = vec[i];
  const size_t n = size_t(M.nb) * BN;
  // the recurrences read phat, shat, s, z, zhat and v of "iteration -1": zero
  for (int i = 7; i < 13; ++i) CUP_CUDA_TRY(cudaMemsetAsync(vec[i], 0, n * sizeof(double), s));
  A.st = st;
  A.mean_mode = P.mean_mode;
  A.zero_mean_row = (P.mean_mode == 1 || P.mean_mode == 3) ? 1 : 0;
  A.ncache = std::max(0, std::min(P.block_cache, KB_CACHE));
  void (*kern)(PArgs, GridSync) = k_pbicg_persistent;
  const size_t dyn = kPersistentSmem;
  static unsigned long long attr = 0;
  if (first_on_device(attr))
    CUP_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn)));
  int per_sm = 0, dev = 0, sms = 0;
  CUP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, PNT, dyn));
  CUP_CUDA_TRY(cudaGetDevice(&dev));
  CUP_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (per_sm < 1) return set_error(CUP_ERR_CUDA, "pipelined BiCGSTAB: kernel does not fit on an SM");
  const int grid = std::max(1, std::min({per_sm * sms, (M.nb + PGROUPS - 1) / PGROUPS, std::max(W.grid, W.ggrid) / 2}));
  CUP_CUDA_TRY(cudaMemsetAsync(W.bar, 0, sizeof(unsigned int), s));
  CUP_CUDA_TRY(cudaMemsetAsync(W.bar_error, 0, sizeof(int), s));
  GridSync Gs{W.bar, W.partial, W.bar_error, W.barrier_cycles > 0 ? W.barrier_cycles : kBarrierClockLimit};
  void* args[] = {(void*)&A, (void*)&Gs};
  {
    ProfScope ps("pbicg_persistent", s);
    CUP_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3(PNT), args, dyn, s));
  }
  PState fin{};
  CUP_CUDA_TRY(cudaMemcpyAsync(&fin, st, sizeof(fin), cudaMemcpyDeviceToHost, s));
  CUP_CUDA_TRY(cudaStreamSynchronize(s));
  if (fin.status == SOLVE_BARRIER_TIMEOUT) return set_error(CUP_ERR_CUDA, "pipelined BiCGSTAB: a grid barrier wait timed out");
  out.iterations = fin.k;
  out.restarts = fin.restarts;
  out.status = fin.status;
  out.err_init = fin.init_norm;
  out.err_opt = fin.min_norm < 1e49 ? fin.min_norm : fin.init_norm;
  return 0;
}

}  // namespace cup3d
