// Obstacle creation on the device: the fill rule, signed distances and chi of
// obstacles.cpp (Sphere.cpp:47-51, the ellipsoid distance of Ellipsoid.cpp:22-300
// in ellipsoid_distance.cuh, and the Towers
// smoothed Heaviside of KernelCharacteristicFunction, ObstaclesCreate.cpp:45-80)
// as kernels, for bodies that are re-created without a host round trip of
// their blocks.
//
// This file is compiled without fused multiply-adds (--fmad=false) and states
// every expression in the host code's order, so the slot list, chi and the
// grid chi equal the host creation's bit for bit (IEEE division and square
// root on both sides).  The chi moments (mass and centre of mass) are summed
// per block in a fixed tree and then over the slots in slot order, so they
// match the host's sequential sums to rounding.
//
// Kernels, one launch each:
//   k_obst_slots  one CTA: bounding-box test per block, slots in block order
//                 (a CTA-wide scan of per-thread counts), the count;
//   k_obst_near   per block: the block or a face neighbour holds a slot;
//   k_obst_chi    one CTA per block: 10^3 signed-distance lab in shared
//                 memory, chi and udef = 0 of its slot, grid chi (0 outside
//                 the body's blocks), the block's four moments;
//   k_obst_kin    one CTA: moments over the slots -> centre of mass, kinematics.
#include <algorithm>
#include <cmath>
#include <vector>

#include "context.h"
#include "obstacles.h"
#include "ellipsoid_distance.cuh"

namespace cup3d {
namespace {

constexpr double kEpsD = 2.220446049250313e-16;  // DBL_EPSILON (the host code's numeric_limits epsilon)

struct Shape {
  int kind;          // 0 sphere, 1 ellipsoid
  double c[3];       // centre
  double r;          // sphere radius
  double ax[3];      // ellipsoid semi-axes
  double L[3][3];    // ellipsoid rotation, lab -> body
  double box[3][2];  // fill box of the body, margin included (sphere_fill_box, ellipsoid_fill_box)
  double vel[3], omega[3];
};

// Result record read back by the host: slot count, mass, kinematics.
struct ObstResult {
  int nslots;
  int pad_;
  double mass;
  double kin[9];
};

__device__ double shape_sdf(const Shape& s, double px, double py, double pz) {
  if (s.kind == 0) {
    const double dx = px - s.c[0], dy = py - s.c[1], dz = pz - s.c[2];
    return s.r - sqrt(dx * dx + dy * dy + dz * dz);
  }
  const double p[3] = {px - s.c[0], py - s.c[1], pz - s.c[2]};
  return ellipsoid_signed_distance(s.ax, s.L, p);
}

__device__ __forceinline__ bool block_touches(const Shape& s, const double* origin, double h, int b) {
  bool touch = true;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double lo = origin[3 * b + d] + 0.5 * h, hi = origin[3 * b + d] + (8 - 0.5) * h;
    const double a = lo < s.box[d][0] ? s.box[d][0] : lo;  // std::max(lo, box lo)
    const double c = s.box[d][1] < hi ? s.box[d][1] : hi;  // std::min(hi, box hi)
    touch &= c - a > 0;
  }
  return touch;
}

constexpr int SLOT_THREADS = 1024;

__global__ void __launch_bounds__(SLOT_THREADS) k_obst_slots(int nb, const double* __restrict__ h,
                                                             const double* __restrict__ origin, Shape s,
                                                             int* __restrict__ slot_of_block,
                                                             int* __restrict__ block_of_slot, ObstResult* res) {
  __shared__ int part[SLOT_THREADS];
  const int t = threadIdx.x;
  const int chunk = (nb + SLOT_THREADS - 1) / SLOT_THREADS;
  const int b0 = min(nb, t * chunk), b1 = min(nb, b0 + chunk);
  int cnt = 0;
  for (int b = b0; b < b1; ++b) cnt += block_touches(s, origin, h[b], b) ? 1 : 0;
  part[t] = cnt;
  __syncthreads();
  // inclusive scan (Hillis-Steele) of the per-thread counts
  for (int off = 1; off < SLOT_THREADS; off <<= 1) {
    const int v = t >= off ? part[t - off] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int slot = part[t] - cnt;
  for (int b = b0; b < b1; ++b) {
    if (block_touches(s, origin, h[b], b)) {
      slot_of_block[b] = slot;
      block_of_slot[slot] = b;
      ++slot;
    } else {
      slot_of_block[b] = -1;
    }
  }
  if (t == SLOT_THREADS - 1) res->nslots = part[t];
}

__global__ void k_obst_near(DevMesh M, const int* __restrict__ slot_of_block, int* __restrict__ near) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < M.nb; b += gridDim.x * blockDim.x) {
    bool nr = slot_of_block[b] >= 0;
    for (int f = 0; f < 6 && !nr; ++f) {
      const int k = M.fkind[6 * b + f];
      const int* nbr = M.fnbr + 24 * b + 4 * f;
      if (k == K_SAME || k == K_COARSER) nr |= slot_of_block[nbr[0]] >= 0;
      if (k == K_FINER)
        for (int q = 0; q < 4; ++q) nr |= slot_of_block[nbr[q]] >= 0;
    }
    near[b] = nr ? 1 : 0;
  }
}

// Sum of v over the 512 threads of the CTA in a fixed order (warp shuffles,
// then the 16 warp sums in order).
__device__ __forceinline__ double cta_sum512(double v, double* sm) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < 16; ++w) s += sm[w];
  __syncthreads();
  return s;
}

// Block b's part of the body: its signed-distance lab, chi and udef = 0 of
// its slot, the grid chi, the block's four moments (one CTA of 512 threads;
// ns: the slot count, udef is component-major [3][ns][512]).
__device__ __forceinline__ void obst_chi_block(int b, const double* __restrict__ h_, const double* __restrict__ origin,
                                               const Shape& s, int slot, size_t ns, double* __restrict__ chi,
                                               double* __restrict__ udef, double* __restrict__ grid_chi,
                                               double* __restrict__ mom) {
  const int t = threadIdx.x;
  if (slot < 0) {
    grid_chi[size_t(b) * BN + t] = 0.0;
    return;
  }
  __shared__ double lab[10][10][10];
  __shared__ double sm[16];
  __shared__ double s_far;
  const double h = h_[b];
  const double ox = origin[3 * b], oy = origin[3 * b + 1], oz = origin[3 * b + 2];
  // A block whose cells all lie more than one cell from the surface has chi
  // 1 (inside) or 0 (outside) in every cell, which is what the lab below
  // would give them: the signed distance is an exact distance (sphere, and
  // the ellipsoid's closest-point solve), so no cell's value is farther than
  // its distance to the block centre (at most 3.5 sqrt(3) h) from the
  // centre's value.  Such blocks skip the lab (1e-6 h of margin for rounding).
  if (t == 0) {
    const double sc = shape_sdf(s, ox + 4.0 * h, oy + 4.0 * h, oz + 4.0 * h);
    const double reach = 3.5 * 1.7320508075688772 * h + 1e-6 * h;
    s_far = sc - reach > h ? 1.0 : (sc + reach < -h ? 0.0 : -1.0);
  }
  __syncthreads();
  const bool far = s_far >= 0.0;
  if (!far) {
    for (int i = t; i < 1000; i += BN) {
      const int x = i % 10 - 1, y = (i / 10) % 10 - 1, z = i / 100 - 1;
      lab[z + 1][y + 1][x + 1] = shape_sdf(s, ox + (x + 0.5) * h, oy + (y + 0.5) * h, oz + (z + 0.5) * h);
    }
    __syncthreads();
  }
  const int x = t & 7, y = (t >> 3) & 7, z = t >> 6;
  const double inv2h = 0.5 / h, vol = h * h * h;
  const double s0 = far ? 0.0 : lab[z + 1][y + 1][x + 1];
  double c;
  if (far) {
    c = s_far;
  } else if (s0 > h || s0 < -h) {
    c = s0 > 0 ? 1 : 0;
  } else {
    const double dPx = lab[z + 1][y + 1][x + 2], dMx = lab[z + 1][y + 1][x];
    const double dPy = lab[z + 1][y + 2][x + 1], dMy = lab[z + 1][y][x + 1];
    const double dPz = lab[z + 2][y + 1][x + 1], dMz = lab[z][y + 1][x + 1];
    const double gUX = inv2h * (dPx - dMx), gUY = inv2h * (dPy - dMy), gUZ = inv2h * (dPz - dMz);
    const double gUSq = gUX * gUX + gUY * gUY + gUZ * gUZ + kEpsD;
    const double gIX = inv2h * ((0.0 < dPx ? dPx : 0.0) - (0.0 < dMx ? dMx : 0.0));
    const double gIY = inv2h * ((0.0 < dPy ? dPy : 0.0) - (0.0 < dMy ? dMy : 0.0));
    const double gIZ = inv2h * ((0.0 < dPz ? dPz : 0.0) - (0.0 < dMz ? dMz : 0.0));
    c = (gIX * gUX + gIY * gUY + gIZ * gUZ) / gUSq;
  }
  chi[size_t(slot) * BN + t] = c;
  for (int d = 0; d < 3; ++d) udef[(d * ns + slot) * BN + t] = 0.0;
  grid_chi[size_t(b) * BN + t] = 0.0 < c ? c : 0.0;  // std::max(0, chi)
  const double px = ox + (x + 0.5) * h, py = oy + (y + 0.5) * h, pz = oz + (z + 0.5) * h;
  const double cv = c * vol;
  const double m0 = cta_sum512(cv * px, sm), m1 = cta_sum512(cv * py, sm), m2 = cta_sum512(cv * pz, sm),
               m3 = cta_sum512(cv, sm);
  if (t == 0) {
    mom[4 * slot + 0] = m0;
    mom[4 * slot + 1] = m1;
    mom[4 * slot + 2] = m2;
    mom[4 * slot + 3] = m3;
  }
}

__global__ void __launch_bounds__(BN) k_obst_chi(const double* __restrict__ h_, const double* __restrict__ origin,
                                                  Shape s, const int* __restrict__ slot_of_block,
                                                  double* __restrict__ chi, double* __restrict__ udef,
                                                  double* __restrict__ grid_chi, double* __restrict__ mom,
                                                  const ObstResult* res) {
  const int b = blockIdx.x;
  obst_chi_block(b, h_, origin, s, slot_of_block[b], size_t(res->nslots), chi, udef, grid_chi, mom);
}

__global__ void __launch_bounds__(BN) k_obst_kin(const double* __restrict__ mom, Shape s, ObstResult* res,
                                                  double* __restrict__ kin_out) {
  __shared__ double sm[16];
  const int n = res->nslots;
  double a[4] = {0, 0, 0, 0};
  for (int i = threadIdx.x; i < n; i += BN)
#pragma unroll
    for (int k = 0; k < 4; ++k) a[k] += mom[4 * i + k];
  double tot[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) tot[k] = cta_sum512(a[k], sm);
  if (threadIdx.x == 0) {
    res->mass = tot[3];
    for (int d = 0; d < 3; ++d) {
      res->kin[d] = tot[3] > 0 ? tot[d] / tot[3] : 0.0;
      res->kin[3 + d] = s.vel[d];
      res->kin[6 + d] = s.omega[d];
    }
    for (int i = 0; i < 9; ++i) kin_out[i] = res->kin[i];
  }
}

// ---- moving bodies in a batch of cases -----------------------------------
// Every case's body created again on the flattened mesh in one pass: the
// slots of all cases in block order (case k's slots follow case k-1's, and
// slot_first[k] is the slot count before the case's first block), each
// block's chi from its case's shape by the single-case arithmetic, and per
// case the kinematics from its own slots' moments in the single-case order.

__global__ void __launch_bounds__(SLOT_THREADS) k_obst_slots_batch(
    int nb, const double* __restrict__ h, const double* __restrict__ origin, const Shape* __restrict__ shapes,
    const int* __restrict__ bcase, const int* __restrict__ first, int ncase, int* __restrict__ slot_of_block,
    int* __restrict__ block_of_slot, int* __restrict__ slot_first, ObstResult* res) {
  __shared__ int part[SLOT_THREADS];
  const int t = threadIdx.x;
  const int chunk = (nb + SLOT_THREADS - 1) / SLOT_THREADS;
  const int b0 = min(nb, t * chunk), b1 = min(nb, b0 + chunk);
  int cnt = 0;
  for (int b = b0; b < b1; ++b) cnt += block_touches(shapes[bcase[b]], origin, h[b], b) ? 1 : 0;
  part[t] = cnt;
  __syncthreads();
  for (int off = 1; off < SLOT_THREADS; off <<= 1) {
    const int v = t >= off ? part[t - off] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int slot = part[t] - cnt;
  for (int b = b0; b < b1; ++b) {
    const int k = bcase[b];
    if (b == first[k]) slot_first[k] = slot;
    if (block_touches(shapes[k], origin, h[b], b)) {
      slot_of_block[b] = slot;
      block_of_slot[slot] = b;
      ++slot;
    } else {
      slot_of_block[b] = -1;
    }
  }
  if (t == SLOT_THREADS - 1) {
    res->nslots = part[t];
    slot_first[ncase] = part[t];
  }
}

__global__ void __launch_bounds__(BN) k_obst_chi_batch(const double* __restrict__ h_, const double* __restrict__ origin,
                                                        const Shape* __restrict__ shapes, const int* __restrict__ bcase,
                                                        const int* __restrict__ slot_of_block, double* __restrict__ chi,
                                                        double* __restrict__ udef, double* __restrict__ grid_chi,
                                                        double* __restrict__ mom, const ObstResult* res) {
  const int b = blockIdx.x;
  const Shape s = shapes[bcase[b]];
  obst_chi_block(b, h_, origin, s, slot_of_block[b], size_t(res->nslots), chi, udef, grid_chi, mom);
}

// One CTA per case: its centre of mass from its slots' moments, and its
// velocities, as k_obst_kin does for one body (kin_out: 9 per case).
__global__ void __launch_bounds__(BN) k_obst_kin_batch(const double* __restrict__ mom, const Shape* __restrict__ shapes,
                                                        const int* __restrict__ slot_first,
                                                        double* __restrict__ kin_out) {
  __shared__ double sm[16];
  const int k = blockIdx.x;
  const int s0 = slot_first[k], n = slot_first[k + 1] - s0;
  double a[4] = {0, 0, 0, 0};
  for (int i = threadIdx.x; i < n; i += BN)
#pragma unroll
    for (int q = 0; q < 4; ++q) a[q] += mom[4 * (s0 + i) + q];
  double tot[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) tot[q] = cta_sum512(a[q], sm);
  if (threadIdx.x == 0) {
    double* kn = kin_out + 9 * k;
    for (int d = 0; d < 3; ++d) {
      kn[d] = tot[3] > 0 ? tot[d] / tot[3] : 0.0;
      kn[3 + d] = shapes[k].vel[d];
      kn[6 + d] = shapes[k].omega[d];
    }
  }
}

// ---- UpdateObstacles ------------------------------------------------------
constexpr int kMomQ = 29;  // momentum integrals per slot (13 explicit + 16 implicit)

// Per slot s, the integrals of KernelIntegrateFluidMomenta
// (ObstaclesUpdate.cpp:25-126) over the cells with chi > 0, arms p taken from
// the centre of mass kin[0..2]:
//   q[0] V, q[1..3] momentum, q[4..6] angular momentum, q[7..12] J0..J5,
//   implicit penalization: q[13] penalM, q[14..16] sum pf p, q[17..22] the
//   pf-weighted J, q[23..25] sum pf (u - udef), q[26..28] sum pf p x (u - udef),
//   with pf = dv lambda dt X1 / (1 + X1 lambda dt), X1 = (chi > 0.5).
__global__ void __launch_bounds__(BN) k_obst_momenta(DevMesh M, const int* __restrict__ block_of_slot,
                                                      const double* __restrict__ chi,
                                                      const double* __restrict__ udef, int nslots,
                                                      const double* __restrict__ vel, const double* __restrict__ kin,
                                                      double lambdt, int implicit, double* __restrict__ qslot) {
  __shared__ double sm[16][kMomQ];
  const int s = blockIdx.x, t = threadIdx.x;
  const int b = block_of_slot[s];
  const size_t n = size_t(M.nb) * BN;
  double q[kMomQ];
#pragma unroll
  for (int k = 0; k < kMomQ; ++k) q[k] = 0.0;
  const double X = chi[size_t(s) * BN + t];
  if (X > 0) {
    const double h = M.h[b], dv = h * h * h;
    const int ix = t & 7, iy = (t >> 3) & 7, iz = t >> 6;
    const double p[3] = {(M.index[3 * b] * 8 + ix + 0.5) * h - kin[0], (M.index[3 * b + 1] * 8 + iy + 0.5) * h - kin[1],
                         (M.index[3 * b + 2] * 8 + iz + 0.5) * h - kin[2]};
    double u[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) u[d] = vel[d * n + size_t(b) * BN + t];
    const double Xdv = X * dv;
    q[0] = Xdv;
    q[1] = Xdv * u[0];
    q[2] = Xdv * u[1];
    q[3] = Xdv * u[2];
    q[4] = Xdv * (p[1] * u[2] - p[2] * u[1]);
    q[5] = Xdv * (p[2] * u[0] - p[0] * u[2]);
    q[6] = Xdv * (p[0] * u[1] - p[1] * u[0]);
    q[7] = Xdv * (p[1] * p[1] + p[2] * p[2]);
    q[8] = Xdv * (p[0] * p[0] + p[2] * p[2]);
    q[9] = Xdv * (p[0] * p[0] + p[1] * p[1]);
    q[10] = -Xdv * p[0] * p[1];
    q[11] = -Xdv * p[0] * p[2];
    q[12] = -Xdv * p[1] * p[2];
    if (implicit) {
      const double X1 = X > 0.5 ? 1.0 : 0.0;
      const double pf = dv * lambdt * X1 / (1 + X1 * lambdt);
      double du[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) du[d] = u[d] - udef[(d * size_t(nslots) + s) * BN + t];
      q[13] = pf;
      q[14] = pf * p[0];
      q[15] = pf * p[1];
      q[16] = pf * p[2];
      q[17] = pf * (p[1] * p[1] + p[2] * p[2]);
      q[18] = pf * (p[0] * p[0] + p[2] * p[2]);
      q[19] = pf * (p[0] * p[0] + p[1] * p[1]);
      q[20] = -pf * p[0] * p[1];
      q[21] = -pf * p[0] * p[2];
      q[22] = -pf * p[1] * p[2];
      q[23] = pf * du[0];
      q[24] = pf * du[1];
      q[25] = pf * du[2];
      q[26] = pf * (p[1] * du[2] - p[2] * du[1]);
      q[27] = pf * (p[2] * du[0] - p[0] * du[2]);
      q[28] = pf * (p[0] * du[1] - p[1] * du[0]);
    }
  }
  // fixed-order CTA sums: warp shuffles, then the 16 warp sums in order
#pragma unroll
  for (int k = 0; k < kMomQ; ++k) {
    double v = q[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((t & 31) == 0) sm[t >> 5][k] = v;
  }
  __syncthreads();
  if (t < kMomQ) {
    double v = 0.0;
    for (int w = 0; w < 16; ++w) v += sm[w][t];
    qslot[size_t(s) * kMomQ + t] = v;
  }
}

// Sums of the per-slot integrals in slot order (one thread per quantity).
__global__ void k_obst_momenta_sum(const double* __restrict__ qslot, int nslots, double* __restrict__ qsum) {
  const int k = threadIdx.x;
  if (k >= kMomQ) return;
  double v = 0.0;
  for (int s = 0; s < nslots; ++s) v += qslot[size_t(s) * kMomQ + k];
  qsum[k] = v;
}

// Solves A x = b (6x6, row-major) by LU decomposition with partial pivoting
// (the method of gsl_linalg_LU_decomp / LU_solve).  Returns false when a
// pivot is zero.
static bool lu_solve6(double A[36], double b[6], double x[6]) {
  for (int k = 0; k < 6; ++k) {
    int piv = k;
    for (int i = k + 1; i < 6; ++i)
      if (std::fabs(A[i * 6 + k]) > std::fabs(A[piv * 6 + k])) piv = i;
    if (A[piv * 6 + k] == 0.0) return false;
    if (piv != k) {
      for (int j = 0; j < 6; ++j) std::swap(A[k * 6 + j], A[piv * 6 + j]);
      std::swap(b[k], b[piv]);
    }
    for (int i = k + 1; i < 6; ++i) {
      const double f = A[i * 6 + k] / A[k * 6 + k];
      A[i * 6 + k] = f;
      for (int j = k + 1; j < 6; ++j) A[i * 6 + j] -= f * A[k * 6 + j];
      b[i] -= f * b[k];
    }
  }
  for (int i = 5; i >= 0; --i) {
    double v = b[i];
    for (int j = i + 1; j < 6; ++j) v -= A[i * 6 + j] * x[j];
    x[i] = v / A[i * 6 + i];
  }
  return true;
}

// Device buffers of a device-created obstacle, sized for every block of the
// mesh (the slot count is known only after k_obst_slots).
int obst_dev_buffers(cup_ctx* c) {
  DevObstacle& o = c->ob;
  const int nb = c->mesh.nb;
  if (o.dev_cap == nb) return 0;
  c->obst_arena.release();
  o = DevObstacle();
  DevArena& A = c->obst_arena;
  if (int rc = A.alloc(&o.slot_of_block, nb)) return rc;
  if (int rc = A.alloc(&o.near, nb)) return rc;
  if (int rc = A.alloc(&o.block_of_slot, nb)) return rc;
  if (int rc = A.alloc(&o.chi, size_t(nb) * BN)) return rc;
  if (int rc = A.alloc(&o.udef, 3 * size_t(nb) * BN)) return rc;
  if (int rc = A.alloc(&o.d_mom, 4 * size_t(nb))) return rc;
  if (int rc = A.alloc(&o.d_origin, 3 * size_t(nb))) return rc;
  ObstResult* r = nullptr;
  if (int rc = A.alloc(&r, 1)) return rc;
  o.d_result = r;
  CUP_CUDA_TRY(stream_h2d(c->stream, o.d_origin, c->mesh.origin.data(), 3 * size_t(nb) * sizeof(double)));
  o.dev_cap = nb;
  return 0;
}

int create_obstacle_dev(cup_ctx* c, Shape& s) {
  graph_reset(c);
  const Mesh& m = c->mesh;
  if (int rc = obst_dev_buffers(c)) return rc;
  DevObstacle& o = c->ob;
  ObstResult* res = static_cast<ObstResult*>(o.d_result);
  cudaStream_t st = c->stream;
  {
    ProfScope ps("obstacle_slots", st);
    k_obst_slots<<<1, SLOT_THREADS, 0, st>>>(m.nb, c->dm.h, o.d_origin, s, o.slot_of_block, o.block_of_slot, res);
  }
  {
    ProfScope ps("obstacle_near", st);
    k_obst_near<<<std::max(1, std::min((m.nb + 255) / 256, c->num_sms * 4)), 256, 0, st>>>(c->dm, o.slot_of_block,
                                                                                         o.near);
  }
  {
    ProfScope ps("obstacle_chi", st);
    k_obst_chi<<<m.nb, BN, 0, st>>>(c->dm.h, o.d_origin, s, o.slot_of_block, o.chi, o.udef, c->F.chi, o.d_mom, res);
  }
  {
    ProfScope ps("obstacle_kin", st);
    k_obst_kin<<<1, BN, 0, st>>>(o.d_mom, s, res, c->d_scalars + SC_KIN);
  }
  CUP_CUDA_TRY(cudaGetLastError());
  ObstResult h{};
  CUP_CUDA_TRY(stream_d2h(st, &h, res, sizeof(h)));
  o.nslots = h.nslots;
  for (int i = 0; i < 9; ++i) o.kin[i] = h.kin[i];
  o.host_stale = true;
  o.udef_zero = true;  // k_obst_chi writes udef = 0
  if (h.nslots == 0) {  // nothing of the body on the mesh: no obstacle
    c->obst_arena.release();
    c->ob = DevObstacle();
  }
  return 0;
}

int shape_args_ok(cup_ctx* c, const char* who) {
  if (!c || c->mesh.nb == 0 || c->host_only) return ctx_fail(c, CUP_ERR_ARG, std::string(who) + ": bad arguments");
  if (c->ncase > 1) return ctx_fail(c, CUP_ERR_STATE, std::string(who) + ": not available on a batch of cases");
  return 0;
}

void set_kinematics(Shape& s, const double* vel, const double* omega) {
  for (int d = 0; d < 3; ++d) {
    s.vel[d] = vel ? vel[d] : 0.0;
    s.omega[d] = omega ? omega[d] : 0.0;
  }
}

// ---- surface forces (ComputeForces, FluidSolidForces.cpp:14-229) ------------
// Surface points of an obstacle block (KernelCharacteristicFunction's second
// loop, ObstaclesCreate.cpp:83-117, and ObstacleBlock::write): cells where the
// gradient of the block's own chi (central inside, one-sided second order at
// the block's faces) is not zero and the smoothed delta
//   Delta = (h^2 / 2) grad(chi) . grad(sdf) / |grad(sdf)|^2
// exceeds machine epsilon; the point's normal is -Delta grad(sdf) (it carries
// h^3).  One CTA per slot; nrm is component-major [3][nslots][512], zero
// where a cell is no surface point.
__global__ void __launch_bounds__(BN) k_obst_surface(const double* __restrict__ h_, const double* __restrict__ origin,
                                                      Shape s, const int* __restrict__ block_of_slot,
                                                      const double* __restrict__ chi, int nslots,
                                                      double* __restrict__ nrm) {
  const int slot = blockIdx.x, t = threadIdx.x;
  const int b = block_of_slot[slot];
  __shared__ double lab[10][10][10];
  __shared__ double ch[8][8][8];
  const double h = h_[b];
  const double ox = origin[3 * b], oy = origin[3 * b + 1], oz = origin[3 * b + 2];
  for (int i = t; i < 1000; i += BN) {
    const int x = i % 10 - 1, y = (i / 10) % 10 - 1, z = i / 100 - 1;
    lab[z + 1][y + 1][x + 1] = shape_sdf(s, ox + (x + 0.5) * h, oy + (y + 0.5) * h, oz + (z + 0.5) * h);
  }
  const int x = t & 7, y = (t >> 3) & 7, z = t >> 6;
  ch[z][y][x] = chi[size_t(slot) * BN + t];
  __syncthreads();
  const double inv2h = 0.5 / h, fac1 = 0.5 * h * h;
  const double dPx = lab[z + 1][y + 1][x + 2], dMx = lab[z + 1][y + 1][x];
  const double dPy = lab[z + 1][y + 2][x + 1], dMy = lab[z + 1][y][x + 1];
  const double dPz = lab[z + 2][y + 1][x + 1], dMz = lab[z][y + 1][x + 1];
  const double gUX = inv2h * (dPx - dMx), gUY = inv2h * (dPy - dMy), gUZ = inv2h * (dPz - dMz);
  const double gUSq = gUX * gUX + gUY * gUY + gUZ * gUZ + kEpsD;
  // d/dx of chi along each axis: one-sided at the block's first and last cells
  auto grad = [&](int i, double m2, double m1, double c0, double p1, double p2) {
    return i == 0 ? 2.0 * (-0.5 * p2 + 2.0 * p1 - 1.5 * c0)
                  : (i == 7 ? 2.0 * (1.5 * c0 - 2.0 * m1 + 0.5 * m2) : (p1 - m1));
  };
  const double c0 = ch[z][y][x];
  const double gHX = grad(x, x > 1 ? ch[z][y][x - 2] : 0.0, x > 0 ? ch[z][y][x - 1] : 0.0, c0,
                          x < 7 ? ch[z][y][x + 1] : 0.0, x < 6 ? ch[z][y][x + 2] : 0.0);
  const double gHY = grad(y, y > 1 ? ch[z][y - 2][x] : 0.0, y > 0 ? ch[z][y - 1][x] : 0.0, c0,
                          y < 7 ? ch[z][y + 1][x] : 0.0, y < 6 ? ch[z][y + 2][x] : 0.0);
  const double gHZ = grad(z, z > 1 ? ch[z - 2][y][x] : 0.0, z > 0 ? ch[z - 1][y][x] : 0.0, c0,
                          z < 7 ? ch[z + 1][y][x] : 0.0, z < 6 ? ch[z + 2][y][x] : 0.0);
  double n3[3] = {0.0, 0.0, 0.0};
  if (!(gHX * gHX + gHY * gHY + gHZ * gHZ < 1e-12)) {
    const double numD = gHX * gUX + gHY * gUY + gHZ * gUZ;
    const double delta = fac1 * numD / gUSq;
    if (delta > kEpsD) {
      n3[0] = -delta * gUX;
      n3[1] = -delta * gUY;
      n3[2] = -delta * gUZ;
    }
  }
  for (int d = 0; d < 3; ++d) nrm[(size_t(d) * nslots + slot) * BN + t] = n3[d];
}

// Quantities summed over the surface points (Obstacle::computeForces order):
// surface force (3), pressure force (3), viscous force (3), torque (3), drag,
// thrust, Pout, PoutBnd, defPower, defPowerBnd, pLocom.
constexpr int kForceQ = 19;
constexpr int kFL = 16;  // force lab cells per side: -4 .. 11 around the block

struct ForceArgs {
  DevMesh M;
  const double* vel;  // [3][n]
  size_t n;
  const double* pres;
  const double* chi;  // grid chi
  const double* origin;
  const int* block_of_slot;
  const double* nrm;   // [3][nslots][512]
  const double* udef;  // [3][nslots][512]
  int nslots;
  double nu;
  double cm[3], utrans[3], omega[3];
  double* qslot;  // nslots * kForceQ
  int* err;       // set when a surface point's stencil leaves the same-level neighbourhood
};

// KernelComputeForces::visit for one slot (one CTA, one thread per cell): the
// velocity and chi labs over -4..11 from the block and its 26 neighbours at
// the same level (through face neighbours x, then y, then z; cells of a
// neighbour that is missing, coarser, finer or beyond a domain boundary are
// NaN, and a surface point whose stencil reads one sets *err and adds
// nothing), then the one-sided velocity gradients at the point moved along
// the normal into the fluid, the pressure and viscous tractions and the sums.
__global__ void __launch_bounds__(BN, 1) k_obst_forces(ForceArgs A) {
  extern __shared__ double fl[];  // [4][kFL^3]: u, v, w, chi
  __shared__ int nbr[27];
  __shared__ double red[BN / 32][kForceQ];
  const int slot = blockIdx.x, t = threadIdx.x;
  const int b = A.block_of_slot[slot];
  const DevMesh& M = A.M;
  if (t < 27) {
    const int off[3] = {t % 3 - 1, (t / 3) % 3 - 1, t / 9 - 1};
    int cur = b;
    for (int d = 0; d < 3 && cur >= 0; ++d) {
      if (off[d] == 0) continue;
      const int f = 2 * d + (off[d] > 0 ? 1 : 0);
      cur = M.fkind[6 * cur + f] == K_SAME ? M.fnbr[24 * cur + 4 * f] : -1;
    }
    nbr[t] = cur;
  }
  __syncthreads();
  constexpr int V = kFL * kFL * kFL;
  for (int i = t; i < V; i += BN) {
    const int x = i % kFL - 4, y = (i / kFL) % kFL - 4, z = i / (kFL * kFL) - 4;
    const int ox = x < 0 ? -1 : (x >= 8 ? 1 : 0), oy = y < 0 ? -1 : (y >= 8 ? 1 : 0),
              oz = z < 0 ? -1 : (z >= 8 ? 1 : 0);
    const int nb = nbr[(ox + 1) + 3 * (oy + 1) + 9 * (oz + 1)];
    const int cell = (x - 8 * ox) + 8 * (y - 8 * oy) + 64 * (z - 8 * oz);
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    for (int c = 0; c < 3; ++c) fl[c * V + i] = nb < 0 ? nan : A.vel[c * A.n + size_t(nb) * BN + cell];
    fl[3 * V + i] = nb < 0 ? nan : A.chi[size_t(nb) * BN + cell];
  }
  __syncthreads();
  auto at = [&](int c, int x, int y, int z) { return fl[c * V + (x + 4) + kFL * ((y + 4) + kFL * (z + 4))]; };
  auto inrange = [](int i) { return i >= -4 && i < 12; };
  double q[kForceQ];
  for (int k = 0; k < kForceQ; ++k) q[k] = 0.0;
  const int ix = t & 7, iy = (t >> 3) & 7, iz = t >> 6;
  const double normX = A.nrm[(0 * size_t(A.nslots) + slot) * BN + t];
  const double normY = A.nrm[(1 * size_t(A.nslots) + slot) * BN + t];
  const double normZ = A.nrm[(2 * size_t(A.nslots) + slot) * BN + t];
  if (normX != 0.0 || normY != 0.0 || normZ != 0.0) {
    const double h = M.h[b], _1oH = A.nu / h;
    const double p[3] = {A.origin[3 * b] + h * (ix + 0.5), A.origin[3 * b + 1] + h * (iy + 0.5),
                         A.origin[3 * b + 2] + h * (iz + 0.5)};
    const double norm = 1.0 / sqrt(normX * normX + normY * normY + normZ * normZ);
    const double dx = normX * norm, dy = normY * norm, dz = normZ * norm;
    // move up to four cells along the normal, out of the body
    int x = ix, y = iy, z = iz;
    for (int kk = 0; kk < 5; ++kk) {
      const int dxi = int(round(kk * dx)), dyi = int(round(kk * dy)), dzi = int(round(kk * dz));
      if (ix + dxi + 1 >= 12 || ix + dxi - 1 < -4) continue;
      if (iy + dyi + 1 >= 12 || iy + dyi - 1 < -4) continue;
      if (iz + dzi + 1 >= 12 || iz + dzi - 1 < -4) continue;
      x = ix + dxi;
      y = iy + dyi;
      z = iz + dzi;
      if (at(3, x, y, z) < 0.01) break;
    }
    const int sx = normX > 0 ? 1 : -1, sy = normY > 0 ? 1 : -1, sz = normZ > 0 ? 1 : -1;
    constexpr double c0 = -137. / 60., c1 = 5., c2 = -5., c3 = 10. / 3., c4 = -5. / 4., c5 = 1. / 5.;
    double g[3][3];  // g[c][d] = d u_c / d x_d at the point (ix, iy, iz)
    for (int c = 0; c < 3; ++c) {
      auto l = [&](int X, int Y, int Z) { return at(c, X, Y, Z); };
      // first derivatives at (x, y, z): sixth-order one-sided, else second, else first order
      auto d1 = [&](int d) {
        const int sd = d == 0 ? sx : (d == 1 ? sy : sz);
        const int e[3] = {d == 0, d == 1, d == 2};
        const int pd = d == 0 ? x : (d == 1 ? y : z);
        auto L = [&](int k) { return l(x + k * e[0], y + k * e[1], z + k * e[2]); };
        if (inrange(pd + 5 * sd))
          return sd * (c0 * L(0) + c1 * L(sd) + c2 * L(2 * sd) + c3 * L(3 * sd) + c4 * L(4 * sd) + c5 * L(5 * sd));
        if (inrange(pd + 2 * sd)) return sd * (-1.5 * L(0) + 2.0 * L(sd) - 0.5 * L(2 * sd));
        // the y branch of the reference multiplies by sx here (FluidSolidForces.cpp:127)
        return (d == 1 ? sx : sd) * (L(sd) - L(0));
      };
      const double dvx = d1(0), dvy = d1(1), dvz = d1(2);
      const double dxx = l(x - 1, y, z) - 2.0 * l(x, y, z) + l(x + 1, y, z);
      const double dyy = l(x, y - 1, z) - 2.0 * l(x, y, z) + l(x, y + 1, z);
      const double dzz = l(x, y, z - 1) - 2.0 * l(x, y, z) + l(x, y, z + 1);
      double dxy, dyz, dxz;
      if (inrange(x + 2 * sx) && inrange(y + 2 * sy))
        dxy = sx * sy *
              (-0.5 * (-1.5 * l(x + 2 * sx, y, z) + 2 * l(x + 2 * sx, y + sy, z) - 0.5 * l(x + 2 * sx, y + 2 * sy, z)) +
               2 * (-1.5 * l(x + sx, y, z) + 2 * l(x + sx, y + sy, z) - 0.5 * l(x + sx, y + 2 * sy, z)) -
               1.5 * (-1.5 * l(x, y, z) + 2 * l(x, y + sy, z) - 0.5 * l(x, y + 2 * sy, z)));
      else
        dxy = sx * sy * (l(x + sx, y + sy, z) - l(x + sx, y, z)) - (l(x, y + sy, z) - l(x, y, z));
      if (inrange(y + 2 * sy) && inrange(z + 2 * sz))
        dyz = sy * sz *
              (-0.5 * (-1.5 * l(x, y + 2 * sy, z) + 2 * l(x, y + 2 * sy, z + sz) - 0.5 * l(x, y + 2 * sy, z + 2 * sz)) +
               2 * (-1.5 * l(x, y + sy, z) + 2 * l(x, y + sy, z + sz) - 0.5 * l(x, y + sy, z + 2 * sz)) -
               1.5 * (-1.5 * l(x, y, z) + 2 * l(x, y, z + sz) - 0.5 * l(x, y, z + 2 * sz)));
      else
        dyz = sy * sz * (l(x, y + sy, z + sz) - l(x, y + sy, z)) - (l(x, y, z + sz) - l(x, y, z));
      if (inrange(x + 2 * sx) && inrange(z + 2 * sz))
        dxz = sx * sz *
              (-0.5 * (-1.5 * l(x, y, z + 2 * sz) + 2 * l(x + sx, y, z + 2 * sz) - 0.5 * l(x + 2 * sx, y, z + 2 * sz)) +
               2 * (-1.5 * l(x, y, z + sz) + 2 * l(x + sx, y, z + sz) - 0.5 * l(x + 2 * sx, y, z + sz)) -
               1.5 * (-1.5 * l(x, y, z) + 2 * l(x + sx, y, z) - 0.5 * l(x + 2 * sx, y, z)));
      else
        dxz = sx * sz * (l(x + sx, y, z + sz) - l(x, y, z + sz)) - (l(x + sx, y, z) - l(x, y, z));
      // Taylor back from (x, y, z) to the surface point
      g[c][0] = dvx + dxx * (ix - x) + dxy * (iy - y) + dxz * (iz - z);
      g[c][1] = dvy + dyy * (iy - y) + dyz * (iz - z) + dxy * (ix - x);
      g[c][2] = dvz + dzz * (iz - z) + dxz * (ix - x) + dyz * (iy - y);
    }
    const double P = A.pres[size_t(b) * BN + t];
    const double fXV = _1oH * (g[0][0] * normX + g[0][1] * normY + g[0][2] * normZ);
    const double fYV = _1oH * (g[1][0] * normX + g[1][1] * normY + g[1][2] * normZ);
    const double fZV = _1oH * (g[2][0] * normX + g[2][1] * normY + g[2][2] * normZ);
    const double fXP = -P * normX, fYP = -P * normY, fZP = -P * normZ;
    const double fXT = fXV + fXP, fYT = fYV + fYP, fZT = fZV + fZP;
    const double vX = at(0, ix, iy, iz), vY = at(1, ix, iy, iz), vZ = at(2, ix, iy, iz);
    const size_t ud = size_t(slot) * BN + t, us = size_t(A.nslots) * BN;
    const double uX = A.udef[ud], uY = A.udef[us + ud], uZ = A.udef[2 * us + ud];
    double velUnit[3] = {0.0, 0.0, 0.0};
    const double vn = sqrt(A.utrans[0] * A.utrans[0] + A.utrans[1] * A.utrans[1] + A.utrans[2] * A.utrans[2]);
    if (vn > 1e-9)
      for (int d = 0; d < 3; ++d) velUnit[d] = A.utrans[d] / vn;
    const double forcePar = fXT * velUnit[0] + fYT * velUnit[1] + fZT * velUnit[2];
    const double powOut = fXT * vX + fYT * vY + fZT * vZ;
    const double powDef = fXT * uX + fYT * uY + fZT * uZ;
    const double r[3] = {p[0] - A.cm[0], p[1] - A.cm[1], p[2] - A.cm[2]};
    const double uS[3] = {A.utrans[0] + A.omega[1] * r[2] - r[1] * A.omega[2],
                          A.utrans[1] + A.omega[2] * r[0] - r[2] * A.omega[0],
                          A.utrans[2] + A.omega[0] * r[1] - r[0] * A.omega[1]};
    const double v[kForceQ] = {fXT, fYT, fZT, fXP, fYP, fZP, fXV, fYV, fZV,
                               r[1] * fZT - r[2] * fYT, r[2] * fXT - r[0] * fZT, r[0] * fYT - r[1] * fXT,
                               -.5 * (forcePar - fabs(forcePar)), .5 * (forcePar + fabs(forcePar)), powOut,
                               fmin(0.0, powOut), powDef, fmin(0.0, powDef),
                               fXT * uS[0] + fYT * uS[1] + fZT * uS[2]};
    bool finite = true;
    for (int k = 0; k < kForceQ; ++k) finite &= isfinite(v[k]);
    if (finite)
      for (int k = 0; k < kForceQ; ++k) q[k] = v[k];
    else
      atomicExch(A.err, 1);
  }
  // CTA sums in a fixed order: warps, then the warps' partials
  for (int k = 0; k < kForceQ; ++k) {
    double a = q[k];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if ((t & 31) == 0) red[t >> 5][k] = a;
  }
  __syncthreads();
  if (t < kForceQ) {
    double a = 0.0;
    for (int w = 0; w < BN / 32; ++w) a += red[w][t];
    A.qslot[size_t(slot) * kForceQ + t] = a;
  }
}

}  // namespace

void body_record(cup_ctx* c, int kind, bool on_device, const double* ctr, const double* r, const double* q,
                 const double* vel, const double* omega) {
  BodyState& B = c->body;
  B = BodyState();
  B.kind = kind;
  B.on_device = on_device;
  for (int d = 0; d < 3; ++d) {
    B.pos[d] = B.old_pos[d] = B.abs_pos[d] = B.old_abs_pos[d] = ctr[d];
    B.vel[d] = vel ? vel[d] : 0.0;
    B.omega[d] = omega ? omega[d] : 0.0;
  }
  if (kind == 0) {
    B.r = r[0];
  } else {
    for (int d = 0; d < 3; ++d) B.ax[d] = r[d];
    for (int i = 0; i < 4; ++i) B.quat[i] = B.old_quat[i] = q[i];
  }
}

bool body_free(const cup_ctx* c) {
  const BodyState& B = c->body;
  if (B.kind < 0 || c->ob.nslots == 0) return false;
  for (int d = 0; d < 3; ++d)
    if (B.free_t[d] || B.free_r[d]) return true;
  return false;
}

int update_obstacles(cup_ctx* c, double dt, double out[12]) {
  DevObstacle& o = c->ob;
  if (o.nslots == 0 || c->host_only || c->body.kind < 0) return 0;  // no body, or raw obstacle data
  if (o.q_cap < o.nslots) {
    if (int rc = c->obst_arena.alloc(&o.d_qslot, size_t(o.nslots) * kMomQ)) return rc;
    if (int rc = c->obst_arena.alloc(&o.d_qsum, kMomQ)) return rc;
    o.q_cap = o.nslots;
  }
  const int implicit = c->cfg.implicit_penalization ? 1 : 0;
  cudaStream_t st = c->stream;
  {
    ProfScope ps("obstacle_momenta", st);
    k_obst_momenta<<<o.nslots, BN, 0, st>>>(c->dm, o.block_of_slot, o.chi, o.udef, o.nslots, c->F.vel[c->F.vcur],
                                            c->d_scalars + SC_KIN, c->cfg.lambda * dt, implicit, o.d_qslot);
    k_obst_momenta_sum<<<1, 32, 0, st>>>(o.d_qslot, o.nslots, o.d_qsum);
  }
  CUP_CUDA_TRY(cudaGetLastError());
  double Mq[kMomQ];
  CUP_CUDA_TRY(stream_d2h(st, Mq, o.d_qsum, sizeof(Mq)));
  // kernelFinalizeObstacleVel (ObstaclesUpdate.cpp:128-186)
  double penalM, penalCM[3], penalJ[6], lmom[3], amom[3];
  if (implicit) {
    penalM = Mq[13];
    for (int d = 0; d < 3; ++d) {
      penalCM[d] = Mq[14 + d];
      lmom[d] = Mq[23 + d];
      amom[d] = Mq[26 + d];
    }
    for (int i = 0; i < 6; ++i) penalJ[i] = Mq[17 + i];
  } else {
    penalM = Mq[0];
    for (int d = 0; d < 3; ++d) {
      penalCM[d] = 0.0;
      lmom[d] = Mq[1 + d];
      amom[d] = Mq[4 + d];
    }
    for (int i = 0; i < 6; ++i) penalJ[i] = Mq[7 + i];
  }
  // Obstacle::computeVelocities (Obstacle.cpp:143-269)
  BodyState& B = c->body;
  double A[36] = {penalM,      0.0,         0.0,         0.0,         +penalCM[2], -penalCM[1],
                  0.0,         penalM,      0.0,         -penalCM[2], 0.0,         +penalCM[0],
                  0.0,         0.0,         penalM,      +penalCM[1], -penalCM[0], 0.0,
                  0.0,         -penalCM[2], +penalCM[1], penalJ[0],   penalJ[3],   penalJ[4],
                  +penalCM[2], 0.0,         -penalCM[0], penalJ[3],   penalJ[1],   penalJ[5],
                  -penalCM[1], +penalCM[0], 0.0,         penalJ[4],   penalJ[5],   penalJ[2]};
  double rhs[6] = {lmom[0], lmom[1], lmom[2], amom[0], amom[1], amom[2]};
  for (int d = 0; d < 3; ++d) {
    if (!B.free_t[d]) {  // forced: the row keeps its diagonal, the velocity is imposed
      for (int j = 0; j < 6; ++j)
        if (j != d) A[d * 6 + j] = 0.0;
      rhs[d] = penalM * B.vel[d];
    }
    if (!B.free_r[d]) {  // rotation imposed (blocked rotation: omega = 0)
      const int r = 3 + d;
      for (int j = 0; j < 6; ++j)
        if (j != r) A[r * 6 + j] = 0.0;
      rhs[r] = A[r * 6 + r] * B.omega[d];
    }
  }
  double x[6];
  if (!lu_solve6(A, rhs, x)) return set_error(CUP_ERR_NAN, "UpdateObstacles: singular 6x6 momentum system");
  const double mass = Mq[0];
  const double J[6] = {Mq[7], Mq[8], Mq[9], Mq[10], Mq[11], Mq[12]};
  double force[3], torque[3], dAv[3];
  for (int d = 0; d < 3; ++d) {
    force[d] = mass * (x[d] - B.vel[d]) / dt;
    dAv[d] = (x[3 + d] - B.omega[d]) / dt;
  }
  torque[0] = J[0] * dAv[0] + J[3] * dAv[1] + J[4] * dAv[2];
  torque[1] = J[3] * dAv[0] + J[1] * dAv[1] + J[5] * dAv[2];
  torque[2] = J[4] * dAv[0] + J[5] * dAv[1] + J[2] * dAv[2];
  for (int d = 0; d < 3; ++d) {
    if (B.free_t[d]) B.vel[d] = x[d];
    if (B.free_r[d]) B.omega[d] = x[3 + d];
    o.kin[3 + d] = B.vel[d];
    o.kin[6 + d] = B.omega[d];
  }
  CUP_CUDA_TRY(stream_h2d(st, c->d_scalars + SC_KIN + 3, o.kin + 3, 6 * sizeof(double)));
  if (out) {
    for (int d = 0; d < 3; ++d) {
      out[d] = B.vel[d];
      out[3 + d] = B.omega[d];
      out[6 + d] = force[d];
      out[9 + d] = torque[d];
    }
  }
  return 0;
}

bool body_update_uinf(cup_ctx* c) {
  const BodyState& B = c->body;
  if (B.kind < 0 || c->ob.nslots == 0) return false;
  bool changed = false;
  for (int d = 0; d < 3; ++d)
    if (B.fix_frame[d] && c->cfg.uinf[d] != -B.vel[d]) {
      c->cfg.uinf[d] = -B.vel[d];
      changed = true;
    }
  return changed;
}

bool body_moves(const cup_ctx* c) {
  const BodyState& B = c->body;
  if (B.kind < 0 || c->cfg.static_obstacles || c->ob.nslots == 0) return false;
  if (body_free(c)) return true;
  for (int d = 0; d < 3; ++d)
    if (B.vel[d] + c->cfg.uinf[d] != 0.0 || B.omega[d] != 0.0) return true;
  return false;
}

void body_coef_u(cup_ctx* c, int step, double dt) {
  if (step > c->cfg.step_2nd_start && c->dt_prev > 0) {  // Simulation.cpp:361-370
    const double a = c->dt_prev, b = dt;
    const double c1 = -(a + b) / (a * b);
    const double c2 = b / (a + b) / a;
    c->coef_u[0] = -b * (c1 + c2);
    c->coef_u[1] = b * c1;
    c->coef_u[2] = b * c2;
  }
}

// Obstacle::update (Obstacle.cpp:306-368) for a body driven by its
// prescribed velocities: explicit Euler for the first step_2nd_start steps,
// BDF2 with coefU after; the quaternion is renormalised.
static void body_update(BodyState& B, const double uinf[3], int step, int step_2nd_start, const double coef[3],
                        double dt) {
  const double* w = B.omega;
  double* q = B.quat;
  const double dqdt[4] = {0.5 * (-w[0] * q[1] - w[1] * q[2] - w[2] * q[3]),
                          0.5 * (+w[0] * q[0] + w[1] * q[3] - w[2] * q[2]),
                          0.5 * (-w[0] * q[3] + w[1] * q[0] + w[2] * q[1]),
                          0.5 * (+w[0] * q[2] - w[1] * q[1] + w[2] * q[0])};
  if (step < step_2nd_start) {
    for (int d = 0; d < 3; ++d) {
      B.old_pos[d] = B.pos[d];
      B.old_abs_pos[d] = B.abs_pos[d];
      B.pos[d] += dt * (B.vel[d] + uinf[d]);
      B.abs_pos[d] += dt * B.vel[d];
    }
    for (int i = 0; i < 4; ++i) {
      B.old_quat[i] = q[i];
      q[i] += dt * dqdt[i];
    }
  } else {
    const double aux = 1.0 / coef[0];
    double tp[3], ta[3], tq[4];
    for (int d = 0; d < 3; ++d) {
      tp[d] = B.pos[d];
      ta[d] = B.abs_pos[d];
      B.pos[d] = aux * (dt * (B.vel[d] + uinf[d]) + (-coef[1] * B.pos[d] - coef[2] * B.old_pos[d]));
      B.abs_pos[d] = aux * (dt * B.vel[d] + (-coef[1] * B.abs_pos[d] - coef[2] * B.old_abs_pos[d]));
    }
    for (int i = 0; i < 4; ++i) {
      tq[i] = q[i];
      q[i] = aux * (dt * dqdt[i] + (-coef[1] * q[i] - coef[2] * B.old_quat[i]));
    }
    for (int d = 0; d < 3; ++d) {
      B.old_pos[d] = tp[d];
      B.old_abs_pos[d] = ta[d];
    }
    for (int i = 0; i < 4; ++i) B.old_quat[i] = tq[i];
  }
  const double invD = 1.0 / std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  for (int i = 0; i < 4; ++i) q[i] *= invD;
}

int body_advance(cup_ctx* c, int step, double dt) {
  body_update(c->body, c->cfg.uinf, step, c->cfg.step_2nd_start, c->coef_u, dt);
  return body_recreate(c);
}

int body_recreate(cup_ctx* c) {
  BodyState& B = c->body;
  if (B.kind < 0) return 0;
  const BodyState keep_state = B;  // the creation calls below record the body afresh
  int rc = 0;
  if (B.kind == 0)
    rc = B.on_device ? cup_obstacle_sphere_dev(c, B.pos, B.r, B.vel, B.omega)
                     : cup_obstacle_sphere(c, B.pos, B.r, B.vel, B.omega);
  else
    rc = B.on_device ? cup_obstacle_ellipsoid_dev(c, B.pos, B.ax, B.quat, B.vel, B.omega)
                     : cup_obstacle_ellipsoid(c, B.pos, B.ax, B.quat, B.vel, B.omega);
  c->body = keep_state;
  return rc;
}

// Moving bodies of a batch of cases (cup_batch_step): each case's pose
// advanced by Obstacle::update with the case's own dt and BDF2 coefficients
// (the order of cup_step: coefU, then the pose), then every body created
// again on the flattened mesh; the per-case kinematics and slot offsets go
// to the batch's step buffers.  A case without a body gets an empty box.
int batch_bodies_advance(cup_ctx* c, int step, const double* dt) {
  const int K = c->ncase;
  std::vector<Shape> shapes(K);
  for (int k = 0; k < K; ++k) {
    BodyState& B = c->case_body[k];
    double* cu = c->case_coef[k].data();
    if (step > c->cfg.step_2nd_start && c->case_dt_prev[k] > 0) {  // Simulation.cpp:361-370
      const double a = c->case_dt_prev[k], b = dt[k];
      const double c1 = -(a + b) / (a * b);
      const double c2 = b / (a + b) / a;
      cu[0] = -b * (c1 + c2);
      cu[1] = b * c1;
      cu[2] = b * c2;
    }
    c->case_dt_prev[k] = dt[k];
    Shape& sh = shapes[k];
    sh = Shape{};
    sh.kind = B.kind;
    if (B.kind < 0) {
      for (int d = 0; d < 3; ++d) {
        sh.box[d][0] = 1.0;
        sh.box[d][1] = 0.0;
      }
      continue;
    }
    body_update(B, c->cfg.uinf, step, c->cfg.step_2nd_start, cu, dt[k]);
    const double hmin = c->case_mesh[k].spec.hmin;
    for (int d = 0; d < 3; ++d) sh.c[d] = B.pos[d];
    if (B.kind == 0) {
      sphere_fill_box(B.pos, B.r, hmin, sh.box);
      sh.r = B.r;
    } else {
      quat_lab_to_body(B.quat, sh.L);
      for (int d = 0; d < 3; ++d) sh.ax[d] = B.ax[d];
      ellipsoid_fill_box(B.pos, B.ax, hmin, sh.box);
    }
    set_kinematics(sh, B.vel, B.omega);
  }
  if (int rc = obst_dev_buffers(c)) return rc;
  if (!c->d_shapes) {
    unsigned char* p = nullptr;
    if (int rc = c->batch_arena.alloc(&p, size_t(K) * sizeof(Shape))) return rc;
    c->d_shapes = p;
  }
  Shape* d_shapes = static_cast<Shape*>(c->d_shapes);
  DevObstacle& o = c->ob;
  ObstResult* res = static_cast<ObstResult*>(o.d_result);
  cudaStream_t st = c->stream;
  const int nb = c->mesh.nb;
  CUP_CUDA_TRY(cudaMemcpyAsync(d_shapes, shapes.data(), size_t(K) * sizeof(Shape), cudaMemcpyHostToDevice, st));
  {
    ProfScope ps("obstacle_slots", st);
    k_obst_slots_batch<<<1, SLOT_THREADS, 0, st>>>(nb, c->dm.h, o.d_origin, d_shapes, c->dm.bcase, c->T.first, K,
                                                  o.slot_of_block, o.block_of_slot, c->T.slot_first, res);
  }
  {
    ProfScope ps("obstacle_near", st);
    k_obst_near<<<std::max(1, std::min((nb + 255) / 256, c->num_sms * 4)), 256, 0, st>>>(c->dm, o.slot_of_block,
                                                                                       o.near);
  }
  {
    ProfScope ps("obstacle_chi", st);
    k_obst_chi_batch<<<nb, BN, 0, st>>>(c->dm.h, o.d_origin, d_shapes, c->dm.bcase, o.slot_of_block, o.chi, o.udef,
                                         c->F.chi, o.d_mom, res);
  }
  {
    ProfScope ps("obstacle_kin", st);
    k_obst_kin_batch<<<K, BN, 0, st>>>(o.d_mom, d_shapes, c->T.slot_first, c->T.kin);
  }
  CUP_CUDA_TRY(cudaGetLastError());
  ObstResult h{};
  CUP_CUDA_TRY(stream_d2h(st, &h, res, sizeof(h)));
  o.nslots = h.nslots;
  o.host_stale = true;
  o.udef_zero = true;  // k_obst_chi_batch writes udef = 0
  return 0;
}

// Host copies of a device-created obstacle (slot list, chi, udef), fetched
// when something reads them.
int ctx_obstacle_host_copies(cup_ctx* c) {
  DevObstacle& o = c->ob;
  if (!o.host_stale) return 0;
  o.h_blocks.resize(o.nslots);
  o.h_chi.resize(size_t(o.nslots) * BN);
  o.h_udef.resize(3 * size_t(o.nslots) * BN);
  CUP_CUDA_TRY(stream_d2h(c->stream, o.h_blocks.data(), o.block_of_slot, o.h_blocks.size() * sizeof(int)));
  CUP_CUDA_TRY(stream_d2h(c->stream, o.h_chi.data(), o.chi, o.h_chi.size() * sizeof(double)));
  CUP_CUDA_TRY(stream_d2h(c->stream, o.h_udef.data(), o.udef, o.h_udef.size() * sizeof(double)));
  o.host_stale = false;
  return 0;
}


// The body's shape for the signed distance (sphere or ellipsoid).
static int body_shape(const cup_ctx* c, Shape& s) {
  const BodyState& B = c->body;
  if (B.kind < 0) return set_error(CUP_ERR_STATE, "ComputeForces: the obstacle is no sphere or ellipsoid body");
  s = Shape{};
  s.kind = B.kind;
  for (int d = 0; d < 3; ++d) s.c[d] = B.pos[d];
  if (B.kind == 0) {
    s.r = B.r;
  } else {
    quat_lab_to_body(B.quat, s.L);
    for (int d = 0; d < 3; ++d) s.ax[d] = B.ax[d];
  }
  return 0;
}

// ComputeForces::operator() (FluidSolidForces.cpp:213-229) and the sums and
// derived quantities of Obstacle::computeForces (Obstacle.cpp:271-300):
// out[0..18] the kForceQ sums, out[19..22] Pthrust, Pdrag, EffPDef, EffPDefBnd.
int compute_forces(cup_ctx* c, double out[23]) {
  DevObstacle& o = c->ob;
  for (int k = 0; k < 23; ++k) out[k] = 0.0;
  if (o.nslots == 0) return 0;
  Shape s{};
  if (int rc = body_shape(c, s)) return rc;
  const int ns = o.nslots, nb = c->mesh.nb;
  cudaStream_t st = c->stream;
  DevArena tmp;
  double *origin = nullptr, *nrm = nullptr, *qslot = nullptr;
  int* err = nullptr;
  if (int rc = tmp.alloc(&origin, 3 * size_t(nb))) return rc;
  if (int rc = tmp.alloc(&nrm, 3 * size_t(ns) * BN)) return rc;
  if (int rc = tmp.alloc(&qslot, size_t(ns) * kForceQ)) return rc;
  if (int rc = tmp.alloc(&err, 1)) return rc;
  CUP_CUDA_TRY(stream_h2d(st, origin, c->mesh.origin.data(), 3 * size_t(nb) * sizeof(double)));
  CUP_CUDA_TRY(stream_zero(st, err, sizeof(int)));
  {
    ProfScope ps("obstacle_surface", st);
    k_obst_surface<<<ns, BN, 0, st>>>(c->dm.h, origin, s, o.block_of_slot, o.chi, ns, nrm);
  }
  ForceArgs A{};
  A.M = c->dm;
  A.vel = c->F.vel[c->F.vcur];
  A.n = nbn(c);
  A.pres = c->F.pres[c->F.pcur];
  A.chi = c->F.chi;
  A.origin = origin;
  A.block_of_slot = o.block_of_slot;
  A.nrm = nrm;
  A.udef = o.udef;
  A.nslots = ns;
  A.nu = c->cfg.nu;
  for (int d = 0; d < 3; ++d) {
    A.cm[d] = o.kin[d];
    A.utrans[d] = o.kin[3 + d];
    A.omega[d] = o.kin[6 + d];
  }
  A.qslot = qslot;
  A.err = err;
  const size_t smem = 4 * size_t(kFL) * kFL * kFL * sizeof(double);
  static unsigned long long attr = 0;
  if (first_on_device(attr))
    CUP_CUDA_TRY(cudaFuncSetAttribute(k_obst_forces, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  {
    ProfScope ps("obstacle_forces", st);
    k_obst_forces<<<ns, BN, smem, st>>>(A);
  }
  CUP_CUDA_TRY(cudaGetLastError());
  std::vector<double> q(size_t(ns) * kForceQ);
  int h_err = 0;
  CUP_CUDA_TRY(stream_d2h(st, q.data(), qslot, q.size() * sizeof(double)));
  CUP_CUDA_TRY(stream_d2h(st, &h_err, err, sizeof(int)));
  if (h_err)
    return set_error(CUP_ERR_MESH, "ComputeForces: a surface point's stencil reaches a block that is not a same-level "
                                   "neighbour of the obstacle block (coarse-fine or domain boundary within 4 cells)");
  for (int sl = 0; sl < ns; ++sl)  // slots in block order, as the reference's sum over blocks
    for (int k = 0; k < kForceQ; ++k) out[k] += q[size_t(sl) * kForceQ + k];
  const double eps = kEpsD;
  const double vn = std::sqrt(o.kin[3] * o.kin[3] + o.kin[4] * o.kin[4] + o.kin[5] * o.kin[5]);
  const double drag = out[12], thrust = out[13], defPower = out[16], defPowerBnd = out[17];
  out[19] = thrust * vn;
  out[20] = drag * vn;
  out[21] = out[19] / (out[19] - std::min(defPower, 0.0) + eps);
  out[22] = out[19] / (out[19] - defPowerBnd + eps);
  return 0;
}
}  // namespace cup3d

using namespace cup3d;

extern "C" {

int cup_obstacle_sphere_dev(cup_ctx* c, const double* ctr, double r, const double* vel, const double* omega) {
  ProfBind pb_(c);
  if (!ctr) return ctx_fail(c, CUP_ERR_ARG, "cup_obstacle_sphere_dev: bad arguments");
  if (int rc = shape_args_ok(c, "cup_obstacle_sphere_dev")) return rc;
  Shape s{};
  s.kind = 0;
  for (int d = 0; d < 3; ++d) s.c[d] = ctr[d];
  sphere_fill_box(ctr, r, c->mesh.spec.hmin, s.box);
  s.r = r;
  set_kinematics(s, vel, omega);
  if (int rc = create_obstacle_dev(c, s)) return ctx_fail(c, rc, "cup_obstacle_sphere_dev failed");
  body_record(c, 0, true, ctr, &r, nullptr, vel, omega);
  return 0;
}

int cup_obstacle_free(cup_ctx* c, const int32_t* free_trans, const int32_t* free_rot) {
  if (!c || c->ncase > 1) return ctx_fail(c, CUP_ERR_ARG, "cup_obstacle_free: bad arguments");
  if (c->body.kind < 0) return ctx_fail(c, CUP_ERR_STATE, "cup_obstacle_free: no sphere or ellipsoid body");
  for (int d = 0; d < 3; ++d) {
    c->body.free_t[d] = free_trans && free_trans[d] ? 1 : 0;
    c->body.free_r[d] = free_rot && free_rot[d] ? 1 : 0;
  }
  graph_reset(c);
  return 0;
}

int cup_create_obstacles(cup_ctx* c, double dt, int32_t step) {
  ProfBind pb_(c);
  if (!c || c->mesh.nb == 0 || c->host_only || !(dt > 0))
    return ctx_fail(c, CUP_ERR_ARG, "cup_create_obstacles: bad arguments");
  if (c->ncase > 1) return ctx_fail(c, CUP_ERR_STATE, "cup_create_obstacles: not available on a batch of cases");
  if (body_update_uinf(c)) graph_reset(c);
  body_coef_u(c, step, dt);
  c->dt_prev = dt;
  if (body_moves(c))
    if (int rc = body_advance(c, step, dt)) return ctx_fail(c, rc, "cup_create_obstacles failed");
  return 0;
}

int cup_obstacle_fix_frame(cup_ctx* c, const int32_t* fix) {
  if (!c || c->ncase > 1) return ctx_fail(c, CUP_ERR_ARG, "cup_obstacle_fix_frame: bad arguments");
  if (c->body.kind < 0) return ctx_fail(c, CUP_ERR_STATE, "cup_obstacle_fix_frame: no sphere or ellipsoid body");
  for (int d = 0; d < 3; ++d) c->body.fix_frame[d] = fix && fix[d] ? 1 : 0;
  body_update_uinf(c);
  graph_reset(c);
  return 0;
}

int cup_get_uinf(const cup_ctx* c, double* uinf) {
  if (!c || !uinf) return ctx_fail(nullptr, CUP_ERR_ARG, "cup_get_uinf: bad arguments");
  for (int d = 0; d < 3; ++d) uinf[d] = c->cfg.uinf[d];
  return 0;
}

int cup_update_obstacles(cup_ctx* c, double dt, double* out12) {
  ProfBind pb_(c);
  if (!c || c->mesh.nb == 0 || c->host_only || !(dt > 0))
    return ctx_fail(c, CUP_ERR_ARG, "cup_update_obstacles: bad arguments");
  if (c->ncase > 1) return ctx_fail(c, CUP_ERR_STATE, "cup_update_obstacles: not available on a batch of cases");
  if (int rc = update_obstacles(c, dt, out12)) return ctx_fail(c, rc, "cup_update_obstacles failed");
  return 0;
}

int cup_obstacle_ellipsoid_dev(cup_ctx* c, const double* ctr, const double* ax, const double* q, const double* vel,
                               const double* omega) {
  ProfBind pb_(c);
  if (!ctr || !ax || !q) return ctx_fail(c, CUP_ERR_ARG, "cup_obstacle_ellipsoid_dev: bad arguments");
  if (int rc = shape_args_ok(c, "cup_obstacle_ellipsoid_dev")) return rc;
  Shape s{};
  s.kind = 1;
  quat_lab_to_body(q, s.L);
  for (int d = 0; d < 3; ++d) {
    s.c[d] = ctr[d];
    s.ax[d] = ax[d];
  }
  ellipsoid_fill_box(ctr, ax, c->mesh.spec.hmin, s.box);
  set_kinematics(s, vel, omega);
  if (int rc = create_obstacle_dev(c, s)) return ctx_fail(c, rc, "cup_obstacle_ellipsoid_dev failed");
  body_record(c, 1, true, ctr, ax, q, vel, omega);
  return 0;
}

int cup_compute_forces(cup_ctx* c, double* out) {
  ProfBind pb_(c);
  if (!c || !out || c->mesh.nb == 0 || c->host_only) return ctx_fail(c, CUP_ERR_ARG, "cup_compute_forces: bad arguments");
  if (c->ncase > 1) return ctx_fail(c, CUP_ERR_STATE, "cup_compute_forces: not available on a batch of cases");
  if (int rc = compute_forces(c, out)) return ctx_fail(c, rc, cup_last_error(nullptr));
  return 0;
}

}  // extern "C"
