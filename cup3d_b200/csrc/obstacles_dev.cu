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

__global__ void __launch_bounds__(BN) k_obst_chi(const double* __restrict__ h_, const double* __restrict__ origin,
                                                  Shape s, const int* __restrict__ slot_of_block,
                                                  double* __restrict__ chi, double* __restrict__ udef,
                                                  double* __restrict__ grid_chi, double* __restrict__ mom,
                                                  const ObstResult* res) {
  const int b = blockIdx.x, t = threadIdx.x;
  const int slot = slot_of_block[b];
  if (slot < 0) {
    grid_chi[size_t(b) * BN + t] = 0.0;
    return;
  }
  __shared__ double lab[10][10][10];
  __shared__ double sm[16];
  const double h = h_[b];
  const double ox = origin[3 * b], oy = origin[3 * b + 1], oz = origin[3 * b + 2];
  for (int i = t; i < 1000; i += BN) {
    const int x = i % 10 - 1, y = (i / 10) % 10 - 1, z = i / 100 - 1;
    lab[z + 1][y + 1][x + 1] = shape_sdf(s, ox + (x + 0.5) * h, oy + (y + 0.5) * h, oz + (z + 0.5) * h);
  }
  __syncthreads();
  const int x = t & 7, y = (t >> 3) & 7, z = t >> 6;
  const double inv2h = 0.5 / h, vol = h * h * h;
  const double s0 = lab[z + 1][y + 1][x + 1];
  double c;
  if (s0 > h || s0 < -h) {
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
  const size_t ns = size_t(res->nslots);  // udef is component-major: [3][nslots][512]
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

}  // extern "C"
