// Block-group primitives of the Poisson kernels.  A CTA of 256 threads works
// on 4 mesh blocks at once, one 64-thread group (two warps) per block; thread
// (gx, gy) of a group owns the z-column of 8 cells (gx, gy, 0..7), so every
// global load of a column is one coalesced 256-byte row per warp and each
// thread keeps 8 independent loads in flight.  Groups synchronise with named
// barriers (bar.sync id, 64), so the four blocks of a CTA proceed
// independently.
#pragma once
#include "common.cuh"

namespace cup3d {

constexpr int GROUP = 64;                 // threads per block group
constexpr int GROUPS = NT / GROUP;        // groups per CTA

struct GroupIdx {
  int g, lane, gx, gy;
  __device__ __forceinline__ GroupIdx() {
    g = threadIdx.x >> 6;
    lane = threadIdx.x & 63;
    gx = lane & 7;
    gy = lane >> 3;
  }
};

__device__ __forceinline__ void group_sync(int g) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(1 + g), "r"(GROUP) : "memory");
}

// Shared tile of one block for the transforms (rows padded to spread banks).
struct FdTile {
  double v[BS][BS][BS + 1];  // [z][y][x]
};

// A block's entries of the mesh tables, staged in shared memory so that the
// operator reads them without a global-memory round trip.
struct BlockInfo {
  int kind[6];   // face kinds (K_SAME, ...)
  int nbr[24];   // face neighbours, four per face (fnbr row)
  double h;      // grid spacing; finer neighbours have h/2, coarser 2h
  int id;        // block index
  int par;       // bit e: parity of the block's index along axis e
  int mean;      // 1: the block holds the mean-constraint row
  int pad_;
};

// Shared tile of one block for the operator: the block with its x/y ghost
// layers in one padded array (v[z][y+1][x+1] holds cell (x, y, z); x = -1, 8
// and y = -1, 8 hold the ghosts, so every neighbour is a fixed offset), the
// face layers of coarser neighbours and the coarse-fine fluxes of x/y faces
// (face-local index tan1 + 8 tan2 in every per-face array), and the block's
// table entries.  The transforms' FdTile aliases the leading member.
struct GroupTile {
  double v[BS][BS + 2][BS + 2];  // [z][y+1][x+1]
  double cl[6][BS * BS];         // per coarser face: the coarse block's layer on that face
  double flx[4][BS * BS];        // x/y coarse-fine face fluxes
  BlockInfo bi;
};

// Orthogonal, symmetric DST-I of size 8: S(n,k) = sqrt(2/9) sin(pi (n+1)(k+1)/9).
// Its entries take only the magnitudes sqrt(2/9) sin(pi r/9), r = 1..4, and
// S(7-n, k) = (-1)^k S(n, k), so y = S x splits into x[n] +- x[7-n] (n < 4)
// followed by two 4x4 products: 32 multiply-adds instead of 64, and the
// coefficients fold into immediate operands once the loops are unrolled.
__host__ __device__ constexpr double dst_mag(int r) {
  return r == 1 ? 0.16122984176531682
       : r == 2 ? 0.30301298511469577
       : r == 3 ? 0.40824829046386296
                : 0.4642428268800126;
}

__host__ __device__ constexpr double dst_coef(int n, int k) {
  const int m = ((n + 1) * (k + 1)) % 18;  // sin(pi m / 9) has period 18
  if (m == 0 || m == 9) return 0.0;
  const int r0 = m < 9 ? m : m - 9;
  const int r = r0 > 4 ? 9 - r0 : r0;
  return (m < 9 ? 1.0 : -1.0) * dst_mag(r);
}

__device__ __forceinline__ void dst8(const double x[8], double y[8]) {
  double u[4], v[4];
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    u[n] = x[n] + x[7 - n];
    v[n] = x[n] - x[7 - n];
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    double s = 0.0;
#pragma unroll
    for (int n = 0; n < 4; ++n)
      if (dst_coef(n, k) != 0.0) s = fma(dst_coef(n, k), (k & 1) ? v[n] : u[n], s);
    y[k] = s;
  }
}

// 1 / (lam_kx + lam_ky + lam_kz) for the eigenvalues lam_j = 2 - 2 cos(pi (j+1)/9)
// of tridiag(-1, 2, -1), laid out [kx][kz][ky] so that thread (ky = gx, kz = gy)
// of a group reads entry kx at inv[kx * 64 + lane] without bank conflicts.
// Filled by the whole CTA; a __syncthreads() must follow.
__device__ __forceinline__ void fd_fill_inverse_eigen(double* inv, const double* lam) {
  for (int i = threadIdx.x; i < BN; i += blockDim.x) {
    const int kx = i >> 6, kz = (i >> 3) & 7, ky = i & 7;
    inv[i] = 1.0 / (lam[kx] + lam[ky] + lam[kz]);
  }
}

// Block inverse scale * L_D^-1 by fast diagonalization on a group,
// L_D^-1 = (S x S x S) diag(1/(lam_x + lam_y + lam_z)) (S x S x S): the
// thread's z-column is transformed in registers, the y and x transforms go
// through the shared tile; forward x, scaling and inverse x happen on one
// register row.  In: col[8] (the thread's column), out: col[8].  4 group
// barriers; the tile may be reused after one more.
__device__ __forceinline__ void fd_group(double col[8], FdTile& t, const GroupIdx& G, double scale,
                                         const double* __restrict__ inv) {
  double w[8], r[8];
  dst8(col, w);  // z transform of the own column
#pragma unroll
  for (int z = 0; z < 8; ++z) t.v[z][G.gy][G.gx] = w[z];
  group_sync(G.g);
  // y transform: thread (x = gx, z = gy) owns row t.v[z][*][x]
#pragma unroll
  for (int i = 0; i < 8; ++i) r[i] = t.v[G.gy][i][G.gx];
  dst8(r, w);
#pragma unroll
  for (int k = 0; k < 8; ++k) t.v[G.gy][k][G.gx] = w[k];
  group_sync(G.g);
  // x transform, scaling, inverse x: thread (y = gx, z = gy) owns row t.v[z][y][*]
#pragma unroll
  for (int i = 0; i < 8; ++i) r[i] = t.v[G.gy][G.gx][i];
  dst8(r, w);
#pragma unroll
  for (int k = 0; k < 8; ++k) w[k] *= scale * inv[k * 64 + G.lane];
  dst8(w, r);
#pragma unroll
  for (int k = 0; k < 8; ++k) t.v[G.gy][G.gx][k] = r[k];
  group_sync(G.g);
  // inverse y: thread (x = gx, z = gy) owns row t.v[z][*][x]
#pragma unroll
  for (int i = 0; i < 8; ++i) r[i] = t.v[G.gy][i][G.gx];
  dst8(r, w);
#pragma unroll
  for (int k = 0; k < 8; ++k) t.v[G.gy][k][G.gx] = w[k];
  group_sync(G.g);
  // inverse z: thread (x = gx, y = gy) owns column t.v[*][y][x]
#pragma unroll
  for (int i = 0; i < 8; ++i) r[i] = t.v[i][G.gy][G.gx];
  dst8(r, col);
}

}  // namespace cup3d
