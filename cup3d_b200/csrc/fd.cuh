// Exact inverse of the 8^3 Dirichlet 7-point block (the reference GPU
// preconditioner P_inv = -(L_D)^-1, PoissonSolverExp.cpp:17-111) applied by
// fast diagonalization: L_D = T(x)I(x)I + I(x)T(x)I + I(x)I(x)T with
// T = tridiag(-1, 2, -1) on 8 points, diagonalised by the orthogonal,
// symmetric DST-I matrix S.  Each translation unit that includes this header
// gets its own constant-memory copy and must call fd_init_constants() once
// its device is current.
#pragma once
#include <cmath>

#include "common.cuh"

namespace cup3d {

static __constant__ double c_S[64];
static __constant__ double c_lam[8];
static bool g_fd_consts_ready = false;

static inline void fd_init_constants() {
  if (g_fd_consts_ready) return;
  double S[64], lam[8];
  const double pi = 3.14159265358979323846;
  for (int j = 0; j < 8; ++j) {
    lam[j] = 2.0 - 2.0 * std::cos(pi * (j + 1) / 9.0);
    for (int k = 0; k < 8; ++k) S[j * 8 + k] = std::sqrt(2.0 / 9.0) * std::sin(pi * (j + 1) * (k + 1) / 9.0);
  }
  cudaMemcpyToSymbol(c_S, S, sizeof(S));
  cudaMemcpyToSymbol(c_lam, lam, sizeof(lam));
  g_fd_consts_ready = true;
}

// ---------------------------------------------------------------------------
// z = (1/h) P_inv v = -(1/h) L_D^-1 v on one block by fast diagonalization.
// Thread t owns mode index k = t&7 along the transformed axis and the two
// transverse positions (t>>3) and (t>>3)+32.  buf holds the block on entry
// and the result on exit.
// ---------------------------------------------------------------------------
struct FdSmem {
  double a[512];
  double b[512];
  double inv_lam[512];
};

static __device__ __forceinline__ void fd_load_scale(FdSmem& sm) {
  for (int i = threadIdx.x; i < 512; i += NT) {
    const int kx = i & 7, ky = (i >> 3) & 7, kz = i >> 6;
    sm.inv_lam[i] = 1.0 / (c_lam[kx] + c_lam[ky] + c_lam[kz]);
  }
}

// one mode product along axis `ax` (0=x,1=y,2=z): out = S x_ax in
static __device__ __forceinline__ void fd_pass(const double* in, double* out, int ax, const double Srow[8]) {
  const int t = threadIdx.x, k = t & 7;
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int o = (t >> 3) + 32 * q;  // transverse pair index 0..63
    const int p0 = o & 7, p1 = o >> 3;
    int base, stride;
    if (ax == 0) { base = 8 * p0 + 64 * p1; stride = 1; }
    else if (ax == 1) { base = p0 + 64 * p1; stride = 8; }
    else { base = p0 + 8 * p1; stride = 64; }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s = fma(Srow[i], in[base + stride * i], s);
    out[base + stride * k] = s;
  }
}

// in: sm.a, result in sm.a.  scale = -1/h
static __device__ __forceinline__ void fd_apply(FdSmem& sm, double scale) {
  const int t = threadIdx.x, k = t & 7;
  double Srow[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) Srow[i] = c_S[k * 8 + i];
  fd_pass(sm.a, sm.b, 0, Srow);
  __syncthreads();
  fd_pass(sm.b, sm.a, 1, Srow);
  __syncthreads();
  fd_pass(sm.a, sm.b, 2, Srow);
  __syncthreads();
  for (int i = t; i < 512; i += NT) sm.b[i] *= scale * sm.inv_lam[i];
  __syncthreads();
  fd_pass(sm.b, sm.a, 0, Srow);
  __syncthreads();
  fd_pass(sm.a, sm.b, 1, Srow);
  __syncthreads();
  fd_pass(sm.b, sm.a, 2, Srow);
  __syncthreads();
}

}  // namespace cup3d
