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
//     scalars, restart rule and best-iterate return, but five fused kernels
//     per iteration and no host round trip inside an iteration.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "cnn.cuh"
#include "fd.cuh"
#include "poisson.cuh"
#include "profiler.h"

namespace cup3d {

void poisson_init_constants() { fd_init_constants(); }

// ---------------------------------------------------------------------------
// Coarse-fine interpolation of PoissonSolverExp::interpolate: the Taylor part
// p_c + s1 D1 + s2 D2' + D2(ds1) + D2(ds2) + s1 s2 Dmixed, evaluated on one
// coarse face layer cl[t1 + 8 t2].  Faces normal to y use ds1 = z (tan2),
// ds2 = x (tan1); the others ds1 = tan1, ds2 = tan2 (PoissonSolverExp.h:159-371).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double cf_taylor(const double* cl, int d, int c1, int c2, double sa, double sb) {
  int u, v;
  double su, sv;
  if (d == 1) {
    u = c2; v = c1; su = sb; sv = sa;
  } else {
    u = c1; v = c2; su = sa; sv = sb;
  }
  auto L = [&](int uu, int vv) -> double { return d == 1 ? cl[vv + 8 * uu] : cl[uu + 8 * vv]; };
  const bool bdu = (u == 7 || u == 3), fdu = (u == 0 || u == 4);
  const bool bdv = (v == 7 || v == 3), fdv = (v == 0 || v == 4);
  const double c = L(u, v);
  double d1u, d1v, d2u, d2v, dm;
  if (bdu) {
    d1u = 1. / 8. * L(u - 2, v) - 1. / 2. * L(u - 1, v) + 3. / 8. * c;
    d2u = 1. / 32. * L(u - 2, v) - 1. / 16. * L(u - 1, v) + 1. / 32. * c;
  } else if (fdu) {
    d1u = -1. / 8. * L(u + 2, v) + 1. / 2. * L(u + 1, v) - 3. / 8. * c;
    d2u = 1. / 32. * L(u + 2, v) - 1. / 16. * L(u + 1, v) + 1. / 32. * c;
  } else {
    d1u = -1. / 8. * L(u - 1, v) + 1. / 8. * L(u + 1, v);
    d2u = 1. / 32. * L(u - 1, v) + 1. / 32. * L(u + 1, v) - 1. / 16. * c;
  }
  if (bdv) {
    d1v = 1. / 8. * L(u, v - 2) - 1. / 2. * L(u, v - 1) + 3. / 8. * c;
    d2v = 1. / 32. * L(u, v - 2) - 1. / 16. * L(u, v - 1) + 1. / 32. * c;
  } else if (fdv) {
    d1v = -1. / 8. * L(u, v + 2) + 1. / 2. * L(u, v + 1) - 3. / 8. * c;
    d2v = 1. / 32. * L(u, v + 2) - 1. / 16. * L(u, v + 1) + 1. / 32. * c;
  } else {
    d1v = -1. / 8. * L(u, v - 1) + 1. / 8. * L(u, v + 1);
    d2v = 1. / 32. * L(u, v - 1) + 1. / 32. * L(u, v + 1) - 1. / 16. * c;
  }
  auto N = [&](int a, int b) { return L(u + a, v + b); };
  if (bdu && bdv)
    dm = 1. / 16. * (N(0, 0) + N(-1, -1) - N(-1, 0) - N(0, -1));
  else if (fdu && bdv)
    dm = 1. / 16. * (N(1, 0) + N(0, -1) - N(1, -1) - N(0, 0));
  else if (bdu && fdv)
    dm = 1. / 16. * (N(0, 1) + N(-1, 0) - N(-1, 1) - N(0, 0));
  else if (fdu && fdv)
    dm = 1. / 16. * (N(1, 1) + N(0, 0) - N(1, 0) - N(0, 1));
  else if (bdu)
    dm = 1. / 32. * (N(0, 1) + N(-1, -1) - N(0, -1) - N(-1, 1));
  else if (fdu)
    dm = 1. / 32. * (N(1, 1) + N(0, -1) - N(1, -1) - N(0, 1));
  else if (bdv)
    dm = 1. / 32. * (N(1, 0) + N(-1, -1) - N(-1, 0) - N(1, -1));
  else if (fdv)
    dm = 1. / 32. * (N(1, 1) + N(-1, 0) - N(-1, 1) - N(1, 0));
  else
    dm = 1. / 64. * (N(1, 1) + N(-1, -1) - N(1, -1) - N(-1, 1));
  return c + su * d1u + sv * d1v + d2u + d2v + su * sv * dm;
}

// ---------------------------------------------------------------------------
// y = A x for one mesh block.  Thread t owns cells t and t+256.  Shared:
// lab[1000] (block + 1 ghost layer), ys[512], cl[64].
// ---------------------------------------------------------------------------
struct SpmvSmem {
  double lab[1000];
  double ys[512];
  double cl[64];
};

__device__ __forceinline__ int lab1(int x, int y, int z) { return (x + 1) + 10 * ((y + 1) + 10 * (z + 1)); }

template <class T>
__device__ void spmv_block(const DevMesh& M, int b, const T* __restrict__ x, double mean_sum,
                           int mean_mode, SpmvSmem& sm, double out[2]) {
  const int t = threadIdx.x;
  const double h = M.h[b];
  const T* xb = x + size_t(b) * BN;
  // interior
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int c = t + q * NT;
    sm.lab[lab1(c & 7, (c >> 3) & 7, c >> 6)] = double(xb[c]);
  }
  // ghosts: same-level neighbour values; zero-flux elsewhere (own value)
  for (int g = t; g < 384; g += NT) {
    const int f = g >> 6, a = g & 7, bb = (g >> 3) & 7;
    const int d = f >> 1, s = f & 1;
    const int kind = M.fkind[b * 6 + f];
    double v;
    if (kind == K_SAME) {
      const int nbk = M.fnbr[b * 24 + 4 * f];
      v = double(x[size_t(nbk) * BN + face_cell(d, 1 - s, 0, a, bb)]);
    } else {
      v = double(xb[face_cell(d, s, 0, a, bb)]);
    }
    int q[3];
    q[d] = s ? BS : -1;
    q[tan1(d)] = a;
    q[tan2(d)] = bb;
    sm.lab[lab1(q[0], q[1], q[2])] = v;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int c = t + q * NT;
    const int X = c & 7, Y = (c >> 3) & 7, Z = c >> 6;
    const double* L = sm.lab;
    sm.ys[c] = h * (L[lab1(X - 1, Y, Z)] + L[lab1(X + 1, Y, Z)] + L[lab1(X, Y - 1, Z)] +
                    L[lab1(X, Y + 1, Z)] + L[lab1(X, Y, Z - 1)] + L[lab1(X, Y, Z + 1)] -
                    6.0 * L[lab1(X, Y, Z)]);
  }
  // coarse-fine faces
  for (int f = 0; f < 6; ++f) {
    const int kind = M.fkind[b * 6 + f];
    if (kind != K_COARSER && kind != K_FINER) continue;
    const int d = f >> 1, s = f & 1;
    const int a = t & 7, bb = (t >> 3) & 7;
    __syncthreads();
    if (kind == K_COARSER) {
      const int cb = M.fnbr[b * 24 + 4 * f];
      if (t < 64) sm.cl[t] = double(x[size_t(cb) * BN + face_cell(d, 1 - s, 0, a, bb)]);
      __syncthreads();
      if (t < 64) {
        const int h1 = M.index[b * 3 + tan1(d)] & 1, h2 = M.index[b * 3 + tan2(d)] & 1;
        const int c1 = h1 * 4 + (a >> 1), c2 = h2 * 4 + (bb >> 1);
        const double tay = cf_taylor(sm.cl, d, c1, c2, (a & 1) ? 1.0 : -1.0, (bb & 1) ? 1.0 : -1.0);
        const int cs = face_cell(d, s, 0, a, bb), ci = face_cell(d, s, 1, a, bb);
        const double xs = double(xb[cs]), xi = double(xb[ci]);
        sm.ys[cs] += h * (2. / 3. * xs - 1. / 5. * xi + 8. / 15. * tay - xs);
      }
    } else {
      if (t < 64) sm.cl[t] = double(xb[face_cell(d, s, 0, a, bb)]);
      __syncthreads();
      if (t < 64) {
        const int ch = M.fnbr[b * 24 + 4 * f + (a >> 2) + 2 * (bb >> 2)];
        const double hf = M.h[ch];
        const T* xc = x + size_t(ch) * BN;
        double acc = 0.0;
#pragma unroll
        for (int q4 = 0; q4 < 4; ++q4) {
          const int f1 = q4 & 1, f2 = q4 >> 1;
          const int fa = 2 * (a & 3) + f1, fb = 2 * (bb & 3) + f2;
          const double close = double(xc[face_cell(d, 1 - s, 0, fa, fb)]);
          const double far = double(xc[face_cell(d, 1 - s, 1, fa, fb)]);
          const double tay = cf_taylor(sm.cl, d, a, bb, f1 ? 1.0 : -1.0, f2 ? 1.0 : -1.0);
          acc += hf * (close - (2. / 3. * close - 1. / 5. * far + 8. / 15. * tay));
        }
        sm.ys[face_cell(d, s, 0, a, bb)] += acc;
      }
    }
  }
  __syncthreads();
  if (mean_mode == 1 && b == M.mean_block && t == 0) sm.ys[0] = mean_sum;
  if (mean_mode == 3 && b == M.mean_block && t == 0) sm.ys[0] = h * double(xb[0]);
  __syncthreads();
  const double h3 = h * h * h;
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    out[q] = sm.ys[t + q * NT];
    if (mean_mode == 2) out[q] += mean_sum * h3;
  }
  __syncthreads();
}

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
  __shared__ SpmvSmem sm;
  const double ms = mean_sum ? *mean_sum : 0.0;
  for (int b = blockIdx.x; b < M.nb; b += gridDim.x) {
    double o[2];
    spmv_block<double>(M, b, x, ms, mean_mode, sm, o);
    y[size_t(b) * BN + threadIdx.x] = o[0];
    y[size_t(b) * BN + threadIdx.x + NT] = o[1];
  }
}

__global__ void __launch_bounds__(NT) k_block_inverse(DevMesh M, const double* __restrict__ in,
                                                      double* __restrict__ out) {
  __shared__ FdSmem sm;
  fd_load_scale(sm);
  for (int b = blockIdx.x; b < M.nb; b += gridDim.x) {
    __syncthreads();
    for (int c = threadIdx.x; c < BN; c += NT) sm.a[c] = in[size_t(b) * BN + c];
    __syncthreads();
    fd_apply(sm, -1.0 / M.h[b]);
    for (int c = threadIdx.x; c < BN; c += NT) out[size_t(b) * BN + c] = sm.a[c];
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
  int ext_precond;    // 1: kernels a and c only update p and s; a separate kernel applies the preconditioner
};

template <class T>
__device__ __forceinline__ T* xslot(const KArgs<T>& A, int i) {
  return i == 0 ? A.xs0 : (i == 1 ? A.xs1 : A.xs2);
}

// x0[mean row] = 0 (getVec, PoissonSolverExp.cpp:402-410) and sum(x0 h^3)
template <class T>
__global__ void __launch_bounds__(NT) k_bicg_prepare(KArgs<T> A) {
  __shared__ double red[64];
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

// r = b - A x0, rhat = r, p = nu = 0; err_init = ||r||
template <class T>
__global__ void __launch_bounds__(NT) k_bicg_init(KArgs<T> A) {
  __shared__ SpmvSmem sm;
  __shared__ double red[64];
  const DevMesh& M = A.M;
  const double ms = A.st->mean_sum;
  double acc[1] = {0.0};
  for (int b = blockIdx.x; b < M.nb; b += gridDim.x) {
    double o[2];
    spmv_block<T>(M, b, A.xs0, ms, A.mean_mode, sm, o);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int c = threadIdx.x + q * NT;
      const size_t i = size_t(b) * BN + c;
      double bi = double(A.b[i]);
      if (A.zero_mean_row && b == M.mean_block && c == 0) bi = 0.0;
      const double ri = bi - o[q];
      A.r[i] = T(ri);
      A.rhat[i] = T(ri);
      A.p[i] = T(0);
      A.nu[i] = T(0);
      acc[0] += ri * ri;
    }
  }
  if (grid_reduce<1>(acc, A.g, red) && threadIdx.x == 0) {
    KrylovState& S = *A.st;
    const double e = sqrt(acc[0]);
    S.err = S.err_init = S.err_opt = e;
    S.rr = S.rr_hat = acc[0];
    S.rho = acc[0];  // (rhat, r) of iteration 0
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
}

// KA: p = r + beta (p - omega nu) (or p = r, rhat = r after a restart);
//     z1 = M^-1 p; sum(z1 h^3)
template <class T>
__global__ void __launch_bounds__(NT) k_bicg_a(KArgs<T> A) {
  __shared__ FdSmem sm;
  __shared__ double red[64];
  const KrylovState& S = *A.st;
  if (S.done) return;
  const double beta = S.beta, omega = S.omega;
  const bool restart = S.restart_pending != 0;
  const DevMesh& M = A.M;
  fd_load_scale(sm);
  double acc[1] = {0.0};
  for (int b = blockIdx.x; b < M.nb; b += gridDim.x) {
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int c = threadIdx.x + q * NT;
      const size_t i = size_t(b) * BN + c;
      const double ri = double(A.r[i]);
      double pi;
      if (restart) {
        pi = ri;
        A.rhat[i] = T(ri);
      } else {
        pi = ri + beta * (double(A.p[i]) - omega * double(A.nu[i]));
      }
      A.p[i] = T(pi);
      sm.a[c] = double(T(pi));
    }
    if (A.ext_precond) continue;  // uniform; z1 comes from the external preconditioner
    __syncthreads();
    const double h = M.h[b];
    fd_apply(sm, -1.0 / h);
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int c = threadIdx.x + q * NT;
      const T zi = T(sm.a[c]);
      A.z1[size_t(b) * BN + c] = zi;
      s += double(zi);
    }
    acc[0] += s * h * h * h;
  }
  if (grid_reduce<1>(acc, A.g, red) && threadIdx.x == 0) {
    KrylovState& W = *A.st;
    W.mean_sum = acc[0];
    if (restart) {
      W.rho = W.rr;
      W.rr_hat = W.rr;
      W.restart_pending = 0;
    }
  }
}

// KB: nu = A z1; alpha = rho / ((rhat, nu) + eps)
template <class T>
__global__ void __launch_bounds__(NT) k_bicg_b(KArgs<T> A) {
  __shared__ SpmvSmem sm;
  __shared__ double red[64];
  const KrylovState& S = *A.st;
  if (S.done) return;
  const DevMesh& M = A.M;
  const double ms = S.mean_sum;
  double acc[1] = {0.0};
  for (int b = blockIdx.x; b < M.nb; b += gridDim.x) {
    double o[2];
    spmv_block<T>(M, b, A.z1, ms, A.mean_mode, sm, o);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const size_t i = size_t(b) * BN + threadIdx.x + q * NT;
      const T v = T(o[q]);
      A.nu[i] = v;
      acc[0] += double(A.rhat[i]) * double(v);
    }
  }
  if (grid_reduce<1>(acc, A.g, red) && threadIdx.x == 0) {
    KrylovState& W = *A.st;
    W.alpha = W.rho / (acc[0] + W.eps);
  }
}

// KC: s = r - alpha nu (in place in r); z2 = M^-1 s; sum(z2 h^3)
template <class T>
__global__ void __launch_bounds__(NT) k_bicg_c(KArgs<T> A) {
  __shared__ FdSmem sm;
  __shared__ double red[64];
  const KrylovState& S = *A.st;
  if (S.done) return;
  const double alpha = S.alpha;
  const DevMesh& M = A.M;
  fd_load_scale(sm);
  double acc[1] = {0.0};
  for (int b = blockIdx.x; b < M.nb; b += gridDim.x) {
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int c = threadIdx.x + q * NT;
      const size_t i = size_t(b) * BN + c;
      const T si = T(double(A.r[i]) - alpha * double(A.nu[i]));
      A.r[i] = si;
      sm.a[c] = double(si);
    }
    if (A.ext_precond) continue;  // uniform; z2 comes from the external preconditioner
    __syncthreads();
    const double h = M.h[b];
    fd_apply(sm, -1.0 / h);
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int c = threadIdx.x + q * NT;
      const T zi = T(sm.a[c]);
      A.z2[size_t(b) * BN + c] = zi;
      s += double(zi);
    }
    acc[0] += s * h * h * h;
  }
  if (grid_reduce<1>(acc, A.g, red) && threadIdx.x == 0) A.st->mean_sum = acc[0];
}

// KD: t = A z2; omega = (t, s) / ((t, t) + eps)
template <class T>
__global__ void __launch_bounds__(NT) k_bicg_d(KArgs<T> A) {
  __shared__ SpmvSmem sm;
  __shared__ double red[64];
  const KrylovState& S = *A.st;
  if (S.done) return;
  const DevMesh& M = A.M;
  const double ms = S.mean_sum;
  double acc[2] = {0.0, 0.0};
  for (int b = blockIdx.x; b < M.nb; b += gridDim.x) {
    double o[2];
    spmv_block<T>(M, b, A.z2, ms, A.mean_mode, sm, o);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const size_t i = size_t(b) * BN + threadIdx.x + q * NT;
      const T v = T(o[q]);
      A.t[i] = v;
      acc[0] += double(v) * double(A.r[i]);
      acc[1] += double(v) * double(v);
    }
  }
  if (grid_reduce<2>(acc, A.g, red) && threadIdx.x == 0) {
    KrylovState& W = *A.st;
    W.omega = acc[0] / (acc[1] + W.eps);
  }
}

// KE: x_new = x + alpha z1 + omega z2; r = s - omega t; (rhat, r), (r, r);
//     convergence, best iterate, restart decision, beta for the next KA.
template <class T>
__global__ void __launch_bounds__(NT) k_bicg_e(KArgs<T> A) {
  __shared__ double red[64];
  const KrylovState& S = *A.st;
  if (S.done) return;
  const double alpha = S.alpha, omega = S.omega;
  const T* xc = xslot(A, S.cur);
  T* xn = xslot(A, S.nxt);
  const DevMesh& M = A.M;
  double acc[2] = {0.0, 0.0};
  const size_t n = size_t(M.nb) * BN;
  for (size_t i = size_t(blockIdx.x) * NT + threadIdx.x; i < n; i += size_t(gridDim.x) * NT) {
    xn[i] = T((double(xc[i]) + alpha * double(A.z1[i])) + omega * double(A.z2[i]));
    const T ri = T(double(A.r[i]) - omega * double(A.t[i]));
    A.r[i] = ri;
    acc[0] += double(A.rhat[i]) * double(ri);
    acc[1] += double(ri) * double(ri);
  }
  if (grid_reduce<2>(acc, A.g, red) && threadIdx.x == 0) {
    KrylovState& W = *A.st;
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
  __shared__ SpmvSmem sm;
  __shared__ double red[64];
  const double ms = st->mean_sum;
  double acc[1] = {0.0};
  for (int blk = blockIdx.x; blk < M.nb; blk += gridDim.x) {
    double o[2];
    spmv_block<double>(M, blk, x, ms, mean_mode, sm, o);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int c = threadIdx.x + q * NT;
      const size_t i = size_t(blk) * BN + c;
      double bi = b[i];
      if (zero_mean_row && blk == M.mean_block && c == 0) bi = 0.0;
      const double ri = bi - o[q];
      if (r32) r32[i] = float(ri);
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
  A.ext_precond = 0;
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
  { ProfScope ps("spmv", s); k_spmv<<<W.grid, NT, 0, s>>>(M, x, y, ms, mean_mode); }
  CUP_CUDA_TRY(cudaGetLastError());
  return 0;
}

int launch_block_inverse(const DevMesh& M, const double* in, double* out, PoissonWork& W,
                         cudaStream_t s) {
  poisson_init_constants();
  { ProfScope ps("block_inverse", s); k_block_inverse<<<W.grid, NT, 0, s>>>(M, in, out); }
  CUP_CUDA_TRY(cudaGetLastError());
  return 0;
}

// Runs BiCGSTAB on vectors of type T; x holds x0 on entry, x_opt on exit.
template <class T>
static int run_bicgstab(const DevMesh& M, const T* b, T* x, T* const v[9], const SolveParams& P, int zero_mean_row,
                        PoissonWork& W, SolveStats& out, cudaStream_t s, int* h_done,
                        const CnnWeights* cnn = nullptr) {
  const bool f32 = sizeof(T) == 4;
  KrylovState init{};
  init.tol_abs = P.tol_abs;
  init.tol_rel = P.tol_rel;
  init.max_iter = P.max_iter;
  init.max_restarts = P.max_restarts;
  init.stall_window = P.stall_window;
  init.eps = 1e-21;
  CUP_CUDA_TRY(cudaMemcpyAsync(W.st, &init, sizeof(init), cudaMemcpyHostToDevice, s));
  KArgs<T> A = make_args<T>(M, b, x, v, W, W.st, P.mean_mode, zero_mean_row, 0);
  A.ext_precond = cnn ? 1 : 0;
  GridReduce gc{W.partial, W.counters + 14};
  { ProfScope ps(f32 ? "bicg32_prepare" : "bicg_prepare", s); k_bicg_prepare<T><<<W.grid, NT, 0, s>>>(A); }
  { ProfScope ps(f32 ? "bicg32_init" : "bicg_init", s); k_bicg_init<T><<<W.grid, NT, 0, s>>>(A); }
  CUP_CUDA_TRY(cudaGetLastError());
  const int chunk = P.check_every > 0 ? P.check_every : 8;
  for (int it = 0; it < P.max_iter; it += chunk) {
    for (int j = 0; j < chunk; ++j) {
      { ProfScope ps(f32 ? "bicg32_a_pupdate_precond" : "bicg_a_pupdate_precond", s); k_bicg_a<T><<<W.grid, NT, 0, s>>>(A); }
      if (cnn)
        if (int rc = cnn_apply<T>(M, A.p, A.z1, *cnn, W.grid, s, gc, &W.st->mean_sum)) return rc;
      { ProfScope ps(f32 ? "bicg32_b_spmv_dot" : "bicg_b_spmv_dot", s); k_bicg_b<T><<<W.grid, NT, 0, s>>>(A); }
      { ProfScope ps(f32 ? "bicg32_c_supdate_precond" : "bicg_c_supdate_precond", s); k_bicg_c<T><<<W.grid, NT, 0, s>>>(A); }
      if (cnn)
        if (int rc = cnn_apply<T>(M, A.r, A.z2, *cnn, W.grid, s, gc, &W.st->mean_sum)) return rc;
      { ProfScope ps(f32 ? "bicg32_d_spmv_dots" : "bicg_d_spmv_dots", s); k_bicg_d<T><<<W.grid, NT, 0, s>>>(A); }
      { ProfScope ps(f32 ? "bicg32_e_xr_update_dots" : "bicg_e_xr_update_dots", s); k_bicg_e<T><<<W.grid, NT, 0, s>>>(A); }
    }
    CUP_CUDA_TRY(cudaGetLastError());
    CUP_CUDA_TRY(cudaMemcpyAsync(h_done, &W.st->done, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUP_CUDA_TRY(cudaStreamSynchronize(s));
    if (*h_done) break;
  }
  KrylovState fin;
  CUP_CUDA_TRY(cudaMemcpyAsync(&fin, W.st, sizeof(fin), cudaMemcpyDeviceToHost, s));
  CUP_CUDA_TRY(cudaStreamSynchronize(s));
  if (fin.best != 0) {
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
                     PoissonWork& W, SolveStats& out, cudaStream_t s, int* h_done, const CnnWeights* cnn) {
  poisson_init_constants();
  double* const v[9] = {W.r, W.rhat, W.p, W.nu, W.t, W.z1, W.z2, W.xs[1], W.xs[2]};
  const int zmr = (P.mean_mode == 1 || P.mean_mode == 3) ? 1 : 0;
  return run_bicgstab<double>(M, b, x, v, P, zmr, W, out, s, h_done, cnn);
}

// Mixed precision: FP64 iterative refinement around FP32 BiCGSTAB inner solves.
// Every outer step recomputes the true residual b - A x in FP64 (the
// convergence test is on it), solves A e = r with FP32 vectors (FP64 dots and
// scalars) to a relative tolerance tied to the remaining reduction, and adds e
// to x in FP64.
int poisson_mixed(const DevMesh& M, const double* b, double* x, const SolveParams& P, PoissonWork& W,
                  SolveStats& out, cudaStream_t s, int* h_done, const CnnWeights* cnn) {
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
      k_true_residual<<<W.grid, NT, 0, s>>>(M, b, x, W.r32, P.mean_mode, zmr, so, g);
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
    if (int rc = run_bicgstab<float>(M, W.r32, e, v, Q, 0, W, in, s, h_done, cnn)) return rc;
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
    k_true_residual<<<W.grid, NT, 0, s>>>(M, b, x, nullptr, mean_mode, zmr, so, g);
  }
  CUP_CUDA_TRY(cudaGetLastError());
  CUP_CUDA_TRY(cudaMemcpyAsync(err_host, &so->err, sizeof(double), cudaMemcpyDeviceToHost, s));
  CUP_CUDA_TRY(cudaStreamSynchronize(s));
  return 0;
}

}  // namespace cup3d
