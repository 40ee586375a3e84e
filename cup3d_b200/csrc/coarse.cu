// Coarse space of the two-level preconditioners: one unknown per mesh block.
//
//   M^-1 r = B^-1 r + P A_c^-1 P^T r
//
// B^-1: the per-block preconditioner (block inverse, or the learned network);
// P: prolongation by a constant over each block; P^T: the sum over a block's
// cells; A_c = P^T A P: the Galerkin coarse operator of the Poisson matrix A
// (the device operator, mean-constraint row included).  No counterpart in
// the reference, whose preconditioner is block-local (PoissonSolverAMR.h:
// 183-222, BiCGSTAB.cu:526-527): the block-local method converges in a number
// of iterations that grows with the number of blocks across the domain, the
// coarse correction removes that growth.
//
// Set-up (once per mesh, coarse_build):
//   * A_c column by column through the device operator: the blocks are given
//     colours such that no two blocks of a colour are face neighbours or
//     share one (distance-2 colouring on the host), and A is applied to the
//     indicator of each colour; the sum of the result over block I's cells is
//     A_c[I][J] for the one block J of the colour at or next to I.  The
//     mean-constraint row (sum over all cells of x h^3) couples its block to
//     every block, J by 512 h_J^3; that part is known and separated.
//   * A_c^-1 by blocked Gauss-Jordan elimination on the device: panels of 32
//     pivots, three launches each (the 32 x 32 pivot block's inverse, the
//     panel products, a rank-32 update of the whole matrix by 64 x 64 tiles),
//     checked by A_c^-1 (A_c v) = v; a failed check repeats it column by
//     column with partial pivoting.
// Apply (two kernels and a reduction per application): r restricted to the
// blocks, one dense matrix-vector product with A_c^-1, the result added to
// every cell of its block; the weighted sum sum(z h^3) that the next
// operator application needs for its mean row gets the added part.
#include <algorithm>
#include <cmath>
#include <set>
#include <vector>

#include "context.h"

namespace cup3d {
namespace {

// x[i] = 1 on the cells of blocks of colour c, else 0
__global__ void k_colour_indicator(int nb, const int* __restrict__ colour, int c, double* __restrict__ x) {
  const size_t n = size_t(nb) * BN;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    x[i] = colour[i / BN] == c ? 1.0 : 0.0;
}

// out[b] = sum of v over block b's cells, in a fixed order
template <class T>
__global__ void __launch_bounds__(NT) k_block_sum(int nb, const T* __restrict__ v, double* __restrict__ out) {
  __shared__ double red[64];
  for (int b = blockIdx.x; b < nb; b += gridDim.x) {
    double s[1] = {0.0};
    for (int c = threadIdx.x; c < BN; c += NT) s[0] += double(v[size_t(b) * BN + c]);
    block_reduce<1>(s, red);
    if (threadIdx.x == 0) out[b] = s[0];
  }
}

// One colour's column entries of A_c: row i gets sums[i] (its block's sum of
// A applied to the colour's indicator) less the known dense part, at column
// jmap[i] (the block of the colour at or next to i; -1: none)
__global__ void k_coarse_scatter(double* __restrict__ Ac, int nb, const int* __restrict__ jmap,
                                 const double* __restrict__ sums, const double* __restrict__ w, double wcol, int mode,
                                 int mb) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
    const int J = jmap[i];
    if (J < 0) continue;
    const double known = (mode == 1 && i == mb) ? wcol : (mode == 2 ? w[i] * wcol : 0.0);
    Ac[size_t(i) * nb + J] += sums[i] - known;
  }
}

// The known dense parts of A_c: mode 1, the mean row of block mb adds
// 512 h_J^3 for every J; mode 2, every row I adds 512 h_I^3 512 h_J^3
__global__ void k_coarse_dense(double* __restrict__ Ac, int nb, const double* __restrict__ w, int mode, int mb) {
  const size_t total = mode == 1 ? size_t(nb) : size_t(nb) * nb;
  for (size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += size_t(gridDim.x) * blockDim.x) {
    if (mode == 1)
      Ac[size_t(mb) * nb + e] += w[e];
    else
      Ac[e] += w[e / nb] * w[e % nb];
  }
}

// Gauss-Jordan on the augmented matrix G = [A | I] (n rows of 2n, row-major),
// step k: the pivot row (largest |G[i][k]|, i >= k) swapped into row k and
// scaled to a unit pivot, and the factors G[i][k] of every row kept in fac.
__global__ void __launch_bounds__(1024) k_gj_pivot(double* G, int n, int k, double* fac, int* singular) {
  __shared__ double sv[1024];
  __shared__ int si[1024];
  const int t = threadIdx.x, w = 2 * n;
  double best = -1.0;
  int arg = k;
  for (int i = k + t; i < n; i += blockDim.x) {
    const double a = fabs(G[size_t(i) * w + k]);
    if (a > best) {
      best = a;
      arg = i;
    }
  }
  sv[t] = best;
  si[t] = arg;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (t < s && (sv[t + s] > sv[t] || (sv[t + s] == sv[t] && si[t + s] < si[t]))) {
      sv[t] = sv[t + s];
      si[t] = si[t + s];
    }
    __syncthreads();
  }
  const int p = si[0];
  if (!(sv[0] > 0.0)) {
    if (t == 0) *singular = 1;
    return;
  }
  if (p != k)
    for (int j = t; j < w; j += blockDim.x) {
      const double a = G[size_t(k) * w + j];
      G[size_t(k) * w + j] = G[size_t(p) * w + j];
      G[size_t(p) * w + j] = a;
    }
  __syncthreads();
  const double inv = 1.0 / G[size_t(k) * w + k];
  __syncthreads();
  for (int j = t; j < w; j += blockDim.x) G[size_t(k) * w + j] *= inv;
  __syncthreads();
  for (int i = t; i < n; i += blockDim.x) fac[i] = i == k ? 0.0 : G[size_t(i) * w + k];
}

// rows i != k: G[i][j] -= fac[i] G[k][j] for columns j >= k
__global__ void k_gj_eliminate(double* G, int n, int k, const double* __restrict__ fac) {
  const int w = 2 * n, cols = w - k;
  const size_t total = size_t(n) * cols;
  for (size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += size_t(gridDim.x) * blockDim.x) {
    const int i = int(e / cols), j = k + int(e % cols);
    const double f = fac[i];
    if (f != 0.0) G[size_t(i) * w + j] -= f * G[size_t(k) * w + j];
  }
}

// inv (n x n) from the right half of G
__global__ void k_gj_extract(const double* __restrict__ G, int n, double* __restrict__ inv) {
  const size_t total = size_t(n) * n;
  for (size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += size_t(gridDim.x) * blockDim.x) {
    const size_t i = e / n, j = e % n;
    inv[e] = G[i * 2 * n + n + j];
  }
}

// G = [A | I] (n rows of 2n) from the device matrix A (n x n)
__global__ void k_gj_augment(const double* __restrict__ A, int n, double* __restrict__ G) {
  const size_t total = size_t(n) * 2 * n;
  for (size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += size_t(gridDim.x) * blockDim.x) {
    const size_t i = e / (2 * size_t(n)), j = e % (2 * size_t(n));
    G[e] = j < size_t(n) ? A[i * n + j] : (j - n == i ? 1.0 : 0.0);
  }
}

// ---- blocked Gauss-Jordan, in place: A -> A^-1 ----
//
// Panel K = [k0, k0 + bk) of the pivot order, with P = M[K][K] and R the
// other indices; one step replaces
//   M[K][K] = P^-1,  M[K][R] = P^-1 M[K][R],
//   M[R][K] = -M[R][K] P^-1,  M[R][R] -= M[R][K] P^-1 M[K][R].
// With T' = P^-1 M[K][:] outside K and P^-1 inside, and C = M[:][K] (old),
// every entry outside the panel rows is base - C T' (base = 0 in the panel
// columns), and the panel rows are T'.  The panels follow the index order
// (no pivoting across them); inside a pivot block, partial pivoting.
constexpr int GJB = 32;  // panel width
constexpr int GJT = 64;  // update tile (GJT x GJT per CTA)

// Pinv (GJB x GJB) = P^-1 by Gauss-Jordan with partial pivoting, one CTA;
// *flag = 1 when a pivot is not above 1e-13 of P's largest entry.
__global__ void __launch_bounds__(256) k_bgj_block_inverse(const double* __restrict__ M, int n, int k0, int bk,
                                                          double* __restrict__ Pinv, int* flag) {
  __shared__ double G[GJB][2 * GJB + 1];
  __shared__ double fac[GJB];
  __shared__ double red[8];
  __shared__ int s_piv, s_bad;
  const int t = threadIdx.x;
  double amax = 0.0;
  for (int e = t; e < GJB * 2 * GJB; e += blockDim.x) {
    const int r = e / (2 * GJB), c = e % (2 * GJB);
    double v;
    if (c < GJB)
      v = (r < bk && c < bk) ? M[size_t(k0 + r) * n + k0 + c] : (r == c ? 1.0 : 0.0);
    else
      v = c - GJB == r ? 1.0 : 0.0;
    G[r][c] = v;
    if (c < bk && r < bk) amax = fmax(amax, fabs(v));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
  if ((t & 31) == 0) red[t >> 5] = amax;
  if (t == 0) s_bad = 0;
  __syncthreads();
  amax = 0.0;
  for (int w = 0; w < int(blockDim.x >> 5); ++w) amax = fmax(amax, red[w]);
  const double tiny = 1e-13 * amax;
  for (int j = 0; j < bk; ++j) {
    if (t < 32) {
      const int r = j + t;
      double a = r < bk ? fabs(G[r][j]) : -1.0;
      int arg = r;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double oa = __shfl_xor_sync(0xffffffffu, a, o);
        const int oarg = __shfl_xor_sync(0xffffffffu, arg, o);
        if (oa > a || (oa == a && oarg < arg)) {
          a = oa;
          arg = oarg;
        }
      }
      if (t == 0) {
        s_piv = arg;
        if (!(a > tiny)) s_bad = 1;
      }
    }
    __syncthreads();
    const int p = s_piv;
    if (p != j && t < 2 * GJB) {
      const double a = G[j][t];
      G[j][t] = G[p][t];
      G[p][t] = a;
    }
    __syncthreads();
    const double ip = 1.0 / G[j][j];
    if (t < GJB) fac[t] = t == j ? 0.0 : G[t][j];
    __syncthreads();
    if (t < 2 * GJB) G[j][t] *= ip;
    __syncthreads();
    for (int e = t; e < GJB * 2 * GJB; e += blockDim.x) {
      const int r = e / (2 * GJB), c = e % (2 * GJB);
      if (r != j) G[r][c] -= fac[r] * G[j][c];
    }
    __syncthreads();
  }
  for (int e = t; e < GJB * GJB; e += blockDim.x) Pinv[e] = G[e / GJB][GJB + e % GJB];
  if (t == 0 && (s_bad || !(amax > 0.0) || !isfinite(amax))) *flag = 1;
}

// T' (GJB rows of n) and C (n rows of GJB) of the panel at k0
__global__ void __launch_bounds__(256) k_bgj_panels(const double* __restrict__ M, int n, int k0, int bk,
                                                   const double* __restrict__ Pinv, double* __restrict__ T,
                                                   double* __restrict__ C) {
  __shared__ double Ps[GJB][GJB];
  for (int e = threadIdx.x; e < GJB * GJB; e += blockDim.x) Ps[e / GJB][e % GJB] = Pinv[e];
  __syncthreads();
  const size_t nt = size_t(n) * (GJB / 8);
  const size_t total = nt + size_t(n) * GJB;
  for (size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += size_t(gridDim.x) * blockDim.x) {
    if (e < nt) {
      // rows 8 kq .. 8 kq + 7 of T', column j
      const int j = int(e % n), kq = int(e / n);
      if (8 * kq >= bk) continue;
      double acc[8];
      if (j >= k0 && j < k0 + bk) {
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[q] = Ps[8 * kq + q][j - k0];
      } else {
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[q] = 0.0;
        for (int m = 0; m < bk; ++m) {
          const double v = M[size_t(k0 + m) * n + j];
#pragma unroll
          for (int q = 0; q < 8; ++q) acc[q] = fma(Ps[8 * kq + q][m], v, acc[q]);
        }
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) T[size_t(8 * kq + q) * n + j] = acc[q];
    } else {
      const size_t f = e - nt;
      const size_t i = f / GJB;
      const int m = int(f % GJB);
      C[f] = m < bk ? M[i * n + k0 + m] : 0.0;
    }
  }
}

// The update of one GJT x GJT tile of M (see above); 256 threads, 4 x 4
// entries each (rows ty + 16 p, columns tx + 16 q).
__global__ void __launch_bounds__(256) k_bgj_update(double* __restrict__ M, int n, int k0, int bk,
                                                   const double* __restrict__ T, const double* __restrict__ C) {
  __shared__ double As[GJT][GJB + 1];
  __shared__ double Bs[GJB][GJT];
  const int i0 = blockIdx.y * GJT, j0 = blockIdx.x * GJT;
  const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
  for (int e = t; e < GJT * GJB; e += blockDim.x) {
    const int r = e / GJB, m = e % GJB, i = i0 + r;
    As[r][m] = (i < n && m < bk) ? C[size_t(i) * GJB + m] : 0.0;
  }
  for (int e = t; e < GJB * GJT; e += blockDim.x) {
    const int m = e / GJT, cc = e % GJT, j = j0 + cc;
    Bs[m][cc] = (j < n && m < bk) ? T[size_t(m) * n + j] : 0.0;
  }
  __syncthreads();
  double acc[4][4];
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[p][q] = 0.0;
#pragma unroll 4
  for (int m = 0; m < GJB; ++m) {
    double a[4], b[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) a[p] = As[ty + 16 * p][m];
#pragma unroll
    for (int q = 0; q < 4; ++q) b[q] = Bs[m][tx + 16 * q];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[p][q] = fma(a[p], b[q], acc[p][q]);
  }
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int i = i0 + ty + 16 * p;
    if (i >= n) continue;
    const bool prow = i >= k0 && i < k0 + bk;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int j = j0 + tx + 16 * q;
      if (j >= n) continue;
      double& dst = M[size_t(i) * n + j];
      if (prow)
        dst = T[size_t(i - k0) * n + j];
      else
        dst = (j >= k0 && j < k0 + bk ? 0.0 : dst) - acc[p][q];
    }
  }
}

// M <- Q M Q with Q the transposition of indices a and b (a != b)
__global__ void k_swap_index(double* M, int n, int a, int b) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    if (k == a) {
      double& aa = M[size_t(a) * n + a];
      double& bb = M[size_t(b) * n + b];
      double& ab = M[size_t(a) * n + b];
      double& ba = M[size_t(b) * n + a];
      const double t0 = aa, t1 = ab;
      aa = bb;
      bb = t0;
      ab = ba;
      ba = t1;
    } else if (k != b) {
      double t0 = M[size_t(a) * n + k];
      M[size_t(a) * n + k] = M[size_t(b) * n + k];
      M[size_t(b) * n + k] = t0;
      t0 = M[size_t(k) * n + a];
      M[size_t(k) * n + a] = M[size_t(k) * n + b];
      M[size_t(k) * n + b] = t0;
    }
  }
}

// the probe vector of the inverse's check: v[i] = 1 + ((37 i) mod 101) / 101
__global__ void k_probe_fill(double* v, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    v[i] = 1.0 + double((37 * i) % 101) / 101.0;
}

// y = A x (n x n, row-major, FP64): one warp per row
__global__ void __launch_bounds__(NT) k_dgemv(const double* __restrict__ A, int n, const double* __restrict__ x,
                                              double* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int warps = blockDim.x >> 5;
  for (int row = blockIdx.x * warps + (threadIdx.x >> 5); row < n; row += gridDim.x * warps) {
    const double* a = A + size_t(row) * n;
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s = fma(a[j], x[j], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[row] = s;
  }
}

// *flag = 1 unless max |u - v| <= tol max |v| (one CTA)
__global__ void __launch_bounds__(NT) k_probe_check(const double* __restrict__ v, const double* __restrict__ u, int n,
                                                    double tol, int* flag) {
  __shared__ double red[64];
  double s[2] = {0.0, 0.0};
  for (int i = threadIdx.x; i < n; i += NT) {
    const double d = fabs(u[i] - v[i]);
    s[0] = (d > s[0] || d != d) ? d : s[0];
    s[1] = fmax(s[1], fabs(v[i]));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double a = __shfl_xor_sync(0xffffffffu, s[0], o), b = __shfl_xor_sync(0xffffffffu, s[1], o);
    s[0] = (a > s[0] || a != a) ? a : s[0];
    s[1] = fmax(s[1], b);
  }
  if ((threadIdx.x & 31) == 0) {
    red[2 * (threadIdx.x >> 5)] = s[0];
    red[2 * (threadIdx.x >> 5) + 1] = s[1];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double e = 0.0, vm = 0.0;
    for (int w = 0; w < NT / 32; ++w) {
      const double a = red[2 * w];
      e = (a > e || a != a) ? a : e;
      vm = fmax(vm, red[2 * w + 1]);
    }
    if (!(e <= tol * vm)) *flag = 1;
  }
}

// FP32 copy of a device array
__global__ void k_to_float(const double* __restrict__ a, size_t n, float* __restrict__ out) {
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    out[i] = float(a[i]);
}

// y = Ainv x (n x n, row-major): one warp per row
__global__ void __launch_bounds__(NT) k_coarse_gemv(const float* __restrict__ Ainv, const double* __restrict__ x,
                                                    int n, double* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int warps = blockDim.x >> 5;
  for (int row = blockIdx.x * warps + (threadIdx.x >> 5); row < n; row += gridDim.x * warps) {
    const float* a = Ainv + size_t(row) * n;
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s += double(a[j]) * __ldg(x + j);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[row] = s;
  }
}

// z += yc on every cell of its block
template <class T>
__global__ void k_coarse_prolong(int nb, const double* __restrict__ yc, T* __restrict__ z) {
  const size_t n = size_t(nb) * BN;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    z[i] = T(double(z[i]) + yc[i / BN]);
}

// *mean_sum += sum_I yc[I] w[I] (w = 512 h^3), one CTA, fixed order
__global__ void __launch_bounds__(NT) k_coarse_mean(int nb, const double* __restrict__ yc,
                                                    const double* __restrict__ w, double* mean_sum) {
  __shared__ double red[64];
  double s[1] = {0.0};
  for (int i = threadIdx.x; i < nb; i += NT) s[0] += yc[i] * w[i];
  block_reduce<1>(s, red);
  if (threadIdx.x == 0) *mean_sum += s[0];
}

}  // namespace

// A^-1 in place of the device matrix M = A (n x n, row-major).  First the
// blocked Gauss-Jordan above, with index `last` (when >= 0) swapped to the
// end of the pivot order, checked by A^-1 (A v) = v to 1e-6 for the probe
// vector v; when a pivot block has a small pivot or the check fails, the
// inverse is redone by column-wise Gauss-Jordan with partial pivoting
// (*fallback = 1).  Returns CUP_ERR_MESH for a singular matrix.
int device_inverse_dev(double* M, int n, int last, int sms, cudaStream_t s, int* fallback,
                       InverseScratch* scratch) {
  if (fallback) *fallback = 0;
  InverseScratch local;
  InverseScratch& X = scratch ? *scratch : local;
  if (X.cap < n) {
    X.arena.release();
    X.cap = 0;
    const size_t cap = scratch ? size_t(n) + n / 4 : size_t(n);
    if (int rc = X.arena.alloc(&X.M0, cap * cap)) return rc;
    if (int rc = X.arena.alloc(&X.Pinv, GJB * GJB)) return rc;
    if (int rc = X.arena.alloc(&X.T, size_t(GJB) * cap)) return rc;
    if (int rc = X.arena.alloc(&X.Cp, size_t(GJB) * cap)) return rc;
    if (int rc = X.arena.alloc(&X.pv, 3 * cap)) return rc;
    if (int rc = X.arena.alloc(&X.flag, 2)) return rc;
    X.cap = int(cap);
  }
  double *M0 = X.M0, *Pinv = X.Pinv, *T = X.T, *Cp = X.Cp, *pv = X.pv;
  int* flag = X.flag;
  const size_t nn = size_t(n) * n;
  DevArena tmp;  // the pivoted form's
  CUP_CUDA_TRY(cudaMemcpyAsync(M0, M, nn * sizeof(double), cudaMemcpyDeviceToDevice, s));
  CUP_CUDA_TRY(cudaMemsetAsync(flag, 0, 2 * sizeof(int), s));
  const int vg = std::max(1, std::min(sms * 8, (n + 7) / 8));
  {
    ProfScope ps("blocked_gauss_jordan_inverse", s);
    k_probe_fill<<<std::max(1, std::min(sms, (n + NT - 1) / NT)), NT, 0, s>>>(pv, n);
    k_dgemv<<<vg, NT, 0, s>>>(M0, n, pv, pv + n);
    const bool swap = last >= 0 && last != n - 1;
    const int sg = std::max(1, std::min(sms, (n + NT - 1) / NT));
    if (swap) k_swap_index<<<sg, NT, 0, s>>>(M, n, last, n - 1);
    const int tiles = (n + GJT - 1) / GJT;
    const int pg = int(std::max<size_t>(1, std::min<size_t>(size_t(sms) * 8, (size_t(n) * (GJB + GJB / 8) + 255) / 256)));
    for (int k0 = 0; k0 < n; k0 += GJB) {
      const int bk = std::min(GJB, n - k0);
      k_bgj_block_inverse<<<1, 256, 0, s>>>(M, n, k0, bk, Pinv, flag);
      k_bgj_panels<<<pg, 256, 0, s>>>(M, n, k0, bk, Pinv, T, Cp);
      k_bgj_update<<<dim3(tiles, tiles), 256, 0, s>>>(M, n, k0, bk, T, Cp);
    }
    if (swap) k_swap_index<<<sg, NT, 0, s>>>(M, n, last, n - 1);
    k_dgemv<<<vg, NT, 0, s>>>(M, n, pv + n, pv + 2 * size_t(n));
    k_probe_check<<<1, NT, 0, s>>>(pv, pv + 2 * size_t(n), n, 1e-6, flag + 1);
    CUP_CUDA_TRY(cudaGetLastError());
  }
  int h_flag[2] = {0, 0};
  CUP_CUDA_TRY(stream_d2h(s, h_flag, flag, sizeof(h_flag)));
  if (!h_flag[0] && !h_flag[1]) return 0;
  // column-wise Gauss-Jordan with partial pivoting on [A | I]
  if (fallback) *fallback = 1;
  double *G = nullptr, *fac = nullptr;
  int* sing = nullptr;
  if (int rc = tmp.alloc(&G, nn * 2)) return rc;
  if (int rc = tmp.alloc(&fac, n)) return rc;
  if (int rc = tmp.alloc(&sing, 1)) return rc;
  CUP_CUDA_TRY(cudaMemsetAsync(sing, 0, sizeof(int), s));
  {
    ProfScope ps("gauss_jordan_inverse", s);
    k_gj_augment<<<std::max(1, sms * 8), NT, 0, s>>>(M0, n, G);
    const int eg = std::max(1, sms * 8);
    for (int k = 0; k < n; ++k) {
      k_gj_pivot<<<1, 1024, 0, s>>>(G, n, k, fac, sing);
      k_gj_eliminate<<<eg, NT, 0, s>>>(G, n, k, fac);
    }
    CUP_CUDA_TRY(cudaGetLastError());
  }
  int h_sing = 0;
  CUP_CUDA_TRY(stream_d2h(s, &h_sing, sing, sizeof(int)));
  if (h_sing) return set_error(CUP_ERR_MESH, "Gauss-Jordan inverse: singular matrix");
  k_gj_extract<<<std::max(1, sms * 8), NT, 0, s>>>(G, n, M);
  CUP_CUDA_TRY(cudaGetLastError());
  CUP_CUDA_TRY(cudaStreamSynchronize(s));  // tmp is free to go
  return 0;
}

// Inverse of the n x n host matrix a (row-major) into d_inv (n x n, device).
int device_inverse(const double* a, int n, double* d_inv, int sms, cudaStream_t s) {
  CUP_CUDA_TRY(cudaMemcpyAsync(d_inv, a, size_t(n) * n * sizeof(double), cudaMemcpyHostToDevice, s));
  return device_inverse_dev(d_inv, n, -1, sms, s, nullptr);
}

// Builds the coarse space of the context's mesh (see above).
int coarse_build(cup_ctx* c) {
  CoarseSpace& C = c->coarse;
  const Mesh& m = c->mesh;
  const int nb = m.nb;
  if (C.nb == nb && C.mesh_version == c->mesh_version) return 0;
  if (nb > kCoarseMaxBlocks)
    return set_error(CUP_ERR_ARG, "two-level preconditioner: more blocks than the dense coarse solve takes (8192)");
  C.nb = 0;
  cudaStream_t s = c->stream;
  // block graph and its distance-2 colouring
  std::vector<std::vector<int>> adj(nb);
  for (int b = 0; b < nb; ++b) {
    std::set<int> nbr;
    for (int f = 0; f < 6; ++f) {
      const int k = m.face_kind[6 * b + f];
      const int* fn = &m.face_nbr[24 * b + 4 * f];
      if (k == FACE_SAME || k == FACE_COARSER) nbr.insert(fn[0]);
      if (k == FACE_FINER)
        for (int q = 0; q < 4; ++q) nbr.insert(fn[q]);
    }
    nbr.erase(b);
    adj[b].assign(nbr.begin(), nbr.end());
  }
  std::vector<int> colour(nb, -1);
  int ncol = 0;
  std::vector<int> mark;
  for (int b = 0; b < nb; ++b) {
    mark.assign(ncol + 1, 0);
    auto forbid = [&](int j) {
      if (colour[j] >= 0) mark[colour[j]] = 1;
    };
    for (int j : adj[b]) {
      forbid(j);
      for (int k : adj[j]) forbid(k);
    }
    int col = 0;
    while (mark[col]) ++col;
    colour[b] = col;
    ncol = std::max(ncol, col + 1);
  }
  // per colour: A applied to its indicator, summed per block, the sums
  // scattered into A_c on the device
  std::vector<double> w(nb);
  for (int b = 0; b < nb; ++b) w[b] = 512.0 * m.h[b] * m.h[b] * m.h[b];
  const int mb = m.mean_block;
  const int mode = c->cfg.mean_constraint;
  std::vector<int> jmap(size_t(ncol) * nb, -1);  // [colour][i]: the block of the colour at or next to i
  std::vector<double> wcol(ncol, 0.0);
  for (int b = 0; b < nb; ++b) wcol[colour[b]] += w[b];
  for (int i = 0; i < nb; ++i) {
    jmap[size_t(colour[i]) * nb + i] = i;
    for (int j : adj[i])
      if (jmap[size_t(colour[j]) * nb + i] < 0) jmap[size_t(colour[j]) * nb + i] = j;
  }
  // storage with room for C.cap blocks, allocated again only to grow
  const size_t nn = size_t(nb) * nb;
  if (C.cap < nb) {
    DevArena& A = C.arena;
    A.release();
    C.cap = 0;
    const size_t cap = size_t(nb) + nb / 4;
    if (int rc = A.alloc(&C.w, cap)) return rc;
    if (int rc = A.alloc(&C.rc, cap)) return rc;
    if (int rc = A.alloc(&C.yc, cap)) return rc;
    if (int rc = A.alloc(&C.rc2, cap)) return rc;
    if (int rc = A.alloc(&C.inv, cap * cap)) return rc;
    if (int rc = A.alloc(&C.ac, cap * cap)) return rc;
    if (int rc = A.alloc(&C.colour, cap)) return rc;
    if (int rc = A.alloc(&C.sum, cap)) return rc;
    C.cap = int(cap);
  }
  if (C.jcap < jmap.size()) {
    C.jarena.release();
    C.jcap = 0;
    if (int rc = C.jarena.alloc(&C.jmap, jmap.size() + jmap.size() / 4)) return rc;
    C.jcap = jmap.size() + jmap.size() / 4;
  }
  int* d_colour = C.colour;
  int* d_jmap = C.jmap;
  double* d_sum = C.sum;
  double* Ac = C.ac;
  CUP_CUDA_TRY(cudaMemcpyAsync(C.w, w.data(), nb * sizeof(double), cudaMemcpyHostToDevice, s));
  CUP_CUDA_TRY(cudaMemcpyAsync(d_colour, colour.data(), nb * sizeof(int), cudaMemcpyHostToDevice, s));
  CUP_CUDA_TRY(cudaMemcpyAsync(d_jmap, jmap.data(), jmap.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  CUP_CUDA_TRY(cudaMemsetAsync(Ac, 0, nn * sizeof(double), s));
  double* x = c->W.z1;
  double* y = c->W.z2;
  const int grid = std::max(1, std::min(c->num_sms * 8, (nb * BN + NT - 1) / NT));
  const int rgrid = std::max(1, std::min(c->num_sms, (nb + NT - 1) / NT));
  for (int col = 0; col < ncol; ++col) {
    k_colour_indicator<<<grid, NT, 0, s>>>(nb, d_colour, col, x);
    CUP_CUDA_TRY(cudaGetLastError());
    if (int rc = launch_poisson_apply(c->dm, x, y, mode, c->W, s)) return rc;
    k_block_sum<double><<<std::min(nb, c->num_sms * 8), NT, 0, s>>>(nb, y, d_sum);
    k_coarse_scatter<<<rgrid, NT, 0, s>>>(Ac, nb, d_jmap + size_t(col) * nb, d_sum, C.w, wcol[col], mode, mb);
    CUP_CUDA_TRY(cudaGetLastError());
  }
  if (mode == 1 || mode == 2) {
    k_coarse_dense<<<std::max(1, std::min(c->num_sms * 8, int((nn + NT - 1) / NT))), NT, 0, s>>>(Ac, nb, C.w, mode, mb);
    CUP_CUDA_TRY(cudaGetLastError());
  }
  if (C.keep_host) {
    C.host_ac.resize(nn);
    CUP_CUDA_TRY(stream_d2h(s, C.host_ac.data(), Ac, nn * sizeof(double)));
  } else {
    std::vector<double>().swap(C.host_ac);
  }
  // A_c^-1 on the device, the mean row's block last in the pivot order (the
  // other blocks' rows are those of a Laplacian); in FP64, kept in FP32: the
  // two coarse corrections of an iteration read it whole (8 nb^2 bytes each
  // in FP64, a large part of an iteration's traffic on meshes of a few
  // thousand blocks)
  {
    int fb = 0;
    if (int rc = device_inverse_dev(Ac, nb, mode == 1 ? mb : -1, c->num_sms, s, &fb, &C.iscratch))
      return rc == CUP_ERR_MESH ? set_error(CUP_ERR_MESH, "two-level preconditioner: singular coarse operator") : rc;
    C.pivoted = fb;
    k_to_float<<<std::max(1, c->num_sms * 8), NT, 0, s>>>(Ac, nn, C.inv);
    CUP_CUDA_TRY(cudaGetLastError());
    CUP_CUDA_TRY(cudaStreamSynchronize(s));
  }
  C.nb = nb;
  C.mesh_version = c->mesh_version;
  C.colours = ncol;
  return 0;
}

template <class T>
int coarse_apply(const CoarseView& C, const T* r, T* z, double* mean_sum, int sms, cudaStream_t s) {
  const int nb = C.nb;
  ProfScope ps("coarse_correction", s);
  k_block_sum<T><<<std::min(nb, sms * 8), NT, 0, s>>>(nb, r, C.rc);
  k_coarse_gemv<<<std::min((nb + 7) / 8, sms * 8), NT, 0, s>>>(C.inv, C.rc, nb, C.yc);
  const size_t n = size_t(nb) * BN;
  k_coarse_prolong<T><<<int(std::min<size_t>((n + NT - 1) / NT, size_t(sms) * 8)), NT, 0, s>>>(nb, C.yc, z);
  if (mean_sum) k_coarse_mean<<<1, NT, 0, s>>>(nb, C.yc, C.w, mean_sum);
  CUP_CUDA_TRY(cudaGetLastError());
  return 0;
}
template int coarse_apply<double>(const CoarseView&, const double*, double*, double*, int, cudaStream_t);
template int coarse_apply<float>(const CoarseView&, const float*, float*, double*, int, cudaStream_t);

}  // namespace cup3d

using namespace cup3d;

extern "C" {

int cup_coarse_matrix(cup_ctx* c, double* out, int32_t* colours) {
  ProfBind pb_(c);
  if (!c || c->mesh.nb == 0 || c->host_only || c->ncase > 1)
    return ctx_fail(c, CUP_ERR_ARG, "cup_coarse_matrix: bad arguments");
  if (!c->coarse.keep_host) {  // rebuilt once, keeping A_c on the host from now on
    c->coarse.keep_host = true;
    c->coarse.nb = 0;
  }
  if (int rc = coarse_build(c)) return ctx_fail(c, rc, cup_last_error(nullptr));
  if (out) std::copy(c->coarse.host_ac.begin(), c->coarse.host_ac.end(), out);
  if (colours) *colours = c->coarse.colours;
  return 0;
}

int cup_dense_inverse_dev(cup_ctx* c, double* d_a, int32_t n, int32_t last, int32_t* pivoted) {
  ProfBind pb_(c);
  if (!c || !d_a || n <= 0 || last < -1 || last >= n || c->host_only)
    return ctx_fail(c, CUP_ERR_ARG, "cup_dense_inverse_dev: bad arguments");
  int fb = 0;
  if (int rc = device_inverse_dev(d_a, n, last, c->num_sms, c->stream, &fb))
    return ctx_fail(c, rc, cup_last_error(nullptr));
  if (pivoted) *pivoted = fb;
  return 0;
}

int cup_coarse_apply_dev(cup_ctx* c, const double* d_r, double* d_z) {
  ProfBind pb_(c);
  if (!c || !d_r || !d_z || c->mesh.nb == 0 || c->host_only || c->ncase > 1)
    return ctx_fail(c, CUP_ERR_ARG, "cup_coarse_apply_dev: bad arguments");
  if (int rc = coarse_build(c)) return ctx_fail(c, rc, cup_last_error(nullptr));
  CUP_CUDA_TRY(cudaMemsetAsync(d_z, 0, nbn(c) * sizeof(double), c->stream));
  const CoarseView v = c->coarse.view();
  if (int rc = coarse_apply<double>(v, d_r, d_z, nullptr, c->num_sms, c->stream))
    return ctx_fail(c, rc, cup_last_error(nullptr));
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return ctx_fail(c, set_cuda_error(e, "coarse_apply", __FILE__, __LINE__), cup_last_error(nullptr));
  return 0;
}

}  // extern "C"
