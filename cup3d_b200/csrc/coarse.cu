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
//   * A_c^-1 by Gauss-Jordan elimination with partial pivoting on the device
//     (nb steps of a pivot kernel and a rank-one elimination kernel).
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

// Inverse of the n x n host matrix a (row-major) by Gauss-Jordan with partial
// pivoting on the device, into d_inv (n x n, device, row-major); returns
// CUP_ERR_MESH for a singular matrix.
int device_inverse(const double* a, int n, double* d_inv, int sms, cudaStream_t s) {
  DevArena tmp;
  double *G = nullptr, *fac = nullptr;
  int* sing = nullptr;
  if (int rc = tmp.alloc(&G, size_t(n) * 2 * n)) return rc;
  if (int rc = tmp.alloc(&fac, n)) return rc;
  if (int rc = tmp.alloc(&sing, 1)) return rc;
  {
    std::vector<double> Gh(size_t(n) * 2 * n, 0.0);
    for (int i = 0; i < n; ++i) {
      std::copy(a + size_t(i) * n, a + size_t(i) * n + n, &Gh[size_t(i) * 2 * n]);
      Gh[size_t(i) * 2 * n + n + i] = 1.0;
    }
    CUP_CUDA_TRY(stream_h2d(s, G, Gh.data(), Gh.size() * sizeof(double)));
  }
  CUP_CUDA_TRY(stream_zero(s, sing, sizeof(int)));
  {
    ProfScope ps("gauss_jordan_inverse", s);
    const int eg = std::max(1, sms * 8);
    for (int k = 0; k < n; ++k) {
      k_gj_pivot<<<1, 1024, 0, s>>>(G, n, k, fac, sing);
      k_gj_eliminate<<<eg, NT, 0, s>>>(G, n, k, fac);
    }
    CUP_CUDA_TRY(cudaGetLastError());
  }
  int h_sing = 0;
  CUP_CUDA_TRY(stream_d2h(s, &h_sing, sing, sizeof(int)));  // synchronises: tmp is free to go
  if (h_sing) return set_error(CUP_ERR_MESH, "Gauss-Jordan inverse: singular matrix");
  k_gj_extract<<<std::max(1, sms * 8), NT, 0, s>>>(G, n, d_inv);
  CUP_CUDA_TRY(cudaGetLastError());
  CUP_CUDA_TRY(cudaStreamSynchronize(s));
  return 0;
}

// Builds the coarse space of the context's mesh (see above).
int coarse_build(cup_ctx* c) {
  CoarseSpace& C = c->coarse;
  const Mesh& m = c->mesh;
  const int nb = m.nb;
  if (C.nb == nb && C.mesh_version == c->mesh_version) return 0;
  if (nb > kCoarseMaxBlocks)
    return set_error(CUP_ERR_ARG, "two-level preconditioner: more blocks than the dense coarse solve takes (8192)");
  C.arena.release();
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
  // per colour: A applied to its indicator, summed per block
  DevArena tmp;
  int* d_colour = nullptr;
  double* d_sum = nullptr;
  if (int rc = tmp.alloc(&d_colour, nb)) return rc;
  if (int rc = tmp.alloc(&d_sum, nb)) return rc;
  CUP_CUDA_TRY(stream_h2d(s, d_colour, colour.data(), nb * sizeof(int)));
  std::vector<double> Ac(size_t(nb) * nb, 0.0), sums(nb);
  std::vector<double> w(nb);
  for (int b = 0; b < nb; ++b) w[b] = 512.0 * m.h[b] * m.h[b] * m.h[b];
  const int mb = m.mean_block;
  const int mode = c->cfg.mean_constraint;
  std::vector<std::vector<int>> members(ncol);
  for (int b = 0; b < nb; ++b) members[colour[b]].push_back(b);
  double* x = c->W.z1;
  double* y = c->W.z2;
  const int grid = std::max(1, std::min(c->num_sms * 8, (nb * BN + NT - 1) / NT));
  for (int col = 0; col < ncol; ++col) {
    k_colour_indicator<<<grid, NT, 0, s>>>(nb, d_colour, col, x);
    CUP_CUDA_TRY(cudaGetLastError());
    if (int rc = launch_poisson_apply(c->dm, x, y, mode, c->W, s)) return rc;
    k_block_sum<double><<<std::min(nb, c->num_sms * 8), NT, 0, s>>>(nb, y, d_sum);
    CUP_CUDA_TRY(cudaGetLastError());
    CUP_CUDA_TRY(stream_d2h(s, sums.data(), d_sum, nb * sizeof(double)));
    double wcol = 0.0;
    for (int j : members[col]) wcol += w[j];
    for (int i = 0; i < nb; ++i) {
      // the one block of this colour at or next to i
      int J = colour[i] == col ? i : -1;
      if (J < 0)
        for (int j : adj[i])
          if (colour[j] == col) {
            J = j;
            break;
          }
      // known dense parts of the row: mode 1, the mean row of block mb adds
      // 512 h_J^3 for every J; mode 2, every row adds 512 h_I^3 512 h_J^3
      double known_i = 0.0;
      if (mode == 1 && i == mb) {
        known_i = wcol;
        for (int j : members[col]) Ac[size_t(i) * nb + j] += w[j];
      } else if (mode == 2) {
        known_i = w[i] * wcol;
        for (int j : members[col]) Ac[size_t(i) * nb + j] += w[i] * w[j];
      }
      if (J >= 0) Ac[size_t(i) * nb + J] += sums[i] - known_i;
    }
  }
  // A_c^-1 by Gauss-Jordan on the device
  // in FP64, kept in FP32: the two coarse corrections of an iteration read
  // it whole (8 nb^2 bytes each in FP64, a large part of an iteration's
  // traffic on meshes of a few thousand blocks)
  DevArena& A = C.arena;
  {
    DevArena tinv;
    double* inv64 = nullptr;
    if (int rc = tinv.alloc(&inv64, size_t(nb) * nb)) return rc;
    if (int rc = device_inverse(Ac.data(), nb, inv64, c->num_sms, s))
      return rc == CUP_ERR_MESH ? set_error(CUP_ERR_MESH, "two-level preconditioner: singular coarse operator") : rc;
    if (int rc = A.alloc(&C.inv, size_t(nb) * nb)) return rc;
    k_to_float<<<std::max(1, c->num_sms * 8), NT, 0, s>>>(inv64, size_t(nb) * nb, C.inv);
    CUP_CUDA_TRY(cudaGetLastError());
    CUP_CUDA_TRY(cudaStreamSynchronize(s));
  }
  if (int rc = A.alloc(&C.rc, nb)) return rc;
  if (int rc = A.alloc(&C.yc, nb)) return rc;
  if (int rc = A.alloc(&C.rc2, nb)) return rc;
  if (int rc = A.alloc(&C.w, nb)) return rc;
  CUP_CUDA_TRY(stream_h2d(s, C.w, w.data(), nb * sizeof(double)));
  C.host_ac.swap(Ac);
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
  if (int rc = coarse_build(c)) return ctx_fail(c, rc, cup_last_error(nullptr));
  if (out) std::copy(c->coarse.host_ac.begin(), c->coarse.host_ac.end(), out);
  if (colours) *colours = c->coarse.colours;
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
