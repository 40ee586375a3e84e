// Learned block preconditioner: CNN inference, training and data gathering.
// The two C->C layers (and their backward passes) run on BF16 tensor cores
// with FP32 accumulation (ldmatrix + mma.sync.m16n8k16); the 1->C and C->1
// layers (27 and 432 MACs per output) run on the FP32 pipes.  See cnn.cuh.
#include <cuda_bf16.h>

#include "cnn.cuh"
#include "fd.cuh"
#include "lab.cuh"
#include "lmap.cuh"
#include "profiler.h"

namespace cup3d {

// ---------------------------------------------------------------------------
// Shared-memory activation layout: two channel halves, padded 10^3 volume,
// 8 BF16 channels per voxel (16 B rows, the ldmatrix row size).
// ---------------------------------------------------------------------------
constexpr int PV = 1000;  // padded voxels
__device__ __forceinline__ int pv(int x, int y, int z) { return (x + 1) + 10 * ((y + 1) + 10 * (z + 1)); }
__device__ __forceinline__ int pv_of_cell(int c) { return pv(c & 7, (c >> 3) & 7, c >> 6); }

struct Act {
  uint16_t v[2][PV][8];
};

__device__ __forceinline__ uint16_t f2bf(float f) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(f));
}
__device__ __forceinline__ float bf2f(uint16_t u) { return __bfloat162float(__ushort_as_bfloat16(u)); }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t r[4]) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(addr));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t addr, uint32_t r[4]) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(addr));
}
__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void zero_act(Act& a) {
  uint32_t* p = reinterpret_cast<uint32_t*>(&a);
  for (int i = threadIdx.x; i < int(sizeof(Act) / 4); i += blockDim.x) p[i] = 0u;
}

// out = in (*) W on the 8^3 interior: C->C, 3^3 'same' (in's zero border is
// the padding), stored BF16.  W: [tap][co][ci] BF16 in shared memory.  8
// warps, each owns 4 M-tiles of 16 voxels; both N-tiles (co 0-7, 8-15).  The
// backward-data pass runs it with the flipped, transposed kernel.
__device__ void conv_cc(const Act& in, const uint16_t* Wsm, Act& out) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float acc[4][2][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[i][j][k] = 0.f;
  const int lm = lane >> 3, lr = lane & 7;
  for (int tap = 0; tap < 27; ++tap) {
    const int dx = tap % 3 - 1, dy = (tap / 3) % 3 - 1, dz = tap / 9 - 1;
    uint32_t b[4];
    {
      // matrices: (co 0-7, ci 0-7), (co 0-7, ci 8-15), (co 8-15, ci 0-7), (co 8-15, ci 8-15)
      const int co = (lm >> 1) * 8 + lr, ci0 = (lm & 1) * 8;
      ldsm_x4(smem_u32(Wsm + (tap * 16 + co) * 16 + ci0), b);
    }
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) {
      const int base = 16 * (4 * warp + mt);
      // matrices: (rows 0-7, ci 0-7), (rows 8-15, ci 0-7), (rows 0-7, ci 8-15), (rows 8-15, ci 8-15)
      const int vox = base + lr + 8 * (lm & 1), half = lm >> 1;
      const int x = (vox & 7) + dx, y = ((vox >> 3) & 7) + dy, z = (vox >> 6) + dz;
      uint32_t a[4];
      ldsm_x4(smem_u32(&in.v[half][pv(x, y, z)][0]), a);
      mma_bf16(acc[mt][0], a, b[0], b[1]);
      mma_bf16(acc[mt][1], a, b[2], b[3]);
    }
  }
  const int g = lane >> 2, tq = lane & 3;
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt)
#pragma unroll
      for (int hr = 0; hr < 2; ++hr) {
        const int vox = 16 * (4 * warp + mt) + g + 8 * hr;
        const int co = nt * 8 + 2 * tq;
        const float v0 = acc[mt][nt][2 * hr], v1 = acc[mt][nt][2 * hr + 1];
        const int p = pv_of_cell(vox);
        const uint32_t packed = uint32_t(f2bf(v0)) | (uint32_t(f2bf(v1)) << 16);
        *reinterpret_cast<uint32_t*>(&out.v[nt][p][2 * tq]) = packed;
      }
}

// Layer 0: 1 -> C, 'valid' 3^3 conv of the 10^3 input, into act (BF16).
__device__ void conv_in(const float* x0, const float* W0, Act& out) {
  for (int c = threadIdx.x; c < BN; c += blockDim.x) {
    const int x = c & 7, y = (c >> 3) & 7, z = c >> 6;
    float acc[CNN_C];
#pragma unroll
    for (int co = 0; co < CNN_C; ++co) acc[co] = 0.f;
    for (int tap = 0; tap < 27; ++tap) {
      const int dx = tap % 3, dy = (tap / 3) % 3, dz = tap / 9;
      const float xv = x0[(x + dx) + 10 * ((y + dy) + 10 * (z + dz))];
#pragma unroll
      for (int co = 0; co < CNN_C; ++co) acc[co] = fmaf(W0[co * 27 + tap], xv, acc[co]);
    }
    const int p = pv(x, y, z);
#pragma unroll
    for (int co = 0; co < CNN_C; ++co) out.v[co >> 3][p][co & 7] = f2bf(acc[co]);
  }
}

// Layer 3: C -> 1, 'same' 3^3 conv, FP32 output z[512].
__device__ void conv_out(const Act& in, const float* W3, float* z) {
  for (int c = threadIdx.x; c < BN; c += blockDim.x) {
    const int x = c & 7, y = (c >> 3) & 7, zz = c >> 6;
    float acc = 0.f;
    for (int tap = 0; tap < 27; ++tap) {
      const int dx = tap % 3 - 1, dy = (tap / 3) % 3 - 1, dz = tap / 9 - 1;
      const int p = pv(x + dx, y + dy, zz + dz);
#pragma unroll
      for (int ci = 0; ci < CNN_C; ++ci) acc = fmaf(W3[ci * 27 + tap], bf2f(in.v[ci >> 3][p][ci & 7]), acc);
    }
    z[c] = acc;
  }
}

struct FwdSmem {
  Act a, b;
  float x0[PV];
  float z[BN];
  uint16_t w1[27 * 16 * 16];
  uint16_t w2[27 * 16 * 16];
  float w0[CNN_W0], w3[CNN_W3];
  double red[64];
};

__device__ void load_weights(FwdSmem& S, const CnnWeights& W) {
  for (int i = threadIdx.x; i < 27 * 256; i += blockDim.x) {
    S.w1[i] = W.w1_bf16[i];
    S.w2[i] = W.w2_bf16[i];
  }
  const float* m = W.master;
  for (int i = threadIdx.x; i < CNN_W0; i += blockDim.x) S.w0[i] = m[OFF_W0 + i];
  for (int i = threadIdx.x; i < CNN_W3; i += blockDim.x) S.w3[i] = m[OFF_W3 + i];
}

// full forward on S.x0 (already normalised) -> S.z; leaves L2 output in S.a
__device__ void forward_block(FwdSmem& S) {
  conv_in(S.x0, S.w0, S.a);
  __syncthreads();
  conv_cc(S.a, S.w1, S.b);
  __syncthreads();
  conv_cc(S.b, S.w2, S.a);
  __syncthreads();
  conv_out(S.a, S.w3, S.z);
  __syncthreads();
}

// Input of one block: its residual lab (block + one-cell face layers, the
// rules of lmap.cuh; edges and corners zero), divided by its RMS; returns
// the RMS.  labd holds the star lab (LabGeom<1>: the block, then its six
// face layers), which is expanded into the 10^3 cube x0.
template <class T>
__device__ float gather_input(const DevMesh& M, int b, const T* v, float* x0, double* labd, double* red,
                              int mean_blk) {
  using LG = LabGeom<1>;
  __shared__ LabMeta meta;
  __syncthreads();
  if (threadIdx.x < 64) lab_meta_load(meta, M, b, threadIdx.x);
  __syncthreads();
  for (int i = threadIdx.x; i < LG::V; i += blockDim.x) {
    const int g = i - BN;
    labd[i] = i < BN ? double(v[size_t(b) * BN + i]) : rlab_ghost(v, meta, g >> 6, g & 7, (g >> 3) & 7, mean_blk);
  }
  __syncthreads();
  double acc[1] = {0.0};
  for (int i = threadIdx.x; i < LG::V; i += blockDim.x) acc[0] += labd[i] * labd[i];
  block_reduce<1>(acc, red);
  __shared__ double s_rms;
  if (threadIdx.x == 0) s_rms = sqrt(acc[0] / PV);
  __syncthreads();
  const double rms = s_rms;
  const double inv = rms > 0 ? 1.0 / rms : 0.0;
  for (int i = threadIdx.x; i < PV; i += blockDim.x) {
    const int x = i % 10 - 1, y = (i / 10) % 10 - 1, z = i / 100 - 1;
    const int outside = (x < 0 || x > 7) + (y < 0 || y > 7) + (z < 0 || z > 7);
    x0[i] = outside > 1 ? 0.f : float(labd[LG::at(x, y, z)] * inv);
  }
  __syncthreads();
  return float(rms);
}

// Block inverse of the normalised input's interior (FdSmem aliased onto an
// activation buffer that is free at this point); result zbj[512] = BJ(x0).
__device__ void block_jacobi_of_input(const float* x0, double h, FdSmem& fs, double* zbj) {
  fd_load_scale(fs);
  for (int c = threadIdx.x; c < BN; c += blockDim.x)
    fs.a[c] = double(x0[((c & 7) + 1) + 10 * ((((c >> 3) & 7) + 1) + 10 * ((c >> 6) + 1))]);
  __syncthreads();
  fd_apply(fs, -1.0 / h);
  for (int c = threadIdx.x; c < BN; c += blockDim.x) zbj[c] = fs.a[c];
  __syncthreads();
}

struct ApplySmem {
  FwdSmem f;
  double zbj[BN];
};

// z = BJ(r) + (s/h) CNN(r_lab / s) per block, and sum(z h^3) for the mean
// constraint of the SpMV that follows (into *mean_sum when given).
template <class T>
__global__ void __launch_bounds__(NT, 1) k_cnn_apply(DevMesh M, const T* __restrict__ r, T* __restrict__ zout,
                                                     CnnWeights W, GridReduce G, double* mean_sum, int mean_blk) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ApplySmem& A = *reinterpret_cast<ApplySmem*>(smem_raw);
  FwdSmem& S = A.f;
  double* labd = reinterpret_cast<double*>(&S.b);  // gather scratch (8 KB of the free act buffer)
  FdSmem& fs = *reinterpret_cast<FdSmem*>(&S.b);  // block-inverse scratch (12 KB), used after the gather
  load_weights(S, W);
  double acc[1] = {0.0};
  for (int b = blockIdx.x; b < M.nb; b += gridDim.x) {
    __syncthreads();
    const float rms = gather_input<T>(M, b, r, S.x0, labd, S.red, mean_blk);
    const double h = M.h[b];
    if (rms > 0.f) block_jacobi_of_input(S.x0, h, fs, A.zbj);
    zero_act(S.a);
    zero_act(S.b);
    __syncthreads();
    if (rms > 0.f) forward_block(S);
    double sum = 0.0;
    for (int c = threadIdx.x; c < BN; c += NT) {
      const T v = rms > 0.f ? T(double(rms) * (A.zbj[c] + double(S.z[c]) / h)) : T(0);
      zout[size_t(b) * BN + c] = v;
      sum += double(v);
    }
    acc[0] += sum * h * h * h;
  }
  __shared__ double red[64];
  if (grid_reduce<1>(acc, G, red) && threadIdx.x == 0 && mean_sum) *mean_sum = acc[0];
}

template <class T>
int cnn_apply(const DevMesh& M, const T* r, T* z, const CnnWeights& W, int grid, cudaStream_t s, GridReduce G,
              double* mean_sum, int mean_blk) {
  fd_init_constants();
  const size_t smem = sizeof(ApplySmem);
  static unsigned long long attr = 0;
  if (first_on_device(attr))
    CUP_CUDA_TRY(cudaFuncSetAttribute(k_cnn_apply<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  ProfScope ps(sizeof(T) == 4 ? "cnn_precond_apply_f32io" : "cnn_precond_apply_f64io", s);
  k_cnn_apply<T><<<grid, NT, smem, s>>>(M, r, z, W, G, mean_sum, mean_blk);
  CUP_CUDA_TRY(cudaGetLastError());
  return 0;
}
template int cnn_apply<double>(const DevMesh&, const double*, double*, const CnnWeights&, int, cudaStream_t,
                               GridReduce, double*, int);
template int cnn_apply<float>(const DevMesh&, const float*, float*, const CnnWeights&, int, cudaStream_t,
                              GridReduce, double*, int);

// Training samples from a residual r and a correction field corr (in the
// units of A^-1 r): input = gather(r)/s, target = corr h / s on the block.
__global__ void __launch_bounds__(NT) k_cnn_dataset(DevMesh M, const double* __restrict__ r,
                                                    const double* __restrict__ corr, float* in, float* target,
                                                    int base, int cap, int* count, int mean_blk) {
  __shared__ double labd[PV];
  __shared__ double red[64];
  __shared__ float x0[PV];
  for (int b = blockIdx.x; b < M.nb; b += gridDim.x) {
    const int slot = base + b;
    if (slot >= cap) break;
    __syncthreads();
    const float rms = gather_input<double>(M, b, r, x0, labd, red, mean_blk);
    const double h = M.h[b];
    const bool live = rms > 0.f;  // uniform across the CTA
    for (int i = threadIdx.x; i < PV; i += NT) in[size_t(slot) * PV + i] = live ? x0[i] : 0.f;
    for (int c = threadIdx.x; c < BN; c += NT)
      target[size_t(slot) * BN + c] = live ? float(corr[size_t(b) * BN + c] * h / double(rms)) : 0.f;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *count = min(cap, base + M.nb);
}

int cnn_dataset_add(const DevMesh& M, const double* r, const double* corr, float* in, float* target, int base,
                    int cap, int* count_dev, int grid, cudaStream_t s, int mean_blk) {
  ProfScope ps("cnn_dataset_add", s);
  k_cnn_dataset<<<grid, NT, 0, s>>>(M, r, corr, in, target, base, cap, count_dev, mean_blk);
  CUP_CUDA_TRY(cudaGetLastError());
  return 0;
}

// BF16 copies: w[tap][co][ci] from master [co][ci][tap]; wt[tap'][ci][co] with
// tap' = 26 - tap (flipped kernel) for the backward-data convolution.
__global__ void k_cnn_pack(const float* m, uint16_t* w1, uint16_t* w2, uint16_t* w1t, uint16_t* w2t) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 27 * 256; i += gridDim.x * blockDim.x) {
    const int tap = i / 256, co = (i / 16) % 16, ci = i % 16;
    w1[i] = f2bf(m[OFF_W1 + (co * 16 + ci) * 27 + tap]);
    w2[i] = f2bf(m[OFF_W2 + (co * 16 + ci) * 27 + tap]);
    // transposed: index i = (tap' * 16 + ci') * 16 + co' holds W[co'][ci'][26 - tap']
    const int tp = tap, cip = co, cop = ci;
    w1t[i] = f2bf(m[OFF_W1 + (cop * 16 + cip) * 27 + (26 - tp)]);
    w2t[i] = f2bf(m[OFF_W2 + (cop * 16 + cip) * 27 + (26 - tp)]);
  }
}

int cnn_pack(const CnnWeights& W, cudaStream_t s) {
  k_cnn_pack<<<27, 256, 0, s>>>(W.master, W.w1_bf16, W.w2_bf16, W.w1t_bf16, W.w2t_bf16);
  CUP_CUDA_TRY(cudaGetLastError());
  return 0;
}

// ---------------------------------------------------------------------------
// Training.  One CTA per sample (grid-stride): forward keeping the three
// hidden activations in shared memory, backward with the C->C layers on the
// tensor cores, per-CTA gradient partials in global memory (no atomics),
// then a fixed-order reduction and an Adam update.
// ---------------------------------------------------------------------------
struct TrainSmem {
  Act a1, a2, a3;     // hidden activations (BF16, zero border)
  Act d, e;           // gradient buffers (BF16, zero border)
  float x0[PV];
  float z[BN];        // output, then dL/dz
  float etmp[BN], rtmp[BN];  // residual-norm loss: error, then its block Laplacian
  uint16_t w1[27 * 256], w2[27 * 256], w1t[27 * 256], w2t[27 * 256];
  float w0[CNN_W0], w3[CNN_W3];
  float red[64];
};

// weight gradient of a C->C layer: dW[tap][co][ci] += sum_v in[v+tap][ci] dout[v][co].
// Tensor cores: M = co (16), N = ci (two n8 tiles), K = voxels (32 steps of
// 16).  Warp w handles taps w, w+8, ...
__device__ void wgrad_cc(const Act& in, const Act& dpre, float* gW /* master layout [co][ci][tap] */) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int lm = lane >> 3, lr = lane & 7, g = lane >> 2, tq = lane & 3;
  for (int tap = warp; tap < 27; tap += 8) {
    const int dx = tap % 3 - 1, dy = (tap / 3) % 3 - 1, dz = tap / 9 - 1;
    float acc[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
    for (int kb = 0; kb < BN; kb += 16) {
      // A (M=co x K=vox) from dpre via transposed loads:
      // matrices (co 0-7, v 0-7), (co 8-15, v 0-7), (co 0-7, v 8-15), (co 8-15, v 8-15)
      uint32_t a[4];
      {
        const int vox = kb + lr + 8 * (lm >> 1), half = lm & 1;
        ldsm_x4_t(smem_u32(&dpre.v[half][pv_of_cell(vox)][0]), a);
      }
      // B (K=vox x N=ci) from in at v+tap via transposed loads:
      // matrices (v 0-7, ci 0-7), (v 8-15, ci 0-7), (v 0-7, ci 8-15), (v 8-15, ci 8-15)
      uint32_t b[4];
      {
        const int vox = kb + lr + 8 * (lm & 1), half = lm >> 1;
        const int x = (vox & 7) + dx, y = ((vox >> 3) & 7) + dy, z = (vox >> 6) + dz;
        ldsm_x4_t(smem_u32(&in.v[half][pv(x, y, z)][0]), b);
      }
      mma_bf16(acc[0], a, b[0], b[1]);
      mma_bf16(acc[1], a, b[2], b[3]);
    }
    // c0,c1: (co = g, ci = nt*8 + 2tq, +1); c2,c3: (co = g + 8, ...)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt)
#pragma unroll
      for (int hr = 0; hr < 2; ++hr) {
        const int co = g + 8 * hr, ci = nt * 8 + 2 * tq;
        gW[(co * 16 + ci) * 27 + tap] += acc[nt][2 * hr];
        gW[(co * 16 + ci + 1) * 27 + tap] += acc[nt][2 * hr + 1];
      }
  }
}

__device__ void load_train_weights(TrainSmem& S, const CnnWeights& W) {
  for (int i = threadIdx.x; i < 27 * 256; i += blockDim.x) {
    S.w1[i] = W.w1_bf16[i];
    S.w2[i] = W.w2_bf16[i];
    S.w1t[i] = W.w1t_bf16[i];
    S.w2t[i] = W.w2t_bf16[i];
  }
  const float* m = W.master;
  for (int i = threadIdx.x; i < CNN_W0; i += blockDim.x) S.w0[i] = m[OFF_W0 + i];
  for (int i = threadIdx.x; i < CNN_W3; i += blockDim.x) S.w3[i] = m[OFF_W3 + i];
}

// grad_partial row of this CTA accumulates dL/dparams over its samples.
// loss partial (sum of squared errors) into lpart[blockIdx].  out (optional):
// network outputs of the samples.
// Block Laplacian of v (8^3, zero outside the block): 6 v - sum of the six neighbours.
__device__ __forceinline__ float block_lap(const float* v, int c) {
  const int x = c & 7, y = (c >> 3) & 7, z = c >> 6;
  float s = 6.f * v[c];
  if (x > 0) s -= v[c - 1];
  if (x < 7) s -= v[c + 1];
  if (y > 0) s -= v[c - 8];
  if (y < 7) s -= v[c + 8];
  if (z > 0) s -= v[c - 64];
  if (z < 7) s -= v[c + 64];
  return s;
}

// loss_mode 0: mean squared error of the output against the target;
// loss_mode 1: the residual norm |L (z - t)|^2 with L the block Laplacian
// (zero outside the block), the quantity a preconditioner's error costs the
// Krylov method: grid-scale errors weigh by their eigenvalue.  zero_pred: the
// loss of the prediction z = 0 (the targets' own norm, for relative losses).
__global__ void __launch_bounds__(NT, 1) k_cnn_train(CnnWeights W, const float* __restrict__ in,
                                                     const float* __restrict__ target, float tscale,
                                                     const int* __restrict__ idx, int n, float grad_scale,
                                                     float* gpart, float* lpart, float* out, int backward,
                                                     int loss_mode, int zero_pred) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TrainSmem& S = *reinterpret_cast<TrainSmem*>(smem_raw);
  load_train_weights(S, W);
  float* gp = gpart + size_t(blockIdx.x) * CNN_NPARAM;
  if (backward)
    for (int i = threadIdx.x; i < CNN_NPARAM; i += NT) gp[i] = 0.f;
  float loss = 0.f;
  for (int sidx = blockIdx.x; sidx < n; sidx += gridDim.x) {
    const int smp = idx ? idx[sidx] : sidx;
    __syncthreads();
    for (int i = threadIdx.x; i < PV; i += NT) S.x0[i] = in[size_t(smp) * PV + i];
    zero_act(S.a1);
    zero_act(S.a2);
    zero_act(S.a3);
    zero_act(S.d);
    zero_act(S.e);
    __syncthreads();
    conv_in(S.x0, S.w0, S.a1);
    __syncthreads();
    conv_cc(S.a1, S.w1, S.a2);
    __syncthreads();
    conv_cc(S.a2, S.w2, S.a3);
    __syncthreads();
    conv_out(S.a3, S.w3, S.z);
    __syncthreads();
    if (loss_mode == 0) {
      // dL/dz = grad_scale * 2 (z - t); loss += (z - t)^2
      for (int c = threadIdx.x; c < BN; c += NT) {
        const float zc = zero_pred ? 0.f : S.z[c];
        const float e = zc - (target ? tscale * target[size_t(smp) * BN + c] : 0.f);
        if (out) out[size_t(sidx) * BN + c] = S.z[c];
        loss += e * e;
        S.z[c] = grad_scale * 2.f * e;
      }
    } else {
      // dL/dz = grad_scale * 2 L^T L (z - t) (L symmetric); loss += |L (z - t)|^2
      for (int c = threadIdx.x; c < BN; c += NT) {
        const float zc = zero_pred ? 0.f : S.z[c];
        if (out) out[size_t(sidx) * BN + c] = S.z[c];
        S.etmp[c] = zc - (target ? tscale * target[size_t(smp) * BN + c] : 0.f);
      }
      __syncthreads();
      for (int c = threadIdx.x; c < BN; c += NT) {
        const float r = block_lap(S.etmp, c);
        S.rtmp[c] = r;
        loss += r * r;
      }
      __syncthreads();
      for (int c = threadIdx.x; c < BN; c += NT) S.z[c] = grad_scale * 2.f * block_lap(S.rtmp, c);
    }
    __syncthreads();
    if (!backward) continue;
    // ---- layer 3 (C -> 1): dW3[ci][tap] = sum_v a3[v+tap][ci] dz[v]
    for (int i = threadIdx.x; i < CNN_W3; i += NT) {
      const int ci = i / 27, tap = i % 27;
      const int dx = tap % 3 - 1, dy = (tap / 3) % 3 - 1, dz = tap / 9 - 1;
      float s = 0.f;
      for (int c = 0; c < BN; ++c) {
        const int x = (c & 7) + dx, y = ((c >> 3) & 7) + dy, z = (c >> 6) + dz;
        s = fmaf(bf2f(S.a3.v[ci >> 3][pv(x, y, z)][ci & 7]), S.z[c], s);
      }
      gp[OFF_W3 + i] += s;
    }
    // da3[u][ci] = sum_tap W3[ci][tap] dz[u - (tap-1)] -> S.d (BF16)
    for (int c = threadIdx.x; c < BN; c += NT) {
      const int x = c & 7, y = (c >> 3) & 7, zz = c >> 6;
      float acc[CNN_C];
#pragma unroll
      for (int ci = 0; ci < CNN_C; ++ci) acc[ci] = 0.f;
      for (int tap = 0; tap < 27; ++tap) {
        const int X = x - (tap % 3 - 1), Y = y - ((tap / 3) % 3 - 1), Z = zz - (tap / 9 - 1);
        if (X < 0 || Y < 0 || Z < 0 || X > 7 || Y > 7 || Z > 7) continue;
        const float dzv = S.z[X + 8 * Y + 64 * Z];
#pragma unroll
        for (int ci = 0; ci < CNN_C; ++ci) acc[ci] = fmaf(S.w3[ci * 27 + tap], dzv, acc[ci]);
      }
      const int p = pv(x, y, zz);
#pragma unroll
      for (int ci = 0; ci < CNN_C; ++ci) {
        S.d.v[ci >> 3][p][ci & 7] = f2bf(acc[ci]);
      }
    }
    __syncthreads();
    // ---- layer 2 (C -> C): weight gradient from a2 and dpre3 (S.d)
    wgrad_cc(S.a2, S.d, gp + OFF_W2);
    __syncthreads();
    // da2 = W2^T (*) da3 -> S.e
    conv_cc(S.d, S.w2t, S.e);
    __syncthreads();
    // ---- layer 1 (C -> C)
    wgrad_cc(S.a1, S.e, gp + OFF_W1);
    __syncthreads();
    conv_cc(S.e, S.w1t, S.d);  // da1 -> S.d
    __syncthreads();
    // ---- layer 0 (1 -> C): dW0[co][tap] = sum_v x0[v+tap] da1[v][co]
    for (int i = threadIdx.x; i < CNN_W0; i += NT) {
      const int co = i / 27, tap = i % 27;
      const int dx = tap % 3, dy = (tap / 3) % 3, dz = tap / 9;
      float s = 0.f;
      for (int c = 0; c < BN; ++c) {
        const int x = c & 7, y = (c >> 3) & 7, z = c >> 6;
        s = fmaf(S.x0[(x + dx) + 10 * ((y + dy) + 10 * (z + dz))], bf2f(S.d.v[co >> 3][pv(x, y, z)][co & 7]), s);
      }
      gp[OFF_W0 + i] += s;
    }
  }
  // loss partial
  for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
  if ((threadIdx.x & 31) == 0) S.red[threadIdx.x >> 5] = loss;
  __syncthreads();
  if (threadIdx.x == 0) {
    float s = 0.f;
    for (int w = 0; w < NT / 32; ++w) s += S.red[w];
    lpart[blockIdx.x] = s;
  }
}

// grad[i] = sum over CTAs of gpart[cta][i] (fixed order); loss = sum lpart * loss_scale
__global__ void k_cnn_reduce(const float* gpart, int ngrad, float* grad, const float* lpart, int nloss,
                             float loss_scale, float* loss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (grad && i < CNN_NPARAM) {
    float s = 0.f;
    for (int p = 0; p < ngrad; ++p) s += gpart[size_t(p) * CNN_NPARAM + i];
    grad[i] = s;
  }
  if (i == 0 && loss) {
    float s = 0.f;
    for (int p = 0; p < nloss; ++p) s += lpart[p];
    *loss = s * loss_scale;
  }
}

__global__ void k_adam(float* w, const float* g, float* m, float* v, int t, float lr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= CNN_NPARAM) return;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float gi = g[i];
  m[i] = b1 * m[i] + (1.f - b1) * gi;
  v[i] = b2 * v[i] + (1.f - b2) * gi * gi;
  const float mh = m[i] / (1.f - powf(b1, float(t)));
  const float vh = v[i] / (1.f - powf(b2, float(t)));
  w[i] -= lr * mh / (sqrtf(vh) + eps);
}

// gpart: >= grid*(CNN_NPARAM+1) floats (gradient rows, then one loss partial per CTA)
static int train_launch(const CnnWeights& W, const float* in, const float* target, float tscale, const int* idx,
                        int n, float* gpart, float* grad, float* loss_dev, float* out, int backward, int grid,
                        cudaStream_t s, int loss_mode = 0, int zero_pred = 0) {
  const size_t smem = sizeof(TrainSmem);
  static unsigned long long attr = 0;
  if (first_on_device(attr))
    CUP_CUDA_TRY(cudaFuncSetAttribute(k_cnn_train, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  const int g = std::max(1, std::min(grid, n));
  // loss = mean over samples and cells; gradients of that mean
  const float scale = 1.0f / (float(n) * BN);
  float* lpart = gpart + size_t(g) * CNN_NPARAM;
  {
    ProfScope ps(backward ? "cnn_train_fwd_bwd" : "cnn_forward_batch", s);
    k_cnn_train<<<g, NT, smem, s>>>(W, in, target, tscale, idx, n, scale, gpart, lpart, out, backward, loss_mode,
                                    zero_pred);
  }
  CUP_CUDA_TRY(cudaGetLastError());
  if (backward || loss_dev) {
    k_cnn_reduce<<<(CNN_NPARAM + 255) / 256, 256, 0, s>>>(gpart, g, backward ? grad : nullptr, lpart, g, scale,
                                                          loss_dev);
    CUP_CUDA_TRY(cudaGetLastError());
  }
  return 0;
}

int cnn_forward_batch(const CnnWeights& W, const float* in, float* out, int n, float* gpart, int grid,
                      cudaStream_t s) {
  return train_launch(W, in, nullptr, 1.0f, nullptr, n, gpart, nullptr, nullptr, out, 0, grid, s);
}

int cnn_grad_batch(const CnnWeights& W, const float* in, const float* target, int n, float* gpart, float* grad,
                   float* loss_dev, int grid, cudaStream_t s) {
  return train_launch(W, in, target, 1.0f, nullptr, n, gpart, grad, loss_dev, nullptr, 1, grid, s);
}

int cnn_residual_loss(const CnnWeights& W, const float* in, const float* target, int n, int zero_pred, float* gpart,
                      float* loss_dev, int grid, cudaStream_t s) {
  return train_launch(W, in, target, 1.0f, nullptr, n, gpart, nullptr, loss_dev, nullptr, 0, grid, s, 1, zero_pred);
}

// Unit inputs of the fold: sample j is 1 at lab entry j's cube position.
__global__ void k_fold_inputs(float* in) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < LMAP_K * PV; i += gridDim.x * blockDim.x) {
    const int j = i / PV, p = i - j * PV;
    int q[3];
    lmap_lab_pos(j, q);
    in[i] = p == pv(q[0], q[1], q[2]) ? 1.f : 0.f;
  }
}

// Fragment-ordered BF16 copy of W[c][j] = out[j][c] (lmap_word's layout).
__global__ void k_fold_pack(const float* __restrict__ out, uint4* __restrict__ wfrag) {
  for (size_t w = size_t(blockIdx.x) * blockDim.x + threadIdx.x; w < LMAP_W_WORDS; w += size_t(gridDim.x) * blockDim.x) {
    const int lane = int(w % 32), ks = int((w / 32) % LMAP_KSTEPS), sw = int(w / (32 * LMAP_KSTEPS));
    const int g = lane >> 2, t = lane & 3;
    const int r0 = (sw / 8) * 128 + (sw % 8) * 16 + g, k0 = ks * 16 + 2 * t;
    auto at = [&](int r, int k) { return uint32_t(f2bf(out[size_t(k) * BN + r])); };
    auto pair = [&](int r, int k) { return at(r, k) | (at(r, k + 1) << 16); };
    wfrag[w] = make_uint4(pair(r0, k0), pair(r0 + 8, k0), pair(r0, k0 + 8), pair(r0 + 8, k0 + 8));
  }
}

int cnn_fold(const CnnWeights& W, float* in, float* out, uint4* wfrag, float* gpart, int grid, cudaStream_t s) {
  ProfScope ps("cnn_fold", s);
  k_fold_inputs<<<256, 256, 0, s>>>(in);
  CUP_CUDA_TRY(cudaGetLastError());
  if (int rc = cnn_forward_batch(W, in, out, LMAP_K, gpart, grid, s)) return rc;
  return lmap_pack(out, wfrag, s);
}

int lmap_pack(const float* out, uint4* wfrag, cudaStream_t s) {
  k_fold_pack<<<(LMAP_W_WORDS + 255) / 256, 256, 0, s>>>(out, wfrag);
  CUP_CUDA_TRY(cudaGetLastError());
  return 0;
}

int cnn_train_step(const CnnWeights& W, float* adam_m, float* adam_v, int t, float lr, const float* in,
                   const float* target, float target_scale, const int* idx, int batch, float* gpart, float* grad,
                   float* loss_dev, int grid, cudaStream_t s) {
  if (int rc = train_launch(W, in, target, target_scale, idx, batch, gpart, grad, loss_dev, nullptr, 1, grid, s,
                            /*loss_mode=*/1))
    return rc;
  k_adam<<<(CNN_NPARAM + 255) / 256, 256, 0, s>>>(W.master, grad, adam_m, adam_v, t, lr);
  CUP_CUDA_TRY(cudaGetLastError());
  // the tensor-core layers read BF16 copies of the weights: refresh them from
  // the updated masters, so the next step's forward and backward use the
  // weights being trained
  if (int rc = cnn_pack(W, s)) return rc;
  return cnn_pack(W, s);
}

}  // namespace cup3d
