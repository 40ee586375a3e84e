// Learned local map of the two-level preconditioner, as the persistent
// solver applies it:
//   z_b += W lab_b(v) / h_b     for every block b,
// with lab_b(v) the block's star lab of v (LabGeom<1>: its 512 cells, then
// the six one-cell face layers, 896 values, lab rules of lab.cuh) and W the
// trained network folded into one 512 x 896 matrix.  The network is linear,
// so W is exact: column j holds the network's output for a unit input at lab
// position j.  This is the slot of the block preconditioner
// (PoissonSolverAMR.h:183-222, BiCGSTAB.cu:526-527,553-554); the network
// itself has no counterpart in the reference.
//
// Two phases, one grid barrier apart:
//   gather: every CTA writes the BF16 labs of its blocks (b = blockIdx.x +
//     k gridDim.x) to a [nb][896] buffer;
//   GEMM: work item (slice, tile) = 128 rows of W times the labs of 32
//     consecutive blocks, on the BF16 tensor cores (mma.sync m16n8k16, FP32
//     accumulation).  The labs of the tile are staged in shared memory; W
//     is stored in fragment order, so every lane loads its A fragment of a
//     k-step as one 16-byte word (coalesced, 512 bytes a warp).  Each item
//     reads 229 KB of W, so one application reads W ceil(nb/32) times
//     (from L2), the labs 4 times and z once.
#pragma once
#include <cuda_bf16.h>

#include "lab.cuh"

namespace cup3d {

constexpr int LMAP_K = LabGeom<1>::V;            // 896
constexpr int LMAP_KSTEPS = LMAP_K / 16;         // 56
constexpr int LMAP_NBLK = 32;                    // blocks per GEMM tile
constexpr int LMAP_LDB = LMAP_K + 8;             // row stride (BF16) of the staged tile: 1808 B
constexpr int LMAP_SLICES = BN / 128;            // 128-row slices of W (8 warps x 16 rows)
constexpr size_t LMAP_W_WORDS = size_t(BN) * LMAP_K / 8;           // 16-byte words of W
constexpr size_t LMAP_TILE_BYTES = size_t(LMAP_NBLK) * LMAP_LDB * 2;  // 57,856
static_assert(LMAP_K % 16 == 0, "the lab must split into k-steps of 16");
static_assert(LMAP_LDB * 2 % 16 == 0 && (LMAP_LDB / 2) % 32 == 4, "conflict-free 32-bit B fragment loads");

// Word of W holding lane `lane`'s A fragment of k-step ks for rows
// 16 (8 slice + warp) .. +15 (PTX m16n8k16 .bf16 A layout: g = lane / 4,
// t = lane % 4; registers (row g, k 2t..2t+1), (g+8, 2t..), (g, 2t+8..),
// (g+8, 2t+8..), lower k in the lower half).
__host__ __device__ __forceinline__ size_t lmap_word(int slice, int warp, int ks, int lane) {
  return (size_t(slice * 8 + warp) * LMAP_KSTEPS + ks) * 32 + lane;
}

// Cube position (x, y, z in -1..8) of lab entry j.
__host__ __device__ __forceinline__ void lmap_lab_pos(int j, int q[3]) {
  if (j < BN) {
    q[0] = j & 7;
    q[1] = (j >> 3) & 7;
    q[2] = j >> 6;
    return;
  }
  const int g = j - BN, f = g >> 6, d = f >> 1, s = f & 1;
  q[d] = s ? BS : -1;
  q[tan1(d)] = g & 7;
  q[tan2(d)] = (g >> 3) & 7;
}

__device__ __forceinline__ uint32_t lmap_pack2(double a, double b) {
  return uint32_t(__bfloat16_as_ushort(__double2bfloat16(a))) |
         (uint32_t(__bfloat16_as_ushort(__double2bfloat16(b))) << 16);
}

__device__ __forceinline__ void lmap_mma(float c[4], const uint4& a, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a.x), "r"(a.y), "r"(a.z), "r"(a.w), "r"(b0), "r"(b1));
}

// Gather phase (whole CTA): BF16 labs of v for blocks blockIdx.x + k gridDim.x
// into lab[b * LMAP_K ...].  labd: LMAP_K doubles of shared scratch.
template <class T>
__device__ void lmap_gather(const DevMesh& M, const T* __restrict__ v, uint16_t* __restrict__ lab, double* labd) {
  for (int b = blockIdx.x; b < M.nb; b += gridDim.x) {
    lab_fill<1, 1>(labd, M, b, [&](int, int blk, int cell) { return double(v[size_t(blk) * BN + cell]); }, false);
    __syncthreads();
    uint32_t* out = reinterpret_cast<uint32_t*>(lab + size_t(b) * LMAP_K);
    for (int i = threadIdx.x; i < LMAP_K / 2; i += blockDim.x) out[i] = lmap_pack2(labd[2 * i], labd[2 * i + 1]);
    __syncthreads();
  }
}

// GEMM phase (whole CTA of 256 threads = 8 warps): z_b += W lab_b / h_b for the
// CTA's work items; returns this thread's part of sum(added z h^3) (the
// change of the stored, rounded values).  Bs: LMAP_TILE_BYTES of shared
// memory, 16-byte aligned.
template <class T>
__device__ double lmap_gemm(const DevMesh& M, const uint4* __restrict__ W, const uint16_t* __restrict__ lab,
                            T* __restrict__ z, uint16_t* Bs) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int ntiles = (M.nb + LMAP_NBLK - 1) / LMAP_NBLK;
  constexpr int WPB = LMAP_K / 8;  // 16-byte words per lab
  double sum = 0.0;
  for (int item = blockIdx.x; item < ntiles * LMAP_SLICES; item += gridDim.x) {
    const int slice = item % LMAP_SLICES, n0 = (item / LMAP_SLICES) * LMAP_NBLK;
    for (int i = threadIdx.x; i < LMAP_NBLK * WPB; i += blockDim.x) {
      const int n = i / WPB, q = i - n * WPB;
      uint4 val = make_uint4(0u, 0u, 0u, 0u);
      if (n0 + n < M.nb) val = __ldcg(reinterpret_cast<const uint4*>(lab + size_t(n0 + n) * LMAP_K) + q);
      *reinterpret_cast<uint4*>(Bs + n * LMAP_LDB + q * 8) = val;
    }
    __syncthreads();
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
    const uint4* wp = W + lmap_word(slice, warp, 0, lane);
    for (int k0 = 0; k0 < LMAP_KSTEPS; k0 += 8) {
      uint4 a[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = __ldg(wp + (k0 + i) * 32);
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int kk = (k0 + i) * 16 + 2 * t;
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          const uint16_t* bp = Bs + (nt * 8 + g) * LMAP_LDB + kk;
          lmap_mma(acc[nt], a[i], *reinterpret_cast<const uint32_t*>(bp), *reinterpret_cast<const uint32_t*>(bp + 8));
        }
      }
    }
    // C fragment: (row g, block 2t), (g, 2t+1), (g+8, 2t), (g+8, 2t+1)
    const int row = slice * 128 + warp * 16 + g;
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int n = n0 + nt * 8 + 2 * t + j;
        if (n >= M.nb) continue;
        const double h = M.h[n], ih = 1.0 / h;
        double s = 0.0;
#pragma unroll
        for (int hr = 0; hr < 2; ++hr) {
          const size_t o = size_t(n) * BN + row + 8 * hr;
          const double old = double(z[o]);
          const T nv = T(old + double(acc[nt][2 * hr + j]) * ih);
          z[o] = nv;
          s += double(nv) - old;
        }
        sum += s * h * h * h;
      }
    __syncthreads();  // the tile is restaged by the next item
  }
  return sum;
}

}  // namespace cup3d
