// Learned local map of the two-level preconditioner, as the persistent
// solver applies it:
//   z_b += W lab_b(v) / h_b     for every block b,
// with lab_b(v) the block's star lab of the residual v (LabGeom<1>: its 512
// cells, then the six one-cell face layers, 896 values; the rules below) and W the
// trained network folded into one 512 x 896 matrix.  The network is linear,
// so W is exact: column j holds the network's output for a unit input at lab
// position j.  This is the slot of the block preconditioner
// (PoissonSolverAMR.h:183-222, BiCGSTAB.cu:526-527,553-554); the network
// itself has no counterpart in the reference.
//
// Two phases, one grid barrier apart:
//   gather: every CTA writes the BF16 residual labs of its blocks (four at
//     a time) to a [nb][896] buffer;
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
static_assert(LMAP_K % 16 == 0 && LMAP_K == 14 * 64, "the lab splits into k-steps of 16 and 14 entries a thread");
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

__device__ __forceinline__ void lmap_mma(float c[4], const uint4& a, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a.x), "r"(a.y), "r"(a.z), "r"(a.w), "r"(b0), "r"(b1));
}

// The lab of a residual.  A residual entry is an integral over its cell (the
// operator's rows are h L ~ h^3 times the Laplacian), so the ghosts are the
// residuals of cells of the block's own size: the sum of the eight finer
// cells of a finer neighbour, an eighth of the value interpolated in a
// coarser neighbour (the lab rules of lab.cuh, rescaled), zero beyond a
// domain boundary.  The mean-constraint row (cell 0 of block mean_blk, -1:
// none) is not a Laplacian row: it enters no other block's lab.
struct LabMeta {
  int kind[6];
  int nbr[24];
  int index[3];
  int pad_;
};

// Loads block b's table entries into m (threads t = 0..32 of a group).
__device__ __forceinline__ void lab_meta_load(LabMeta& m, const DevMesh& M, int b, int t) {
  if (t < 6)
    m.kind[t] = M.fkind[6 * b + t];
  else if (t < 30)
    m.nbr[t - 6] = M.fnbr[24 * b + (t - 6)];
  else if (t < 33)
    m.index[t - 30] = M.index[3 * b + (t - 30)];
}

// Ghost entry (face f, tangential a, bb) of block b's residual lab.
template <class T>
__device__ __forceinline__ double rlab_ghost(const T* __restrict__ v, const LabMeta& m, int f, int a, int bb,
                                             int mean_blk) {
  const int d = f >> 1, s = f & 1, kind = m.kind[f];
  auto get = [&](int blk, int cell) {
    return (blk == mean_blk && cell == 0) ? 0.0 : double(v[size_t(blk) * BN + cell]);
  };
  if (kind == K_SAME) return get(m.nbr[4 * f], face_cell(d, 1 - s, 0, a, bb));
  if (kind == K_BOUNDARY) return 0.0;
  if (kind == K_FINER) {
    const int ch = m.nbr[4 * f + (a >> 2) + 2 * (bb >> 2)];
    double sum = 0.0;
#pragma unroll
    for (int e2 = 0; e2 < 2; ++e2)
#pragma unroll
      for (int e1 = 0; e1 < 2; ++e1)
#pragma unroll
        for (int en = 0; en < 2; ++en) sum += get(ch, face_cell(d, 1 - s, en, 2 * (a & 3) + e1, 2 * (bb & 3) + e2));
    return sum;
  }
  const int cb = m.nbr[4 * f];  // K_COARSER
  const int h1 = m.index[tan1(d)] & 1, h2 = m.index[tan2(d)] & 1;
  return 0.125 * c2f_ghost([&](int cell) { return get(cb, cell); }, d, s, 1, a, bb, h1, h2);
}

// Entry k (0..13) of thread t (0..63) of block b's residual lab: lab index
// j = t + 64 k (the cells for k < 8, face k - 8's ghost layer after).
template <class T>
__device__ __forceinline__ double rlab_entry(const T* __restrict__ v, const LabMeta& m, int b, int t, int k,
                                             int mean_blk) {
  if (k < 8) return double(v[size_t(b) * BN + t + 64 * k]);
  return rlab_ghost(v, m, k - 8, t & 7, t >> 3, mean_blk);
}

// Gather phase (whole CTA of 256 threads): the four 64-thread groups write
// the BF16 residual labs of four consecutive blocks at once (blocks
// 4 blockIdx.x + k 4 gridDim.x ...) to lab[b * LMAP_K ...].  meta: LMAP_GATHER
// entries of shared memory.
constexpr int LMAP_GATHER = 4;
template <class T>
__device__ void lmap_gather(const DevMesh& M, const T* __restrict__ v, uint16_t* __restrict__ lab, LabMeta* meta,
                            int mean_blk) {
  const int g = threadIdx.x >> 6, t = threadIdx.x & 63;
  for (int b0 = blockIdx.x * LMAP_GATHER; b0 < M.nb; b0 += gridDim.x * LMAP_GATHER) {
    const int b = b0 + g;
    if (b < M.nb) lab_meta_load(meta[g], M, b, t);
    __syncthreads();
    if (b < M.nb) {
      double e[LMAP_K / 64];
#pragma unroll
      for (int k = 0; k < LMAP_K / 64; ++k) e[k] = rlab_entry(v, meta[g], b, t, k, mean_blk);
      uint16_t* out = lab + size_t(b) * LMAP_K + t;
#pragma unroll
      for (int k = 0; k < LMAP_K / 64; ++k) out[64 * k] = __bfloat16_as_ushort(__double2bfloat16(e[k]));
    }
    __syncthreads();  // meta is reloaded by the next round
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
    // the A fragments of eight k-steps in flight while the previous eight
    // are multiplied
    const uint4* wp = W + lmap_word(slice, warp, 0, lane);
    uint4 a[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = __ldg(wp + i * 32);
#pragma unroll
    for (int k0 = 0; k0 < LMAP_KSTEPS; k0 += 8) {
      uint4 nx[8];
      if (k0 + 8 < LMAP_KSTEPS)
#pragma unroll
        for (int i = 0; i < 8; ++i) nx[i] = __ldg(wp + (k0 + 8 + i) * 32);
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int kk = (k0 + i) * 16 + 2 * t;
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          const uint16_t* bp = Bs + (nt * 8 + g) * LMAP_LDB + kk;
          lmap_mma(acc[nt], a[i], *reinterpret_cast<const uint32_t*>(bp), *reinterpret_cast<const uint32_t*>(bp + 8));
        }
      }
      if (k0 + 8 < LMAP_KSTEPS)
#pragma unroll
        for (int i = 0; i < 8; ++i) a[i] = nx[i];
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
