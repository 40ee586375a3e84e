// Staged block pipeline for the one-ghost-layer stencil kernels (pressure
// RHS, gradient update).  A CTA walks its blocks (blockIdx.x, + gridDim.x, ...)
// through a two-stage ring in shared memory.  While it computes block k, the
// copies of block k+1 are in flight and those of block k+2 are issued as soon
// as block k's stage is free:
//   * each field component's 4 KB block interior by one bulk copy (TMA
//     engine, mbarrier completion with the byte count);
//   * the one-layer ghosts of same-level faces by per-thread 8-byte cp.async
//     from the neighbours (commit groups);
//   * the table entries of block k+2 two stages ahead (4/8-byte cp.async),
//     so no copy waits on a dependent load.
// Ghosts of boundary faces are filled from the staged interior and those of
// coarse-fine faces by the lab rules (lab.cuh) once the stage has landed.
// The star lab layout is LabGeom<1>'s: interior [0, 512), face f's ghost
// layer at 512 + 64 f + (tan1 + 8 tan2).
#pragma once
#include "async_copy.cuh"
#include "lab.cuh"

namespace cup3d {

// One block's table entries, staged by cp.async.
struct StageMeta {
  int kind[6];
  int nbr[24];
  int index[3];
  int flag;   // per-block flag of the kernel (e.g. near an obstacle), 0 if none
  double h;
};
static_assert(sizeof(StageMeta) == 144, "StageMeta layout");

// Issues the copies of block b's table entries into m (threads 0..34).
__device__ __forceinline__ void meta_issue(StageMeta* m, const DevMesh& M, int b, const int* flag) {
  const int t = threadIdx.x;
  if (t < 6)
    cp_async4(&m->kind[t], M.fkind + 6 * b + t);
  else if (t < 30)
    cp_async4(&m->nbr[t - 6], M.fnbr + 24 * b + (t - 6));
  else if (t < 33)
    cp_async4(&m->index[t - 30], M.index + 3 * b + (t - 30));
  else if (t == 33)
    cp_async8(&m->h, M.h + b);
  else if (t == 34) {
    if (flag)
      cp_async4(&m->flag, flag + b);
    else
      m->flag = 0;
  }
}

// The same with plain loads (the pipeline's first two blocks).
__device__ __forceinline__ void meta_load(StageMeta* m, const DevMesh& M, int b, const int* flag) {
  const int t = threadIdx.x;
  if (t < 6)
    m->kind[t] = M.fkind[6 * b + t];
  else if (t < 30)
    m->nbr[t - 6] = M.fnbr[24 * b + (t - 6)];
  else if (t < 33)
    m->index[t - 30] = M.index[3 * b + (t - 30)];
  else if (t == 33)
    m->h = M.h[b];
  else if (t == 34)
    m->flag = flag ? flag[b] : 0;
}

__device__ __forceinline__ bool meta_has_finer(const StageMeta& m) {
  bool r = false;
#pragma unroll
  for (int f = 0; f < 6; ++f) r |= m.kind[f] == K_FINER;
  return r;
}

// Ghosts of block b that the copies do not bring: boundary faces from the
// staged interior (vector_bc: the normal component, or all components at a
// wall, change sign), coarse-fine faces by the lab rules from global memory
// (get(c, blk, cell) reads component c).  Same-level ghosts are left as staged.
template <int NC, class Get>
__device__ void stage_fixup(double* lab, const DevMesh& M, const StageMeta& m, Get get, bool vector_bc) {
  using LG = LabGeom<1>;
  for (int g = threadIdx.x; g < 6 * 64; g += blockDim.x) {
    const int f = g >> 6, a = g & 7, bb = (g >> 3) & 7;
    const int kind = m.kind[f];
    if (kind == K_SAME) continue;
    const int d = f >> 1, s = f & 1;
    const int li = BN + g;
    if (kind == K_BOUNDARY) {
      const int cell = face_cell(d, s, 0, a, bb);
      const bool wall = m.nbr[4 * f] == BCK_WALL;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const double v = lab[c * LG::V + cell];
        lab[c * LG::V + li] = (vector_bc && (wall || c == d)) ? -v : v;
      }
    } else if (kind == K_FINER) {
      const int ch = m.nbr[4 * f + (a >> 2) + 2 * (bb >> 2)];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        double sum = 0.0;
#pragma unroll
        for (int e2 = 0; e2 < 2; ++e2)
#pragma unroll
          for (int e1 = 0; e1 < 2; ++e1)
#pragma unroll
            for (int en = 0; en < 2; ++en)
              sum += get(c, ch, face_cell(d, 1 - s, en, 2 * (a & 3) + e1, 2 * (bb & 3) + e2));
        lab[c * LG::V + li] = 0.125 * sum;
      }
    } else {  // K_COARSER
      const int cb = m.nbr[4 * f];
      const int h1 = m.index[tan1(d)] & 1, h2 = m.index[tan2(d)] & 1;
#pragma unroll
      for (int c = 0; c < NC; ++c)
        lab[c * LG::V + li] = c2f_ghost([&](int cell) { return get(c, cb, cell); }, d, s, 1, a, bb, h1, h2);
    }
  }
}

// Shared memory of the pipeline: two stages of NCH star labs (components with
// ghosts) and NCI interiors (components without), a ring of four table
// entries and two mbarriers.
template <int NCH, int NCI>
struct StagedShape {
  static constexpr int kStage = NCH * LabGeom<1>::V + NCI * BN;  // doubles per stage
  static constexpr size_t kBytes = 2 * kStage * sizeof(double) + 4 * sizeof(StageMeta) + 2 * sizeof(uint64_t);
};

// Runs body(k, b, meta, stage) for this CTA's blocks b = blockIdx.x + k gridDim.x
// with stage = the block's NCH labs followed by its NCI interiors, the
// interiors and same-level ghosts landed.  src[c]: component c's field (block
// b's cells at src[c] + 512 b).  The body fills the remaining ghosts
// (stage_fixup), computes, and ends with __syncthreads (the stage is then
// refilled).  A bulk-copy wait that runs out sets *err and ends the CTA.
template <int NCH, int NCI, class Body>
__device__ void staged_blocks(const DevMesh& M, const double* const (&src)[NCH + NCI], const int* flag,
                              unsigned char* smem, int* err, Body body) {
  using SS = StagedShape<NCH, NCI>;
  using LG = LabGeom<1>;
  double* stage0 = reinterpret_cast<double*>(smem);
  StageMeta* meta = reinterpret_cast<StageMeta*>(smem + 2 * SS::kStage * sizeof(double));
  uint64_t* bar = reinterpret_cast<uint64_t*>(meta + 4);
  const int t = threadIdx.x;
  const int nk = int(blockIdx.x) < M.nb ? (M.nb - 1 - int(blockIdx.x)) / int(gridDim.x) + 1 : 0;
  if (nk == 0) return;
  auto blk = [&](int k) { return int(blockIdx.x) + k * int(gridDim.x); };
  if (t == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init_fence();
  }
  meta_load(&meta[0], M, blk(0), flag);
  if (nk > 1) meta_load(&meta[1], M, blk(1), flag);
  __syncthreads();
  auto issue = [&](int k) {
    const int b = blk(k), s = k & 1;
    const StageMeta& m = meta[k & 3];
    double* st = stage0 + s * SS::kStage;
    if (t == 0) {
      fence_proxy_async_smem();  // the stage's last readers were threads
      mbar_arrive_expect_tx(&bar[s], (NCH + NCI) * BN * sizeof(double));
#pragma unroll
      for (int c = 0; c < NCH; ++c) bulk_g2s(st + c * LG::V, src[c] + size_t(b) * BN, BN * sizeof(double), &bar[s]);
#pragma unroll
      for (int c = 0; c < NCI; ++c)
        bulk_g2s(st + NCH * LG::V + c * BN, src[NCH + c] + size_t(b) * BN, BN * sizeof(double), &bar[s]);
    }
    for (int g = t; g < 6 * 64; g += blockDim.x) {
      const int f = g >> 6;
      if (m.kind[f] != K_SAME) continue;
      const int d = f >> 1, sd = f & 1;
      const size_t from = size_t(m.nbr[4 * f]) * BN + face_cell(d, 1 - sd, 0, g & 7, (g >> 3) & 7);
#pragma unroll
      for (int c = 0; c < NCH; ++c) cp_async8(st + c * LG::V + BN + g, src[c] + from);
    }
    if (k + 2 < nk) meta_issue(&meta[(k + 2) & 3], M, blk(k + 2), flag);
    cp_async_commit();
  };
  issue(0);
  if (nk > 1)
    issue(1);
  else
    cp_async_commit();
  for (int k = 0; k < nk; ++k) {
    cp_async_wait<1>();  // block k's ghosts and block k+2's table entries
    const bool ok = mbar_wait_bounded(&bar[k & 1], (k >> 1) & 1);
    if (__syncthreads_or(!ok)) {
      if (t == 0) atomicExch(err, 1);
      cp_async_wait<0>();
      if (k + 1 < nk) mbar_wait_bounded(&bar[(k + 1) & 1], ((k + 1) >> 1) & 1);
      return;
    }
    body(k, blk(k), meta[k & 3], stage0 + (k & 1) * SS::kStage);
    if (k + 2 < nk)
      issue(k + 2);
    else
      cp_async_commit();
  }
  cp_async_wait<0>();
}

}  // namespace cup3d
