// Shared device definitions: block geometry, mesh tables, reductions.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>

namespace cup3d {

constexpr int BS = 8;     // cells per block edge (CUP_BLOCK_SIZE)
constexpr int BN = 512;   // cells per block
constexpr int NT = 256;   // threads per CTA for block kernels

enum : int { K_SAME = 0, K_BOUNDARY = 1, K_COARSER = 2, K_FINER = 3 };
enum : int { BCK_FREESPACE = 0, BCK_PERIODIC = 1, BCK_WALL = 2 };

// Mesh tables as uploaded by the host (see mesh.h for their meaning).
struct DevMesh {
  int nb;
  int mean_block;               // block with index (0,0,0), -1 if none
  const int* __restrict__ fkind;  // 6*nb
  const int* __restrict__ fnbr;   // 24*nb
  const int* __restrict__ index;  // 3*nb
  const double* __restrict__ h;   // nb
  // Order in which the block-group kernels visit the blocks (a permutation of
  // 0..nb-1, or null for 0..nb-1): visit slot i holds block order[i].
  const int* __restrict__ order;
  // Batches of independent cases (null for one case): the case of each block
  // and each case's mean-constraint block, time step, (sum phi h^3, sum h^3)
  // of the pressure increment, and obstacle kinematics (CM, vel, omega).
  const int* __restrict__ bcase;
  const int* __restrict__ case_mean;
  const double* __restrict__ case_dt;
  const double* __restrict__ case_sums;
  const double* __restrict__ case_kin;
  // Error word of the staged stencil kernels: set to 1 when a wait for a
  // block's bulk copies runs out (zero otherwise; read by the host).
  int* kerr;
};

// Time step of block b: its case's in a batch, the device-computed one of a
// captured step (case_dt set, bcase null), else dt.
__device__ __forceinline__ double block_dt(const DevMesh& M, int b, double dt) {
  return M.case_dt ? M.case_dt[M.bcase ? M.bcase[b] : 0] : dt;
}

#ifndef CUP3D_TAN_HELPERS
#define CUP3D_TAN_HELPERS
__host__ __device__ __forceinline__ int tan1(int d) { return d == 0 ? 1 : 0; }
__host__ __device__ __forceinline__ int tan2(int d) { return d == 2 ? 1 : 2; }
#endif

// Cell of a block on its own face (d, side) at `layer` cells inward, at
// tangential position (a along tan1, b along tan2).
__device__ __forceinline__ int face_cell(int d, int side, int layer, int a, int b) {
  const int c = side ? BS - 1 - layer : layer;
  return d == 0 ? c + BS * a + BS * BS * b : (d == 1 ? a + BS * c + BS * BS * b : a + BS * b + BS * BS * c);
}

// ---------------------------------------------------------------------------
// Deterministic reductions: every CTA writes NR partial sums, the last CTA to
// arrive (ticket counter) sums all partials in CTA order and runs `fin`.
// ---------------------------------------------------------------------------
template <int NR>
__device__ __forceinline__ void block_reduce(double (&v)[NR], double* sm /* >= 8*NR */) {
#pragma unroll
  for (int r = 0; r < NR; ++r)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[r] += __shfl_xor_sync(0xffffffffu, v[r], o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0)
#pragma unroll
    for (int r = 0; r < NR; ++r) sm[w * NR + r] = v[r];
  __syncthreads();
  if (threadIdx.x < 32) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      double s = l < nw ? sm[l * NR + r] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      v[r] = s;
    }
  }
  __syncthreads();
}

// Programmatic dependent launch.  A kernel launched with the programmatic
// stream-serialization attribute may start while the previous kernel of its
// stream is finishing; pdl_wait() blocks until that kernel has completed and
// its memory is visible, so everything before it must read only data the
// previous kernel does not write.  Without the attribute both are no-ops.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Plain (weak, L1-cached) load of solver vectors.  Within a launch, data
// that other CTAs wrote before a grid barrier is read only after the
// barrier's acquire and the CTA barrier behind it; the memory model orders
// these weak loads after the writes, so they may hit L1 (halo values that
// neighbouring blocks on the same SM read again) and still see fresh data.
template <class V>
__device__ __forceinline__ V ld_stream(const V* p) {
  return *p;
}

struct GridReduce {
  double* partial;        // gridDim.x * 8 doubles
  unsigned int* counter;  // one per reduction site, zero between launches
};

// Returns true in the last CTA, with the grid totals in v (all threads of it).
template <int NR>
__device__ bool grid_reduce(double (&v)[NR], const GridReduce& g, double* sm) {
  block_reduce<NR>(v, sm);
  __shared__ unsigned int s_ticket;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int r = 0; r < NR; ++r) g.partial[blockIdx.x * 8 + r] = v[r];
    __threadfence();
    s_ticket = atomicAdd(g.counter, 1u);
  }
  __syncthreads();
  if (s_ticket != gridDim.x - 1) return false;
  __threadfence();
  double acc[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) acc[r] = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x)
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] += __ldcg(&g.partial[i * 8 + r]);
  block_reduce<NR>(acc, sm);
  // broadcast lane-0 totals to the whole CTA
  __shared__ double s_tot[NR];
  if (threadIdx.x == 0) {
#pragma unroll
    for (int r = 0; r < NR; ++r) s_tot[r] = acc[r];
    *g.counter = 0u;
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < NR; ++r) v[r] = s_tot[r];
  return true;
}

// Max-reduction counterpart of grid_reduce for one non-negative value.
__device__ __forceinline__ bool grid_reduce_max(double& v, const GridReduce& g, double* sm) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sm[w] = v;
  __syncthreads();
  __shared__ unsigned int s_ticket_m;
  __shared__ double s_max;
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) m = fmax(m, sm[i]);
    g.partial[blockIdx.x * 8] = m;
    __threadfence();
    s_ticket_m = atomicAdd(g.counter, 1u);
  }
  __syncthreads();
  if (s_ticket_m != gridDim.x - 1) return false;
  __threadfence();
  // the last CTA takes the maximum over all partials with all its threads
  double m = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) m = fmax(m, __ldcg(&g.partial[i * 8]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (l == 0) sm[w] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mm = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) mm = fmax(mm, sm[i]);
    s_max = mm;
    *g.counter = 0u;
  }
  __syncthreads();
  v = s_max;
  return true;
}

// ---------------------------------------------------------------------------
// Grid-wide barrier with a reduction, for cooperative (co-resident) launches.
// Each CTA writes its NR partial sums into the slot of this barrier (two slots
// alternate, so a CTA that runs ahead to the next barrier cannot overwrite
// partials another CTA is still reading), arrives on a counter that only
// grows, and waits until every CTA has arrived at this barrier.  Then every
// CTA sums all partials itself, in the same order, so all CTAs hold the same
// totals and no CTA has to publish them.  The wait is bounded: after about a
// second of polling a waiter sets *error and returns false, so a barrier that
// can never complete ends the kernel instead of hanging the device.
// Ordering: the CTA's stores precede its arrival through the CTA barrier and
// the arrival's release; the waiter's acquire load and the CTA barrier after
// it order every later load of the CTA behind all arrivals it has seen.
// ---------------------------------------------------------------------------
struct GridSync {
  unsigned int* arrive;  // arrivals since the launch (zero before it)
  double* partial;       // 2 * gridDim.x * 8
  int* error;            // set on a timed-out wait
  long long limit;       // longest wait of one CTA at one barrier, in SM clock cycles
};

constexpr long long kBarrierClockLimit = 1ll << 31;  // default wait limit: about 1 s

// GPU-scope release add (no result) and acquire load.
__device__ __forceinline__ void red_add_release(unsigned int* p, unsigned int v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// epoch: the number of barriers this CTA has passed (shared, zero at launch)
template <int NR>
__device__ bool grid_allreduce(double (&v)[NR], const GridSync& G, unsigned int& epoch, double* sm) {
  const unsigned int k = epoch;
  double* part = G.partial + size_t(k & 1u) * gridDim.x * 8;
  block_reduce<NR>(v, sm);  // ends with __syncthreads: the CTA's writes precede the arrival
  __shared__ int s_ok;
  __shared__ double s_tot[8];
  if (threadIdx.x == 0) {
#pragma unroll
    for (int r = 0; r < NR; ++r) part[blockIdx.x * 8 + r] = v[r];
    red_add_release(G.arrive, 1u);
    const unsigned int target = (k + 1u) * gridDim.x;
    const long long t0 = clock64();
    int ok = 1;
    while (ld_acquire(G.arrive) < target) {
      if (clock64() - t0 > G.limit) {
        ok = 0;
        break;
      }
    }
    if (!ok) atomicExch(G.error, 1);
    s_ok = ok;
    epoch = k + 1u;
  }
  __syncthreads();
  if (!s_ok) return false;
  double acc[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) acc[r] = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x)
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] += __ldcg(&part[i * 8 + r]);
  block_reduce<NR>(acc, sm);
  if (threadIdx.x == 0)
#pragma unroll
    for (int r = 0; r < NR; ++r) s_tot[r] = acc[r];
  __syncthreads();
#pragma unroll
  for (int r = 0; r < NR; ++r) v[r] = s_tot[r];
  return true;
}

}  // namespace cup3d

namespace cup3d {
// Function attributes (cudaFuncSetAttribute) hold per device: `done` keeps one
// bit per device ordinal.  True, and marks the bit, the first time a launch
// site asks on the current device.
inline bool first_on_device(unsigned long long& done) {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d > 63) return true;
  const unsigned long long bit = 1ull << d;
  if (done & bit) return false;
  done |= bit;
  return true;
}
}  // namespace cup3d

#define CUP_CUDA_TRY(expr)                                                     \
  do {                                                                            \
    cudaError_t e_ = (expr);                                                      \
    if (e_ != cudaSuccess) return ::cup3d::set_cuda_error(e_, #expr, __FILE__, __LINE__); \
  } while (0)

namespace cup3d {
int set_cuda_error(cudaError_t e, const char* what, const char* file, int line);
// Records a message for cup_last_error() and returns code.
int set_error(int code, const char* msg);
}
