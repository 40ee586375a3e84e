// Poisson operator, block preconditioner and BiCGSTAB solver on the device.
#pragma once
#include "common.cuh"

namespace cup3d {

// Device-resident Krylov state.  Written only by the last CTA of a reduction
// ("finalizer"), read by the kernels that follow on the same stream.
struct KrylovState {
  double rho, rho_prev, alpha, omega, beta;
  double rr, rr_hat;                 // (r,r) and (rhat,rhat)
  double err, err_init, err_opt;     // ||r||_2 now, initially, best so far
  double tol_abs, tol_rel;
  double mean_sum;                   // sum(v h^3) of the vector the next SpMV reads
  double ms_zr;                      // three-phase solvers: sum(zr h^3) of the current zr
  double eps;
  int k, restarts, max_restarts, max_iter;
  int done, converged, restart_pending, status;
  int cur, best, nxt;                // x buffer rotation (x_opt without copies)
  int stall_window;                  // > 0: stop when ||r|| has not dropped 10% in this many iterations
  int last_improve_k;
  double stall_ref;
};

enum SolveStatus : int {
  SOLVE_RUNNING = 0,
  SOLVE_CONVERGED = 1,
  SOLVE_MAXITER = 2,
  SOLVE_RESTARTS = 3,
  SOLVE_NAN = 4,
  SOLVE_STALL = 5,
  SOLVE_BARRIER_TIMEOUT = 6  // persistent solver: a grid barrier wait timed out
};

// The operator and preconditioner kernels give each mesh block a 64-thread
// group, four groups per 256-thread CTA.
constexpr int GROUPS_PER_CTA = 4;
// Block groups per CTA of the persistent solvers.
constexpr int PERSISTENT_GROUPS_PER_CTA = 4;

struct PoissonWork {
  // vectors, nb*512 each
  double *r, *rhat, *p, *nu, *t, *z1, *z2, *xs[3];
  // FP32 inner-solve vectors of the mixed-precision solver; fxs[0] = correction e
  float *fr, *frhat, *fp, *fnu, *ft, *fz1, *fz2, *fxs[3], *r32;
  KrylovState* st;
  KrylovState* st2;         // outer (refinement) state
  KrylovState* st_init;     // captured solves: the initial state, uploaded before capture
  double* partial;          // grid * 8
  unsigned int* counters;   // 16
  unsigned int* bar;        // persistent solver: grid-barrier arrivals
  int* bar_error;           // persistent solver: set on a timed-out barrier wait
  long long barrier_cycles; // persistent solvers: grid-barrier wait limit in SM cycles (0: default)
  int grid;                 // CTAs for block kernels
  int pgrid;                // CTAs of the persistent solver (set with the visit order)
  int ggrid;                // CTAs for block-group kernels (4 mesh blocks per CTA pass)
};

// Batched solves: independent cases on disjoint blocks of one flattened mesh
// (no face joins two cases), all in one cooperative launch.  Every block
// group of the batched solver works for one case at a time; the groups are
// dealt to the running cases in proportion to their blocks and dealt again
// whenever a case stops.
struct BatchWork {
  int ncase = 0;
  int grid = 0;                  // CTAs of the batched solver
  int groups = 0;                // grid * groups per CTA
  int* cfirst = nullptr;         // ncase + 1: case c owns blocks cfirst[c] .. cfirst[c+1]-1
  int* cblocks = nullptr;        // nb: each case's blocks by decreasing operator cost, at its own offsets
  double* part = nullptr;        // 2 * groups * 8 partial sums
  int* case_done = nullptr;      // ncase: 1 once the case has stopped
  KrylovState* st = nullptr;     // ncase
  KrylovState* st_init = nullptr;  // ncase: initial states of captured solves
};

// The cases' two-level preconditioners in a batch: each case's A_c^-1
// (nb_c x nb_c, FP32, row-major) packed in case order (case c at off[c]),
// the restriction buffers and 512 h^3 over the batch's blocks.
struct BatchCoarse {
  const float* inv = nullptr;
  const long long* off = nullptr;
  double* rc = nullptr;
  double* rc2 = nullptr;
  const double* w = nullptr;
};

struct SolveParams {
  double tol_abs, tol_rel;
  int max_iter, max_restarts, mean_mode;
  int check_every;   // host checks convergence every this many iterations
  int stall_window;  // 0: off (reference behaviour)
  int persistent;    // 1: all iterations in one cooperative launch (plain and mixed solvers)
  int block_cache;   // persistent solver: table entries staged per block group at launch (0-4)
  int graph;         // 1: being captured into a CUDA graph: the initial state comes from
                     //    PoissonWork::st_init and nothing is read back (plain persistent solver only)
};

struct SolveStats {
  int iterations, restarts, status, outer;
  double err_init, err_opt;
};

// Standalone operators (parity tests and the mixed/learned solvers).
int launch_poisson_apply(const DevMesh& M, const double* x, double* y, int mean_mode,
                         PoissonWork& W, cudaStream_t s);
int launch_block_inverse(const DevMesh& M, const double* in, double* out, PoissonWork& W,
                         cudaStream_t s);
// Solves A x = b; x holds the initial guess on entry and x_opt on exit.
// Coarse space of the two-level preconditioners (built by coarse_build):
// A_c^-1 (nb x nb, row-major), two restriction buffers, the apply buffer and
// the blocks' 512 h^3.  nb = 0: no coarse correction.
struct CoarseView {
  int nb;
  const float* inv;  // FP32: the correction only has to be a fixed linear map
  double* rc;
  double* rc2;
  double* yc;
  const double* w;
};

// Learned local map of the preconditioner (lmap.cuh): the folded network in
// fragment order (LMAP_W_WORDS words) and a [nb][896] BF16 lab buffer.
struct LocalMap {
  const uint4* w;
  uint16_t* lab;
};

// coarse != nullptr: the coarse correction of the two-level preconditioners
// is added to the per-block preconditioner (sms: the device's SM count).
// lmap != nullptr: the learned local map is added as well (persistent solver
// only).
int poisson_bicgstab(const DevMesh& M, const double* b, double* x, const SolveParams& P,
                     PoissonWork& W, SolveStats& out, cudaStream_t s, int* h_done_pinned,
                     const LocalMap* lmap = nullptr, const CoarseView* coarse = nullptr, int sms = 148);

// Mixed precision: FP32 inner BiCGSTAB inside FP64 iterative refinement.
int poisson_mixed(const DevMesh& M, const double* b, double* x, const SolveParams& P, PoissonWork& W,
                  SolveStats& out, cudaStream_t s, int* h_done_pinned, const LocalMap* lmap = nullptr,
                  const CoarseView* coarse = nullptr, int sms = 148);
// The reference's pipelined BiCGSTAB with the exact block inverse
// (PoissonSolverAMR.cpp:13-358), in one cooperative launch; vec: 16 vectors
// of nb*512 doubles (scratch).
int poisson_pipelined(const DevMesh& M, const double* b, double* x, const SolveParams& P, PoissonWork& W,
                      double* const vec[16], SolveStats& out, cudaStream_t s);
// FP64 ||b - A x||_2 with the solvers' mean-row convention.
int true_residual_norm(const DevMesh& M, const double* b, const double* x, int mean_mode, PoissonWork& W,
                       double* err_host, cudaStream_t s);

// sum over cells of v*h^3 and of h^3 (zero-mean projection), into d_out[2]
int launch_weighted_sum(const DevMesh& M, const double* v, double* d_out, PoissonWork& W,
                        cudaStream_t s);

void poisson_init_constants();

// Two-level preconditioners: z += P A_c^-1 P^T r over the mesh blocks
// (coarse.cu); mean_sum (may be null) gets the added sum(z h^3).
constexpr int kCoarseMaxBlocks = 8192;
template <class T>
int coarse_apply(const CoarseView& C, const T* r, T* z, double* mean_sum, int sms, cudaStream_t s);

// Number of 64-thread groups of the persistent solver on a mesh of nb blocks
// (the visit order is balanced for this many groups).
int persistent_solver_groups(int nb, PoissonWork& W, int* groups);
// Largest co-resident grid of the persistent solver for nb blocks.
int persistent_grid_max(int nb, const PoissonWork& W, int* grid);
// Programmatic dependent launch of the solver kernels on this thread (on by
// default; off while capturing a CUDA graph).
void solver_pdl(bool on);
// The solver state before the first kernel (tolerances and caps of P).
void krylov_init_state(const SolveParams& P, KrylovState& init);
// CTAs and block groups of the batched solver for ncase cases (all co-resident).
int batch_solver_shape(int nb, int ncase, int* grid, int* groups);
// One BiCGSTAB per case of the batch (x holds x0 on entry and each case's
// best iterate on exit); out[c] per case.
int poisson_bicgstab_batched(const DevMesh& M, const double* b, double* x, const SolveParams& P,
                             PoissonWork& W, BatchWork& B, SolveStats* out, cudaStream_t s,
                             const BatchCoarse* coarse = nullptr);
// Mixed precision in a batch: FP32 batched inner solves inside per-case FP64
// iterative refinement.  d_first / first: the cases' block offsets (device /
// host, ncase + 1); bpart: nb doubles of scratch; d_case: 2 ncase doubles.
int poisson_mixed_batched(const DevMesh& M, const double* b, double* x, const SolveParams& P, PoissonWork& W,
                          BatchWork& B, SolveStats* out, cudaStream_t s, const BatchCoarse* coarse,
                          const int* d_first, const int* first, double* bpart, double* d_case);

}  // namespace cup3d
