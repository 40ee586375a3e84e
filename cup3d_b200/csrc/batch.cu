// Batches of independent cases: one context over the concatenated meshes of
// several contexts, whose Poisson solves run in one cooperative launch.
//
// No reference counterpart: the reference advances one case per process.
// Each case keeps its own mesh, its own mean-constraint row and its own
// BiCGSTAB scalars; only the device launch is shared.
#include <algorithm>
#include <cstring>
#include <numeric>

#include "context.h"
#include "stencils.cuh"

namespace cup3d {

// Concatenates the cases' meshes: blocks of case k follow those of case k-1,
// face-table entries that name blocks are shifted by the case's offset
// (boundary entries hold a BC kind and stay), and no face joins two cases.
static void concat_meshes(const std::vector<Mesh>& cases, Mesh& m, std::vector<int>& first,
                          std::vector<int>& mean) {
  m = Mesh();
  m.spec = cases[0].spec;
  first.assign(cases.size() + 1, 0);
  mean.assign(cases.size(), -1);
  for (size_t k = 0; k < cases.size(); ++k) first[k + 1] = first[k] + cases[k].nb;
  m.nb = first.back();
  for (size_t k = 0; k < cases.size(); ++k) {
    const Mesh& c = cases[k];
    const int off = first[k];
    m.level.insert(m.level.end(), c.level.begin(), c.level.end());
    m.index.insert(m.index.end(), c.index.begin(), c.index.end());
    m.h.insert(m.h.end(), c.h.begin(), c.h.end());
    m.origin.insert(m.origin.end(), c.origin.begin(), c.origin.end());
    m.face_kind.insert(m.face_kind.end(), c.face_kind.begin(), c.face_kind.end());
    for (int b = 0; b < c.nb; ++b)
      for (int f = 0; f < 6; ++f) {
        const int kind = c.face_kind[6 * b + f];
        for (int q = 0; q < 4; ++q) {
          const int v = c.face_nbr[24 * b + 4 * f + q];
          m.face_nbr.push_back(kind != FACE_BOUNDARY && v >= 0 ? v + off : v);
        }
      }
    mean[k] = c.mean_block >= 0 ? c.mean_block + off : -1;
    m.max_level_used = std::max(m.max_level_used, c.max_level_used);
  }
  m.mean_block = mean[0];
}

// Each case's blocks by decreasing operator cost (2 + coarser faces + 2 x
// finer faces, the estimate of mesh_visit_order), at the case's own offsets:
// the batched solver deals them round-robin to the case's groups.
static std::vector<int> cost_sorted_blocks(const std::vector<Mesh>& cases, const std::vector<int>& first) {
  std::vector<int> out(first.back());
  for (size_t k = 0; k < cases.size(); ++k) {
    const Mesh& m = cases[k];
    std::vector<int> cost(m.nb, 2);
    for (int b = 0; b < m.nb; ++b)
      for (int f = 0; f < 6; ++f) {
        const int kind = m.face_kind[6 * b + f];
        cost[b] += kind == FACE_COARSER ? 1 : (kind == FACE_FINER ? 2 : 0);
      }
    std::vector<int> idx(m.nb);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return cost[x] > cost[y]; });
    for (int i = 0; i < m.nb; ++i) out[first[k] + i] = first[k] + idx[i];
  }
  return out;
}

// Keeps the thread's last error message on the context.
static int keep_err(cup_ctx* c, int rc) {
  c->err = cup_last_error(nullptr);
  return rc;
}

static int upload_ints(cup_ctx* c, int** dst, const std::vector<int>& v) {
  if (int rc = c->batch_arena.alloc(dst, v.size())) return rc;
  CUP_CUDA_TRY(stream_h2d(c->stream, *dst, v.data(), v.size() * sizeof(int)));
  return 0;
}

static int batch_setup(cup_ctx* c, const std::vector<Mesh>& cases) {
  std::vector<int> first, mean;
  concat_meshes(cases, c->mesh, first, mean);
  c->ncase = int(cases.size());
  c->case_first = first;
  c->case_mesh = cases;
  if (int rc = ctx_upload_mesh(c)) return rc;
  if (int rc = ctx_alloc_fields(c)) return rc;
  std::vector<int> bcase(c->mesh.nb);
  for (int k = 0; k < c->ncase; ++k)
    for (int b = first[k]; b < first[k + 1]; ++b) bcase[b] = k;
  int *d_bcase = nullptr, *d_mean = nullptr;
  if (int rc = upload_ints(c, &d_bcase, bcase)) return rc;
  if (int rc = upload_ints(c, &d_mean, mean)) return rc;
  c->dm.bcase = d_bcase;
  c->dm.case_mean = d_mean;
  BatchWork& B = c->B;
  B.ncase = c->ncase;
  if (int rc = batch_solver_shape(c->mesh.nb, c->ncase, &B.grid, &B.groups)) return rc;
  if (B.groups < c->ncase) return set_error(CUP_ERR_ARG, "batch: more cases than block groups of the batched solver");
  if (int rc = upload_ints(c, &B.cfirst, first)) return rc;
  if (int rc = upload_ints(c, &B.cblocks, cost_sorted_blocks(cases, first))) return rc;
  if (int rc = c->batch_arena.alloc(&B.part, size_t(2) * B.groups * 8)) return rc;
  if (int rc = c->batch_arena.alloc(&B.case_done, size_t(B.ncase))) return rc;
  if (int rc = c->batch_arena.alloc(&B.st, size_t(B.ncase))) return rc;
  return 0;
}

// The batch's two-level preconditioners, when built.
static const BatchCoarse* batch_coarse(const cup_ctx* c) { return c->bcoarse.inv ? &c->bcoarse : nullptr; }

// With the two-level solver configured: each case's coarse space, built on
// the case's own context (its A_c, mean-constraint row included, and the
// FP32 inverse), copied into one packed, block-diagonal array in case order.
// No face joins two cases, so the batch's coarse operator is exactly that.
static int batch_coarse_setup(cup_ctx* c, cup_ctx* const* cases) {
  if (c->cfg.poisson_solver != CUP_POISSON_B200_TWOLEVEL && c->cfg.poisson_solver != CUP_POISSON_B200_TWOLEVEL_MIXED)
    return 0;
  std::vector<long long> off(c->ncase);
  long long total = 0;
  for (int k = 0; k < c->ncase; ++k) {
    const long long n = c->case_first[k + 1] - c->case_first[k];
    off[k] = total;
    total += n * n;
  }
  DevArena& A = c->bcoarse_arena;
  float* inv = nullptr;
  long long* d_off = nullptr;
  double *rc = nullptr, *rc2 = nullptr, *w = nullptr;
  const int nb = c->mesh.nb;
  if (int rc_ = A.alloc(&inv, size_t(total))) return rc_;
  if (int rc_ = A.alloc(&d_off, size_t(c->ncase))) return rc_;
  if (int rc_ = A.alloc(&rc, size_t(nb))) return rc_;
  if (int rc_ = A.alloc(&rc2, size_t(nb))) return rc_;
  if (int rc_ = A.alloc(&w, size_t(nb))) return rc_;
  CUP_CUDA_TRY(stream_h2d(c->stream, d_off, off.data(), off.size() * sizeof(long long)));
  std::vector<double> hw(nb);
  for (int b = 0; b < nb; ++b) hw[b] = 512.0 * c->mesh.h[b] * c->mesh.h[b] * c->mesh.h[b];
  CUP_CUDA_TRY(stream_h2d(c->stream, w, hw.data(), hw.size() * sizeof(double)));
  for (int k = 0; k < c->ncase; ++k) {
    cup_ctx* s = cases[k];
    if (int rc_ = coarse_build(s)) return rc_;
    const long long n = c->case_first[k + 1] - c->case_first[k];
    if (s->coarse.nb != n) return set_error(CUP_ERR_STATE, "batch two-level: a case's coarse space does not match");
    CUP_CUDA_TRY(cudaMemcpyAsync(inv + off[k], s->coarse.inv, size_t(n * n) * sizeof(float), cudaMemcpyDeviceToDevice,
                                 s->stream));
    CUP_CUDA_TRY(cudaStreamSynchronize(s->stream));
  }
  c->bcoarse = BatchCoarse{inv, d_off, rc, rc2, w};
  return 0;
}

// The cases' current fields (velocity, pressure, grid chi) into the batch's.
static int copy_case_fields(cup_ctx* c, const std::vector<const cup_ctx*>& cases) {
  const size_t N = size_t(c->mesh.nb) * BN;
  for (size_t k = 0; k < cases.size(); ++k) {
    const cup_ctx* s = cases[k];
    CUP_CUDA_TRY(cudaStreamSynchronize(s->stream));
    const size_t n = size_t(s->mesh.nb) * BN, off = size_t(c->case_first[k]) * BN;
    for (int d = 0; d < 3; ++d)
      CUP_CUDA_TRY(cudaMemcpyAsync(c->F.vel[c->F.vcur] + d * N + off, s->F.vel[s->F.vcur] + d * n, n * 8,
                                   cudaMemcpyDeviceToDevice, c->stream));
    CUP_CUDA_TRY(cudaMemcpyAsync(c->F.pres[c->F.pcur] + off, s->F.pres[s->F.pcur], n * 8, cudaMemcpyDeviceToDevice,
                                 c->stream));
    CUP_CUDA_TRY(cudaMemcpyAsync(c->F.chi + off, s->F.chi, n * 8, cudaMemcpyDeviceToDevice, c->stream));
  }
  CUP_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return 0;
}

// The cases' obstacles, concatenated in case order (slots of case k are
// slot_first[k] .. slot_first[k+1]-1), and the per-case buffers of the step.
static int batch_step_setup(cup_ctx* c, const std::vector<const cup_ctx*>& cases) {
  const int K = c->ncase;
  std::vector<int> blocks, slot_first(K + 1, 0);
  std::vector<double> chi, udef, kin(9 * size_t(K), 0.0);
  for (int k = 0; k < K; ++k) {
    if (int rc = ctx_obstacle_host_copies(const_cast<cup_ctx*>(cases[k]))) return rc;
    const DevObstacle& o = cases[k]->ob;
    slot_first[k + 1] = slot_first[k] + o.nslots;
    for (int sl = 0; sl < o.nslots; ++sl) blocks.push_back(o.h_blocks[sl] + c->case_first[k]);
    chi.insert(chi.end(), o.h_chi.begin(), o.h_chi.end());
    for (int i = 0; i < 9; ++i) kin[9 * k + i] = o.kin[i];
  }
  const int NS = slot_first[K];
  udef.assign(3 * size_t(NS) * BN, 0.0);
  for (int d = 0; d < 3; ++d)
    for (int k = 0; k < K; ++k) {
      const DevObstacle& o = cases[k]->ob;
      for (int sl = 0; sl < o.nslots; ++sl)
        std::copy_n(o.h_udef.begin() + (size_t(d) * o.nslots + sl) * BN, BN,
                    udef.begin() + (size_t(d) * NS + slot_first[k] + sl) * BN);
    }
  if (NS > 0)
    if (int rc = ctx_upload_obstacle(c, NS, blocks.data(), chi.data(), udef.data(), kin.data())) return rc;
  BatchStep& T = c->T;
  DevArena& A = c->batch_arena;
  if (int rc = upload_ints(c, &T.first, c->case_first)) return rc;
  if (int rc = upload_ints(c, &T.slot_first, slot_first)) return rc;
  if (int rc = A.alloc(&T.dt, size_t(K))) return rc;
  if (int rc = A.alloc(&T.sums, 2 * size_t(K))) return rc;
  if (int rc = A.alloc(&T.kin, 9 * size_t(K))) return rc;
  if (int rc = A.alloc(&T.umax, size_t(K))) return rc;
  if (int rc = A.alloc(&T.force, 6 * size_t(K))) return rc;
  if (int rc = A.alloc(&T.bscratch, 2 * size_t(c->mesh.nb))) return rc;
  if (int rc = A.alloc(&T.slot_force, 6 * size_t(std::max(NS, 1)))) return rc;
  CUP_CUDA_TRY(stream_h2d(c->stream, T.kin, kin.data(), kin.size() * 8));
  CUP_CUDA_TRY(stream_zero(c->stream, T.force, 6 * size_t(K) * 8));
  std::vector<double> hmin(K);
  for (int k = 0; k < K; ++k) hmin[k] = c->case_mesh[k].spec.hmin;
  if (int rc = A.alloc(&T.hmin, size_t(K))) return rc;
  if (int rc = A.alloc(&T.mixed, 2 * size_t(K))) return rc;
  CUP_CUDA_TRY(stream_h2d(c->stream, T.hmin, hmin.data(), K * sizeof(double)));
  if (int rc = A.alloc(&c->B.st_init, size_t(K))) return rc;
  // pinned host copies for captured steps
  const size_t bytes = sizeof(KrylovState) * K + sizeof(double) * 7 * K + sizeof(int) * 4;
  CUP_CUDA_TRY(cudaMallocHost(&T.h_block, bytes));
  T.h_st = static_cast<KrylovState*>(T.h_block);
  T.h_dt = reinterpret_cast<double*>(T.h_st + K);
  T.h_force = T.h_dt + K;
  T.h_err = reinterpret_cast<int*>(T.h_force + 6 * K);
  c->dm.case_dt = T.dt;
  c->dm.case_sums = T.sums;
  c->dm.case_kin = T.kin;
  return 0;
}

// Moving bodies (unless -StaticObstacles): when a case's body moves, every
// case's pose is advanced and its chi created again at each launched step
// (batch_bodies_advance), as cup_step does for one case; each case keeps its
// own BDF2 history.  Free bodies and frames that follow a body stay with
// single cases.
static int batch_bodies_setup(cup_ctx* c, const std::vector<const cup_ctx*>& cases) {
  if (c->cfg.static_obstacles) return 0;
  bool any = false;
  for (const cup_ctx* k : cases) any |= body_moves(k);
  if (!any) return 0;
  for (size_t k = 0; k < cases.size(); ++k) {
    const BodyState& B = cases[k]->body;
    bool frame = false;
    for (int d = 0; d < 3; ++d) frame |= B.fix_frame[d] != 0;
    if (body_free(cases[k]) || frame)
      return set_error(CUP_ERR_ARG, ("batch of cases with moving bodies: case " + std::to_string(k) +
                                     " has a free body or a frame that follows it (single cases only)").c_str());
    if (B.kind < 0 && cases[k]->ob.nslots > 0)
      return set_error(CUP_ERR_ARG, ("batch of cases with moving bodies: case " + std::to_string(k) +
                                     " holds obstacle data that cannot be created again").c_str());
  }
  c->batch_moving = true;
  c->case_body.clear();
  c->case_coef.clear();
  c->case_dt_prev.clear();
  for (const cup_ctx* k : cases) {
    c->case_body.push_back(k->body);
    c->case_coef.push_back({k->coef_u[0], k->coef_u[1], k->coef_u[2]});
    c->case_dt_prev.push_back(k->dt_prev);
  }
  // per-slot force sums for any slot count
  return c->batch_arena.alloc(&c->T.slot_force, 6 * size_t(c->mesh.nb));
}

static ObstacleView batch_ob_view(const cup_ctx* c) {
  ObstacleView v;
  v.nslots = c->ob.nslots;
  v.slot = c->ob.slot_of_block;
  v.near = c->ob.near;
  v.chi = c->ob.chi;
  v.udef = c->ob.udef;
  v.blk = c->ob.block_of_slot;
  v.udef_zero = c->ob.udef_zero ? 1 : 0;
  return v;
}

static SolveParams batch_params(const cup_ctx* c) {
  SolveParams P{};
  P.tol_abs = c->cfg.poisson_tol;
  P.tol_rel = c->cfg.poisson_tol_rel;
  P.max_iter = c->cfg.poisson_max_iter;
  P.max_restarts = c->cfg.poisson_max_restarts;
  P.mean_mode = c->cfg.mean_constraint;
  P.persistent = 1;
  P.block_cache = c->cfg.poisson_block_cache;
  return P;
}

// The batch's Poisson solve: FP64 (block inverse, or two-level when the
// cases' coarse spaces were built), or mixed precision (-poissonSolver
// b200_mixed, or b200_twolevel_mixed with the coarse spaces: FP32 batched
// inner solves, FP64 refinement per case).  The learned, Schwarz and
// pipelined solvers are single-case only.
static int batch_solve(cup_ctx* c, const double* b, double* x, const SolveParams& P, SolveStats* S) {
  const int sv = c->cfg.poisson_solver;
  if (sv == CUP_POISSON_B200_LEARNED || sv == CUP_POISSON_B200_LEARNED_MIXED || sv == CUP_POISSON_B200_SCHWARZ ||
      sv == CUP_POISSON_B200_PIPELINED)
    return set_error(CUP_ERR_ARG, "batch of cases: the learned, Schwarz and pipelined solvers are single-case only "
                                  "(b200, b200_mixed, b200_twolevel, b200_twolevel_mixed)");
  if (sv == CUP_POISSON_B200_MIXED || sv == CUP_POISSON_B200_TWOLEVEL_MIXED)
    return poisson_mixed_batched(c->dm, b, x, P, c->W, c->B, S, c->stream, batch_coarse(c), c->T.first,
                                 c->case_first.data(), c->T.bscratch, c->T.mixed);
  return poisson_bicgstab_batched(c->dm, b, x, P, c->W, c->B, S, c->stream, batch_coarse(c));
}

// Worst outcome over the cases, stats per case.
static int batch_stats(cup_ctx* c, const std::vector<SolveStats>& S, float ms, cup_solve_stats* stats) {
  int rc = CUP_OK;
  for (int k = 0; k < c->ncase; ++k) {
    if (stats) {
      cup_solve_stats& o = stats[k];
      o.iterations = S[k].iterations;
      o.restarts = S[k].restarts;
      o.status = S[k].status;
      o.fallback = 0;
      o.err_init = S[k].err_init;
      o.err_final = S[k].err_opt;
      o.true_rel = -1.0;
      o.milliseconds = ms;
    }
    if (S[k].status == SOLVE_NAN) rc = ctx_fail(c, CUP_ERR_NAN, "batched Poisson solve produced NaN");
    else if (S[k].status != SOLVE_CONVERGED && rc == CUP_OK) rc = CUP_SOFT_MAXITER;
  }
  return rc;
}

// A batch step with every case at its CFL dt, captured as a CUDA graph: the
// per-case dt comes from k_case_calc_dt (the host supplies the step's CFL
// factor through pinned memory), the solver starts from device templates and
// moves its best iterates itself, and dt, forces, solver states and the
// barrier flag are copied back by the graph.
static int batch_graph_capture(cup_ctx* c, int vcur, int pcur, int use_pold, cudaGraphExec_t* out) {
  const int K = c->ncase;
  Fields& F = c->F;
  BatchStep& T = c->T;
  cudaStream_t s = c->stream;
  const int grid = c->W.grid;
  poisson_init_constants();
  SolveParams P = batch_params(c);
  P.graph = 1;
  std::vector<KrylovState> init(K);
  for (KrylovState& k : init) krylov_init_state(P, k);
  CUP_CUDA_TRY(stream_h2d(s, c->B.st_init, init.data(), K * sizeof(KrylovState)));
  const ObstacleView ob = batch_ob_view(c);
  const int step_arg = use_pold ? c->cfg.step_2nd_start + 1 : 0;
  CUP_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  auto run = [&]() -> int {
    CUP_CUDA_TRY(cudaMemcpyAsync(c->d_scalars + SC_GFAC, &c->gio->cfl_fac, sizeof(double), cudaMemcpyHostToDevice, s));
    if (int r = launch_case_max_u(c->dm, F.vel[vcur], c->cfg.uinf, T.bscratch, T.first, K, T.umax, grid, s)) return r;
    if (int r = launch_case_calc_dt(T.umax, c->d_scalars + SC_GFAC, c->cfg.nu, T.hmin, K, T.dt, s)) return r;
    int v = vcur;
    for (int st = 0; st < 3; ++st) {
      if (int r = launch_advect_stage(c->dm, F.vel[v], F.vel[1 - v], F.tmpV, 0.0, c->cfg.nu, c->cfg.uinf,
                                      c->cfg.advection, st, kgrid(c, TG_ADVECT), s))
        return r;
      v = 1 - v;
    }
    if (ob.nslots > 0) {
      if (int r = launch_penalize(c->dm, F.vel[v], F.chi, ob, T.kin, 0.0, c->cfg.lambda, c->cfg.implicit_penalization,
                                  nullptr, c->W.partial, c->W.counters + 11, s, T.slot_force))
        return r;
      if (int r = launch_case_forces(T.slot_force, T.slot_first, K, T.force, s)) return r;
    }
    double* pold = F.pres[pcur];
    double* pnew = F.pres[1 - pcur];
    if (int r = launch_pressure_rhs(c->dm, F.vel[v], pold, F.chi, ob, 0.0, step_arg, c->cfg.step_2nd_start, F.lhs,
                                    F.phi, kgrid(c, TG_RHS), s))
      return r;
    CUP_CUDA_TRY(cudaEventRecordWithFlags(c->ev0, s, cudaEventRecordExternal));
    if (int r = poisson_bicgstab_batched(c->dm, F.lhs, F.phi, P, c->W, c->B, nullptr, s, batch_coarse(c))) return r;
    CUP_CUDA_TRY(cudaEventRecordWithFlags(c->ev1, s, cudaEventRecordExternal));
    if (int r = launch_case_sums(c->dm, F.phi, T.bscratch, T.first, K, T.sums, grid, s)) return r;
    if (int r = launch_grad_update(c->dm, F.vel[v], F.phi, pold, pnew, nullptr, 0.0, step_arg,
                                   c->cfg.step_2nd_start, kgrid(c, TG_GRAD), s))
      return r;
    CUP_CUDA_TRY(cudaMemcpyAsync(T.h_dt, T.dt, K * sizeof(double), cudaMemcpyDeviceToHost, s));
    CUP_CUDA_TRY(cudaMemcpyAsync(T.h_force, T.force, 6 * K * sizeof(double), cudaMemcpyDeviceToHost, s));
    CUP_CUDA_TRY(cudaMemcpyAsync(T.h_st, c->B.st, K * sizeof(KrylovState), cudaMemcpyDeviceToHost, s));
    CUP_CUDA_TRY(cudaMemcpyAsync(T.h_err, c->W.bar_error, sizeof(int), cudaMemcpyDeviceToHost, s));
    return 0;
  };
  solver_pdl(false);
  const int rc = run();
  solver_pdl(true);
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s, &graph);
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (e != cudaSuccess) return set_cuda_error(e, "cudaStreamEndCapture", __FILE__, __LINE__);
  const cudaError_t e2 = cudaGraphInstantiate(out, graph, 0);
  cudaGraphDestroy(graph);
  if (e2 != cudaSuccess) return set_cuda_error(e2, "cudaGraphInstantiate", __FILE__, __LINE__);
  return 0;
}

static int batch_graph_step(cup_ctx* c, int step, double* dt_used, double* force, cup_solve_stats* stats) {
  const int K = c->ncase;
  Fields& F = c->F;
  BatchStep& T = c->T;
  const int use_pold = step > c->cfg.step_2nd_start ? 1 : 0;
  const int key = F.vcur | (F.pcur << 1) | (use_pold << 2);
  if (!c->gexec[key])
    if (int rc = batch_graph_capture(c, F.vcur, F.pcur, use_pold, &c->gexec[key])) return keep_err(c, rc);
  c->gio->cfl_fac = ctx_cfl_factor(c->cfg, step);
  CUP_CUDA_TRY(cudaGraphLaunch(c->gexec[key], c->stream));
  CUP_CUDA_TRY(cudaStreamSynchronize(c->stream));
  F.vcur = 1 - F.vcur;  // three advection stages
  F.pcur = 1 - F.pcur;
  if (*T.h_err) return ctx_fail(c, CUP_ERR_CUDA, "batched BiCGSTAB: a grid barrier wait timed out");
  for (int k = 0; k < K; ++k) {
    dt_used[k] = T.h_dt[k];
    if (!(T.h_dt[k] > 0)) return ctx_fail(c, CUP_ERR_NAN, "cup_batch_step: dt <= 0 or NaN in case " + std::to_string(k));
  }
  if (force) std::copy_n(T.h_force, 6 * K, force);
  float ms = 0;
  CUP_CUDA_TRY(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  std::vector<SolveStats> S(K);
  for (int k = 0; k < K; ++k) {
    const KrylovState& st = T.h_st[k];
    S[k].iterations = st.k;
    S[k].restarts = st.restarts;
    S[k].status = st.done ? st.status : SOLVE_MAXITER;
    S[k].err_init = st.err_init;
    S[k].err_opt = st.err_opt;
  }
  return batch_stats(c, S, ms, stats);
}

}  // namespace cup3d

using namespace cup3d;

extern "C" {

cup_ctx* cup_batch_create(int32_t ncases, cup_ctx* const* cases) {
  if (ncases < 1 || !cases) {
    set_error(CUP_ERR_ARG, "cup_batch_create: no cases");
    return nullptr;
  }
  std::vector<Mesh> meshes;
  for (int k = 0; k < ncases; ++k) {
    const cup_ctx* c = cases[k];
    if (!c || c->host_only || c->mesh.nb == 0 || c->ncase != 1) {
      set_error(CUP_ERR_ARG, "cup_batch_create: every case must be a device context with a mesh (not a batch)");
      return nullptr;
    }
    if (c->cfg.device != cases[0]->cfg.device || c->cfg.mean_constraint != cases[0]->cfg.mean_constraint) {
      set_error(CUP_ERR_ARG, "cup_batch_create: the cases must share the device and -bMeanConstraint");
      return nullptr;
    }
    meshes.push_back(c->mesh);
  }
  cup_ctx* c = cup_create(&cases[0]->cfg);
  if (!c) return nullptr;
  const std::vector<const cup_ctx*> cs(cases, cases + ncases);
  int rc = batch_setup(c, meshes);
  if (rc == 0) rc = copy_case_fields(c, cs);
  if (rc == 0) rc = batch_step_setup(c, cs);
  if (rc == 0) rc = batch_bodies_setup(c, cs);
  if (rc == 0) rc = batch_coarse_setup(c, cases);
  if (rc) {
    (void)rc;
    const std::string msg = "cup_batch_create: " + std::string(cup_last_error(nullptr));
    cup_destroy(c);
    set_error(CUP_ERR_CUDA, msg.c_str());
    return nullptr;
  }
  return c;
}

int32_t cup_batch_num_cases(const cup_ctx* c) { return c ? c->ncase : 0; }

int cup_batch_case_blocks(const cup_ctx* c, int32_t k, int32_t* first, int32_t* nblocks) {
  if (!c || k < 0 || k >= c->ncase || !first || !nblocks) return set_error(CUP_ERR_ARG, "cup_batch_case_blocks: bad arguments");
  if (c->ncase == 1) {
    *first = 0;
    *nblocks = c->mesh.nb;
  } else {
    *first = c->case_first[k];
    *nblocks = c->case_first[k + 1] - c->case_first[k];
  }
  return 0;
}

int cup_batch_poisson_solve_dev(cup_ctx* c, const double* b, double* x, cup_solve_stats* stats) {
  ProfBind pb_(c);
  if (!c || !b || !x || !stats || c->ncase < 2) return ctx_fail(c, CUP_ERR_ARG, "cup_batch_poisson_solve_dev: not a batch or bad arguments");
  if (reinterpret_cast<uintptr_t>(x) % 16 != 0 || reinterpret_cast<uintptr_t>(b) % 16 != 0)
    return ctx_fail(c, CUP_ERR_ARG, "cup_batch_poisson_solve_dev: b and x must be 16-byte aligned");
  const SolveParams P = batch_params(c);
  std::vector<SolveStats> S(c->ncase);
  CUP_CUDA_TRY(cudaEventRecord(c->ev0, c->stream));
  if (int rc = batch_solve(c, b, x, P, S.data())) return keep_err(c, rc);
  CUP_CUDA_TRY(cudaEventRecord(c->ev1, c->stream));
  CUP_CUDA_TRY(cudaEventSynchronize(c->ev1));
  float ms = 0;
  CUP_CUDA_TRY(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  return batch_stats(c, S, ms, stats);
}

int cup_batch_step(cup_ctx* c, int32_t step, const double* dt_in, double* dt_used, double* force,
                   cup_solve_stats* stats) {
  ProfBind pb_(c);
  if (!c || c->ncase < 2 || !dt_used) return ctx_fail(c, CUP_ERR_ARG, "cup_batch_step: not a batch or bad arguments");
  const bool fp64 = c->cfg.poisson_solver == CUP_POISSON_B200 || c->cfg.poisson_solver == CUP_POISSON_B200_TWOLEVEL;
  if (!dt_in && c->cfg.step_graph && !c->prof.on && !c->batch_moving && fp64)
    return batch_graph_step(c, step, dt_used, force, stats);
  const int K = c->ncase;
  BatchStep& T = c->T;
  Fields& F = c->F;
  const int grid = c->W.grid;
  // each case's dt: given, or Simulation::calcMaxTimestep from its own max |u| and hmin
  std::vector<double> dt(K, 0.0), umax(K, 0.0);
  bool need_umax = !dt_in;
  for (int k = 0; k < K && !need_umax; ++k) need_umax = !(dt_in[k] > 0);
  if (need_umax) {
    if (int rc = launch_case_max_u(c->dm, F.vel[F.vcur], c->cfg.uinf, T.bscratch, T.first, K, T.umax, grid,
                                   c->stream))
      return keep_err(c, rc);
    CUP_CUDA_TRY(stream_d2h(c->stream, umax.data(), T.umax, K * sizeof(double)));
  }
  for (int k = 0; k < K; ++k) {
    dt[k] = dt_in && dt_in[k] > 0 ? dt_in[k] : ctx_calc_dt(c->cfg, c->case_mesh[k].spec.hmin, umax[k], step);
    if (!(dt[k] > 0)) return ctx_fail(c, CUP_ERR_NAN, "cup_batch_step: dt <= 0 or NaN in case " + std::to_string(k));
    dt_used[k] = dt[k];
  }
  CUP_CUDA_TRY(cudaMemcpyAsync(T.dt, dt.data(), K * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  // CreateObstacles: the cases' bodies at their new poses
  if (c->batch_moving)
    if (int rc = batch_bodies_advance(c, step, dt.data())) return keep_err(c, rc);
  // advection-diffusion, penalization, pressure projection: the single-case
  // kernels over all blocks, each block with its case's dt, kinematics and mean
  for (int st = 0; st < 3; ++st) {
    if (int rc = launch_advect_stage(c->dm, F.vel[F.vcur], F.vel[1 - F.vcur], F.tmpV, 0.0, c->cfg.nu, c->cfg.uinf,
                                     c->cfg.advection, st, kgrid(c, TG_ADVECT), c->stream))
      return keep_err(c, rc);
    F.vcur = 1 - F.vcur;
  }
  const ObstacleView ob = batch_ob_view(c);
  if (ob.nslots > 0) {
    if (int rc = launch_penalize(c->dm, F.vel[F.vcur], F.chi, ob, T.kin, 0.0, c->cfg.lambda,
                                 c->cfg.implicit_penalization, nullptr, c->W.partial, c->W.counters + 11, c->stream,
                                 T.slot_force))
      return keep_err(c, rc);
    if (int rc = launch_case_forces(T.slot_force, T.slot_first, K, T.force, c->stream)) return keep_err(c, rc);
  }
  double* pold = F.pres[F.pcur];
  double* pnew = F.pres[1 - F.pcur];
  if (int rc = launch_pressure_rhs(c->dm, F.vel[F.vcur], pold, F.chi, ob, 0.0, step, c->cfg.step_2nd_start, F.lhs,
                                   F.phi, kgrid(c, TG_RHS), c->stream))
    return keep_err(c, rc);
  std::vector<SolveStats> S(K);
  CUP_CUDA_TRY(cudaEventRecord(c->ev0, c->stream));
  if (int rc = batch_solve(c, F.lhs, F.phi, batch_params(c), S.data())) return keep_err(c, rc);
  CUP_CUDA_TRY(cudaEventRecord(c->ev1, c->stream));
  if (int rc = launch_case_sums(c->dm, F.phi, T.bscratch, T.first, K, T.sums, grid, c->stream)) return keep_err(c, rc);
  if (int rc = launch_grad_update(c->dm, F.vel[F.vcur], F.phi, pold, pnew, nullptr, 0.0, step,
                                  c->cfg.step_2nd_start, kgrid(c, TG_GRAD), c->stream))
    return keep_err(c, rc);
  F.pcur = 1 - F.pcur;
  if (force) CUP_CUDA_TRY(cudaMemcpyAsync(force, T.force, 6 * K * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUP_CUDA_TRY(cudaStreamSynchronize(c->stream));
  float ms = 0;
  CUP_CUDA_TRY(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  return batch_stats(c, S, ms, stats);
}

}  // extern "C"
