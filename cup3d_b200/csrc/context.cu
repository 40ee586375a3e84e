// C-ABI implementation: context, mesh, fields, Poisson entry points.
#include <cmath>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <sstream>

#include "context.h"
#include "obstacles.h"
#include "stencils.cuh"

namespace cup3d {

static thread_local std::string g_last_error;
thread_local Profiler* t_prof = nullptr;

int set_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
  std::ostringstream os;
  os << "CUDA error " << int(e) << " (" << cudaGetErrorString(e) << ") in " << what << " at "
     << file << ":" << line;
  g_last_error = os.str();
  return CUP_ERR_CUDA;
}

int set_error(int code, const char* msg) {
  g_last_error = msg;
  return code;
}

int ctx_fail(cup_ctx* c, int code, const std::string& msg) {
  g_last_error = msg;
  if (c) c->err = msg;
  return code;
}

size_t nbn(const cup_ctx* c) { return size_t(c->mesh.nb) * BN; }

cudaError_t stream_h2d(cudaStream_t s, void* dst, const void* src, size_t bytes) {
  const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
  return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
}

cudaError_t stream_d2h(cudaStream_t s, void* dst, const void* src, size_t bytes) {
  const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
  return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
}

cudaError_t stream_zero(cudaStream_t s, void* dst, size_t bytes) {
  const cudaError_t e = cudaMemsetAsync(dst, 0, bytes, s);
  return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
}

// Propagates the thread-local message of a failed internal call into ctx.
static int keep(cup_ctx* c, int rc) {
  if (rc < 0 && c) c->err = g_last_error;
  return rc;
}

int ctx_upload_mesh(cup_ctx* c, int set) {
  Mesh& m = c->mesh;
  if (set < 0) set = c->tab_cur;
  MeshTables& T = c->tabs[set];
  if (T.cap < m.nb) {
    T.arena.release();
    T.cap = 0;
    const size_t cap = size_t(m.nb) + m.nb / 4;
    if (int rc = T.arena.alloc(&T.kerr, 1)) return rc;
    if (int rc = T.arena.alloc(&T.fk, 6 * cap)) return rc;
    if (int rc = T.arena.alloc(&T.fn, 24 * cap)) return rc;
    if (int rc = T.arena.alloc(&T.ix, 3 * cap)) return rc;
    if (int rc = T.arena.alloc(&T.plan, 9 * cap)) return rc;
    if (int rc = T.arena.alloc(&T.h, cap)) return rc;
    T.cap = int(cap);
  }
  cudaStream_t s = c->stream;
  CUP_CUDA_TRY(cudaMemsetAsync(T.kerr, 0, sizeof(int), s));
  CUP_CUDA_TRY(cudaMemcpyAsync(T.fk, m.face_kind.data(), 6 * size_t(m.nb) * 4, cudaMemcpyHostToDevice, s));
  CUP_CUDA_TRY(cudaMemcpyAsync(T.fn, m.face_nbr.data(), 24 * size_t(m.nb) * 4, cudaMemcpyHostToDevice, s));
  CUP_CUDA_TRY(cudaMemcpyAsync(T.ix, m.index.data(), 3 * size_t(m.nb) * 4, cudaMemcpyHostToDevice, s));
  CUP_CUDA_TRY(cudaMemcpyAsync(T.h, m.h.data(), size_t(m.nb) * 8, cudaMemcpyHostToDevice, s));
  c->dm.nb = m.nb;
  c->dm.mean_block = m.mean_block;
  c->dm.fkind = T.fk;
  c->dm.fnbr = T.fn;
  c->dm.index = T.ix;
  c->dm.h = T.h;
  c->dm.order = c->d_order;  // set again by fields_reset
  c->dm.bcase = nullptr;  // set for batches
  c->dm.case_mean = nullptr;
  c->dm.case_dt = nullptr;
  c->dm.case_sums = nullptr;
  c->dm.case_kin = nullptr;
  c->dm.kerr = T.kerr;
  ++c->mesh_version;
  return 0;
}

// Reads the staged kernels' error word after the stream has been synchronised.
int ctx_check_kernels(cup_ctx* c) {
  int e = 0;
  CUP_CUDA_TRY(stream_d2h(c->stream, &e, c->dm.kerr, sizeof(int)));
  if (e) return ctx_fail(c, CUP_ERR_CUDA, "stencil kernel: a wait for a block's bulk copies timed out");
  return 0;
}

int fields_reserve(cup_ctx* c, int nb) {
  if (c->field_cap >= nb) return 0;
  graph_reset(c);
  c->field_arena.release();
  c->field_cap = 0;
  c->d_diag = nullptr;
  c->diag_cap = 0;
  c->d_order = nullptr;
  const int cap = nb + nb / 4;
  const size_t n = size_t(cap) * BN;
  DevArena& A = c->field_arena;
  Fields& F = c->F;
  for (int i = 0; i < 2; ++i) {
    if (int rc = A.alloc(&F.vel[i], 3 * n)) return rc;
    if (int rc = A.alloc(&F.pres[i], n)) return rc;
  }
  if (int rc = A.alloc(&F.tmpV, 3 * n)) return rc;
  if (int rc = A.alloc(&F.lhs, n)) return rc;
  if (int rc = A.alloc(&F.chi, n)) return rc;
  if (int rc = A.alloc(&F.phi, n)) return rc;
  PoissonWork& W = c->W;
  double** vecs[] = {&W.r, &W.rhat, &W.p, &W.nu, &W.t, &W.z1, &W.z2, &W.xs[1], &W.xs[2]};
  for (double** v : vecs)
    if (int rc = A.alloc(v, n)) return rc;
  W.xs[0] = nullptr;
  float** fvecs[] = {&W.fr, &W.frhat, &W.fp, &W.fnu, &W.ft, &W.fz1, &W.fz2, &W.fxs[0], &W.fxs[1], &W.fxs[2], &W.r32};
  for (float** v : fvecs)
    if (int rc = A.alloc(v, n)) return rc;
  // partial sums for the largest grid of any mesh: a few CTAs per SM, and
  // the penalization's 1184 CTAs
  if (int rc = A.alloc(&W.partial, size_t(std::max(c->num_sms * 8, 1184)) * 8)) return rc;
  if (int rc = A.alloc(&W.counters, 32)) return rc;
  if (int rc = A.alloc(&W.bar, 1)) return rc;
  if (int rc = A.alloc(&W.bar_error, 1)) return rc;
  if (int rc = A.alloc(&W.st, 1)) return rc;
  if (int rc = A.alloc(&W.st2, 1)) return rc;
  if (int rc = A.alloc(&W.st_init, 1)) return rc;
  if (int rc = A.alloc(&c->d_order, size_t(cap))) return rc;
  c->field_cap = cap;
  return 0;
}

int fields_reset(cup_ctx* c, bool keep_current) {
  const size_t n = nbn(c);
  cudaStream_t s = c->stream;
  Fields& F = c->F;
  PoissonWork& W = c->W;
  for (int i = 0; i < 2; ++i) {
    if (!keep_current || i != F.vcur) CUP_CUDA_TRY(cudaMemsetAsync(F.vel[i], 0, 3 * n * 8, s));
    if (!keep_current || i != F.pcur) CUP_CUDA_TRY(cudaMemsetAsync(F.pres[i], 0, n * 8, s));
  }
  CUP_CUDA_TRY(cudaMemsetAsync(F.tmpV, 0, 3 * n * 8, s));
  CUP_CUDA_TRY(cudaMemsetAsync(F.lhs, 0, n * 8, s));
  CUP_CUDA_TRY(cudaMemsetAsync(F.chi, 0, n * 8, s));
  CUP_CUDA_TRY(cudaMemsetAsync(F.phi, 0, n * 8, s));
  CUP_CUDA_TRY(cudaMemsetAsync(W.counters, 0, 32 * sizeof(unsigned int), s));
  CUP_CUDA_TRY(cudaMemsetAsync(W.bar, 0, sizeof(unsigned int), s));
  CUP_CUDA_TRY(cudaMemsetAsync(W.bar_error, 0, sizeof(int), s));
  // grid: a few CTAs per SM, never more than blocks
  W.grid = std::max(1, std::min(c->mesh.nb, c->num_sms * 8));
  W.ggrid = std::max(1, std::min((c->mesh.nb + GROUPS_PER_CTA - 1) / GROUPS_PER_CTA, c->num_sms * 8));
  // visit order of the block-group kernels, balanced for the persistent solver's groups
  int groups = 0;
  if (int rc = persistent_solver_groups(c->mesh.nb, W, &groups)) return rc;
  const std::vector<int32_t> order = mesh_visit_order(c->mesh, groups);
  CUP_CUDA_TRY(cudaMemcpyAsync(c->d_order, order.data(), order.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  c->dm.order = c->d_order;
  return 0;
}

int ctx_alloc_fields(cup_ctx* c) {
  graph_reset(c);
  c->obst_arena.release();
  c->ob = DevObstacle();
  c->proj_open = 0;
  if (int rc = fields_reserve(c, c->mesh.nb)) return rc;
  c->F.vcur = 0;
  c->F.pcur = 0;
  return fields_reset(c, false);
}

static int install_mesh(cup_ctx* c, const std::vector<std::array<int32_t, 4>>& leaves) {
  if (c->ncase > 1) return ctx_fail(c, CUP_ERR_STATE, "a batch of cases keeps the meshes it was made from");
  MeshSpec spec;
  for (int d = 0; d < 3; ++d) {
    spec.bpd[d] = c->cfg.bpd[d];
    spec.bc[d] = c->cfg.bc[d];
  }
  spec.level_max = c->cfg.level_max;
  spec.extent = c->cfg.extent;
  std::string err;
  Mesh m;
  if (!mesh_build(spec, leaves, m, err)) return ctx_fail(c, CUP_ERR_MESH, "mesh: " + err);
  c->mesh = std::move(m);
  if (c->host_only) return 0;
  if (int rc = ctx_upload_mesh(c)) return keep(c, rc);
  if (int rc = ctx_alloc_fields(c)) return keep(c, rc);
  return 0;
}

static double* field_ptr(cup_ctx* c, int field, int* ncomp) {
  *ncomp = 1;
  if (c->host_only) return nullptr;
  switch (field) {
    case CUP_FIELD_VEL: *ncomp = 3; return c->F.vel[c->F.vcur];
    case CUP_FIELD_PRES: return c->proj_open ? c->F.phi : c->F.pres[c->F.pcur];
    case CUP_FIELD_CHI: return c->F.chi;
    case CUP_FIELD_LHS: return c->F.lhs;
    case CUP_FIELD_TMPV: *ncomp = 3; return c->F.tmpV;
    default: return nullptr;
  }
}

}  // namespace cup3d

using namespace cup3d;

extern "C" {

void cup_config_default(cup_config* c) {
  std::memset(c, 0, sizeof(*c));
  c->bpd[0] = c->bpd[1] = c->bpd[2] = 1;
  c->level_max = 1;
  c->bc[0] = c->bc[1] = c->bc[2] = CUP_BC_FREESPACE;
  c->extent = 1.0;
  c->nu = 0.0;
  c->cfl = 0.1;
  c->rampup = 100;
  c->lambda = 1e6;
  c->implicit_penalization = 1;
  c->advection = CUP_ADV_UPWIND5;
  c->mean_constraint = 1;
  c->poisson_tol = 1e-6;
  c->poisson_tol_rel = 1e-4;
  c->poisson_solver = CUP_POISSON_B200;
  c->poisson_max_iter = 1000;
  c->poisson_max_restarts = 100;
  c->step_2nd_start = 2;
  c->device = 0;
  c->poisson_block_cache = 4;
  c->step_graph = 1;
  c->static_obstacles = 0;
  c->rtol = 1.0;
  c->ctol = 0.1;
  c->level_max_vorticity = -1;  // levelMax unless given
  c->level_start = -1;          // levelMax - 1 unless given (SimulationData.cpp:38)
  c->poisson_persistent = 1;
}

static int parse_bc(const std::string& v) {
  if (v == "periodic") return CUP_BC_PERIODIC;
  if (v == "wall") return CUP_BC_WALL;
  if (v == "freespace") return CUP_BC_FREESPACE;
  return -1;
}

int cup_config_parse(cup_config* c, const char* args) {
  if (!c || !args) return ctx_fail(nullptr, CUP_ERR_ARG, "cup_config_parse: null argument");
  std::istringstream is(args);
  std::string k, v;
  while (is >> k) {
    if (!(is >> v)) return ctx_fail(nullptr, CUP_ERR_ARG, "missing value for " + k);
    std::string key = k;
    while (!key.empty() && key[0] == '-') key.erase(0, 1);
    char* end = nullptr;
    const double dv = std::strtod(v.c_str(), &end);
    const bool num = end && *end == '\0';
    auto need_num = [&]() { return num ? 0 : ctx_fail(nullptr, CUP_ERR_ARG, "bad number for " + k); };
    if (key == "bpdx" || key == "bpdy" || key == "bpdz") {
      if (need_num()) return CUP_ERR_ARG;
      c->bpd[key[3] - 'x'] = int(dv);
    } else if (key == "levelMax") {
      if (need_num()) return CUP_ERR_ARG;
      c->level_max = int(dv);
    } else if (key == "BC_x" || key == "BC_y" || key == "BC_z") {
      const int bc = parse_bc(v);
      if (bc < 0) return ctx_fail(nullptr, CUP_ERR_ARG, "BC not recognized " + v);
      c->bc[key[3] - 'x'] = bc;
    } else if (key == "extent") {
      if (need_num()) return CUP_ERR_ARG;
      c->extent = dv;
    } else if (key == "nu") {
      if (need_num()) return CUP_ERR_ARG;
      c->nu = dv;
    } else if (key == "CFL") {
      if (need_num()) return CUP_ERR_ARG;
      c->cfl = dv;
    } else if (key == "rampup") {
      if (need_num()) return CUP_ERR_ARG;
      c->rampup = int(dv);
    } else if (key == "lambda") {
      if (need_num()) return CUP_ERR_ARG;
      c->lambda = dv;
    } else if (key == "implicitPenalization") {
      c->implicit_penalization = (v == "1" || v == "true");
    } else if (key == "uinfx" || key == "uinfy" || key == "uinfz") {
      if (need_num()) return CUP_ERR_ARG;
      c->uinf[key[4] - 'x'] = dv;
    } else if (key == "advection") {
      if (v == "upwind5" || v == "upwind3") c->advection = CUP_ADV_UPWIND5;
      else if (v == "weno5") c->advection = CUP_ADV_WENO5;
      else return ctx_fail(nullptr, CUP_ERR_ARG, "unknown advection scheme " + v);
    } else if (key == "bMeanConstraint") {
      if (need_num()) return CUP_ERR_ARG;
      c->mean_constraint = int(dv);
    } else if (key == "poissonTol") {
      if (need_num()) return CUP_ERR_ARG;
      c->poisson_tol = dv;
    } else if (key == "poissonTolRel") {
      if (need_num()) return CUP_ERR_ARG;
      c->poisson_tol_rel = dv;
    } else if (key == "poissonSolver") {
      // the reference's own names ("iterative": PoissonSolverAMR, "cuda_iterative":
      // PoissonSolverExp; PoissonSolverBase.cpp:10-32) select the plain FP64 solver
      if (v == "b200" || v == "iterative" || v == "cuda_iterative") c->poisson_solver = CUP_POISSON_B200;
      else if (v == "b200_mixed") c->poisson_solver = CUP_POISSON_B200_MIXED;
      else if (v == "b200_learned") c->poisson_solver = CUP_POISSON_B200_LEARNED;
      else if (v == "b200_learned_mixed") c->poisson_solver = CUP_POISSON_B200_LEARNED_MIXED;
      else if (v == "b200_twolevel") c->poisson_solver = CUP_POISSON_B200_TWOLEVEL;
      else if (v == "b200_twolevel_mixed") c->poisson_solver = CUP_POISSON_B200_TWOLEVEL_MIXED;
      else if (v == "b200_schwarz") c->poisson_solver = CUP_POISSON_B200_SCHWARZ;
      else if (v == "b200_pipelined") c->poisson_solver = CUP_POISSON_B200_PIPELINED;
      else return ctx_fail(nullptr, CUP_ERR_ARG, "Poisson solver: \"" + v + "\" unrecognized!");
    } else if (key == "device") {
      if (need_num()) return CUP_ERR_ARG;
      c->device = int(dv);
    } else if (key == "stepGraph") {
      if (need_num()) return CUP_ERR_ARG;
      c->step_graph = dv != 0 ? 1 : 0;
    } else if (key == "Rtol") {
      if (need_num()) return CUP_ERR_ARG;
      c->rtol = dv;
    } else if (key == "Ctol") {
      if (need_num()) return CUP_ERR_ARG;
      c->ctol = dv;
    } else if (key == "levelMaxVorticity") {
      if (need_num()) return CUP_ERR_ARG;
      c->level_max_vorticity = int(dv);
    } else if (key == "levelStart") {
      if (need_num()) return CUP_ERR_ARG;
      c->level_start = int(dv);
    } else if (key == "poissonPersistent") {
      if (need_num()) return CUP_ERR_ARG;
      c->poisson_persistent = int(dv) != 0 ? 1 : 0;
    } else if (key == "StaticObstacles") {
      if (need_num()) return CUP_ERR_ARG;
      c->static_obstacles = dv != 0 ? 1 : 0;
    } else if (key == "poissonBlockCache") {
      if (need_num()) return CUP_ERR_ARG;
      if (dv < 0 || dv > 4) return ctx_fail(nullptr, CUP_ERR_ARG, "poissonBlockCache must be 0-4");
      c->poisson_block_cache = int(dv);
    } else {
      return ctx_fail(nullptr, CUP_ERR_ARG, "unknown flag " + k);
    }
  }
  return 0;
}

cup_ctx* cup_create(const cup_config* cfg) {
  if (!cfg) {
    ctx_fail(nullptr, CUP_ERR_ARG, "cup_create: null config");
    return nullptr;
  }
  if (cfg->level_max < 1 || cfg->bpd[0] < 1 || cfg->bpd[1] < 1 || cfg->bpd[2] < 1 ||
      !(cfg->extent > 0)) {
    ctx_fail(nullptr, CUP_ERR_ARG, "cup_create: invalid bpd/levelMax/extent");
    return nullptr;
  }
  cup_ctx* c = new cup_ctx();
  c->cfg = *cfg;
  if (cfg->device < 0) {  // host-only context: mesh construction and tables, no device work
    c->host_only = true;
    return c;
  }
  cudaError_t e = cudaSetDevice(cfg->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
  if (e == cudaSuccess) e = cudaMallocHost(&c->h_pinned, 4096);
  if (e == cudaSuccess) e = cudaMallocHost(&c->gio, sizeof(GraphIO));
  if (e == cudaSuccess) e = cudaMalloc(&c->d_scalars, 64 * sizeof(double));
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, cfg->device);
  if (e != cudaSuccess) {
    set_cuda_error(e, "cup_create", __FILE__, __LINE__);
    cup_destroy(c);
    return nullptr;
  }
  poisson_init_constants();
  return c;
}

void cup_destroy(cup_ctx* c) {
  if (!c) return;
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (MeshTables& T : c->tabs) T.arena.release();
  c->field_arena.release();
  c->obst_arena.release();
  if (c->d_scalars) cudaFree(c->d_scalars);
  for (cudaGraphExec_t& g : c->gexec)
    if (g) cudaGraphExecDestroy(g);
  if (c->T.h_block) cudaFreeHost(c->T.h_block);
  if (c->h_pinned) cudaFreeHost(c->h_pinned);
  if (c->gio) cudaFreeHost(c->gio);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

const char* cup_last_error(const cup_ctx* c) {
  if (c && !c->err.empty()) return c->err.c_str();
  return g_last_error.c_str();
}

int cup_set_mesh(cup_ctx* c, int32_t nblocks, const int32_t* level, const int32_t* index) {
  if (!c || nblocks <= 0 || !level || !index) return ctx_fail(c, CUP_ERR_ARG, "cup_set_mesh: bad arguments");
  std::vector<std::array<int32_t, 4>> leaves(nblocks);
  for (int i = 0; i < nblocks; ++i) leaves[i] = {level[i], index[3 * i], index[3 * i + 1], index[3 * i + 2]};
  return install_mesh(c, leaves);
}

static MeshSpec spec_of(const cup_ctx* c) {
  MeshSpec s;
  for (int d = 0; d < 3; ++d) {
    s.bpd[d] = c->cfg.bpd[d];
    s.bc[d] = c->cfg.bc[d];
  }
  s.level_max = c->cfg.level_max;
  s.extent = c->cfg.extent;
  mesh_spec_finalize(s);
  return s;
}

int cup_set_mesh_uniform(cup_ctx* c) {
  if (!c) return ctx_fail(c, CUP_ERR_ARG, "null ctx");
  // every block at -levelStart (levelMax - 1 by default), as the reference's
  // grids start (Simulation.cpp:162-168)
  const int l = c->cfg.level_start >= 0 ? std::min(c->cfg.level_start, c->cfg.level_max - 1) : c->cfg.level_max - 1;
  std::vector<std::array<int32_t, 4>> leaves;
  for (int k = 0; k < c->cfg.bpd[2] << l; ++k)
    for (int j = 0; j < c->cfg.bpd[1] << l; ++j)
      for (int i = 0; i < c->cfg.bpd[0] << l; ++i) leaves.push_back({l, i, j, k});
  return install_mesh(c, leaves);
}

int cup_set_mesh_sphere_wake(cup_ctx* c, const double* ctr, double r, int32_t flow_dir,
                             double near_radius, double wake_len, double wake_radius) {
  if (!c || !ctr) return ctx_fail(c, CUP_ERR_ARG, "null argument");
  return install_mesh(c, mesh_sphere_wake_leaves(spec_of(c), ctr, r, flow_dir, near_radius,
                                                 wake_len, wake_radius));
}

int cup_set_mesh_random(cup_ctx* c, uint64_t seed, double p) {
  if (!c) return ctx_fail(c, CUP_ERR_ARG, "null ctx");
  return install_mesh(c, mesh_random_leaves(spec_of(c), seed, p));
}

int32_t cup_num_blocks(const cup_ctx* c) { return c ? c->mesh.nb : 0; }

int cup_get_blocks(const cup_ctx* c, int32_t* level, int32_t* index, double* h) {
  if (!c) return ctx_fail(nullptr, CUP_ERR_ARG, "null ctx");
  const Mesh& m = c->mesh;
  if (level) std::memcpy(level, m.level.data(), m.nb * sizeof(int32_t));
  if (index) std::memcpy(index, m.index.data(), 3 * m.nb * sizeof(int32_t));
  if (h) std::memcpy(h, m.h.data(), m.nb * sizeof(double));
  return 0;
}

int cup_get_faces(const cup_ctx* c, int32_t* kinds, int32_t* nbrs) {
  if (!c) return ctx_fail(nullptr, CUP_ERR_ARG, "null ctx");
  const Mesh& m = c->mesh;
  if (kinds) std::memcpy(kinds, m.face_kind.data(), 6 * m.nb * sizeof(int32_t));
  if (nbrs) std::memcpy(nbrs, m.face_nbr.data(), 24 * m.nb * sizeof(int32_t));
  return 0;
}

int cup_upload_field(cup_ctx* c, int32_t field, const double* host) {
  if (!c || !host || c->mesh.nb == 0 || c->host_only) return ctx_fail(c, CUP_ERR_ARG, "cup_upload_field: bad arguments or no mesh");
  int nc;
  double* d = field_ptr(c, field, &nc);
  if (!d) return ctx_fail(c, CUP_ERR_ARG, "unknown field id");
  cudaError_t e = cudaMemcpyAsync(d, host, nc * nbn(c) * 8, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return keep(c, set_cuda_error(e, "upload", __FILE__, __LINE__));
  return 0;
}

int cup_download_field(cup_ctx* c, int32_t field, double* host) {
  if (!c || !host || c->mesh.nb == 0 || c->host_only) return ctx_fail(c, CUP_ERR_ARG, "cup_download_field: bad arguments or no mesh");
  int nc;
  double* d = field_ptr(c, field, &nc);
  if (!d) return ctx_fail(c, CUP_ERR_ARG, "unknown field id");
  cudaError_t e = cudaMemcpyAsync(host, d, nc * nbn(c) * 8, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return keep(c, set_cuda_error(e, "download", __FILE__, __LINE__));
  return 0;
}

// Reference block storage <-> SoA device field.  Block k of the caller is
// (level[k], index[3k..3k+2]) at block_ptrs[k]: GridBlock data[iz][iy][ix] of
// VectorElement {u[3]} or ScalarElement {s} (Definitions.h:528-539), Real =
// double.  Every leaf must appear exactly once.
static int blocks_transfer(cup_ctx* c, int32_t field, int32_t n, const int32_t* level, const int32_t* index,
                           double* const* ptrs, bool upload) {
  const char* fn = upload ? "cup_upload_field_blocks" : "cup_download_field_blocks";
  if (!c || c->mesh.nb == 0 || c->host_only || !level || !index || !ptrs)
    return ctx_fail(c, CUP_ERR_ARG, std::string(fn) + ": bad arguments or no mesh");
  if (n != c->mesh.nb)
    return ctx_fail(c, CUP_ERR_ARG, std::string(fn) + ": block count differs from the mesh");
  int nc;
  double* d = field_ptr(c, field, &nc);
  if (!d) return ctx_fail(c, CUP_ERR_ARG, "unknown field id");
  const size_t nbc = nbn(c);
  std::vector<int32_t> slot(n);
  std::vector<char> seen(n, 0);
  for (int k = 0; k < n; ++k) {
    const int b = c->mesh.find(level[k], index[3 * k], index[3 * k + 1], index[3 * k + 2]);
    if (b < 0 || seen[b] || !ptrs[k])
      return ctx_fail(c, CUP_ERR_ARG, std::string(fn) + ": block " + std::to_string(k) +
                                          " is not a leaf of the mesh, repeats one, or has no data");
    seen[b] = 1;
    slot[k] = b;
  }
  std::vector<double> soa(nc * nbc);
  cudaError_t e = cudaSuccess;
  if (!upload) {
    e = cudaMemcpyAsync(soa.data(), d, soa.size() * 8, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return keep(c, set_cuda_error(e, fn, __FILE__, __LINE__));
  }
  for (int k = 0; k < n; ++k) {
    double* blk = ptrs[k];
    const size_t base = size_t(slot[k]) * BN;
    for (int q = 0; q < nc; ++q)
      for (int cell = 0; cell < BN; ++cell) {
        double& s = soa[q * nbc + base + cell];
        double& r = blk[cell * nc + q];
        if (upload)
          s = r;
        else
          r = s;
      }
  }
  if (upload) {
    e = cudaMemcpyAsync(d, soa.data(), soa.size() * 8, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return keep(c, set_cuda_error(e, fn, __FILE__, __LINE__));
  }
  return 0;
}

int cup_upload_field_blocks(cup_ctx* c, int32_t field, int32_t nblocks, const int32_t* level,
                            const int32_t* index, const double* const* block_ptrs) {
  return blocks_transfer(c, field, nblocks, level, index, const_cast<double* const*>(block_ptrs), true);
}

int cup_download_field_blocks(cup_ctx* c, int32_t field, int32_t nblocks, const int32_t* level,
                              const int32_t* index, double* const* block_ptrs) {
  return blocks_transfer(c, field, nblocks, level, index, block_ptrs, false);
}

void* cup_stream(cup_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

double* cup_field_device_ptr(cup_ctx* c, int32_t field) {
  if (!c) return nullptr;
  int nc;
  return field_ptr(c, field, &nc);
}

int cup_poisson_apply_dev(cup_ctx* c, const double* x, double* y, int32_t mean_mode) {
  ProfBind pb_(c);
  if (!c || !x || !y || c->mesh.nb == 0 || c->host_only) return ctx_fail(c, CUP_ERR_ARG, "cup_poisson_apply_dev: bad arguments");
  const int mm = mean_mode >= 0 ? mean_mode : c->cfg.mean_constraint;
  if (int rc = launch_poisson_apply(c->dm, x, y, mm, c->W, c->stream)) return keep(c, rc);
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return keep(c, set_cuda_error(e, "poisson_apply", __FILE__, __LINE__));
  return 0;
}

int cup_block_inverse_dev(cup_ctx* c, const double* in, double* out) {
  ProfBind pb_(c);
  if (!c || !in || !out || c->mesh.nb == 0 || c->host_only) return ctx_fail(c, CUP_ERR_ARG, "cup_block_inverse_dev: bad arguments");
  if (int rc = launch_block_inverse(c->dm, in, out, c->W, c->stream)) return keep(c, rc);
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return keep(c, set_cuda_error(e, "block_inverse", __FILE__, __LINE__));
  return 0;
}

// The pipelined solver's 16 scratch vectors, allocated on its first use for
// the current mesh size.
static int pipelined_vectors(cup_ctx* c, double* vec[16]) {
  const size_t n = nbn(c);
  if (c->pipe_cap < n) {
    c->pipe_arena.release();
    c->pipe_cap = 0;
    for (int i = 0; i < 16; ++i)
      if (int rc = c->pipe_arena.alloc(&c->pipe_vec[i], n)) return rc;
    c->pipe_cap = n;
  }
  for (int i = 0; i < 16; ++i) vec[i] = c->pipe_vec[i];
  return 0;
}

// check_true: recompute ||b - A x||_2 in FP64 after the solve (stats.true_rel);
// the time-step path skips it (-1) since the solvers already test their own
// FP64 residual.
static int solve_impl(cup_ctx* c, const double* b, double* x, cup_solve_stats* stats, bool check_true = true) {
  if (c->ncase > 1) return ctx_fail(c, CUP_ERR_STATE, "a batch of cases solves with cup_batch_poisson_solve_dev");
  SolveParams P{};
  P.tol_abs = c->cfg.poisson_tol;
  P.tol_rel = c->cfg.poisson_tol_rel;
  P.max_iter = c->cfg.poisson_max_iter;
  P.max_restarts = c->cfg.poisson_max_restarts;
  P.mean_mode = c->cfg.mean_constraint;
  P.check_every = 8;
  P.stall_window = 0;
  P.persistent = c->cfg.poisson_persistent;
  P.block_cache = c->cfg.poisson_block_cache;
  SolveStats S{};
  int rc = 0;
  const int solver = c->cfg.poisson_solver;
  const bool learned = solver == CUP_POISSON_B200_LEARNED || solver == CUP_POISSON_B200_LEARNED_MIXED;
  // the two-level solvers: the coarse space of the mesh, built once per mesh
  // (outside the solve's timed region)
  const bool schwarz = solver == CUP_POISSON_B200_SCHWARZ;
  const bool twolevel =
      learned || schwarz || solver == CUP_POISSON_B200_TWOLEVEL || solver == CUP_POISSON_B200_TWOLEVEL_MIXED;
  if (twolevel)
    if (int rc2 = coarse_build(c)) return keep(c, rc2);
  if (learned && !c->cnn.ready)
    return ctx_fail(c, CUP_ERR_STATE, "learned preconditioner has no weights (cup_cnn_init / cup_cnn_set_params)");
  // the local map: the learned one of the current weights (folded outside
  // the timed region), or the exact overlap solve
  LocalMap lm{};
  if (learned)
    if (int rc2 = lmap_prepare(c, &lm)) return keep(c, rc2);
  if (schwarz)
    if (int rc2 = schwarz_prepare(c, &lm)) return keep(c, rc2);
  const LocalMap* lmap = (learned || schwarz) ? &lm : nullptr;
  CUP_CUDA_TRY(cudaEventRecord(c->ev0, c->stream));
  int fallback = 0;
  if (learned) P.stall_window = 40;  // a stall hands over to block-Jacobi below
  const CoarseView cview = c->coarse.view();
  const CoarseView* coarse = twolevel ? &cview : nullptr;
  if (solver == CUP_POISSON_B200_PIPELINED) {
    double* vec[16];
    if (int rc2 = pipelined_vectors(c, vec)) return keep(c, rc2);
    rc = poisson_pipelined(c->dm, b, x, P, c->W, vec, S, c->stream);
  } else if (solver == CUP_POISSON_B200_MIXED || solver == CUP_POISSON_B200_LEARNED_MIXED ||
             solver == CUP_POISSON_B200_TWOLEVEL_MIXED)
    rc = poisson_mixed(c->dm, b, x, P, c->W, S, c->stream, c->h_pinned, lmap, coarse, c->num_sms);
  else
    rc = poisson_bicgstab(c->dm, b, x, P, c->W, S, c->stream, c->h_pinned, lmap, coarse, c->num_sms);
  if (rc) return keep(c, rc);
  if (learned && S.status != SOLVE_CONVERGED && S.status != SOLVE_NAN) {
    // The learned preconditioner stalled: plain block-Jacobi BiCGSTAB from the
    // best iterate, against the original initial residual.
    SolveParams Q = P;
    Q.stall_window = 0;
    Q.max_iter = std::max(1, P.max_iter - S.iterations);
    // the original target as an absolute residual (the restart's own initial
    // residual is not the learned solve's)
    Q.tol_abs = std::max(P.tol_abs, P.tol_rel * S.err_init);
    Q.tol_rel = 0.0;
    SolveStats F{};
    if (int rc2 = poisson_bicgstab(c->dm, b, x, Q, c->W, F, c->stream, c->h_pinned)) return keep(c, rc2);
    S.iterations += F.iterations;
    S.restarts += F.restarts;
    S.status = F.status;
    S.err_opt = F.err_opt;
    fallback = 1;
  }
  CUP_CUDA_TRY(cudaEventRecord(c->ev1, c->stream));
  CUP_CUDA_TRY(cudaEventSynchronize(c->ev1));
  float ms = 0;
  CUP_CUDA_TRY(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  double true_rel = -1.0;
  if (check_true && S.status != SOLVE_NAN) {
    double e = 0;
    if (int rc2 = true_residual_norm(c->dm, b, x, P.mean_mode, c->W, &e, c->stream)) return keep(c, rc2);
    true_rel = S.err_init > 0 ? e / S.err_init : 0.0;
  }
  if (stats) {
    stats->iterations = S.iterations;
    stats->restarts = S.restarts;
    stats->status = S.status;
    stats->fallback = fallback;
    stats->err_init = S.err_init;
    stats->err_final = S.err_opt;
    stats->true_rel = true_rel;
    stats->milliseconds = ms;
  }
  if (S.status == SOLVE_NAN) return ctx_fail(c, CUP_ERR_NAN, "Poisson solve produced NaN");
  if (S.status != SOLVE_CONVERGED) return CUP_SOFT_MAXITER;
  return fallback ? CUP_SOFT_FALLBACK : CUP_OK;
}

int cup_poisson_solve_dev(cup_ctx* c, const double* b, double* x, cup_solve_stats* stats) {
  ProfBind pb_(c);
  if (!c || !b || !x || c->mesh.nb == 0 || c->host_only) return ctx_fail(c, CUP_ERR_ARG, "cup_poisson_solve_dev: bad arguments");
  if (reinterpret_cast<uintptr_t>(x) % 16 != 0)
    return ctx_fail(c, CUP_ERR_ARG, "cup_poisson_solve_dev: d_x must be 16-byte aligned (the solver reads it as 2-wide vectors)");
  return solve_impl(c, b, x, stats);
}

int cup_poisson_solve(cup_ctx* c, cup_solve_stats* stats) {
  ProfBind pb_(c);
  if (!c || c->mesh.nb == 0 || c->host_only) return ctx_fail(c, CUP_ERR_ARG, "cup_poisson_solve: no mesh");
  return solve_impl(c, c->F.lhs, c->proj_open ? c->F.phi : c->F.pres[c->F.pcur], stats);
}

}  // extern "C"

// ===========================================================================
// Obstacles and time-step operators
// ===========================================================================
namespace cup3d {

static ObstacleView ob_view(const cup_ctx* c) {
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

int ctx_upload_obstacle(cup_ctx* c, int nslots, const int32_t* blocks, const double* chi, const double* udef,
                        const double* kin) {
  graph_reset(c);
  const Mesh& m = c->mesh;
  c->obst_arena.release();
  c->ob = DevObstacle();
  if (nslots <= 0) return 0;
  std::vector<int> slot(m.nb, -1), near(m.nb, 0);
  for (int s = 0; s < nslots; ++s) {
    if (blocks[s] < 0 || blocks[s] >= m.nb || slot[blocks[s]] >= 0)
      return ctx_fail(c, CUP_ERR_ARG, "obstacle: invalid or repeated block id");
    slot[blocks[s]] = s;
  }
  for (int b = 0; b < m.nb; ++b) {
    bool nr = slot[b] >= 0;
    for (int f = 0; f < 6 && !nr; ++f) {
      const int k = m.face_kind[6 * b + f];
      const int* nb = &m.face_nbr[24 * b + 4 * f];
      if (k == FACE_SAME || k == FACE_COARSER) nr |= slot[nb[0]] >= 0;
      if (k == FACE_FINER)
        for (int q = 0; q < 4; ++q) nr |= slot[nb[q]] >= 0;
    }
    near[b] = nr;
  }
  DevObstacle& o = c->ob;
  o.nslots = nslots;
  o.h_blocks.assign(blocks, blocks + nslots);
  o.h_chi.assign(chi, chi + size_t(nslots) * BN);
  if (udef)
    o.h_udef.assign(udef, udef + 3 * size_t(nslots) * BN);
  else
    o.h_udef.assign(3 * size_t(nslots) * BN, 0.0);
  for (int i = 0; i < 9; ++i) o.kin[i] = kin ? kin[i] : 0.0;
  o.udef_zero = std::all_of(o.h_udef.begin(), o.h_udef.end(), [](double v) { return v == 0.0; });
  if (c->host_only) return 0;  // host copies only
  DevArena& A = c->obst_arena;
  if (int rc = A.alloc(&o.slot_of_block, m.nb)) return keep(c, rc);
  if (int rc = A.alloc(&o.near, m.nb)) return keep(c, rc);
  if (int rc = A.alloc(&o.block_of_slot, nslots)) return keep(c, rc);
  if (int rc = A.alloc(&o.chi, size_t(nslots) * BN)) return keep(c, rc);
  if (int rc = A.alloc(&o.udef, 3 * size_t(nslots) * BN)) return keep(c, rc);
  CUP_CUDA_TRY(stream_h2d(c->stream, o.slot_of_block, slot.data(), m.nb * sizeof(int)));
  CUP_CUDA_TRY(stream_h2d(c->stream, o.near, near.data(), m.nb * sizeof(int)));
  CUP_CUDA_TRY(stream_h2d(c->stream, o.block_of_slot, blocks, nslots * sizeof(int)));
  CUP_CUDA_TRY(stream_h2d(c->stream, o.chi, o.h_chi.data(), o.h_chi.size() * 8));
  CUP_CUDA_TRY(stream_h2d(c->stream, o.udef, o.h_udef.data(), o.h_udef.size() * 8));
  CUP_CUDA_TRY(stream_h2d(c->stream, c->d_scalars + SC_KIN, o.kin, 9 * sizeof(double)));
  return 0;
}

static int install_host_obstacle(cup_ctx* c, const HostObstacle& h) {
  if (int rc = ctx_upload_obstacle(c, int(h.blocks.size()), h.blocks.data(), h.chi.data(), h.udef.data(), h.kin))
    return rc;
  if (c->host_only) return 0;
  CUP_CUDA_TRY(stream_h2d(c->stream, c->F.chi, h.grid_chi.data(), h.grid_chi.size() * 8));
  return 0;
}

// The CFL number of step `step`, ramped up from 1e-3 over the first `rampup`
// steps (Simulation.cpp:329-333).
double ctx_cfl_factor(const cup_config& cfg, int step) {
  if (step < cfg.rampup) {
    const double x = step / double(cfg.rampup);
    return std::exp(std::log(1e-3) * (1 - x) + std::log(cfg.cfl) * x);
  }
  return cfg.cfl;
}

double ctx_calc_dt(const cup_config& cfg, double hmin, double umax, int step) {
  // Simulation::calcMaxTimestep (Simulation.cpp:326-338); k_calc_dt repeats
  // these operations on the device for captured steps
  const double dtDiffusion = (1.0 / 6.0) * hmin * hmin / (cfg.nu + (1.0 / 6.0) * hmin * umax);
  const double dtAdvection = hmin / (umax + 1e-8);
  return std::min(dtDiffusion, ctx_cfl_factor(cfg, step) * dtAdvection);
}

static int grid_of(const cup_ctx* c) { return c->W.grid; }

static int advect(cup_ctx* c, double dt) {
  Fields& F = c->F;
  for (int s = 0; s < 3; ++s) {
    if (int rc = launch_advect_stage(c->dm, F.vel[F.vcur], F.vel[1 - F.vcur], F.tmpV, dt, c->cfg.nu, c->cfg.uinf,
                                     c->cfg.advection, s, kgrid(c, TG_ADVECT), c->stream))
      return keep(c, rc);
    F.vcur = 1 - F.vcur;
  }
  return 0;
}

static int penalize(cup_ctx* c, double dt) {
  return keep(c, launch_penalize(c->dm, c->F.vel[c->F.vcur], c->F.chi, ob_view(c), c->d_scalars + SC_KIN, dt,
                                 c->cfg.lambda, c->cfg.implicit_penalization, c->d_scalars + SC_FORCE, c->W.partial,
                                 c->W.counters + 11, c->stream));
}

static int project(cup_ctx* c, double dt, int step, cup_solve_stats* stats) {
  Fields& F = c->F;
  c->proj_open = 0;
  double* pold = F.pres[F.pcur];
  double* pnew = F.pres[1 - F.pcur];
  if (int rc = launch_pressure_rhs(c->dm, F.vel[F.vcur], pold, F.chi, ob_view(c), dt, step, c->cfg.step_2nd_start,
                                   F.lhs, F.phi, kgrid(c, TG_RHS), c->stream))
    return keep(c, rc);
  cup_solve_stats st{};
  const int rs = solve_impl(c, F.lhs, F.phi, &st, false);
  if (rs < 0) return rs;
  if (int rc = launch_weighted_sum(c->dm, F.phi, c->d_scalars + SC_SUMS, c->W, c->stream)) return keep(c, rc);
  if (int rc = launch_grad_update(c->dm, F.vel[F.vcur], F.phi, pold, pnew, c->d_scalars + SC_SUMS, dt, step,
                                  c->cfg.step_2nd_start, kgrid(c, TG_GRAD), c->stream))
    return keep(c, rc);
  F.pcur = 1 - F.pcur;
  if (stats) *stats = st;
  return rs;
}

// ---------------------------------------------------------------------------
// Captured time steps.  A step with the CFL dt and the plain solver has no
// host decision inside: dt comes from k_calc_dt (the host supplies only the
// CFL factor of the step, through pinned memory), the kernels read it from
// the device (DevMesh::case_dt), the persistent solver moves its best iterate
// itself, and the state is read back after the step.  The step is captured
// once per (velocity buffer, pressure buffer, p_old term) and replayed.
// ---------------------------------------------------------------------------
void graph_reset(cup_ctx* c) {
  for (cudaGraphExec_t& g : c->gexec)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
}

static SolveParams plain_params(const cup_ctx* c) {
  SolveParams P{};
  P.tol_abs = c->cfg.poisson_tol;
  P.tol_rel = c->cfg.poisson_tol_rel;
  P.max_iter = c->cfg.poisson_max_iter;
  P.max_restarts = c->cfg.poisson_max_restarts;
  P.mean_mode = c->cfg.mean_constraint;
  P.check_every = 8;
  P.stall_window = 0;
  P.persistent = 1;
  P.block_cache = c->cfg.poisson_block_cache;
  return P;
}

static int graph_capture(cup_ctx* c, int vcur, int pcur, int use_pold, cudaGraphExec_t* out) {
  Fields& F = c->F;
  cudaStream_t s = c->stream;
  const int grid = grid_of(c);
  poisson_init_constants();  // before the capture: it writes constant memory
  SolveParams P = plain_params(c);
  P.graph = 1;
  KrylovState init;
  krylov_init_state(P, init);
  CUP_CUDA_TRY(stream_h2d(s, c->W.st_init, &init, sizeof(init)));
  DevMesh dmg = c->dm;
  dmg.case_dt = c->d_scalars + SC_GDT;
  // the two-level solver's coarse space (built before the capture by graph_step)
  const CoarseView cview = c->coarse.view();
  const CoarseView* coarse = c->cfg.poisson_solver == CUP_POISSON_B200_TWOLEVEL ? &cview : nullptr;
  const int step_arg = use_pold ? c->cfg.step_2nd_start + 1 : 0;
  CUP_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  int rc = 0;
  auto run = [&]() -> int {
    CUP_CUDA_TRY(cudaMemcpyAsync(c->d_scalars + SC_GFAC, &c->gio->cfl_fac, sizeof(double), cudaMemcpyHostToDevice, s));
    if (int r = launch_max_u(c->dm, F.vel[vcur], c->cfg.uinf, c->d_scalars + SC_UMAX, c->W.partial,
                             c->W.counters + 10, grid, s))
      return r;
    if (int r = launch_calc_dt(c->d_scalars + SC_UMAX, c->d_scalars + SC_GFAC, c->cfg.nu, c->mesh.spec.hmin,
                               c->d_scalars + SC_GDT, s))
      return r;
    int v = vcur;
    for (int st = 0; st < 3; ++st) {
      if (int r = launch_advect_stage(dmg, F.vel[v], F.vel[1 - v], F.tmpV, 0.0, c->cfg.nu, c->cfg.uinf,
                                      c->cfg.advection, st, kgrid(c, TG_ADVECT), s))
        return r;
      v = 1 - v;
    }
    if (c->ob.nslots > 0)
      if (int r = launch_penalize(dmg, F.vel[v], F.chi, ob_view(c), c->d_scalars + SC_KIN, 0.0, c->cfg.lambda,
                                  c->cfg.implicit_penalization, c->d_scalars + SC_FORCE, c->W.partial,
                                  c->W.counters + 11, s))
        return r;
    double* pold = F.pres[pcur];
    double* pnew = F.pres[1 - pcur];
    if (int r = launch_pressure_rhs(dmg, F.vel[v], pold, F.chi, ob_view(c), 0.0, step_arg, c->cfg.step_2nd_start,
                                    F.lhs, F.phi, kgrid(c, TG_RHS), s))
      return r;
    // event record nodes (external): the solve's device time, read after replay
    CUP_CUDA_TRY(cudaEventRecordWithFlags(c->ev0, s, cudaEventRecordExternal));
    SolveStats S{};
    if (int r = poisson_bicgstab(c->dm, F.lhs, F.phi, P, c->W, S, s, c->h_pinned, nullptr, coarse, c->num_sms))
      return r;
    CUP_CUDA_TRY(cudaEventRecordWithFlags(c->ev1, s, cudaEventRecordExternal));
    if (int r = launch_weighted_sum(c->dm, F.phi, c->d_scalars + SC_SUMS, c->W, s)) return r;
    if (int r = launch_grad_update(dmg, F.vel[v], F.phi, pold, pnew, c->d_scalars + SC_SUMS, 0.0, step_arg,
                                   c->cfg.step_2nd_start, kgrid(c, TG_GRAD), s))
      return r;
    CUP_CUDA_TRY(cudaMemcpyAsync(&c->gio->dt, c->d_scalars + SC_GDT, sizeof(double), cudaMemcpyDeviceToHost, s));
    CUP_CUDA_TRY(cudaMemcpyAsync(&c->gio->st, c->W.st, sizeof(KrylovState), cudaMemcpyDeviceToHost, s));
    CUP_CUDA_TRY(cudaMemcpyAsync(&c->gio->bar_error, c->W.bar_error, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUP_CUDA_TRY(cudaMemcpyAsync(&c->gio->kerr, c->dm.kerr, sizeof(int), cudaMemcpyDeviceToHost, s));
    return 0;
  };
  solver_pdl(false);
  rc = run();
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

static int graph_step(cup_ctx* c, int step, double* dt_used, cup_solve_stats* stats) {
  Fields& F = c->F;
  const int use_pold = step > c->cfg.step_2nd_start ? 1 : 0;
  const int key = F.vcur | (F.pcur << 1) | (use_pold << 2);
  if (c->cfg.poisson_solver == CUP_POISSON_B200_TWOLEVEL) {
    // the captured steps hold the coarse space's buffers: a rebuilt one (a
    // new mesh) needs new captures
    const int before = c->coarse.mesh_version;
    const float* inv = c->coarse.inv;
    if (int rc = coarse_build(c)) return keep(c, rc);
    if (c->coarse.mesh_version != before || c->coarse.inv != inv) graph_reset(c);
  }
  if (!c->gexec[key])
    if (int rc = graph_capture(c, F.vcur, F.pcur, use_pold, &c->gexec[key])) return keep(c, rc);
  c->gio->cfl_fac = ctx_cfl_factor(c->cfg, step);
  CUP_CUDA_TRY(cudaGraphLaunch(c->gexec[key], c->stream));
  CUP_CUDA_TRY(cudaStreamSynchronize(c->stream));
  F.vcur = 1 - F.vcur;  // three advection stages
  F.pcur = 1 - F.pcur;
  const KrylovState& K = c->gio->st;
  if (c->gio->bar_error) return ctx_fail(c, CUP_ERR_CUDA, "persistent BiCGSTAB: a grid barrier wait timed out");
  if (c->gio->kerr) return ctx_fail(c, CUP_ERR_CUDA, "stencil kernel: a wait for a block's bulk copies timed out");
  if (dt_used) *dt_used = c->gio->dt;
  if (!(c->gio->dt > 0)) return ctx_fail(c, CUP_ERR_NAN, "dt <= 0 or NaN (Simulation.cpp:344-347)");
  float ms = 0;
  CUP_CUDA_TRY(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  const int status = K.done ? K.status : SOLVE_MAXITER;
  if (stats) {
    stats->iterations = K.k;
    stats->restarts = K.restarts;
    stats->status = status;
    stats->fallback = 0;
    stats->err_init = K.err_init;
    stats->err_final = K.err_opt;
    stats->true_rel = -1.0;
    stats->milliseconds = ms;
  }
  if (status == SOLVE_NAN) return ctx_fail(c, CUP_ERR_NAN, "Poisson solve produced NaN");
  return status == SOLVE_CONVERGED ? CUP_OK : CUP_SOFT_MAXITER;
}

}  // namespace cup3d

extern "C" {

int cup_obstacle_sphere(cup_ctx* c, const double* ctr, double r, const double* vel, const double* omega) {
  if (!c || !ctr || c->mesh.nb == 0) return ctx_fail(c, CUP_ERR_ARG, "cup_obstacle_sphere: bad arguments");
  if (c->ncase > 1) return ctx_fail(c, CUP_ERR_STATE, "cup_obstacle_sphere: not available on a batch of cases");
  const double z[3] = {0, 0, 0};
  HostObstacle h;
  make_sphere(c->mesh, ctr, r, vel ? vel : z, omega ? omega : z, h);
  body_record(c, 0, false, ctr, &r, nullptr, vel, omega);
  return install_host_obstacle(c, h);
}

int cup_obstacle_ellipsoid(cup_ctx* c, const double* ctr, const double* ax, const double* q, const double* vel,
                           const double* omega) {
  if (!c || !ctr || !ax || !q || c->mesh.nb == 0)
    return ctx_fail(c, CUP_ERR_ARG, "cup_obstacle_ellipsoid: bad arguments");
  if (c->ncase > 1) return ctx_fail(c, CUP_ERR_STATE, "cup_obstacle_ellipsoid: not available on a batch of cases");
  const double z[3] = {0, 0, 0};
  HostObstacle h;
  make_ellipsoid(c->mesh, ctr, ax, q, vel ? vel : z, omega ? omega : z, h);
  body_record(c, 1, false, ctr, ax, q, vel, omega);
  return install_host_obstacle(c, h);
}

int cup_set_obstacle(cup_ctx* c, int32_t nslots, const int32_t* blocks, const double* chi, const double* udef,
                     const double* kin) {
  if (!c || c->mesh.nb == 0 || (nslots > 0 && (!blocks || !chi)))
    return ctx_fail(c, CUP_ERR_ARG, "cup_set_obstacle: bad arguments");
  if (c->ncase > 1) return ctx_fail(c, CUP_ERR_STATE, "cup_set_obstacle: not available on a batch of cases");
  c->body = BodyState();  // raw data: no shape to move
  return ctx_upload_obstacle(c, nslots, blocks, chi, udef, kin);
}

int cup_get_obstacle(const cup_ctx* cc, int32_t* blocks, double* chi, double* udef, double* kin) {
  if (!cc) return ctx_fail(nullptr, CUP_ERR_ARG, "null ctx");
  cup_ctx* c = const_cast<cup_ctx*>(cc);  // a device-created body fetches its host copies here
  if ((blocks || chi || udef) && !c->host_only)
    if (int rc = ctx_obstacle_host_copies(c)) return keep(c, rc);
  const DevObstacle& o = c->ob;
  if (blocks) std::copy(o.h_blocks.begin(), o.h_blocks.end(), blocks);
  if (chi) std::copy(o.h_chi.begin(), o.h_chi.end(), chi);
  if (udef) std::copy(o.h_udef.begin(), o.h_udef.end(), udef);
  if (kin) std::copy(o.kin, o.kin + 9, kin);
  return o.nslots;
}

int cup_max_u(cup_ctx* c, double* umax) {
  ProfBind pb_(c);
  if (!c || !umax || c->mesh.nb == 0 || c->host_only) return ctx_fail(c, CUP_ERR_ARG, "cup_max_u: bad arguments");
  if (c->ncase > 1) return ctx_fail(c, CUP_ERR_STATE, "cup_max_u: not available on a batch of cases");
  if (int rc = launch_max_u(c->dm, c->F.vel[c->F.vcur], c->cfg.uinf, c->d_scalars + SC_UMAX, c->W.partial,
                            c->W.counters + 10, grid_of(c), c->stream))
    return keep(c, rc);
  cudaError_t e = cudaMemcpyAsync(umax, c->d_scalars + SC_UMAX, sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return keep(c, set_cuda_error(e, "max_u", __FILE__, __LINE__));
  return 0;
}

int cup_compute_dt(cup_ctx* c, int32_t step, double* dt) {
  double umax = 0;
  if (int rc = cup_max_u(c, &umax)) return rc;
  *dt = ctx_calc_dt(c->cfg, c->mesh.spec.hmin, umax, step);
  if (!(*dt > 0)) return ctx_fail(c, CUP_ERR_NAN, "dt <= 0 or NaN (Simulation.cpp:344-347)");
  return 0;
}

int cup_advect_diffuse(cup_ctx* c, double dt) {
  ProfBind pb_(c);
  if (!c || c->mesh.nb == 0 || c->host_only) return ctx_fail(c, CUP_ERR_ARG, "cup_advect_diffuse: no mesh");
  if (c->ncase > 1) return ctx_fail(c, CUP_ERR_STATE, "cup_advect_diffuse: not available on a batch of cases");
  if (int rc = advect(c, dt)) return rc;
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return keep(c, set_cuda_error(e, "advect_diffuse", __FILE__, __LINE__));
  return 0;
}

int cup_penalize(cup_ctx* c, double dt, double* force6) {
  ProfBind pb_(c);
  if (!c || c->mesh.nb == 0 || c->host_only) return ctx_fail(c, CUP_ERR_ARG, "cup_penalize: no mesh");
  if (c->ncase > 1) return ctx_fail(c, CUP_ERR_STATE, "cup_penalize: not available on a batch of cases");
  if (int rc = penalize(c, dt)) return rc;
  cudaError_t e = cudaSuccess;
  if (force6) e = cudaMemcpyAsync(force6, c->d_scalars + SC_FORCE, 6 * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return keep(c, set_cuda_error(e, "penalize", __FILE__, __LINE__));
  return 0;
}

int cup_pressure_rhs(cup_ctx* c, double dt, int32_t step) {
  ProfBind pb_(c);
  if (!c || c->mesh.nb == 0 || c->host_only) return ctx_fail(c, CUP_ERR_ARG, "cup_pressure_rhs: no mesh");
  if (c->ncase > 1) return ctx_fail(c, CUP_ERR_STATE, "cup_pressure_rhs: not available on a batch of cases");
  Fields& F = c->F;
  c->proj_open = 0;  // a second call starts the projection again from the same pressure
  if (int rc = launch_pressure_rhs(c->dm, F.vel[F.vcur], F.pres[F.pcur], F.chi, ob_view(c), dt, step,
                                   c->cfg.step_2nd_start, F.lhs, F.phi, kgrid(c, TG_RHS), c->stream))
    return keep(c, rc);
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return keep(c, set_cuda_error(e, "pressure_rhs", __FILE__, __LINE__));
  if (int rk = ctx_check_kernels(c)) return rk;
  c->proj_open = 1;
  return 0;
}

int cup_pressure_finish(cup_ctx* c, double dt, int32_t step) {
  ProfBind pb_(c);
  if (!c || c->mesh.nb == 0 || c->host_only) return ctx_fail(c, CUP_ERR_ARG, "cup_pressure_finish: no mesh");
  if (!c->proj_open)
    return ctx_fail(c, CUP_ERR_STATE, "cup_pressure_finish: no projection open (call cup_pressure_rhs first)");
  Fields& F = c->F;
  double* pold = F.pres[F.pcur];
  double* pnew = F.pres[1 - F.pcur];
  if (int rc = launch_weighted_sum(c->dm, F.phi, c->d_scalars + SC_SUMS, c->W, c->stream)) return keep(c, rc);
  if (int rc = launch_grad_update(c->dm, F.vel[F.vcur], F.phi, pold, pnew, c->d_scalars + SC_SUMS, dt, step,
                                  c->cfg.step_2nd_start, kgrid(c, TG_GRAD), c->stream))
    return keep(c, rc);
  F.pcur = 1 - F.pcur;
  c->proj_open = 0;
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return keep(c, set_cuda_error(e, "pressure_finish", __FILE__, __LINE__));
  return ctx_check_kernels(c);
}

int cup_pressure_project(cup_ctx* c, double dt, int32_t step, cup_solve_stats* stats) {
  ProfBind pb_(c);
  if (!c || c->mesh.nb == 0 || c->host_only) return ctx_fail(c, CUP_ERR_ARG, "cup_pressure_project: no mesh");
  if (c->ncase > 1) return ctx_fail(c, CUP_ERR_STATE, "cup_pressure_project: not available on a batch of cases");
  const int rc = project(c, dt, step, stats);
  if (rc < 0) return rc;
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return keep(c, set_cuda_error(e, "pressure_project", __FILE__, __LINE__));
  if (int rk = ctx_check_kernels(c)) return rk;
  return rc;
}

int cup_step(cup_ctx* c, int32_t step, double dt, double* dt_used, cup_solve_stats* stats) {
  ProfBind pb_(c);
  if (!c || c->mesh.nb == 0 || c->host_only) return ctx_fail(c, CUP_ERR_ARG, "cup_step: no mesh");
  if (c->ncase > 1) return ctx_fail(c, CUP_ERR_STATE, "cup_step: not available on a batch of cases");
  c->proj_open = 0;
  if (body_update_uinf(c)) graph_reset(c);  // CreateObstacles: the frame follows the body
  const bool moving = body_moves(c);
  if (!(dt > 0) && c->cfg.step_graph &&
      (c->cfg.poisson_solver == CUP_POISSON_B200 || c->cfg.poisson_solver == CUP_POISSON_B200_TWOLEVEL) &&
      !c->prof.on && !moving) {
    const int rc = graph_step(c, step, dt_used, stats);
    if (rc >= 0) {
      body_coef_u(c, step, c->gio->dt);
      c->dt_prev = c->gio->dt;
    }
    return rc;
  }
  if (!(dt > 0))
    if (int rc = cup_compute_dt(c, step, &dt)) return rc;
  if (dt_used) *dt_used = dt;
  body_coef_u(c, step, dt);
  c->dt_prev = dt;
  if (moving)  // CreateObstacles: Obstacle::update, then chi at the new pose
    if (int rc = body_advance(c, step, dt)) return keep(c, rc);
  if (int rc = advect(c, dt)) return rc;
  if (body_free(c))  // UpdateObstacles: free degrees of freedom from the fluid momentum
    if (int rc = update_obstacles(c, dt, nullptr)) return keep(c, rc);
  if (c->ob.nslots > 0)
    if (int rc = penalize(c, dt)) return rc;
  const int rc = project(c, dt, step, stats);
  if (rc < 0) return rc;
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return keep(c, set_cuda_error(e, "step", __FILE__, __LINE__));
  if (int rk = ctx_check_kernels(c)) return rk;
  return rc;
}

}  // extern "C"

extern "C" {

int cup_profile(cup_ctx* c, int32_t enable) {
  if (!c || c->host_only) return ctx_fail(c, CUP_ERR_ARG, "cup_profile: no device context");
  c->prof.reset();
  c->prof.on = enable != 0;
  return 0;
}

int cup_profile_read(cup_ctx* c, char* buf, int32_t len) {
  if (!c || !buf || len <= 0) return ctx_fail(c, CUP_ERR_ARG, "cup_profile_read: bad arguments");
  c->prof.flush();
  std::ostringstream os;
  os.precision(9);
  os << "{";
  for (size_t i = 0; i < c->prof.names.size(); ++i) {
    if (i) os << ",";
    os << "\"" << c->prof.names[i] << "\":[" << c->prof.acc[i].launches << "," << c->prof.acc[i].ms << "]";
  }
  os << "}";
  const std::string js = os.str();
  if (int(js.size()) + 1 > len) return ctx_fail(c, CUP_ERR_ARG, "cup_profile_read: buffer too small");
  std::memcpy(buf, js.c_str(), js.size() + 1);
  return int(js.size());
}

}  // extern "C"
