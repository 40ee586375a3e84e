// Internal definition of cup_ctx (the C-ABI handle).
#pragma once
#include <string>
#include <array>
#include <vector>

#include "../../include/cup3d_b200.h"
#include "common.cuh"
#include "mesh.h"
#include "cnn.cuh"
#include "poisson.cuh"
#include "profiler.h"

namespace cup3d {

struct DevArena {
  std::vector<void*> ptrs;
  ~DevArena() { release(); }
  void release() {
    for (void* p : ptrs) cudaFree(p);
    ptrs.clear();
  }
  template <class T>
  int alloc(T** out, size_t n) {
    void* p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc(&p, n * sizeof(T));
    if (e != cudaSuccess) return set_cuda_error(e, "cudaMalloc", __FILE__, __LINE__);
    ptrs.push_back(p);
    *out = static_cast<T*>(p);
    return 0;
  }
};

// Obstacle data on the device: per-slot chi and udef blocks, and the rigid
// body kinematics (ObstacleBlock.h:41-42, Obstacle.h getters).
struct DevObstacle {
  int nslots = 0;
  int* slot_of_block = nullptr;   // nb, -1 when the block holds no obstacle cells
  int* near = nullptr;            // nb, block or a face neighbour holds obstacle cells
  int* block_of_slot = nullptr;   // nslots
  double* chi = nullptr;          // nslots*512
  double* udef = nullptr;         // 3*nslots*512 (component-major)
  double kin[9] = {0};            // CM[3], vel[3], omega[3]
  std::vector<int> h_blocks;      // host copies for cup_get_obstacle
  std::vector<double> h_chi, h_udef;
  // created on the device (cup_obstacle_*_dev): buffers sized for every block
  // of the mesh, the host copies fetched when read
  int dev_cap = 0;
  bool host_stale = false;
  bool udef_zero = false;  // every slot's udef is zero (bodies created by the library: rigid)
  double* d_mom = nullptr;        // 4 per slot: sum chi h^3 (x, y, z), sum chi h^3
  double* d_origin = nullptr;     // 3 nb block origins
  void* d_result = nullptr;       // slot count, mass, kinematics
  // momentum integrals of UpdateObstacles: 29 per slot, then their sums
  double* d_qslot = nullptr;
  double* d_qsum = nullptr;
  int q_cap = 0;
};

// Learned preconditioner state: weights, Adam moments, training scratch and
// the device dataset of (input, target) samples.
struct CnnState {
  DevArena arena, data_arena;
  CnnWeights W{};
  float *adam_m = nullptr, *adam_v = nullptr, *grad = nullptr, *gpart = nullptr, *loss = nullptr;
  float *ds_in = nullptr, *ds_target = nullptr;
  int *ds_count = nullptr, *idx = nullptr;
  int cap = 0, count = 0, adam_t = 0, train_grid = 148, idx_cap = 0;
  int ntest = 0;  // the last ntest samples are held out of training (cup_cnn_eval)
  bool ready = false;
  // the network folded into the solver's matrix (lmap.cuh), refolded when the
  // weights change; the fold's scratch; the solver's lab buffer
  DevArena lab_arena;
  uint4* lmap_w = nullptr;
  float *fold_in = nullptr, *fold_out = nullptr;
  uint16_t* lmap_lab = nullptr;
  uint4* schwarz_w = nullptr;  // the one-cell-overlap local solve (schwarz_prepare)
  size_t lab_cap = 0;
  bool folded = false;
};

// Per-case device buffers of a batch's time step.
struct BatchStep {
  int* first = nullptr;         // ncase + 1 block offsets
  int* slot_first = nullptr;    // ncase + 1 obstacle-slot offsets
  double* dt = nullptr;         // ncase
  double* sums = nullptr;       // 2 ncase: (sum phi h^3, sum h^3)
  double* kin = nullptr;        // 9 ncase: CM, velocity, angular velocity
  double* umax = nullptr;       // ncase
  double* force = nullptr;      // 6 ncase: penalization force and torque
  double* bscratch = nullptr;   // 2 nb
  double* slot_force = nullptr; // 6 nslots
  double* hmin = nullptr;       // ncase: finest spacing of each case
  double* mixed = nullptr;      // 2 ncase: the mixed-precision batch's per-case sums
  // pinned host copies filled by captured steps
  double* h_dt = nullptr;       // ncase
  double* h_force = nullptr;    // 6 ncase
  KrylovState* h_st = nullptr;  // ncase
  int* h_err = nullptr;
  void* h_block = nullptr;      // the pinned allocation holding them
};

// Scratch of the blocked dense inverse (coarse.cu), with room for cap x cap.
struct InverseScratch {
  DevArena arena;
  int cap = 0;
  double *M0 = nullptr, *Pinv = nullptr, *T = nullptr, *Cp = nullptr, *pv = nullptr;
  int* flag = nullptr;
};

// Coarse space of the two-level preconditioners (coarse.cu): A_c^-1 of the
// Galerkin coarse operator (one unknown per block) and the apply buffers.
struct CoarseSpace {
  DevArena arena;               // the arrays below, with room for cap blocks
  int cap = 0;
  int nb = 0;                   // blocks it was built for (0: not built)
  int mesh_version = -1;        // cup_ctx::mesh_version it was built for
  int colours = 0;              // colours of the set-up
  float* inv = nullptr;         // A_c^-1, nb x nb, row-major, FP32 (a preconditioner needs no more)
  double* rc = nullptr;         // nb: restricted vector
  double* rc2 = nullptr;        // nb: the second one of the persistent solver
  double* yc = nullptr;         // nb: coarse correction
  double* w = nullptr;          // nb: 512 h^3 of each block
  // set-up scratch: A_c (FP64, then its inverse in place), colours, block sums,
  // the per-colour neighbour map (jcap entries)
  double* ac = nullptr;
  int* colour = nullptr;
  double* sum = nullptr;
  DevArena jarena;
  size_t jcap = 0;
  int* jmap = nullptr;
  InverseScratch iscratch;
  std::vector<double> host_ac;  // A_c (row-major), for checks (kept when keep_host)
  bool keep_host = false;
  int pivoted = 0;              // A_c^-1 came from the column-wise pivoted Gauss-Jordan
  CoarseView view() const { return CoarseView{nb, inv, rc, rc2, yc, w}; }
};

// Offsets into cup_ctx::d_scalars
enum : int { SC_SUMS = 0, SC_UMAX = 2, SC_FORCE = 8, SC_KIN = 16, SC_TARGET_SUMSQ = 32, SC_GFAC = 48, SC_GDT = 49 };

// Host side of a captured step: the CFL factor going in, the state coming out.
struct GraphIO {
  double cfl_fac;
  double dt;
  int bar_error;
  int kerr;  // the staged kernels' error word
  KrylovState st;
};

// Shape, pose and motion of the context's body (Obstacle.h: position,
// quaternion, transVel, angVel and their previous values for BDF2).
struct BodyState {
  int kind = -1;           // -1: none (or raw data), 0 sphere, 1 ellipsoid
  bool on_device = false;  // re-created by the device path
  double pos[3] = {0, 0, 0}, quat[4] = {1, 0, 0, 0};
  double r = 0, ax[3] = {0, 0, 0};
  double vel[3] = {0, 0, 0}, omega[3] = {0, 0, 0};
  double old_pos[3] = {0, 0, 0}, old_quat[4] = {1, 0, 0, 0};
  double abs_pos[3] = {0, 0, 0}, old_abs_pos[3] = {0, 0, 0};  // position in the lab frame (absPos)
  // free degrees of freedom: velocities from the fluid momentum
  // (!bForcedInSimFrame[d], !bBlockRotation[d]); the others keep vel / omega
  int free_t[3] = {0, 0, 0}, free_r[3] = {0, 0, 0};
  // frame of reference following the body along these axes (bFixFrameOfRef)
  int fix_frame[3] = {0, 0, 0};
};

// Device copies of a mesh's tables, with room for `cap` blocks; a context
// keeps two sets, so that a mesh adaptation fills one while its field
// transfer still reads the other.
struct MeshTables {
  DevArena arena;
  int cap = 0;
  int *fk = nullptr, *fn = nullptr, *ix = nullptr, *kerr = nullptr;
  int* plan = nullptr;  // 9 per block: where an adapted mesh's block takes its values from
  double* h = nullptr;
};

struct Fields {
  double* vel[2] = {nullptr, nullptr};  // ping-pong, 3*nb*512 each
  int vcur = 0;
  double* tmpV = nullptr;               // 3*nb*512
  double* pres[2] = {nullptr, nullptr}; // ping-pong pressure
  int pcur = 0;
  double* lhs = nullptr;
  double* chi = nullptr;
  double* phi = nullptr;                // Poisson unknown (increment)
};

}  // namespace cup3d

struct cup_ctx {
  cup_config cfg;
  cup3d::Mesh mesh;
  cup3d::DevMesh dm{};
  cup3d::DevArena field_arena, obst_arena;
  // mesh tables in two sets (tabs[tab_cur] in use); the field arena holds
  // room for field_cap blocks and is allocated again only to grow, so a mesh
  // adaptation within that room allocates and frees nothing
  cup3d::MeshTables tabs[2];
  int tab_cur = 0;
  int field_cap = 0;
  int* d_order = nullptr;  // the block-group kernels' visit order (field arena)
  cup3d::Fields F;
  cup3d::PoissonWork W{};
  cup3d::DevObstacle ob;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int* h_pinned = nullptr;        // small pinned host buffer
  double* d_scalars = nullptr;    // 64 device doubles for misc reductions
  int num_sms = 148;
  bool host_only = false;         // device < 0: mesh work only
  cup3d::Profiler prof;
  cup3d::CnnState cnn;
  std::string err;
  // batches of independent cases (cup_batch_create); ncase == 1 otherwise
  int ncase = 1;
  std::vector<int> case_first;        // ncase + 1 block offsets
  std::vector<cup3d::Mesh> case_mesh;  // each case's own mesh
  cup3d::BatchWork B{};
  cup3d::BatchStep T{};
  // launch grids of the stencil kernels chosen by cup_autotune (0: W.grid)
  int tgrid[3] = {0, 0, 0};
  // captured time steps, by (velocity buffer, pressure buffer, p_old term)
  cudaGraphExec_t gexec[8] = {};
  cup3d::GraphIO* gio = nullptr;      // pinned
  cup3d::DevArena batch_arena;
  // moving bodies: pose, the previous step's dt and the BDF2 coefficients of
  // the pose update (SimulationData::coefU)
  cup3d::BodyState body;
  double* d_diag = nullptr;  // ComputeDissipation partial sums (field arena)
  int diag_cap = 0;
  double dt_prev = 0.0;
  double coef_u[3] = {1.5, -2.0, 0.5};
  // A projection split at its solve (cup_pressure_rhs ... cup_pressure_finish):
  // while open, CUP_FIELD_PRES is the pressure increment phi that the Poisson
  // solve reads as its guess and writes, as sim.pres is in the reference
  // between `pres = 0` and `pres += pOld` (PressureProjection.cpp:388-446).
  int proj_open = 0;
  // incremented whenever the mesh changes (keys what is built per mesh)
  int mesh_version = 0;
  cup3d::CoarseSpace coarse;
  // a batch's two-level preconditioners (cup_batch_create with b200_twolevel)
  cup3d::DevArena bcoarse_arena;
  cup3d::BatchCoarse bcoarse;
  // moving bodies of a batch of cases (batch_bodies_advance): each case's
  // body, BDF2 coefficients and previous dt; the shapes on the device
  bool batch_moving = false;
  std::vector<cup3d::BodyState> case_body;
  std::vector<std::array<double, 3>> case_coef;
  std::vector<double> case_dt_prev;
  void* d_shapes = nullptr;
  // scratch vectors of the pipelined solver (allocated on first use)
  cup3d::DevArena pipe_arena;
  double* pipe_vec[16] = {nullptr};
  size_t pipe_cap = 0;
};

namespace cup3d {
enum : int { TG_ADVECT = 0, TG_RHS = 1, TG_GRAD = 2 };
// Launch grid of stencil kernel k (TG_*): the tuned one, else the default.
inline int kgrid(const cup_ctx* c, int k) { return c->tgrid[k] > 0 ? c->tgrid[k] : c->W.grid; }
// Binds the context's profiler to this thread for the duration of an API call.
struct ProfBind {
  Profiler* prev;
  ProfBind(cup_ctx* c) : prev(t_prof) { t_prof = (c && c->prof.on) ? &c->prof : nullptr; }
  ~ProfBind() { t_prof = prev; }  // nested API calls restore the caller's binding
};
int ctx_fail(cup_ctx* c, int code, const std::string& msg);
// Uploads c->mesh into table set `set` (-1: the set in use) and points the
// device mesh at it.
int ctx_upload_mesh(cup_ctx* c, int set = -1);
// CUP_ERR_CUDA with a message when a staged stencil kernel reported a timed-out
// wait (call after synchronising the context's stream).
int ctx_check_kernels(cup_ctx* c);
// Room for the fields and solver work of c->mesh, all zeroed; the obstacle
// data dropped.
int ctx_alloc_fields(cup_ctx* c);
// Room for nb blocks in the field arena (allocated again, a quarter larger,
// only when nb exceeds it; then every field pointer changes).
int fields_reserve(cup_ctx* c, int nb);
// Zeroes the fields (but vel[vcur] and pres[pcur] when keep_current), sets
// the launch grids and uploads the visit order of c->mesh.
int fields_reset(cup_ctx* c, bool keep_current);
// Installs an obstacle (nslots blocks with chi, udef and kinematics kin[9]).
int ctx_upload_obstacle(cup_ctx* c, int nslots, const int32_t* blocks, const double* chi, const double* udef,
                        const double* kin);
// Moving bodies (obstacles_dev.cu).  body_record keeps the shape and motion
// of a body just created (r: the sphere radius or the ellipsoid axes; q null
// for a sphere); body_moves: the body is not static and its velocity + uinf
// or angular velocity is non-zero; body_coef_u: the BDF2 coefficients of the
// step (Simulation.cpp:361-370); body_advance: Obstacle::update with dt, then
// chi at the new pose by the path the body was created with.
void body_record(cup_ctx* c, int kind, bool on_device, const double* ctr, const double* r, const double* q,
                 const double* vel, const double* omega);
bool body_moves(const cup_ctx* c);
// ObstacleVector::updateUinf (ObstacleVector.h:74-83) for the axes the body
// fixes: uinf = -velocity there; returns true when uinf changed.
bool body_update_uinf(cup_ctx* c);
// The body has a free degree of freedom (UpdateObstacles runs every step).
bool body_free(const cup_ctx* c);
// UpdateObstacles (ObstaclesUpdate.cpp:189-216): momentum integrals over the
// body, Obstacle::computeVelocities, the new kinematics on the device.
// out (may be null): translational and angular velocity, force, torque.
int update_obstacles(cup_ctx* c, double dt, double out[12]);
void body_coef_u(cup_ctx* c, int step, double dt);
int body_advance(cup_ctx* c, int step, double dt);
// chi of the context's body at its current pose, by the path it was created
// with, keeping its motion history (after a mesh change).
int body_recreate(cup_ctx* c);
// A batch's moving bodies: every case's pose advanced with its dt[k], then all
// bodies created again on the flattened mesh (obstacles_dev.cu).
int batch_bodies_advance(cup_ctx* c, int step, const double* dt);
// Mesh adaptation (adapt.cu): the per-block refinement indicator, and one
// adaptation of the mesh with the fields moved onto it (*changed = 0 when
// the mesh stays as it is).
int adapt_indicator(cup_ctx* c, std::vector<double>& out);
int adapt_mesh(cup_ctx* c, int* changed);
// Builds (once per mesh) the coarse space of the two-level preconditioners.
int coarse_build(cup_ctx* c);
// Inverse of an n x n host matrix (row-major) on the device (coarse.cu).
int device_inverse(const double* a, int n, double* d_inv, int sms, cudaStream_t s);
// The inverse in place of an n x n device matrix, index `last` (>= 0) last in
// the pivot order; *fallback = 1 when the pivoted column-wise form ran.
// Scratch from `scratch` when given (kept for the next call), else allocated for the call.
int device_inverse_dev(double* M, int n, int last, int sms, cudaStream_t s, int* fallback,
                       InverseScratch* scratch = nullptr);
// The learned map of the current weights for the solver (folds them when they
// changed; the lab buffer for the current mesh).
int lmap_prepare(cup_ctx* c, LocalMap* out);
// The exact one-cell-overlap local solve as a local map (built once).
int schwarz_prepare(cup_ctx* c, LocalMap* out);
// The block of the mean-constraint row when the mean mode replaces a row, else -1.
int mean_block_of(const cup_ctx* c);
// Fetches the host copies of a device-created obstacle (no-op otherwise).
int ctx_obstacle_host_copies(cup_ctx* c);
// Drops the captured time steps (after any change of mesh, obstacle or
// solver settings).
void graph_reset(cup_ctx* c);
// The CFL number of a step (ramped up over the first -rampup steps).
double ctx_cfl_factor(const cup_config& cfg, int step);
// Simulation::calcMaxTimestep for spacing hmin and max |u| umax.
double ctx_calc_dt(const cup_config& cfg, double hmin, double umax, int step);
size_t nbn(const cup_ctx* c);
// Host<->device copies and fills ordered on a stream, waiting for it before
// returning.  The context stream is non-blocking, so cudaMemcpy / cudaMemset
// on the legacy default stream are not ordered with the kernels that follow
// on it (a pageable cudaMemcpy may return before its DMA has landed).
cudaError_t stream_h2d(cudaStream_t s, void* dst, const void* src, size_t bytes);
cudaError_t stream_d2h(cudaStream_t s, void* dst, const void* src, size_t bytes);
cudaError_t stream_zero(cudaStream_t s, void* dst, size_t bytes);
}  // namespace cup3d
