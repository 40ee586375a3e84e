/* cup3d_b200 — C ABI of the B200-native CUP3D time-step hot path.
 *
 * One context holds one simulation's mesh and fields on one GPU.  Every call
 * returns an int status: 0 OK, > 0 soft (solver stopped without reaching the
 * tolerance, fallback used), < 0 hard error (CUDA failure, bad argument, bad
 * mesh, NaN).  cup_last_error() gives the message.  No C++ exception crosses
 * this boundary.  A context is used by one host thread at a time.
 *
 * Field layout on the host side of this ABI: structure-of-arrays, component c
 * of block b, cell (ix,iy,iz) at f[c*nb*512 + b*512 + iz*64 + iy*8 + ix], blocks
 * in the order cup_get_blocks() reports (the space-filling-curve order set by
 * cup_set_mesh).  cup_upload_field_blocks / cup_download_field_blocks take
 * the reference's block storage instead (one pointer per block, VectorBlock =
 * 512 x {u,v,w}, ScalarBlock = 512 x s, [iz][iy][ix]; Definitions.h:528-539).
 */
#ifndef CUP3D_B200_H
#define CUP3D_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CUP_OK 0
#define CUP_SOFT_MAXITER 1      /* Poisson solve stopped at the iteration/restart cap */
#define CUP_SOFT_FALLBACK 2     /* learned preconditioner stalled; block-Jacobi used */
#define CUP_ERR_CUDA (-1)
#define CUP_ERR_ARG (-2)
#define CUP_ERR_MESH (-3)
#define CUP_ERR_NAN (-4)
#define CUP_ERR_STATE (-5)

/* boundary conditions (BCflag, Definitions.h:38) */
#define CUP_BC_FREESPACE 0
#define CUP_BC_PERIODIC 1
#define CUP_BC_WALL 2

/* advection schemes (AdvectionDiffusion.cpp:32-103) */
#define CUP_ADV_UPWIND5 0
#define CUP_ADV_WENO5 1

/* Poisson solvers selectable by -poissonSolver (PoissonSolverBase.cpp:30-52) */
#define CUP_POISSON_B200 0          /* "b200": FP64 BiCGSTAB, exact block inverse */
#define CUP_POISSON_B200_MIXED 1    /* "b200_mixed": FP32 inner, FP64 refinement */
#define CUP_POISSON_B200_LEARNED 2  /* "b200_learned": flexible BiCGSTAB, two-level preconditioner
                                       with the CNN on each block (coarse correction + block
                                       inverse + learned correction) */
#define CUP_POISSON_B200_LEARNED_MIXED 3 /* "b200_learned_mixed": both */
#define CUP_POISSON_B200_TWOLEVEL 4 /* "b200_twolevel": BiCGSTAB, two-level preconditioner without
                                       the network (coarse correction + block inverse); the
                                       method the learned one is compared with */
#define CUP_POISSON_B200_PIPELINED 6 /* "b200_pipelined": the reference CPU solver's pipelined BiCGSTAB
                                       (PoissonSolverAMR.cpp:13-358: exact block inverse, residual
                                       replacement every 50 iterations, restarts, best iterate), in
                                       one persistent launch with two grid barriers per iteration */
#define CUP_POISSON_B200_SCHWARZ 5  /* "b200_schwarz": the two-level preconditioner with the exact
                                       one-cell-overlap local solve of each block (restricted
                                       additive Schwarz) in place of the block inverse; the local
                                       map the network is trained to reproduce */
#define CUP_POISSON_B200_TWOLEVEL_MIXED 7 /* "b200_twolevel_mixed": the two-level preconditioner in
                                       FP32 inner solves inside FP64 iterative refinement */

/* field ids */
#define CUP_FIELD_VEL 0   /* 3 components */
#define CUP_FIELD_PRES 1
#define CUP_FIELD_CHI 2
#define CUP_FIELD_LHS 3   /* Poisson right-hand side (sim.lhs) */
#define CUP_FIELD_TMPV 4  /* 3 components */

typedef struct cup_ctx cup_ctx;

/* Run parameters; names follow the reference's command-line flags
 * (SimulationData.cpp:21-132). */
typedef struct cup_config {
  int32_t bpd[3];              /* -bpdx -bpdy -bpdz */
  int32_t level_max;           /* -levelMax */
  int32_t bc[3];               /* -BC_x -BC_y -BC_z */
  double extent;               /* -extent (largest side) */
  double nu;                   /* -nu */
  double cfl;                  /* -CFL */
  int32_t rampup;              /* -rampup */
  double lambda;               /* -lambda */
  int32_t implicit_penalization; /* -implicitPenalization */
  double uinf[3];              /* frame velocity sim.uinf */
  int32_t advection;           /* CUP_ADV_* */
  int32_t mean_constraint;     /* -bMeanConstraint */
  double poisson_tol;          /* -poissonTol (absolute, on ||r||_2) */
  double poisson_tol_rel;      /* -poissonTolRel */
  int32_t poisson_solver;      /* CUP_POISSON_* */
  int32_t poisson_max_iter;    /* 1000 in the reference */
  int32_t poisson_max_restarts;/* 100 in the reference */
  int32_t step_2nd_start;      /* 2 in the reference */
  int32_t device;              /* CUDA device ordinal */
  int32_t poisson_block_cache; /* -poissonBlockCache: mesh-table entries per block group kept in
                                  shared memory by the persistent solver (0-4; 4 by default);
                                  a tuning knob with no reference counterpart */
  int32_t step_graph;          /* -stepGraph: cup_step with dt <= 0 and the plain solver replays a
                                  CUDA graph of the whole step (1, default) or launches the
                                  kernels one by one (0); the same kernels either way */
  int32_t static_obstacles;    /* -StaticObstacles (default 0): bodies created by cup_obstacle_sphere(_dev)
                                  / cup_obstacle_ellipsoid(_dev) whose velocity + uinf or angular
                                  velocity is non-zero move every cup_step (Obstacle::update) and
                                  their chi is re-created at the new pose (CreateObstacles) */
  double rtol;                 /* -Rtol: refine a block whose indicator reaches it (default 1) */
  double ctol;                 /* -Ctol: compress blocks whose indicators stay below it (default 0.1) */
  int32_t level_max_vorticity; /* -levelMaxVorticity (default levelMax) */
  int32_t level_start;         /* -levelStart: level of cup_set_mesh_uniform (default levelMax - 1) */
  int32_t poisson_persistent;  /* -poissonPersistent: 1 (default) one cooperative launch per solve; 0 the
                                  host-driven form, five kernels per iteration and a host check every 8
                                  (plain, mixed and two-level solvers; for per-phase profiles) */
} cup_config;

typedef struct cup_solve_stats {
  int32_t iterations;
  int32_t restarts;
  int32_t status;      /* 1 converged, 2 iteration cap, 3 restart cap, 4 NaN */
  int32_t fallback;    /* learned solver fell back to block-Jacobi */
  double err_init;     /* ||b - A x0||_2 */
  double err_final;    /* best ||r||_2 (the iterate returned) */
  double true_rel;     /* FP64 ||b - A x||_2 / ||b - A x0||_2 of the returned x */
  double milliseconds; /* device time of the solve */
} cup_solve_stats;

/* Defaults of the reference (SimulationData.cpp:21-132) and the "b200" solver. */
void cup_config_default(cup_config* cfg);
/* ParseArguments-style: "-key value" pairs, e.g. "-bpdx 4 -levelMax 2 -nu 0.01". */
int cup_config_parse(cup_config* cfg, const char* args);

cup_ctx* cup_create(const cup_config* cfg);      /* NULL on failure: cup_last_error(NULL) */
void cup_destroy(cup_ctx* ctx);
const char* cup_last_error(const cup_ctx* ctx);  /* ctx may be NULL */

/* ---- mesh (host C++: ordering, neighbour tables; Cubism's role) ---- */
/* Leaf blocks in any order: level[n], index[3n].  Reordered along the
 * space-filling curve; fields are reallocated and zeroed. */
int cup_set_mesh(cup_ctx* ctx, int32_t nblocks, const int32_t* level, const int32_t* index);
/* Uniform mesh at level 0 of cfg->bpd. */
int cup_set_mesh_uniform(cup_ctx* ctx);
/* Refined around a sphere (centre c, radius r) and its wake along flow_dir
 * (+1/-1 in x), refined to level_max-1, 2:1 balanced. */
int cup_set_mesh_sphere_wake(cup_ctx* ctx, const double* c, double r, int32_t flow_dir,
                             double near_radius, double wake_len, double wake_radius);
/* Random 2:1-balanced refinement (tests). */
int cup_set_mesh_random(cup_ctx* ctx, uint64_t seed, double refine_prob);
int32_t cup_num_blocks(const cup_ctx* ctx);
/* level[n], index[3n], h[n] in device order; any pointer may be NULL */
int cup_get_blocks(const cup_ctx* ctx, int32_t* level, int32_t* index, double* h);
/* face tables: kinds[6n] (0 same, 1 boundary, 2 coarser, 3 finer), nbrs[24n] */
int cup_get_faces(const cup_ctx* ctx, int32_t* kinds, int32_t* nbrs);

/* ---- fields ---- */
int cup_upload_field(cup_ctx* ctx, int32_t field, const double* host);
int cup_download_field(cup_ctx* ctx, int32_t field, double* host);
/* The same in the reference's block storage: block k is (level[k],
 * index[3k..3k+2]) with its GridBlock data (Real = double, cells [iz][iy][ix],
 * VectorElement {u[3]} interleaved) at block_ptrs[k], blocks in any order
 * (e.g. the order of the reference's vInfo()).  Every leaf exactly once. */
int cup_upload_field_blocks(cup_ctx* ctx, int32_t field, int32_t nblocks, const int32_t* level,
                            const int32_t* index, const double* const* block_ptrs);
int cup_download_field_blocks(cup_ctx* ctx, int32_t field, int32_t nblocks, const int32_t* level,
                              const int32_t* index, double* const* block_ptrs);
/* Device pointer of a field (SoA), for zero-copy use by device-resident callers. */
double* cup_field_device_ptr(cup_ctx* ctx, int32_t field);
/* The context's CUDA stream (cudaStream_t) on which every call enqueues its work. */
void* cup_stream(cup_ctx* ctx);

/* ---- raw device-side operators on caller device buffers (nb*512 doubles) ---- */
/* y = A x: the AMR Poisson operator of PoissonSolverExp::getMat with the
 * mean constraint of the config (or mean_mode >= 0 to override). */
int cup_poisson_apply_dev(cup_ctx* ctx, const double* d_x, double* d_y, int32_t mean_mode);
/* out = (1/h) P_inv in per block (the preconditioner of BiCGSTAB.cu:526-527). */
int cup_block_inverse_dev(cup_ctx* ctx, const double* d_in, double* d_out);
/* Solves A x = b on device buffers; x: initial guess in, solution out
 * (d_x 16-byte aligned, as cudaMalloc returns it). */
int cup_poisson_solve_dev(cup_ctx* ctx, const double* d_b, double* d_x, cup_solve_stats* stats);

/* ---- PoissonSolverBase::solve(): RHS in CUP_FIELD_LHS, guess and result in CUP_FIELD_PRES ---- */
int cup_poisson_solve(cup_ctx* ctx, cup_solve_stats* stats);

/* ---- batches of independent cases (no counterpart in the reference, which
 * runs one case per process) ---- */
/* A new context over the meshes of ncases device contexts, concatenated in
 * case order (case k's blocks follow case k-1's, each case in its own block
 * order); the cases keep their own mean-constraint rows, boundary
 * conditions, obstacles and current velocity, pressure and chi fields, which
 * are copied in.  The other settings (tolerances, -bMeanConstraint, nu, CFL,
 * rampup, lambda, uinf, advection scheme, device) are case 0's; every case
 * must use the same device and -bMeanConstraint.  The cases are not
 * modified.  NULL on failure: cup_last_error(NULL). */
cup_ctx* cup_batch_create(int32_t ncases, cup_ctx* const* cases);
int32_t cup_batch_num_cases(const cup_ctx* batch);  /* 1 for a plain context */
/* Blocks first .. first+nblocks-1 of the batch (and of its fields) are case k's. */
int cup_batch_case_blocks(const cup_ctx* batch, int32_t k, int32_t* first, int32_t* nblocks);
/* One BiCGSTAB per case, all in one device launch: each case has its own
 * scalars, restarts, stopping test and best iterate.  d_x (16-byte aligned):
 * initial guess in, each case's solution out; stats[ncases].  Returns the
 * worst outcome over the cases (true_rel is not computed: -1). */
int cup_batch_poisson_solve_dev(cup_ctx* batch, const double* d_b, double* d_x, cup_solve_stats* stats);
/* One time step of every case (cup_step per case: advection-diffusion,
 * penalization, pressure projection), each case with its own dt: dt_in[k]
 * (or, when dt_in is NULL or dt_in[k] <= 0, Simulation::calcMaxTimestep from
 * the case's own max |u| and finest spacing).  dt_used[ncases]; force[6 ncases]
 * (penalization force and torque per case, may be NULL); stats[ncases] (may
 * be NULL).  The Poisson solves of all cases run in one device launch.
 * Bodies move unless -StaticObstacles 1: when a case's sphere or ellipsoid
 * moves, every step advances each case's pose with that case's dt
 * (Obstacle::update, the case's own BDF2 history) and creates every body
 * again at its new pose, as cup_step does for one case; such a batch steps
 * kernel by kernel.  cup_batch_create refuses free bodies and frames that
 * follow a body when bodies move. */
int cup_batch_step(cup_ctx* batch, int32_t step, const double* dt_in, double* dt_used, double* force,
                   cup_solve_stats* stats);

/* ---- launch-shape tuning (no reference counterpart) ---- */
/* Times candidate launch shapes on the context's own mesh and fields and
 * keeps the fastest: the grids of the advection, pressure-RHS and gradient
 * kernels (multiples of the SM count) and the CTA count of the persistent
 * solver (one to two per SM; a plain context only), which sets how many
 * blocks each block group takes per phase.  choice[4] = the chosen grids
 * (advection, RHS, gradient, solver); best_ms[4] (may be NULL) = their times
 * (per launch; per iteration for the solver).  Overwrites the scratch fields
 * (CUP_FIELD_LHS, CUP_FIELD_TMPV and the buffers a step writes next); call it
 * between steps.  Results do not depend on the grids except for the solver's
 * summation order. */
int cup_autotune(cup_ctx* ctx, int32_t* choice, float* best_ms);

/* ---- obstacles (host-side CreateObstacles; one body per context) ---- */
/* Sphere of radius r at c (Sphere.cpp); chi by ObstaclesCreate.cpp:18-121;
 * kin = velocity[3], angular velocity[3] (may be NULL).  Also sets CUP_FIELD_CHI. */
int cup_obstacle_sphere(cup_ctx* ctx, const double* c, double r, const double* vel, const double* omega);
/* Ellipsoid with semi-axes ax[3] rotated by the unit quaternion q = (w,x,y,z). */
int cup_obstacle_ellipsoid(cup_ctx* ctx, const double* c, const double* ax, const double* q,
                           const double* vel, const double* omega);
/* The same bodies created on the device (no host work on the blocks): the slot
 * list, chi, udef and CUP_FIELD_CHI equal those of cup_obstacle_sphere /
 * cup_obstacle_ellipsoid bit for bit, the centre of mass to rounding (other
 * summation order).  One 96-byte device-to-host read of the slot count and
 * kinematics; cup_get_obstacle fetches the host copies when called. */
int cup_obstacle_sphere_dev(cup_ctx* ctx, const double* c, double r, const double* vel, const double* omega);
int cup_obstacle_ellipsoid_dev(cup_ctx* ctx, const double* c, const double* ax, const double* q,
                               const double* vel, const double* omega);
/* Free degrees of freedom of the body (1 = free): translation along x, y, z
 * (!bForcedInSimFrame) and rotation about x, y, z (!bBlockRotation).  Free
 * ones take their velocity from the fluid momentum in every cup_step
 * (UpdateObstacles); the others keep the creation's velocity / angular
 * velocity.  Bodies are created with every degree of freedom imposed. */
int cup_obstacle_free(cup_ctx* ctx, const int32_t* free_trans, const int32_t* free_rot);
/* Frame of reference following the body (bFixFrameOfRef; ObstacleVector::
 * updateUinf): along the axes with fix[d] = 1, uinf = -the body's velocity at
 * the start of every step.  Other axes keep the configured uinf (the
 * reference sets them to 0 whenever it updates uinf). */
int cup_obstacle_fix_frame(cup_ctx* ctx, const int32_t* fix);
/* The frame velocity uinf[3] in use. */
int cup_get_uinf(const cup_ctx* ctx, double* uinf);
/* CreateObstacles (ObstaclesCreate.cpp:303-323) for the step `step` of length
 * dt: the body's pose advanced by Obstacle::update and its chi re-created,
 * when it moves (see static_obstacles); cup_step does this itself. */
int cup_create_obstacles(cup_ctx* ctx, double dt, int32_t step);
/* UpdateObstacles (ObstaclesUpdate.cpp:189-216): the momentum integrals of the
 * current velocity over the body and Obstacle::computeVelocities (6x6 solve).
 * out12 (may be NULL): translational velocity[3], angular velocity[3],
 * force[3] = mass dV/dt, torque[3] = J dOmega/dt. */
int cup_update_obstacles(cup_ctx* ctx, double dt, double* out12);
/* Raw obstacle data: nslots obstacle blocks, block_of_slot[nslots] (device
 * order), chi[nslots*512], udef[3*nslots*512] (component-major), kin[9] =
 * centre of mass, velocity, angular velocity.  nslots = 0 removes the body. */
int cup_set_obstacle(cup_ctx* ctx, int32_t nslots, const int32_t* block_of_slot, const double* chi,
                     const double* udef, const double* kin);
/* Reads back the obstacle data; returns nslots (arrays may be NULL to query). */
int cup_get_obstacle(const cup_ctx* ctx, int32_t* block_of_slot, double* chi, double* udef, double* kin);

/* ---- diagnostics ---- */
/* ComputeDissipation (ComputeDissipation.cpp:17-140) of the current velocity,
 * pressure and chi: out20 = circulation[3], linear impulse[3], linear
 * momentum[3], angular impulse[3], angular momentum[3], pressure power,
 * viscous power, helicity, kinetic energy, enstrophy (the columns of the
 * reference's diagnostics.dat after step and time). */
int cup_compute_dissipation(cup_ctx* ctx, double* out20);

/* ---- restart files (Simulation::serialize / deserialize) ---- */
/* Writes dir/field.restart and dir/shape_0.restart in the reference's text
 * formats (SimulationData.cpp:200-250, Obstacle.cpp:443-472; the body file
 * adds the shape after the reference's keys) and dir/restart_<step>.cupf with
 * the leaves, velocity and pressure (the reference's HDF5 dumps; no HDF5 here). */
int cup_write_restart(cup_ctx* ctx, const char* dir, int32_t step, double time);
/* Reads them back: mesh from the leaves, fields, uinf, the previous dt, the
 * body with its pose history and its chi; *time (may be NULL) = the saved
 * time.  Stepping on from step + 1... gives the results of the uninterrupted
 * run bit for bit. */
int cup_read_restart(cup_ctx* ctx, const char* dir, int32_t step, double* time);

/* ---- mesh adaptation (Simulation::adaptMesh, Simulation.cpp:128-149) ----
 * cup_adapt_indicator: each block's refinement indicator (nblocks values in
 * cup_get_blocks order): the largest vorticity magnitude over its cells with
 * GradChiOnTmp's rules (ProcessHelpers.h:17-69): 1e10 where the body's
 * interface (0.00001 < chi < 0.9) meets the block or its face ghost layers,
 * 0 for cells inside the body, (Rtol+Ctol)/2 for cells at or above Rtol on
 * level levelMaxVorticity-1.
 * cup_adapt_mesh: refines blocks whose indicator is >= Rtol, merges eight
 * siblings whose indicators are all < Ctol, keeps the 2:1 balance, moves
 * velocity and pressure to the new mesh (copy, linear prolongation with
 * central slopes, 8-cell means), zeroes tmpV and the right-hand side and
 * creates the body's chi again.  Cubism's MeshAdaptation, which does this in
 * the reference, is not in its tree: these rules are this library's.
 * *changed (may be NULL): 1 when the mesh changed.  Obstacle data given by
 * cup_set_obstacle cannot be re-created: CUP_ERR_STATE. */
int cup_adapt_indicator(cup_ctx* ctx, double* out);
int cup_adapt_mesh(cup_ctx* ctx, int32_t* changed);

/* ---- the time-step operators (Operator::operator()(dt) of the reference) ---- */
int cup_max_u(cup_ctx* ctx, double* umax);                          /* findMaxU */
/* calcMaxTimestep (Simulation.cpp:309-375) for `step`: dt from max|u+uinf|. */
int cup_compute_dt(cup_ctx* ctx, int32_t step, double* dt);
int cup_advect_diffuse(cup_ctx* ctx, double dt);                    /* AdvectionDiffusion */
int cup_penalize(cup_ctx* ctx, double dt, double* force_torque6);   /* Penalization */
int cup_pressure_project(cup_ctx* ctx, double dt, int32_t step, cup_solve_stats* stats);
/* PressureProjection split at its Poisson solve, as the reference runs it
 * (PressureProjection.cpp:331-468, solve() at :402):
 *   cup_pressure_rhs    KernelPressureRHS and, for step > 2, KernelDivPressure
 *                       (:340-394) into CUP_FIELD_LHS from the current velocity,
 *                       pressure, chi and body; keeps the pressure as p_old and
 *                       opens the projection: CUP_FIELD_PRES is then the
 *                       pressure increment, zero, as sim.pres after `pres = 0`;
 *   cup_poisson_solve   (PoissonSolverBase::solve) solves into that increment;
 *   cup_pressure_finish zero mean, p += p_old for step > 2, KernelGradP and the
 *                       velocity update (:404-467); closes the projection.
 * cup_pressure_finish without an open projection returns CUP_ERR_STATE.
 * cup_pressure_project and cup_step run all three in one call. */
int cup_pressure_rhs(cup_ctx* ctx, double dt, int32_t step);
int cup_pressure_finish(cup_ctx* ctx, double dt, int32_t step);
/* One time step: AdvectionDiffusion, Penalization (if a body is set),
 * PressureProjection.  dt <= 0: computed by calcMaxTimestep; *dt_used gets it. */
int cup_step(cup_ctx* ctx, int32_t step, double dt, double* dt_used, cup_solve_stats* stats);

/* Changes the Poisson solver settings of a context (-poissonSolver,
 * -poissonTol, -poissonTolRel and the iteration cap). */
int cup_set_poisson(cup_ctx* ctx, int32_t solver, double tol_abs, double tol_rel, int32_t max_iter);
/* Longest wait, in SM clock cycles, of one CTA at one grid barrier of the
 * persistent Poisson solvers (0: the default, 2^31 cycles, about a second).
 * A wait that runs out ends the solve: every CTA leaves at its next barrier,
 * the solve returns CUP_ERR_CUDA with "a grid barrier wait timed out", and
 * the next solve starts afresh (the solution buffer holds partial results). */
int cup_set_barrier_limit(cup_ctx* ctx, int64_t cycles);

/* ComputeForces::operator() (FluidSolidForces.cpp:213-229, run by Simulation::advance after
 * the projection, Simulation.cpp:214-215) with the sums and derived quantities of
 * Obstacle::computeForces (Obstacle.cpp:271-300), for the context's sphere or ellipsoid body
 * on the current velocity and pressure.  out[23]: surfForce[3], presForce[3], viscForce[3],
 * surfTorque[3], drag, thrust, Pout, PoutBnd, defPower, defPowerBnd, pLocom, Pthrust, Pdrag,
 * EffPDef, EffPDefBnd (all zero without a body).  The velocity stencil of a surface point
 * reaches up to 4 cells beyond its block; these cells are read at the block's own level, so
 * a point whose stencil reaches a coarser or finer block, or beyond a non-periodic domain
 * boundary, returns CUP_ERR_MESH (bodies inside a region of uniform refinement satisfy it). */
int cup_compute_forces(cup_ctx* ctx, double* out);

/* ---- learned preconditioner (no counterpart in the reference: the new slot at
 * the preconditioner call sites PoissonSolverAMR.h:183-222, BiCGSTAB.cu:526-527).
 * z = P A_c^-1 P^T r + BJ(r) + (s/h) CNN(r_lab / s): the coarse correction, the exact
 * block inverse and a per-block 3-D CNN correction of the block's residual lab (4 linear
 * conv 3^3 layers, 16 channels, BF16 weights, FP32 accumulation; no biases, so the
 * preconditioner is a fixed linear map).  The solver applies the network folded into one
 * 512 x 896 matrix on the tensor cores. ---- */
int32_t cup_cnn_num_params(void);
int cup_cnn_init(cup_ctx* ctx, uint64_t seed);                 /* random initial weights */
int cup_cnn_set_params(cup_ctx* ctx, const float* params);     /* cup_cnn_num_params() floats */
int cup_cnn_get_params(cup_ctx* ctx, float* params);
int cup_cnn_dataset_reserve(cup_ctx* ctx, int32_t capacity);   /* samples (one per block per pair) */
/* adds one sample per block from a device residual r of a solver iterate: the input is r's
 * block lab (block + one-cell face layers, residual rules), the target the correction of the
 * one-cell-overlap local solve over the block inverse, [L_s^-1 lab]_interior - B^-1 r (the
 * "b200_schwarz" local map).  d_e (the iterate's error x* - x) is accepted and not used (may
 * be NULL): a local map fitted to the error itself is a poor preconditioner, because the
 * error's smooth part cannot be told from a block's lab (a least-squares fit of it made the
 * two-level solve of a uniform test problem take 534 instead of 28 iterations). */
int cup_cnn_dataset_add(cup_ctx* ctx, const double* d_r, const double* d_e);
int32_t cup_cnn_dataset_size(const cup_ctx* ctx);
/* the last ntest samples are held out of training; cup_cnn_eval: the network's
 * residual-norm loss on them (|L (z - t)|^2, L the block Laplacian, the loss the
 * training minimises) relative to that of the zero prediction */
int cup_cnn_holdout(cup_ctx* ctx, int32_t ntest);
int cup_cnn_eval(cup_ctx* ctx, float* rel_loss);
/* `steps` Adam steps on random minibatches (seeded) minimising the residual-norm loss
 * |L (z - t)|^2 (L: the 7-point Laplacian of the 8^3 block, zero outside), relative to
 * the targets' scale; per-step loss into loss_out (or NULL) */
int cup_cnn_train(cup_ctx* ctx, int32_t steps, int32_t batch, float lr, uint64_t seed, float* loss_out);
/* network forward / loss and gradient on host arrays (n samples of 10^3 inputs, 8^3 targets) */
int cup_cnn_forward_host(cup_ctx* ctx, const float* in, float* out, int32_t n);
int cup_cnn_grad_host(cup_ctx* ctx, const float* in, const float* target, int32_t n, float* grad, float* loss);
/* z = block inverse of r + the network on r's block labs (the network's own
 * convolution layers), per block */
int cup_cnn_precond_dev(cup_ctx* ctx, const double* d_r, double* d_z);
/* The same through the solver's path: block inverse + the network folded into
 * one 512 x 896 matrix (BF16 tensor-core GEMM on the BF16 star labs of r). */
int cup_cnn_map_apply_dev(cup_ctx* ctx, const double* d_r, double* d_z);
/* z = block inverse of r + the one-cell-overlap local solve's correction (the
 * "b200_schwarz" local map), per block, on the same path */
int cup_schwarz_apply_dev(cup_ctx* ctx, const double* d_r, double* d_z);

/* Network forward on host arrays, as cup_cnn_forward_host, without allocating
 * or freeing device memory.  No counterpart in the reference.
 *
 * For callers that cannot allocate: cup_cnn_forward_host allocates and frees
 * staging buffers on every call, and cudaFree waits until the whole device is
 * idle, which stalls a solve or time step running on other streams; a caller
 * whose device memory is owned by another allocator may have none to give.
 * This variant stages the samples in one static device array instead, so it
 * takes at most CUP_CNN_FORWARD_NOALLOC_MAX samples per call (387,072 bytes
 * of staging per device) and returns CUP_ERR_ARG, with a message, for more.
 *
 * The staging array is shared by every context on a device within the
 * process: concurrent calls would race on it, so the library serialises the
 * calls with a process-wide lock and each call returns only after its
 * outputs are on the host.  The first call on a device looks the array's
 * address up (cudaGetSymbolAddress) and keeps it; make that first call before
 * beginning any stream capture on the device. */
#define CUP_CNN_FORWARD_NOALLOC_MAX 64
int cup_cnn_forward_host_noalloc(cup_ctx* ctx, const float* in, float* out, int32_t n);

/* ---- coarse space of the two-level solvers (no counterpart in the reference,
 * whose preconditioner is block-local).  One unknown per block; A_c = P^T A P
 * with P constant over each block, built through the device operator once
 * per mesh (at most 8192 blocks), inverted once on the device. ----
 * cup_coarse_matrix: builds it; out (may be NULL): A_c, nblocks^2 doubles,
 * row-major, blocks in cup_get_blocks order; *colours (may be NULL): the
 * colours of the set-up's block colouring.
 * cup_coarse_apply_dev: d_z = P A_c^-1 P^T d_r on device buffers.
 * cup_dense_inverse_dev: the inverse that the coarse space uses, in place of
 * the n x n row-major FP64 device matrix d_a: blocked Gauss-Jordan (panels of
 * 32 pivots, no pivoting across panels) with index `last` (-1: none) moved to
 * the end of the pivot order, checked by A^-1 (A v) = v to 1e-6 for a fixed
 * probe v; when a pivot block is near-singular or the check fails, column-wise
 * Gauss-Jordan with partial pivoting, and *pivoted (may be NULL) = 1.
 * CUP_ERR_MESH for a singular matrix. */
int cup_coarse_matrix(cup_ctx* ctx, double* out, int32_t* colours);
int cup_coarse_apply_dev(cup_ctx* ctx, const double* d_r, double* d_z);
int cup_dense_inverse_dev(cup_ctx* ctx, double* d_a, int32_t n, int32_t last, int32_t* pivoted);

/* ---- profiling (the reference's DeviceProfiler, Utils/DeviceProfiler.cuh) ---- */
/* Enables per-kernel CUDA-event timing (resets the counters). */
int cup_profile(cup_ctx* ctx, int32_t enable);
/* JSON object {"phase": [launches, milliseconds], ...} into buf; returns its length. */
int cup_profile_read(cup_ctx* ctx, char* buf, int32_t len);

#ifdef __cplusplus
}
#endif
#endif
