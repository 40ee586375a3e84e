/* CPU FP64 oracle for the CUP3D time-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library restates, in plain C++/OpenMP, the
 * reference algorithms of the per-time-step path (AdvectionDiffusion,
 * Penalization, PressureProjection, the Poisson operator and both BiCGSTAB
 * solvers with their block preconditioners).  Only tests/, the smoke() entry
 * and bench.py's CPU-baseline leg may load it; the product never does.
 *
 * Parity status: the reference tree cannot be compiled here (its Cubism
 * submodule is empty, no MPI/HDF5/GSL), so the oracle is pinned against
 * known-answer tests built from the reference's own formulas and tests
 * (tests/cubismup3d/TestBoundaries.cpp ghost-shift test, P_inv * L = I,
 * polynomial exactness of the upwind/WENO stencils, RK3 coefficients).  On
 * uniform meshes every formula is the reference's; at coarse-fine faces the
 * ghost interpolation for lab-based stencils is our documented definition
 * (Cubism's is absent), while the Poisson operator follows
 * PoissonSolverExp.cpp:112-373 exactly.
 *
 * Field layout everywhere: SoA, component c of block b cell (ix,iy,iz) at
 *   f[c*nb*512 + b*512 + iz*64 + iy*8 + ix].
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_mesh orc_mesh;

/* Mesh from a leaf list (levels[nb], index[3*nb]) in the caller's block order.
 * bc[d]: 0 freespace, 1 periodic, 2 wall.  Returns NULL on an invalid mesh. */
orc_mesh* orc_mesh_create(int nb, const int32_t* level, const int32_t* index, const int32_t* bpd,
                          int level_max, const int32_t* bc, double extent);
void orc_mesh_destroy(orc_mesh* m);
int orc_mesh_nb(const orc_mesh* m);
double orc_mesh_h(const orc_mesh* m, int b);
double orc_mesh_hmin(const orc_mesh* m);
/* face kinds as the oracle sees them: 6*nb ints (0 same,1 boundary,2 coarser,3 finer) */
void orc_mesh_faces(const orc_mesh* m, int32_t* kinds, int32_t* nbrs /* 24*nb */);

/* ---- Poisson operator (PoissonSolverExp.cpp:221-373, PoissonSolverAMR.h:108-172) ---- */
int64_t orc_poisson_nnz(orc_mesh* m, int mean_constraint);
void orc_poisson_csr(orc_mesh* m, int mean_constraint, int64_t* rowptr, int64_t* col, double* val);
void orc_poisson_apply(orc_mesh* m, int mean_constraint, const double* x, double* y);

/* ---- block preconditioners ---- */
void orc_pinv(double* P /* 512*512 row major */);                       /* PoissonSolverExp.cpp:17-111 */
void orc_precond_pinv(orc_mesh* m, const double* P, const double* in, double* out); /* BiCGSTAB.cu:526-527 */
void orc_precond_cg(orc_mesh* m, const double* in, double* out);       /* PoissonSolverAMRKernels.cpp:268-332 */

/* ---- Krylov solvers.  stats[0]=iterations, [1]=restarts, [2]=initial norm,
 *      [3]=final (best) norm, [4]=converged flag. ---- */
int orc_bicgstab_gpu(orc_mesh* m, int mean_constraint, int precond, const double* b, double* x,
                     double tol, double tol_rel, int max_restarts, int max_iter, double* stats);
int orc_bicgstab_pipelined(orc_mesh* m, int mean_constraint, int precond, const double* b,
                           double* x, double tol, double tol_rel, int max_iter, double* stats);

/* ---- lab (block + ghost layers), for ghost-fill tests ---- */
void orc_fill_lab(orc_mesh* m, const double* field, int ncomp, int G, int block, int vector_bc,
                  double* lab /* ncomp*(8+2G)^3 */);

/* ---- operators ---- */
double orc_max_u(orc_mesh* m, const double* vel, const double* uinf);
double orc_dt(double hmin, double nu, double cfl, double umax, int step, int rampup);
/* scheme: 0 upwind5, 1 weno5.  One full low-storage RK3 step. */
void orc_advect_diffuse(orc_mesh* m, double* vel, double* tmpV, double dt, double nu,
                        const double* uinf, int scheme);
/* one RK stage only (tmpV += RHS(vel) with flux correction, no update) */
void orc_advect_rhs(orc_mesh* m, const double* vel, double* tmpV, double dt, double nu,
                    const double* uinf, int scheme, double coef);

/* Obstacle data on obstacle blocks.  obst_slot[nb]: -1 or slot s; chi_o and
 * udef_o hold per-slot blocks (chi_o[s*512+cell], udef_o[(c*nslots+s)*512+cell]).
 * ob: CM[3], vel[3], omega[3]. force_out: 6 reals (F, T). */
void orc_penalize(orc_mesh* m, double* vel, const double* chi, const int32_t* obst_slot,
                  int nslots, const double* chi_o, const double* udef_o, const double* ob,
                  double dt, double lambda, int implicit, double* force_out);

/* Pressure projection (PressureProjection.cpp:331-468).  solver: 0 GPU-style
 * BiCGSTAB with exact block inverse, 1 pipelined BiCGSTAB with block CG. */
void orc_pressure_project(orc_mesh* m, double* vel, double* pres, const double* chi,
                          const int32_t* obst_slot, int nslots, const double* chi_o,
                          const double* udef_o, double dt, int step, int mean_constraint,
                          int solver, double tol, double tol_rel, double* stats,
                          double* lhs_out /* optional: RHS handed to the solver */);

/* the RHS kernel alone (KernelPressureRHS + optional KernelDivPressure) */
void orc_pressure_rhs(orc_mesh* m, const double* vel, const double* pres, const double* chi,
                      const int32_t* obst_slot, int nslots, const double* chi_o,
                      const double* udef_o, double dt, int step, double* lhs);
/* grad p update alone: vel += (-dt h^2/2 grad p + flux corr)/h^3 */
void orc_grad_update(orc_mesh* m, double* vel, const double* pres, double dt);
// ComputeDissipation's 20 diagnostics (ComputeDissipation.cpp:17-109).
void orc_dissipation(orc_mesh* m, const double* vel, const double* pres, const double* chi, double nu, double* out);

/* ---- obstacle creation (ObstaclesCreate.cpp:18-148, Sphere.cpp:19-51,
 * Ellipsoid.cpp:22-300).  kind 0 sphere (shape[0] = radius), 1 ellipsoid
 * (shape = semi-axes, q = unit quaternion w, x, y, z).  Fill margin 3 hmin,
 * hmin the finest possible spacing of the mesh (SimulationData.cpp:162).
 * Outputs: obst_slot[nb] (-1 or the slot, slots in block order),
 * block_of_slot[nb], chi_o[nb*512] (per slot), chi_grid[nb*512],
 * mom[4] = sum chi h^3 (x, y, z), sum chi h^3.  Returns the slot count. ---- */
int orc_create_obstacle(orc_mesh* m, int kind, const double* centre, const double* shape, const double* q,
                        int32_t* obst_slot, int32_t* block_of_slot, double* chi_o, double* chi_grid,
                        double* mom);

/* surface points of the obstacle blocks (normals [3][ns][512]) and the sums of
 * ComputeForces (FluidSolidForces.cpp:14-229); returns the points whose result
 * is not finite */
void orc_obstacle_surface(orc_mesh* m, int kind, const double* centre, const double* shape, const double* q,
                          int ns, const int32_t* block_of_slot, const double* chi_o, double* nrm);
int orc_compute_forces(orc_mesh* m, const double* vel, const double* pres, const double* chi_grid, int ns,
                       const int32_t* block_of_slot, const double* nrm, const double* udef, double nu,
                       const double* kin, double* qoi);

/* ---- learned preconditioner network (see oracle.cpp for the layout) ---- */
int orc_cnn_nparam(int C);
/* forward (out may be NULL), loss and gradient (target/grad may be NULL) */
void orc_cnn_fwd_grad(int nblk, int C, const double* params, const float* in, const float* target,
                      float* out, double* grad, double* loss);

#ifdef __cplusplus
}
#endif
