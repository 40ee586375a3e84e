// Time-step stencil operators on the device (advection-diffusion, penalization,
// pressure RHS, gradient update, max velocity).
#pragma once
#include "common.cuh"

namespace cup3d {

struct ObstacleView {
  int nslots;
  const int* slot;      // nb: obstacle slot of each block or -1 (nullptr: none)
  const int* near;      // nb: 1 if the block or a face neighbour holds obstacle cells
  const double* chi;    // nslots*512 obstacle chi
  const double* udef;   // 3*nslots*512
  const int* blk;       // nslots: block of each slot
  int udef_zero = 0;    // 1: every slot's udef is zero (rigid bodies)
};

// One RK3 stage (AdvectionDiffusion.cpp:286-320) fused with its update:
// tmp = tmpV_in + RHS(vel_in) + flux correction; vel_out = vel_in + alpha/h^3 tmp;
// tmpV_out = beta tmp.  stage 0 ignores tmpV_in; stage 2 skips tmpV_out.
int launch_advect_stage(const DevMesh& M, const double* vel_in, double* vel_out, double* tmpV,
                        double dt, double nu, const double* uinf, int scheme, int stage,
                        int grid, cudaStream_t s);

// lhs = KernelPressureRHS (+ flux correction) - [step > 2] KernelDivPressure(p_old);
// phi = 0 (initial guess).  PressureProjection.cpp:340-394.
int launch_pressure_rhs(const DevMesh& M, const double* vel, const double* pold, const double* chi,
                        const ObstacleView& ob, double dt, int step, int step_2nd_start, double* lhs,
                        double* phi, int grid, cudaStream_t s);

// p_new = phi - avg + [step > 2] p_old; vel += (KernelGradP(p_new) + flux corr)/h^3.
// avg = sums[0]/sums[1] from the weighted sum of phi.  PressureProjection.cpp:404-467.
int launch_grad_update(const DevMesh& M, double* vel, const double* phi, const double* pold,
                       double* pnew, const double* sums, double dt, int step, int step_2nd_start,
                       int grid, cudaStream_t s);

// KernelPenalization + kernelFinalizePenalizationForce (Penalization.cpp:18-109).
// kin = CM[3], vel[3], omega[3]; force[6] (F, T) reduced on the device.  In a
// batch (slot_force set) the sums go per obstacle slot into slot_force[6 s].
int launch_penalize(const DevMesh& M, double* vel, const double* chi, const ObstacleView& ob,
                    const double* kin_dev, double dt, double lambda, int implicit, double* force,
                    double* partial, unsigned* counter, cudaStream_t s, double* slot_force = nullptr);

// max |u + uinf| (findMaxU, ProcessHelpers.h:71-94) into *out.
int launch_max_u(const DevMesh& M, const double* vel, const double* uinf, double* out,
                 double* partial, unsigned* counter, int grid, cudaStream_t s);

// Batches: per-case max |u + uinf| (out[ncase]; bmax: nb scratch), per-case
// (sum phi h^3, sum h^3) (out[2 ncase]; bsum: 2 nb scratch) and per-case
// obstacle force/torque (out[6 ncase]) from per-slot sums.  first / slot_first:
// the cases' block / obstacle-slot ranges (ncase + 1 entries).
int launch_case_max_u(const DevMesh& M, const double* vel, const double* uinf, double* bmax, const int* first,
                      int ncase, double* out, int grid, cudaStream_t s);
int launch_case_sums(const DevMesh& M, const double* phi, double* bsum, const int* first, int ncase, double* out,
                     int grid, cudaStream_t s);
int launch_case_forces(const double* slot_force, const int* slot_first, int ncase, double* out, cudaStream_t s);

// dt = min(dtDiffusion, cfl_fac * dtAdvection) of Simulation::calcMaxTimestep
// from the device's max |u|, bit-identical to the host computation.
int launch_calc_dt(const double* umax, const double* cfl_fac, double nu, double hmin, double* dt, cudaStream_t s);
// The same for every case of a batch (hmin[ncase], umax[ncase] -> dt[ncase]).
int launch_case_calc_dt(const double* umax, const double* cfl_fac, double nu, const double* hmin, int ncase,
                        double* dt, cudaStream_t s);

}  // namespace cup3d
