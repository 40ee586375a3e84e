// Drives the hot path through the C++ operator layer the way the reference's
// Simulation::advance does: calcMaxTimestep, then each Operator in order.
// Configuration: the Taylor-Green vortex of the uniform periodic case.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "cup3d_b200_operators.hpp"

using namespace cubismup3d_b200;

int main() {
  Simulation S("-bpdx 4 -bpdy 4 -bpdz 4 -levelMax 1 -extent 6.283185307179586 -BC_x periodic "
               "-BC_y periodic -BC_z periodic -nu 0.01 -CFL 0.3 -rampup 0 -poissonTolRel 1e-8 -poissonTol 0");
  check(cup_set_mesh_uniform(S.sim.ctx), S.sim.ctx);
  const int nb = cup_num_blocks(S.sim.ctx);
  std::vector<int> level(nb), index(3 * nb);
  std::vector<double> h(nb);
  check(cup_get_blocks(S.sim.ctx, level.data(), index.data(), h.data()), S.sim.ctx);
  const size_t n = size_t(nb) * 512;
  std::vector<double> vel(3 * n, 0.0);
  for (int b = 0; b < nb; ++b)
    for (int c = 0; c < 512; ++c) {
      const double x = (index[3 * b] * 8 + c % 8 + 0.5) * h[b];
      const double y = (index[3 * b + 1] * 8 + (c / 8) % 8 + 0.5) * h[b];
      const double z = (index[3 * b + 2] * 8 + c / 64 + 0.5) * h[b];
      vel[b * 512 + c] = std::sin(x) * std::cos(y) * std::cos(z);
      vel[n + b * 512 + c] = -std::cos(x) * std::sin(y) * std::cos(z);
    }
  check(cup_upload_field(S.sim.ctx, CUP_FIELD_VEL, vel.data()), S.sim.ctx);
  S.sim.freqDiagnostics = 1;
  for (int s = 0; s < 3; ++s) {
    const Real dt = S.calcMaxTimestep();
    S.advance(dt);
    std::printf("step %d dt %.6e poisson iterations %d status %d\n", S.sim.step, dt, S.sim.last_solve.iterations,
                S.sim.last_solve.status);
    if (S.sim.last_solve.status != 1) return 2;
    // the decaying vortex: kinetic energy (the 19th diagnostic) below pi^3
    std::printf("  kinetic energy %.9f\n", S.sim.diagnostics[18]);
    if (!(S.sim.diagnostics[18] > 0.9 * 31.00627668 && S.sim.diagnostics[18] < 31.00627668)) return 7;
  }
  double umax = 0;
  check(cup_max_u(S.sim.ctx, &umax), S.sim.ctx);
  std::printf("umax %.12f\n", umax);
  // the decaying vortex keeps |u| <= 1 and loses energy slowly
  if (!(umax > 0.9 && umax <= 1.0)) return 3;

  // makePoissonSolver for every solver name: a Simulation is built with each
  // and steps, its projection calling pressureSolver->solve() in the middle
  for (const char* name : {"b200", "b200_mixed", "b200_learned", "b200_learned_mixed", "b200_twolevel",
                           "b200_twolevel_mixed", "iterative"}) {
    Simulation T(std::string("-bpdx 4 -bpdy 4 -bpdz 4 -levelMax 1 -extent 6.283185307179586 -BC_x periodic "
                             "-BC_y periodic -BC_z periodic -nu 0.01 -CFL 0.3 -rampup 0 -poissonTolRel 1e-8 "
                             "-poissonTol 0 -poissonSolver ") + name);
    if (T.sim.poissonSolver != (std::string(name) == "iterative" ? "b200" : name)) {
      std::printf("solver %s: named %s\n", name, T.sim.poissonSolver.c_str());
      return 10;
    }
    check(cup_set_mesh_uniform(T.sim.ctx), T.sim.ctx);
    check(cup_upload_field(T.sim.ctx, CUP_FIELD_VEL, vel.data()), T.sim.ctx);
    if (T.sim.poissonSolver.find("learned") != std::string::npos) check(cup_cnn_init(T.sim.ctx, 5), T.sim.ctx);
    for (int s = 0; s < 2; ++s) {
      const Real dt = T.calcMaxTimestep();
      T.advance(dt);
      if (T.sim.last_solve.status != 1) {
        std::printf("solver %s: step %d status %d\n", name, s, T.sim.last_solve.status);
        return 8;
      }
    }
    double um = 0;
    check(cup_max_u(T.sim.ctx, &um), T.sim.ctx);
    std::printf("solver %s: 2 steps, umax %.12f\n", name, um);
    if (!(std::fabs(um - umax) < 0.02)) return 9;
  }

  // A moving sphere: the pipeline of this layer (CreateObstacles, ...,
  // UpdateObstacles, Penalization, ...) against cup_step on a second context,
  // bit for bit.
  const char* flags =
      "-bpdx 4 -bpdy 4 -bpdz 4 -levelMax 1 -extent 6.283185307179586 -BC_x periodic -BC_y periodic "
      "-BC_z periodic -nu 0.01 -CFL 0.3 -rampup 0 -poissonTolRel 1e-8 -poissonTol 0 -lambda 1e6";
  Simulation A(flags), B(flags);
  const double ctr[3] = {3.0, 3.1, 2.9}, bvel[3] = {0.5, 0.0, 0.1}, bom[3] = {0.0, 0.0, 0.0};
  for (Simulation* X : {&A, &B}) {
    check(cup_set_mesh_uniform(X->sim.ctx), X->sim.ctx);
    check(cup_upload_field(X->sim.ctx, CUP_FIELD_VEL, vel.data()), X->sim.ctx);
    check(cup_obstacle_sphere(X->sim.ctx, ctr, 0.8, bvel, bom), X->sim.ctx);
    X->sim.has_obstacle = true;
  }
  std::vector<double> va(3 * n), vb(3 * n), ca(n), c0(n);
  check(cup_download_field(A.sim.ctx, CUP_FIELD_CHI, c0.data()), A.sim.ctx);
  for (int s = 0; s < 3; ++s) {
    const Real dt = A.calcMaxTimestep();
    A.advance(dt);
    double dtb = 0;
    cup_solve_stats st{};
    if (cup_step(B.sim.ctx, s, 0.0, &dtb, &st) < 0) return 4;
    check(cup_download_field(A.sim.ctx, CUP_FIELD_VEL, va.data()), A.sim.ctx);
    check(cup_download_field(B.sim.ctx, CUP_FIELD_VEL, vb.data()), B.sim.ctx);
    if (dtb != dt || va != vb) {
      std::printf("moving sphere: step %d differs (dt %.17g vs %.17g)\n", s, dt, dtb);
      return 5;
    }
  }
  check(cup_download_field(A.sim.ctx, CUP_FIELD_CHI, ca.data()), A.sim.ctx);
  double moved = 0;
  for (size_t i = 0; i < n; ++i) moved = std::max(moved, std::fabs(ca[i] - c0[i]));
  std::printf("moving sphere: 3 steps equal to cup_step, chi changed by %.3f\n", moved);
  // ComputeForces ran after each projection (the pipeline's own operator)
  std::printf("moving sphere: surface force %.6e %.6e %.6e, drag %.6e\n", A.sim.forces[0], A.sim.forces[1],
              A.sim.forces[2], A.sim.forces[12]);
  for (Real f : A.sim.forces)
    if (!std::isfinite(f)) return 7;
  if (A.sim.forces[0] == 0.0) return 8;
  return moved > 0.01 ? 0 : 6;
}
