// C++ host layer over the C ABI with the reference's operator interfaces:
//   class Operator { virtual void operator()(Real dt) = 0; virtual std::string getName() = 0; }
//     (operators/Operator.h:12-20)
//   class PoissonSolverBase { virtual void solve() = 0; } + makePoissonSolver(SimulationData&)
//     (poisson/PoissonSolverBase.h:10-19, PoissonSolverBase.cpp:30-52)
//   Simulation::calcMaxTimestep / advance (Simulation.cpp:309-412)
//
// Header-only; link against libcup3d_b200.so.  Hard errors of the C ABI become
// std::runtime_error (the reference throws or aborts); soft statuses (Poisson
// solve stopped at its caps) are recorded in SimulationData::last_solve.
#pragma once
#include <array>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "cup3d_b200.h"

namespace cubismup3d_b200 {

using Real = double;

inline void check(int rc, const cup_ctx* ctx) {
  if (rc < 0) throw std::runtime_error(std::string("cup3d_b200: ") + cup_last_error(ctx));
}

// The run state the operators share (the reference's SimulationData, reduced
// to what the time-step path reads).  Fields live on the device in `ctx`.
struct SimulationData {
  cup_config cfg{};
  cup_ctx* ctx = nullptr;
  int step = 0;
  Real time = 0, dt = 0, uMax_measured = 0;
  std::string poissonSolver = "b200";
  cup_solve_stats last_solve{};
  std::array<Real, 6> force_torque{};  // last Penalization force and torque
  bool has_obstacle = false;
  int freqDiagnostics = 0;             // ComputeDissipation every this many steps (0: never)
  bool adapt = true;                   // adaptMesh on the reference's cadence in Simulation::advance
  bool meshChanged = false;            // set when an adaptation changed the mesh
  std::array<Real, 20> diagnostics{};  // its last values (the columns of diagnostics.dat)
  bool computeForces = true;           // ComputeForces after the projection, as the reference does
  std::array<Real, 23> forces{};       // its last values (cup_compute_forces' order)

  explicit SimulationData(const std::string& flags) {
    cup_config_default(&cfg);
    check(cup_config_parse(&cfg, flags.c_str()), nullptr);
    static const char* names[] = {"b200",          "b200_mixed",   "b200_learned",   "b200_learned_mixed",
                                  "b200_twolevel", "b200_schwarz", "b200_pipelined", "b200_twolevel_mixed"};
    if (cfg.poisson_solver < 0 || cfg.poisson_solver >= int(sizeof(names) / sizeof(names[0])))
      throw std::runtime_error("cup3d_b200: Poisson solver id without a name");
    poissonSolver = names[cfg.poisson_solver];
    ctx = cup_create(&cfg);
    if (!ctx) throw std::runtime_error(std::string("cup3d_b200: ") + cup_last_error(nullptr));
  }
  ~SimulationData() { cup_destroy(ctx); }
  SimulationData(const SimulationData&) = delete;
  SimulationData& operator=(const SimulationData&) = delete;
};

class Operator {
 public:
  SimulationData& sim;
  explicit Operator(SimulationData& s) noexcept : sim(s) {}
  virtual ~Operator() = default;
  virtual void operator()(Real dt) = 0;
  virtual std::string getName() = 0;
};

class AdvectionDiffusion : public Operator {
 public:
  using Operator::Operator;
  void operator()(Real dt) override { check(cup_advect_diffuse(sim.ctx, dt), sim.ctx); }
  std::string getName() override { return "AdvectionDiffusion"; }
};

// CreateObstacles (ObstaclesCreate.cpp:303-323): a moving body's pose and chi.
class CreateObstacles : public Operator {
 public:
  using Operator::Operator;
  void operator()(Real dt) override {
    if (!sim.has_obstacle) return;
    check(cup_create_obstacles(sim.ctx, dt, sim.step), sim.ctx);
  }
  std::string getName() override { return "CreateObstacles"; }
};

// UpdateObstacles (ObstaclesUpdate.cpp:189-216): velocities of the free
// degrees of freedom from the fluid momentum; body_state = velocity, angular
// velocity, force, torque.
class UpdateObstacles : public Operator {
 public:
  using Operator::Operator;
  std::array<Real, 12> body_state{};
  void operator()(Real dt) override {
    if (!sim.has_obstacle) return;
    check(cup_update_obstacles(sim.ctx, dt, body_state.data()), sim.ctx);
  }
  std::string getName() override { return "UpdateObstacles"; }
};

class Penalization : public Operator {
 public:
  using Operator::Operator;
  void operator()(Real dt) override {
    if (!sim.has_obstacle) return;  // Penalization.cpp:513
    check(cup_penalize(sim.ctx, dt, sim.force_torque.data()), sim.ctx);
  }
  std::string getName() override { return "Penalization"; }
};

class PoissonSolverBase {
 public:
  virtual ~PoissonSolverBase() = default;
  virtual void solve() = 0;
};

// "b200", "b200_mixed", "b200_learned", "b200_learned_mixed", "b200_twolevel",
// "b200_twolevel_mixed", "b200_schwarz", "b200_pipelined": RHS in
// sim.lhs, initial guess and result in sim.pres (PoissonSolverAMR.cpp:20-21).
// The variant is the context's -poissonSolver setting.
class PoissonSolverB200 : public PoissonSolverBase {
  SimulationData& sim;

 public:
  explicit PoissonSolverB200(SimulationData& s) : sim(s) {}
  void solve() override { check(cup_poisson_solve(sim.ctx, &sim.last_solve), sim.ctx); }
};

// PoissonSolverBase.cpp:10-32: the solver named by -poissonSolver.  The
// reference's "iterative" / "cuda_iterative" select the plain FP64 solver.
inline std::shared_ptr<PoissonSolverBase> makePoissonSolver(SimulationData& s) {
  static const char* known[] = {"b200",           "b200_mixed",          "b200_learned", "b200_learned_mixed",
                                "b200_twolevel",  "b200_twolevel_mixed", "b200_schwarz", "b200_pipelined",
                                "iterative",      "cuda_iterative"};
  for (const char* k : known)
    if (s.poissonSolver == k) return std::make_shared<PoissonSolverB200>(s);
  throw std::invalid_argument("Poisson solver: \"" + s.poissonSolver + "\" unrecognized!");
}

// PressureProjection::operator() (PressureProjection.cpp:331-468): the RHS
// and p_old, then pressureSolver->solve() on sim.lhs / sim.pres (:402), then
// zero mean, p += p_old and the gradient update.
class PressureProjection : public Operator {
 public:
  std::shared_ptr<PoissonSolverBase> pressureSolver;
  explicit PressureProjection(SimulationData& s) : Operator(s), pressureSolver(makePoissonSolver(s)) {}
  void operator()(Real dt) override {
    check(cup_pressure_rhs(sim.ctx, dt, sim.step), sim.ctx);
    pressureSolver->solve();
    check(cup_pressure_finish(sim.ctx, dt, sim.step), sim.ctx);
  }
  std::string getName() override { return "PressureProjection"; }
};

// ComputeDissipation (ComputeDissipation.cpp:111-140): the 20 diagnostics
// every freqDiagnostics steps.
class ComputeDissipation : public Operator {
 public:
  using Operator::Operator;
  void operator()(Real) override {
    if (sim.freqDiagnostics == 0 || sim.step % sim.freqDiagnostics) return;
    check(cup_compute_dissipation(sim.ctx, sim.diagnostics.data()), sim.ctx);
  }
  std::string getName() override { return "ComputeDissipation"; }
};

// ComputeForces (FluidSolidForces.cpp:213-229): the body's surface forces
// after the projection (Simulation.cpp:214-215).
class ComputeForces : public Operator {
 public:
  using Operator::Operator;
  void operator()(Real) override {
    if (!sim.computeForces || !sim.has_obstacle) return;
    check(cup_compute_forces(sim.ctx, sim.forces.data()), sim.ctx);
  }
  std::string getName() override { return "ComputeForces"; }
};

// The time-step driver restricted to the hot path (Simulation.cpp:300-412),
// with the reference's operator order (Simulation.cpp:186-215); mesh
// adaptation stays with the caller.
class Simulation {
 public:
  SimulationData sim;
  std::vector<std::shared_ptr<Operator>> pipeline;

  explicit Simulation(const std::string& flags) : sim(flags) {
    pipeline.push_back(std::make_shared<CreateObstacles>(sim));
    pipeline.push_back(std::make_shared<AdvectionDiffusion>(sim));
    pipeline.push_back(std::make_shared<UpdateObstacles>(sim));
    pipeline.push_back(std::make_shared<Penalization>(sim));
    pipeline.push_back(std::make_shared<PressureProjection>(sim));
    pipeline.push_back(std::make_shared<ComputeForces>(sim));
    pipeline.push_back(std::make_shared<ComputeDissipation>(sim));
  }
  Real calcMaxTimestep() {
    Real dt = 0;
    check(cup_compute_dt(sim.ctx, sim.step, &dt), sim.ctx);
    sim.dt = dt;
    return dt;
  }
  // Simulation::adaptMesh (Simulation.cpp:128-149): the mesh adapts to the
  // vorticity and the body (cup_adapt_mesh); the body's chi is created again
  // on the new mesh.
  void adaptMesh() {
    int32_t changed = 0;
    check(cup_adapt_mesh(sim.ctx, &changed), sim.ctx);
    sim.meshChanged = sim.meshChanged || changed != 0;
  }
  // The mesh adapts before the pipeline every 20 steps and in the first 10
  // (Simulation.cpp:384-385); adapt = false keeps it as it is.
  void advance(Real dt) {
    if (sim.adapt && (sim.step % 20 == 0 || sim.step < 10)) adaptMesh();
    for (auto& op : pipeline) (*op)(dt);
    sim.step++;
    sim.time += dt;
  }
};

}  // namespace cubismup3d_b200
