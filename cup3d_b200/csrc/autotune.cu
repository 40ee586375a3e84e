// Launch-shape tuning on a context's own mesh and fields (no reference
// counterpart): the grid of each stencil kernel and the CTA count of the
// persistent solver (block groups per CTA are fixed, so this sets the
// blocks each group takes per phase) are chosen by timing candidates.
#include <algorithm>
#include <functional>
#include <random>

#include "context.h"
#include "stencils.cuh"

namespace cup3d {

static int keep_last(cup_ctx* c, int rc) {
  c->err = cup_last_error(nullptr);
  return rc;
}

// Mean device time of `reps` launches after one untimed launch.
static int time_launch(cup_ctx* c, const std::function<int()>& launch, int reps, float* ms) {
  if (int rc = launch()) return rc;
  CUP_CUDA_TRY(cudaEventRecord(c->ev0, c->stream));
  for (int i = 0; i < reps; ++i)
    if (int rc = launch()) return rc;
  CUP_CUDA_TRY(cudaEventRecord(c->ev1, c->stream));
  CUP_CUDA_TRY(cudaEventSynchronize(c->ev1));
  CUP_CUDA_TRY(cudaEventElapsedTime(ms, c->ev0, c->ev1));
  *ms /= reps;
  return 0;
}

// Sets the persistent solver's CTA count and deals the visit order for its
// block groups.
static int set_solver_grid(cup_ctx* c, int grid) {
  c->W.pgrid = grid;
  const std::vector<int32_t> order = mesh_visit_order(c->mesh, grid * PERSISTENT_GROUPS_PER_CTA);
  CUP_CUDA_TRY(stream_h2d(c->stream, const_cast<int*>(c->dm.order), order.data(), order.size() * sizeof(int32_t)));
  return 0;
}

}  // namespace cup3d

using namespace cup3d;

extern "C" {

int cup_autotune(cup_ctx* c, int32_t* choice, float* best_ms) {
  ProfBind pb_(c);
  if (!c || c->host_only || c->mesh.nb == 0 || !choice) return ctx_fail(c, CUP_ERR_ARG, "cup_autotune: bad arguments");
  Fields& F = c->F;
  const int nb = c->mesh.nb, sms = c->num_sms;
  graph_reset(c);
  // stencil grids: multiples of the SM count, at most one CTA per block
  std::vector<int> cand;
  for (int k : {1, 2, 3, 4, 6, 8}) cand.push_back(std::min(nb, k * sms));
  std::sort(cand.begin(), cand.end());
  cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
  const double dt = 1e-4;
  const double* vel = F.vel[F.vcur];
  double* scratch = F.vel[1 - F.vcur];
  const ObstacleView ob{c->ob.nslots, c->ob.slot_of_block, c->ob.near, c->ob.chi, c->ob.udef, c->ob.block_of_slot,
                       c->ob.udef_zero ? 1 : 0};
  std::function<int(int)> kernels[3] = {
      // one RK3 stage: writes the other velocity buffer and tmpV
      [&](int g) { return launch_advect_stage(c->dm, vel, scratch, F.tmpV, dt, c->cfg.nu, c->cfg.uinf,
                                              c->cfg.advection, 0, g, c->stream); },
      // the pressure RHS: writes lhs and phi
      [&](int g) { return launch_pressure_rhs(c->dm, vel, F.pres[F.pcur], F.chi, ob, dt, 0, c->cfg.step_2nd_start,
                                              F.lhs, F.phi, g, c->stream); },
      // the gradient update on a copy of the velocity (and the other pressure buffer)
      [&](int g) { return launch_grad_update(c->dm, scratch, F.phi, F.pres[F.pcur], F.pres[1 - F.pcur],
                                             c->d_scalars + SC_SUMS, dt, 0, c->cfg.step_2nd_start, g, c->stream); },
  };
  CUP_CUDA_TRY(cudaMemcpyAsync(scratch, vel, 3 * nbn(c) * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  if (int rc = launch_pressure_rhs(c->dm, vel, F.pres[F.pcur], F.chi, ob, dt, 0, c->cfg.step_2nd_start, F.lhs, F.phi,
                                   c->W.grid, c->stream))
    return keep_last(c, rc);
  if (int rc = launch_weighted_sum(c->dm, F.phi, c->d_scalars + SC_SUMS, c->W, c->stream)) return keep_last(c, rc);
  for (int k = 0; k < 3; ++k) {
    float best = 0;
    int arg = cand[0];
    for (int g : cand) {
      float ms = 0;
      if (int rc = time_launch(c, [&]() { return kernels[k](g); }, 3, &ms)) return keep_last(c, rc);
      if (g == cand[0] || ms < best) {
        best = ms;
        arg = g;
      }
    }
    c->tgrid[k] = arg;
    choice[k] = arg;
    if (best_ms) best_ms[k] = best;
  }
  // persistent solver CTAs: one or two per SM (up to the co-resident maximum),
  // timed over 16 iterations of a seeded problem (lhs and phi as scratch)
  choice[3] = c->W.pgrid;
  if (best_ms) best_ms[3] = 0.0f;
  if (c->ncase == 1) {
    int gmax = 0;
    if (int rc = persistent_grid_max(nb, c->W, &gmax)) return keep_last(c, rc);
    std::vector<int> sg;
    for (int g : {sms, (3 * sms) / 2, 2 * sms}) sg.push_back(std::max(1, std::min(gmax, g)));
    sg.push_back(gmax);
    std::sort(sg.begin(), sg.end());
    sg.erase(std::unique(sg.begin(), sg.end()), sg.end());
    std::vector<double> b(nbn(c));
    std::mt19937_64 rng(1234);
    std::normal_distribution<double> nd;
    for (double& v : b) v = nd(rng);
    CUP_CUDA_TRY(stream_h2d(c->stream, F.lhs, b.data(), b.size() * sizeof(double)));
    SolveParams P{};
    P.tol_abs = 0.0;
    P.tol_rel = 0.0;
    P.max_iter = 16;
    P.max_restarts = c->cfg.poisson_max_restarts;
    P.mean_mode = c->cfg.mean_constraint;
    P.check_every = 8;
    P.persistent = 1;
    P.block_cache = c->cfg.poisson_block_cache;
    float best = 0;
    int arg = sg.back();
    for (int g : sg) {
      if (int rc = set_solver_grid(c, g)) return keep_last(c, rc);
      float ms = 0;
      SolveStats S{};
      auto solve = [&]() {
        if (cudaMemsetAsync(F.phi, 0, nbn(c) * sizeof(double), c->stream) != cudaSuccess)
          return set_error(CUP_ERR_CUDA, "cup_autotune: memset");
        return poisson_bicgstab(c->dm, F.lhs, F.phi, P, c->W, S, c->stream, c->h_pinned, nullptr);
      };
      if (int rc = time_launch(c, solve, 2, &ms)) return keep_last(c, rc);
      const float per_it = ms / std::max(1, S.iterations);
      if (g == sg.front() || per_it < best) {
        best = per_it;
        arg = g;
      }
    }
    if (int rc = set_solver_grid(c, arg)) return keep_last(c, rc);
    choice[3] = arg;
    if (best_ms) best_ms[3] = best;
  }
  CUP_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return 0;
}

}  // extern "C"
