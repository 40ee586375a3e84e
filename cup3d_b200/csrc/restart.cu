// Restart files (Simulation::serialize / deserialize, Simulation.cpp:225-298;
// SimulationData::writeRestartFiles / readRestartFiles, SimulationData.cpp:200-297;
// Obstacle::saveRestart / loadRestart, Obstacle.cpp:443-504).
//
// A restart directory holds:
//   field.restart       the reference's text file, key for key: time, stepid,
//                       uinf, dt (%20.20e, exact round trip);
//   shape_0.restart     the reference's body file, key for key (pose, lab
//                       position, quaternion, velocities, previous pose), then
//                       the shape: kind, radius or axes, free degrees of
//                       freedom, creation path;
//   restart_<step>.cupf the fields the reference dumps to HDF5 (vel_restart_*,
//                       pres_restart_*), which this build keeps in its own
//                       binary: magic, block count, the leaves (level, index)
//                       in device order, velocity (3 nb 512) and pressure
//                       (nb 512) in FP64, the BDF2 coefficients of the bodies.
// Reading one rebuilds the mesh from the leaves, uploads the fields, restores
// the body and re-creates its chi (the reference runs pipeline[0],
// CreateObstacles), so that the run continues bit for bit.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "context.h"

namespace cup3d {
namespace {

constexpr char kMagic[8] = {'C', 'U', 'P', '3', 'D', 'R', 'S', '1'};

std::string field_path(const std::string& dir, int step) {
  char name[64];
  std::snprintf(name, sizeof(name), "/restart_%09d.cupf", step);
  return dir + name;
}

struct File {
  FILE* f;
  explicit File(const std::string& p, const char* mode) : f(std::fopen(p.c_str(), mode)) {}
  ~File() {
    if (f) std::fclose(f);
  }
};

int write_text(cup_ctx* c, const std::string& dir, int step, double time) {
  File ff(dir + "/field.restart", "w");
  if (!ff.f) return set_error(CUP_ERR_ARG, ("cannot write " + dir + "/field.restart").c_str());
  std::fprintf(ff.f, "time: %20.20e\n", time);
  std::fprintf(ff.f, "stepid: %d\n", step);
  std::fprintf(ff.f, "uinfx: %20.20e\n", c->cfg.uinf[0]);
  std::fprintf(ff.f, "uinfy: %20.20e\n", c->cfg.uinf[1]);
  std::fprintf(ff.f, "uinfz: %20.20e\n", c->cfg.uinf[2]);
  std::fprintf(ff.f, "dt: %20.20e\n", c->dt_prev);
  const BodyState& B = c->body;
  if (B.kind < 0) return 0;
  File fs(dir + "/shape_0.restart", "w");
  if (!fs.f) return set_error(CUP_ERR_ARG, ("cannot write " + dir + "/shape_0.restart").c_str());
  FILE* f = fs.f;
  std::fprintf(f, "x:       %20.20e\n", B.pos[0]);
  std::fprintf(f, "y:       %20.20e\n", B.pos[1]);
  std::fprintf(f, "z:       %20.20e\n", B.pos[2]);
  std::fprintf(f, "xAbs:    %20.20e\n", B.abs_pos[0]);
  std::fprintf(f, "yAbs:    %20.20e\n", B.abs_pos[1]);
  std::fprintf(f, "zAbs:    %20.20e\n", B.abs_pos[2]);
  for (int i = 0; i < 4; ++i) std::fprintf(f, "quat_%d:  %20.20e\n", i, B.quat[i]);
  std::fprintf(f, "u_x:     %20.20e\n", B.vel[0]);
  std::fprintf(f, "u_y:     %20.20e\n", B.vel[1]);
  std::fprintf(f, "u_z:     %20.20e\n", B.vel[2]);
  std::fprintf(f, "omega_x: %20.20e\n", B.omega[0]);
  std::fprintf(f, "omega_y: %20.20e\n", B.omega[1]);
  std::fprintf(f, "omega_z: %20.20e\n", B.omega[2]);
  for (int d = 0; d < 3; ++d) std::fprintf(f, "old_position_%d:    %20.20e\n", d, B.old_pos[d]);
  for (int d = 0; d < 3; ++d) std::fprintf(f, "old_absPos_%d:      %20.20e\n", d, B.old_abs_pos[d]);
  for (int i = 0; i < 4; ++i) std::fprintf(f, "old_quaternion_%d:  %20.20e\n", i, B.old_quat[i]);
  // the shape (no counterpart in the reference's file, which keeps it in the
  // run's settings)
  std::fprintf(f, "kind: %d\n", B.kind);
  std::fprintf(f, "radius: %20.20e\n", B.r);
  for (int d = 0; d < 3; ++d) std::fprintf(f, "axis_%d: %20.20e\n", d, B.ax[d]);
  for (int d = 0; d < 3; ++d) std::fprintf(f, "free_trans_%d: %d\n", d, B.free_t[d]);
  for (int d = 0; d < 3; ++d) std::fprintf(f, "free_rot_%d: %d\n", d, B.free_r[d]);
  std::fprintf(f, "on_device: %d\n", B.on_device ? 1 : 0);
  for (int d = 0; d < 3; ++d) std::fprintf(f, "fix_frame_%d: %d\n", d, B.fix_frame[d]);
  return 0;
}

bool scan(FILE* f, const char* fmt, double* v) { return std::fscanf(f, fmt, v) == 1; }
bool scan_i(FILE* f, const char* fmt, int* v) { return std::fscanf(f, fmt, v) == 1; }

int read_body(const std::string& dir, BodyState& B) {
  File fs(dir + "/shape_0.restart", "r");
  if (!fs.f) return 1;  // no body
  FILE* f = fs.f;
  bool ok = true;
  const char* pk[3] = {"x:       %le\n", "y:       %le\n", "z:       %le\n"};
  const char* ak[3] = {"xAbs:    %le\n", "yAbs:    %le\n", "zAbs:    %le\n"};
  const char* uk[3] = {"u_x:     %le\n", "u_y:     %le\n", "u_z:     %le\n"};
  const char* ok3[3] = {"omega_x: %le\n", "omega_y: %le\n", "omega_z: %le\n"};
  char key[64];
  for (int d = 0; d < 3; ++d) ok = ok && scan(f, pk[d], &B.pos[d]);
  for (int d = 0; d < 3; ++d) ok = ok && scan(f, ak[d], &B.abs_pos[d]);
  for (int i = 0; i < 4; ++i) {
    std::snprintf(key, sizeof(key), "quat_%d:  %%le\n", i);
    ok = ok && scan(f, key, &B.quat[i]);
  }
  for (int d = 0; d < 3; ++d) ok = ok && scan(f, uk[d], &B.vel[d]);
  for (int d = 0; d < 3; ++d) ok = ok && scan(f, ok3[d], &B.omega[d]);
  for (int d = 0; d < 3; ++d) {
    std::snprintf(key, sizeof(key), "old_position_%d:    %%le\n", d);
    ok = ok && scan(f, key, &B.old_pos[d]);
  }
  for (int d = 0; d < 3; ++d) {
    std::snprintf(key, sizeof(key), "old_absPos_%d:      %%le\n", d);
    ok = ok && scan(f, key, &B.old_abs_pos[d]);
  }
  for (int i = 0; i < 4; ++i) {
    std::snprintf(key, sizeof(key), "old_quaternion_%d:  %%le\n", i);
    ok = ok && scan(f, key, &B.old_quat[i]);
  }
  int on_dev = 0;
  ok = ok && scan_i(f, "kind: %d\n", &B.kind);
  ok = ok && scan(f, "radius: %le\n", &B.r);
  for (int d = 0; d < 3; ++d) {
    std::snprintf(key, sizeof(key), "axis_%d: %%le\n", d);
    ok = ok && scan(f, key, &B.ax[d]);
  }
  for (int d = 0; d < 3; ++d) {
    std::snprintf(key, sizeof(key), "free_trans_%d: %%d\n", d);
    ok = ok && scan_i(f, key, &B.free_t[d]);
  }
  for (int d = 0; d < 3; ++d) {
    std::snprintf(key, sizeof(key), "free_rot_%d: %%d\n", d);
    ok = ok && scan_i(f, key, &B.free_r[d]);
  }
  ok = ok && scan_i(f, "on_device: %d\n", &on_dev);
  // fix_frame_* came later: a file without them (written before the frame of
  // reference could follow a body) restores a body that fixes no axis
  for (int d = 0; d < 3; ++d) {
    std::snprintf(key, sizeof(key), "fix_frame_%d: %%d\n", d);
    B.fix_frame[d] = 0;
    if (ok && !scan_i(f, key, &B.fix_frame[d])) {
      B.fix_frame[d] = 0;
      break;  // end of file: the remaining axes stay 0
    }
  }
  B.on_device = on_dev != 0;
  if (!ok || (B.kind != 0 && B.kind != 1)) return set_error(CUP_ERR_ARG, ("malformed " + dir + "/shape_0.restart").c_str());
  return 0;
}

}  // namespace
}  // namespace cup3d

using namespace cup3d;

extern "C" {

int cup_write_restart(cup_ctx* c, const char* dir, int32_t step, double time) {
  if (!c || !dir || c->mesh.nb == 0 || c->host_only || c->ncase > 1)
    return ctx_fail(c, CUP_ERR_ARG, "cup_write_restart: bad arguments");
  const std::string d(dir);
  if (int rc = write_text(c, d, step, time)) return ctx_fail(c, rc, "cup_write_restart failed");
  const Mesh& m = c->mesh;
  const size_t n = size_t(m.nb) * BN;
  std::vector<double> vel(3 * n), pres(n);
  CUP_CUDA_TRY(stream_d2h(c->stream, vel.data(), c->F.vel[c->F.vcur], vel.size() * sizeof(double)));
  CUP_CUDA_TRY(stream_d2h(c->stream, pres.data(), c->F.pres[c->F.pcur], pres.size() * sizeof(double)));
  File fb(field_path(d, step), "wb");
  if (!fb.f) return ctx_fail(c, CUP_ERR_ARG, "cannot write " + field_path(d, step));
  const int32_t nb = m.nb;
  bool ok = std::fwrite(kMagic, 1, 8, fb.f) == 8 && std::fwrite(&nb, 4, 1, fb.f) == 1 &&
            std::fwrite(m.level.data(), 4, nb, fb.f) == size_t(nb) &&
            std::fwrite(m.index.data(), 4, 3 * size_t(nb), fb.f) == 3 * size_t(nb) &&
            std::fwrite(vel.data(), 8, vel.size(), fb.f) == vel.size() &&
            std::fwrite(pres.data(), 8, pres.size(), fb.f) == pres.size() &&
            std::fwrite(c->coef_u, 8, 3, fb.f) == 3;
  if (!ok) return ctx_fail(c, CUP_ERR_ARG, "short write to " + field_path(d, step));
  return 0;
}

int cup_read_restart(cup_ctx* c, const char* dir, int32_t step, double* time) {
  if (!c || !dir || c->host_only || c->ncase > 1) return ctx_fail(c, CUP_ERR_ARG, "cup_read_restart: bad arguments");
  const std::string d(dir);
  double t = 0, uinf[3] = {0, 0, 0}, dt = 0;
  int stepid = -1;
  {
    File ff(d + "/field.restart", "r");
    if (!ff.f) return ctx_fail(c, CUP_ERR_ARG, "cannot read " + d + "/field.restart");
    bool ok = scan(ff.f, "time: %le\n", &t) && scan_i(ff.f, "stepid: %d\n", &stepid) &&
              scan(ff.f, "uinfx: %le\n", &uinf[0]) && scan(ff.f, "uinfy: %le\n", &uinf[1]) &&
              scan(ff.f, "uinfz: %le\n", &uinf[2]) && scan(ff.f, "dt: %le\n", &dt);
    if (!ok || stepid < 0 || t < 0) return ctx_fail(c, CUP_ERR_ARG, "error reading " + d + "/field.restart");
    if (stepid != step) return ctx_fail(c, CUP_ERR_ARG, "field.restart holds another step");
  }
  File fb(field_path(d, step), "rb");
  if (!fb.f) return ctx_fail(c, CUP_ERR_ARG, "cannot read " + field_path(d, step));
  char magic[8];
  int32_t nb = 0;
  if (std::fread(magic, 1, 8, fb.f) != 8 || std::memcmp(magic, kMagic, 8) != 0 || std::fread(&nb, 4, 1, fb.f) != 1 ||
      nb <= 0)
    return ctx_fail(c, CUP_ERR_ARG, "not a restart field file: " + field_path(d, step));
  std::vector<int32_t> level(nb), index(3 * size_t(nb));
  const size_t n = size_t(nb) * BN;
  std::vector<double> vel(3 * n), pres(n);
  double coef[3];
  const bool ok = std::fread(level.data(), 4, nb, fb.f) == size_t(nb) &&
                  std::fread(index.data(), 4, index.size(), fb.f) == index.size() &&
                  std::fread(vel.data(), 8, vel.size(), fb.f) == vel.size() &&
                  std::fread(pres.data(), 8, pres.size(), fb.f) == pres.size() &&
                  std::fread(coef, 8, 3, fb.f) == 3;
  if (!ok) return ctx_fail(c, CUP_ERR_ARG, "truncated " + field_path(d, step));
  if (int rc = cup_set_mesh(c, nb, level.data(), index.data())) return rc;
  if (c->mesh.level != level || c->mesh.index != index)
    return ctx_fail(c, CUP_ERR_ARG, "restart leaves are not in this build's block order");
  CUP_CUDA_TRY(stream_h2d(c->stream, c->F.vel[c->F.vcur], vel.data(), vel.size() * sizeof(double)));
  CUP_CUDA_TRY(stream_h2d(c->stream, c->F.pres[c->F.pcur], pres.data(), pres.size() * sizeof(double)));
  for (int k = 0; k < 3; ++k) {
    c->cfg.uinf[k] = uinf[k];
    c->coef_u[k] = coef[k];
  }
  c->dt_prev = dt;
  // the body: re-created at its pose (CreateObstacles), then its history restored
  BodyState B;
  const int rb = read_body(d, B);
  if (rb < 0 || rb > 1) return ctx_fail(c, rb, "cup_read_restart: body");
  if (rb == 0) {
    int rc;
    if (B.kind == 0)
      rc = B.on_device ? cup_obstacle_sphere_dev(c, B.pos, B.r, B.vel, B.omega)
                       : cup_obstacle_sphere(c, B.pos, B.r, B.vel, B.omega);
    else
      rc = B.on_device ? cup_obstacle_ellipsoid_dev(c, B.pos, B.ax, B.quat, B.vel, B.omega)
                       : cup_obstacle_ellipsoid(c, B.pos, B.ax, B.quat, B.vel, B.omega);
    if (rc) return rc;
    c->body = B;
  }
  graph_reset(c);
  if (time) *time = t;
  return 0;
}

}  // extern "C"
