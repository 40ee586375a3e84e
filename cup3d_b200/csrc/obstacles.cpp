// Host-side obstacle creation: see obstacles.h.
#include "obstacles.h"

#include "ellipsoid_distance.cuh"

#include <algorithm>
#include <cmath>
#include <functional>
#include <limits>

namespace cup3d {

namespace {

constexpr double kEps = std::numeric_limits<double>::epsilon();

// Fills obstacle blocks from a signed distance (positive inside) on the
// blocks whose cell-centre range meets `box` (Obstacle::create_base,
// Obstacle.h:139-160).  chi per ObstaclesCreate.cpp:45-80 (Towers, "Finite
// difference methods for approximating Heaviside functions", eq. 14).
void fill_from_sdf(const Mesh& m, const std::function<double(double, double, double)>& sdf,
                   const double box[3][2], const double vel[3], const double omega[3], HostObstacle& out) {
  out = HostObstacle();
  out.grid_chi.assign(size_t(m.nb) * 512, 0.0);
  double mom[4] = {0, 0, 0, 0};
  for (int b = 0; b < m.nb; ++b) {
  const double h = m.h[b];
    double lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
      lo[d] = m.origin[3 * b + d] + 0.5 * h;          // info.pos(.., 0, 0, 0)
      hi[d] = m.origin[3 * b + d] + (8 - 0.5) * h;    // info.pos(.., 7, 7, 7)
    }
    bool touch = true;
    for (int d = 0; d < 3; ++d) {
      const double a = std::max(lo[d], box[d][0]), c = std::min(hi[d], box[d][1]);
      touch &= c - a > 0;
    }
    if (!touch) continue;
    // signed distance on the block and a one-cell halo (sdfLab)
    double lab[10][10][10];
    for (int z = -1; z <= 8; ++z)
      for (int y = -1; y <= 8; ++y)
        for (int x = -1; x <= 8; ++x)
          lab[z + 1][y + 1][x + 1] = sdf(m.origin[3 * b] + (x + 0.5) * h, m.origin[3 * b + 1] + (y + 0.5) * h,
                                         m.origin[3 * b + 2] + (z + 0.5) * h);
    const int slot = int(out.blocks.size());
    out.blocks.push_back(b);
    out.chi.resize(size_t(slot + 1) * 512, 0.0);
    const double inv2h = 0.5 / h, vol = h * h * h;
    for (int z = 0; z < 8; ++z)
      for (int y = 0; y < 8; ++y)
        for (int x = 0; x < 8; ++x) {
          const double s0 = lab[z + 1][y + 1][x + 1];
          double chi;
          if (s0 > h || s0 < -h) {
            chi = s0 > 0 ? 1 : 0;
          } else {
            const double dPx = lab[z + 1][y + 1][x + 2], dMx = lab[z + 1][y + 1][x];
            const double dPy = lab[z + 1][y + 2][x + 1], dMy = lab[z + 1][y][x + 1];
            const double dPz = lab[z + 2][y + 1][x + 1], dMz = lab[z][y + 1][x + 1];
            const double gUX = inv2h * (dPx - dMx), gUY = inv2h * (dPy - dMy), gUZ = inv2h * (dPz - dMz);
            const double gUSq = gUX * gUX + gUY * gUY + gUZ * gUZ + kEps;
            const double gIX = inv2h * (std::max(0.0, dPx) - std::max(0.0, dMx));
            const double gIY = inv2h * (std::max(0.0, dPy) - std::max(0.0, dMy));
            const double gIZ = inv2h * (std::max(0.0, dPz) - std::max(0.0, dMz));
            chi = (gIX * gUX + gIY * gUY + gIZ * gUZ) / gUSq;
          }
          const int cell = x + 8 * y + 64 * z;
          out.chi[size_t(slot) * 512 + cell] = chi;
          double& g = out.grid_chi[size_t(b) * 512 + cell];
          g = std::max(g, chi);
          const double px = m.origin[3 * b] + (x + 0.5) * h, py = m.origin[3 * b + 1] + (y + 0.5) * h,
                       pz = m.origin[3 * b + 2] + (z + 0.5) * h;
          mom[0] += chi * vol * px;
          mom[1] += chi * vol * py;
          mom[2] += chi * vol * pz;
          mom[3] += chi * vol;
        }
  }
  out.udef.assign(3 * out.chi.size(), 0.0);
  out.mass = mom[3];
  for (int d = 0; d < 3; ++d) {
    out.kin[d] = mom[3] > 0 ? mom[d] / mom[3] : 0.0;
    out.kin[3 + d] = vel[d];
    out.kin[6 + d] = omega[d];
  }
}

}  // namespace

void sphere_fill_box(const double c[3], double r, double hmin, double box[3][2]) {
  const double safety = (2 + 1) * hmin;
  for (int d = 0; d < 3; ++d) {
    box[d][0] = c[d] - (r + safety);
    box[d][1] = c[d] + (r + safety);
  }
}

void ellipsoid_fill_box(const double c[3], const double ax[3], double hmin, double box[3][2]) {
  const double safety = (2 + 1) * hmin;
  const double amax = std::max({ax[0], ax[1], ax[2]});
  for (int d = 0; d < 3; ++d) {
    box[d][0] = c[d] - 2 * (amax + safety);
    box[d][1] = c[d] + 2 * (amax + safety);
  }
}

void make_sphere(const Mesh& m, const double c[3], double r, const double vel[3], const double omega[3],
                 HostObstacle& out) {
  double box[3][2];
  sphere_fill_box(c, r, m.spec.hmin, box);
  auto sdf = [&](double x, double y, double z) {
    const double dx = x - c[0], dy = y - c[1], dz = z - c[2];
    return r - std::sqrt(dx * dx + dy * dy + dz * dz);
  };
  fill_from_sdf(m, sdf, box, vel, omega, out);
}

void quat_rotation(const double q[4], double R[3][3]) {
  const double w = q[0], x = q[1], y = q[2], z = q[3];
  const double M[3][3] = {{1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)},
                          {2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)},
                          {2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)}};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) R[i][j] = M[i][j];
}

void make_ellipsoid(const Mesh& m, const double c[3], const double ax[3], const double q[4], const double vel[3],
                    const double omega[3], HostObstacle& out) {
  double L[3][3], box[3][2];
  quat_lab_to_body(q, L);
  ellipsoid_fill_box(c, ax, m.spec.hmin, box);
  auto sdf = [&](double px, double py, double pz) {
    const double p[3] = {px - c[0], py - c[1], pz - c[2]};
    return ellipsoid_signed_distance(ax, L, p);
  };
  fill_from_sdf(m, sdf, box, vel, omega, out);
}

}  // namespace cup3d
