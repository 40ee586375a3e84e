// Host-side obstacle creation (the reference's CreateObstacles step, kept on
// the host): signed distance -> characteristic function chi on the blocks the
// body touches, deformation velocity udef, rigid-body kinematics.
#pragma once
#include <vector>

#include "mesh.h"

namespace cup3d {

struct HostObstacle {
  std::vector<int> blocks;       // obstacle slot -> block id (device order)
  std::vector<double> chi;       // nslots*512
  std::vector<double> udef;      // 3*nslots*512, component-major
  std::vector<double> grid_chi;  // nb*512: max over obstacles (sim.chi)
  double kin[9] = {0};           // centre of mass[3], velocity[3], angular velocity[3]
  double mass = 0;               // sum chi h^3
};

// Sphere (Sphere.cpp:19-51 fill rule and SDF) with chi from the Towers FDMH
// smoothed Heaviside of KernelCharacteristicFunction (ObstaclesCreate.cpp:18-121).
// Rigid body: udef = 0; centre of mass from the chi moments.
void make_sphere(const Mesh& m, const double c[3], double r, const double vel[3], const double omega[3],
                 HostObstacle& out);

// Rotation matrix (body -> lab) of the unit quaternion q = (w, x, y, z).
void quat_rotation(const double q[4], double R[3][3]);

// Bounding-box margin of the fill rule: (2 + 1) times the coarsest spacing.
constexpr double kObstacleSafety = 2.0 + 1.0;

// Ellipsoid with semi-axes ax[3] rotated by quaternion q (w, x, y, z); the
// signed distance is the ellipsoid's algebraic level set scaled to distance
// units near the surface (see obstacles.cpp).
void make_ellipsoid(const Mesh& m, const double c[3], const double ax[3], const double q[4], const double vel[3],
                    const double omega[3], HostObstacle& out);

}  // namespace cup3d
