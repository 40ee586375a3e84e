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

// Fill boxes of the bodies: a block holds obstacle data when the range of its
// cell centres meets the box (isTouching).  The margin is (2 + SURFDH) hmin,
// SURFDH = 1 (ObstacleBlock.h:16), hmin the finest spacing the mesh may have
// (SimulationData.cpp:162).  Sphere: centre +- (r + margin) (Sphere.cpp:22-27);
// ellipsoid: centre +- 2 (largest semi-axis + margin) (Ellipsoid.cpp:252-258).
void sphere_fill_box(const double c[3], double r, double hmin, double box[3][2]);
void ellipsoid_fill_box(const double c[3], const double ax[3], double hmin, double box[3][2]);

// Ellipsoid with semi-axes ax[3] rotated by quaternion q (w, x, y, z); the
// signed distance is the exact distance to the surface (Eberly's bisection,
// ellipsoid_distance.cuh), positive inside.
void make_ellipsoid(const Mesh& m, const double c[3], const double ax[3], const double q[4], const double vel[3],
                    const double omega[3], HostObstacle& out);

}  // namespace cup3d
