// Distance from a point to an ellipsoid by root bisection: D. Eberly,
// "Distance from a Point to an Ellipse, an Ellipsoid, or a Hyperellipsoid"
// (Geometric Tools, 2013), the method the reference's Ellipsoid obstacle uses
// for its signed distance (Ellipsoid.cpp:22-258).
//
// For a query y in the first octant and semi-axes e0 >= e1 >= e2, the closest
// surface point is x_i = e_i^2 y_i / (t + e_i^2), t the root of
//   F(t) = sum_i (e_i y_i / (t + e_i^2))^2 - 1,
// which is monotone for t > -e2^2 and bracketed by [-e2^2 + e2 y2,
// -e2^2 + |e.y|].  Zero coordinates reduce the problem to an ellipse (or to
// an axis endpoint); the ellipse case brackets its root the same way.  The
// bisection stops when the midpoint no longer moves by more than the machine
// epsilon (absolute), after at most 2 * 1024 halvings.
//
// The operations and their order are those of the published method as the
// reference states it, so that host, device and the checker produce the same
// bits: the chi of a body is compared bit for bit across them.  Used from
// code compiled without fused multiply-adds.
#pragma once
#include <math.h>

namespace cup3d {

constexpr double kEllEps = 2.220446049250313e-16;  // DBL_EPSILON
constexpr int kEllMaxHalvings = 2 * 1024;            // 2 * DBL_MAX_EXP

// Ellipse (x0/e0)^2 + (x1/e1)^2 = 1, e0 >= e1, query y0, y1 >= 0: distance,
// closest point into x.
__host__ __device__ inline double ellipse_distance_q1(const double e[2], const double y[2], double x[2]) {
  if (y[1] > 0) {
    if (y[0] > 0) {
      const double e2[2] = {e[0] * e[0], e[1] * e[1]};
      const double ey[2] = {e[0] * y[0], e[1] * y[1]};
      double lo = -e2[1] + ey[1];
      double hi = -e2[1] + sqrt(ey[0] * ey[0] + ey[1] * ey[1]);
      double t = lo;
      for (int k = 0; k < kEllMaxHalvings; ++k) {
        t = 0.5 * (lo + hi);
        if (fabs(t - lo) < kEllEps || fabs(t - hi) < kEllEps) break;
        const double r0 = ey[0] / (t + e2[0]), r1 = ey[1] / (t + e2[1]);
        const double f = r0 * r0 + r1 * r1 - 1;
        if (f > 0)
          lo = t;
        else if (f < 0)
          hi = t;
        else
          break;
      }
      x[0] = e2[0] * y[0] / (t + e2[0]);
      x[1] = e2[1] * y[1] / (t + e2[1]);
      const double d0 = x[0] - y[0], d1 = x[1] - y[1];
      return sqrt(d0 * d0 + d1 * d1);
    }
    x[0] = 0;
    x[1] = e[1];
    return fabs(y[1] - e[1]);
  }
  const double den = e[0] * e[0] - e[1] * e[1];
  const double e0y0 = e[0] * y[0];
  if (e0y0 < den) {
    const double u = e0y0 / den;
    const double u2 = u * u;
    x[0] = e[0] * u;
    x[1] = e[1] * sqrt(fabs(1.0 - u2));
    const double d0 = x[0] - y[0];
    return sqrt(d0 * d0 + x[1] * x[1]);
  }
  x[0] = e[0];
  x[1] = 0;
  return fabs(y[0] - e[0]);
}

// Ellipsoid with e0 >= e1 >= e2, query in the first octant.
__host__ __device__ inline double ellipsoid_distance_q1(const double e[3], const double y[3], double x[3]) {
  if (y[2] > 0) {
    if (y[1] > 0) {
      if (y[0] > 0) {
        const double e2[3] = {e[0] * e[0], e[1] * e[1], e[2] * e[2]};
        const double ey[3] = {e[0] * y[0], e[1] * y[1], e[2] * y[2]};
        double lo = -e2[2] + ey[2];
        double hi = -e2[2] + sqrt(ey[0] * ey[0] + ey[1] * ey[1] + ey[2] * ey[2]);
        double t = lo;
        for (int k = 0; k < kEllMaxHalvings; ++k) {
          t = 0.5 * (lo + hi);
          if (fabs(t - lo) < kEllEps || fabs(t - hi) < kEllEps) break;
          const double r0 = ey[0] / (t + e2[0]), r1 = ey[1] / (t + e2[1]), r2 = ey[2] / (t + e2[2]);
          const double f = r0 * r0 + r1 * r1 + r2 * r2 - 1;
          if (f > 0)
            lo = t;
          else if (f < 0)
            hi = t;
          else
            break;
        }
        x[0] = e2[0] * y[0] / (t + e2[0]);
        x[1] = e2[1] * y[1] / (t + e2[1]);
        x[2] = e2[2] * y[2] / (t + e2[2]);
        const double d0 = x[0] - y[0], d1 = x[1] - y[1], d2 = x[2] - y[2];
        return sqrt(d0 * d0 + d1 * d1 + d2 * d2);
      }
      // y0 = 0: the ellipse of axes (e1, e2) in the plane x0 = 0
      x[0] = 0;
      const double es[2] = {e[1], e[2]}, ys[2] = {y[1], y[2]};
      double xs[2];
      const double d = ellipse_distance_q1(es, ys, xs);
      x[1] = xs[0];
      x[2] = xs[1];
      return d;
    }
    x[1] = 0;
    if (y[0] > 0) {  // y1 = 0: the ellipse of axes (e0, e2)
      const double es[2] = {e[0], e[2]}, ys[2] = {y[0], y[2]};
      double xs[2];
      const double d = ellipse_distance_q1(es, ys, xs);
      x[0] = xs[0];
      x[2] = xs[1];
      return d;
    }
    x[0] = 0;
    x[2] = e[2];
    return fabs(y[2] - e[2]);
  }
  // y2 = 0: the closest point is above the (x0, x1) plane when (y0, y1) lies
  // inside the sub-ellipse of the focal radii, on the boundary ellipse otherwise
  const double den[2] = {e[0] * e[0] - e[2] * e[2], e[1] * e[1] - e[2] * e[2]};
  const double ey[2] = {e[0] * y[0], e[1] * y[1]};
  if (ey[0] < den[0] && ey[1] < den[1]) {
    const double u[2] = {ey[0] / den[0], ey[1] / den[1]};
    const double u2[2] = {u[0] * u[0], u[1] * u[1]};
    const double disc = 1 - u2[0] - u2[1];
    if (disc > 0) {
      x[0] = e[0] * u[0];
      x[1] = e[1] * u[1];
      x[2] = e[2] * sqrt(disc);
      const double d0 = x[0] - y[0], d1 = x[1] - y[1];
      return sqrt(d0 * d0 + d1 * d1 + x[2] * x[2]);
    }
  }
  x[2] = 0;
  return ellipse_distance_q1(e, y, x);
}

// Any query point and any order of the semi-axes: the query is reflected into
// the first octant and the axes sorted by decreasing length (ties keep the
// reference's choice), then the closest point mapped back.
__host__ __device__ inline double ellipsoid_distance(const double e[3], const double y[3], double x[3]) {
  int perm[3];
  if (e[0] < e[1]) {
    if (e[2] < e[0]) {
      perm[0] = 1; perm[1] = 0; perm[2] = 2;
    } else if (e[2] < e[1]) {
      perm[0] = 1; perm[1] = 2; perm[2] = 0;
    } else {
      perm[0] = 2; perm[1] = 1; perm[2] = 0;
    }
  } else {
    if (e[2] < e[1]) {
      perm[0] = 0; perm[1] = 1; perm[2] = 2;
    } else if (e[2] < e[0]) {
      perm[0] = 0; perm[1] = 2; perm[2] = 1;
    } else {
      perm[0] = 2; perm[1] = 0; perm[2] = 1;
    }
  }
  double le[3], ly[3], lx[3];
  for (int i = 0; i < 3; ++i) {
    const int j = perm[i];
    le[i] = e[j];
    ly[i] = y[j] < 0 ? -y[j] : y[j];
  }
  const double d = ellipsoid_distance_q1(le, ly, lx);
  for (int i = 0; i < 3; ++i) {
    const int j = perm[i];
    x[j] = y[j] < 0 ? -lx[i] : lx[i];
  }
  return d;
}

// Signed distance of the ellipsoid obstacle (positive inside, the sign
// convention of every obstacle's signedDistance, ObstacleLibrary.h:30-32):
// the query p (relative to the centre) is taken to body axes by the rows of
// L (lab -> body), and its distance is negative when p lies farther from the
// centre than its closest surface point.
__host__ __device__ inline double ellipsoid_signed_distance(const double e[3], const double L[3][3],
                                                           const double p[3]) {
  const double t[3] = {L[0][0] * p[0] + L[0][1] * p[1] + L[0][2] * p[2],
                       L[1][0] * p[0] + L[1][1] * p[1] + L[1][2] * p[2],
                       L[2][0] * p[0] + L[2][1] * p[1] + L[2][2] * p[2]};
  double xs[3];
  const double dist = ellipsoid_distance(e, t, xs);
  const double dc = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
  const double ds = xs[0] * xs[0] + xs[1] * xs[1] + xs[2] * xs[2];
  return dc > ds ? -dist : dist;
}

// Lab -> body rotation of the unit quaternion q = (w, x, y, z), the matrix
// the reference's ellipsoid applies to p (Ellipsoid.cpp:262-267).
__host__ __device__ inline void quat_lab_to_body(const double q[4], double L[3][3]) {
  const double w = q[0], x = q[1], y = q[2], z = q[3];
  L[0][0] = 1 - 2 * (y * y + z * z);
  L[0][1] = 2 * (x * y + z * w);
  L[0][2] = 2 * (x * z - y * w);
  L[1][0] = 2 * (x * y - z * w);
  L[1][1] = 1 - 2 * (x * x + z * z);
  L[1][2] = 2 * (y * z + x * w);
  L[2][0] = 2 * (x * z + y * w);
  L[2][1] = 2 * (y * z - x * w);
  L[2][2] = 1 - 2 * (x * x + y * y);
}

}  // namespace cup3d
