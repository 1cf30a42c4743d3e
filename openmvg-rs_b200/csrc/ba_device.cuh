// ba_device.cuh — device-side numerics of the bundle-adjustment hot path (sm_100a).
//
// Each function restates the reference computation it cites (paths relative to the openmvg-rs root);
// the GPU kernels in ba_kernels.cu build on these. All functions are __host__ __device__ so the
// host-side bookkeeping (final metrics, weak points) uses the identical arithmetic.
#pragma once

#include <cmath>
#include <cstdint>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

namespace omvgba {

#ifndef __CUDACC__
using std::copysign;
using std::fabs;
using std::fma;
using std::fmax;
using std::fmin;
using std::hypot;
using std::isfinite;
using std::log1p;
using std::sqrt;
#endif

#define BA_HD __host__ __device__ __forceinline__

constexpr double kEps = 2.220446049250313e-16;
constexpr double kMinPositive = 2.2250738585072014e-308;

enum LossKindDev : int32_t { kLossL2 = 0, kLossHuber = 1, kLossCauchy = 2 };

// Robust loss (numerics/robust.rs:7-44, numerics/refine/api.rs:369-387). scale: Huber delta or
// Cauchy scale already divided by sqrt(2) (problem.rs:372-382).
struct LossDev {
  int32_t kind;
  double scale;
  BA_HD double sqrt_weight(double r) const {
    if (kind == kLossHuber) {
      double m = fabs(r);
      if (m <= scale || m == 0.0) return 1.0;
      return sqrt(scale / m);
    }
    if (kind == kLossCauchy) {
      double x2 = (r / scale) * (r / scale);
      return sqrt(1.0 / (scale * scale * (0.5 * x2 + 1.0)));
    }
    return 1.0;
  }
  BA_HD double cost(double r) const {
    if (kind == kLossHuber) {
      double m = fabs(r);
      return m <= scale ? 0.5 * r * r : scale * (m - 0.5 * scale);
    }
    if (kind == kLossCauchy) {
      double x2 = (r / scale) * (r / scale);
      return log1p(0.5 * x2);
    }
    return 0.5 * r * r;
  }
};

BA_HD bool finite3(double a, double b, double c) { return isfinite(a) && isfinite(b) && isfinite(c); }

// Fixed perspective camera: pinhole or Brown–Conrady with k1..k3, p1, p2
// (openmvg-core camera/brown_conrady.rs:134-252, camera/distortion.rs:227-635, camera/pinhole.rs:276-321).
struct FixedCameraDev {
  double fx, fy, cx, cy;
  double k1, k2, k3, p1, p2;  // zero when the discriminant does not declare them
  int32_t radial_kind, tangential_kind;
  double turn_squared;  // first positive root of 1 + 3 k1 q + 5 k2 q^2, or +inf
  int32_t has_turn;

  BA_HD bool has_distortion() const { return radial_kind != 0 || tangential_kind != 0; }
  BA_HD double radial_apply(double r2) const {
    if (radial_kind == 0) return 1.0;
    if (radial_kind == 1) return 1.0 + k1 * r2;
    double r4 = r2 * r2;
    if (radial_kind == 2) return 1.0 + k1 * r2 + k2 * r4;
    return 1.0 + k1 * r2 + k2 * r4 + k3 * (r4 * r2);
  }
  BA_HD void apply_distortion(double x, double y, double* xd, double* yd) const {
    double r2 = x * x + y * y;
    double f = radial_apply(r2);
    double tx = 0.0, ty = 0.0;
    if (tangential_kind == 1) {
      tx = 2.0 * p1 * x * y;
      ty = p1 * (r2 + 2.0 * y * y);
    } else if (tangential_kind == 2) {
      tx = 2.0 * p1 * x * y + p2 * (r2 + 2.0 * x * x);
      ty = p1 * (r2 + 2.0 * y * y) + 2.0 * p2 * x * y;
    }
    *xd = x * f + tx;
    *yd = y * f + ty;
  }
  // distortion_jacobian (distortion.rs:613-635)
  BA_HD bool distortion_jacobian(double x, double y, double* j11, double* j12, double* j22, double* det) const {
    double r2 = fma(x, x, y * y);
    double rf = radial_apply(r2);
    double rd = k1 + 2.0 * (k2 * r2) + 3.0 * (k3 * r2 * r2);
    *j11 = rf + 2.0 * x * x * rd + 2.0 * p1 * y + 6.0 * p2 * x;
    *j12 = 2.0 * x * y * rd + 2.0 * p1 * x + 2.0 * p2 * y;
    *j22 = rf + 2.0 * y * y * rd + 6.0 * p1 * y + 2.0 * p2 * x;
    *det = fma(*j11, *j22, -(*j12) * (*j12));
    return isfinite(*j11) && isfinite(*j12) && isfinite(*j22) && isfinite(*det);
  }
  // is_validated_distortion_invertible_at (distortion.rs:580-602): 33 samples with k3 or p terms
  BA_HD bool invertible_at(double x, double y) const {
    double a, b, c, d;
    if (k3 == 0.0 && p1 == 0.0 && p2 == 0.0) {
      double r2 = fma(x, x, y * y);
      if (!isfinite(r2) || (has_turn && r2 >= turn_squared)) return false;
      return distortion_jacobian(x, y, &a, &b, &c, &d) && d > 1e-12;
    }
    for (int i = 0; i <= 32; ++i) {
      double s = double(i) / 32.0;
      if (!(distortion_jacobian(x * s, y * s, &a, &b, &c, &d) && d > 1e-12)) return false;
    }
    return true;
  }
  // validate_forward_domain (brown_conrady.rs:134-166)
  BA_HD bool forward_domain(double x, double y) const {
    if (!isfinite(x) || !isfinite(y)) return false;
    if (!has_distortion()) return true;
    if (k3 == 0.0 && p1 == 0.0 && p2 == 0.0) {
      double r2 = fma(x, x, y * y);
      if (!isfinite(r2)) return false;
      if (has_turn && r2 >= turn_squared) return false;
      double a, b, c, d;
      if (!distortion_jacobian(x, y, &a, &b, &c, &d)) return false;
      return d > 1e-12;
    }
    return invertible_at(x, y);
  }
  // project (brown_conrady.rs:200-223) -> pixel
  BA_HD bool project(double X, double Y, double Z, double* u, double* v) const {
    if (!finite3(X, Y, Z) || Z <= 0.0) return false;
    double xn = X / Z, yn = Y / Z;
    if (!forward_domain(xn, yn)) return false;
    double xd, yd;
    apply_distortion(xn, yn, &xd, &yd);
    *u = fma(fx, xd, cx);
    *v = fma(fy, yd, cy);
    return isfinite(*u) && isfinite(*v);
  }
  // project_with_jacobian (brown_conrady.rs:225-252; pinhole.rs:301-321): residual and d pixel / d X
  BA_HD bool linearize(double X, double Y, double Z, double ox, double oy, double r[2], double J[2][3]) const {
    double u, v;
    if (!project(X, Y, Z, &u, &v)) return false;
    double iz = 1.0 / Z;
    if (!has_distortion()) {
      double iz2 = iz * iz;
      J[0][0] = fx * iz;
      J[0][1] = 0.0;
      J[0][2] = -fx * X * iz2;
      J[1][0] = 0.0;
      J[1][1] = fy * iz;
      J[1][2] = -fy * Y * iz2;
    } else {
      double x = X * iz, y = Y * iz, j11, j12, j22, det;
      if (!distortion_jacobian(x, y, &j11, &j12, &j22, &det)) return false;
      J[0][0] = fx * j11 * iz;
      J[0][1] = fx * j12 * iz;
      J[0][2] = -fx * (j11 * x + j12 * y) * iz;
      J[1][0] = fy * j12 * iz;
      J[1][1] = fy * j22 * iz;
      J[1][2] = -fy * (j12 * x + j22 * y) * iz;
    }
    r[0] = u - ox;
    r[1] = v - oy;
    for (int i = 0; i < 2; ++i)
      if (!finite3(J[i][0], J[i][1], J[i][2])) return false;
    return isfinite(r[0]) && isfinite(r[1]);
  }
  // remove_validated_distortion (distortion.rs:637-720): damped Newton, used for invertibility counts
  BA_HD bool remove_distortion(double xd, double yd) const {
    double x, y;
    return remove_distortion(xd, yd, &x, &y);
  }
  BA_HD bool remove_distortion(double xd, double yd, double* xo, double* yo) const {
    if (!isfinite(xd) || !isfinite(yd)) return false;
    if (!has_distortion()) {
      *xo = xd;
      *yo = yd;
      return true;
    }
    double x = xd, y = yd;
    for (int it = 1; it <= 30; ++it) {
      double dxx, dyy;
      apply_distortion(x, y, &dxx, &dyy);
      double dx = xd - dxx, dy = yd - dyy;
      double e2 = fma(dx, dx, dy * dy);
      if (e2 <= 1e-24) {
        if (!invertible_at(x, y)) return false;
        *xo = x;
        *yo = y;
        return true;
      }
      double j11, j12, j22, det;
      if (!distortion_jacobian(x, y, &j11, &j12, &j22, &det)) return false;
      if (fabs(det) <= 1e-15) return false;
      double sx = (j22 * dx - j12 * dy) / det, sy = (j11 * dy - j12 * dx) / det;
      if (!isfinite(sx) || !isfinite(sy)) return false;
      double damping = 1.0;
      bool accepted = false;
      for (int h = 0; h < 16; ++h) {
        double cxv = x + damping * sx, cyv = y + damping * sy, ex, ey;
        apply_distortion(cxv, cyv, &ex, &ey);
        double cdx = xd - ex, cdy = yd - ey;
        double ce = fma(cdx, cdx, cdy * cdy);
        if (isfinite(ce) && ce < e2) {
          x = cxv;
          y = cyv;
          accepted = true;
          break;
        }
        damping *= 0.5;
      }
      if (!accepted) return false;
    }
    return false;
  }
};

// ---- angular residuals (kernel/projection.rs:89-195) -------------------------------------------
BA_HD double dot3(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
BA_HD void cross3(const double a[3], const double b[3], double out[3]) {
  out[0] = a[1] * b[2] - a[2] * b[1];
  out[1] = a[2] * b[0] - a[0] * b[2];
  out[2] = a[0] * b[1] - a[1] * b[0];
}
// normalize (projection.rs:156-169): vectors already of unit length to 8 eps stay as they are
BA_HD bool normalize3(const double v[3], double out[3]) {
  const double n2 = dot3(v, v);
  if (!finite3(v[0], v[1], v[2]) || !(isfinite(n2) && n2 > kMinPositive)) return false;
  if (fabs(n2 - 1.0) <= 8.0 * kEps) {
    out[0] = v[0];
    out[1] = v[1];
    out[2] = v[2];
    return true;
  }
  const double inv = 1.0 / sqrt(n2);
  for (int k = 0; k < 3; ++k) out[k] = v[k] * inv;
  return true;
}
// tangent_basis (projection.rs:171-186)
BA_HD void tangent_basis3(const double u[3], double b0[3], double b1[3]) {
  double ref[3] = {0.0, 0.0, 0.0};
  if (fabs(u[0]) <= fabs(u[1]) && fabs(u[0]) <= fabs(u[2]))
    ref[0] = 1.0;
  else if (fabs(u[1]) <= fabs(u[2]))
    ref[1] = 1.0;
  else
    ref[2] = 1.0;
  cross3(u, ref, b0);
  const double inv = 1.0 / sqrt(dot3(b0, b0));
  for (int k = 0; k < 3; ++k) b0[k] *= inv;
  cross3(u, b0, b1);
}
// angular_projection (projection.rs:89-149): the residual angle(observation, prediction) times the
// unit direction in the observation's tangent plane, and its Jacobian d r / d X in the camera frame.
BA_HD bool angular_linearize(const double raw_obs[3], const double X[3], double r[2], double J[2][3]) {
  double obs[3], pred[3], b0[3], b1[3];
  if (!normalize3(raw_obs, obs) || !normalize3(X, pred)) return false;
  tangent_basis3(obs, b0, b1);
  const double a = dot3(b0, pred), b = dot3(b1, pred), c = dot3(obs, pred);
  const double s2 = a * a + b * b, s = sqrt(s2);
  if (c < 0.0 && s < 1e-6) return false;  // near the antipode
  double factor, fscale = 0.0, angle = 0.0;
  if (s < 1e-6) {
    const double s4 = s2 * s2;
    factor = 1.0 + s2 / 6.0 + 3.0 * s4 / 40.0;
    fscale = 1.0 / 3.0 + 3.0 * s2 / 10.0;
  } else {
    angle = atan2(s, c);
    factor = angle / s;
  }
  double dp[2][3];
  for (int k = 0; k < 3; ++k) {
    const double da = b0[k], db = b1[k], dc = obs[k];
    double fd;
    if (s < 1e-6) {
      fd = fscale * (a * da + b * db);
    } else {
      const double ds = (a * da + b * db) / s;
      const double ad = (c * ds - s * dc) / (s2 + c * c);
      fd = (ad * s - angle * ds) / s2;
    }
    dp[0][k] = factor * da + a * fd;
    dp[1][k] = factor * db + b * fd;
  }
  const double pn = sqrt(dot3(X, X));
  for (int row = 0; row < 2; ++row)
    for (int col = 0; col < 3; ++col) {
      double acc = 0.0;
      for (int k = 0; k < 3; ++k) acc += dp[row][k] * (((col == k) ? 1.0 : 0.0) - pred[col] * pred[k]) / pn;
      J[row][col] = acc;
    }
  r[0] = factor * a;
  r[1] = factor * b;
  for (int i = 0; i < 2; ++i)
    if (!finite3(J[i][0], J[i][1], J[i][2])) return false;
  return isfinite(r[0]) && isfinite(r[1]);
}

// Pinhole pixel projection with the 64-eps depth floor (kernel/projection.rs:47-87), skew 0.
BA_HD bool pixel_linearize(const FixedCameraDev& c, double X, double Y, double Z, double ox, double oy, double r[2],
                           double J[2][3]) {
  double s = fmax(fmax(fabs(X), fabs(Y)), fabs(Z));
  if (!finite3(X, Y, Z) || Z <= 64.0 * kEps * s) return false;
  double iz = 1.0 / Z, iz2 = iz * iz, xn = c.fx * X;
  r[0] = xn * iz + c.cx - ox;
  r[1] = c.fy * Y * iz + c.cy - oy;
  J[0][0] = c.fx * iz;
  J[0][1] = 0.0;
  J[0][2] = -xn * iz2;
  J[1][0] = 0.0;
  J[1][1] = c.fy * iz;
  J[1][2] = -c.fy * Y * iz2;
  for (int i = 0; i < 2; ++i)
    if (!finite3(J[i][0], J[i][1], J[i][2])) return false;
  return isfinite(r[0]) && isfinite(r[1]);
}

// first_positive_radial_turn (self_calibration/model.rs:245-268)
BA_HD bool first_radial_turn_squared(double k1, double k2, double* out) {
  double scale = fmax(fmax(fabs(k1), fabs(k2)), 1.0);
  double a = 5.0 * (k2 / scale), b = 3.0 * (k1 / scale), c = 1.0 / scale;
  if (a == 0.0) {
    double root = -c / b;
    if (b < 0.0 && isfinite(root) && root > 0.0) {
      *out = root;
      return true;
    }
    return false;
  }
  double disc = fma(b, b, -4.0 * a * c);
  if (disc < 0.0 || !isfinite(disc)) return false;
  double q = -0.5 * (b + copysign(sqrt(disc), b));
  double r0, r1;
  if (q == 0.0) {
    r0 = -b / (2.0 * a);
    r1 = NAN;
  } else {
    r0 = q / a;
    r1 = c / q;
  }
  bool have = false;
  double best = 0.0;
  if (isfinite(r0) && r0 > 0.0) {
    best = r0;
    have = true;
  }
  if (isfinite(r1) && r1 > 0.0 && (!have || r1 < best)) {
    best = r1;
    have = true;
  }
  *out = best;
  return have;
}

// Centred radial camera (log f, k1, k2): self_calibration/model.rs:26-324.
struct RadialDev {
  double focal, k1, k2;
  double turn;   // first radial turn squared, valid when has_turn
  int32_t has_turn;
};
// radial_linearization (positive depth): residual, d pred / d X, intrinsic Jacobian (log f, k1, k2)
BA_HD bool radial_linearize(const RadialDev& c, double X, double Y, double Z, double ox, double oy, double r[2],
                            double J[2][3], double Ji[2][3]) {
  double s = fmax(fmax(fabs(X), fabs(Y)), fabs(Z));
  if (!finite3(X, Y, Z) || !(Z > 64.0 * kEps * s)) return false;
  double iz = 1.0 / Z;
  double n0 = X * iz, n1 = Y * iz;
  double r2 = n0 * n0 + n1 * n1;
  if (c.has_turn && r2 >= c.turn) return false;
  double r4 = r2 * r2;
  double dist = 1.0 + c.k1 * r2 + c.k2 * r4;
  double rd = c.k1 + 2.0 * (c.k2 * r2);
  double slope = dist + 2.0 * r2 * rd;
  double det = dist * slope;
  if (!isfinite(det) || det <= 1e-12) return false;
  double p0 = c.focal * dist * n0, p1 = c.focal * dist * n1;
  if (!(isfinite(p0) && isfinite(p1) && isfinite(r2) && isfinite(r4) && isfinite(dist))) return false;
  double dx = 2.0 * n0 * rd, dy = 2.0 * n1 * rd;
  double nj00 = c.focal * (dist + n0 * dx), nj01 = c.focal * n0 * dy;
  double nj10 = c.focal * n1 * dx, nj11 = c.focal * (dist + n1 * dy);
  J[0][0] = nj00 * iz;
  J[0][1] = nj01 * iz;
  J[0][2] = -(nj00 * n0 + nj01 * n1) * iz;
  J[1][0] = nj10 * iz;
  J[1][1] = nj11 * iz;
  J[1][2] = -(nj10 * n0 + nj11 * n1) * iz;
  r[0] = p0 - ox;
  r[1] = p1 - oy;
  Ji[0][0] = p0;
  Ji[0][1] = c.focal * r2 * n0;
  Ji[0][2] = c.focal * r4 * n0;
  Ji[1][0] = p1;
  Ji[1][1] = c.focal * r2 * n1;
  Ji[1][2] = c.focal * r4 * n1;
  for (int i = 0; i < 2; ++i)
    if (!finite3(J[i][0], J[i][1], J[i][2]) || !finite3(Ji[i][0], Ji[i][1], Ji[i][2])) return false;
  return isfinite(r[0]) && isfinite(r[1]);
}

// radial_bearing (self_calibration/model.rs:171-230): can the measurement be inverted?
BA_HD bool radial_bearing_ok(const RadialDev& c, double mx, double my) {
  if (!(c.focal > 0.0 && isfinite(c.focal) && isfinite(c.k1) && isfinite(c.k2))) return false;
  if (!isfinite(mx) || !isfinite(my)) return false;
  double d0 = mx / c.focal, d1 = my / c.focal;
  double dr = hypot(d0, d1);
  if (!isfinite(dr)) return false;
  if (dr == 0.0) return true;
  double upper;
  if (c.has_turn) {
    upper = sqrt(c.turn);
    double u2 = upper * upper;
    double maximum = upper * (1.0 + c.k1 * u2 + c.k2 * u2 * u2);
    double tol = 64.0 * kEps * (1.0 + fabs(maximum));
    if (!isfinite(maximum) || dr >= maximum - tol) return false;
  } else {
    upper = fmax(dr, 1.0);
    for (int guard = 0; guard < 2100; ++guard) {
      double u2 = upper * upper;
      double pr = upper * (1.0 + c.k1 * u2 + c.k2 * u2 * u2);
      if (!isfinite(pr)) return false;
      if (pr >= dr) break;
      upper *= 2.0;
      if (!isfinite(upper)) return false;
    }
  }
  double tol = 1e-14 * (1.0 + dr);
  double lower = 0.0, rr = fmin(dr, 0.5 * upper);
  for (int i = 0; i < 48; ++i) {
    double r2 = rr * rr;
    double v = rr * (1.0 + c.k1 * r2 + c.k2 * r2 * r2) - dr;
    if (fabs(v) <= tol) {
      double s = rr / dr;
      double b0 = d0 * s, b1 = d1 * s;
      double nrm = sqrt(b0 * b0 + b1 * b1 + 1.0);
      return isfinite(nrm) && nrm > kMinPositive;
    }
    if (v < 0.0)
      lower = rr;
    else
      upper = rr;
    double der = 1.0 + 3.0 * c.k1 * r2 + 5.0 * c.k2 * r2 * r2;
    double newton = rr - v / der;
    rr = (isfinite(der) && der > 0.0 && newton > lower && newton < upper) ? newton : 0.5 * (lower + upper);
  }
  return false;
}

// PointBlockFactor (kernel/point_block.rs:78-160): Jacobi-scaled Cholesky of the damped 3x3 block.
// V packed lower (00, 10, 11, 20, 21, 22). Returns false when the block cannot be factored.
BA_HD bool point_damping_diagonal(const double V[6], double d[3]) {
  double ds = fmax(fmax(fmax(0.0, V[0]), V[2]), V[5]);
  if (!(isfinite(ds) && ds > 0.0)) return false;
  double fl = 64.0 * kEps * ds;
  d[0] = fmax(V[0], fl);
  d[1] = fmax(V[2], fl);
  d[2] = fmax(V[5], fl);
  return true;
}
// With fac non-null it also receives N = (S L)^-1 (S the scaling, L the factor of the scaled block),
// lower packed like inv: Vhat^-1 = N^T N. Applying N and then N^T to a vector is linear and
// symmetric to rounding even for a badly conditioned block, where a product with the explicit
// inverse is not: a track-2 point close to a camera centre (cond 1e9) gives that product rounding
// noise near 1e-5 of its size, which changes from one vector to the next.
BA_HD bool point_factor(const double V[6], double lambda, double damped[6], double inv[6], double* fac = nullptr) {
  double d[3];
  if (!point_damping_diagonal(V, d)) return false;
  double a[3][3] = {{V[0] + lambda * d[0], V[1], V[3]}, {V[1], V[2] + lambda * d[1], V[4]}, {V[3], V[4], V[5] + lambda * d[2]}};
  damped[0] = a[0][0];
  damped[1] = a[1][0];
  damped[2] = a[1][1];
  damped[3] = a[2][0];
  damped[4] = a[2][1];
  damped[5] = a[2][2];
  double ds = fmax(fmax(fmax(0.0, a[0][0]), a[1][1]), a[2][2]);
  double fl = 64.0 * kEps * ds;
  double sc[3] = {sqrt(fmax(a[0][0], fl)), sqrt(fmax(a[1][1], fl)), sqrt(fmax(a[2][2], fl))};
  double l[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c <= r; ++c) {
      double v = 0.5 * (a[r][c] + a[c][r]) / (sc[r] * sc[c]);
      for (int k = 0; k < c; ++k) v -= l[r][k] * l[c][k];
      if (r == c) {
        if (!(isfinite(v) && v > 64.0 * kEps)) return false;
        l[r][c] = sqrt(v);
      } else {
        l[r][c] = v / l[c][c];
      }
    }
  double m00 = 1.0 / l[0][0], m11 = 1.0 / l[1][1], m22 = 1.0 / l[2][2];
  double m10 = -l[1][0] * m00 * m11;
  double m21 = -l[2][1] * m11 * m22;
  double m20 = -(l[2][0] * m00 + l[2][1] * m10) * m22;
  double d0 = 1.0 / sc[0], d1 = 1.0 / sc[1], d2 = 1.0 / sc[2];
  inv[0] = (m00 * m00 + m10 * m10 + m20 * m20) * (d0 * d0);
  inv[1] = (m11 * m10 + m21 * m20) * (d1 * d0);
  inv[2] = (m11 * m11 + m21 * m21) * (d1 * d1);
  inv[3] = (m22 * m20) * (d2 * d0);
  inv[4] = (m22 * m21) * (d2 * d1);
  inv[5] = (m22 * m22) * (d2 * d2);
  if (fac) {
    fac[0] = m00 * d0;
    fac[1] = m10 * d0;
    fac[2] = m11 * d1;
    fac[3] = m20 * d0;
    fac[4] = m21 * d1;
    fac[5] = m22 * d2;
  }
  return true;
}
BA_HD void sym3_apply(const double P[6], const double x[3], double y[3]) {
  y[0] = P[0] * x[0] + P[1] * x[1] + P[3] * x[2];
  y[1] = P[1] * x[0] + P[2] * x[1] + P[4] * x[2];
  y[2] = P[3] * x[0] + P[4] * x[1] + P[5] * x[2];
}
// reciprocal_condition_number (point_block.rs:163-184) with infinity norms
BA_HD double point_rcond(const double V[6], const double inv[6]) {
  double nV = fmax(fmax(fabs(V[0]) + fabs(V[1]) + fabs(V[3]), fabs(V[1]) + fabs(V[2]) + fabs(V[4])),
                   fabs(V[3]) + fabs(V[4]) + fabs(V[5]));
  double nI = fmax(fmax(fabs(inv[0]) + fabs(inv[1]) + fabs(inv[3]), fabs(inv[1]) + fabs(inv[2]) + fabs(inv[4])),
                   fabs(inv[3]) + fabs(inv[4]) + fabs(inv[5]));
  double den = nV * nI;
  return (isfinite(den) && den > 0.0) ? 1.0 / den : 0.0;
}

// Track geometry admission (kernel/point_geometry.rs:16-130).
struct TrackGeometryDev {
  double near2, far2, scene2;
  double f0, f1, f2;
  int32_t has_first, parallax, observations, invalid;
  BA_HD void init(double scene) {
    near2 = INFINITY;
    far2 = scene * scene;
    scene2 = scene * scene;
    has_first = 0;
    parallax = 0;
    observations = 0;
    invalid = 0;
    f0 = f1 = f2 = 0.0;
  }
  BA_HD void push(double x, double y, double z) {
    double sq = x * x + y * y + z * z;
    if (!(isfinite(sq) && sq > 0.0)) {
      invalid = 1;
      return;
    }
    observations++;
    near2 = fmin(near2, sq);
    far2 = fmax(far2, sq);
    double inv = 1.0 / sqrt(sq);
    double r0 = x * inv, r1 = y * inv, r2 = z * inv;
    if (!has_first) {
      has_first = 1;
      f0 = r0;
      f1 = r1;
      f2 = r2;
      return;
    }
    if (parallax) return;
    double d = r0 * f0 + r1 * f1 + r2 * f2;
    double c0 = r1 * f2 - r2 * f1, c1 = r2 * f0 - r0 * f2, c2 = r0 * f1 - r1 * f0;
    double s2 = c0 * c0 + c1 * c1 + c2 * c2;
    parallax = (d < 0.0 || s2 >= 1.7e-5 * 1.7e-5) ? 1 : 0;
  }
  BA_HD bool degenerate() const { return invalid || (observations >= 2 && (!parallax || near2 < 1e-8 * far2)); }
  BA_HD bool collapsed() const { return invalid || (observations >= 2 && near2 < 1e-8 * scene2); }
};

}  // namespace omvgba
