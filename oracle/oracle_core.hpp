// oracle_core.hpp — TEST INFRASTRUCTURE ONLY. CPU restatement of the numeric building blocks of
// openmvg-rs `openmvg-ba` (and the Brown–Conrady camera of `openmvg-core`) that the bundle-adjustment
// hot path uses. Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may use it,
// as the checker; the shipped solver never links it.
//
// Parity pins: the reference Rust crate cannot be compiled in this environment (no Rust toolchain),
// so this restatement is pinned against the reference's own unit-test known answers
// (tests/test_oracle_pins.py) and against finite differences; see each function's citation.
// All paths cited are relative to the openmvg-rs repository root.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <limits>
#include <optional>

namespace oracle {

constexpr double kEps = std::numeric_limits<double>::epsilon();
constexpr double kMinPositive = std::numeric_limits<double>::min();
constexpr double kInf = std::numeric_limits<double>::infinity();

using Vec2 = std::array<double, 2>;
using Vec3 = std::array<double, 3>;
using Mat3 = std::array<std::array<double, 3>, 3>;
using Mat23 = std::array<std::array<double, 3>, 2>;

inline double dot3(const Vec3& a, const Vec3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline double norm3(const Vec3& a) { return std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }
inline bool all_finite(const double* v, int n) {
  for (int i = 0; i < n; ++i)
    if (!std::isfinite(v[i])) return false;
  return true;
}
inline Mat3 mat_mul(const Mat3& a, const Mat3& b) {  // numerics/manifold.rs:58-70
  Mat3 c{};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) c[i][j] += a[i][k] * b[k][j];
  return c;
}
inline Vec3 rotate(const Mat3& r, const Vec3& x) {  // kernel/multi_view/model.rs:694-703
  return {r[0][0] * x[0] + r[0][1] * x[1] + r[0][2] * x[2], r[1][0] * x[0] + r[1][1] * x[1] + r[1][2] * x[2],
          r[2][0] * x[0] + r[2][1] * x[1] + r[2][2] * x[2]};
}
inline Vec3 rotate_transposed(const Mat3& r, const Vec3& v) {  // schur/point.rs:836-845
  return {r[0][0] * v[0] + r[1][0] * v[1] + r[2][0] * v[2], r[0][1] * v[0] + r[1][1] * v[1] + r[2][1] * v[2],
          r[0][2] * v[0] + r[1][2] * v[1] + r[2][2] * v[2]};
}

// ---------------------------------------------------------------------------------------------
// Robust losses: numerics/robust.rs:7-44, numerics/refine/api.rs:369-387.
// ---------------------------------------------------------------------------------------------
enum class LossKind { L2 = 0, Huber = 1, Cauchy = 2 };
struct Loss {
  LossKind kind = LossKind::L2;
  double scale = 0.0;  // Huber delta, or Cauchy scale already divided by sqrt(2) (problem.rs:372-382)
  bool operator==(const Loss& o) const { return kind == o.kind && scale == o.scale; }
  double sqrt_weight(double r) const {
    switch (kind) {
      case LossKind::L2: return 1.0;
      case LossKind::Huber: {
        double m = std::fabs(r);
        if (m <= scale || m == 0.0) return 1.0;
        return std::sqrt(scale / m);
      }
      case LossKind::Cauchy: {
        double x2 = (r / scale) * (r / scale);
        return std::sqrt(1.0 / (scale * scale * (0.5 * x2 + 1.0)));
      }
    }
    return 1.0;
  }
  double cost(double r) const {
    switch (kind) {
      case LossKind::L2: return 0.5 * r * r;
      case LossKind::Huber: {
        double m = std::fabs(r);
        return m <= scale ? 0.5 * r * r : scale * (m - 0.5 * scale);
      }
      case LossKind::Cauchy: {
        double x2 = (r / scale) * (r / scale);
        return std::log1p(0.5 * x2);
      }
    }
    return 0.0;
  }
};

// ---------------------------------------------------------------------------------------------
// Projection result shared by the kernels: kernel/projection.rs:9-13.
// ---------------------------------------------------------------------------------------------
struct Projection {
  Vec2 residual;
  Mat23 jacobian;  // d(prediction)/d(camera point)
};
inline bool projection_finite(const Projection& p) {
  return all_finite(p.residual.data(), 2) && all_finite(&p.jacobian[0][0], 3) && all_finite(&p.jacobian[1][0], 3);
}

// Pinhole pixel projection with the 64 eps depth floor: kernel/projection.rs:47-87 (skew = 0).
inline std::optional<Projection> pixel_projection(double fx, double fy, double cx, double cy, const Vec2& obs,
                                                  const Vec3& p) {
  double scale = std::max({std::fabs(p[0]), std::fabs(p[1]), std::fabs(p[2])});
  if (!all_finite(p.data(), 3) || p[2] <= 64.0 * kEps * scale) return std::nullopt;
  double iz = 1.0 / p[2];
  double iz2 = iz * iz;
  double xn = fx * p[0];
  Projection pr;
  pr.residual = {xn * iz + cx - obs[0], fy * p[1] * iz + cy - obs[1]};
  pr.jacobian = {{{fx * iz, 0.0, -xn * iz2}, {0.0, fy * iz, -fy * p[1] * iz2}}};
  if (!projection_finite(pr)) return std::nullopt;
  return pr;
}

// ---------------------------------------------------------------------------------------------
// Brown–Conrady camera: openmvg-core camera/brown_conrady.rs:225-355, camera/distortion.rs:227-700,
// camera/pinhole.rs:276-321.
// ---------------------------------------------------------------------------------------------
struct BrownConrady {
  double fx = 1, fy = 1, cx = 0, cy = 0;
  int radial_kind = 0;      // 0 None, 1 K1, 2 K1K2, 3 K1K2K3
  int tangential_kind = 0;  // 0 None, 1 P1, 2 P1P2
  double k1 = 0, k2 = 0, k3 = 0, p1 = 0, p2 = 0;
  std::optional<double> turn_squared;  // first_radial_turn_squared(k1, k2)

  double rk1() const { return radial_kind >= 1 ? k1 : 0.0; }
  double rk2() const { return radial_kind >= 2 ? k2 : 0.0; }
  double rk3() const { return radial_kind >= 3 ? k3 : 0.0; }
  double tp1() const { return tangential_kind >= 1 ? p1 : 0.0; }
  double tp2() const { return tangential_kind >= 2 ? p2 : 0.0; }
  bool has_distortion() const { return radial_kind != 0 || tangential_kind != 0; }

  // RadialDistortion::apply (distortion.rs:227-241)
  double radial_apply(double r2) const {
    switch (radial_kind) {
      case 0: return 1.0;
      case 1: return 1.0 + k1 * r2;
      case 2: {
        double r4 = r2 * r2;
        return 1.0 + k1 * r2 + k2 * r4;
      }
      default: {
        double r4 = r2 * r2, r6 = r4 * r2;
        return 1.0 + k1 * r2 + k2 * r4 + k3 * r6;
      }
    }
  }
  // TangentialDistortion::apply (distortion.rs:493-509)
  Vec2 tangential_apply(double x, double y, double r2) const {
    switch (tangential_kind) {
      case 0: return {0.0, 0.0};
      case 1: return {2.0 * p1 * x * y, p1 * (r2 + 2.0 * y * y)};
      default: return {2.0 * p1 * x * y + p2 * (r2 + 2.0 * x * x), p1 * (r2 + 2.0 * y * y) + 2.0 * p2 * x * y};
    }
  }
  // apply_distortion (distortion.rs:530-551)
  Vec2 apply_distortion(double x, double y) const {
    double r2 = x * x + y * y;
    double f = radial_apply(r2);
    Vec2 t = tangential_apply(x, y, r2);
    return {x * f + t[0], y * f + t[1]};
  }
  // distortion_jacobian (distortion.rs:613-635): (j11, j12, j22, det)
  std::optional<std::array<double, 4>> distortion_jacobian(double x, double y) const {
    double r2 = std::fma(x, x, y * y);
    double rf = radial_apply(r2);
    double rd = rk1() + 2.0 * (rk2() * r2) + 3.0 * (rk3() * r2 * r2);
    double P1 = tp1(), P2 = tp2();
    double j11 = rf + 2.0 * x * x * rd + 2.0 * P1 * y + 6.0 * P2 * x;
    double j12 = 2.0 * x * y * rd + 2.0 * P1 * x + 2.0 * P2 * y;
    double j22 = rf + 2.0 * y * y * rd + 6.0 * P1 * y + 2.0 * P2 * x;
    double det = std::fma(j11, j22, -j12 * j12);
    if (!(std::isfinite(j11) && std::isfinite(j12) && std::isfinite(j22) && std::isfinite(det))) return std::nullopt;
    return std::array<double, 4>{j11, j12, j22, det};
  }
  // is_validated_distortion_invertible_at (distortion.rs:580-602), 33 samples when k3/p terms exist
  bool invertible_at(double x, double y) const {
    if (rk3() == 0.0 && tp1() == 0.0 && tp2() == 0.0) {
      double r2 = std::fma(x, x, y * y);
      if (!std::isfinite(r2) || (turn_squared && r2 >= *turn_squared)) return false;
      auto j = distortion_jacobian(x, y);
      return j && (*j)[3] > 1e-12;
    }
    for (int i = 0; i <= 32; ++i) {
      double s = double(i) / 32.0;
      auto j = distortion_jacobian(x * s, y * s);
      if (!(j && (*j)[3] > 1e-12)) return false;
    }
    return true;
  }
  // validate_forward_domain (brown_conrady.rs:134-166)
  bool forward_domain(double x, double y) const {
    if (!std::isfinite(x) || !std::isfinite(y)) return false;
    if (!has_distortion()) return true;
    if (rk3() == 0.0 && tp1() == 0.0 && tp2() == 0.0) {
      double r2 = std::fma(x, x, y * y);
      if (!std::isfinite(r2)) return false;
      if (turn_squared && r2 >= *turn_squared) return false;
      auto j = distortion_jacobian(x, y);
      if (!j) return false;
      if ((*j)[3] <= 1e-12) return false;
      return true;
    }
    return invertible_at(x, y);
  }
  // CameraModel::project (brown_conrady.rs:200-223; pinhole.rs:276-299)
  std::optional<Vec2> project(const Vec3& p) const {
    if (!all_finite(p.data(), 3)) return std::nullopt;
    if (p[2] <= 0.0) return std::nullopt;
    double xn = p[0] / p[2], yn = p[1] / p[2];
    if (!forward_domain(xn, yn)) return std::nullopt;
    Vec2 d = apply_distortion(xn, yn);
    // pinhole project of (xd, yd, 1): fx.mul_add(x * 1, cx)
    Vec2 px = {std::fma(fx, d[0], cx), std::fma(fy, d[1], cy)};
    if (!all_finite(px.data(), 2)) return std::nullopt;
    return px;
  }
  // project_with_jacobian (brown_conrady.rs:225-252); for no distortion pinhole.rs:301-321
  std::optional<Projection> project_with_jacobian(const Vec2& obs, const Vec3& p) const {
    auto px = project(p);
    if (!px) return std::nullopt;
    double iz = 1.0 / p[2];
    Projection pr;
    if (!has_distortion()) {
      double iz2 = iz * iz;
      pr.jacobian = {{{fx * iz, 0.0, -fx * p[0] * iz2}, {0.0, fy * iz, -fy * p[1] * iz2}}};
    } else {
      double x = p[0] * iz, y = p[1] * iz;
      auto j = distortion_jacobian(x, y);
      if (!j) return std::nullopt;
      double j11 = (*j)[0], j12 = (*j)[1], j22 = (*j)[2];
      pr.jacobian = {{{fx * j11 * iz, fx * j12 * iz, -fx * (j11 * x + j12 * y) * iz},
                      {fy * j12 * iz, fy * j22 * iz, -fy * (j12 * x + j22 * y) * iz}}};
    }
    pr.residual = {(*px)[0] - obs[0], (*px)[1] - obs[1]};
    if (!projection_finite(pr)) return std::nullopt;
    return pr;
  }
  // remove_validated_distortion (distortion.rs:637-720): damped Newton, 30 iterations, 16 halvings
  bool remove_distortion(double xd, double yd, double* xo, double* yo) const {
    if (!std::isfinite(xd) || !std::isfinite(yd)) return false;
    if (!has_distortion()) {
      *xo = xd;
      *yo = yd;
      return true;
    }
    double x = xd, y = yd;
    for (int it = 1; it <= 30; ++it) {
      Vec2 d = apply_distortion(x, y);
      double dx = xd - d[0], dy = yd - d[1];
      double e2 = std::fma(dx, dx, dy * dy);
      if (e2 <= 1e-24) {
        if (!invertible_at(x, y)) return false;
        *xo = x;
        *yo = y;
        return true;
      }
      auto j = distortion_jacobian(x, y);
      if (!j) return false;
      double j11 = (*j)[0], j12 = (*j)[1], j22 = (*j)[2], det = (*j)[3];
      if (std::fabs(det) <= 1e-15) return false;
      double sx = (j22 * dx - j12 * dy) / det, sy = (j11 * dy - j12 * dx) / det;
      if (!std::isfinite(sx) || !std::isfinite(sy)) return false;
      double damping = 1.0;
      bool accepted = false;
      for (int h = 0; h < 16; ++h) {
        double cxv = x + damping * sx, cyv = y + damping * sy;
        Vec2 cd = apply_distortion(cxv, cyv);
        double cdx = xd - cd[0], cdy = yd - cd[1];
        double ce = std::fma(cdx, cdx, cdy * cdy);
        if (std::isfinite(ce) && ce < e2) {
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

// first_radial_turn_squared / first_positive_radial_turn (distortion.rs:553-578,
// self_calibration/model.rs:245-268): first positive root of 1 + 3 k1 q + 5 k2 q^2.
inline std::optional<double> first_radial_turn_squared(double k1, double k2) {
  double scale = std::max({std::fabs(k1), std::fabs(k2), 1.0});
  double a = 5.0 * (k2 / scale), b = 3.0 * (k1 / scale), c = 1.0 / scale;
  if (a == 0.0) {
    double root = -c / b;
    if (b < 0.0 && std::isfinite(root) && root > 0.0) return root;
    return std::nullopt;
  }
  double disc = std::fma(b, b, -4.0 * a * c);
  if (disc < 0.0 || !std::isfinite(disc)) return std::nullopt;
  double q = -0.5 * (b + std::copysign(std::sqrt(disc), b));
  double roots[2];
  if (q == 0.0) {
    roots[0] = -b / (2.0 * a);
    roots[1] = std::nan("");
  } else {
    roots[0] = q / a;
    roots[1] = c / q;
  }
  std::optional<double> best;
  for (double r : roots)
    if (std::isfinite(r) && r > 0.0 && (!best || r < *best)) best = r;
  return best;
}

// ---------------------------------------------------------------------------------------------
// Centred radial camera (log f, k1, k2): kernel/multi_view/self_calibration/model.rs:16-350.
// ---------------------------------------------------------------------------------------------
struct Radial {
  double focal = 1, k1 = 0, k2 = 0;
};
struct RadialTerms {
  Vec2 normalized;
  double r2, r4, distortion;
  Vec2 prediction;
  double inverse_depth;
};
// radial_terms_with_depth, positive-depth branch (model.rs:26-75)
inline std::optional<RadialTerms> radial_terms(const Radial& cam, const Vec3& p) {
  double scale = std::max({std::fabs(p[0]), std::fabs(p[1]), std::fabs(p[2])});
  double floor = 64.0 * kEps * scale;
  if (!all_finite(p.data(), 3) || !(p[2] > floor)) return std::nullopt;
  RadialTerms t;
  t.inverse_depth = 1.0 / p[2];
  t.normalized = {p[0] * t.inverse_depth, p[1] * t.inverse_depth};
  t.r2 = t.normalized[0] * t.normalized[0] + t.normalized[1] * t.normalized[1];
  auto turn = first_radial_turn_squared(cam.k1, cam.k2);
  if (turn && t.r2 >= *turn) return std::nullopt;
  t.r4 = t.r2 * t.r2;
  t.distortion = 1.0 + cam.k1 * t.r2 + cam.k2 * t.r4;
  double rd = cam.k1 + 2.0 * (cam.k2 * t.r2);
  double slope = t.distortion + 2.0 * t.r2 * rd;
  double det = t.distortion * slope;
  if (!std::isfinite(det) || det <= 1e-12) return std::nullopt;
  t.prediction = {cam.focal * t.distortion * t.normalized[0], cam.focal * t.distortion * t.normalized[1]};
  if (!(std::isfinite(t.prediction[0]) && std::isfinite(t.prediction[1]) && std::isfinite(t.r2) &&
        std::isfinite(t.r4) && std::isfinite(t.distortion)))
    return std::nullopt;
  return t;
}
// radial_projection_from_terms (model.rs:86-125)
inline std::optional<Projection> radial_projection(const Radial& cam, const Vec2& obs, const RadialTerms& t) {
  double rd = cam.k1 + 2.0 * (cam.k2 * t.r2);
  double dx = 2.0 * t.normalized[0] * rd, dy = 2.0 * t.normalized[1] * rd;
  double nj[2][2] = {{cam.focal * (t.distortion + t.normalized[0] * dx), cam.focal * t.normalized[0] * dy},
                     {cam.focal * t.normalized[1] * dx, cam.focal * (t.distortion + t.normalized[1] * dy)}};
  Projection pr;
  for (int r = 0; r < 2; ++r) {
    pr.jacobian[r][0] = nj[r][0] * t.inverse_depth;
    pr.jacobian[r][1] = nj[r][1] * t.inverse_depth;
    pr.jacobian[r][2] = -(nj[r][0] * t.normalized[0] + nj[r][1] * t.normalized[1]) * t.inverse_depth;
  }
  pr.residual = {t.prediction[0] - obs[0], t.prediction[1] - obs[1]};
  if (!projection_finite(pr)) return std::nullopt;
  return pr;
}
// radial_intrinsic_jacobian_from_terms (model.rs:298-315): columns (log f, k1, k2)
inline std::optional<Mat23> radial_intrinsic_jacobian(const Radial& cam, const RadialTerms& t) {
  Mat23 j;
  for (int r = 0; r < 2; ++r) {
    j[r][0] = t.prediction[r];
    j[r][1] = cam.focal * t.r2 * t.normalized[r];
    j[r][2] = cam.focal * t.r4 * t.normalized[r];
  }
  if (!all_finite(&j[0][0], 3) || !all_finite(&j[1][0], 3)) return std::nullopt;
  return j;
}
// radial_bearing (model.rs:171-230): principal-branch inverse, used for invertibility counts
inline bool radial_bearing_ok(const Radial& cam, const Vec2& m) {
  if (!(cam.focal > 0.0 && std::isfinite(cam.focal) && std::isfinite(cam.k1) && std::isfinite(cam.k2))) return false;
  if (!std::isfinite(m[0]) || !std::isfinite(m[1])) return false;
  Vec2 d = {m[0] / cam.focal, m[1] / cam.focal};
  double dr = std::hypot(d[0], d[1]);
  if (!std::isfinite(dr)) return false;
  if (dr == 0.0) return true;
  auto radius_fn = [&](double r) {
    double r2 = r * r;
    return r * (1.0 + cam.k1 * r2 + cam.k2 * r2 * r2);
  };
  auto turn = first_radial_turn_squared(cam.k1, cam.k2);
  double upper;
  if (turn) {
    upper = std::sqrt(*turn);
    double maximum = radius_fn(upper);
    double tol = 64.0 * kEps * (1.0 + std::fabs(maximum));
    if (!std::isfinite(maximum) || dr >= maximum - tol) return false;
  } else {
    upper = std::max(dr, 1.0);
    for (;;) {
      double pr = radius_fn(upper);
      if (!std::isfinite(pr)) return false;
      if (pr >= dr) break;
      upper *= 2.0;
      if (!std::isfinite(upper)) return false;
    }
  }
  double tol = 1e-14 * (1.0 + dr);
  double lower = 0.0, r = std::min(dr, 0.5 * upper);
  for (int i = 0; i < 48; ++i) {
    double v = radius_fn(r) - dr;
    if (std::fabs(v) <= tol) {
      double s = r / dr;
      double b0 = d[0] * s, b1 = d[1] * s;
      double n = std::sqrt(b0 * b0 + b1 * b1 + 1.0);
      return std::isfinite(n) && n > kMinPositive;
    }
    if (v < 0.0)
      lower = r;
    else
      upper = r;
    double r2 = r * r;
    double der = 1.0 + 3.0 * cam.k1 * r2 + 5.0 * cam.k2 * r2 * r2;
    double newton = r - v / der;
    r = (std::isfinite(der) && der > 0.0 && newton > lower && newton < upper) ? newton : 0.5 * (lower + upper);
  }
  return false;
}

// ---------------------------------------------------------------------------------------------
// Manifold maps: numerics/manifold/so3.rs:254-265,420-423; numerics/manifold.rs:118-158.
// ---------------------------------------------------------------------------------------------
inline Mat3 skew(const Vec3& v) { return {{{0.0, -v[2], v[1]}, {v[2], 0.0, -v[0]}, {-v[1], v[0], 0.0}}}; }
inline Mat3 matrix_polynomial(const Vec3& v, double identity, double linear, double quadratic) {
  Mat3 k = skew(v);
  Mat3 k2 = mat_mul(k, k);
  Mat3 out{};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) out[i][j] = (i == j ? identity : 0.0) + k[i][j] * linear + k2[i][j] * quadratic;
  return out;
}
inline Mat3 exp_so3(const Vec3& v) {
  double th2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  double th = std::sqrt(th2);
  if (th < 1e-10) return matrix_polynomial(v, 1.0, 1.0, 0.5);
  Vec3 axis = {v[0] / th, v[1] / th, v[2] / th};
  return matrix_polynomial(axis, 1.0, std::sin(th), 1.0 - std::cos(th));
}
inline Vec3 normalize3(const Vec3& v) {
  double n = norm3(v);
  return {v[0] / n, v[1] / n, v[2] / n};
}
inline Vec3 cross3(const Vec3& a, const Vec3& b) {
  return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
// s2_tangent_basis (manifold.rs:118-131)
inline std::array<Vec3, 2> s2_tangent_basis(const Vec3& t) {
  Vec3 tv = normalize3(t);
  Vec3 ref;
  if (std::fabs(tv[0]) <= std::fabs(tv[1]) && std::fabs(tv[0]) <= std::fabs(tv[2]))
    ref = {1, 0, 0};
  else if (std::fabs(tv[1]) <= std::fabs(tv[2]))
    ref = {0, 1, 0};
  else
    ref = {0, 0, 1};
  Vec3 b0 = normalize3(cross3(tv, ref));
  Vec3 b1 = normalize3(cross3(tv, b0));
  return {b0, b1};
}
// retract_s2 (manifold.rs:133-147)
inline Vec3 retract_s2(const Vec3& t, const std::array<Vec3, 2>& basis, double d0, double d1) {
  Vec3 v = {basis[0][0] * d0 + basis[1][0] * d1, basis[0][1] * d0 + basis[1][1] * d1,
            basis[0][2] * d0 + basis[1][2] * d1};
  double th = norm3(v);
  Vec3 tv = normalize3(t);
  if (th < 1e-10) return normalize3({tv[0] + v[0], tv[1] + v[1], tv[2] + v[2]});
  double c = std::cos(th), s = std::sin(th) / th;
  return {tv[0] * c + v[0] * s, tv[1] * c + v[1] * s, tv[2] * c + v[2] * s};
}

// ---------------------------------------------------------------------------------------------
// Point blocks: kernel/point_block.rs:78-184.
// ---------------------------------------------------------------------------------------------
struct PointBlockFactor {
  double inverse[6];  // packed lower: 00, 10, 11, 20, 21, 22
  Vec3 solve(const Vec3& x) const {
    const double* i = inverse;
    return {i[0] * x[0] + i[1] * x[1] + i[3] * x[2], i[1] * x[0] + i[2] * x[1] + i[4] * x[2],
            i[3] * x[0] + i[4] * x[1] + i[5] * x[2]};
  }
};
inline std::optional<Vec3> damping_diagonal(const Mat3& m) {
  double ds = std::max({0.0, m[0][0], m[1][1], m[2][2]});
  if (!(std::isfinite(ds) && ds > 0.0)) return std::nullopt;
  double floor = 64.0 * kEps * ds;
  return Vec3{std::max(m[0][0], floor), std::max(m[1][1], floor), std::max(m[2][2], floor)};
}
inline std::optional<Mat3> damped_matrix(const Mat3& m, double lambda) {
  auto d = damping_diagonal(m);
  if (!d) return std::nullopt;
  Mat3 out = m;
  for (int c = 0; c < 3; ++c) out[c][c] += lambda * (*d)[c];
  return out;
}
inline std::optional<PointBlockFactor> factor_damped(const Mat3& a) {
  double ds = std::max({0.0, a[0][0], a[1][1], a[2][2]});
  double floor = 64.0 * kEps * ds;
  double sc[3];
  for (int i = 0; i < 3; ++i) sc[i] = std::sqrt(std::max(a[i][i], floor));
  double l[3][3] = {};
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c <= r; ++c) {
      double v = 0.5 * (a[r][c] + a[c][r]) / (sc[r] * sc[c]);
      for (int k = 0; k < c; ++k) v -= l[r][k] * l[c][k];
      if (r == c) {
        if (!(std::isfinite(v) && v > 64.0 * kEps)) return std::nullopt;
        l[r][c] = std::sqrt(v);
      } else {
        l[r][c] = v / l[c][c];
      }
    }
  double m00 = 1.0 / l[0][0], m11 = 1.0 / l[1][1], m22 = 1.0 / l[2][2];
  double m10 = -l[1][0] * m00 * m11;
  double m21 = -l[2][1] * m11 * m22;
  double m20 = -(l[2][0] * m00 + l[2][1] * m10) * m22;
  double d0 = 1.0 / sc[0], d1 = 1.0 / sc[1], d2 = 1.0 / sc[2];
  PointBlockFactor f;
  f.inverse[0] = (m00 * m00 + m10 * m10 + m20 * m20) * (d0 * d0);
  f.inverse[1] = (m11 * m10 + m21 * m20) * (d1 * d0);
  f.inverse[2] = (m11 * m11 + m21 * m21) * (d1 * d1);
  f.inverse[3] = (m22 * m20) * (d2 * d0);
  f.inverse[4] = (m22 * m21) * (d2 * d1);
  f.inverse[5] = (m22 * m22) * (d2 * d2);
  return f;
}
inline std::optional<PointBlockFactor> point_block_factor(const Mat3& m, double lambda) {
  auto d = damped_matrix(m, lambda);
  if (!d) return std::nullopt;
  return factor_damped(*d);
}
// reciprocal_condition_number (point_block.rs:163-184), infinity norms
inline double point_rcond(const PointBlockFactor& f, const Mat3& m) {
  Mat3 inv;
  for (int c = 0; c < 3; ++c) {
    Vec3 e = {0, 0, 0};
    e[c] = 1.0;
    Vec3 col = f.solve(e);
    for (int r = 0; r < 3; ++r) inv[r][c] = col[r];
  }
  auto inf_norm = [](const Mat3& a) {
    double best = 0.0;
    for (int r = 0; r < 3; ++r) best = std::max(best, std::fabs(a[r][0]) + std::fabs(a[r][1]) + std::fabs(a[r][2]));
    return best;
  };
  double den = inf_norm(m) * inf_norm(inv);
  return (std::isfinite(den) && den > 0.0) ? 1.0 / den : 0.0;
}
// ---------------------------------------------------------------------------------------------
// Angular residuals: kernel/projection.rs:89-195.
// ---------------------------------------------------------------------------------------------
inline double odot(const Vec3& a, const Vec3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline Vec3 ocross(const Vec3& a, const Vec3& b) {
  return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
// normalize (projection.rs:156-169)
inline std::optional<Vec3> unit_or_none(const Vec3& v) {
  const double n2 = odot(v, v);
  if (!all_finite(v.data(), 3) || !(std::isfinite(n2) && n2 > kMinPositive)) return std::nullopt;
  if (std::fabs(n2 - 1.0) <= 8.0 * kEps) return v;
  const double inv = 1.0 / std::sqrt(n2);
  return Vec3{v[0] * inv, v[1] * inv, v[2] * inv};
}
// tangent_basis (projection.rs:171-186)
inline std::array<Vec3, 2> angular_tangent_basis(const Vec3& u) {
  Vec3 ref{0.0, 0.0, 0.0};
  if (std::fabs(u[0]) <= std::fabs(u[1]) && std::fabs(u[0]) <= std::fabs(u[2]))
    ref[0] = 1.0;
  else if (std::fabs(u[1]) <= std::fabs(u[2]))
    ref[1] = 1.0;
  else
    ref[2] = 1.0;
  Vec3 first = ocross(u, ref);
  const double inv = 1.0 / std::sqrt(odot(first, first));
  for (double& x : first) x *= inv;
  return {first, ocross(u, first)};
}
// angular_projection (projection.rs:89-149)
inline std::optional<Projection> angular_projection(const Vec3& raw_obs, const Vec3& point) {
  auto obs = unit_or_none(raw_obs);
  auto pred = unit_or_none(point);
  if (!obs || !pred) return std::nullopt;
  const auto basis = angular_tangent_basis(*obs);
  const double a = odot(basis[0], *pred), b = odot(basis[1], *pred), c = odot(*obs, *pred);
  const double s2 = a * a + b * b, s = std::sqrt(s2);
  if (c < 0.0 && s < 1e-6) return std::nullopt;
  double factor, fscale = 0.0;
  if (s < 1e-6) {
    const double s4 = s2 * s2;
    factor = 1.0 + s2 / 6.0 + 3.0 * s4 / 40.0;
    fscale = 1.0 / 3.0 + 3.0 * s2 / 10.0;
  } else {
    factor = std::atan2(s, c) / s;
  }
  double dp[2][3];
  for (int k = 0; k < 3; ++k) {
    const double da = basis[0][k], db = basis[1][k], dc = (*obs)[k];
    double fd;
    if (s < 1e-6) {
      fd = fscale * (a * da + b * db);
    } else {
      const double ds = (a * da + b * db) / s;
      const double angle = std::atan2(s, c);
      const double ad = (c * ds - s * dc) / (s2 + c * c);
      fd = (ad * s - angle * ds) / s2;
    }
    dp[0][k] = factor * da + a * fd;
    dp[1][k] = factor * db + b * fd;
  }
  const double pn = std::sqrt(odot(point, point));
  Projection pr;
  for (int row = 0; row < 2; ++row)
    for (int col = 0; col < 3; ++col) {
      double acc = 0.0;
      for (int k = 0; k < 3; ++k) acc += dp[row][k] * (((col == k) ? 1.0 : 0.0) - (*pred)[col] * (*pred)[k]) / pn;
      pr.jacobian[row][col] = acc;
    }
  pr.residual = {factor * a, factor * b};
  if (!projection_finite(pr)) return std::nullopt;
  return pr;
}

constexpr double kPointBlockRcondThreshold = 64.0 * kEps * 3.0;  // point_block.rs:10
constexpr double kPointBlockQuarantineRcond = 1.0e-5;             // point_block.rs:20

// ---------------------------------------------------------------------------------------------
// Track geometry admission: kernel/point_geometry.rs:16-130.
// ---------------------------------------------------------------------------------------------
constexpr double kMinNearFarRatio = 1e-4;
constexpr double kMinParallaxSine = 1.7e-5;
struct TrackGeometry {
  double near2 = kInf, far2, scene2;
  bool has_first = false;
  Vec3 first{};
  bool parallax = false;
  int observations = 0;
  bool invalid = false;
  explicit TrackGeometry(double scene) : far2(scene * scene), scene2(scene * scene) {}
  void push(const Vec3& off) {
    double sq = off[0] * off[0] + off[1] * off[1] + off[2] * off[2];
    if (!(std::isfinite(sq) && sq > 0.0)) {
      invalid = true;
      return;
    }
    observations++;
    near2 = std::min(near2, sq);
    far2 = std::max(far2, sq);
    double inv = 1.0 / std::sqrt(sq);
    Vec3 ray = {off[0] * inv, off[1] * inv, off[2] * inv};
    if (!has_first) {
      has_first = true;
      first = ray;
      return;
    }
    if (parallax) return;
    double d = dot3(ray, first);
    Vec3 c = cross3(ray, first);
    double s2 = dot3(c, c);
    parallax = d < 0.0 || s2 >= kMinParallaxSine * kMinParallaxSine;
  }
  bool degenerate() const {
    return invalid || (observations >= 2 && (!parallax || near2 < kMinNearFarRatio * kMinNearFarRatio * far2));
  }
  bool collapsed() const {
    return invalid || (observations >= 2 && near2 < kMinNearFarRatio * kMinNearFarRatio * scene2);
  }
};
enum class Admission { Projection, Collapse, Geometry };
inline bool admits(Admission a, const TrackGeometry& g) {
  switch (a) {
    case Admission::Projection: return true;
    case Admission::Collapse: return !g.collapsed();
    case Admission::Geometry: return !g.degenerate();
  }
  return false;
}

// ---------------------------------------------------------------------------------------------
// Nielsen damping and LM run state: numerics/refine/nonlinear/{controller,run_state,continuation}.rs
// ---------------------------------------------------------------------------------------------
struct Nielsen {
  double value, nu = 2.0;
  bool has_gain = false;
  double gain = 0.0;
  explicit Nielsen(double v = 1e-4) : value(v) {}
  void increase() {
    value = std::min(value * nu, 1e12);
    nu = std::min(nu * 2.0, 1e12);
  }
  void reject() {
    has_gain = false;
    increase();
  }
  bool accept(double actual, double predicted) {
    double g = (std::isfinite(actual) && std::isfinite(predicted) && predicted > 0.0) ? actual / predicted
                                                                                      : std::nan("");
    has_gain = std::isfinite(g);
    gain = g;
    if (!(std::isfinite(g) && g > 0.0)) {
      increase();
      return false;
    }
    double c = 2.0 * g - 1.0;
    double factor = std::max(1.0 - c * c * c, 1.0 / 3.0);
    value = std::max(value * factor, 1e-12);
    nu = 2.0;
    return true;
  }
};
enum class Criterion { None = -1, Cost = 0, Gradient = 1, Step = 2 };
struct Criteria {
  double gradient, step, relative_cost;
};
struct RunState {
  Nielsen damping;
  uint64_t iterations = 0, accepted = 0, target_accepted = 0;
  uint64_t rej_lin = 0, rej_solve = 0, rej_cand = 0, rej_insuff = 0;
  double step_norm = 0.0;
  Criterion convergence = Criterion::None;
  explicit RunState(double initial) : damping(initial) {}
  uint64_t rejected() const { return rej_lin + rej_solve + rej_cand + rej_insuff; }
  bool accept_gain(double a, double p) {
    if (damping.accept(a, p)) return true;
    rej_insuff++;
    return false;
  }
  bool gradient_converged(double g, double cost, const Criteria& c) {
    if (convergence == Criterion::None && std::isfinite(g) && g >= 0.0 && std::isfinite(cost) &&
        g <= c.gradient * (1.0 + std::fabs(cost))) {
      convergence = Criterion::Gradient;
      return true;
    }
    return false;
  }
  Criterion record_accepted(double sn, double reduction, double prev, bool target, const Criteria& c) {
    accepted++;
    step_norm = sn;
    if (!target) return Criterion::None;
    target_accepted++;
    double rel = reduction / (1.0 + std::fabs(prev));
    if (sn <= c.step) return Criterion::Step;
    if (rel <= c.relative_cost) return Criterion::Cost;
    return Criterion::None;
  }
  bool certify(Criterion c) {
    convergence = c;
    return c != Criterion::None;
  }
  // status (run_state.rs:170-181): 0 converged, 1 max, 2 stalled, 3 degenerate
  int status(bool well_constrained) const {
    if (!well_constrained) return 3;
    if (convergence != Criterion::None) return 0;
    if (iterations > 0 && target_accepted == 0) return 2;
    return 1;
  }
};
struct Stage {
  Loss loss;
  uint64_t max_iterations;
};
// stages (continuation.rs:18-74)
inline std::array<Stage, 3> stages(const Loss& loss, uint64_t max_iterations) {
  Loss l2{};
  if (loss.kind == LossKind::Cauchy) {
    uint64_t w = std::min<uint64_t>(max_iterations / 4, 5);
    return {Stage{l2, w}, Stage{loss, max_iterations - w}, Stage{l2, 0}};
  }
  return {Stage{loss, max_iterations}, Stage{l2, 0}, Stage{l2, 0}};
}
inline int final_stage_index(const std::array<Stage, 3>& s) {
  for (int i = 2; i >= 0; --i)
    if (s[i].max_iterations > 0) return i;
  return 0;
}

}  // namespace oracle
