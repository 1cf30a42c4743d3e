// camera_models.cuh — openmvg-core's camera models as the SfM side evaluates them, host and device.
//
// The bundle adjustment itself projects through its own admissibility rules (ba_device.cuh); the
// steps either side of it in openmvg-sfm measure observations with the camera model's plain
// projection and unprojection (camera/camera_model.rs, camera_enum.rs). These are restated here for
// the four models of the C ABI: pinhole, Brown-Conrady, fisheye and spherical.
#pragma once

#include "ba_cuda.h"
#include "ba_device.cuh"

namespace omvgba {

constexpr double kPi = 3.141592653589793;
constexpr double kFisheyeMaxIncidentAngle = kPi - 1e-10;  // camera/fisheye.rs:32

// FisheyeDistortion (camera/distortion.rs:244-460): theta_d = theta (1 + k1 t^2 + k2 t^4 + k3 t^6 + k4 t^8)
struct FisheyePoly {
  int kind;  // 0 None .. 4 K1K2K3K4
  double k1, k2, k3, k4;
  BA_HD double apply(double t) const {
    const double t2 = t * t, t4 = t2 * t2;
    switch (kind) {
      case 0: return t;
      case 1: return t * (1.0 + k1 * t2);
      case 2: return t * (1.0 + k1 * t2 + k2 * t4);
      case 3: return t * (1.0 + k1 * t2 + k2 * t4 + k3 * (t4 * t2));
      default: return t * (1.0 + k1 * t2 + k2 * t4 + k3 * (t4 * t2) + k4 * (t4 * t4));
    }
  }
  BA_HD double derivative(double t) const {
    const double t2 = t * t, t4 = t2 * t2, t6 = t4 * t2, t8 = t4 * t4;
    return 1.0 + 3.0 * k1 * t2 + 5.0 * k2 * t4 + 7.0 * k3 * t6 + 9.0 * k4 * t8;
  }
  // max_invertible_angle (distortion.rs:416-455)
  BA_HD bool max_invertible_angle(double max_theta, double* out) const {
    if (!(isfinite(k1) && isfinite(k2) && isfinite(k3) && isfinite(k4))) return false;
    if (k3 == 0.0 && k4 == 0.0) {
      double q;
      *out = first_radial_turn_squared(k1, k2, &q) ? fmin(sqrt(q), max_theta) : max_theta;
      return true;
    }
    if (k1 >= 0.0 && k2 >= 0.0 && k3 >= 0.0 && k4 >= 0.0) {
      *out = max_theta;
      return true;
    }
    double previous = 0.0;
    for (int i = 1; i <= 1024; ++i) {
      const double t = max_theta * i / 1024.0;
      if (derivative(t) <= 0.0) {
        double lo = previous, hi = t;
        for (int k = 0; k < 64; ++k) {
          const double mid = 0.5 * (lo + hi);
          if (derivative(mid) > 0.0)
            lo = mid;
          else
            hi = mid;
        }
        *out = lo;
        return true;
      }
      previous = t;
    }
    *out = max_theta;
    return true;
  }
  // invert_on_validated_interval (distortion.rs:359-409)
  BA_HD bool invert(double td, double upper, double* out) const {
    if (!isfinite(td) || !isfinite(upper) || td < 0.0 || upper <= 0.0) return false;
    const double mapped = apply(upper);
    if (!isfinite(mapped) || td > mapped + 1e-12) return false;
    double lo = 0.0, hi = upper, t = fmin(td, upper);
    for (int i = 0; i < 48; ++i) {
      const double r = apply(t) - td;
      if (fabs(r) <= 1e-13) {
        *out = t;
        return true;
      }
      if (r < 0.0)
        lo = t;
      else
        hi = t;
      const double d = derivative(t), nt = t - r / d;
      t = (isfinite(d) && d > 1e-15 && nt > lo && nt < hi) ? nt : 0.5 * (lo + hi);
    }
    if (fabs(apply(t) - td) <= 1e-12) {
      *out = t;
      return true;
    }
    return false;
  }
};

// try_normalize_bearing (camera/camera_model.rs:91-109)
BA_HD bool normalize_bearing(const double d[3], double b[3]) {
  if (!finite3(d[0], d[1], d[2])) return false;
  const double s = fmax(fmax(fabs(d[0]), fabs(d[1])), fabs(d[2]));
  if (s == 0.0) return false;
  const double x[3] = {d[0] / s, d[1] / s, d[2] / s};
  const double n = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  if (!isfinite(n) || n == 0.0) return false;
  for (int k = 0; k < 3; ++k) b[k] = x[k] / n;
  return true;
}

// One camera of the C ABI in the form the kernels read (built on the host by make_camera_dev).
struct CameraDev {
  int32_t model;        // OMVGBA_CAMERA_*
  uint32_t width;       // spherical image width (its height is width / 2)
  FixedCameraDev pin;   // pinhole part, with the Brown-Conrady distortion when the model has it
  FisheyePoly fish;     // fisheye polynomial
  double max_angle;     // fisheye: largest incident angle the polynomial inverts
  int32_t fish_ok;      // fisheye: the invertible angle exists
};

// Camera::project (camera_enum.rs): pinhole (pinhole.rs:276-298) and Brown-Conrady
// (brown_conrady.rs:310-332) reject points at or behind the camera and outside the distortion's
// forward domain; fisheye (fisheye.rs:182-210) rejects incident angles past the invertible range;
// spherical (spherical.rs:147-209) accepts every finite direction.
BA_HD bool camera_project(const CameraDev& c, const double X[3], double* u, double* v) {
  if (c.model == OMVGBA_CAMERA_PINHOLE || c.model == OMVGBA_CAMERA_BROWN_CONRADY)
    return c.pin.project(X[0], X[1], X[2], u, v);
  double d[3];
  if (!normalize_bearing(X, d)) return false;
  if (c.model == OMVGBA_CAMERA_FISHEYE) {
    if (!c.fish_ok) return false;
    const double radial = hypot(d[0], d[1]);
    if (radial == 0.0) {
      if (!(d[2] > 0.0)) return false;
      *u = c.pin.cx;
      *v = c.pin.cy;
      return true;
    }
    const double theta = atan2(radial, d[2]);
    if (theta > c.max_angle + 1e-12) return false;
    const double scale = c.fish.apply(theta) / radial;
    *u = fma(c.pin.fx, d[0] * scale, c.pin.cx);
    *v = fma(c.pin.fy, d[1] * scale, c.pin.cy);
    return isfinite(*u) && isfinite(*v);
  }
  if (c.model == OMVGBA_CAMERA_SPHERICAL) {
    const double lon = atan2(d[0], d[2]), lat = atan2(d[1], hypot(d[0], d[2]));
    const double w = (double)c.width, h = (double)(c.width / 2);
    double x = fmod((lon + kPi) * w / (2.0 * kPi), w);
    if (x < 0.0) x += w;
    *u = x - 0.5;
    *v = (lat + kPi / 2.0) * h / kPi - 0.5;
    return true;
  }
  return false;
}

// The unit bearing of pixel (u, v): CameraModel::unproject of the pinhole (pinhole.rs:324-340),
// Brown-Conrady (brown_conrady.rs:365-383), fisheye (fisheye.rs:271-299) and spherical
// (spherical.rs:113-257) models, then normalized.
BA_HD bool camera_unproject_bearing(const CameraDev& c, double u, double v, double b[3]) {
  if (!isfinite(u) || !isfinite(v)) return false;
  double d[3];
  switch (c.model) {
    case OMVGBA_CAMERA_PINHOLE:
    case OMVGBA_CAMERA_BROWN_CONRADY: {
      d[0] = (u - c.pin.cx) / c.pin.fx;
      d[1] = (v - c.pin.cy) / c.pin.fy;
      d[2] = 1.0;
      if (!finite3(d[0], d[1], d[2])) return false;
      if (c.model == OMVGBA_CAMERA_BROWN_CONRADY) {
        double x, y;
        if (!c.pin.remove_distortion(d[0], d[1], &x, &y)) return false;
        d[0] = x;
        d[1] = y;
      }
      break;
    }
    case OMVGBA_CAMERA_FISHEYE: {
      const double xd = (u - c.pin.cx) / c.pin.fx, yd = (v - c.pin.cy) / c.pin.fy;
      if (!isfinite(xd) || !isfinite(yd)) return false;
      const double td = hypot(xd, yd);
      if (td <= kEps) {
        d[0] = 0.0;
        d[1] = 0.0;
        d[2] = 1.0;
        break;
      }
      double theta;
      if (!c.fish_ok || !c.fish.invert(td, c.max_angle, &theta)) return false;
      const double sc = sin(theta) / td;
      d[0] = xd * sc;
      d[1] = yd * sc;
      d[2] = cos(theta);
      if (!finite3(d[0], d[1], d[2])) return false;
      break;
    }
    case OMVGBA_CAMERA_SPHERICAL: {
      const double w = (double)c.width, h = (double)(c.width / 2);
      if (v < -0.5 || v > h - 0.5) return false;
      double x = fmod(u + 0.5, w);
      if (x < 0.0) x += w;
      x -= 0.5;
      const double lon = (x + 0.5) * (2.0 * kPi) / w - kPi, lat = (v + 0.5) * kPi / h - kPi / 2.0;
      if (!isfinite(lon) || !isfinite(lat) || lat < -kPi / 2.0 || lat > kPi / 2.0) return false;
      const double cl = cos(lat);
      d[0] = cl * sin(lon);
      d[1] = sin(lat);
      d[2] = cl * cos(lon);
      break;
    }
    default:
      return false;
  }
  return normalize_bearing(d, b);
}

// nominal_pixels_per_radian (openmvg-sfm ops/reconstruction/residual.rs:96-115): the spherical image's
// width over a full turn, else the smaller focal length; NaN when not finite and positive.
BA_HD double camera_pixels_per_radian(const CameraDev& c) {
  const double s = c.model == OMVGBA_CAMERA_SPHERICAL ? (double)c.width / (2.0 * kPi)
                                                       : fmin(fabs(c.pin.fx), fabs(c.pin.fy));
  return (isfinite(s) && s > 0.0) ? s : NAN;
}

BA_HD bool camera_is_generalized(const CameraDev& c) {  // is_generalized_camera (residual.rs:149-151)
  return c.model == OMVGBA_CAMERA_FISHEYE || c.model == OMVGBA_CAMERA_SPHERICAL;
}

// The pixel-equivalent residual of CameraResidualPolicy::evaluate with an unbounded limit
// (openmvg-sfm ops/reconstruction/residual.rs:57-90): perspective cameras the pixel distance of the
// projection (camera_pixel_residual, :117-138); fisheye and spherical cameras the bearing angle
// 2 asin(|b_predicted - b_observed| / 2) (Camera::bearing_error_rad, camera_model.rs:238-269) times
// the nominal pixels per radian. False when the camera point or the pixel is outside the model's
// domain or the value is not finite.
BA_HD bool camera_pixel_equivalent(const CameraDev& c, const double Xc[3], double u, double v, double* out) {
  double pu, pv;
  if (!camera_project(c, Xc, &pu, &pv)) return false;
  double r;
  if (!camera_is_generalized(c)) {
    if (!isfinite(pu) || !isfinite(pv) || !isfinite(u) || !isfinite(v)) {
      r = INFINITY;
    } else {
      r = hypot(pu - u, pv - v);
    }
  } else {
    double bo[3], bp[3];
    if (!camera_unproject_bearing(c, u, v, bo) || !normalize_bearing(Xc, bp)) return false;
    const double e0 = bp[0] - bo[0], e1 = bp[1] - bo[1], e2 = bp[2] - bo[2];
    double chord2 = e0 * e0 + e1 * e1 + e2 * e2;
    if (!isfinite(chord2)) return false;
    chord2 = fmin(fmax(chord2, 0.0), 4.0);
    const double angle = 2.0 * asin(fmin(fmax(0.5 * sqrt(chord2), 0.0), 1.0));
    r = angle * camera_pixels_per_radian(c);
  }
  if (!isfinite(r)) return false;
  *out = r;
  return true;
}

// Host-side construction from the C ABI's intrinsic record.
inline FixedCameraDev make_fixed_camera(const omvgba_intrinsic& in) {
  FixedCameraDev m{};
  m.fx = in.fx;
  m.fy = in.fy;
  m.cx = in.cx;
  m.cy = in.cy;
  if (in.model == OMVGBA_CAMERA_BROWN_CONRADY) {
    m.radial_kind = in.radial_kind;
    m.tangential_kind = in.tangential_kind;
    m.k1 = in.radial_kind >= 1 ? in.k1 : 0.0;
    m.k2 = in.radial_kind >= 2 ? in.k2 : 0.0;
    m.k3 = in.radial_kind >= 3 ? in.k3 : 0.0;
    m.p1 = in.tangential_kind >= 1 ? in.p1 : 0.0;
    m.p2 = in.tangential_kind >= 2 ? in.p2 : 0.0;
    double t;
    m.has_turn = first_radial_turn_squared(m.k1, m.k2, &t) ? 1 : 0;
    m.turn_squared = m.has_turn ? t : INFINITY;
  } else {
    m.radial_kind = 0;
    m.tangential_kind = 0;
    m.has_turn = 0;
    m.turn_squared = INFINITY;
  }
  return m;
}

inline FisheyePoly make_fisheye_poly(const omvgba_intrinsic& in) {
  return FisheyePoly{in.radial_kind, in.radial_kind >= 1 ? in.k1 : 0.0, in.radial_kind >= 2 ? in.k2 : 0.0,
                     in.radial_kind >= 3 ? in.k3 : 0.0, in.radial_kind >= 4 ? in.k4 : 0.0};
}

inline CameraDev make_camera_dev(const omvgba_intrinsic& in) {
  CameraDev c{};
  c.model = in.model;
  c.width = in.width;
  c.pin = make_fixed_camera(in);
  if (in.model == OMVGBA_CAMERA_FISHEYE) {
    c.fish = make_fisheye_poly(in);
    c.fish_ok = c.fish.max_invertible_angle(kFisheyeMaxIncidentAngle, &c.max_angle) ? 1 : 0;
  }
  return c;
}

}  // namespace omvgba
