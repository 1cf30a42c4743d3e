// host.cpp — C ABI (include/ba_cuda.h) of the B200 bundle-adjustment solver: problem validation,
// native lowering, quarantine re-solves, report and Solution construction around the GPU LM loop.
//
// Reference (paths relative to the openmvg-rs root):
//   NativeBundleAdjuster::solve ...... native/mod.rs:235-367 (routing, quarantine)
//   problem / config checks .......... problem.rs:492-577, solver.rs:122-141
//   gauge plans ...................... native/gauge.rs:9-330
//   world rebase ..................... native/world_rebase.rs:19-87
//   calibrated lowering .............. native/calibrated.rs:200-460
//   self-calibrating lowering ........ native/self_calibration.rs:47-198, 442-512
//   report mapping ................... native/reporting.rs:24-141
//   Solution metrics ................. solver.rs:803-1131; weak points solver.rs:1149-1226
//   quarantine ....................... quarantine.rs:34-96
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ba_cuda.h"
#include "camera_models.cuh"
#include "gpu_solver.hpp"
#include "fixed_rotation.hpp"

namespace omvgba {
namespace {

using Mat3 = std::array<std::array<double, 3>, 3>;
using Vec3 = std::array<double, 3>;

[[noreturn]] void fail(int code, const std::string& msg) { throw SolveFailure{code, msg}; }

Mat3 pose_R(const omvgba_pose& p) {
  Mat3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r[i][j] = p.rotation[i * 3 + j];
  return r;
}
Vec3 pose_C(const omvgba_pose& p) { return {p.center[0], p.center[1], p.center[2]}; }
Vec3 point_at(const omvgba_problem& pr, size_t i) { return {pr.points[3 * i], pr.points[3 * i + 1], pr.points[3 * i + 2]}; }
bool point_fixed(const omvgba_problem& pr, size_t i) { return pr.point_fixed && pr.point_fixed[i]; }
bool all_finite(const double* v, int n) {
  for (int i = 0; i < n; ++i)
    if (!std::isfinite(v[i])) return false;
  return true;
}
Mat3 mat_mul(const Mat3& a, const Mat3& b) {
  Mat3 c{};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) c[i][j] += a[i][k] * b[k][j];
  return c;
}
Vec3 rotate(const Mat3& r, const Vec3& x) {
  return {r[0][0] * x[0] + r[0][1] * x[1] + r[0][2] * x[2], r[1][0] * x[0] + r[1][1] * x[1] + r[1][2] * x[2],
          r[2][0] * x[0] + r[2][1] * x[1] + r[2][2] * x[2]};
}
Vec3 rotate_t(const Mat3& r, const Vec3& v) {
  return {r[0][0] * v[0] + r[1][0] * v[1] + r[2][0] * v[2], r[0][1] * v[0] + r[1][1] * v[1] + r[2][1] * v[2],
          r[0][2] * v[0] + r[1][2] * v[1] + r[2][2] * v[2]};
}
double sqdist(const Vec3& a, const Vec3& b) {
  double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
  return dx * dx + dy * dy + dz * dz;
}


LossDev problem_loss(const omvgba_problem& pr) {
  if (pr.loss_kind == OMVGBA_LOSS_HUBER) return {kLossHuber, pr.loss_scale};
  if (pr.loss_kind == OMVGBA_LOSS_CAUCHY) return {kLossCauchy, pr.loss_scale / std::sqrt(2.0)};
  return {kLossL2, 0.0};
}

// Runs body(chunk, begin, end) over `count` items cut into a fixed number of contiguous chunks, on
// up to host_thread_limit() threads. Callers combine per-chunk results in chunk order, so every
// result is independent of the thread count.
template <typename Body>
void for_fixed_chunks(size_t count, size_t chunks, Body body) {
  const size_t per = (count + chunks - 1) / std::max<size_t>(chunks, 1);
  const unsigned hw = host_thread_limit();
  const size_t nthreads = std::min<size_t>(std::min<size_t>(hw, chunks), count / 65536 + 1);
  std::atomic<size_t> next{0};
  auto worker = [&]() {
    for (size_t c; (c = next.fetch_add(1)) < chunks;) {
      const size_t b = std::min(count, c * per), e = std::min(count, b + per);
      body(c, b, e);
    }
  };
  std::vector<std::thread> pool;
  for (size_t i = 1; i < nthreads; ++i) pool.emplace_back(worker);
  worker();
  for (auto& t : pool) t.join();
}

// ---- validation ----------------------------------------------------------------------------
void validate_problem(const omvgba_problem& pr) {
  if (pr.pose_count == 0) fail(OMVGBA_INVALID_PROBLEM, "bundle adjustment requires at least one pose");
  if (pr.intrinsic_count == 0) fail(OMVGBA_INVALID_PROBLEM, "bundle adjustment requires at least one intrinsic");
  if (pr.point_count == 0) fail(OMVGBA_INVALID_PROBLEM, "bundle adjustment requires at least one point");
  if (pr.observation_count == 0) fail(OMVGBA_INVALID_PROBLEM, "bundle adjustment requires at least one observation");
  if (!pr.poses || !pr.intrinsics || !pr.points || !pr.observation_pose || !pr.observation_intrinsic ||
      !pr.observation_point || !pr.observation_pixel)
    fail(OMVGBA_INVALID_ARGUMENT, "problem arrays must not be null");
  for (size_t i = 0; i < pr.pose_count; ++i) {
    Mat3 R = pose_R(pr.poses[i]);
    bool ok = all_finite(pr.poses[i].rotation, 9) && all_finite(pr.poses[i].center, 3);
    for (int a = 0; a < 3 && ok; ++a)
      for (int b = 0; b < 3; ++b) {
        double s = R[0][a] * R[0][b] + R[1][a] * R[1][b] + R[2][a] * R[2][b];
        if (std::fabs(s - (a == b ? 1.0 : 0.0)) > 9.5367431640625e-7) ok = false;
      }
    double det = R[0][0] * (R[1][1] * R[2][2] - R[1][2] * R[2][1]) - R[0][1] * (R[1][0] * R[2][2] - R[1][2] * R[2][0]) +
                 R[0][2] * (R[1][0] * R[2][1] - R[1][1] * R[2][0]);
    if (!ok || !(det > 0.0)) fail(OMVGBA_INVALID_PROBLEM, "pose " + std::to_string(i) + " is not a valid rigid transform");
  }
  for (size_t i = 0; i < pr.intrinsic_count; ++i)
    if (pr.intrinsics[i].fixed_model && pr.intrinsics[i].variables != 0)
      fail(OMVGBA_INVALID_PROBLEM, "a fixed intrinsic cannot expose variable coordinates");
  for (size_t i = 0; i < pr.point_count; ++i)
    if (!all_finite(pr.points + 3 * i, 3)) fail(OMVGBA_INVALID_PROBLEM, "point coordinates must be finite");
  for (size_t o = 0; o < pr.observation_count; ++o) {
    if (!all_finite(pr.observation_pixel + 2 * o, 2)) fail(OMVGBA_INVALID_PROBLEM, "observation pixels must be finite");
    if (pr.observation_pose[o] >= pr.pose_count)
      fail(OMVGBA_INVALID_PROBLEM, "observation " + std::to_string(o) + " references pose out of bounds");
    if (pr.observation_point[o] >= pr.point_count)
      fail(OMVGBA_INVALID_PROBLEM, "observation " + std::to_string(o) + " references point out of bounds");
    if (pr.observation_intrinsic[o] >= pr.intrinsic_count)
      fail(OMVGBA_INVALID_PROBLEM, "observation " + std::to_string(o) + " references intrinsic out of bounds");
  }
  if (pr.loss_kind != OMVGBA_LOSS_SQUARED && pr.loss_scale_space != pr.residual_space)
    fail(OMVGBA_INVALID_PROBLEM, "robust-loss scale units do not match the problem residual space");
  if (pr.gauge_kind == OMVGBA_GAUGE_FIXED_BASELINE) {
    if (pr.gauge_first >= pr.pose_count || pr.gauge_second >= pr.pose_count)
      fail(OMVGBA_INVALID_PROBLEM, "fixed-baseline gauge references an out-of-range pose");
    if (pr.gauge_first == pr.gauge_second) fail(OMVGBA_INVALID_PROBLEM, "fixed-baseline gauge requires two distinct poses");
    if (!std::isfinite(pr.gauge_distance) || pr.gauge_distance <= 0.0)
      fail(OMVGBA_INVALID_PROBLEM, "fixed-baseline distance must be finite and positive");
  }
}

void validate_config(const omvgba_config& c) {
  if (c.max_iterations == 0) fail(OMVGBA_INVALID_CONFIG, "max_iterations must be positive");
  const char* names[3] = {"function_tolerance", "gradient_tolerance", "parameter_tolerance"};
  double vals[3] = {c.function_tolerance, c.gradient_tolerance, c.parameter_tolerance};
  for (int i = 0; i < 3; ++i)
    if (!std::isfinite(vals[i]) || vals[i] <= 0.0) fail(OMVGBA_INVALID_CONFIG, names[i]);
  if (c.has_workspace_budget && c.workspace_budget_bytes == 0)
    fail(OMVGBA_INVALID_CONFIG, "workspace_budget_bytes must be positive");
  if (c.precision != OMVGBA_PRECISION_FP64 && c.precision != OMVGBA_PRECISION_MIXED)
    fail(OMVGBA_INVALID_CONFIG, "precision must be FP64 or MIXED");
}

// ---- gauge plans ---------------------------------------------------------------------------
std::vector<uint8_t> observed_cameras(const omvgba_problem& pr) {
  std::vector<uint8_t> o(pr.pose_count, 0);
  for (size_t i = 0; i < pr.observation_count; ++i) o[pr.observation_pose[i]] = 1;
  return o;
}
int farthest_camera(const std::vector<std::pair<int, double>>& cands) {
  int best = -1;
  double bs = 0.0;
  for (auto& c : cands) {
    if (!std::isfinite(c.second)) continue;
    if (best < 0 || c.second > bs || (c.second == bs && c.first < best)) {
      best = c.first;
      bs = c.second;
    }
  }
  return (best >= 0 && bs > 0.0) ? best : -1;
}

struct GaugePlan {
  size_t anchor = 0;
  double scale = 1.0;
  int native_cam = -1;
  std::vector<uint32_t> masks;
};

GaugePlan gauge_plan(const omvgba_problem& pr) {
  auto observed = observed_cameras(pr);
  bool controls = false;
  for (size_t o = 0; o < pr.observation_count; ++o) controls = controls || point_fixed(pr, pr.observation_point[o]);
  if (pr.gauge_kind == OMVGBA_GAUGE_FREE && controls) {
    bool any = false;
    for (size_t i = 0; i < pr.pose_count; ++i) any = any || (observed[i] && pr.poses[i].variables == 0);
    if (!any)
      fail(OMVGBA_UNSUPPORTED,
           "native BA with fixed world points requires an explicitly fixed observed pose or fixed-baseline anchor");
  }
  GaugePlan plan;
  for (size_t i = 0; i < pr.pose_count; ++i) plan.masks.push_back(pr.poses[i].variables);
  if (pr.gauge_kind == OMVGBA_GAUGE_FREE) {
    size_t anchor = SIZE_MAX, first = SIZE_MAX;
    for (size_t i = 0; i < pr.pose_count; ++i) {
      if (observed[i] && pr.poses[i].variables == 0) {
        anchor = i;
        break;
      }
      if (observed[i] && first == SIZE_MAX) first = i;
    }
    if (anchor == SIZE_MAX) anchor = first == SIZE_MAX ? 0 : first;
    Vec3 ac = pose_C(pr.poses[anchor]);
    bool sets = false;
    for (size_t i = 0; i < pr.pose_count; ++i)
      sets = sets || (i != anchor && observed[i] && pr.poses[i].variables == 0 && sqdist(pose_C(pr.poses[i]), ac) > 0.0);
    for (size_t o = 0; o < pr.observation_count; ++o) {
      size_t p = pr.observation_point[o];
      sets = sets || (point_fixed(pr, p) && sqdist(point_at(pr, p), ac) > 0.0);
    }
    plan.anchor = anchor;
    if (!sets) {
      std::vector<std::pair<int, double>> c;
      for (size_t i = 0; i < pr.pose_count; ++i)
        if (i != anchor && observed[i] && pr.poses[i].variables != 0) c.push_back({(int)i, sqdist(pose_C(pr.poses[i]), ac)});
      int cam = farthest_camera(c);
      if (cam < 0) fail(OMVGBA_UNSUPPORTED, "free-scale BA has no nonzero active baseline");
      plan.native_cam = cam;
    }
    return plan;
  }
  Vec3 c1 = pose_C(pr.poses[pr.gauge_first]), c2 = pose_C(pr.poses[pr.gauge_second]);
  double current = std::sqrt(sqdist(c2, c1));
  if (!std::isfinite(current) || current <= 0.0) fail(OMVGBA_UNSUPPORTED, "fixed-baseline cameras have no usable separation");
  double raw = pr.gauge_distance / current;
  double tol = 256.0 * kEps * std::max({std::fabs(current), std::fabs(pr.gauge_distance), 1.0});
  double scale = std::fabs(current - pr.gauge_distance) <= tol ? 1.0 : raw;
  if (scale != 1.0) {
    bool moves = false;
    for (size_t i = 0; i < pr.pose_count; ++i)
      moves = moves || (i != pr.gauge_first && !(pr.poses[i].variables & OMVGBA_POSE_TRANSLATION));
    for (size_t i = 0; i < pr.point_count; ++i) moves = moves || point_fixed(pr, i);
    if (moves) fail(OMVGBA_UNSUPPORTED, "fixed-baseline scaling would move fixed state");
  }
  plan.anchor = pr.gauge_first;
  plan.scale = scale;
  plan.native_cam = (pr.poses[pr.gauge_second].variables & OMVGBA_POSE_TRANSLATION) ? (int)pr.gauge_second : -1;
  return plan;
}

GaugePlan calibrated_gauge_plan(const omvgba_problem& pr) {
  auto observed = observed_cameras(pr);
  if (pr.gauge_kind == OMVGBA_GAUGE_FIXED_BASELINE) {
    GaugePlan p = gauge_plan(pr);
    p.masks[p.anchor] = 0;
    return p;
  }
  GaugePlan plan;
  for (size_t i = 0; i < pr.pose_count; ++i) plan.masks.push_back(pr.poses[i].variables);
  size_t first = SIZE_MAX;
  for (size_t i = 0; i < pr.pose_count; ++i)
    if (observed[i]) {
      first = i;
      break;
    }
  if (first == SIZE_MAX) fail(OMVGBA_INTERNAL, "checked bundle has no observed pose");
  size_t fixed_anchor = SIZE_MAX;
  for (size_t i = 0; i < pr.pose_count; ++i)
    if (observed[i] && plan.masks[i] == 0) {
      fixed_anchor = i;
      break;
    }
  bool controls = false;
  for (size_t o = 0; o < pr.observation_count; ++o) controls = controls || point_fixed(pr, pr.observation_point[o]);
  if (controls && fixed_anchor == SIZE_MAX) {
    plan.anchor = first;
    return plan;
  }
  std::vector<size_t> held;
  size_t known_rot = SIZE_MAX;
  for (size_t i = 0; i < pr.pose_count; ++i) {
    if (observed[i] && !(plan.masks[i] & OMVGBA_POSE_TRANSLATION)) held.push_back(i);
    if (known_rot == SIZE_MAX && observed[i] && !(plan.masks[i] & OMVGBA_POSE_ROTATION)) known_rot = i;
  }
  size_t anchor = fixed_anchor != SIZE_MAX ? fixed_anchor : (!held.empty() ? held[0] : (known_rot != SIZE_MAX ? known_rot : first));
  Vec3 ac = pose_C(pr.poses[anchor]);
  bool distinct = false;
  for (size_t c : held) distinct = distinct || sqdist(pose_C(pr.poses[c]), ac) > 0.0;
  if (!controls && held.empty())
    plan.masks[anchor] = 0;
  else if (!controls && known_rot == SIZE_MAX && !distinct)
    plan.masks[anchor] = 0;
  bool control_scale = false;
  for (size_t o = 0; o < pr.observation_count; ++o) {
    size_t p = pr.observation_point[o];
    control_scale = control_scale || (point_fixed(pr, p) && sqdist(point_at(pr, p), ac) > 0.0);
  }
  plan.anchor = anchor;
  if (!(distinct || control_scale)) {
    std::vector<std::pair<int, double>> c;
    for (size_t i = 0; i < pr.pose_count; ++i)
      if (i != anchor && observed[i] && (plan.masks[i] & OMVGBA_POSE_TRANSLATION))
        c.push_back({(int)i, sqdist(pose_C(pr.poses[i]), ac)});
    int cam = farthest_camera(c);
    if (cam < 0) fail(OMVGBA_UNSUPPORTED, "free-scale BA has no nonzero active baseline");
    plan.native_cam = cam;
  }
  return plan;
}

// ---- lowering --------------------------------------------------------------------------------
struct Rebase {
  Mat3 R;
  Vec3 C;
  double scale = 1.0;
  std::vector<size_t> camera_source_order;
};

void set_anchor(const omvgba_problem& pr, Rebase& rb, size_t anchor, double scale) {
  rb.R = pose_R(pr.poses[anchor]);
  rb.C = pose_C(pr.poses[anchor]);
  rb.scale = scale;
  if (!std::isfinite(scale) || scale <= 0.0) fail(OMVGBA_UNSUPPORTED, "world scale must be finite and positive");
  rb.camera_source_order.clear();
  rb.camera_source_order.push_back(anchor);
  for (size_t i = 0; i < pr.pose_count; ++i)
    if (i != anchor) rb.camera_source_order.push_back(i);
}
void pose_to_native(const Rebase& rb, const omvgba_pose& p, double* R9, double* t3) {
  Mat3 R = pose_R(p);
  Vec3 C = pose_C(p);
  if (R == rb.R && C == rb.C) {
    for (int k = 0; k < 9; ++k) R9[k] = (k % 4 == 0) ? 1.0 : 0.0;
    t3[0] = t3[1] = t3[2] = 0.0;
    return;
  }
  Mat3 AT;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) AT[i][j] = rb.R[j][i];
  Mat3 rot = mat_mul(R, AT);
  Vec3 t = rotate(R, {rb.C[0] - C[0], rb.C[1] - C[1], rb.C[2] - C[2]});
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) R9[3 * i + j] = rot[i][j];
  for (int k = 0; k < 3; ++k) t3[k] = t[k] * rb.scale;
}
Vec3 point_to_native(const Rebase& rb, const Vec3& X) {
  Vec3 r = rotate(rb.R, {X[0] - rb.C[0], X[1] - rb.C[1], X[2] - rb.C[2]});
  return {r[0] * rb.scale, r[1] * rb.scale, r[2] * rb.scale};
}
void pose_from_native(const Rebase& rb, const double* R9, const double* t3, double* Rout, double* Cout) {
  Mat3 Rr;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) Rr[i][j] = R9[3 * i + j];
  Mat3 R = mat_mul(Rr, rb.R);
  Vec3 rc = rotate_t(Rr, {t3[0], t3[1], t3[2]});
  Vec3 wc = rotate_t(rb.R, {-rc[0], -rc[1], -rc[2]});
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) Rout[3 * i + j] = R[i][j];
  for (int k = 0; k < 3; ++k) Cout[k] = rb.C[k] + wc[k];
}
Vec3 point_from_native(const Rebase& rb, const double* X) {
  Vec3 r = rotate_t(rb.R, {X[0], X[1], X[2]});
  return {rb.C[0] + r[0], rb.C[1] + r[1], rb.C[2] + r[2]};
}

bool has_free_intrinsics(const omvgba_problem& pr) {
  for (size_t o = 0; o < pr.observation_count; ++o)
    if (pr.intrinsics[pr.observation_intrinsic[o]].variables != 0) return true;
  return false;
}
bool single_pose_intrinsics(const omvgba_problem& pr, std::vector<size_t>* out) {
  std::vector<size_t> idx(pr.pose_count, SIZE_MAX);
  for (size_t o = 0; o < pr.observation_count; ++o) {
    size_t& s = idx[pr.observation_pose[o]];
    if (s != SIZE_MAX && s != pr.observation_intrinsic[o]) return false;
    s = pr.observation_intrinsic[o];
  }
  for (auto& s : idx)
    if (s == SIZE_MAX) s = 0;
  *out = idx;
  return true;
}

// point-major CSR with a stable sort by point (counting sort keeps source order within a track)
void sort_observations(const omvgba_problem& pr, NativeProblem& n, const std::vector<size_t>& dest,
                       FillVector<size_t>* order_out) {
  size_t N = pr.observation_count, P = pr.point_count;
  n.pt_off.assign(P + 1, 0);
  for (size_t o = 0; o < N; ++o) n.pt_off[pr.observation_point[o] + 1]++;
  for (size_t p = 0; p < P; ++p) n.pt_off[p + 1] += n.pt_off[p];
  FillVector<size_t> order(N);  // every position is written below
  std::vector<uint64_t> fill(n.pt_off.begin(), n.pt_off.end() - 1);
  for (size_t o = 0; o < N; ++o) order[fill[pr.observation_point[o]]++] = o;
  n.obs_cam.resize(N);
  n.obs_src.resize(N);
  for_fixed_chunks(N, 64, [&](size_t, size_t b, size_t e) {
    for (size_t i = b; i < e; ++i) {
      n.obs_cam[i] = (uint32_t)dest[pr.observation_pose[order[i]]];
      n.obs_src[i] = order[i];
    }
  });
  *order_out = std::move(order);
}

struct Lowered {
  NativeProblem n;
  Rebase rb;
};

// ---- bearings of measured pixels (Camera::bearing, openmvg-core camera/camera_enum.rs:128-132) ----
bool camera_bearing(const omvgba_intrinsic& in, double u, double v, double b[3]) {
  return camera_unproject_bearing(make_camera_dev(in), u, v, b);
}

// The calibrated lowering (native/calibrated.rs:200-494). Angular residuals (PreparedAngularProblem,
// calibrated.rs:27-123) keep the same frame, gauge and masks and carry each observation's unit bearing.
Lowered lower_calibrated(const omvgba_problem& pr, bool angular = false) {
  if (!angular)
    for (size_t o = 0; o < pr.observation_count; ++o) {
      int m = pr.intrinsics[pr.observation_intrinsic[o]].model;
      if (m == OMVGBA_CAMERA_FISHEYE || m == OMVGBA_CAMERA_SPHERICAL)
        fail(OMVGBA_UNSUPPORTED,
             "pixel BA supports fixed pinhole and Brown-Conrady cameras; use angular residuals for wide-angle cameras");
    }
  GaugePlan plan = calibrated_gauge_plan(pr);
  auto observed = observed_cameras(pr);
  Lowered L;
  NativeProblem& n = L.n;
  n.self_cal = false;
  n.explicit_masks = true;
  // CameraPoseVariables of the prepared problem (native/calibrated.rs:226-234): translation-only when
  // no free mask moves a rotation (vacuously so when every pose is fixed)
  n.translation_only = true;
  for (size_t i = 0; i < pr.pose_count; ++i)
    if (plan.masks[i] != 0 && (plan.masks[i] & OMVGBA_POSE_ROTATION)) n.translation_only = false;
  set_anchor(pr, L.rb, plan.anchor, plan.scale);
  n.ncam = (int)pr.pose_count;
  std::vector<size_t> dest(pr.pose_count);
  for (size_t d = 0; d < L.rb.camera_source_order.size(); ++d) dest[L.rb.camera_source_order[d]] = d;
  n.rotation.resize(9 * pr.pose_count);
  n.translation.resize(3 * pr.pose_count);
  for (size_t d = 0; d < L.rb.camera_source_order.size(); ++d) {
    size_t s = L.rb.camera_source_order[d];
    if (observed[s]) {
      pose_to_native(L.rb, pr.poses[s], &n.rotation[9 * d], &n.translation[3 * d]);
    } else {
      for (int k = 0; k < 9; ++k) n.rotation[9 * d + k] = (k % 4 == 0) ? 1.0 : 0.0;
      for (int k = 0; k < 3; ++k) n.translation[3 * d + k] = 0.0;
    }
    n.fixed_poses.push_back(plan.masks[s] == 0);
    n.pose_mask.push_back((uint8_t)((plan.masks[s] & OMVGBA_POSE_ROTATION ? 1 : 0) |
                                    (plan.masks[s] & OMVGBA_POSE_TRANSLATION ? 2 : 0)));
  }
  std::vector<uint8_t> pobs(pr.point_count, 0);
  for (size_t o = 0; o < pr.observation_count; ++o) pobs[pr.observation_point[o]] = 1;
  n.points.resize(3 * pr.point_count);
  for (size_t i = 0; i < pr.point_count; ++i) {
    Vec3 X = (point_fixed(pr, i) && !pobs[i]) ? Vec3{0, 0, 0} : point_to_native(L.rb, point_at(pr, i));
    for (int k = 0; k < 3; ++k) n.points[3 * i + k] = X[k];
    n.fixed_points.push_back(point_fixed(pr, i) ? 1 : 0);
  }
  std::vector<size_t> pose_intr;
  bool single = single_pose_intrinsics(pr, &pose_intr);
  bool uses_full = !single;
  for (size_t o = 0; o < pr.observation_count && !uses_full; ++o) {
    const auto& in = pr.intrinsics[pr.observation_intrinsic[o]];
    uses_full = in.model == OMVGBA_CAMERA_BROWN_CONRADY && (in.radial_kind != 0 || in.tangential_kind != 0);
  }
  n.pixel_model = !uses_full;
  for (size_t i = 0; i < pr.intrinsic_count; ++i) n.models.push_back(make_fixed_camera(pr.intrinsics[i]));
  n.gauge_cam = plan.native_cam >= 0 ? (int)dest[plan.native_cam] : -1;
  FillVector<size_t> order;
  sort_observations(pr, n, dest, &order);
  n.obs_px.resize(2 * order.size());
  n.obs_model.resize(order.size());
  for (size_t i = 0; i < order.size(); ++i) {
    n.obs_px[2 * i] = pr.observation_pixel[2 * order[i]];
    n.obs_px[2 * i + 1] = pr.observation_pixel[2 * order[i] + 1];
    n.obs_model[i] = pr.observation_intrinsic[order[i]];
  }
  if (angular) {
    n.angular = true;
    n.obs_bearing.resize(3 * order.size());
    std::atomic<size_t> bad{SIZE_MAX};
    for_fixed_chunks(order.size(), 64, [&](size_t, size_t b, size_t e) {
      for (size_t i = b; i < e; ++i)
        if (!camera_bearing(pr.intrinsics[n.obs_model[i]], n.obs_px[2 * i], n.obs_px[2 * i + 1], &n.obs_bearing[3 * i])) {
          size_t cur = bad.load();
          while (i < cur && !bad.compare_exchange_weak(cur, i)) {
          }
        }
    });
    if (bad.load() != SIZE_MAX)
      fail(OMVGBA_NUMERICAL, "observation " + std::to_string(order[bad.load()]) +
                                 ": the measured pixel does not define a bearing of its camera model");
  }
  return L;
}

int free_radial_dimension(const omvgba_intrinsic& in) {
  if (in.model == OMVGBA_CAMERA_BROWN_CONRADY && (in.variables & OMVGBA_INTRINSIC_RADIAL)) {
    if (in.radial_kind == 0) return 1;
    if (in.radial_kind == 1) return 2;
    return 3;
  }
  return 1;
}

Lowered lower_self_calibrating(const omvgba_problem& pr) {
  std::vector<size_t> pose_intr;
  if (!single_pose_intrinsics(pr, &pose_intr))
    fail(OMVGBA_UNSUPPORTED, "native self-calibration requires one intrinsic group per observed pose");
  auto observed = observed_cameras(pr);
  for (size_t i = 0; i < pr.pose_count; ++i) {
    uint32_t v = pr.poses[i].variables;
    if (!observed[i] || v == 0) continue;
    if (!(v & OMVGBA_POSE_TRANSLATION))
      fail(OMVGBA_UNSUPPORTED, "direct native lowering cannot optimize rotation without translation");
    if (!(v & OMVGBA_POSE_ROTATION)) fail(OMVGBA_UNSUPPORTED, "self-calibration requires full-pose or fixed camera blocks");
  }
  for (size_t i = 0; i < pr.intrinsic_count; ++i) {
    const auto& in = pr.intrinsics[i];
    if ((in.variables & OMVGBA_INTRINSIC_RADIAL) && in.model == OMVGBA_CAMERA_BROWN_CONRADY && in.radial_kind == 3)
      fail(OMVGBA_UNSUPPORTED, "native self-calibration refines at most two declared radial coefficients");
    if (in.variables != 0 && (!(in.variables & OMVGBA_INTRINSIC_FOCAL) || (in.variables & OMVGBA_INTRINSIC_PRINCIPAL_POINT) ||
                              (in.variables & OMVGBA_INTRINSIC_TANGENTIAL)))
      fail(OMVGBA_UNSUPPORTED,
           "self-calibration refines the focal length and radial coefficients with a fixed principal point");
  }
  GaugePlan plan = gauge_plan(pr);
  Lowered L;
  NativeProblem& n = L.n;
  n.self_cal = true;
  set_anchor(pr, L.rb, plan.anchor, plan.scale);
  n.ncam = (int)pr.pose_count;
  std::vector<size_t> dest(pr.pose_count);
  for (size_t d = 0; d < L.rb.camera_source_order.size(); ++d) dest[L.rb.camera_source_order[d]] = d;
  n.rotation.resize(9 * pr.pose_count);
  n.translation.resize(3 * pr.pose_count);
  for (size_t d = 0; d < L.rb.camera_source_order.size(); ++d) {
    size_t s = L.rb.camera_source_order[d];
    pose_to_native(L.rb, pr.poses[s], &n.rotation[9 * d], &n.translation[3 * d]);
    n.fixed_poses.push_back((s == plan.anchor || pr.poses[s].variables == 0) ? 1 : 0);
    n.cam_group.push_back((uint32_t)pose_intr[s]);
  }
  n.points.resize(3 * pr.point_count);
  for (size_t i = 0; i < pr.point_count; ++i) {
    Vec3 X = point_to_native(L.rb, point_at(pr, i));
    for (int k = 0; k < 3; ++k) n.points[3 * i + k] = X[k];
    n.fixed_points.push_back(point_fixed(pr, i) ? 1 : 0);
  }
  for (size_t i = 0; i < pr.intrinsic_count; ++i) {
    const auto& in = pr.intrinsics[i];
    if (in.model == OMVGBA_CAMERA_FISHEYE || in.model == OMVGBA_CAMERA_SPHERICAL)
      fail(OMVGBA_UNSUPPORTED, "self-calibration supports perspective cameras only");
    double k1 = 0, k2 = 0, k3 = 0, p1 = 0, p2 = 0;
    if (in.model == OMVGBA_CAMERA_BROWN_CONRADY) {
      k1 = in.radial_kind >= 1 ? in.k1 : 0.0;
      k2 = in.radial_kind >= 2 ? in.k2 : 0.0;
      k3 = in.radial_kind >= 3 ? in.k3 : 0.0;
      p1 = in.tangential_kind >= 1 ? in.p1 : 0.0;
      p2 = in.tangential_kind >= 2 ? in.p2 : 0.0;
    }
    if (in.fx != in.fy || k3 != 0.0 || p1 != 0.0 || p2 != 0.0)
      fail(OMVGBA_UNSUPPORTED,
           "self-calibration requires isotropic focal length, k1+k2 radial distortion, and no tangential distortion");
    n.groups.push_back(in.fx);
    n.groups.push_back(k1);
    n.groups.push_back(k2);
    n.group_dim.push_back(in.variables == 0 ? 0 : free_radial_dimension(in));
  }
  n.gauge_cam = plan.native_cam >= 0 ? (int)dest[plan.native_cam] : -1;
  FillVector<size_t> order;
  sort_observations(pr, n, dest, &order);
  n.obs_px.resize(2 * order.size());
  for_fixed_chunks(order.size(), 64, [&](size_t, size_t b, size_t e) {
    for (size_t i = b; i < e; ++i) {
      const auto& in = pr.intrinsics[pr.observation_intrinsic[order[i]]];
      n.obs_px[2 * i] = pr.observation_pixel[2 * order[i]] - in.cx;
      n.obs_px[2 * i + 1] = pr.observation_pixel[2 * order[i] + 1] - in.cy;
    }
  });
  return L;
}

// Regroups points so that consecutive points share cameras: stable order by the smallest native
// camera index of the track. Points are independent given the cameras, so this changes only the
// grouping of the camera-side sums; it lets the GPU kernels reduce each tile of points into few
// camera segments. Observations stay point-major and keep their source order within a track.
void reorder_points_for_locality(NativeProblem& n) {
  size_t P = n.points.size() / 3, N = n.obs_cam.size();
  // key: the smallest camera index of the track (ncam for a point without observations)
  std::vector<uint32_t> key(P);
  const uint32_t none = (uint32_t)n.ncam;
  for_fixed_chunks(P, 64, [&](size_t, size_t b, size_t e) {
    for (size_t p = b; p < e; ++p) {
      uint32_t k = UINT32_MAX;
      for (uint64_t o = n.pt_off[p]; o < n.pt_off[p + 1]; ++o) k = std::min(k, n.obs_cam[o]);
      key[p] = std::min(k, none);
    }
  });
  // stable order by key: a counting sort (equal keys keep their point order)
  std::vector<uint64_t> start((size_t)none + 2, 0);
  for (size_t p = 0; p < P; ++p) start[key[p] + 1]++;
  for (size_t k = 0; k <= none; ++k) start[k + 1] += start[k];
  FillVector<uint64_t> order(P);  // every array below is written completely before it is read
  for (size_t p = 0; p < P; ++p) order[start[key[p]]++] = p;
  FillVector<double> points(3 * P);
  std::vector<uint8_t> fixed(P);
  FillVector<uint64_t> off(P + 1, 0);
  for (size_t q = 0; q < P; ++q) off[q + 1] = off[q] + (n.pt_off[order[q] + 1] - n.pt_off[order[q]]);
  FillVector<uint32_t> cam(N), model(n.obs_model.empty() ? 0 : N);
  FillVector<double> px(2 * N), bearing(n.angular ? 3 * N : 0);
  FillVector<uint64_t> src(N);
  for_fixed_chunks(P, 64, [&](size_t, size_t b, size_t e) {
    for (size_t q = b; q < e; ++q) {
      uint64_t p = order[q];
      for (int k = 0; k < 3; ++k) points[3 * q + k] = n.points[3 * p + k];
      fixed[q] = n.fixed_points[p];
      uint64_t w = off[q];
      for (uint64_t o = n.pt_off[p]; o < n.pt_off[p + 1]; ++o, ++w) {
        cam[w] = n.obs_cam[o];
        if (!model.empty()) model[w] = n.obs_model[o];
        px[2 * w] = n.obs_px[2 * o];
        px[2 * w + 1] = n.obs_px[2 * o + 1];
        if (n.angular)
          for (int k = 0; k < 3; ++k) bearing[3 * w + k] = n.obs_bearing[3 * o + k];
        src[w] = n.obs_src[o];
      }
    }
  });
  n.points.swap(points);
  n.fixed_points.swap(fixed);
  n.pt_off.swap(off);
  n.obs_cam.swap(cam);
  if (!model.empty()) n.obs_model.swap(model);
  n.obs_px.swap(px);
  if (n.angular) n.obs_bearing.swap(bearing);
  n.obs_src.swap(src);
  n.point_source = std::move(order);
}

Lowered lower(const omvgba_problem& pr) {
  if (pr.residual_space == OMVGBA_RESIDUAL_ANGULAR && has_free_intrinsics(pr))
    fail(OMVGBA_UNSUPPORTED, "angular BA requires fixed intrinsics");
  Lowered L = pr.residual_space == OMVGBA_RESIDUAL_ANGULAR ? lower_calibrated(pr, true)
              : has_free_intrinsics(pr)                    ? lower_self_calibrating(pr)
                                                           : lower_calibrated(pr);
  reorder_points_for_locality(L.n);
  return L;
}

int reduced_dimension(const NativeProblem& n) {
  int D = 0;
  for (int c = 0; c < n.ncam; ++c) D += pose_block_dim(n, c);
  if (n.self_cal)
    for (int d : n.group_dim) D += d;
  return D;
}

LmOptions lm_options(const omvgba_problem& pr, const omvgba_config& cfg, const NativeProblem& n) {
  LmOptions o;
  o.max_iterations = cfg.max_iterations;
  o.loss = problem_loss(pr);
  o.gradient_tolerance = cfg.gradient_tolerance;
  o.step_tolerance = cfg.parameter_tolerance;
  o.relative_cost_tolerance = cfg.function_tolerance;
  int D = reduced_dimension(n);
  (void)D;
  // Auto is resolved by the solver once it knows the reduced pattern (execution_policy.rs:122-253)
  o.linear_solver = cfg.linear_solver;
  o.iterative = cfg.linear_solver == OMVGBA_SOLVER_ITERATIVE;
  o.workspace_budget = cfg.has_workspace_budget ? cfg.workspace_budget_bytes : 0;
  o.pcg_tolerance = cfg.pcg_relative_tolerance > 0.0 ? cfg.pcg_relative_tolerance : 1e-1;
  o.pcg_max_iterations = cfg.pcg_max_iterations > 0 ? cfg.pcg_max_iterations : 600;
  o.precision = cfg.precision;
  o.matvec = cfg.matvec;
  o.stream = cfg.stream;
  return o;
}

// ---- solution ----------------------------------------------------------------------------------
struct Result {
  std::vector<omvgba_pose> poses;
  std::vector<omvgba_intrinsic> intrinsics;
  std::vector<double> points;
  std::vector<uint64_t> quarantined;
  std::vector<uint64_t> unconstrained;  // intrinsic groups held at their input values by the certificate
  omvgba_report report{};
};

// Largest accepted marginal standard deviation of each free intrinsic parameter's contribution to the
// relative radial displacement at the farthest image corner (native/self_calibration.rs:215-222).
constexpr double kMaxIntrinsicCornerStd = 0.01;

// Free intrinsic groups that the final information does not constrain
// (native/self_calibration.rs:255-303): sigma(log f), sigma(k1) r^2 and sigma(k2) r^4 of the marginal
// covariance (S^-1)_gg times the zero-residual weight, with r the normalized radius of the farthest
// corner at the final focal length; a NaN deviation holds even a waived group, a deviation above the
// bound holds a required one. Every free group when S does not factor or any marginal is not finite.
std::vector<uint64_t> unconstrained_groups(const omvgba_problem& pr, const NativeProblem& n,
                                           const std::vector<double>& groups, const NativeReport& nr,
                                           const LossDev& loss) {
  std::vector<uint64_t> all, out;
  for (size_t g = 0; g < n.group_dim.size(); ++g)
    if (n.group_dim[g] > 0) all.push_back(g);
  if (all.empty()) return out;
  if (!nr.marginals_ok || nr.marginals.size() < 9 * n.group_dim.size()) return all;
  const double zw = loss.sqrt_weight(0.0);
  const double wn = zw * zw;
  for (uint64_t g : all) {
    const int dim = n.group_dim[g];
    for (int a = 0; a < dim; ++a)
      for (int b = 0; b < dim; ++b)
        if (!std::isfinite(nr.marginals[9 * g + 3 * a + b] * wn)) return all;
  }
  for (uint64_t g : all) {
    const omvgba_intrinsic& in = pr.intrinsics[g];
    const double f = groups[3 * g];
    const double ux = std::max(in.cx, double(in.width) - in.cx) / f, uy = std::max(in.cy, double(in.height) - in.cy) / f;
    const double r2 = ux * ux + uy * uy;
    const double scales[3] = {1.0, r2, r2 * r2};
    const bool waived = in.certification == 1;
    bool held = false;
    for (int k = 0; k < n.group_dim[g]; ++k) {
      const double dev = std::sqrt(nr.marginals[9 * g + 4 * k] * wn) * scales[k];
      held = held || std::isnan(dev) || (!waived && dev > kMaxIntrinsicCornerStd);
    }
    if (held) out.push_back(g);
  }
  return out;
}

// The poses' rotations and centres and the intrinsics' camera models of one state, built once so
// that per-observation residuals only rotate and project.
struct StateView {
  std::vector<Mat3> R;
  std::vector<Vec3> C;
  std::vector<FixedCameraDev> model;
  std::vector<uint8_t> supported;
  bool angular = false;
  const omvgba_intrinsic* intrinsics = nullptr;
  StateView(const omvgba_problem& pr, const omvgba_pose* poses, const omvgba_intrinsic* intrinsics)
      : R(pr.pose_count), C(pr.pose_count), model(pr.intrinsic_count), supported(pr.intrinsic_count),
        angular(pr.residual_space == OMVGBA_RESIDUAL_ANGULAR), intrinsics(intrinsics) {
    for (size_t i = 0; i < pr.pose_count; ++i) {
      R[i] = pose_R(poses[i]);
      C[i] = pose_C(poses[i]);
    }
    for (size_t i = 0; i < pr.intrinsic_count; ++i) {
      const omvgba_intrinsic& in = intrinsics[i];
      supported[i] = in.model == OMVGBA_CAMERA_PINHOLE || in.model == OMVGBA_CAMERA_BROWN_CONRADY;
      if (supported[i]) model[i] = make_fixed_camera(in);
    }
  }
};

// Residual norm of observation o with the point at X (solver.rs:1405-1432): pixels, or the angle
// between the measured bearing and the camera point.
bool residual_norm(const omvgba_problem& pr, const StateView& sv, size_t o, const double* X, double* out) {
  const size_t pi = pr.observation_pose[o], ii = pr.observation_intrinsic[o];
  const Vec3& C = sv.C[pi];
  Vec3 xc = rotate(sv.R[pi], {X[0] - C[0], X[1] - C[1], X[2] - C[2]});
  if (sv.angular) {
    double b[3], r[2], J[2][3];
    if (!camera_bearing(sv.intrinsics[ii], pr.observation_pixel[2 * o], pr.observation_pixel[2 * o + 1], b)) return false;
    if (!angular_linearize(b, xc.data(), r, J)) return false;
    const double nrm = std::hypot(r[0], r[1]);
    if (!std::isfinite(nrm)) return false;
    *out = nrm;
    return true;
  }
  if (!sv.supported[ii]) return false;
  double u, v;
  if (!sv.model[ii].project(xc[0], xc[1], xc[2], &u, &v)) return false;
  double nrm = std::hypot(u - pr.observation_pixel[2 * o], v - pr.observation_pixel[2 * o + 1]);
  if (!std::isfinite(nrm)) return false;
  *out = nrm;
  return true;
}

bool active_metrics(const omvgba_problem& pr, const std::vector<uint8_t>& active, const Result* sol, double* cost,
                    double* rmse);


// Inlier count and RMSE of the solution (solver.rs:1317-1402): residual norms of the active
// observations within the loss scale (every one for squared loss). 64 fixed chunks.
void refresh_inliers(const omvgba_problem& pr, const std::vector<uint8_t>& active, Result& res) {
  double limit = pr.loss_kind == OMVGBA_LOSS_SQUARED ? INFINITY : pr.loss_scale;
  constexpr size_t kChunks = 64;
  std::vector<uint64_t> count(kChunks, 0);
  std::vector<double> ss(kChunks, 0.0);
  std::vector<uint8_t> ok(kChunks, 1);
  res.report.has_inlier_count = 0;
  res.report.has_final_inlier_rmse = 0;
  const StateView sv(pr, res.poses.data(), res.intrinsics.data());
  const double* X = res.points.data();
  for_fixed_chunks(pr.observation_count, kChunks, [&](size_t c, size_t b, size_t e) {
    uint64_t n = 0;  // locals: the chunks' slots share cache lines
    double sum = 0.0;
    for (size_t o = b; o < e; ++o) {
      size_t p = pr.observation_point[o];
      if (!active[p]) continue;
      double nrm;
      if (!residual_norm(pr, sv, o, X + 3 * p, &nrm)) {
        ok[c] = 0;
        return;
      }
      if (nrm <= limit) {
        n++;
        sum += nrm * nrm;
      }
    }
    count[c] = n;
    ss[c] = sum;
  });
  uint64_t total = 0;
  double sum = 0.0;
  for (size_t c = 0; c < kChunks; ++c) {
    if (!ok[c]) return;
    total += count[c];
    sum += ss[c];
  }
  res.report.has_inlier_count = 1;
  res.report.inlier_count = total;
  if (total > 0) {
    double r = std::sqrt(sum / double(total));
    if (std::isfinite(r)) {
      res.report.has_final_inlier_rmse = 1;
      res.report.final_inlier_rmse = r;
    }
  }
}

// Objective and RMSE of the active observations at the input state (sol == nullptr) or at a
// solution (solver.rs:1052-1131): the RMSE accumulates a scaled sum of squares (largest norm and
// the sum of squares relative to it) so it cannot overflow. 64 fixed chunks combined in order.
// One chunk's share of the objective and of the scaled sum of squares of the residual norms.
struct MetricPart {
  double total = 0.0, rs = 0.0, ssr = 1.0;
  size_t count = 0;
  bool ok = true;
  void add(const LossDev& loss, double nrm) {
    total += loss.cost(nrm);
    if (nrm > 0.0) {
      if (rs < nrm) {
        ssr = 1.0 + ssr * (rs / nrm) * (rs / nrm);
        rs = nrm;
      } else {
        ssr += (nrm / rs) * (nrm / rs);
      }
    }
    count++;
  }
};
bool merge_metrics(const std::vector<MetricPart>& parts, double* cost, double* rmse);

bool active_metrics(const omvgba_problem& pr, const std::vector<uint8_t>& active, const Result* sol, double* cost,
                    double* rmse) {
  LossDev loss = problem_loss(pr);
  constexpr size_t kChunks = 64;
  std::vector<MetricPart> parts(kChunks);
  const StateView sv(pr, sol ? sol->poses.data() : pr.poses, sol ? sol->intrinsics.data() : pr.intrinsics);
  const double* X0 = sol ? sol->points.data() : pr.points;
  for_fixed_chunks(pr.observation_count, kChunks, [&](size_t c, size_t b, size_t e) {
    MetricPart pt;  // a local: the chunks' slots share cache lines
    for (size_t o = b; o < e && pt.ok; ++o) {
      size_t p = pr.observation_point[o];
      if (!active[p]) continue;
      double nrm;
      if (!residual_norm(pr, sv, o, X0 + 3 * p, &nrm))
        pt.ok = false;
      else
        pt.add(loss, nrm);
    }
    parts[c] = pt;
  });
  return merge_metrics(parts, cost, rmse);
}

// Chunks combined in order: objective, count and the scaled sums of squares of the RMSE.
bool merge_metrics(const std::vector<MetricPart>& parts, double* cost, double* rmse) {
  double total = 0.0, rs = 0.0, ssr = 1.0;
  size_t count = 0;
  for (const MetricPart& pt : parts) {
    if (!pt.ok) return false;
    total += pt.total;
    count += pt.count;
    if (pt.rs > 0.0) {  // merge the chunk's scaled sum of squares
      if (rs < pt.rs) {
        ssr = pt.ssr + ssr * (rs / pt.rs) * (rs / pt.rs);
        rs = pt.rs;
      } else {
        ssr += pt.ssr * (pt.rs / rs) * (pt.rs / rs);
      }
    }
  }
  if (count == 0 || !std::isfinite(total) || total < 0.0) return false;
  double r = rs * std::sqrt(ssr / double(count));
  if (!std::isfinite(r)) return false;
  *cost = total;
  *rmse = r;
  return true;
}

Result raise(const omvgba_problem& pr, const Lowered& L, const std::vector<double>& rot, const std::vector<double>& tr,
             const std::vector<double>& points, const std::vector<double>& groups, const NativeReport& nr,
             bool iterative) {
  Result res;
  auto observed = observed_cameras(pr);
  const NativeProblem& n = L.n;
  res.poses.assign(pr.poses, pr.poses + pr.pose_count);
  for (size_t d = 0; d < L.rb.camera_source_order.size(); ++d) {
    size_t s = L.rb.camera_source_order[d];
    const omvgba_pose& in = pr.poses[s];
    if (in.variables == 0 || !observed[s]) continue;
    double R[9], C[3];
    pose_from_native(L.rb, &rot[9 * d], &tr[3 * d], R, C);
    if (in.variables & OMVGBA_POSE_ROTATION) std::memcpy(res.poses[s].rotation, R, sizeof(R));
    if (in.variables & OMVGBA_POSE_TRANSLATION) std::memcpy(res.poses[s].center, C, sizeof(C));
  }
  res.points.resize(3 * pr.point_count);
  for (size_t q = 0; q < pr.point_count; ++q) {
    size_t i = n.point_source[q];
    Vec3 X = point_fixed(pr, i) ? point_at(pr, i) : point_from_native(L.rb, &points[3 * q]);
    if (!all_finite(X.data(), 3)) fail(OMVGBA_NUMERICAL, "native BA returned a non-finite point");
    for (int k = 0; k < 3; ++k) res.points[3 * i + k] = X[k];
  }
  res.intrinsics.assign(pr.intrinsics, pr.intrinsics + pr.intrinsic_count);
  if (n.self_cal)
    for (size_t i = 0; i < pr.intrinsic_count; ++i) {
      auto& out = res.intrinsics[i];
      if (out.variables == 0) continue;
      out.fx = groups[3 * i];
      out.fy = groups[3 * i];
      if (out.model == OMVGBA_CAMERA_BROWN_CONRADY) {
        if (out.radial_kind >= 1) out.k1 = groups[3 * i + 1];
        if (out.radial_kind >= 2) out.k2 = groups[3 * i + 2];
      }
    }
  omvgba_report& r = res.report;
  std::memset(&r, 0, sizeof(r));
  r.status = nr.status == 0 ? OMVGBA_STATUS_CONVERGED
                            : (nr.status == 1 ? OMVGBA_STATUS_MAX_ITERATIONS
                                              : (nr.status == 2 ? OMVGBA_STATUS_STALLED : OMVGBA_STATUS_DEGENERATE));
  r.convergence_reason = nr.status == 0 ? nr.reason : OMVGBA_REASON_NONE;
  r.iteration_count = nr.iterations;
  r.initial_objective = nr.initial_cost;
  r.final_objective = nr.final_cost;
  r.initial_rmse = nr.initial_rmse * std::sqrt(2.0);
  r.final_rmse = nr.final_rmse * std::sqrt(2.0);
  r.accepted_step_count = nr.accepted;
  r.rejected_step_count = nr.rejected;
  r.rejected_linearization = nr.rej[0];
  r.rejected_step_solve = nr.rej[1];
  r.rejected_candidate = nr.rej[2];
  r.rejected_insufficient_reduction = nr.rej[3];
  if (!std::isfinite(nr.gradient_inf_norm) || nr.gradient_inf_norm < 0.0)
    fail(OMVGBA_NUMERICAL, "stationarity audit requires a finite non-negative gradient norm");
  r.has_stationarity = 1;
  r.scaled_gradient_inf_norm = nr.gradient_inf_norm;
  r.observability = nr.rank == 0 ? OMVGBA_OBS_FULL_RANK : (nr.rank == 2 ? OMVGBA_OBS_RANK_DEFICIENT : OMVGBA_OBS_NOT_ASSESSED);
  r.has_weak_point_count = 1;
  r.weak_point_count = nr.weak;
  r.has_noninvertible_observation_count = 1;
  r.noninvertible_observation_count = nr.noninvertible;
  if (r.observability != OMVGBA_OBS_NOT_ASSESSED && nr.D > 0) {
    r.has_observability_details = 1;
    r.details_pose_rank = r.observability == OMVGBA_OBS_FULL_RANK ? nr.D : 0;
    r.details_pose_dimension = nr.D;
    r.details_weak_point_count = nr.weak;
  }
  r.has_linear_solver = 1;
  r.linear_solver = iterative ? OMVGBA_SOLVER_ITERATIVE : OMVGBA_SOLVER_DIRECT;
  r.pcg_iteration_count = nr.pcg_terms;
  r.reduced_dimension = nr.D;
  r.final_damping = nr.final_damping;
  double vals[4] = {r.initial_objective, r.final_objective, r.initial_rmse, r.final_rmse};
  for (double v : vals)
    if (!std::isfinite(v) || v < 0.0) fail(OMVGBA_INTERNAL, "bundle-adjustment report is invalid");
  if (r.accepted_step_count > r.iteration_count) fail(OMVGBA_INTERNAL, "bundle-adjustment report is invalid");
  return res;
}

// The solution's report over the active observations (points not held out): their count, and, with
// points held out, the objective and RMSE at the input state and at the solution; then the inlier
// count and RMSE of the solution. One pass over the observations: each quantity is accumulated per
// chunk as active_metrics and refresh_inliers accumulate it and combined in the same chunk order, and
// the solution's residual norm, which both use, is evaluated once.
// The input-state metrics of a problem with held-out points (the report's initial objective and RMSE)
// depend only on the input and on the held-out set, so a plan keeps them from one solve to the next.
struct InputMetrics {
  bool valid = false;
  std::vector<uint64_t> quarantined;
  std::vector<MetricPart> parts;
};

void finish_solution(const omvgba_problem& pr, Result& res, InputMetrics* cache = nullptr) {
  std::vector<uint8_t> active(pr.point_count, 1);
  for (auto q : res.quarantined) active[q] = 0;
  const bool held_out = !res.quarantined.empty();
  const bool reuse_input = held_out && cache && cache->valid && cache->quarantined == res.quarantined;
  const LossDev loss = problem_loss(pr);
  const double limit = pr.loss_kind == OMVGBA_LOSS_SQUARED ? INFINITY : pr.loss_scale;
  constexpr size_t kChunks = 64;
  std::vector<uint64_t> seen(kChunks, 0), inliers(kChunks, 0);
  std::vector<double> inlier_ss(kChunks, 0.0);
  std::vector<MetricPart> at_input(kChunks), at_solution(kChunks);  // at_solution[c].ok: chunk c's norms
  const StateView sv(pr, res.poses.data(), res.intrinsics.data());
  std::unique_ptr<StateView> sv_input;
  if (held_out) sv_input = std::make_unique<StateView>(pr, pr.poses, pr.intrinsics);
  // each chunk accumulates in locals and stores once: the chunks' slots share cache lines
  const double* X1 = res.points.data();
  for_fixed_chunks(pr.observation_count, kChunks, [&](size_t c, size_t b, size_t e) {
    MetricPart m1, m0;
    uint64_t n_seen = 0, n_in = 0;
    double ss = 0.0;
    for (size_t o = b; o < e; ++o) {
      const size_t p = pr.observation_point[o];
      if (!active[p]) continue;
      n_seen++;
      if (m1.ok) {
        double nrm;
        if (!residual_norm(pr, sv, o, X1 + 3 * p, &nrm)) {
          m1.ok = false;
        } else {
          if (held_out) m1.add(loss, nrm);
          if (nrm <= limit) {
            n_in++;
            ss += nrm * nrm;
          }
        }
      }
      if (held_out && !reuse_input && m0.ok) {
        double nrm;
        if (!residual_norm(pr, *sv_input, o, pr.points + 3 * p, &nrm))
          m0.ok = false;
        else
          m0.add(loss, nrm);
      }
    }
    at_solution[c] = m1;
    at_input[c] = m0;
    seen[c] = n_seen;
    inliers[c] = n_in;
    inlier_ss[c] = ss;
  });
  if (reuse_input) {
    at_input = cache->parts;
  } else if (held_out && cache) {
    cache->valid = true;
    cache->quarantined = res.quarantined;
    cache->parts = at_input;
  }
  uint64_t cnt = 0;
  for (uint64_t k : seen) cnt += k;
  res.report.has_observation_count = 1;
  res.report.observation_count = cnt;
  res.report.quarantined_point_count = res.quarantined.size();
  if (held_out) {
    double c0, r0, c1, r1;
    if (!merge_metrics(at_input, &c0, &r0) || !merge_metrics(at_solution, &c1, &r1))
      fail(OMVGBA_INTERNAL, "bundle-adjustment report is invalid");
    res.report.initial_objective = c0;
    res.report.initial_rmse = r0;
    res.report.final_objective = c1;
    res.report.final_rmse = r1;
  }
  // inlier count and RMSE, as refresh_inliers reports them
  res.report.has_inlier_count = 0;
  res.report.has_final_inlier_rmse = 0;
  uint64_t total = 0;
  double sum = 0.0;
  for (size_t c = 0; c < kChunks; ++c) {
    if (!at_solution[c].ok) return;
    total += inliers[c];
    sum += inlier_ss[c];
  }
  res.report.has_inlier_count = 1;
  res.report.inlier_count = total;
  if (total > 0) {
    double r = std::sqrt(sum / double(total));
    if (std::isfinite(r)) {
      res.report.has_final_inlier_rmse = 1;
      res.report.final_inlier_rmse = r;
    }
  }
}

void canonicalize(const omvgba_problem& pr, Result& res) {
  if (pr.gauge_kind == OMVGBA_GAUGE_FIXED_BASELINE) {
    double init = std::sqrt(sqdist(pose_C(pr.poses[pr.gauge_first]), pose_C(pr.poses[pr.gauge_second])));
    if (!std::isfinite(init) || std::fabs(init - pr.gauge_distance) > 512.0 * kEps * std::max(init, pr.gauge_distance))
      return;
  }
  auto& r = res.report;
  double inc = r.final_objective - r.initial_objective;
  double tol = 2.0 * std::sqrt(kEps) * std::max(std::fabs(r.initial_objective), 1.0);
  if (!(inc > 0.0 && inc <= tol && r.status == OMVGBA_STATUS_CONVERGED && r.observability != OMVGBA_OBS_RANK_DEFICIENT))
    return;
  std::vector<uint8_t> active(pr.point_count, 1);
  for (auto q : res.quarantined) active[q] = 0;
  double c0, r0;
  if (!active_metrics(pr, active, nullptr, &c0, &r0)) return;
  bool same = true;
  for (size_t i = 0; i < pr.pose_count && same; ++i)
    same = std::memcmp(res.poses[i].rotation, pr.poses[i].rotation, sizeof(double) * 9) == 0 &&
           std::memcmp(res.poses[i].center, pr.poses[i].center, sizeof(double) * 3) == 0;
  for (size_t i = 0; i < pr.intrinsic_count && same; ++i)
    same = std::memcmp(&res.intrinsics[i], &pr.intrinsics[i], sizeof(omvgba_intrinsic)) == 0;
  same = same && std::memcmp(res.points.data(), pr.points, sizeof(double) * 3 * pr.point_count) == 0;
  if (!same) {
    res.poses.assign(pr.poses, pr.poses + pr.pose_count);
    res.intrinsics.assign(pr.intrinsics, pr.intrinsics + pr.intrinsic_count);
    res.points.assign(pr.points, pr.points + 3 * pr.point_count);
    r.has_stationarity = 0;
    r.observability = OMVGBA_OBS_NOT_ASSESSED;
    r.has_weak_point_count = 0;
    r.has_noninvertible_observation_count = 0;
    r.has_observability_details = 0;
  }
  r.initial_objective = c0;
  r.final_objective = c0;
  r.initial_rmse = r0;
  r.final_rmse = r0;
  r.status = OMVGBA_STATUS_SKIPPED;
  r.convergence_reason = OMVGBA_REASON_NONE;
  refresh_inliers(pr, active, res);
}

// ---- translation-only observability: the preflight and the post-solve probe -------------------
// common_pose_variables (native/gauge.rs:9-40): 1 when every observed free pose moves only its
// centre, 0 when they move rotation and translation (or none is free), -1 when the masks are not one
// of those forms (a rotation without translation, or a mixture).
int common_pose_variables(const omvgba_problem& pr) {
  const auto observed = observed_cameras(pr);
  int selected = -1;
  for (size_t i = 0; i < pr.pose_count; ++i) {
    const uint32_t v = pr.poses[i].variables;
    if (!observed[i] || v == 0) continue;
    if (!(v & OMVGBA_POSE_TRANSLATION)) return -1;
    const int candidate = (v & OMVGBA_POSE_ROTATION) ? 0 : 1;
    if (selected >= 0 && selected != candidate) return -1;
    selected = candidate;
  }
  return selected < 0 ? 0 : selected;
}

// can_probe_scale_representative (native/mod.rs:510-521)
bool can_probe_scale_representative(const omvgba_problem& pr) {
  if (pr.gauge_kind != OMVGBA_GAUGE_FIXED_BASELINE) return true;
  const auto observed = observed_cameras(pr);
  const double* f = pr.poses[pr.gauge_first].center;
  for (size_t c = 0; c < pr.pose_count; ++c) {
    const double* x = pr.poses[c].center;
    if (c != pr.gauge_first && observed[c] && !(pr.poses[c].variables & OMVGBA_POSE_TRANSLATION) &&
        !(x[0] == f[0] && x[1] == f[1] && x[2] == f[2]))
      return false;
  }
  return true;
}

// The probe's problem on the prepared (rebased) frame of a calibrated lowering with the native state
// rot / tr / pts (probe_prepared, native/fixed_rotation.rs:50-165): centres C = -R^T t, one camera
// model per pose (the pinhole of its intrinsics, or the full Brown-Conrady camera when the lowering
// uses full models), the tracks in the lowering's point order, the scale camera of the native gauge.
ProbeProblem prepared_probe_problem(const omvgba_problem& pr, const Lowered& L, const std::vector<double>& rot,
                                    const std::vector<double>& tr, const std::vector<double>& pts) {
  const NativeProblem& n = L.n;
  ProbeProblem q;
  std::vector<size_t> pose_intr;
  single_pose_intrinsics(pr, &pose_intr);
  const auto observed = observed_cameras(pr);
  const size_t fallback = pr.observation_count ? pr.observation_intrinsic[0] : 0;
  q.cameras.resize(n.ncam);
  for (int c = 0; c < n.ncam; ++c) {
    ProbeCamera& cam = q.cameras[c];
    for (int k = 0; k < 9; ++k) cam.R[k] = rot[9 * (size_t)c + k];
    const double* t = &tr[3 * (size_t)c];
    for (int j = 0; j < 3; ++j) cam.C[j] = -(cam.R[j] * t[0] + cam.R[3 + j] * t[1] + cam.R[6 + j] * t[2]);
    cam.fixed = n.fixed_poses[c] != 0;
    const size_t src = L.rb.camera_source_order[c];
    for (double& v : cam.intrinsics) v = 0.0;
    if (!observed[src] && n.pixel_model) {
      cam.intrinsics[0] = cam.intrinsics[1] = 1.0;  // PinholeCamera::new(1, 1, 0, 0)
      continue;
    }
    const omvgba_intrinsic& in = pr.intrinsics[observed[src] ? pose_intr[src] : fallback];
    cam.intrinsics[0] = in.fx;
    cam.intrinsics[1] = in.fy;
    cam.intrinsics[2] = in.cx;
    cam.intrinsics[3] = in.cy;
    if (!n.pixel_model && in.model == OMVGBA_CAMERA_BROWN_CONRADY) {
      cam.intrinsics[4] = in.radial_kind >= 1 ? in.k1 : 0.0;
      cam.intrinsics[5] = in.radial_kind >= 2 ? in.k2 : 0.0;
      cam.intrinsics[6] = in.radial_kind >= 3 ? in.k3 : 0.0;
      cam.intrinsics[7] = in.tangential_kind >= 1 ? in.p1 : 0.0;
      cam.intrinsics[8] = in.tangential_kind >= 2 ? in.p2 : 0.0;
    }
  }
  // tracks in the prepared point order (the lowering regroups points for locality; point_source maps
  // them back), observations of a track in their input order
  const size_t P = n.points.size() / 3;
  std::vector<size_t> native_of(P);
  for (size_t p = 0; p < P; ++p) native_of[n.point_source[p]] = p;
  q.points.resize(3 * P);
  q.track_off.assign(P + 1, 0);
  for (size_t i = 0; i < P; ++i) {
    const size_t p = native_of[i];
    for (int k = 0; k < 3; ++k) q.points[3 * i + k] = pts[3 * p + k];
    q.track_off[i + 1] = q.track_off[i] + (n.pt_off[p + 1] - n.pt_off[p]);
  }
  q.obs_cam.resize(q.track_off[P]);
  q.obs_px.resize(2 * q.track_off[P]);
  for (size_t i = 0; i < P; ++i) {
    const size_t p = native_of[i];
    uint64_t w = q.track_off[i];
    for (uint64_t o = n.pt_off[p]; o < n.pt_off[p + 1]; ++o, ++w) {
      q.obs_cam[w] = n.obs_cam[o];
      q.obs_px[2 * w] = n.obs_px[2 * o];
      q.obs_px[2 * w + 1] = n.obs_px[2 * o + 1];
    }
  }
  q.fixed_baseline = pr.gauge_kind == OMVGBA_GAUGE_FIXED_BASELINE;
  q.anchor = 0;
  q.scale_camera = (uint64_t)std::max(n.gauge_cam, 0);
  if (q.fixed_baseline) {
    const double* a = q.cameras[0].C;
    const double* b = q.cameras[q.scale_camera].C;
    const double d[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    q.distance = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  }
  q.loss = problem_loss(pr);
  return q;
}

// probe_prepared + native_preflight_from_probe (native/fixed_rotation.rs:50-202)
omvgba_preflight preflight_from_prepared(Context* ctx, const omvgba_problem& pr, const Lowered& L,
                                         const std::vector<double>& rot, const std::vector<double>& tr,
                                         const std::vector<double>& pts) {
  omvgba_probe_options opt;
  probe_options_default(&opt);
  omvgba_probe_report probe;
  try {
    probe = probe_fixed_rotation(ctx, prepared_probe_problem(pr, L, rot, tr, pts), opt);
  } catch (const SolveFailure& f) {
    if (f.code == OMVGBA_INVALID_PROBLEM || f.code == OMVGBA_INVALID_ARGUMENT) fail(OMVGBA_NUMERICAL, f.message);
    throw;
  }
  uint64_t required = 0;
  for (int c = 1; c < L.n.ncam; ++c) required += L.n.fixed_poses[c] ? 0 : 1;
  omvgba_preflight out{};
  out.has_counts = 1;
  out.pose_dimension = probe.pose_dimension;
  out.covered_free_pose_count = probe.covered_free_cameras;
  out.weak_point_count = probe.weak_point_count;
  switch (probe.status) {
    case OMVGBA_PROBE_FULL_RANK_CERTIFIED: out.status = OMVGBA_PREFLIGHT_PROCEED; break;
    case OMVGBA_PROBE_INSUFFICIENT_CAMERA_COVERAGE: out.status = OMVGBA_PREFLIGHT_INSUFFICIENT_CAMERA_COVERAGE; break;
    case OMVGBA_PROBE_RESOURCE_LIMIT: out.status = OMVGBA_PREFLIGHT_RESOURCE_LIMIT; break;
    case OMVGBA_PROBE_WEAK_POINT_GEOMETRY: out.status = OMVGBA_PREFLIGHT_WEAK_POINT_GEOMETRY; break;
    default:
      if (probe.weak_point_count == 0 && probe.covered_free_cameras >= required) {
        out.status = OMVGBA_PREFLIGHT_PROCEED;
        out.dense_observability_escalation = 1;
      } else {
        out.status = OMVGBA_PREFLIGHT_OBSERVABILITY_NOT_CERTIFIED;
      }
  }
  return out;
}

// The probe a translation-only calibrated solve runs on its accepted geometry (native/mod.rs:435-447).
bool wants_post_solve_probe(const omvgba_problem& pr, const NativeProblem& n) {
  bool fixed_points = false;
  for (size_t i = 0; i < pr.point_count && !fixed_points; ++i) fixed_points = point_fixed(pr, i);
  return !n.self_cal && !n.angular && n.translation_only && !fixed_points && n.pixel_model &&
         can_probe_scale_representative(pr) && n.gauge_cam >= 0;
}

// certified_observability and the probe's observability details (native/reporting.rs:24-134).
void apply_preflight(const omvgba_problem& pr, const omvgba_preflight& pf, omvgba_report& r) {
  const bool certifies =
      pf.status == OMVGBA_PREFLIGHT_PROCEED && !pf.dense_observability_escalation && pf.weak_point_count == 0;
  if (r.observability == OMVGBA_OBS_NOT_ASSESSED && certifies)
    r.observability = pr.gauge_kind == OMVGBA_GAUGE_FIXED_BASELINE ? OMVGBA_OBS_FULL_RANK : OMVGBA_OBS_ONLY_EXPECTED_GAUGE;
  const bool ranked = pf.status == OMVGBA_PREFLIGHT_PROCEED &&
                      (!pf.dense_observability_escalation || r.observability == OMVGBA_OBS_FULL_RANK ||
                       r.observability == OMVGBA_OBS_ONLY_EXPECTED_GAUGE);
  if (pf.pose_dimension == 0) fail(OMVGBA_INTERNAL, "bundle-adjustment report is invalid");
  r.has_observability_details = 1;
  r.details_pose_rank = ranked ? pf.pose_dimension : 0;
  r.details_pose_dimension = pf.pose_dimension;
  r.details_weak_point_count = pf.weak_point_count;
}

// NativeBundleAdjuster::preflight (native/mod.rs:184-230)
omvgba_preflight preflight_check(Context* ctx, const omvgba_problem& pr, const omvgba_config& cfg) {
  validate_config(cfg);
  omvgba_preflight none{};
  none.status = OMVGBA_PREFLIGHT_PROCEED;
  bool fixed_points = false;
  for (size_t i = 0; i < pr.point_count && !fixed_points; ++i) fixed_points = point_fixed(pr, i);
  if (common_pose_variables(pr) != 1 || pr.residual_space == OMVGBA_RESIDUAL_ANGULAR || fixed_points) return none;
  if (has_free_intrinsics(pr)) fail(OMVGBA_UNSUPPORTED, "direct native lowering does not support self-calibration");
  Lowered L = lower(pr);
  std::vector<size_t> pose_intr;
  if (L.n.gauge_cam < 0 || !single_pose_intrinsics(pr, &pose_intr) || !can_probe_scale_representative(pr))
    return none;
  std::vector<double> pts(L.n.points.begin(), L.n.points.end());
  return preflight_from_prepared(ctx, pr, L, L.n.rotation, L.n.translation, pts);
}

// ---- two-view solves (native/two_view.rs) --------------------------------------------------------
// unobserved_free_intrinsics (native/mod.rs:465-478): free intrinsic blocks no observation uses; the
// calibrated, angular and two-view solutions report them unconstrained
std::vector<uint64_t> unobserved_free_intrinsics(const omvgba_problem& pr) {
  std::vector<uint8_t> seen(pr.intrinsic_count, 0);
  for (size_t o = 0; o < pr.observation_count; ++o) seen[pr.observation_intrinsic[o]] = 1;
  std::vector<uint64_t> out;
  for (size_t i = 0; i < pr.intrinsic_count; ++i)
    if (!seen[i] && pr.intrinsics[i].variables != 0) out.push_back(i);
  return out;
}

// can_use_two_view (native/two_view.rs:14-48): two poses, the anchor fixed and the other fully
// free, every point seen exactly once by each (no fixed point, no repeated pose-point pair), one
// calibration per pose, and undistorted perspective cameras unless the residuals are angular.
bool can_use_two_view(const omvgba_problem& pr) {
  if (pr.pose_count != 2 || pr.observation_count != 2 * pr.point_count || has_free_intrinsics(pr)) return false;
  for (size_t i = 0; i < pr.point_count; ++i)
    if (point_fixed(pr, i)) return false;
  std::vector<uint8_t> seen(2 * pr.point_count, 0);
  for (size_t o = 0; o < pr.observation_count; ++o) {
    uint8_t& s = seen[2 * pr.observation_point[o] + pr.observation_pose[o]];
    if (s) return false;  // has_repeated_pose_points (native/mod.rs:500-506)
    s = 1;
  }
  std::vector<size_t> intr;
  if (!single_pose_intrinsics(pr, &intr)) return false;
  size_t anchor;
  if (pr.gauge_kind == OMVGBA_GAUGE_FIXED_BASELINE) {
    anchor = pr.gauge_first;
  } else if (pr.poses[0].variables == 0) {
    anchor = 0;
  } else if (pr.poses[1].variables == 0) {
    anchor = 1;
  } else {
    return false;
  }
  if (pr.poses[anchor].variables != 0 || pr.poses[1 - anchor].variables != OMVGBA_POSE_FREE) return false;
  if (pr.residual_space == OMVGBA_RESIDUAL_ANGULAR) return true;
  for (size_t k : intr) {
    const omvgba_intrinsic& in = pr.intrinsics[k];
    const bool undistorted = in.model == OMVGBA_CAMERA_PINHOLE ||
                             (in.model == OMVGBA_CAMERA_BROWN_CONRADY && in.radial_kind == 0 && in.tangential_kind == 0);
    if (!undistorted) return false;
  }
  return true;
}

// solve_two_view (native/two_view.rs:50-185): rebase on the anchor, refine on the device, raise,
// and the two-view report (native/reporting.rs:143-182).
Result solve_two_view(Context* ctx, const omvgba_problem& pr, const omvgba_config& cfg) {
  std::vector<size_t> intr;
  if (!single_pose_intrinsics(pr, &intr)) fail(OMVGBA_UNSUPPORTED, "two-view lowering requires one calibration per pose");
  GaugePlan plan = gauge_plan(pr);
  const size_t var = plan.anchor == 0 ? 1 : 0;
  if (pr.poses[var].variables != OMVGBA_POSE_FREE || pr.poses[plan.anchor].variables != 0)
    fail(OMVGBA_UNSUPPORTED, "direct two-view lowering requires one fixed anchor and one full-pose camera");
  Rebase rb;
  set_anchor(pr, rb, plan.anchor, plan.scale);
  TwoViewProblem tv;
  tv.angular = pr.residual_space == OMVGBA_RESIDUAL_ANGULAR;
  pose_to_native(rb, pr.poses[var], tv.R, tv.t);
  const size_t P = pr.point_count;
  tv.points.resize(3 * P);
  for (size_t i = 0; i < P; ++i) {
    const Vec3 X = point_to_native(rb, point_at(pr, i));
    for (int k = 0; k < 3; ++k) tv.points[3 * i + k] = X[k];
  }
  std::vector<int64_t> at(2 * P, -1);
  for (size_t o = 0; o < pr.observation_count; ++o)
    at[(pr.observation_pose[o] == plan.anchor ? 0 : P) + pr.observation_point[o]] = (int64_t)o;
  if (tv.angular)
    tv.bearing.resize(2 * 3 * P);
  else
    tv.obs.resize(2 * 2 * P);
  for (int v = 0; v < 2; ++v) {
    const omvgba_intrinsic& in = pr.intrinsics[intr[v == 0 ? plan.anchor : var]];
    tv.cam[v][0] = in.fx;
    tv.cam[v][1] = in.fy;
    tv.cam[v][2] = in.cx;
    tv.cam[v][3] = in.cy;
    if (!tv.angular && !(std::isfinite(in.fx) && std::isfinite(in.fy) && std::isfinite(in.cx) && std::isfinite(in.cy) &&
                         in.fx > 0.0 && in.fy > 0.0))
      fail(OMVGBA_NUMERICAL, "two-view bundle adjustment intrinsics are invalid");
    for (size_t i = 0; i < P; ++i) {
      const int64_t o = at[v * P + i];
      if (o < 0) fail(OMVGBA_UNSUPPORTED, "direct two-view lowering requires complete two-view tracks");
      const double u = pr.observation_pixel[2 * o], w = pr.observation_pixel[2 * o + 1];
      if (tv.angular) {
        if (!camera_bearing(in, u, w, &tv.bearing[3 * (v * P + i)]))
          fail(OMVGBA_NUMERICAL, "a measured pixel does not define a bearing of its camera model");
      } else {
        tv.obs[2 * (v * P + i)] = u;
        tv.obs[2 * (v * P + i) + 1] = w;
      }
    }
  }
  LmOptions opt = lm_options(pr, cfg, NativeProblem{});
  TwoViewReport tr = gpu_two_view(ctx, tv, opt);
  Result res;
  res.poses.assign(pr.poses, pr.poses + pr.pose_count);
  pose_from_native(rb, tr.R, tr.t, res.poses[var].rotation, res.poses[var].center);
  res.points.resize(3 * P);
  for (size_t i = 0; i < P; ++i) {
    const Vec3 X = point_from_native(rb, &tv.points[3 * i]);
    if (!all_finite(X.data(), 3)) fail(OMVGBA_NUMERICAL, "native BA returned a non-finite point");
    for (int k = 0; k < 3; ++k) res.points[3 * i + k] = X[k];
  }
  res.intrinsics.assign(pr.intrinsics, pr.intrinsics + pr.intrinsic_count);
  omvgba_report& r = res.report;
  std::memset(&r, 0, sizeof(r));
  r.status = tr.status == 0 ? OMVGBA_STATUS_CONVERGED
                            : (tr.status == 1 ? OMVGBA_STATUS_MAX_ITERATIONS
                                              : (tr.status == 2 ? OMVGBA_STATUS_STALLED : OMVGBA_STATUS_DEGENERATE));
  r.convergence_reason = tr.status == 0 ? tr.reason : OMVGBA_REASON_NONE;
  r.iteration_count = tr.iterations;
  r.initial_objective = tr.initial_cost;
  r.final_objective = tr.final_cost;
  r.initial_rmse = tr.initial_rmse * std::sqrt(2.0);
  r.final_rmse = tr.final_rmse * std::sqrt(2.0);
  r.accepted_step_count = tr.accepted;
  r.rejected_step_count = tr.rej[0] + tr.rej[1] + tr.rej[2] + tr.rej[3];
  r.rejected_linearization = tr.rej[0];
  r.rejected_step_solve = tr.rej[1];
  r.rejected_candidate = tr.rej[2];
  r.rejected_insufficient_reduction = tr.rej[3];
  if (!std::isfinite(tr.grad_norm) || tr.grad_norm < 0.0)
    fail(OMVGBA_NUMERICAL, "stationarity audit requires a finite non-negative gradient norm");
  r.has_stationarity = 1;
  r.scaled_gradient_inf_norm = tr.grad_norm;
  r.observability = tr.rank == 5 ? OMVGBA_OBS_FULL_RANK : OMVGBA_OBS_RANK_DEFICIENT;
  r.has_weak_point_count = 1;
  r.weak_point_count = tr.weak;
  r.has_noninvertible_observation_count = 1;
  r.noninvertible_observation_count = 0;
  r.has_linear_solver = 1;
  r.linear_solver = OMVGBA_SOLVER_DIRECT;
  r.reduced_dimension = 5;
  r.final_damping = tr.final_damping;
  const double vals[4] = {r.initial_objective, r.final_objective, r.initial_rmse, r.final_rmse};
  for (double v : vals)
    if (!std::isfinite(v) || v < 0.0) fail(OMVGBA_INTERNAL, "bundle-adjustment report is invalid");
  res.unconstrained = unobserved_free_intrinsics(pr);
  r.unconstrained_intrinsic_count = res.unconstrained.size();
  return res;
}

// finish = false leaves the report's observation and inlier metrics to the caller: the quarantine
// protocol evaluates them once more over the original problem whenever points are held out.
Result solve_once(Context* ctx, const omvgba_problem& pr, const omvgba_config& cfg, bool finish = true) {
  validate_config(cfg);
  if (!(pr.residual_space != OMVGBA_RESIDUAL_ANGULAR && has_free_intrinsics(pr)) && can_use_two_view(pr)) {
    Result res = solve_two_view(ctx, pr, cfg);
    if (finish) finish_solution(pr, res);
    canonicalize(pr, res);
    return res;
  }
  const auto t0 = std::chrono::steady_clock::now();
  Lowered L = lower(pr);
  const double t_lower = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  LmOptions opt = lm_options(pr, cfg, L.n);
  std::vector<double> rot, tr, pts, grp;
  NativeReport nr = gpu_refine(ctx, L.n, opt, rot, tr, pts, grp);
  std::vector<uint64_t> held;
  if (L.n.self_cal) {
    held = unconstrained_groups(pr, L.n, grp, nr, opt.loss);
    if (!held.empty()) {
      // re-solve from the input state with the unconstrained groups fixed
      // (native/self_calibration.rs:236-249); the second solve is not certified again
      for (uint64_t g : held) L.n.group_dim[g] = 0;
      LmOptions again = lm_options(pr, cfg, L.n);
      again.certify_intrinsics = false;
      nr = gpu_refine(ctx, L.n, again, rot, tr, pts, grp);
    }
  }
  const double t_gpu = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() - t_lower;
  Result res = raise(pr, L, rot, tr, pts, grp, nr, nr.iterative != 0);
  res.unconstrained = L.n.self_cal ? held : unobserved_free_intrinsics(pr);
  res.report.unconstrained_intrinsic_count = res.unconstrained.size();
  if (wants_post_solve_probe(pr, L.n)) apply_preflight(pr, preflight_from_prepared(ctx, pr, L, rot, tr, pts), res.report);
  if (finish) finish_solution(pr, res);
  canonicalize(pr, res);
  if (std::getenv("OMVGBA_PHASE_TIMES"))
    std::fprintf(stderr, "[omvgba] solve_once: lower %.3fs gpu %.3fs raise+finish %.3fs\n", t_lower, t_gpu,
                 std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() - t_lower - t_gpu);
  return res;
}

// ---- quarantine --------------------------------------------------------------------------------
// The k-th smallest of v (k < v.size()), as std::nth_element would place it; v is reordered. Values
// that are all non-negative and not NaN (distances) order like their bit patterns, so a histogram
// of the top 16 bits, taken in parallel, finds the bucket that holds the k-th value, and only that
// bucket is selected from. Anything else takes std::nth_element over the whole vector.
double kth_smallest(std::vector<double>& v, size_t k) {
  const size_t n = v.size();
  constexpr size_t kChunks = 64, kBins = 1 << 16;
  std::vector<uint32_t> hist(kChunks * kBins, 0);
  std::atomic<bool> plain{true};
  for_fixed_chunks(n, kChunks, [&](size_t c, size_t b, size_t e) {
    uint32_t* h = &hist[c * kBins];
    for (size_t i = b; i < e; ++i) {
      if (!(v[i] >= 0.0)) {  // negative or NaN
        plain = false;
        return;
      }
      uint64_t bits;
      std::memcpy(&bits, &v[i], 8);
      h[bits >> 48]++;
    }
  });
  if (!plain || n < (1u << 20)) {
    std::nth_element(v.begin(), v.begin() + k, v.end());
    return v[k];
  }
  size_t below = 0, bucket = 0;
  for (; bucket < kBins; ++bucket) {
    size_t cnt = 0;
    for (size_t c = 0; c < kChunks; ++c) cnt += hist[c * kBins + bucket];
    if (below + cnt > k) break;
    below += cnt;
  }
  std::vector<double> in_bucket;
  for (size_t i = 0; i < n; ++i) {
    uint64_t bits;
    std::memcpy(&bits, &v[i], 8);
    if ((bits >> 48) == bucket) in_bucket.push_back(v[i]);
  }
  std::nth_element(in_bucket.begin(), in_bucket.begin() + (k - below), in_bucket.end());
  return in_bucket[k - below];
}

std::vector<size_t> degenerate_points(const omvgba_problem& pr, const omvgba_pose* poses, const double* points) {
  size_t N = pr.observation_count;
  // the ray from the camera centre to the point (recomputed where it is used, bit for bit)
  auto offset = [&](size_t o) -> Vec3 {
    const size_t p = pr.observation_point[o];
    const double* C = poses[pr.observation_pose[o]].center;
    return {points[3 * p] - C[0], points[3 * p + 1] - C[1], points[3 * p + 2] - C[2]};
  };
  std::vector<double> dist(N);
  for_fixed_chunks(N, 64, [&](size_t, size_t b, size_t e) {
    for (size_t o = b; o < e; ++o) {
      const Vec3 v = offset(o);
      dist[o] = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    }
  });
  const double scene = N > 0 ? kth_smallest(dist, N / 2) : 0.0;
  // each point's observations in input order: the input itself when it is grouped by point in
  // ascending order (a track per point, the usual layout), else a stable counting sort
  const size_t P = pr.point_count;
  std::vector<uint64_t> start(P + 1, 0);
  std::vector<uint64_t> order;
  std::atomic<bool> grouped{true};
  for_fixed_chunks(N, 64, [&](size_t, size_t b, size_t e) {
    for (size_t o = std::max<size_t>(b, 1); o < e; ++o)
      if (pr.observation_point[o] < pr.observation_point[o - 1]) {
        grouped = false;
        return;
      }
  });
  for (size_t o = 0; o < N; ++o) start[pr.observation_point[o] + 1]++;
  for (size_t p = 0; p < P; ++p) start[p + 1] += start[p];
  if (!grouped) {
    order.resize(N);
    std::vector<uint64_t> next(start.begin(), start.end() - 1);
    for (size_t o = 0; o < N; ++o) order[next[pr.observation_point[o]]++] = o;
  }
  std::vector<uint8_t> deg(P, 0);
  for_fixed_chunks(P, 64, [&](size_t, size_t b, size_t e) {
    for (size_t p = b; p < e; ++p) {
      TrackGeometryDev g;
      g.init(scene);
      for (uint64_t i = start[p]; i < start[p + 1]; ++i) {
        const Vec3 v = offset(grouped ? i : order[i]);
        g.push(v[0], v[1], v[2]);
      }
      deg[p] = g.degenerate() ? 1 : 0;
    }
  });
  std::vector<size_t> out;
  for (size_t p = 0; p < P; ++p)
    if (deg[p]) out.push_back(p);
  return out;
}

struct Restricted {
  std::vector<omvgba_pose> poses;
  std::vector<omvgba_intrinsic> intrinsics;
  std::vector<double> points;
  std::vector<uint8_t> fixed;
  FillVector<uint32_t> op, oi, opt;  // written completely by without_points
  FillVector<double> px;
  omvgba_problem view{};
  std::vector<size_t> kept;
};

void without_points(const omvgba_problem& pr, const Result* warm, const std::set<size_t>& dropped, Restricted& r) {
  r.poses.assign(pr.poses, pr.poses + pr.pose_count);
  r.intrinsics.assign(pr.intrinsics, pr.intrinsics + pr.intrinsic_count);
  if (warm) {
    for (size_t i = 0; i < pr.pose_count; ++i) {
      uint32_t v = pr.poses[i].variables;
      r.poses[i] = warm->poses[i];
      r.poses[i].variables = v;
    }
    for (size_t i = 0; i < pr.intrinsic_count; ++i) {
      uint32_t v = pr.intrinsics[i].variables;
      int32_t c = pr.intrinsics[i].certification;
      r.intrinsics[i] = warm->intrinsics[i];
      r.intrinsics[i].variables = v;
      r.intrinsics[i].certification = c;
    }
  }
  std::vector<uint8_t> drop(pr.point_count, 0);
  size_t ndrop = 0;
  for (size_t i : dropped)
    if (i < pr.point_count) {
      drop[i] = 1;
      ++ndrop;
    }
  std::vector<size_t> ni(pr.point_count, SIZE_MAX);
  r.kept.clear();
  r.kept.reserve(pr.point_count - ndrop);
  r.points.reserve(r.points.size() + 3 * (pr.point_count - ndrop));
  r.fixed.reserve(r.fixed.size() + pr.point_count - ndrop);
  for (size_t i = 0; i < pr.point_count; ++i) {
    if (drop[i]) continue;
    ni[i] = r.kept.size();
    r.kept.push_back(i);
    for (int k = 0; k < 3; ++k) r.points.push_back(warm ? warm->points[3 * i + k] : pr.points[3 * i + k]);
    r.fixed.push_back(point_fixed(pr, i) ? 1 : 0);
  }
  // the observations of kept points, in order: per-chunk counts, then each chunk fills its range
  constexpr size_t kChunks = 64;
  std::vector<size_t> at(kChunks + 1, 0);
  for_fixed_chunks(pr.observation_count, kChunks, [&](size_t c, size_t b, size_t e) {
    size_t k = 0;
    for (size_t o = b; o < e; ++o) k += ni[pr.observation_point[o]] != SIZE_MAX;
    at[c + 1] = k;
  });
  for (size_t c = 0; c < kChunks; ++c) at[c + 1] += at[c];
  const size_t base = r.op.size(), M = at[kChunks];
  r.op.resize(base + M);
  r.oi.resize(base + M);
  r.opt.resize(base + M);
  r.px.resize(2 * (base + M));
  for_fixed_chunks(pr.observation_count, kChunks, [&](size_t c, size_t b, size_t e) {
    size_t w = base + at[c];
    for (size_t o = b; o < e; ++o) {
      const size_t q = ni[pr.observation_point[o]];
      if (q == SIZE_MAX) continue;
      r.op[w] = pr.observation_pose[o];
      r.oi[w] = pr.observation_intrinsic[o];
      r.opt[w] = (uint32_t)q;
      r.px[2 * w] = pr.observation_pixel[2 * o];
      r.px[2 * w + 1] = pr.observation_pixel[2 * o + 1];
      ++w;
    }
  });
  r.view = pr;
  r.view.poses = r.poses.data();
  r.view.intrinsics = r.intrinsics.data();
  r.view.point_count = r.kept.size();
  r.view.points = r.points.data();
  r.view.point_fixed = r.fixed.data();
  r.view.observation_count = r.op.size();
  r.view.observation_pose = r.op.data();
  r.view.observation_intrinsic = r.oi.data();
  r.view.observation_point = r.opt.data();
  r.view.observation_pixel = r.px.data();
  validate_problem(r.view);
}

// smallest/largest eigenvalue of a symmetric 3x3 by cyclic Jacobi rotations
void sym3_eigen_extrema(double A[3][3], double* mn, double* mx) {
  for (int sweep = 0; sweep < 50; ++sweep) {
    double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
    if (off < 1e-300) break;
    for (int a = 0; a < 3; ++a)
      for (int b = a + 1; b < 3; ++b) {
        double apq = A[a][b];
        if (std::fabs(apq) < 1e-300) continue;
        double th = (A[b][b] - A[a][a]) / (2.0 * apq);
        double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
        double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 3; ++k) {
          double x = A[k][a], y = A[k][b];
          A[k][a] = c * x - s * y;
          A[k][b] = s * x + c * y;
        }
        for (int k = 0; k < 3; ++k) {
          double x = A[a][k], y = A[b][k];
          A[a][k] = c * x - s * y;
          A[b][k] = s * x + c * y;
        }
      }
  }
  *mx = std::max({A[0][0], A[1][1], A[2][2]});
  *mn = std::min({A[0][0], A[1][1], A[2][2]});
}

std::vector<size_t> weak_points(const omvgba_problem& pr, const Result& sol) {
  LossDev loss = problem_loss(pr);
  size_t P = pr.point_count;
  std::vector<std::array<double, 9>> blocks(P, std::array<double, 9>{});
  std::vector<uint8_t> ok(P, 1);
  for (size_t o = 0; o < pr.observation_count; ++o) {
    size_t p = pr.observation_point[o];
    if (!ok[p]) continue;
    const omvgba_pose& pose = sol.poses[pr.observation_pose[o]];
    Mat3 R = pose_R(pose);
    Vec3 C = pose_C(pose);
    Vec3 xc = rotate(R, {sol.points[3 * p] - C[0], sol.points[3 * p + 1] - C[1], sol.points[3 * p + 2] - C[2]});
    double r[2], J[2][3];
    bool good;
    if (pr.residual_space == OMVGBA_RESIDUAL_ANGULAR) {  // Solution::weak_points (solver.rs:1149-1226)
      double b[3];
      good = camera_bearing(sol.intrinsics[pr.observation_intrinsic[o]], pr.observation_pixel[2 * o],
                            pr.observation_pixel[2 * o + 1], b) &&
             angular_linearize(b, xc.data(), r, J);
    } else {
      FixedCameraDev m = make_fixed_camera(sol.intrinsics[pr.observation_intrinsic[o]]);
      good = m.linearize(xc[0], xc[1], xc[2], pr.observation_pixel[2 * o], pr.observation_pixel[2 * o + 1], r, J);
    }
    double rn = good ? std::hypot(r[0], r[1]) : INFINITY;
    if (!good || !std::isfinite(rn)) {
      ok[p] = 0;
      continue;
    }
    double Jw[2][3];
    for (int a = 0; a < 2; ++a)
      for (int c = 0; c < 3; ++c) Jw[a][c] = J[a][0] * R[0][c] + J[a][1] * R[1][c] + J[a][2] * R[2][c];
    double w = loss.sqrt_weight(rn);
    w *= w;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) blocks[p][3 * i + j] += w * (Jw[0][i] * Jw[0][j] + Jw[1][i] * Jw[1][j]);
  }
  std::vector<uint8_t> deg(P, 0);
  for (auto q : sol.quarantined) deg[q] = 1;
  for (size_t p : degenerate_points(pr, sol.poses.data(), sol.points.data()))
    if (!point_fixed(pr, p)) deg[p] = 1;
  std::vector<size_t> out;
  for (size_t p = 0; p < P; ++p) {
    bool weak = deg[p];
    if (!weak && !point_fixed(pr, p)) {
      if (!ok[p]) {
        weak = true;
      } else {
        double A[3][3];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) A[i][j] = blocks[p][3 * i + j];
        double mn, mx;
        sym3_eigen_extrema(A, &mn, &mx);
        weak = !(mn > 1.0e-5 * mx);
      }
    }
    if (weak) out.push_back(p);
  }
  return out;
}

bool needs_resolve(const Result& r) {
  return (r.report.has_weak_point_count && r.report.weak_point_count > 0) ||
         r.report.observability == OMVGBA_OBS_RANK_DEFICIENT || r.report.status == OMVGBA_STATUS_DEGENERATE;
}

void add_origin(omvgba_report& r, const omvgba_report& origin) {
  r.initial_objective = origin.initial_objective;
  r.initial_rmse = origin.initial_rmse;
  r.iteration_count += origin.iteration_count;
  r.accepted_step_count += origin.accepted_step_count;
  r.rejected_step_count += origin.rejected_step_count;
  r.rejected_linearization += origin.rejected_linearization;
  r.rejected_step_solve += origin.rejected_step_solve;
  r.rejected_candidate += origin.rejected_candidate;
  r.rejected_insufficient_reduction += origin.rejected_insufficient_reduction;
  r.pcg_iteration_count += origin.pcg_iteration_count;
}

// The part of the quarantine protocol before the first solve (quarantine.rs:34-96): points seen
// fewer than twice or without parallax in the input are held out of the problem that is solved.
struct Prepared {
  Restricted first;
  const omvgba_problem* working = nullptr;
  std::vector<size_t> kept;
  size_t quarantined = 0;
  bool changes_scale = false;
};

void prepare_quarantine(const omvgba_problem& pr, const omvgba_config& cfg, Prepared& out) {
  validate_config(cfg);
  std::vector<uint64_t> counts(pr.point_count, 0);
  for (size_t o = 0; o < pr.observation_count; ++o) counts[pr.observation_point[o]]++;
  std::vector<uint8_t> weak(pr.point_count, 0);
  for (size_t p = 0; p < pr.point_count; ++p) weak[p] = counts[p] < 2;
  for (size_t p : degenerate_points(pr, pr.poses, pr.points)) weak[p] = 1;
  std::set<size_t> input_deg;
  for (size_t p = 0; p < pr.point_count; ++p)
    if (weak[p] && !point_fixed(pr, p)) input_deg.insert(p);
  if (input_deg.size() == pr.point_count)
    fail(OMVGBA_UNSUPPORTED, "no point can be adjusted: every point is seen fewer than twice or without parallax");
  out.working = &pr;
  out.kept.resize(pr.point_count);
  std::iota(out.kept.begin(), out.kept.end(), 0);
  if (!input_deg.empty()) {
    without_points(pr, nullptr, input_deg, out.first);
    out.working = &out.first.view;
    out.kept = out.first.kept;
  }
  out.quarantined = input_deg.size();
  out.changes_scale = false;
  if (pr.gauge_kind == OMVGBA_GAUGE_FIXED_BASELINE) out.changes_scale = std::fabs(gauge_plan(pr).scale - 1.0) > 1e-9;
  if (out.changes_scale && out.quarantined > 0)
    fail(OMVGBA_UNSUPPORTED, "native BA cannot change its physical baseline while holding out points");
}

// The rest of the protocol after the first solve `sol` of prep.working: up to four re-solves
// without the weak points of the previous solution, then the solution in the input's indexing.
Result finish_quarantine(Context* ctx, const omvgba_problem& pr, const omvgba_config& cfg, const Prepared& prep,
                         Result sol, InputMetrics* input_cache = nullptr) {
  std::vector<size_t> kept = prep.kept;
  size_t quarantined = prep.quarantined;
  const bool changes_scale = prep.changes_scale;
  omvgba_config retry = cfg;
  retry.max_iterations = std::min<uint64_t>(cfg.max_iterations, 8);
  std::vector<Restricted> chain;
  chain.reserve(4);
  const omvgba_problem* current = prep.working;
  bool have_origin = false;
  omvgba_report origin{};
  for (int round = 0; round < 4; ++round) {
    if (!needs_resolve(sol)) break;
    std::set<size_t> wk;
    for (size_t p : weak_points(*current, sol))
      if (!point_fixed(*current, p)) wk.insert(p);
    if (wk.empty()) break;
    chain.emplace_back();
    Restricted& next = chain.back();
    try {
      without_points(*current, &sol, wk, next);
    } catch (const SolveFailure&) {
      chain.pop_back();
      break;
    }
    Result resolved;
    try {
      resolved = solve_once(ctx, next.view, retry, false);  // held-out points: finished below
    } catch (const SolveFailure& f) {
      if (f.code == OMVGBA_CUDA_ERROR) throw;
      chain.pop_back();
      break;
    }
    std::vector<size_t> nk;
    for (size_t k : next.kept) nk.push_back(kept[k]);
    kept = nk;
    quarantined += wk.size();
    omvgba_report prev = sol.report;
    if (have_origin) add_origin(prev, origin);
    origin = prev;
    have_origin = true;
    sol = resolved;
    current = &next.view;
  }
  if (changes_scale && quarantined > 0)
    fail(OMVGBA_UNSUPPORTED, "native BA cannot change its physical baseline while holding out points");
  if (quarantined == 0) return sol;
  Result out;
  out.poses = sol.poses;
  out.intrinsics = sol.intrinsics;
  out.points.assign(pr.points, pr.points + 3 * pr.point_count);
  std::vector<uint8_t> retained(pr.point_count, 0);
  for (size_t r = 0; r < kept.size(); ++r) {
    retained[kept[r]] = 1;
    for (int k = 0; k < 3; ++k) out.points[3 * kept[r] + k] = sol.points[3 * r + k];
  }
  for (size_t p = 0; p < pr.point_count; ++p)
    if (!retained[p]) out.quarantined.push_back(p);
  out.unconstrained = sol.unconstrained;
  out.report = sol.report;
  if (have_origin) add_origin(out.report, origin);
  finish_solution(pr, out, input_cache);
  return out;
}

double seconds_since(std::chrono::steady_clock::time_point t) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t).count();
}

Result solve_with_quarantine(Context* ctx, const omvgba_problem& pr, const omvgba_config& cfg) {
  const auto t0 = std::chrono::steady_clock::now();
  Prepared prep;
  prepare_quarantine(pr, cfg, prep);
  const double t_prep = seconds_since(t0);
  Result sol = solve_once(ctx, *prep.working, cfg, prep.quarantined == 0);
  const double t_solve = seconds_since(t0) - t_prep;
  Result out = finish_quarantine(ctx, pr, cfg, prep, std::move(sol));
  if (std::getenv("OMVGBA_PHASE_TIMES"))
    std::fprintf(stderr, "[omvgba] host: prepare %.3fs solve_once %.3fs finish %.3fs\n", t_prep, t_solve,
                 seconds_since(t0) - t_prep - t_solve);
  return out;
}

int write_error(omvgba_error* e, int code, const std::string& msg) {
  if (e) {
    e->code = code;
    e->detail = -1;
    std::snprintf(e->message, sizeof(e->message), "%s", msg.c_str());
  }
  return code;
}

}  // namespace
}  // namespace omvgba

struct omvgba_context {
  omvgba::Context* ctx;
};

using namespace omvgba;

struct omvgba_plan {
  Context* ctx = nullptr;
  bool two_view = false;  // solved by the two-view path (no resident multi-view solver)
  const omvgba_problem* problem = nullptr;
  omvgba_config config{};
  Prepared prep;
  Lowered lowered;
  LmOptions options;
  Resident* resident = nullptr;
  InputMetrics input_metrics;  // the held-out report's input-state metrics, kept across solves
  ~omvgba_plan() { resident_destroy(resident); }
};

namespace {

struct Telemetry {
  uint64_t launches = 0, h2d = 0, d2h = 0;
};

Telemetry telemetry_now() {
  Telemetry t;
  telemetry_read(&t.launches, &t.h2d, &t.d2h);
  return t;
}

void stamp_telemetry(omvgba_report& r, const Telemetry& before, std::chrono::steady_clock::time_point t0) {
  const Telemetry after = telemetry_now();
  r.kernel_launches = after.launches - before.launches;
  r.h2d_bytes = after.h2d - before.h2d;
  r.d2h_bytes = after.d2h - before.d2h;
  r.solve_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void write_solution(const omvgba_problem& problem, const Result& r, omvgba_solution* solution) {
  std::memcpy(solution->poses, r.poses.data(), sizeof(omvgba_pose) * problem.pose_count);
  std::memcpy(solution->intrinsics, r.intrinsics.data(), sizeof(omvgba_intrinsic) * problem.intrinsic_count);
  std::memcpy(solution->points, r.points.data(), sizeof(double) * 3 * problem.point_count);
  if (solution->quarantined_points)
    for (size_t i = 0; i < r.quarantined.size(); ++i) solution->quarantined_points[i] = r.quarantined[i];
  if (solution->unconstrained_intrinsics)
    for (size_t i = 0; i < r.unconstrained.size(); ++i) solution->unconstrained_intrinsics[i] = r.unconstrained[i];
  solution->report = r.report;
  solution->report.unconstrained_intrinsic_count = r.unconstrained.size();
}

void clear_error(omvgba_error* error) {
  if (!error) return;
  error->code = 0;
  error->detail = -1;
  error->message[0] = 0;
}

}  // namespace

extern "C" {

uint32_t omvgba_abi_version(void) { return OMVGBA_ABI_VERSION; }
const char* omvgba_adjuster_name(void) { return "openmvg-ba-cuda-b200"; }

void omvgba_config_default(omvgba_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->max_iterations = 50;
  c->function_tolerance = 1.0e-6;
  c->gradient_tolerance = 1.0e-10;
  c->parameter_tolerance = 1.0e-8;
  c->linear_solver = OMVGBA_SOLVER_AUTO;
  c->precision = OMVGBA_PRECISION_FP64;
  c->matvec = OMVGBA_MATVEC_AUTO;
}

// Reports the struct sizes this library was compiled with, so bindings can check their layout.
void omvgba_struct_sizes(uint64_t* out) {
  out[0] = sizeof(omvgba_error);
  out[1] = sizeof(omvgba_pose);
  out[2] = sizeof(omvgba_intrinsic);
  out[3] = sizeof(omvgba_problem);
  out[4] = sizeof(omvgba_config);
  out[5] = sizeof(omvgba_report);
  out[6] = sizeof(omvgba_solution);
}

int32_t omvgba_device_count(void) { return device_count(); }

omvgba_context* omvgba_context_create(int32_t device, omvgba_error* error) {
  std::string msg;
  Context* c = context_create(device, &msg);
  if (!c) {
    write_error(error, OMVGBA_CUDA_ERROR, "context creation failed: " + msg);
    return nullptr;
  }
  if (error) {
    error->code = 0;
    error->message[0] = 0;
  }
  return new omvgba_context{c};
}

void omvgba_context_destroy(omvgba_context* context) {
  if (!context) return;
  context_destroy(context->ctx);
  delete context;
}

int32_t omvgba_solve(omvgba_context* context, const omvgba_problem* problem, const omvgba_config* config,
                     omvgba_solution* solution, omvgba_error* error) {
  if (error) {
    error->code = 0;
    error->detail = -1;
    error->message[0] = 0;
  }
  if (!context || !problem || !config || !solution || !solution->poses || !solution->intrinsics || !solution->points)
    return write_error(error, OMVGBA_INVALID_ARGUMENT, "null argument");
  auto t0 = std::chrono::steady_clock::now();
  try {
    validate_problem(*problem);
    const Telemetry before = telemetry_now();
    Result r = solve_with_quarantine(context->ctx, *problem, *config);
    write_solution(*problem, r, solution);
    stamp_telemetry(solution->report, before, t0);
    if (std::getenv("OMVGBA_PHASE_TIMES")) std::fprintf(stderr, "[omvgba] omvgba_solve %.3fs\n", seconds_since(t0));
    return OMVGBA_OK;
  } catch (const SolveFailure& f) {
    return write_error(error, f.code, f.message);
  } catch (const std::exception& ex) {
    return write_error(error, OMVGBA_INTERNAL, ex.what());
  }
}

void omvgba_probe_options_default(omvgba_probe_options* options) {
  if (options) probe_options_default(options);
}

int32_t omvgba_probe_fixed_rotation(omvgba_context* context, const omvgba_fixed_rotation_problem* problem,
                                    const omvgba_probe_options* options, omvgba_probe_report* report,
                                    omvgba_error* error) {
  clear_error(error);
  if (!context || !problem || !options || !report) return write_error(error, OMVGBA_INVALID_ARGUMENT, "null argument");
  const omvgba_fixed_rotation_problem& fp = *problem;
  const uint64_t nobs = (fp.track_offsets && fp.point_count) ? fp.track_offsets[fp.point_count] : 0;
  if ((fp.camera_count && (!fp.rotations || !fp.centers || !fp.intrinsics || !fp.fixed_cameras)) ||
      (fp.point_count && (!fp.points || !fp.track_offsets)) || (nobs && (!fp.observation_camera || !fp.observation_pixel)))
    return write_error(error, OMVGBA_INVALID_ARGUMENT, "null array");
  try {
    ProbeProblem q;
    q.cameras.resize(fp.camera_count);
    for (uint64_t c = 0; c < fp.camera_count; ++c) {
      ProbeCamera& cam = q.cameras[c];
      std::memcpy(cam.R, fp.rotations + 9 * c, sizeof(cam.R));
      std::memcpy(cam.C, fp.centers + 3 * c, sizeof(cam.C));
      std::memcpy(cam.intrinsics, fp.intrinsics + 9 * c, sizeof(cam.intrinsics));
      cam.fixed = fp.fixed_cameras[c] != 0;
    }
    q.points.assign(fp.points, fp.points + 3 * fp.point_count);
    if (fp.point_count) q.track_off.assign(fp.track_offsets, fp.track_offsets + fp.point_count + 1);
    for (size_t k = 0; k + 1 < q.track_off.size(); ++k)
      if (q.track_off[k + 1] < q.track_off[k] || q.track_off[k + 1] > nobs)
        return write_error(error, OMVGBA_INVALID_PROBLEM, "fixed-rotation BA dimensions are inconsistent");
    q.obs_cam.assign(fp.observation_camera, fp.observation_camera + nobs);
    q.obs_px.assign(fp.observation_pixel, fp.observation_pixel + 2 * nobs);
    q.fixed_baseline = fp.gauge_kind == OMVGBA_GAUGE_FIXED_BASELINE;
    q.anchor = fp.anchor;
    q.scale_camera = fp.scale_camera;
    q.distance = fp.distance;
    if (fp.loss_kind == OMVGBA_LOSS_SQUARED)
      q.loss = {kLossL2, 0.0};
    else if ((fp.loss_kind == OMVGBA_LOSS_HUBER || fp.loss_kind == OMVGBA_LOSS_CAUCHY) && std::isfinite(fp.loss_scale) &&
             fp.loss_scale > 0.0)
      q.loss = {fp.loss_kind == OMVGBA_LOSS_HUBER ? kLossHuber : kLossCauchy, fp.loss_scale};
    else
      return write_error(error, OMVGBA_INVALID_ARGUMENT, "invalid robust loss");
    *report = probe_fixed_rotation(context->ctx, q, *options);
    return OMVGBA_OK;
  } catch (const SolveFailure& f) {
    return write_error(error, f.code, f.message);
  } catch (const std::exception& ex) {
    return write_error(error, OMVGBA_INTERNAL, ex.what());
  }
}

int32_t omvgba_preflight_check(omvgba_context* context, const omvgba_problem* problem, const omvgba_config* config,
                               omvgba_preflight* preflight, omvgba_error* error) {
  clear_error(error);
  if (!context || !problem || !config || !preflight) return write_error(error, OMVGBA_INVALID_ARGUMENT, "null argument");
  try {
    validate_problem(*problem);
    *preflight = preflight_check(context->ctx, *problem, *config);
    return OMVGBA_OK;
  } catch (const SolveFailure& f) {
    return write_error(error, f.code, f.message);
  } catch (const std::exception& ex) {
    return write_error(error, OMVGBA_INTERNAL, ex.what());
  }
}

// Windows solved concurrently by a pool of host threads, each with its own context and stream;
// each window goes through exactly the omvgba_solve path, so its solution is the one omvgba_solve
// returns for it alone, whichever worker takes it.
int32_t omvgba_solve_batched(omvgba_context* context, uint64_t window_count, const omvgba_problem* windows,
                             const omvgba_config* config, omvgba_solution* solutions, omvgba_error* error) {
  clear_error(error);
  if (!context || !config || (window_count > 0 && (!windows || !solutions)))
    return write_error(error, OMVGBA_INVALID_ARGUMENT, "null argument");
  for (uint64_t i = 0; i < window_count; ++i)
    if (!solutions[i].poses || !solutions[i].intrinsics || !solutions[i].points)
      return write_error(error, OMVGBA_INVALID_ARGUMENT, "null solution buffer for window " + std::to_string(i));
  try {
    validate_config(*config);
  } catch (const SolveFailure& f) {
    return write_error(error, f.code, f.message);
  }
  // 16 workers measured best for 256 windows of 5-40 cameras on one B200 (4: 1.9k, 16: 2.3k, 32: 2.1k
  // LM iterations/s); OMVGBA_BATCH_WORKERS overrides it
  uint64_t batch_workers = 16;
  if (const char* w = std::getenv("OMVGBA_BATCH_WORKERS")) batch_workers = std::max(1, std::atoi(w));
  const int device = context_device(context->ctx);
  const uint64_t workers = std::min<uint64_t>(window_count, batch_workers);
  std::vector<int32_t> codes(window_count, OMVGBA_OK);
  std::vector<std::string> messages(window_count);
  std::atomic<uint64_t> next{0};
  std::string setup_error;
  std::mutex setup_mutex;
  omvgba_config cfg = *config;
  cfg.stream = nullptr;  // every worker runs on its own context's stream
  auto worker = [&]() {
    std::string msg;
    Context* ctx = context_create(device, &msg);
    if (!ctx) {
      std::lock_guard<std::mutex> lock(setup_mutex);
      setup_error = "worker context creation failed: " + msg;
      return;
    }
    for (uint64_t i; (i = next.fetch_add(1)) < window_count;) {
      const auto t0 = std::chrono::steady_clock::now();
      try {
        validate_problem(windows[i]);
        const Telemetry before = telemetry_now();
        Result r = solve_with_quarantine(ctx, windows[i], cfg);
        write_solution(windows[i], r, &solutions[i]);
        stamp_telemetry(solutions[i].report, before, t0);
      } catch (const SolveFailure& f) {
        codes[i] = f.code;
        messages[i] = f.message;
      } catch (const std::exception& ex) {
        codes[i] = OMVGBA_INTERNAL;
        messages[i] = ex.what();
      }
    }
    context_destroy(ctx);
  };
  std::vector<std::thread> pool;
  for (uint64_t w = 0; w < workers; ++w) pool.emplace_back(worker);
  for (auto& t : pool) t.join();
  if (!setup_error.empty() && next.load() < window_count) return write_error(error, OMVGBA_CUDA_ERROR, setup_error);
  for (uint64_t i = 0; i < window_count; ++i)
    if (codes[i] != OMVGBA_OK) {
      const int32_t code = write_error(error, codes[i], "window " + std::to_string(i) + ": " + messages[i]);
      if (error) error->detail = (int32_t)i;
      return code;
    }
  return OMVGBA_OK;
}

int32_t omvgba_debug_linearize(omvgba_context* context, const omvgba_problem* problem, const omvgba_config* config,
                               double* residual, double* sqrt_weight, double* point_jacobian, double* camera_jacobian,
                               uint64_t* source_index, omvgba_error* error) {
  if (!context || !problem || !config || !residual || !sqrt_weight || !point_jacobian || !camera_jacobian || !source_index)
    return write_error(error, OMVGBA_INVALID_ARGUMENT, "null argument");
  try {
    validate_problem(*problem);
    validate_config(*config);
    Lowered L = lower(*problem);
    LmOptions opt = lm_options(*problem, *config, L.n);
    gpu_debug_linearize(context->ctx, L.n, opt, residual, sqrt_weight, point_jacobian, camera_jacobian);
    for (size_t o = 0; o < L.n.obs_src.size(); ++o) source_index[o] = L.n.obs_src[o];
    return OMVGBA_OK;
  } catch (const SolveFailure& f) {
    return write_error(error, f.code, f.message);
  }
}

// Debug: digest of the host side of a solve's set-up (quarantine preparation, lowering, block
// tables and matvec tiles) built with at most `threads` host threads (0: all); uses no GPU. Every
// parallel loop of the set-up is arranged so that this does not depend on `threads`.
int32_t omvgba_debug_execution_plan(const omvgba_problem* problem, const omvgba_config* config, int32_t* iterative,
                                    uint64_t* direct_estimate, uint64_t* cached_estimate, omvgba_error* error) {
  clear_error(error);
  if (!problem || !config || !iterative || !direct_estimate || !cached_estimate)
    return write_error(error, OMVGBA_INVALID_ARGUMENT, "null argument");
  try {
    validate_problem(*problem);
    validate_config(*config);
    Prepared prep;
    prepare_quarantine(*problem, *config, prep);
    Lowered L = lower(*prep.working);
    LmOptions opt = lm_options(*prep.working, *config, L.n);
    ExecutionPlan plan = execution_plan(L.n, opt);
    *iterative = plan.iterative ? 1 : 0;
    *direct_estimate = plan.direct_estimate;
    *cached_estimate = plan.cached_estimate;
    return OMVGBA_OK;
  } catch (const SolveFailure& f) {
    return write_error(error, f.code, f.message);
  } catch (const std::exception& ex) {
    return write_error(error, OMVGBA_INTERNAL, ex.what());
  }
}

int32_t omvgba_debug_setup_digest(const omvgba_problem* problem, const omvgba_config* config, uint32_t threads,
                                  uint64_t* digest, omvgba_error* error) {
  clear_error(error);
  if (!problem || !config || !digest) return write_error(error, OMVGBA_INVALID_ARGUMENT, "null argument");
  struct Limit {
    explicit Limit(unsigned t) { set_host_thread_limit(t); }
    ~Limit() { set_host_thread_limit(0); }
  } limit(threads);
  try {
    validate_problem(*problem);
    validate_config(*config);
    Prepared prep;
    prepare_quarantine(*problem, *config, prep);
    const omvgba_problem& w = *prep.working;
    Lowered L = lower(w);
    LmOptions opt = lm_options(w, *config, L.n);
    const NativeProblem& n = L.n;
    uint64_t h = 1469598103934665603ull;
    auto add = [&](const void* p, size_t bytes) { h = fnv1a(p, bytes, h); };
    add(prep.kept.data(), sizeof(size_t) * prep.kept.size());
    add(w.points, sizeof(double) * 3 * w.point_count);
    add(w.observation_pose, sizeof(uint32_t) * w.observation_count);
    add(w.observation_intrinsic, sizeof(uint32_t) * w.observation_count);
    add(w.observation_point, sizeof(uint32_t) * w.observation_count);
    add(w.observation_pixel, sizeof(double) * 2 * w.observation_count);
    add(n.points.data(), sizeof(double) * n.points.size());
    add(n.fixed_points.data(), n.fixed_points.size());
    add(n.pt_off.data(), sizeof(uint64_t) * n.pt_off.size());
    add(n.obs_cam.data(), sizeof(uint32_t) * n.obs_cam.size());
    add(n.obs_px.data(), sizeof(double) * n.obs_px.size());
    add(n.obs_src.data(), sizeof(uint64_t) * n.obs_src.size());
    add(n.point_source.data(), sizeof(uint64_t) * n.point_source.size());
    add(n.rotation.data(), sizeof(double) * n.rotation.size());
    add(n.translation.data(), sizeof(double) * n.translation.size());
    const uint64_t tables = setup_digest(n, opt);
    add(&tables, sizeof(tables));
    *digest = h;
    return OMVGBA_OK;
  } catch (const SolveFailure& f) {
    return write_error(error, f.code, f.message);
  } catch (const std::exception& ex) {
    return write_error(error, OMVGBA_INTERNAL, ex.what());
  }
}

// Debug: the reduced camera system product S_lambda x at the first linearization, by the
// matrix-free kernel (y_matvec) and by the explicit dense Schur complement (y_dense). Call with
// x == NULL to query the dimension into *dimension.
int32_t omvgba_debug_schur_product(omvgba_context* context, const omvgba_problem* problem, const omvgba_config* config,
                                   double lambda, const double* x, double* y_matvec, double* y_dense,
                                   int32_t* dimension, omvgba_error* error) {
  if (!context || !problem || !config || !dimension) return write_error(error, OMVGBA_INVALID_ARGUMENT, "null argument");
  try {
    validate_problem(*problem);
    validate_config(*config);
    Lowered L = lower(*problem);
    LmOptions opt = lm_options(*problem, *config, L.n);
    int d = 0;
    gpu_debug_schur_product(context->ctx, L.n, opt, lambda, x, y_matvec, y_dense, &d);
    *dimension = d;
    return OMVGBA_OK;
  } catch (const SolveFailure& f) {
    return write_error(error, f.code, f.message);
  }
}

int32_t omvgba_plan_create(omvgba_context* context, const omvgba_problem* problem, const omvgba_config* config,
                           omvgba_plan** plan, omvgba_error* error) {
  clear_error(error);
  if (!context || !problem || !config || !plan) return write_error(error, OMVGBA_INVALID_ARGUMENT, "null argument");
  *plan = nullptr;
  try {
    validate_problem(*problem);
    validate_config(*config);
    std::unique_ptr<omvgba_plan> p(new omvgba_plan());
    p->ctx = context->ctx;
    p->problem = problem;
    p->config = *config;
    prepare_quarantine(*problem, p->config, p->prep);
    const omvgba_problem& working = *p->prep.working;
    // a problem omvgba_solve would hand to the two-view solver keeps that route
    p->two_view = !(working.residual_space != OMVGBA_RESIDUAL_ANGULAR && has_free_intrinsics(working)) &&
                  can_use_two_view(working);
    if (!p->two_view) {
      p->lowered = lower(working);
      p->options = lm_options(working, p->config, p->lowered.n);
      p->resident = resident_create(p->ctx, p->lowered.n, p->options);
    }
    *plan = p.release();
    return OMVGBA_OK;
  } catch (const SolveFailure& f) {
    return write_error(error, f.code, f.message);
  } catch (const std::exception& ex) {
    return write_error(error, OMVGBA_INTERNAL, ex.what());
  }
}

int32_t omvgba_plan_solve(omvgba_plan* plan, omvgba_solution* solution, omvgba_error* error) {
  clear_error(error);
  if (!plan || !solution || !solution->poses || !solution->intrinsics || !solution->points)
    return write_error(error, OMVGBA_INVALID_ARGUMENT, "null argument");
  auto t0 = std::chrono::steady_clock::now();
  try {
    const Telemetry before = telemetry_now();
    const omvgba_problem& working = *plan->prep.working;
    if (plan->two_view) {
      Result first = solve_two_view(plan->ctx, working, plan->config);
      if (plan->prep.quarantined == 0) finish_solution(working, first);
      canonicalize(working, first);
      Result r = finish_quarantine(plan->ctx, *plan->problem, plan->config, plan->prep, std::move(first),
                                   &plan->input_metrics);
      write_solution(*plan->problem, r, solution);
      stamp_telemetry(solution->report, before, t0);
      return OMVGBA_OK;
    }
    std::vector<double> rot, tr, pts, grp;
    double laps[6];
    NativeReport nr = resident_refine(plan->resident, rot, tr, pts, grp);
    std::vector<uint64_t> held;
    Lowered held_lowering;
    const Lowered* lowered = &plan->lowered;
    if (plan->lowered.n.self_cal) {
      held = unconstrained_groups(working, plan->lowered.n, grp, nr, plan->options.loss);
      if (!held.empty()) {  // re-solve from the input state with the unconstrained groups fixed
        held_lowering = plan->lowered;
        for (uint64_t g : held) held_lowering.n.group_dim[g] = 0;
        LmOptions again = lm_options(working, plan->config, held_lowering.n);
        again.certify_intrinsics = false;
        nr = gpu_refine(plan->ctx, held_lowering.n, again, rot, tr, pts, grp);
        lowered = &held_lowering;
      }
    }
    laps[0] = seconds_since(t0);
    Result first = raise(working, *lowered, rot, tr, pts, grp, nr, nr.iterative != 0);
    first.unconstrained = lowered->n.self_cal ? held : unobserved_free_intrinsics(working);
    first.report.unconstrained_intrinsic_count = first.unconstrained.size();
    if (wants_post_solve_probe(working, lowered->n))
      apply_preflight(working, preflight_from_prepared(plan->ctx, working, *lowered, rot, tr, pts), first.report);
    laps[1] = seconds_since(t0);
    // with points held out, the quarantine protocol evaluates the report's metrics over the original
    // problem, so the working problem's pass would be discarded
    if (plan->prep.quarantined == 0) finish_solution(working, first);
    laps[2] = seconds_since(t0);
    canonicalize(working, first);
    laps[3] = seconds_since(t0);
    Result r = finish_quarantine(plan->ctx, *plan->problem, plan->config, plan->prep, std::move(first),
                                 &plan->input_metrics);
    laps[4] = seconds_since(t0);
    write_solution(*plan->problem, r, solution);
    laps[5] = seconds_since(t0);
    if (std::getenv("OMVGBA_PHASE_TIMES"))
      std::fprintf(stderr,
                   "[omvgba] plan_solve: refine %.3fs raise %.3fs finish %.3fs canonicalize %.3fs quarantine %.3fs "
                   "write %.3fs\n",
                   laps[0], laps[1] - laps[0], laps[2] - laps[1], laps[3] - laps[2], laps[4] - laps[3],
                   laps[5] - laps[4]);
    stamp_telemetry(solution->report, before, t0);
    return OMVGBA_OK;
  } catch (const SolveFailure& f) {
    return write_error(error, f.code, f.message);
  } catch (const std::exception& ex) {
    return write_error(error, OMVGBA_INTERNAL, ex.what());
  }
}

int32_t omvgba_plan_info_get(const omvgba_plan* plan, omvgba_plan_info* info, omvgba_error* error) {
  clear_error(error);
  if (!plan || !info) return write_error(error, OMVGBA_INVALID_ARGUMENT, "null argument");
  if (plan->two_view) {  // the two-view path keeps no resident multi-view solver
    std::memset(info, 0, sizeof(*info));
    info->observation_count = plan->prep.working->observation_count;
    info->point_count = plan->prep.working->point_count;
    info->camera_count = 2;
    info->reduced_dimension = 5;
    return OMVGBA_OK;
  }
  ResidentInfo r = resident_info(plan->resident);
  std::memset(info, 0, sizeof(*info));
  info->observation_count = r.observations;
  info->point_count = r.points;
  info->camera_count = r.cameras;
  info->reduced_dimension = r.dimension;
  info->jacobian_entries = r.jacobian_entries;
  info->tile_count_fp64 = r.tiles64;
  info->tile_count_fp32 = r.tiles32;
  info->record_bytes_fp64 = r.record_bytes64;
  info->record_bytes_fp32 = r.record_bytes32;
  info->metadata_bytes_fp64 = r.metadata_bytes64;
  info->metadata_bytes_fp32 = r.metadata_bytes32;
  info->iterative = r.iterative;
  info->mixed = r.mixed;
  return OMVGBA_OK;
}

int32_t omvgba_plan_schur_product(omvgba_plan* plan, double lambda, int32_t fp32, int32_t stage, const double* x,
                                  double* y, omvgba_error* error) {
  clear_error(error);
  if (plan && plan->two_view)
    return write_error(error, OMVGBA_UNSUPPORTED, "a two-view plan has no reduced camera product");
  if (!plan || !x || (stage == 0 && !y)) return write_error(error, OMVGBA_INVALID_ARGUMENT, "null argument");
  if (stage < 0 || stage > 3) return write_error(error, OMVGBA_INVALID_ARGUMENT, "stage must be 0, 1, 2 or 3");
  if (!(std::isfinite(lambda) && lambda >= 0.0))
    return write_error(error, OMVGBA_INVALID_ARGUMENT, "lambda must be finite and non-negative");
  try {
    resident_schur_product(plan->resident, lambda, fp32 != 0, stage, x, y);
    return OMVGBA_OK;
  } catch (const SolveFailure& f) {
    return write_error(error, f.code, f.message);
  } catch (const std::exception& ex) {
    return write_error(error, OMVGBA_INTERNAL, ex.what());
  }
}

void omvgba_plan_destroy(omvgba_plan* plan) { delete plan; }

}  // extern "C"

extern "C" int32_t omvgba_sfm_refresh_reprojection(omvgba_context* context, uint64_t pose_count,
                                                   const omvgba_pose* poses, uint64_t intrinsic_count,
                                                   const omvgba_intrinsic* intrinsics,
                                                   const omvgba_landmark_tracks* tracks,
                                                   omvgba_refresh_result* result, omvgba_error* error) {
  clear_error(error);
  if (!context || !tracks || !result || (pose_count && !poses) || (intrinsic_count && !intrinsics))
    return write_error(error, OMVGBA_INVALID_ARGUMENT, "null argument");
  const uint64_t L = tracks->landmark_count;
  if (!tracks->track_offset || (L && (!tracks->points || !tracks->active || !result->landmark_update ||
                                      !result->reprojection_error)))
    return write_error(error, OMVGBA_INVALID_ARGUMENT, "null landmark array");
  try {
    if (tracks->track_offset[0] != 0) fail(OMVGBA_INVALID_PROBLEM, "track offsets must start at zero");
    for (uint64_t l = 0; l < L; ++l)
      if (tracks->track_offset[l + 1] < tracks->track_offset[l])
        fail(OMVGBA_INVALID_PROBLEM, "track offsets must not decrease");
    const uint64_t N = tracks->track_offset[L];
    if (N && (!tracks->track_pose || !tracks->track_intrinsic || !tracks->track_pixel || !tracks->track_support ||
              !result->track_support))
      return write_error(error, OMVGBA_INVALID_ARGUMENT, "null track array");
    std::vector<uint8_t> used(intrinsic_count, 0);
    for (uint64_t o = 0; o < N; ++o) {
      const uint32_t p = tracks->track_pose[o], i = tracks->track_intrinsic[o];
      if (p != OMVGBA_NO_POSE && p >= pose_count) fail(OMVGBA_INVALID_PROBLEM, "track pose index out of range");
      if (i >= intrinsic_count) fail(OMVGBA_INVALID_PROBLEM, "track intrinsic index out of range");
      if (p != OMVGBA_NO_POSE && tracks->track_support[o]) used[i] = 1;
    }
    // CameraResidualPolicy::from_pixel_limit (residual.rs:37-55) fails for a wide-angle camera
    // without a positive finite pixel-to-angle scale
    for (uint64_t i = 0; i < intrinsic_count; ++i) {
      const CameraDev c = make_camera_dev(intrinsics[i]);
      if (used[i] && camera_is_generalized(c) && !std::isfinite(camera_pixels_per_radian(c)))
        fail(OMVGBA_INVALID_PROBLEM, "camera residual policy requires a positive finite pixel-to-angle scale");
    }
    std::vector<double> rot(9 * pose_count), cen(3 * pose_count);
    for (uint64_t p = 0; p < pose_count; ++p) {
      for (int k = 0; k < 9; ++k) rot[9 * p + k] = poses[p].rotation[k];
      for (int k = 0; k < 3; ++k) cen[3 * p + k] = poses[p].center[k];
    }
    SfmRefreshInput in{pose_count, intrinsic_count, L, N, rot.data(), cen.data(), intrinsics, tracks->points,
                       tracks->active, tracks->track_offset, tracks->track_pose, tracks->track_intrinsic,
                       tracks->track_pixel, tracks->track_support};
    SfmRefreshOutput out{result->landmark_update, result->reprojection_error, result->track_support};
    gpu_sfm_refresh(context->ctx, in, out);
    result->rejected_landmarks = out.rejected_landmarks;
    result->removed_observations = out.removed_observations;
    return OMVGBA_OK;
  } catch (const SolveFailure& f) {
    return write_error(error, f.code, f.message);
  } catch (const std::exception& ex) {
    return write_error(error, OMVGBA_INTERNAL, ex.what());
  }
}
