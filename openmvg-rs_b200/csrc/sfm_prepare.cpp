// sfm_prepare.cpp — building the bundle-adjustment problem from an SfM reconstruction's tables
// (prepare_bundle_adjustment_problem, crates/openmvg-sfm/src/ops/reconstruction/bundle.rs:707-989).
//
// The reference walks its workspace's maps; here the workspace arrives as flat tables (views with
// their pose and intrinsic rows, poses, intrinsic groups, landmarks with their tracks) and the
// problem leaves as the C ABI's structure-of-arrays. Ordering follows the reference: poses of the
// registered views in ascending row, the intrinsic groups those views use in ascending row, active
// landmarks not excluded in row order, and each landmark's supporting observations from registered
// views in track order. The observation gather counts per landmark in parallel chunks, then fills
// at prefix-summed offsets, so its output does not depend on the thread count.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ba_cuda.h"

namespace {

struct Failure {
  int32_t code;
  std::string message;
};

[[noreturn]] void fail(int32_t code, const std::string& message) { throw Failure{code, message}; }

bool generalized(const omvgba_intrinsic& c) {
  return c.model == OMVGBA_CAMERA_FISHEYE || c.model == OMVGBA_CAMERA_SPHERICAL;
}

// for_each over [0, n) in fixed chunks on up to hardware_concurrency threads
template <typename F>
void parallel_chunks(size_t n, size_t chunks, F f) {
  chunks = std::max<size_t>(1, std::min(chunks, n));
  const size_t workers = std::max<unsigned>(1, std::min<unsigned>(std::thread::hardware_concurrency(), 32));
  std::vector<std::thread> pool;
  for (size_t w = 0; w < std::min(workers, chunks); ++w)
    pool.emplace_back([&, w]() {
      for (size_t c = w; c < chunks; c += std::min(workers, chunks)) f(c, n * c / chunks, n * (c + 1) / chunks);
    });
  for (auto& t : pool) t.join();
}

struct Tables {
  std::vector<uint32_t> pose_rows, intrinsic_rows, landmark_rows;
  std::vector<uint32_t> pose_index, intrinsic_index;  // workspace row -> problem index (UINT32_MAX: none)
  std::vector<uint32_t> pose_vars;
  std::vector<omvgba_intrinsic> intrinsics;
  std::vector<uint8_t> point_fixed;
  std::vector<uint64_t> obs_offset;  // per kept landmark: its first observation
  int32_t residual_space = OMVGBA_RESIDUAL_PIXELS;
  int32_t loss_kind = OMVGBA_LOSS_SQUARED, loss_space = OMVGBA_RESIDUAL_PIXELS;
  double loss_scale = 0.0;
  int32_t gauge_kind = OMVGBA_GAUGE_FREE;
  uint64_t gauge_first = 0, gauge_second = 0;
  double gauge_distance = 0.0;
};

void validate(const omvgba_sfm_workspace& ws, const omvgba_sfm_prepare_config& cfg) {
  if (cfg.scope < OMVGBA_SCOPE_FULL || cfg.scope > OMVGBA_SCOPE_SELF_CALIBRATION)
    fail(OMVGBA_INVALID_CONFIG, "unknown optimization scope");
  if (cfg.loss_kind < OMVGBA_LOSS_SQUARED || cfg.loss_kind > OMVGBA_LOSS_CAUCHY)
    fail(OMVGBA_INVALID_CONFIG, "unknown robust loss");
  if (cfg.loss_kind != OMVGBA_LOSS_SQUARED && !(std::isfinite(cfg.loss_scale) && cfg.loss_scale > 0.0))
    fail(OMVGBA_INVALID_CONFIG, "robust loss scale must be positive and finite");
  for (uint64_t v = 0; v < ws.view_count; ++v) {
    if (ws.view_pose[v] != OMVGBA_NO_POSE && ws.view_pose[v] >= ws.pose_count)
      fail(OMVGBA_INVALID_PROBLEM, "view pose row out of range");
    if (ws.view_intrinsic[v] >= ws.intrinsic_count) fail(OMVGBA_INVALID_PROBLEM, "view intrinsic row out of range");
  }
  const omvgba_landmark_tracks& lt = ws.landmarks;
  if (lt.landmark_count && (!lt.points || !lt.active || !lt.track_offset))
    fail(OMVGBA_INVALID_PROBLEM, "null landmark array");
  if (lt.track_offset && lt.track_offset[0] != 0) fail(OMVGBA_INVALID_PROBLEM, "track offsets must start at zero");
  for (uint64_t l = 0; l < lt.landmark_count; ++l)
    if (lt.track_offset[l + 1] < lt.track_offset[l]) fail(OMVGBA_INVALID_PROBLEM, "track offsets must not decrease");
  const uint64_t N = lt.track_offset ? lt.track_offset[lt.landmark_count] : 0;
  for (uint64_t o = 0; o < N; ++o)
    if (lt.track_pose[o] >= ws.view_count) fail(OMVGBA_INVALID_PROBLEM, "track view row out of range");
  for (uint64_t i = 0; i < cfg.fixed_view_count; ++i)
    if (cfg.fixed_views[i] >= ws.view_count) fail(OMVGBA_INVALID_PROBLEM, "fixed view row out of range");
  for (uint64_t i = 0; i < cfg.fixed_landmark_count; ++i)
    if (cfg.fixed_landmarks[i] >= lt.landmark_count) fail(OMVGBA_INVALID_PROBLEM, "fixed landmark row out of range");
  for (uint64_t i = 0; i < cfg.excluded_landmark_count; ++i)
    if (cfg.excluded_landmarks[i] >= lt.landmark_count)
      fail(OMVGBA_INVALID_PROBLEM, "excluded landmark row out of range");
}

// Poses (bundle.rs:715-784) and intrinsic groups (:745-846) of the registered views.
void cameras(const omvgba_sfm_workspace& ws, const omvgba_sfm_prepare_config& cfg, Tables& t) {
  std::vector<uint8_t> pose_used(ws.pose_count, 0), intr_used(ws.intrinsic_count, 0), pose_fixed(ws.pose_count, 0);
  for (uint64_t v = 0; v < ws.view_count; ++v)
    if (ws.view_pose[v] != OMVGBA_NO_POSE) {
      pose_used[ws.view_pose[v]] = 1;
      intr_used[ws.view_intrinsic[v]] = 1;
    }
  for (uint64_t i = 0; i < cfg.fixed_view_count; ++i) {
    const uint32_t p = ws.view_pose[cfg.fixed_views[i]];
    if (p == OMVGBA_NO_POSE) fail(OMVGBA_INVALID_PROBLEM, "a fixed view has no pose");
    pose_fixed[p] = 1;
  }
  t.pose_index.assign(ws.pose_count, UINT32_MAX);
  for (uint64_t p = 0; p < ws.pose_count; ++p)
    if (pose_used[p]) {
      t.pose_index[p] = (uint32_t)t.pose_rows.size();
      t.pose_rows.push_back((uint32_t)p);
      uint32_t vars = OMVGBA_POSE_FREE;
      if (pose_fixed[p] || cfg.scope == OMVGBA_SCOPE_POINTS_ONLY)
        vars = 0;
      else if (cfg.scope == OMVGBA_SCOPE_TRANSLATIONS_AND_POINTS)
        vars = OMVGBA_POSE_TRANSLATION;
      t.pose_vars.push_back(vars);
    }
  t.intrinsic_index.assign(ws.intrinsic_count, UINT32_MAX);
  for (uint64_t i = 0; i < ws.intrinsic_count; ++i) {
    if (!intr_used[i]) continue;
    // every view of the group (registered or not) must share one image size
    bool seen = false;
    uint32_t w = 0, h = 0;
    for (uint64_t v = 0; v < ws.view_count; ++v) {
      if (ws.view_intrinsic[v] != i) continue;
      const uint32_t vw = ws.view_size[2 * v], vh = ws.view_size[2 * v + 1];
      if (!seen) {
        w = vw;
        h = vh;
        seen = true;
      } else if (vw != w || vh != h) {
        fail(OMVGBA_INVALID_PROBLEM, "intrinsic " + std::to_string(i) + " is shared by images with different dimensions");
      }
    }
    omvgba_intrinsic c = ws.intrinsics[i];
    c.width = w;
    c.height = h;
    // A spherical or fisheye camera has no intrinsic the pipeline estimates (bundle.rs:810-813)
    const bool fixed = cfg.scope != OMVGBA_SCOPE_SELF_CALIBRATION || generalized(c);
    c.fixed_model = fixed ? 1 : 0;
    c.variables = fixed ? 0u : (OMVGBA_INTRINSIC_FOCAL | OMVGBA_INTRINSIC_RADIAL);
    c.certification = ws.intrinsic_guess && ws.intrinsic_guess[i] ? 1 : 0;
    t.intrinsic_index[i] = (uint32_t)t.intrinsic_rows.size();
    t.intrinsic_rows.push_back((uint32_t)i);
    t.intrinsics.push_back(c);
  }
}

}  // namespace

namespace {

// Points (bundle.rs:847-870) and the observation offsets of the kept landmarks (:871-920).
void landmarks(const omvgba_sfm_workspace& ws, const omvgba_sfm_prepare_config& cfg, Tables& t) {
  const omvgba_landmark_tracks& lt = ws.landmarks;
  std::vector<uint8_t> excluded(lt.landmark_count, 0), fixed(lt.landmark_count, 0);
  for (uint64_t i = 0; i < cfg.excluded_landmark_count; ++i) excluded[cfg.excluded_landmarks[i]] = 1;
  for (uint64_t i = 0; i < cfg.fixed_landmark_count; ++i) fixed[cfg.fixed_landmarks[i]] = 1;
  for (uint64_t l = 0; l < lt.landmark_count; ++l)
    if (lt.active[l] && !excluded[l]) {
      t.landmark_rows.push_back((uint32_t)l);
      t.point_fixed.push_back(fixed[l] || cfg.scope == OMVGBA_SCOPE_POSES_ONLY ? 1 : 0);
    }
  const size_t K = t.landmark_rows.size();
  std::vector<uint64_t> count(K, 0);
  parallel_chunks(K, 256, [&](size_t, size_t b, size_t e) {
    for (size_t k = b; k < e; ++k) {
      const uint32_t l = t.landmark_rows[k];
      uint64_t n = 0;
      for (uint64_t o = lt.track_offset[l]; o < lt.track_offset[l + 1]; ++o)
        n += lt.track_support[o] && ws.view_pose[lt.track_pose[o]] != OMVGBA_NO_POSE ? 1 : 0;
      count[k] = n;
    }
  });
  t.obs_offset.assign(K + 1, 0);
  for (size_t k = 0; k < K; ++k) t.obs_offset[k + 1] = t.obs_offset[k] + count[k];
}

// Gauge (bundle.rs:937-963), residual space (:964-973) and the robust loss in the residual's units
// (mean_radians_per_pixel :991-1004, canonical_robust_loss :1006-1032).
void gauge_and_loss(const omvgba_sfm_workspace& ws, const omvgba_sfm_prepare_config& cfg, Tables& t) {
  t.gauge_kind = cfg.gauge_kind;
  if (cfg.gauge_kind == OMVGBA_GAUGE_FIXED_BASELINE) {
    auto pose_of = [&](uint32_t view) -> uint64_t {
      if (view >= ws.view_count || ws.view_pose[view] == OMVGBA_NO_POSE ||
          t.pose_index[ws.view_pose[view]] == UINT32_MAX)
        fail(OMVGBA_INVALID_PROBLEM, "fixed-baseline anchor is missing");
      return t.pose_index[ws.view_pose[view]];
    };
    t.gauge_first = pose_of(cfg.gauge_first_view);
    t.gauge_second = pose_of(cfg.gauge_second_view);
    t.gauge_distance = cfg.gauge_distance;
  } else if (cfg.gauge_kind != OMVGBA_GAUGE_FREE) {
    fail(OMVGBA_INVALID_CONFIG, "unknown gauge");
  }
  t.residual_space = OMVGBA_RESIDUAL_PIXELS;
  for (const auto& c : t.intrinsics)
    if (generalized(c)) t.residual_space = OMVGBA_RESIDUAL_ANGULAR;
  double sum = 0.0;
  size_t steps = 0;
  for (const auto& c : t.intrinsics) {
    sum += c.model == OMVGBA_CAMERA_SPHERICAL ? 2.0 * 3.141592653589793 / (double)c.width : 1.0 / c.fx;
    ++steps;
  }
  const double radians_per_pixel = sum / (double)std::max<size_t>(steps, 1);
  t.loss_kind = cfg.loss_kind;
  t.loss_scale = cfg.loss_scale;
  t.loss_space = cfg.loss_scale_space;
  if (cfg.loss_kind == OMVGBA_LOSS_SQUARED || cfg.loss_scale_space == t.residual_space) return;
  if (cfg.loss_scale_space != OMVGBA_RESIDUAL_PIXELS)
    fail(OMVGBA_INVALID_PROBLEM, "robust-loss units do not match the BA residual domain");
  const double angular = cfg.loss_scale * radians_per_pixel;
  if (!(std::isfinite(angular) && angular > 0.0)) fail(OMVGBA_INVALID_PROBLEM, "invalid angular loss threshold");
  t.loss_scale = angular;
  t.loss_space = OMVGBA_RESIDUAL_ANGULAR;
}

int32_t write(omvgba_error* e, int32_t code, const std::string& m) {
  if (e) {
    e->code = code;
    e->detail = -1;
    std::snprintf(e->message, sizeof(e->message), "%s", m.c_str());
  }
  return code;
}

}  // namespace

extern "C" int32_t omvgba_sfm_prepare_problem(const omvgba_sfm_workspace* workspace,
                                              const omvgba_sfm_prepare_config* config,
                                              omvgba_sfm_prepared* prepared, omvgba_error* error) {
  if (error) {
    error->code = 0;
    error->detail = -1;
    error->message[0] = 0;
  }
  if (!workspace || !config || !prepared) return write(error, OMVGBA_INVALID_ARGUMENT, "null argument");
  const omvgba_sfm_workspace& ws = *workspace;
  if ((ws.view_count && (!ws.view_pose || !ws.view_intrinsic || !ws.view_size)) || (ws.pose_count && !ws.poses) ||
      (ws.intrinsic_count && !ws.intrinsics))
    return write(error, OMVGBA_INVALID_ARGUMENT, "null workspace table");
  try {
    validate(ws, *config);
    Tables t;
    cameras(ws, *config, t);
    landmarks(ws, *config, t);
    gauge_and_loss(ws, *config, t);
    omvgba_problem& p = prepared->problem;
    const size_t K = t.landmark_rows.size();
    const uint64_t N = t.obs_offset[K];
    const bool sizing = !p.poses;
    p.pose_count = t.pose_rows.size();
    p.intrinsic_count = t.intrinsics.size();
    p.point_count = K;
    p.observation_count = N;
    p.residual_space = t.residual_space;
    p.loss_kind = t.loss_kind;
    p.loss_scale = t.loss_scale;
    p.loss_scale_space = t.loss_space;
    p.gauge_kind = t.gauge_kind;
    p.gauge_first = t.gauge_first;
    p.gauge_second = t.gauge_second;
    p.gauge_distance = t.gauge_distance;
    if (sizing) return 0;
    if ((p.intrinsic_count && !p.intrinsics) || (K && (!p.points || !p.point_fixed)) ||
        (N && (!p.observation_pose || !p.observation_intrinsic || !p.observation_point || !p.observation_pixel)))
      return write(error, OMVGBA_INVALID_ARGUMENT, "null output array");
    omvgba_pose* poses = const_cast<omvgba_pose*>(p.poses);
    for (size_t i = 0; i < t.pose_rows.size(); ++i) {
      poses[i] = ws.poses[t.pose_rows[i]];
      poses[i].variables = t.pose_vars[i];
      if (prepared->pose_rows) prepared->pose_rows[i] = t.pose_rows[i];
    }
    omvgba_intrinsic* intr = const_cast<omvgba_intrinsic*>(p.intrinsics);
    for (size_t i = 0; i < t.intrinsics.size(); ++i) {
      intr[i] = t.intrinsics[i];
      if (prepared->intrinsic_rows) prepared->intrinsic_rows[i] = t.intrinsic_rows[i];
    }
    double* pts = const_cast<double*>(p.points);
    uint8_t* pf = const_cast<uint8_t*>(p.point_fixed);
    uint32_t* op = const_cast<uint32_t*>(p.observation_pose);
    uint32_t* oi = const_cast<uint32_t*>(p.observation_intrinsic);
    uint32_t* ot = const_cast<uint32_t*>(p.observation_point);
    double* ox = const_cast<double*>(p.observation_pixel);
    const omvgba_landmark_tracks& lt = ws.landmarks;
    parallel_chunks(K, 256, [&](size_t, size_t b, size_t e) {
      for (size_t k = b; k < e; ++k) {
        const uint32_t l = t.landmark_rows[k];
        for (int c = 0; c < 3; ++c) pts[3 * k + c] = lt.points[3 * (size_t)l + c];
        pf[k] = t.point_fixed[k];
        if (prepared->landmark_rows) prepared->landmark_rows[k] = l;
        uint64_t w = t.obs_offset[k];
        for (uint64_t o = lt.track_offset[l]; o < lt.track_offset[l + 1]; ++o) {
          const uint32_t v = lt.track_pose[o];
          if (!lt.track_support[o] || ws.view_pose[v] == OMVGBA_NO_POSE) continue;
          op[w] = t.pose_index[ws.view_pose[v]];
          oi[w] = t.intrinsic_index[ws.view_intrinsic[v]];
          ot[w] = (uint32_t)k;
          ox[2 * w] = lt.track_pixel[2 * o];
          ox[2 * w + 1] = lt.track_pixel[2 * o + 1];
          ++w;
        }
      }
    });
    return 0;
  } catch (const Failure& f) {
    return write(error, f.code, f.message);
  } catch (const std::exception& ex) {
    return write(error, OMVGBA_INTERNAL, ex.what());
  }
}
