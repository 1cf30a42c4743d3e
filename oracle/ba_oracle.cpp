// ba_oracle.cpp — TEST INFRASTRUCTURE ONLY: a CPU restatement of openmvg-rs `openmvg-ba`'s native
// Levenberg–Marquardt bundle adjustment (NativeBundleAdjuster::solve), used as the parity checker
// for the GPU solver and as the timed CPU baseline ("port"). It is never linked into the shipped
// library. Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs use it.
//
// Parity pins: the Rust reference cannot be built here (no toolchain), so this restatement is pinned
// against the reference's unit-test known answers and central differences (tests/test_oracle_pins.py)
// and against fixtures it generated itself (tests/golden/).
//
// File map (reference paths relative to the openmvg-rs root):
//   lowering .......... native/mod.rs:235-367, native/gauge.rs:123-330, native/world_rebase.rs:19-87,
//                       native/calibrated.rs:200-494, native/self_calibration.rs:47-198
//   quarantine ........ quarantine.rs:34-96, native/mod.rs:260-340, solver.rs:1149-1226
//   assembly .......... schur/point.rs:176-448, schur/assembly.rs:691-1069
//   camera step ....... sparse/calibrated/camera_step.rs:152-266, sparse/direct.rs:235-283,
//                       sparse/pcg.rs:23-157, sparse/retained/mod.rs:620-934, retained/block.rs:148-246
//   candidate ......... sparse/calibrated/candidate.rs:23-333, schur/point.rs:537-728,
//                       kernel/multi_view/optimizer.rs:380-702, self_calibration/optimizer.rs:565-587
//   LM driver ......... sparse/calibrated/mod.rs:169-589, sparse/self_calibration/mod.rs:212-640
//   final certificate . sparse/direct.rs:288-460, schur/diagnostics.rs:18-140
//   report/solution ... native/reporting.rs:24-141, solver.rs:803-1131
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <set>
#include <string>
#include <vector>

#include "../include/ba_cuda.h"
#include "oracle_core.hpp"
#include "fixed_rotation_probe.hpp"

// Phase timer printed to stderr when OMVGBA_ORACLE_TIMES is set (diagnostics only).
static double oracle_now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
static void oracle_phase(const char* what, double t0) {
  static const bool on = std::getenv("OMVGBA_ORACLE_TIMES") != nullptr;
  if (on) std::fprintf(stderr, "[oracle] %s %.3fs\n", what, oracle_now() - t0);
}

#ifdef _OPENMP
#include <omp.h>
#endif

namespace oracle {

struct SolveFailure {
  int code;
  std::string message;
};

struct NPose {
  Mat3 R;
  Vec3 t;
};

// ------------------------------------------------------------------------------------------
// Lowered ("native") problem.
// ------------------------------------------------------------------------------------------
struct Native {
  bool self_cal = false;
  int ncam = 0;
  std::vector<NPose> poses;
  std::vector<Vec3> points;
  std::vector<uint8_t> fixed_points;
  std::vector<uint8_t> fixed_poses;  // native camera order
  // Calibrated solves carry explicit per-camera pose masks (native camera order; bit 0 rotation, bit 1
  // translation, 0 fixed): the block of camera c has 3 rotation and 3 (2 on the baseline camera)
  // translation coordinates as its mask allows, camera 0 included
  // (workspace/topology.rs:305-347). Self-calibration keeps the legacy layout: camera 0 fixed, every
  // other camera full or fixed (topology.rs:364-380).
  bool explicit_masks = false;
  std::vector<uint8_t> pose_mask;
  bool translation_only = false;  // CameraPoseVariables::TranslationOnly (calibrated)
  bool angular = false;           // angular residuals (native/calibrated.rs:27-123)
  std::vector<Vec3> obs_bearing;  // per observation: the measured pixel's bearing
  std::vector<uint32_t> obs_cam;
  std::vector<Vec2> obs_px;
  std::vector<uint64_t> obs_src;
  std::vector<uint32_t> obs_model;  // calibrated: fixed camera model per observation
  std::vector<uint64_t> pt_off;
  bool pixel_model = true;  // Pixel (pinhole, 64 eps depth floor) versus full Brown–Conrady model
  std::vector<BrownConrady> models;
  std::vector<Radial> groups;
  std::vector<uint32_t> cam_group;
  std::vector<int> group_dim;
  int gauge_cam = -1;
  Mat3 anchor_R;
  Vec3 anchor_C;
  double scale = 1.0;
  std::vector<size_t> camera_source_order;
};

struct Layout {
  int D = 0;
  std::vector<int> pose_off, pose_dim;  // per camera
  std::vector<int> intr_off, intr_dim;  // per group (self-calibration)
  std::vector<int> block_off, block_dim;
  std::vector<int> param_block;
  std::vector<int> param_camera;  // camera owning each pose parameter, -1 for intrinsic parameters
};

struct GaugeState {
  int fixed_camera = -1;
  double baseline = 0.0, scene_scale = 1.0;
  Vec3 direction{};
  std::array<Vec3, 2> basis{};
};

// GaugeState::new (schur/layout.rs:79-125), FixedBaseline and Free only.
static GaugeState make_gauge(const Native& n, const std::vector<NPose>& poses, double scene) {
  GaugeState g;
  g.scene_scale = scene;
  if (n.gauge_cam >= 0) {
    g.fixed_camera = n.gauge_cam;
    const Vec3& t = poses[n.gauge_cam].t;
    g.baseline = norm3(t);
    g.direction = {t[0] / g.baseline, t[1] / g.baseline, t[2] / g.baseline};
    g.basis = s2_tangent_basis(g.direction);
  }
  return g;
}

static Layout make_layout(const Native& n) {
  Layout L;
  L.pose_off.resize(n.ncam);
  L.pose_dim.resize(n.ncam);
  int off = 0;
  for (int c = 0; c < n.ncam; ++c) {
    int d;
    if (n.explicit_masks) {
      const int m = n.pose_mask[c];
      d = (n.fixed_poses[c] || m == 0) ? 0 : 3 * (m & 1) + ((m & 2) ? (c == n.gauge_cam ? 2 : 3) : 0);
    } else {
      d = (c == 0 || n.fixed_poses[c]) ? 0 : (c == n.gauge_cam ? 5 : 6);
    }
    L.pose_off[c] = off;
    L.pose_dim[c] = d;
    off += d;
  }
  if (n.self_cal) {
    L.intr_off.resize(n.groups.size());
    L.intr_dim.resize(n.groups.size());
    for (size_t g = 0; g < n.groups.size(); ++g) {
      L.intr_off[g] = off;
      L.intr_dim[g] = n.group_dim[g];
      off += n.group_dim[g];
    }
  }
  L.D = off;
  L.param_block.assign(off, -1);
  L.param_camera.assign(off, -1);
  for (int c = 0; c < n.ncam; ++c)
    if (L.pose_dim[c] > 0) {
      int b = (int)L.block_off.size();
      L.block_off.push_back(L.pose_off[c]);
      L.block_dim.push_back(L.pose_dim[c]);
      for (int k = 0; k < L.pose_dim[c]; ++k) {
        L.param_block[L.pose_off[c] + k] = b;
        L.param_camera[L.pose_off[c] + k] = c;
      }
    }
  for (size_t g = 0; g < L.intr_dim.size(); ++g)
    if (L.intr_dim[g] > 0) {
      int b = (int)L.block_off.size();
      L.block_off.push_back(L.intr_off[g]);
      L.block_dim.push_back(L.intr_dim[g]);
      for (int k = 0; k < L.intr_dim[g]; ++k) L.param_block[L.intr_off[g] + k] = b;
    }
  return L;
}

// ------------------------------------------------------------------------------------------
// Observation model (kernel/multi_view/model.rs:287-317, self_calibration/model.rs:143-160).
// ------------------------------------------------------------------------------------------
struct ObsLin {
  Projection p;
  bool has_intr = false;
  Mat23 jint{};
};
static bool project_obs(const Native& n, const std::vector<Radial>& groups, size_t o, const Vec3& xc,
                        ObsLin* out) {
  if (n.self_cal) {
    const Radial& cam = groups[n.cam_group[n.obs_cam[o]]];
    auto t = radial_terms(cam, xc);
    if (!t) return false;
    auto pr = radial_projection(cam, n.obs_px[o], *t);
    if (!pr) return false;
    auto ji = radial_intrinsic_jacobian(cam, *t);
    if (!ji) return false;
    out->p = *pr;
    out->has_intr = true;
    out->jint = *ji;
    return true;
  }
  if (n.angular) {  // ObservationModel::project, Angular (kernel/multi_view/model.rs:287-292)
    auto pr = angular_projection(n.obs_bearing[o], xc);
    if (!pr) return false;
    out->p = *pr;
    out->has_intr = false;
    return true;
  }
  const BrownConrady& m = n.models[n.obs_model[o]];
  std::optional<Projection> pr =
      n.pixel_model ? pixel_projection(m.fx, m.fy, m.cx, m.cy, n.obs_px[o], xc) : m.project_with_jacobian(n.obs_px[o], xc);
  if (!pr) return false;
  out->p = *pr;
  out->has_intr = false;
  return true;
}

// ------------------------------------------------------------------------------------------
// Hessian accumulators (schur/assembly.rs:25-160).
// ------------------------------------------------------------------------------------------
struct Hessian {
  // dense == true: full D x D matrix; otherwise block diagonal + pose/intrinsic edges.
  bool dense = false;
  int D = 0;
  std::vector<double> S;  // dense
  const Layout* L = nullptr;
  const Native* N = nullptr;
  std::vector<std::vector<double>> blocks;       // per parameter block, dim x dim full
  std::vector<std::vector<double>> edges;        // per camera: pose_dim x intr_dim (self-cal)
  std::vector<int> edge_cam_of_group_param;      // unused helper
  bool valid = true;
  void init_dense(int d) {
    dense = true;
    D = d;
    S.assign((size_t)d * d, 0.0);
  }
  void init_blocks(const Layout& l, const Native& n) {
    dense = false;
    L = &l;
    N = &n;
    D = l.D;
    blocks.assign(l.block_off.size(), {});
    for (size_t b = 0; b < l.block_off.size(); ++b) blocks[b].assign((size_t)l.block_dim[b] * l.block_dim[b], 0.0);
    edges.assign(n.ncam, {});
    if (n.self_cal)
      for (int c = 0; c < n.ncam; ++c) {
        int g = n.cam_group[c];
        if (l.pose_dim[c] > 0 && l.intr_dim[g] > 0) edges[c].assign((size_t)l.pose_dim[c] * l.intr_dim[g], 0.0);
      }
  }
  void clear() {
    valid = true;
    if (dense)
      std::fill(S.begin(), S.end(), 0.0);
    else {
      for (auto& b : blocks) std::fill(b.begin(), b.end(), 0.0);
      for (auto& e : edges) std::fill(e.begin(), e.end(), 0.0);
    }
  }
  // row >= column is not required; adds value at (row, col) and (col, row)
  void add_symmetric(int row, int col, double v) {
    if (dense) {
      S[(size_t)row * D + col] += v;
      if (row != col) S[(size_t)col * D + row] += v;
      return;
    }
    int br = L->param_block[row], bc = L->param_block[col];
    if (br == bc) {
      int o = L->block_off[br], d = L->block_dim[br];
      blocks[br][(size_t)(row - o) * d + (col - o)] += v;
      if (row != col) blocks[br][(size_t)(col - o) * d + (row - o)] += v;
      return;
    }
    // pose/intrinsic edge: find the camera owning the pose parameter
    int pose_param = row, intr_param = col;
    if (row >= L->intr_off.front()) std::swap(pose_param, intr_param);
    const int cam = L->param_camera[pose_param];
    if (cam < 0) {
      valid = false;
      return;
    }
    int g = N->cam_group[cam];
    int pi = pose_param - L->pose_off[cam], ii = intr_param - L->intr_off[g];
    if (edges[cam].empty()) {
      valid = false;
      return;
    }
    edges[cam][(size_t)pi * L->intr_dim[g] + ii] += v;
  }
  bool finite() const {
    if (!valid) return false;
    if (dense) {
      for (double v : S)
        if (!std::isfinite(v)) return false;
      return true;
    }
    for (auto& b : blocks)
      for (double v : b)
        if (!std::isfinite(v)) return false;
    for (auto& e : edges)
      for (double v : e)
        if (!std::isfinite(v)) return false;
    return true;
  }
};

// Per-point caches kept by assembly for the camera step and the candidate.
struct PointCache {
  std::vector<uint8_t> valid;
  std::vector<std::array<double, 6>> vhat;   // damped V packed lower (00,10,11,20,21,22)
  std::vector<PointBlockFactor> factor;
  std::vector<Vec3> inv_grad;                // Vhat^-1 g_p
  std::vector<Vec3> damp_diag;               // damping diagonal
  std::vector<uint64_t> row_off;             // per point into rows
  std::vector<int> row_param;                // active parameter index
  std::vector<Vec3> row_y;                   // Vhat^-1 W row for that parameter
};

struct Assembly {
  bool valid = true;
  uint64_t weak = 0;
  double min_rcond = 1.0;
  double grad_norm = 0.0;
  double point_red = 0.0;
  double cost = 0.0, sq = 0.0;
  double min_diag = 0.0, max_diag = 0.0;
  uint64_t clamp_count = 0;
};

struct Workspace {
  std::vector<double> grad, full_grad, diag;
  Hessian H;
  PointCache cache;
};

// pose_motion (schur/point.rs:730-762)
static void pose_motion(const Vec3& r, int cam, const GaugeState& g, double m[3][6]) {
  double base[3][6] = {{0.0, r[2], -r[1], 0, 0, 0}, {-r[2], 0.0, r[0], 0, 0, 0}, {r[1], -r[0], 0.0, 0, 0, 0}};
  std::memcpy(m, base, sizeof(base));
  if (g.fixed_camera == cam) {
    for (int c = 0; c < 3; ++c) {
      m[c][3] = g.baseline * g.basis[0][c];
      m[c][4] = g.baseline * g.basis[1][c];
    }
  } else {
    for (int c = 0; c < 3; ++c) m[c][3 + c] = g.scene_scale;
  }
}

// The pose columns of one observation's camera Jacobian (schur/point.rs:286-313): a block without
// rotation moves only its translation (translation_motion, point.rs:764-786); a block with rotation
// uses pose_motion at the rotated point RX, or, when the translation is held, at the camera point
// RX + t, since then the camera turns about its fixed centre. J is the 2 x 3 projection Jacobian.
static int pose_columns(const Native& n, const Layout& L, const GaugeState& g, int cam, const Vec3& rot,
                        const Vec3& xc, const Mat23& J, double Jc[2][9]) {
  const int pd = L.pose_dim[cam];
  if (pd == 0) return 0;
  const int mask = n.explicit_masks ? n.pose_mask[cam] : 3;
  double m[3][6];
  if (!(mask & 1)) {
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 6; ++c) m[r][c] = 0.0;
    if (g.fixed_camera == cam) {
      for (int c = 0; c < 3; ++c) {
        m[c][0] = g.baseline * g.basis[0][c];
        m[c][1] = g.baseline * g.basis[1][c];
      }
    } else {
      for (int c = 0; c < 3; ++c) m[c][c] = g.scene_scale;
    }
  } else {
    pose_motion((mask & 2) ? rot : xc, cam, g, m);
  }
  for (int r = 0; r < 2; ++r)
    for (int c = 0; c < pd; ++c) Jc[r][c] = J[r][0] * m[0][c] + J[r][1] * m[1][c] + J[r][2] * m[2][c];
  return pd;
}

// Shard-local assembly output, combined in shard order (retained/parallel.rs:15-31).
struct ShardOut {
  std::vector<double> grad, full_grad, diag;
  Hessian H;
  Assembly a;
};

static void assemble_range(const Native& n, const std::vector<NPose>& poses, const std::vector<Vec3>& points,
                           const std::vector<Radial>& groups, const Layout& L, const GaugeState& g,
                           const Loss& loss, double lambda, bool materialize, size_t p0, size_t p1, ShardOut& out,
                           PointCache& cache) {
  std::vector<Vec3> cross(L.D, Vec3{0, 0, 0});
  std::vector<uint8_t> marks(L.D, 0);
  std::vector<int> active;
  active.reserve(64);
  Assembly& a = out.a;
  for (size_t p = p0; p < p1; ++p) {
    // linearize_point_with_hessian_and_active (schur/point.rs:176-236)
    Mat3 V{};
    Vec3 gp{0, 0, 0};
    double cost = 0.0, sq = 0.0;
    bool ok = true;
    active.clear();
    const Vec3& X = points[p];
    for (uint64_t o = n.pt_off[p]; o < n.pt_off[p + 1]; ++o) {
      int cam = n.obs_cam[o];
      const NPose& P = poses[cam];
      Vec3 rot = rotate(P.R, X);
      Vec3 xc = {rot[0] + P.t[0], rot[1] + P.t[1], rot[2] + P.t[2]};
      ObsLin ol;
      if (!project_obs(n, groups, o, xc, &ol)) {
        ok = false;
        break;
      }
      // accumulate_observation (schur/point.rs:239-355)
      double rn = std::sqrt(ol.p.residual[0] * ol.p.residual[0] + ol.p.residual[1] * ol.p.residual[1]);
      double sw = loss.sqrt_weight(rn);
      Mat23 Jp;
      for (int r = 0; r < 2; ++r)
        for (int c = 0; c < 3; ++c)
          Jp[r][c] = (ol.p.jacobian[r][0] * P.R[0][c] + ol.p.jacobian[r][1] * P.R[1][c] + ol.p.jacobian[r][2] * P.R[2][c]) *
                     g.scene_scale;
      cost += loss.cost(rn);
      sq += rn * rn;
      for (int r = 0; r < 2; ++r) {  // accumulate_point (schur/point.rs:357-372)
        double wr = sw * ol.p.residual[r];
        double wp[3] = {sw * Jp[r][0], sw * Jp[r][1], sw * Jp[r][2]};
        for (int i = 0; i < 3; ++i) {
          gp[i] += wp[i] * wr;
          for (int j = 0; j < 3; ++j) V[i][j] += wp[i] * wp[j];
        }
      }
      int pd = L.pose_dim[cam];
      int grp = n.self_cal ? (int)n.cam_group[cam] : -1;
      int id = (grp >= 0) ? L.intr_dim[grp] : 0;
      if (pd == 0 && id == 0) continue;
      double Jc[2][9] = {};
      int params[9];
      if (pd > 0) {
        pose_columns(n, L, g, cam, rot, xc, ol.p.jacobian, Jc);
        for (int k = 0; k < pd; ++k) params[k] = L.pose_off[cam] + k;
      }
      if (id > 0) {
        for (int r = 0; r < 2; ++r)
          for (int c = 0; c < id; ++c) Jc[r][pd + c] = ol.jint[r][c];
        for (int k = 0; k < id; ++k) params[pd + k] = L.intr_off[grp] + k;
      }
      int cd = pd + id;
      // ActiveParameterTracker::register (schur/layout.rs:229-250)
      int runs[2][2] = {{0, pd}, {pd, cd}};
      for (auto& run : runs) {
        if (run[1] == run[0]) continue;
        int start = params[run[0]];
        if (marks[start]) continue;
        marks[start] = 1;
        for (int k = run[0]; k < run[1]; ++k) {
          active.push_back(params[k]);
          cross[params[k]] = {0, 0, 0};
        }
      }
      // accumulate_camera (schur/point.rs:380-448)
      double first[9], second[9];
      for (int k = 0; k < cd; ++k) {
        first[k] = sw * Jc[0][k];
        second[k] = sw * Jc[1][k];
      }
      double pf[3] = {sw * Jp[0][0], sw * Jp[0][1], sw * Jp[0][2]};
      double ps[3] = {sw * Jp[1][0], sw * Jp[1][1], sw * Jp[1][2]};
      for (int k = 0; k < cd; ++k) {
        Vec3& t = cross[params[k]];
        for (int i = 0; i < 3; ++i) {
          t[i] += pf[i] * first[k];
          t[i] += ps[i] * second[k];
        }
      }
      double res[2] = {sw * ol.p.residual[0], sw * ol.p.residual[1]};
      for (int k = 0; k < cd; ++k) {
        int q = params[k];
        out.grad[q] += first[k] * res[0];
        out.grad[q] += second[k] * res[1];
        out.full_grad[q] += first[k] * res[0];
        out.full_grad[q] += second[k] * res[1];
        out.diag[q] += first[k] * first[k];
        out.diag[q] += second[k] * second[k];
      }
      // add_gram over runs: run0 x run0 (lower), run1 x run0, run1 x run1 (lower)
      for (int ri = 0; ri < 2; ++ri) {
        if (runs[ri][1] == runs[ri][0]) continue;
        for (int ci = 0; ci < ri; ++ci) {
          if (runs[ci][1] == runs[ci][0]) continue;
          for (int i = runs[ri][0]; i < runs[ri][1]; ++i)
            for (int j = runs[ci][0]; j < runs[ci][1]; ++j) {
              out.H.add_symmetric(params[i], params[j], first[i] * first[j]);
              out.H.add_symmetric(params[i], params[j], second[i] * second[j]);
            }
        }
        for (int i = runs[ri][0]; i < runs[ri][1]; ++i)
          for (int j = runs[ri][0]; j <= i; ++j) {
            out.H.add_symmetric(params[i], params[j], first[i] * first[j]);
            out.H.add_symmetric(params[i], params[j], second[i] * second[j]);
          }
      }
    }
    for (int q : active) marks[q] = 0;
    cache.valid[p] = 0;
    if (!ok) {
      a.valid = false;
      continue;
    }
    // assemble_with_hessian_problem_impl point body (schur/assembly.rs:893-1040)
    a.cost += cost;
    a.sq += sq;
    if (n.fixed_points[p]) continue;
    {
      double scale = std::max({0.0, V[0][0], V[1][1], V[2][2]});
      double gn;
      if (!(std::isfinite(scale) && scale > 0.0)) {
        gn = (gp[0] == 0.0 && gp[1] == 0.0 && gp[2] == 0.0) ? 0.0 : kInf;
      } else {
        double fl = 64.0 * kEps * scale;
        gn = 0.0;
        for (int i = 0; i < 3; ++i) gn = std::max(gn, std::fabs(gp[i]) / std::sqrt(std::max(V[i][i], fl)));
      }
      a.grad_norm = std::max(a.grad_norm, gn);
    }
    auto f = point_block_factor(V, lambda);
    if (!f) {
      a.valid = false;
      if (lambda == 0.0) {
        a.weak++;
        a.min_rcond = 0.0;
      }
      continue;
    }
    auto dd = damping_diagonal(V);
    auto dm = damped_matrix(V, lambda);
    if (!dd || !dm) {
      a.valid = false;
      continue;
    }
    cache.damp_diag[p] = *dd;
    cache.vhat[p] = {(*dm)[0][0], (*dm)[1][0], (*dm)[1][1], (*dm)[2][0], (*dm)[2][1], (*dm)[2][2]};
    cache.factor[p] = *f;
    if (lambda == 0.0) {
      double rc = point_rcond(*f, V);
      a.min_rcond = std::min(a.min_rcond, rc);
      if (rc <= kPointBlockRcondThreshold) a.weak++;
    }
    Vec3 ig = f->solve(gp);
    a.point_red += 0.5 * dot3(gp, ig);
    cache.inv_grad[p] = ig;
    cache.valid[p] = 1;
    uint64_t ro = cache.row_off[p];
    uint64_t cap = cache.row_off[p + 1] - ro;
    if (active.size() > cap) {
      a.valid = false;
      cache.valid[p] = 0;
      continue;
    }
    std::vector<Vec3> yrows(active.size());
    for (size_t i = 0; i < active.size(); ++i) {
      int q = active[i];
      out.grad[q] -= dot3(cross[q], ig);
      yrows[i] = f->solve(cross[q]);
      cache.row_param[ro + i] = q;
      cache.row_y[ro + i] = yrows[i];
    }
    for (size_t i = active.size(); i < cap; ++i) cache.row_param[ro + i] = -1;
    if (materialize)
      for (size_t i = 0; i < active.size(); ++i)
        for (size_t j = 0; j <= i; ++j) out.H.add_symmetric(active[i], active[j], -dot3(yrows[i], cross[active[j]]));
  }
}

static int g_forced_shards = 0;  // test hook: a different (still fixed) summation grouping

struct Solver {
  const Native& n;
  Layout L;
  int nshards = 1;
  std::vector<size_t> shard_begin;
  explicit Solver(const Native& nat) : n(nat), L(make_layout(nat)) {
    // Topology-defined contiguous point shards: at most 32, about 8192 observations each.
    size_t P = n.points.size();
    size_t obs = n.obs_cam.size();
    size_t want = std::max<size_t>(1, std::min<size_t>(32, (obs + 8191) / 8192));
    if (g_forced_shards > 0) want = std::min<size_t>((size_t)g_forced_shards, std::max<size_t>(P, 1));
    shard_begin.push_back(0);
    for (size_t s = 1; s < want; ++s) {
      uint64_t target = obs * s / want;
      size_t p = std::lower_bound(n.pt_off.begin(), n.pt_off.end(), target) - n.pt_off.begin();
      p = std::min(std::max(p, shard_begin.back()), P);
      shard_begin.push_back(p);
    }
    shard_begin.push_back(P);
    nshards = (int)shard_begin.size() - 1;
  }

  // Full assembly; materialize: dense S (Direct), else block storage (retained PCG).
  Assembly assemble(const std::vector<NPose>& poses, const std::vector<Vec3>& points, const std::vector<Radial>& groups,
                    const GaugeState& g, const Loss& loss, double lambda, bool materialize, Workspace& ws) {
    int D = L.D;
    size_t P = points.size();
    auto& c = ws.cache;
    if (c.valid.size() != P) {
      c.valid.assign(P, 0);
      c.vhat.assign(P, {});
      c.factor.assign(P, {});
      c.inv_grad.assign(P, {});
      c.damp_diag.assign(P, {});
      c.row_off.assign(P + 1, 0);
      for (size_t p = 0; p < P; ++p) {
        // capacity: every observation can add one pose run and one intrinsic run
        uint64_t cap = 0;
        for (uint64_t o = n.pt_off[p]; o < n.pt_off[p + 1]; ++o) cap += 9;
        c.row_off[p + 1] = c.row_off[p] + cap;
      }
      c.row_param.assign(c.row_off[P], -1);
      c.row_y.assign(c.row_off[P], {});
    }
    std::vector<ShardOut> shards(nshards);
    for (auto& s : shards) {
      s.grad.assign(D, 0.0);
      s.full_grad.assign(D, 0.0);
      s.diag.assign(D, 0.0);
      if (materialize)
        s.H.init_dense(D);
      else
        s.H.init_blocks(L, n);
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int s = 0; s < nshards; ++s)
      assemble_range(n, poses, points, groups, L, g, loss, lambda, materialize, shard_begin[s], shard_begin[s + 1],
                     shards[s], c);
    ws.grad.assign(D, 0.0);
    ws.full_grad.assign(D, 0.0);
    ws.diag.assign(D, 0.0);
    if (materialize)
      ws.H.init_dense(D);
    else
      ws.H.init_blocks(L, n);
    Assembly a;
    for (int s = 0; s < nshards; ++s) {  // fixed shard order
      auto& so = shards[s];
      for (int i = 0; i < D; ++i) {
        ws.grad[i] += so.grad[i];
        ws.full_grad[i] += so.full_grad[i];
        ws.diag[i] += so.diag[i];
      }
      if (materialize)
        for (size_t i = 0; i < so.H.S.size(); ++i) ws.H.S[i] += so.H.S[i];
      else {
        for (size_t b = 0; b < so.H.blocks.size(); ++b)
          for (size_t i = 0; i < so.H.blocks[b].size(); ++i) ws.H.blocks[b][i] += so.H.blocks[b][i];
        for (size_t e = 0; e < so.H.edges.size(); ++e)
          for (size_t i = 0; i < so.H.edges[e].size(); ++i) ws.H.edges[e][i] += so.H.edges[e][i];
      }
      ws.H.valid = ws.H.valid && so.H.valid;
      a.valid = a.valid && so.a.valid;
      a.weak += so.a.weak;
      a.min_rcond = std::min(a.min_rcond, so.a.min_rcond);
      a.grad_norm = std::max(a.grad_norm, so.a.grad_norm);
      a.point_red += so.a.point_red;
      a.cost += so.a.cost;
      a.sq += so.a.sq;
    }
    // finalize_assembly (schur/assembly.rs:691-727)
    double scale = 0.0, mn = kInf;
    for (int i = 0; i < D; ++i) {
      scale = std::max(scale, ws.diag[i]);
      mn = std::min(mn, ws.diag[i]);
    }
    a.min_diag = D == 0 ? 0.0 : mn;
    a.max_diag = scale;
    a.clamp_count = 0;
    for (size_t b = 0; b < L.block_off.size(); ++b) {  // clamp_damping_block, pose blocks then intrinsic
      int o = L.block_off[b], d = L.block_dim[b];
      double s = 0.0;
      for (int k = 0; k < d; ++k) s = std::max(s, ws.diag[o + k]);
      double fl = s > 0.0 ? 64.0 * kEps * s : 1.0;
      for (int k = 0; k < d; ++k)
        if (ws.diag[o + k] < fl) {
          ws.diag[o + k] = fl;
          a.clamp_count++;
        }
    }
    for (int i = 0; i < D; ++i) ws.H.add_symmetric(i, i, lambda * ws.diag[i]);
    double gn = 0.0;
    for (int i = 0; i < D; ++i) {
      double cv = ws.diag[i], v = ws.full_grad[i];
      double t = (std::isfinite(cv) && cv > 0.0) ? std::fabs(v) / std::sqrt(cv) : (v == 0.0 ? 0.0 : kInf);
      gn = std::max(gn, t);
    }
    a.grad_norm = std::max(a.grad_norm, gn);
    bool gf = true;
    for (int i = 0; i < D; ++i) gf = gf && std::isfinite(ws.grad[i]);
    a.valid = a.valid && ws.H.finite() && gf;
    return a;
  }

  // Dense Cholesky (stands in for faer's sparse LLT; exact to rounding).
  static bool cholesky(std::vector<double>& A, int D) {
    for (int j = 0; j < D; ++j) {
      double s = A[(size_t)j * D + j];
      for (int k = 0; k < j; ++k) s -= A[(size_t)j * D + k] * A[(size_t)j * D + k];
      if (!(std::isfinite(s) && s > 0.0)) return false;
      double d = std::sqrt(s);
      A[(size_t)j * D + j] = d;
#pragma omp parallel for schedule(static) if (D > 256)
      for (int i = j + 1; i < D; ++i) {
        double v = A[(size_t)i * D + j];
        for (int k = 0; k < j; ++k) v -= A[(size_t)i * D + k] * A[(size_t)j * D + k];
        A[(size_t)i * D + j] = v / d;
      }
    }
    return true;
  }
  static void cholesky_solve(const std::vector<double>& Lf, int D, std::vector<double>& x) {
    for (int i = 0; i < D; ++i) {
      double v = x[i];
      for (int k = 0; k < i; ++k) v -= Lf[(size_t)i * D + k] * x[k];
      x[i] = v / Lf[(size_t)i * D + i];
    }
    for (int i = D - 1; i >= 0; --i) {
      double v = x[i];
      for (int k = i + 1; k < D; ++k) v -= Lf[(size_t)k * D + i] * x[k];
      x[i] = v / Lf[(size_t)i * D + i];
    }
  }

  // Retained operator y = S_lambda x (retained/operator.rs:137-227): U_lambda blocks and edges minus
  // the point coupling through cached Vhat^-1 W rows.
  void apply_operator(const Workspace& ws, const std::vector<double>& x, std::vector<double>& y) const {
    int D = L.D;
    y.assign(D, 0.0);
    const Hessian& H = ws.H;
    for (size_t b = 0; b < L.block_off.size(); ++b) {
      int o = L.block_off[b], d = L.block_dim[b];
      for (int i = 0; i < d; ++i) {
        double s = 0.0;
        for (int j = 0; j < d; ++j) s += H.blocks[b][(size_t)i * d + j] * x[o + j];
        y[o + i] += s;
      }
    }
    if (n.self_cal)
      for (int c = 0; c < n.ncam; ++c) {
        if (H.edges[c].empty()) continue;
        int g = n.cam_group[c];
        int pd = L.pose_dim[c], id = L.intr_dim[g], po = L.pose_off[c], io = L.intr_off[g];
        for (int i = 0; i < pd; ++i)
          for (int j = 0; j < id; ++j) {
            double e = H.edges[c][(size_t)i * id + j];
            y[po + i] += e * x[io + j];
            y[io + j] += e * x[po + i];
          }
      }
    std::vector<std::vector<double>> part(nshards, std::vector<double>(D, 0.0));
#pragma omp parallel for schedule(dynamic, 1)
    for (int s = 0; s < nshards; ++s) {
      auto& yp = part[s];
      const auto& c = ws.cache;
      for (size_t p = shard_begin[s]; p < shard_begin[s + 1]; ++p) {
        if (!c.valid[p]) continue;
        Vec3 z{0, 0, 0};
        for (uint64_t r = c.row_off[p]; r < c.row_off[p + 1] && c.row_param[r] >= 0; ++r)
          for (int i = 0; i < 3; ++i) z[i] += c.row_y[r][i] * x[c.row_param[r]];
        const auto& v = c.vhat[p];
        Vec3 w = {v[0] * z[0] + v[1] * z[1] + v[3] * z[2], v[1] * z[0] + v[2] * z[1] + v[4] * z[2],
                  v[3] * z[0] + v[4] * z[1] + v[5] * z[2]};
        for (uint64_t r = c.row_off[p]; r < c.row_off[p + 1] && c.row_param[r] >= 0; ++r)
          yp[c.row_param[r]] -= dot3(c.row_y[r], w);
      }
    }
    for (int s = 0; s < nshards; ++s)
      for (int i = 0; i < D; ++i) y[i] += part[s][i];
  }

  // Block-Jacobi factors of the exact diagonal blocks of S (retained/mod.rs:904-934).
  struct BlockFactor {
    std::vector<double> lower, scale;
    int d = 0;
  };
  bool factor_blocks(const Workspace& ws, std::vector<BlockFactor>& out) const {
    size_t nb = L.block_off.size();
    std::vector<std::vector<double>> coupling(nb);
    for (size_t b = 0; b < nb; ++b) coupling[b].assign((size_t)L.block_dim[b] * L.block_dim[b], 0.0);
    const auto& c = ws.cache;
    for (size_t p = 0; p < n.points.size(); ++p) {
      if (!c.valid[p]) continue;
      const auto& v = c.vhat[p];
      for (uint64_t r = c.row_off[p]; r < c.row_off[p + 1] && c.row_param[r] >= 0; ++r)
        for (uint64_t q = c.row_off[p]; q <= r; ++q) {
          int pr = c.row_param[r], pq = c.row_param[q];
          int b = L.param_block[pr];
          if (L.param_block[pq] != b) continue;
          const Vec3& a = c.row_y[r];
          const Vec3& z = c.row_y[q];
          Vec3 w = {v[0] * z[0] + v[1] * z[1] + v[3] * z[2], v[1] * z[0] + v[2] * z[1] + v[4] * z[2],
                    v[3] * z[0] + v[4] * z[1] + v[5] * z[2]};
          double val = dot3(a, w);
          int d = L.block_dim[b], o = L.block_off[b];
          int i = pr - o, j = pq - o;
          coupling[b][(size_t)i * d + j] += val;
          if (i != j) coupling[b][(size_t)j * d + i] += val;
        }
    }
    out.assign(nb, {});
    for (size_t b = 0; b < nb; ++b) {
      int d = L.block_dim[b];
      std::vector<double> m(ws.H.blocks[b]);
      for (size_t i = 0; i < m.size(); ++i) m[i] -= coupling[b][i];
      // PackedCameraBlockFactor::factor (retained/block.rs:171-218)
      BlockFactor& f = out[b];
      f.d = d;
      f.lower.assign((size_t)d * d, 0.0);
      f.scale.assign(d, 0.0);
      double ds = 0.0;
      for (int i = 0; i < d; ++i) ds = std::max(ds, m[(size_t)i * d + i]);
      if (!(std::isfinite(ds) && ds > 0.0)) return false;
      double fl = 64.0 * kEps * ds;
      for (int i = 0; i < d; ++i) f.scale[i] = std::sqrt(std::max(m[(size_t)i * d + i], fl));
      for (int r = 0; r < d; ++r)
        for (int cc = 0; cc <= r; ++cc) {
          double val = m[(size_t)r * d + cc] / (f.scale[r] * f.scale[cc]);
          for (int k = 0; k < cc; ++k) val -= f.lower[(size_t)r * d + k] * f.lower[(size_t)cc * d + k];
          if (r == cc) {
            if (!(std::isfinite(val) && val > 64.0 * kEps)) return false;
            f.lower[(size_t)r * d + cc] = std::sqrt(val);
          } else {
            f.lower[(size_t)r * d + cc] = val / f.lower[(size_t)cc * d + cc];
          }
        }
    }
    return true;
  }
  void apply_preconditioner(const std::vector<BlockFactor>& fs, const std::vector<double>& r,
                            std::vector<double>& z) const {
    z.assign(L.D, 0.0);
    for (size_t b = 0; b < fs.size(); ++b) {
      const auto& f = fs[b];
      int o = L.block_off[b], d = f.d;
      double s[9];
      for (int i = 0; i < d; ++i) {
        double v = r[o + i] / f.scale[i];
        for (int k = 0; k < i; ++k) v -= f.lower[(size_t)i * d + k] * s[k];
        s[i] = v / f.lower[(size_t)i * d + i];
      }
      for (int i = d - 1; i >= 0; --i) {
        double v = s[i];
        for (int k = i + 1; k < d; ++k) v -= f.lower[(size_t)k * d + i] * s[k];
        s[i] = v / f.lower[(size_t)i * d + i];
      }
      for (int i = 0; i < d; ++i) z[o + i] = s[i] / f.scale[i];
    }
  }

  struct PcgResult {
    bool accepted = false;
    uint64_t terms = 0;
    double relative_residual = std::nan("");
  };
  static double dotv(const std::vector<double>& a, const std::vector<double>& b) {
    double s = 0.0;
    for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
    return s;
  }
  // pcg::solve (sparse/pcg.rs:23-119) with require_bounded_residual = true
  PcgResult pcg(const Workspace& ws, const std::vector<BlockFactor>& fs, uint64_t max_it, double tol,
                std::vector<double>& x) const {
    int D = L.D;
    PcgResult res;
    x.assign(D, 0.0);
    std::vector<double> r(D), z(D), d(D), q(D);
    for (int i = 0; i < D; ++i) r[i] = -ws.grad[i];
    double n0 = std::sqrt(dotv(r, r));
    if (!std::isfinite(n0)) return res;
    if (n0 == 0.0) {
      res.accepted = true;
      res.relative_residual = 0.0;
      return res;
    }
    apply_preconditioner(fs, r, z);
    d = z;
    double rho = dotv(r, z);
    if (!(std::isfinite(rho) && rho > 0.0)) return res;
    auto recompute = [&]() {
      apply_operator(ws, x, q);
      for (int i = 0; i < D; ++i) r[i] = -ws.grad[i] - q[i];
    };
    for (uint64_t it = 1; it <= max_it; ++it) {
      apply_operator(ws, d, q);
      double curv = dotv(d, q);
      if (!(std::isfinite(curv) && curv > 0.0)) {
        res.terms = it - 1;
        return res;
      }
      double alpha = rho / curv;
      if (!std::isfinite(alpha)) {
        res.terms = it - 1;
        return res;
      }
      for (int i = 0; i < D; ++i) {
        x[i] += alpha * d[i];
        r[i] -= alpha * q[i];
      }
      double ratio = std::sqrt(dotv(r, r)) / n0;
      if (!std::isfinite(ratio)) {
        res.terms = it;
        return res;
      }
      if (ratio <= tol) {
        recompute();
        double tr = std::sqrt(dotv(r, r)) / n0;
        if (std::isfinite(tr) && tr <= tol) {
          res.accepted = true;
          res.terms = it;
          res.relative_residual = tr;
          return res;
        }
        if (!std::isfinite(tr)) {
          res.terms = it;
          return res;
        }
        apply_preconditioner(fs, r, z);
        d = z;
        rho = dotv(r, z);
        if (!(std::isfinite(rho) && rho > 0.0)) {
          res.terms = it;
          res.relative_residual = tr;
          return res;
        }
        continue;
      }
      apply_preconditioner(fs, r, z);
      double nrho = dotv(r, z);
      if (!(std::isfinite(nrho) && nrho > 0.0)) {
        res.terms = it;
        return res;
      }
      double beta = nrho / rho;
      if (!std::isfinite(beta)) {
        res.terms = it;
        return res;
      }
      for (int i = 0; i < D; ++i) d[i] = z[i] + beta * d[i];
      rho = nrho;
    }
    recompute();
    double rr = std::sqrt(dotv(r, r)) / n0;
    res.terms = max_it;
    res.relative_residual = rr;
    return res;  // require_bounded_residual: rejected
  }
};

// ------------------------------------------------------------------------------------------
// Candidate evaluation (sparse/calibrated/candidate.rs:23-333, schur/point.rs:586-728).
// ------------------------------------------------------------------------------------------
static std::optional<double> admitted_point_cost(const Native& n, const std::vector<NPose>& poses,
                                                 const std::vector<Radial>& groups, const Vec3& X, size_t p,
                                                 const Loss& loss, double scene, Admission adm) {
  double total = 0.0;
  TrackGeometry geo(scene);
  for (uint64_t o = n.pt_off[p]; o < n.pt_off[p + 1]; ++o) {
    const NPose& P = poses[n.obs_cam[o]];
    Vec3 r = rotate(P.R, X);
    Vec3 xc = {r[0] + P.t[0], r[1] + P.t[1], r[2] + P.t[2]};
    ObsLin ol;
    if (!project_obs(n, groups, o, xc, &ol)) return std::nullopt;
    geo.push(rotate_transposed(P.R, xc));
    double rn = std::sqrt(ol.p.residual[0] * ol.p.residual[0] + ol.p.residual[1] * ol.p.residual[1]);
    total += loss.cost(rn);
  }
  if (!admits(adm, geo)) return std::nullopt;
  return total;
}

struct CandidatePoint {
  Vec3 position;
  double cost;
  bool moved;
};
// candidate_rule (point_geometry.rs:110-130)
static std::optional<CandidatePoint> candidate_point(const Native& n, const std::vector<NPose>& cur,
                                                     const std::vector<Radial>& cur_groups,
                                                     const std::vector<NPose>& cand,
                                                     const std::vector<Radial>& cand_groups, const Vec3& prev,
                                                     const Vec3& stepped, size_t p, const Loss& loss, double scene) {
  if (auto m = admitted_point_cost(n, cand, cand_groups, stepped, p, loss, scene, Admission::Geometry))
    return CandidatePoint{stepped, *m, true};
  auto held = admitted_point_cost(n, cand, cand_groups, prev, p, loss, scene, Admission::Collapse);
  if (!held) {
    if (admitted_point_cost(n, cur, cur_groups, prev, p, loss, scene, Admission::Collapse)) return std::nullopt;
    held = admitted_point_cost(n, cand, cand_groups, prev, p, loss, scene, Admission::Projection);
    if (!held) return std::nullopt;
  }
  return CandidatePoint{prev, *held, false};
}

// ------------------------------------------------------------------------------------------
// LM driver (sparse/calibrated/mod.rs:169-589; sparse/self_calibration/mod.rs:212-640).
// ------------------------------------------------------------------------------------------
struct Options {
  uint64_t max_iterations;
  Loss loss;
  Criteria criteria;
  bool iterative;
  double pcg_tol;
  uint64_t pcg_max;
  bool certify_intrinsics = true;  // self-calibration: compute the intrinsic marginal covariances
};

struct NativeReport {
  int status;  // run_state status
  Criterion reason;
  uint64_t iterations, accepted, rejected, rej[4];
  double initial_cost, initial_rmse, final_cost, final_rmse;
  double gradient_inf_norm;
  int rank;  // 0 full, 1 expected gauge, 2 deficient, 3 not assessed
  uint64_t weak;
  uint64_t noninvertible;
  uint64_t pcg_terms;
  double final_damping;
  int D;
  std::vector<double> marginals;  // self-calibration: (S^-1)_gg per group, 9 values (row-major corner)
  bool marginals_ok = false;
};

// ------------------------------------------------------------------------------------------
// Explicit reduced camera system in a band, its Cholesky factor, and the intrinsic marginal
// covariances of the final undamped system (stands in for faer's sparse LLT, numerics/sparse.rs:119-250;
// sparse/direct.rs:288-330 factors S for the rank, sparse/covariance.rs:564-587 solves S x = e_p for
// the marginals). Parameters are ordered camera by camera -- each pose block, then the intrinsic
// blocks it introduces -- which keeps the reduced system of a survey in a narrow band.
// ------------------------------------------------------------------------------------------
static bool g_certificate = true;  // test hook: timing runs skip the final certificate's factorization

// Wall time of every LM iteration of the calling thread's last solve (the bench's per-iteration CPU
// rate); each refine appends its iterations.
thread_local std::vector<double> tl_iteration_seconds;

struct Band {
  int n = 0, w = 0;
  std::vector<double> a;  // row i, column j (i - w <= j <= i) at a[i (w + 1) + (i - j)]
  double& at(int i, int j) { return a[(size_t)i * (w + 1) + (i - j)]; }
  double at(int i, int j) const { return a[(size_t)i * (w + 1) + (i - j)]; }
};

// Position of every parameter in the factorization order.
static std::vector<int> factor_order(const Native& n, const Layout& L) {
  std::vector<int> pos(L.D, 0);
  std::vector<int> home(L.intr_dim.size(), -1);
  if (n.self_cal)
    for (int c = n.ncam - 1; c >= 0; --c) home[n.cam_group[c]] = c;
  int at = 0;
  auto place_group = [&](size_t g) {
    for (int k = 0; k < L.intr_dim[g]; ++k) pos[L.intr_off[g] + k] = at++;
  };
  for (int c = 0; c < n.ncam; ++c) {
    for (int k = 0; k < L.pose_dim[c]; ++k) pos[L.pose_off[c] + k] = at++;
    for (size_t g = 0; g < L.intr_dim.size(); ++g)
      if (home[g] == c) place_group(g);
  }
  for (size_t g = 0; g < L.intr_dim.size(); ++g)
    if (home[g] < 0) place_group(g);
  return pos;
}

// Per point of the final state: the weighted camera rows of each observation and the point's
// coupling terms, added into the rows of the band that [r0, r1) owns (lower triangle in the
// factorization order). Every element receives its terms in point order, observation order.
static void band_point_terms(const Native& n, const Layout& L, const std::vector<NPose>& poses,
                             const std::vector<Vec3>& points, const std::vector<Radial>& groups, const GaugeState& g,
                             const Loss& loss, const std::vector<int>& pos, size_t p, int r0, int r1, Band& B) {
  struct ObsRows {
    int cd;
    int params[9];
    double first[9], second[9];
  };
  std::vector<ObsRows> rows;
  std::vector<int> qs;
  std::vector<Vec3> cross;
  Mat3 V{};
  const Vec3& X = points[p];
  for (uint64_t o = n.pt_off[p]; o < n.pt_off[p + 1]; ++o) {
    const int cam = n.obs_cam[o];
    const NPose& P = poses[cam];
    Vec3 rot = rotate(P.R, X);
    Vec3 xc = {rot[0] + P.t[0], rot[1] + P.t[1], rot[2] + P.t[2]};
    ObsLin ol;
    if (!project_obs(n, groups, o, xc, &ol)) return;
    const double rn = std::sqrt(ol.p.residual[0] * ol.p.residual[0] + ol.p.residual[1] * ol.p.residual[1]);
    const double sw = loss.sqrt_weight(rn);
    Mat23 Jp;
    for (int r = 0; r < 2; ++r)
      for (int c = 0; c < 3; ++c)
        Jp[r][c] = (ol.p.jacobian[r][0] * P.R[0][c] + ol.p.jacobian[r][1] * P.R[1][c] + ol.p.jacobian[r][2] * P.R[2][c]) *
                   g.scene_scale;
    for (int r = 0; r < 2; ++r)
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) V[i][j] += (sw * Jp[r][i]) * (sw * Jp[r][j]);
    const int pd = L.pose_dim[cam];
    const int grp = n.self_cal ? (int)n.cam_group[cam] : -1;
    const int id = grp >= 0 ? L.intr_dim[grp] : 0;
    if (pd == 0 && id == 0) continue;
    ObsRows orow{};
    double Jc[2][9] = {};
    if (pd > 0) {
      pose_columns(n, L, g, cam, rot, xc, ol.p.jacobian, Jc);
      for (int k = 0; k < pd; ++k) orow.params[k] = L.pose_off[cam] + k;
    }
    for (int r = 0; r < 2; ++r)
      for (int c = 0; c < id; ++c) Jc[r][pd + c] = ol.jint[r][c];
    for (int k = 0; k < id; ++k) orow.params[pd + k] = L.intr_off[grp] + k;
    orow.cd = pd + id;
    for (int k = 0; k < orow.cd; ++k) {
      orow.first[k] = sw * Jc[0][k];
      orow.second[k] = sw * Jc[1][k];
      const int q = orow.params[k];
      size_t at = 0;
      while (at < qs.size() && qs[at] != q) ++at;
      if (at == qs.size()) {
        qs.push_back(q);
        cross.push_back({0, 0, 0});
      }
      for (int i = 0; i < 3; ++i) cross[at][i] += (sw * Jp[0][i]) * orow.first[k] + (sw * Jp[1][i]) * orow.second[k];
    }
    rows.push_back(orow);
  }
  auto add = [&](int a, int b, double v) {
    int P = pos[a], Q = pos[b];
    if (P < Q) std::swap(P, Q);
    if (P >= r0 && P < r1) B.at(P, Q) += v;
  };
  for (const ObsRows& r : rows)
    for (int i = 0; i < r.cd; ++i)
      for (int j = 0; j <= i; ++j) add(r.params[i], r.params[j], r.first[i] * r.first[j] + r.second[i] * r.second[j]);
  if (n.fixed_points[p]) return;
  auto f = point_block_factor(V, 0.0);
  if (!f) return;
  std::vector<Vec3> y(qs.size());
  for (size_t i = 0; i < qs.size(); ++i) y[i] = f->solve(cross[i]);
  for (size_t i = 0; i < qs.size(); ++i)
    for (size_t j = 0; j <= i; ++j) add(qs[i], qs[j], -dot3(y[i], cross[j]));
}

// S of the final undamped state in the band; false when a projection or a point factor fails.
static bool assemble_band(const Native& n, const Layout& L, const std::vector<NPose>& poses,
                          const std::vector<Vec3>& points, const std::vector<Radial>& groups, const GaugeState& g,
                          const Loss& loss, const std::vector<int>& pos, Band& B) {
  const int D = L.D;
  B.n = D;
  B.w = 0;
  for (size_t p = 0; p < points.size(); ++p) {
    int lo = D, hi = -1;
    for (uint64_t o = n.pt_off[p]; o < n.pt_off[p + 1]; ++o) {
      const int cam = n.obs_cam[o];
      for (int k = 0; k < L.pose_dim[cam]; ++k) {
        lo = std::min(lo, pos[L.pose_off[cam] + k]);
        hi = std::max(hi, pos[L.pose_off[cam] + k]);
      }
      if (n.self_cal) {
        const int grp = n.cam_group[cam];
        for (int k = 0; k < L.intr_dim[grp]; ++k) {
          lo = std::min(lo, pos[L.intr_off[grp] + k]);
          hi = std::max(hi, pos[L.intr_off[grp] + k]);
        }
      }
    }
    if (hi >= lo) B.w = std::max(B.w, hi - lo);
  }
  B.a.assign((size_t)D * (B.w + 1), 0.0);
  // rows of the band in contiguous ranges, one per thread; each thread adds the terms of its rows
  int nth = 1;
#ifdef _OPENMP
  nth = omp_get_max_threads();
#endif
  const int per = (D + nth - 1) / std::max(nth, 1);
#pragma omp parallel for schedule(static, 1)
  for (int t = 0; t < nth; ++t) {
    const int r0 = t * per, r1 = std::min(D, r0 + per);
    if (r0 >= r1) continue;
    for (size_t p = 0; p < points.size(); ++p) band_point_terms(n, L, poses, points, groups, g, loss, pos, p, r0, r1, B);
  }
  for (double v : B.a)
    if (!std::isfinite(v)) return false;
  return true;
}

// In-place left-looking band Cholesky; false when a pivot is not finite and positive.
static bool band_cholesky(Band& B) {
  const int n = B.n, w = B.w;
  for (int j = 0; j < n; ++j) {
    double d = B.at(j, j);
    for (int k = std::max(0, j - w); k < j; ++k) d -= B.at(j, k) * B.at(j, k);
    if (!(std::isfinite(d) && d > 0.0)) return false;
    const double piv = std::sqrt(d);
    B.at(j, j) = piv;
    const int i1 = std::min(n - 1, j + w);
#pragma omp parallel for schedule(static)
    for (int i = j + 1; i <= i1; ++i) {
      double v = B.at(i, j);
      for (int k = std::max(0, i - w); k < j; ++k) v -= B.at(i, k) * B.at(j, k);
      B.at(i, j) = v / piv;
    }
  }
  return true;
}

// (S^-1)_pq = (L^-1 e_P) . (L^-1 e_Q): forward solves from each parameter's position.
static bool band_marginals(const Native& n, const Layout& L, const Band& B, const std::vector<int>& pos,
                           std::vector<double>& out) {
  const size_t ng = L.intr_dim.size();
  out.assign(9 * std::max<size_t>(ng, 1), 0.0);
  bool finite = true;
#pragma omp parallel for schedule(dynamic, 1) reduction(&& : finite)
  for (long long g = 0; g < (long long)ng; ++g) {
    const int dim = L.intr_dim[g];
    if (dim == 0) continue;
    std::vector<std::vector<double>> y(dim, std::vector<double>(B.n, 0.0));
    int lo = B.n;
    for (int k = 0; k < dim; ++k) lo = std::min(lo, pos[L.intr_off[g] + k]);
    for (int k = 0; k < dim; ++k) {
      const int P = pos[L.intr_off[g] + k];
      std::vector<double>& v = y[k];
      for (int i = P; i < B.n; ++i) {
        double s = i == P ? 1.0 : 0.0;
        for (int c = std::max(P, i - B.w); c < i; ++c) s -= B.at(i, c) * v[c];
        v[i] = s / B.at(i, i);
      }
    }
    for (int a = 0; a < dim; ++a)
      for (int b = 0; b < dim; ++b) {
        double s = 0.0;
        for (int i = lo; i < B.n; ++i) s += y[a][i] * y[b][i];
        out[9 * g + 3 * a + b] = s;
        finite = finite && std::isfinite(s);
      }
  }
  return finite;
}

static double scene_scale_observed(const Native& n, const std::vector<NPose>& poses, const std::vector<Vec3>& points) {
  // observed_scene_scale (optimizer.rs:630-675); FixedBaseline gauges use the baseline norm
  if (n.gauge_cam >= 0) return norm3(poses[n.gauge_cam].t);
  double scale = 0.0, sq = 1.0;
  size_t count = 0;
  for (size_t p = 0; p < points.size(); ++p) {
    if (n.pt_off[p] == n.pt_off[p + 1]) continue;
    count++;
    for (double c : points[p]) {
      double m = std::fabs(c);
      if (m == 0.0) continue;
      if (scale < m) {
        double r = scale / m;
        sq = 1.0 + sq * r * r;
        scale = m;
      } else {
        double r = m / scale;
        sq += r * r;
      }
    }
  }
  if (scale == 0.0 || count == 0) return kMinPositive;
  double rms = scale * std::sqrt(sq / double(count));
  return std::isfinite(rms) ? std::max(rms, kMinPositive) : scale;
}
static double scene_scale_plain(const Native& n, const std::vector<NPose>& poses, const std::vector<Vec3>& points) {
  // scene_scale (optimizer.rs:620-628)
  if (n.gauge_cam >= 0) return norm3(poses[n.gauge_cam].t);
  double s = 0.0;
  for (auto& p : points) s += p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
  return std::max(std::sqrt(s / double(points.size())), kMinPositive);
}

// spectral rank of a symmetric PSD matrix after Jacobi equilibration (sparse/direct.rs:410-455), with the
// eigenvalues from cyclic Jacobi rotations (a published symmetric eigenvalue method).
static int spectral_rank(std::vector<double> A, int D, bool* ok) {
  *ok = false;
  if (const char* dump = std::getenv("OMVGBA_ORACLE_DUMP_S")) {
    if (FILE* f = std::fopen(dump, "ab")) {
      std::fwrite(&D, sizeof(int), 1, f);
      std::fwrite(A.data(), sizeof(double), A.size(), f);
      std::fclose(f);
    }
  }
  double ds = 0.0;
  for (int i = 0; i < D; ++i) ds = std::max(ds, std::fabs(A[(size_t)i * D + i]));
  if (!(std::isfinite(ds) && ds > 0.0)) return 0;
  double fl = 64.0 * kEps * ds;
  std::vector<double> sc(D);
  for (int i = 0; i < D; ++i) {
    double d = A[(size_t)i * D + i];
    if (!std::isfinite(d)) return 0;
    sc[i] = 1.0 / std::sqrt(std::max(d, fl));
  }
  for (int i = 0; i < D; ++i)
    for (int j = 0; j < D; ++j) {
      double v = A[(size_t)i * D + j] * sc[i] * sc[j];
      if (!std::isfinite(v)) return 0;
      A[(size_t)i * D + j] = v;
    }
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int i = 0; i < D; ++i)
      for (int j = i + 1; j < D; ++j) off += A[(size_t)i * D + j] * A[(size_t)i * D + j];
    if (off < 1e-30) break;
    for (int p = 0; p < D; ++p)
      for (int q = p + 1; q < D; ++q) {
        double apq = A[(size_t)p * D + q];
        if (std::fabs(apq) < 1e-300) continue;
        double app = A[(size_t)p * D + p], aqq = A[(size_t)q * D + q];
        double theta = (aqq - app) / (2.0 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < D; ++k) {
          double akp = A[(size_t)k * D + p], akq = A[(size_t)k * D + q];
          A[(size_t)k * D + p] = c * akp - s * akq;
          A[(size_t)k * D + q] = s * akp + c * akq;
        }
        for (int k = 0; k < D; ++k) {
          double apk = A[(size_t)p * D + k], aqk = A[(size_t)q * D + k];
          A[(size_t)p * D + k] = c * apk - s * aqk;
          A[(size_t)q * D + k] = s * apk + c * aqk;
        }
      }
  }
  double largest = 0.0, smallest = kInf;
  for (int i = 0; i < D; ++i) {
    largest = std::max(largest, std::fabs(A[(size_t)i * D + i]));
    smallest = std::min(smallest, A[(size_t)i * D + i]);
  }
  if (!(std::isfinite(largest) && largest > 0.0)) return 0;
  double tol = 64.0 * kEps * D * largest;
  if (std::getenv("OMVGBA_ORACLE_TRACE"))
    std::fprintf(stderr, "rank: lambda_max %.6e lambda_min %.6e tol %.3e\n", largest, smallest, tol);
  int rank = 0;
  for (int i = 0; i < D; ++i) {
    double v = A[(size_t)i * D + i];
    if (!std::isfinite(v) || v < -tol) return 0;
    rank += v > tol ? 1 : 0;
  }
  *ok = true;
  return rank;
}

static uint64_t noninvertible_count(const Native& n, const std::vector<Radial>& groups) {
  uint64_t count = 0;
  for (size_t o = 0; o < n.obs_cam.size(); ++o) {
    if (n.self_cal) {
      if (!radial_bearing_ok(groups[n.cam_group[n.obs_cam[o]]], n.obs_px[o])) count++;
    } else if (!n.pixel_model) {
      const BrownConrady& m = n.models[n.obs_model[o]];
      double xd = (n.obs_px[o][0] - m.cx) / m.fx, yd = (n.obs_px[o][1] - m.cy) / m.fy, x, y;
      if (!m.remove_distortion(xd, yd, &x, &y)) count++;
    }
  }
  return count;
}

static const int kDenseRankLimit = 2048;

static NativeReport refine(const Native& n, std::vector<NPose>& poses, std::vector<Vec3>& points,
                           std::vector<Radial>& groups, const Options& opt) {
  Solver S(n);
  const Layout& L = S.L;
  int D = L.D;
  bool direct = !opt.iterative;
  double scene = n.self_cal ? scene_scale_plain(n, poses, points) : scene_scale_observed(n, poses, points);
  auto schedule = stages(opt.loss, opt.max_iterations);
  int target = final_stage_index(schedule);
  bool have_initial = false;
  double init_cost = kInf, init_rmse = kInf;
  size_t N = n.obs_cam.size();
  auto metrics = [&](const Loss& loss, double* cost, double* rmse) {
    double total = 0.0, sq = 0.0;
    for (size_t p = 0; p < points.size(); ++p)
      for (uint64_t o = n.pt_off[p]; o < n.pt_off[p + 1]; ++o) {
        const NPose& P = poses[n.obs_cam[o]];
        Vec3 r = rotate(P.R, points[p]);
        Vec3 xc = {r[0] + P.t[0], r[1] + P.t[1], r[2] + P.t[2]};
        ObsLin ol;
        if (!project_obs(n, groups, o, xc, &ol)) {
          *cost = kInf;
          *rmse = kInf;
          return;
        }
        double rn = std::hypot(ol.p.residual[0], ol.p.residual[1]);
        rn = std::sqrt(ol.p.residual[0] * ol.p.residual[0] + ol.p.residual[1] * ol.p.residual[1]);
        total += loss.cost(rn);
        sq += rn * rn;
      }
    *cost = total;
    *rmse = std::sqrt(sq / double(2 * N));
  };
  bool reuse = false;
  for (auto& st : schedule)
    if (st.max_iterations > 0) {
      reuse = st.loss == opt.loss;
      break;
    }
  if (!reuse) {
    metrics(opt.loss, &init_cost, &init_rmse);
    have_initial = true;
  }
  double initial_damping = direct ? 1e-4 : 1e-1;  // SparseCameraSolver::default_initial_damping (api.rs:300-305)
  RunState run(initial_damping);
  double iter_tol = std::min(std::sqrt(opt.criteria.relative_cost), 1e-6);
  Workspace ws;
  uint64_t pcg_terms = 0;
  std::vector<NPose> cand_poses(poses.size());
  std::vector<Vec3> cand_points(points.size());
  std::vector<Radial> cand_groups(groups);
  std::vector<double> step(D, 0.0), Lf;
  bool done = false;
  for (int si = 0; si < 3 && !done; ++si) {
    const Stage& st = schedule[si];
    bool confirm = false;
    double t_iter = 0.0;
    auto close_iteration = [&]() {
      if (t_iter > 0.0) tl_iteration_seconds.push_back(oracle_now() - t_iter);
      t_iter = 0.0;
    };
    for (uint64_t it = 0; it < st.max_iterations; ++it) {
      close_iteration();
      t_iter = oracle_now();
      run.iterations++;
      GaugeState g = make_gauge(n, poses, scene);
      double t_it = oracle_now();
      Assembly a = S.assemble(poses, points, groups, g, st.loss, run.damping.value, direct, ws);
      oracle_phase("assemble", t_it);
      t_it = oracle_now();
      if (!have_initial && std::isfinite(a.cost) && std::isfinite(a.sq) && N > 0) {
        init_cost = a.cost;
        init_rmse = std::sqrt(a.sq / double(2 * N));
        have_initial = true;
      }
      if (!a.valid) {
        run.rej_lin++;
        run.damping.reject();
        continue;
      }
      double current = a.cost;
      if (si == target && run.gradient_converged(a.grad_norm, current, opt.criteria)) {
        done = true;
        break;
      }
      // camera step
      bool iterative_step = false;
      double rel_res = 0.0;
      if (direct) {
        Lf = ws.H.S;
        if (!Solver::cholesky(Lf, D)) {
          run.rej_solve++;
          run.damping.reject();
          continue;
        }
        for (int i = 0; i < D; ++i) step[i] = -ws.grad[i];
        Solver::cholesky_solve(Lf, D, step);
      } else {
        std::vector<Solver::BlockFactor> fs;
        if (!S.factor_blocks(ws, fs)) {
          run.rej_solve++;
          run.damping.reject();
          continue;
        }
        double tol = confirm ? std::min(opt.pcg_tol, iter_tol) : opt.pcg_tol;
        uint64_t limit = confirm ? opt.pcg_max : std::min<uint64_t>(opt.pcg_max, (uint64_t)D);
        auto r = S.pcg(ws, fs, limit, tol, step);
        pcg_terms += r.terms;
        if (!r.accepted) {
          run.rej_solve++;
          run.damping.reject();
          continue;
        }
        iterative_step = true;
        rel_res = r.relative_residual;
      }
      oracle_phase("camera step", t_it);
      t_it = oracle_now();
      // candidate: step cap (calibrated only), retraction
      if (!n.self_cal) {
        double largest = 0.0;
        for (int c = 0; c < n.ncam; ++c) {
          int d = L.pose_dim[c];
          if (d == 0) continue;
          int o = L.pose_off[c], fd = std::min(d, 3);
          double s1 = 0, s2 = 0;
          for (int k = 0; k < fd; ++k) s1 += step[o + k] * step[o + k];
          for (int k = fd; k < d; ++k) s2 += step[o + k] * step[o + k];
          largest = std::max({largest, std::sqrt(s1), std::sqrt(s2)});
        }
        if (largest > 0.5) {
          double sc = 0.5 / largest;
          for (auto& v : step) v *= sc;
        }
      }
      // retract_poses_with_masks (optimizer.rs:442-510); with every mask full it is retract_poses
      // (optimizer.rs:376-424)
      for (int c = 0; c < n.ncam; ++c) {
        int d = L.pose_dim[c], o = L.pose_off[c];
        if (d == 0) {
          cand_poses[c] = poses[c];
          continue;
        }
        const int mask = n.explicit_masks ? n.pose_mask[c] : 3;
        Mat3 R = poses[c].R, up{};
        int ts = 0;
        if (mask & 1) {
          up = exp_so3({step[o], step[o + 1], step[o + 2]});
          R = mat_mul(up, poses[c].R);
          ts = 3;
        }
        Vec3 t;
        if (!(mask & 2)) {  // t' = Exp(w) t keeps the centre -R^T t
          t = (mask & 1) ? rotate(up, poses[c].t) : poses[c].t;
        } else if (g.fixed_camera == c) {
          Vec3 dir = retract_s2(g.direction, g.basis, step[o + ts], step[o + ts + 1]);
          t = {g.baseline * dir[0], g.baseline * dir[1], g.baseline * dir[2]};
        } else {
          for (int k = 0; k < 3; ++k) t[k] = poses[c].t[k] + g.scene_scale * step[o + ts + k];
        }
        cand_poses[c] = {R, t};
      }
      if (n.self_cal)
        for (size_t gi = 0; gi < groups.size(); ++gi) {  // retract_cameras (self_calibration/optimizer.rs:565-587)
          int d = L.intr_dim[gi], o = L.intr_off[gi];
          cand_groups[gi] = groups[gi];
          if (d == 0) continue;
          double dl[3] = {0, 0, 0};
          for (int k = 0; k < d; ++k) dl[k] = step[o + k];
          cand_groups[gi] = {groups[gi].focal * std::exp(dl[0]), groups[gi].k1 + dl[1], groups[gi].k2 + dl[2]};
        }
      // candidate points (cached back-substitution)
      size_t P = points.size();
      std::vector<double> pc(P, 0.0), ps(P, 0.0), pdn(P, 0.0);
      std::vector<uint8_t> pok(P, 1);
#pragma omp parallel for schedule(dynamic, 1024)
      for (size_t p = 0; p < P; ++p) {
        if (n.fixed_points[p]) {
          cand_points[p] = points[p];
          auto c = admitted_point_cost(n, cand_poses, cand_groups, points[p], p, st.loss, 0.0, Admission::Projection);
          if (!c)
            pok[p] = 0;
          else
            pc[p] = *c;
          continue;
        }
        const auto& cc = ws.cache;
        if (!cc.valid[p]) {
          pok[p] = 0;
          continue;
        }
        Vec3 sp = cc.inv_grad[p];
        for (uint64_t r = cc.row_off[p]; r < cc.row_off[p + 1] && cc.row_param[r] >= 0; ++r)
          for (int i = 0; i < 3; ++i) sp[i] += cc.row_y[r][i] * step[cc.row_param[r]];
        sp = {-sp[0], -sp[1], -sp[2]};
        Vec3 stepped = {points[p][0] + g.scene_scale * sp[0], points[p][1] + g.scene_scale * sp[1],
                        points[p][2] + g.scene_scale * sp[2]};
        auto ev = candidate_point(n, poses, groups, cand_poses, cand_groups, points[p], stepped, p, st.loss,
                                  g.scene_scale);
        if (!ev) {
          pok[p] = 0;
          continue;
        }
        cand_points[p] = ev->position;
        pc[p] = ev->cost;
        if (ev->moved) {
          ps[p] = sp[0] * sp[0] + sp[1] * sp[1] + sp[2] * sp[2];
          const Vec3& dd = cc.damp_diag[p];
          pdn[p] = dd[0] * sp[0] * sp[0] + dd[1] * sp[1] * sp[1] + dd[2] * sp[2] * sp[2];
        }
      }
      bool cand_ok = true;
      double cand_cost = 0.0, sqs = 0.0, pdamp = 0.0;
      size_t free_points = 0;
      for (size_t p = 0; p < P; ++p) {
        cand_ok = cand_ok && pok[p];
        cand_cost += pc[p];
        sqs += ps[p];
        pdamp += pdn[p];
        if (!n.fixed_points[p]) free_points++;
      }
      if (!cand_ok) {
        run.rej_cand++;
        run.damping.reject();
        continue;
      }
      double point_rms = std::sqrt(sqs / double(n.self_cal ? std::max<size_t>(P, 1) : std::max<size_t>(free_points, 1)));
      // model reduction
      double damped;
      if (!iterative_step) {
        double quad = 0.0;  // hessian_quadratic_form over the damped S (sparse/direct.rs:235-257)
        for (int i = 0; i < D; ++i) {
          double row = 0.0;
          for (int j = 0; j < D; ++j) row += ws.H.S[(size_t)i * D + j] * step[j];
          quad += step[i] * row;
        }
        double gs = 0.0;
        for (int i = 0; i < D; ++i) gs += ws.grad[i] * step[i];
        damped = a.point_red - gs - 0.5 * quad;
      } else {
        std::vector<double> q;
        S.apply_operator(ws, step, q);
        double gs = 0.0, sq = 0.0;
        for (int i = 0; i < D; ++i) {
          gs += ws.grad[i] * step[i];
          sq += step[i] * q[i];
        }
        damped = a.point_red + (-gs - 0.5 * sq);
        if (!(std::isfinite(damped) && damped > 0.0)) damped = std::nan("");
      }
      double cdn = 0.0;
      for (int i = 0; i < D; ++i) cdn += ws.diag[i] * step[i] * step[i];
      double predicted = damped + 0.5 * run.damping.value * (cdn + pdamp);
      double reduction = current - cand_cost;
      if (std::getenv("OMVGBA_ORACLE_TRACE"))
        std::fprintf(stderr, "it=%llu stage=%d cost=%.12e cand=%.12e pred=%.6e lambda=%.3e gn=%.3e\n",
                     (unsigned long long)run.iterations, si, current, cand_cost, predicted, run.damping.value, a.grad_norm);
      if (run.accept_gain(reduction, predicted)) {
        poses = cand_poses;
        points = cand_points;
        if (n.self_cal) groups = cand_groups;
        double ss = 0.0;
        for (double v : step) ss += v * v;
        double crms = std::sqrt(ss / double(std::max(D, 1)));
        double sn = std::sqrt(crms * crms + point_rms * point_rms);
        bool is_target = si == target;
        Criterion cc = run.record_accepted(sn, reduction, current, is_target, opt.criteria);
        if (is_target) {
          bool converged;
          if (iterative_step && cc != Criterion::None && rel_res > iter_tol) {
            confirm = true;
            converged = run.certify(Criterion::None);
          } else {
            confirm = false;
            converged = run.certify(cc);
          }
          if (converged) {
            done = true;
            break;
          }
        }
      }
    }
    close_iteration();
  }
  // final undamped assembly and certificate
  NativeReport rep{};
  GaugeState g = make_gauge(n, poses, scene);
  bool dense_rank = D <= kDenseRankLimit;
  Assembly fa = S.assemble(poses, points, groups, g, opt.loss, 0.0, dense_rank, ws);
  // the expected gauge nullity is zero: the native lowering fixes the gauge with pose masks
  rep.rank = 3;
  Band band;
  bool band_factored = false;
  std::vector<int> order;
  if (!fa.valid) {
    rep.rank = 2;
  } else if (D == 0) {
    rep.rank = 0;
  } else if (dense_rank) {
    bool ok;
    int rank = spectral_rank(ws.H.S, D, &ok);
    rep.rank = (ok && rank == D) ? 0 : 2;
  } else if (g_certificate) {  // sparse/direct.rs:300-304: S factors
    order = factor_order(n, L);
    band_factored = assemble_band(n, L, poses, points, groups, g, opt.loss, order, band) && band_cholesky(band);
    rep.rank = band_factored ? 0 : 2;
  }
  if (n.self_cal && opt.certify_intrinsics && g_certificate && fa.valid) {
    if (order.empty()) {
      order = factor_order(n, L);
      band_factored = assemble_band(n, L, poses, points, groups, g, opt.loss, order, band) && band_cholesky(band);
    }
    rep.marginals_ok = band_factored && band_marginals(n, L, band, order, rep.marginals);
  }
  bool well = rep.rank != 2 && fa.weak == 0;
  rep.status = run.status(well);
  if (std::getenv("OMVGBA_ORACLE_TRACE"))
    std::fprintf(stderr, "final: valid=%d rank=%d weak=%llu status=%d D=%d min_rcond=%.3e\n", (int)fa.valid, rep.rank,
                 (unsigned long long)fa.weak, rep.status, D, fa.min_rcond);
  rep.reason = run.convergence;
  if (fa.valid) {
    rep.final_cost = fa.cost;
    rep.final_rmse = std::sqrt(fa.sq / double(2 * N));
    rep.gradient_inf_norm = fa.grad_norm;
  } else {
    metrics(opt.loss, &rep.final_cost, &rep.final_rmse);
    // unreduced scaled gradient with zero damping: same assembly without point factorization failures
    rep.gradient_inf_norm = fa.grad_norm;
  }
  rep.initial_cost = init_cost;
  rep.initial_rmse = init_rmse;
  rep.iterations = run.iterations;
  rep.accepted = run.accepted;
  rep.rejected = run.rejected();
  rep.rej[0] = run.rej_lin;
  rep.rej[1] = run.rej_solve;
  rep.rej[2] = run.rej_cand;
  rep.rej[3] = run.rej_insuff;
  rep.weak = fa.weak;
  rep.noninvertible = noninvertible_count(n, groups);
  rep.pcg_terms = pcg_terms;
  rep.final_damping = run.damping.value;
  rep.D = D;
  return rep;
}

// ------------------------------------------------------------------------------------------
// Problem validation and lowering.
// ------------------------------------------------------------------------------------------
static Mat3 pose_R(const omvgba_pose& p) {
  Mat3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r[i][j] = p.rotation[i * 3 + j];
  return r;
}
static Vec3 pose_C(const omvgba_pose& p) { return {p.center[0], p.center[1], p.center[2]}; }
static Vec3 point_at(const omvgba_problem& pr, size_t i) {
  return {pr.points[3 * i], pr.points[3 * i + 1], pr.points[3 * i + 2]};
}
static bool point_fixed(const omvgba_problem& pr, size_t i) { return pr.point_fixed && pr.point_fixed[i]; }

static void fail(int code, const std::string& msg) { throw SolveFailure{code, msg}; }

// BundleProblemBuilder::build (problem.rs:492-577) and BundleIntrinsic::try_new (problem.rs:120-134)
static void validate_problem(const omvgba_problem& pr) {
  if (pr.pose_count == 0) fail(OMVGBA_INVALID_PROBLEM, "bundle adjustment requires at least one pose");
  if (pr.intrinsic_count == 0) fail(OMVGBA_INVALID_PROBLEM, "bundle adjustment requires at least one intrinsic");
  if (pr.point_count == 0) fail(OMVGBA_INVALID_PROBLEM, "bundle adjustment requires at least one point");
  if (pr.observation_count == 0) fail(OMVGBA_INVALID_PROBLEM, "bundle adjustment requires at least one observation");
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

static void validate_config(const omvgba_config& c) {  // SolveConfig::validate (solver.rs:122-141)
  if (c.max_iterations == 0) fail(OMVGBA_INVALID_CONFIG, "max_iterations must be positive");
  const char* names[3] = {"function_tolerance", "gradient_tolerance", "parameter_tolerance"};
  double vals[3] = {c.function_tolerance, c.gradient_tolerance, c.parameter_tolerance};
  for (int i = 0; i < 3; ++i)
    if (!std::isfinite(vals[i]) || vals[i] <= 0.0) fail(OMVGBA_INVALID_CONFIG, names[i]);
  if (c.has_workspace_budget && c.workspace_budget_bytes == 0)
    fail(OMVGBA_INVALID_CONFIG, "workspace_budget_bytes must be positive");
}

static std::vector<uint8_t> observed_cameras(const omvgba_problem& pr) {
  std::vector<uint8_t> o(pr.pose_count, 0);
  for (size_t i = 0; i < pr.observation_count; ++i) o[pr.observation_pose[i]] = 1;
  return o;
}
static double sqdist(const Vec3& a, const Vec3& b) {
  double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
  return dx * dx + dy * dy + dz * dz;
}
// farthest_camera (native/gauge.rs:64-75): max squared distance, ties to the lower index
static int farthest_camera(const std::vector<std::pair<int, double>>& cands) {
  int best = -1;
  double bs = 0.0;
  for (auto& c : cands) {
    if (!std::isfinite(c.second)) continue;
    if (best < 0 || c.second > bs || (c.second == bs && c.first < best)) {
      best = c.first;
      bs = c.second;
    }
  }
  if (best >= 0 && bs > 0.0) return best;
  return -1;
}

struct GaugePlan {
  size_t anchor;
  double scale;
  int native_cam;  // -1 Free
  std::vector<uint32_t> masks;
};

// gauge_plan (native/gauge.rs:239-330)
static GaugePlan gauge_plan(const omvgba_problem& pr) {
  auto observed = observed_cameras(pr);
  bool controls = false;
  for (size_t o = 0; o < pr.observation_count; ++o) controls = controls || point_fixed(pr, pr.observation_point[o]);
  if (pr.gauge_kind == OMVGBA_GAUGE_FREE && controls) {  // validate_anchor_policy (gauge.rs:77-100)
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
    for (size_t i = 0; i < pr.pose_count; ++i) {  // free_scale_anchor (gauge.rs:50-62)
      if (observed[i] && pr.poses[i].variables == 0) {
        anchor = i;
        break;
      }
      if (observed[i] && first == SIZE_MAX) first = i;
    }
    if (anchor == SIZE_MAX) anchor = first == SIZE_MAX ? 0 : first;
    Vec3 ac = pose_C(pr.poses[anchor]);
    bool pose_sets = false, point_sets = false;
    for (size_t i = 0; i < pr.pose_count; ++i)
      pose_sets = pose_sets || (i != anchor && observed[i] && pr.poses[i].variables == 0 && sqdist(pose_C(pr.poses[i]), ac) > 0.0);
    for (size_t o = 0; o < pr.observation_count; ++o) {
      size_t p = pr.observation_point[o];
      point_sets = point_sets || (point_fixed(pr, p) && sqdist(point_at(pr, p), ac) > 0.0);
    }
    plan.anchor = anchor;
    plan.scale = 1.0;
    plan.native_cam = -1;
    if (!(pose_sets || point_sets)) {
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

// calibrated_gauge_plan (native/gauge.rs:123-237)
static GaugePlan calibrated_gauge_plan(const omvgba_problem& pr) {
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
    plan.scale = 1.0;
    plan.native_cam = -1;
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
  plan.scale = 1.0;
  plan.native_cam = -1;
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

static BrownConrady to_model(const omvgba_intrinsic& in) {
  BrownConrady m;
  m.fx = in.fx;
  m.fy = in.fy;
  m.cx = in.cx;
  m.cy = in.cy;
  if (in.model == OMVGBA_CAMERA_BROWN_CONRADY) {
    m.radial_kind = in.radial_kind;
    m.tangential_kind = in.tangential_kind;
    m.k1 = in.k1;
    m.k2 = in.k2;
    m.k3 = in.k3;
    m.p1 = in.p1;
    m.p2 = in.p2;
    m.turn_squared = first_radial_turn_squared(m.rk1(), m.rk2());
  }
  return m;
}

// WorldRebase (native/world_rebase.rs:19-87)
static NPose pose_to_native(const Native& n, const omvgba_pose& p) {
  Mat3 R = pose_R(p);
  Vec3 C = pose_C(p);
  if (R == n.anchor_R && C == n.anchor_C) return {{{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}}, {0, 0, 0}};
  Mat3 AT;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) AT[i][j] = n.anchor_R[j][i];
  Mat3 rot = mat_mul(R, AT);
  Vec3 d = {n.anchor_C[0] - C[0], n.anchor_C[1] - C[1], n.anchor_C[2] - C[2]};
  Vec3 t = rotate(R, d);
  return {rot, {t[0] * n.scale, t[1] * n.scale, t[2] * n.scale}};
}
static Vec3 point_to_native(const Native& n, const Vec3& X) {
  Vec3 d = {X[0] - n.anchor_C[0], X[1] - n.anchor_C[1], X[2] - n.anchor_C[2]};
  Vec3 r = rotate(n.anchor_R, d);
  return {r[0] * n.scale, r[1] * n.scale, r[2] * n.scale};
}
static void pose_from_native(const Native& n, const NPose& p, double R_out[9], double C_out[3]) {
  Mat3 R = mat_mul(p.R, n.anchor_R);
  Vec3 rc = rotate_transposed(p.R, p.t);
  rc = {-rc[0], -rc[1], -rc[2]};
  Vec3 wc = rotate_transposed(n.anchor_R, rc);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) R_out[i * 3 + j] = R[i][j];
  for (int i = 0; i < 3; ++i) C_out[i] = n.anchor_C[i] + wc[i];
}
static Vec3 point_from_native(const Native& n, const Vec3& X) {
  Vec3 r = rotate_transposed(n.anchor_R, X);
  return {n.anchor_C[0] + r[0], n.anchor_C[1] + r[1], n.anchor_C[2] + r[2]};
}

static bool has_free_intrinsics(const omvgba_problem& pr) {
  for (size_t o = 0; o < pr.observation_count; ++o)
    if (pr.intrinsics[pr.observation_intrinsic[o]].variables != 0) return true;
  return false;
}

// single_pose_intrinsics (native/mod.rs:393-409)
static bool single_pose_intrinsics(const omvgba_problem& pr, std::vector<size_t>* out) {
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

static void sort_observations(const omvgba_problem& pr, Native& n, const std::vector<size_t>& cam_dest,
                              std::vector<size_t>* order_out) {
  std::vector<size_t> order(pr.observation_count);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](size_t a, size_t b) { return pr.observation_point[a] < pr.observation_point[b]; });
  n.obs_cam.resize(order.size());
  n.obs_src.resize(order.size());
  for (size_t i = 0; i < order.size(); ++i) {
    n.obs_cam[i] = (uint32_t)cam_dest[pr.observation_pose[order[i]]];
    n.obs_src[i] = order[i];
  }
  n.pt_off.assign(pr.point_count + 1, 0);
  for (size_t o = 0; o < pr.observation_count; ++o) n.pt_off[pr.observation_point[o] + 1]++;
  for (size_t p = 0; p < pr.point_count; ++p) n.pt_off[p + 1] += n.pt_off[p];
  *order_out = order;
}

static void set_anchor(const omvgba_problem& pr, Native& n, size_t anchor, double scale) {
  n.anchor_R = pose_R(pr.poses[anchor]);
  n.anchor_C = pose_C(pr.poses[anchor]);
  n.scale = scale;
  if (!std::isfinite(scale) || scale <= 0.0) fail(OMVGBA_UNSUPPORTED, "world scale must be finite and positive");
  n.camera_source_order.clear();
  n.camera_source_order.push_back(anchor);
  for (size_t i = 0; i < pr.pose_count; ++i)
    if (i != anchor) n.camera_source_order.push_back(i);
}

// PreparedCalibratedProblem::try_new (native/calibrated.rs:200-391), full-pose masks only.
// Camera::bearing (openmvg-core camera/camera_enum.rs:128-132): unproject (pinhole.rs:324-340,
// brown_conrady.rs:365-383, fisheye.rs:271-299 with distortion.rs:319-455, spherical.rs:113-257),
// then try_normalize_bearing (camera_model.rs:91-109).
static double fisheye_apply(int kind, const double k[4], double t) {
  const double t2 = t * t, t4 = t2 * t2;
  switch (kind) {
    case 0: return t;
    case 1: return t * (1.0 + k[0] * t2);
    case 2: return t * (1.0 + k[0] * t2 + k[1] * t4);
    case 3: return t * (1.0 + k[0] * t2 + k[1] * t4 + k[2] * (t4 * t2));
    default: return t * (1.0 + k[0] * t2 + k[1] * t4 + k[2] * (t4 * t2) + k[3] * (t4 * t4));
  }
}
static double fisheye_derivative(const double k[4], double t) {
  const double t2 = t * t, t4 = t2 * t2, t6 = t4 * t2, t8 = t4 * t4;
  return 1.0 + 3.0 * k[0] * t2 + 5.0 * k[1] * t4 + 7.0 * k[2] * t6 + 9.0 * k[3] * t8;
}
static std::optional<Vec3> camera_bearing(const omvgba_intrinsic& in, double u, double v) {
  if (!std::isfinite(u) || !std::isfinite(v)) return std::nullopt;
  Vec3 d;
  if (in.model == OMVGBA_CAMERA_PINHOLE || in.model == OMVGBA_CAMERA_BROWN_CONRADY) {
    d = {(u - in.cx) / in.fx, (v - in.cy) / in.fy, 1.0};
    if (!all_finite(d.data(), 3)) return std::nullopt;
    if (in.model == OMVGBA_CAMERA_BROWN_CONRADY) {
      double x, y;
      if (!to_model(in).remove_distortion(d[0] / d[2], d[1] / d[2], &x, &y)) return std::nullopt;
      d = {x, y, 1.0};
    }
  } else if (in.model == OMVGBA_CAMERA_FISHEYE) {
    const double xd = (u - in.cx) / in.fx, yd = (v - in.cy) / in.fy;
    if (!std::isfinite(xd) || !std::isfinite(yd)) return std::nullopt;
    const double td = std::hypot(xd, yd);
    if (td <= kEps) {
      d = {0.0, 0.0, 1.0};
    } else {
      const int kind = in.radial_kind;
      const double k[4] = {kind >= 1 ? in.k1 : 0.0, kind >= 2 ? in.k2 : 0.0, kind >= 3 ? in.k3 : 0.0,
                           kind >= 4 ? in.k4 : 0.0};
      if (!all_finite(k, 4)) return std::nullopt;
      // FisheyeCamera::try_new: the end of the positive-derivative branch up to pi - 1e-10
      const double cap = 3.141592653589793 - 1e-10;
      double upper = cap;
      if (k[2] == 0.0 && k[3] == 0.0) {
        auto q = first_radial_turn_squared(k[0], k[1]);
        upper = q ? std::min(std::sqrt(*q), cap) : cap;
      } else if (!(k[0] >= 0.0 && k[1] >= 0.0 && k[2] >= 0.0 && k[3] >= 0.0)) {
        double prev = 0.0;
        for (int i = 1; i <= 1024; ++i) {
          const double t = cap * i / 1024.0;
          if (fisheye_derivative(k, t) <= 0.0) {
            double lo = prev, hi = t;
            for (int it = 0; it < 64; ++it) {
              const double mid = 0.5 * (lo + hi);
              (fisheye_derivative(k, mid) > 0.0 ? lo : hi) = mid;
            }
            upper = lo;
            break;
          }
          prev = t;
        }
      }
      // invert_on_validated_interval: safeguarded Newton, 48 steps
      const double mapped = fisheye_apply(kind, k, upper);
      if (!std::isfinite(mapped) || td > mapped + 1e-12) return std::nullopt;
      double lo = 0.0, hi = upper, t = std::min(td, upper);
      bool done = false;
      for (int it = 0; it < 48 && !done; ++it) {
        const double r = fisheye_apply(kind, k, t) - td;
        if (std::fabs(r) <= 1e-13) {
          done = true;
          break;
        }
        if (r < 0.0)
          lo = t;
        else
          hi = t;
        const double dv = fisheye_derivative(k, t), nt = t - r / dv;
        t = (std::isfinite(dv) && dv > 1e-15 && nt > lo && nt < hi) ? nt : 0.5 * (lo + hi);
      }
      if (!done && !(std::fabs(fisheye_apply(kind, k, t) - td) <= 1e-12)) return std::nullopt;
      const double sc = std::sin(t) / td;
      d = {xd * sc, yd * sc, std::cos(t)};
      if (!all_finite(d.data(), 3)) return std::nullopt;
    }
  } else if (in.model == OMVGBA_CAMERA_SPHERICAL) {
    const double w = (double)in.width, h = (double)(in.width / 2);
    if (v < -0.5 || v > h - 0.5) return std::nullopt;
    double x = std::fmod(u + 0.5, w);
    if (x < 0.0) x += w;
    x -= 0.5;
    const double pi = 3.141592653589793;
    const double lon = (x + 0.5) * (2.0 * pi) / w - pi, lat = (v + 0.5) * pi / h - pi / 2.0;
    if (!std::isfinite(lon) || !std::isfinite(lat) || lat < -pi / 2.0 || lat > pi / 2.0) return std::nullopt;
    d = {std::cos(lat) * std::sin(lon), std::sin(lat), std::cos(lat) * std::cos(lon)};
  } else {
    return std::nullopt;
  }
  if (!all_finite(d.data(), 3)) return std::nullopt;
  const double sc = std::max({0.0, std::fabs(d[0]), std::fabs(d[1]), std::fabs(d[2])});
  if (sc == 0.0) return std::nullopt;
  const Vec3 x = {d[0] / sc, d[1] / sc, d[2] / sc};
  const double nrm = std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  if (!std::isfinite(nrm) || nrm == 0.0) return std::nullopt;
  return Vec3{x[0] / nrm, x[1] / nrm, x[2] / nrm};
}

static Native lower_calibrated(const omvgba_problem& pr, bool angular = false) {
  for (size_t o = 0; o < pr.observation_count && !angular; ++o) {
    int m = pr.intrinsics[pr.observation_intrinsic[o]].model;
    if (m == OMVGBA_CAMERA_FISHEYE || m == OMVGBA_CAMERA_SPHERICAL)
      fail(OMVGBA_UNSUPPORTED,
           "pixel BA supports fixed pinhole and Brown-Conrady cameras; use angular residuals for wide-angle cameras");
  }
  GaugePlan plan = calibrated_gauge_plan(pr);
  auto observed = observed_cameras(pr);
  // CameraPoseVariables of the prepared problem (native/calibrated.rs:226-234): translation-only when
  // no free mask moves a rotation (vacuously so when every pose is fixed)
  bool translation_only = true;
  for (size_t i = 0; i < pr.pose_count; ++i)
    if (plan.masks[i] != 0 && (plan.masks[i] & OMVGBA_POSE_ROTATION)) translation_only = false;
  Native n;
  n.self_cal = false;
  n.explicit_masks = true;
  n.translation_only = translation_only;
  set_anchor(pr, n, plan.anchor, plan.scale);
  n.ncam = (int)pr.pose_count;
  std::vector<size_t> dest(pr.pose_count);
  for (size_t d = 0; d < n.camera_source_order.size(); ++d) dest[n.camera_source_order[d]] = d;
  for (size_t d = 0; d < n.camera_source_order.size(); ++d) {
    size_t s = n.camera_source_order[d];
    n.poses.push_back(observed[s] ? pose_to_native(n, pr.poses[s]) : NPose{{{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}}, {0, 0, 0}});
    n.fixed_poses.push_back(plan.masks[s] == 0);
    n.pose_mask.push_back((uint8_t)((plan.masks[s] & OMVGBA_POSE_ROTATION ? 1 : 0) |
                                    (plan.masks[s] & OMVGBA_POSE_TRANSLATION ? 2 : 0)));
  }
  std::vector<uint8_t> pobs(pr.point_count, 0);
  for (size_t o = 0; o < pr.observation_count; ++o) pobs[pr.observation_point[o]] = 1;
  for (size_t i = 0; i < pr.point_count; ++i) {
    n.points.push_back((point_fixed(pr, i) && !pobs[i]) ? Vec3{0, 0, 0} : point_to_native(n, point_at(pr, i)));
    n.fixed_points.push_back(point_fixed(pr, i));
  }
  std::vector<size_t> pose_intr;
  bool single = single_pose_intrinsics(pr, &pose_intr);
  bool uses_full = !single;
  for (size_t o = 0; o < pr.observation_count && !uses_full; ++o) {
    const auto& in = pr.intrinsics[pr.observation_intrinsic[o]];
    uses_full = in.model == OMVGBA_CAMERA_BROWN_CONRADY && (in.radial_kind != 0 || in.tangential_kind != 0);
  }
  n.pixel_model = !uses_full;
  if (!uses_full)
    for (size_t o = 0; o < pr.observation_count; ++o) {
      const auto& in = pr.intrinsics[pr.observation_intrinsic[o]];
      if (in.model == OMVGBA_CAMERA_BROWN_CONRADY && (in.radial_kind != 0 || in.tangential_kind != 0))
        fail(OMVGBA_UNSUPPORTED, "direct calibrated lowering requires an undistorted perspective camera");
    }
  for (size_t i = 0; i < pr.intrinsic_count; ++i) n.models.push_back(to_model(pr.intrinsics[i]));
  n.gauge_cam = plan.native_cam >= 0 ? (int)dest[plan.native_cam] : -1;
  std::vector<size_t> order;
  sort_observations(pr, n, dest, &order);
  n.obs_px.resize(order.size());
  n.obs_model.resize(order.size());
  for (size_t i = 0; i < order.size(); ++i) {
    n.obs_px[i] = {pr.observation_pixel[2 * order[i]], pr.observation_pixel[2 * order[i] + 1]};
    n.obs_model[i] = pr.observation_intrinsic[order[i]];
  }
  if (angular) {  // bearings in the sorted order; the first failure is the error
    n.angular = true;
    n.obs_bearing.resize(order.size());
    for (size_t i = 0; i < order.size(); ++i) {
      auto b = camera_bearing(pr.intrinsics[n.obs_model[i]], n.obs_px[i][0], n.obs_px[i][1]);
      if (!b)
        fail(OMVGBA_NUMERICAL, "observation " + std::to_string(order[i]) +
                                   ": the measured pixel does not define a bearing of its camera model");
      n.obs_bearing[i] = *b;
    }
  }
  return n;
}

// free_radial_dimension (native/self_calibration.rs:442-451)
static int free_radial_dimension(const omvgba_intrinsic& in) {
  if (in.model == OMVGBA_CAMERA_BROWN_CONRADY && (in.variables & OMVGBA_INTRINSIC_RADIAL)) {
    switch (in.radial_kind) {
      case 0: return 1;
      case 1: return 2;
      default: return 3;
    }
  }
  return 1;
}

// PreparedSelfCalibratingProblem::try_new (native/self_calibration.rs:47-198)
static Native lower_self_calibrating(const omvgba_problem& pr) {
  std::vector<size_t> pose_intr;
  if (!single_pose_intrinsics(pr, &pose_intr))
    fail(OMVGBA_UNSUPPORTED, "native self-calibration requires one intrinsic group per observed pose");
  // common_pose_variables (gauge.rs:9-39)
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
  Native n;
  n.self_cal = true;
  set_anchor(pr, n, plan.anchor, plan.scale);
  n.ncam = (int)pr.pose_count;
  std::vector<size_t> dest(pr.pose_count);
  for (size_t d = 0; d < n.camera_source_order.size(); ++d) dest[n.camera_source_order[d]] = d;
  for (size_t d = 0; d < n.camera_source_order.size(); ++d) {
    size_t s = n.camera_source_order[d];
    n.poses.push_back(pose_to_native(n, pr.poses[s]));
    n.fixed_poses.push_back(s == plan.anchor || pr.poses[s].variables == 0);
    n.cam_group.push_back((uint32_t)pose_intr[s]);
  }
  for (size_t i = 0; i < pr.point_count; ++i) {
    n.points.push_back(point_to_native(n, point_at(pr, i)));
    n.fixed_points.push_back(point_fixed(pr, i));
  }
  for (size_t i = 0; i < pr.intrinsic_count; ++i) {  // radial_camera (native/self_calibration.rs:483-512)
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
    n.groups.push_back({in.fx, k1, k2});
    n.group_dim.push_back(in.variables == 0 ? 0 : free_radial_dimension(in));
  }
  n.gauge_cam = plan.native_cam >= 0 ? (int)dest[plan.native_cam] : -1;
  std::vector<size_t> order;
  sort_observations(pr, n, dest, &order);
  n.obs_px.resize(order.size());
  for (size_t i = 0; i < order.size(); ++i) {
    const auto& in = pr.intrinsics[pr.observation_intrinsic[order[i]]];
    n.obs_px[i] = {pr.observation_pixel[2 * order[i]] - in.cx, pr.observation_pixel[2 * order[i] + 1] - in.cy};
  }
  return n;
}

// ------------------------------------------------------------------------------------------
// Solution building (native/calibrated.rs:393-460, native/reporting.rs:24-141, solver.rs:803-1131).
// ------------------------------------------------------------------------------------------
struct Result {
  std::vector<omvgba_pose> poses;
  std::vector<omvgba_intrinsic> intrinsics;
  std::vector<double> points;
  std::vector<uint64_t> quarantined;
  std::vector<uint64_t> unconstrained;  // intrinsic groups the self-calibration certificate held
  omvgba_report report;
};

// Largest accepted marginal standard deviation of a free intrinsic parameter's contribution to the
// relative radial displacement at the farthest image corner (native/self_calibration.rs:215-222).
static const double kMaxIntrinsicCornerStd = 0.01;

// unconstrained_intrinsics (native/self_calibration.rs:255-303): free groups whose sigma(log f),
// sigma(k1) r^2 or sigma(k2) r^4 -- from (S^-1)_gg times the zero-residual weight, r the normalized
// radius of the farthest corner at the final focal length -- is NaN, or above the bound for a group
// whose certification is required; every free group when S does not factor or a marginal is not
// finite.
static std::vector<uint64_t> unconstrained_groups(const omvgba_problem& pr, const Native& n,
                                                  const std::vector<Radial>& groups, const NativeReport& nr,
                                                  const Loss& loss) {
  std::vector<uint64_t> all, out;
  for (size_t g = 0; g < n.group_dim.size(); ++g)
    if (n.group_dim[g] > 0) all.push_back(g);
  if (all.empty()) return out;
  if (!nr.marginals_ok || nr.marginals.size() < 9 * n.group_dim.size()) return all;
  const double zw = loss.sqrt_weight(0.0);
  const double wn = zw * zw;
  for (uint64_t g : all)
    for (int a = 0; a < n.group_dim[g]; ++a)
      for (int b = 0; b < n.group_dim[g]; ++b)
        if (!std::isfinite(nr.marginals[9 * g + 3 * a + b] * wn)) return all;
  for (uint64_t g : all) {
    const omvgba_intrinsic& in = pr.intrinsics[g];
    const double f = groups[g].focal;
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

static bool camera_project_pixel(const omvgba_intrinsic& in, const Vec3& xc, Vec2* px) {
  if (in.model != OMVGBA_CAMERA_PINHOLE && in.model != OMVGBA_CAMERA_BROWN_CONRADY) return false;
  BrownConrady m = to_model(in);
  auto p = m.project(xc);
  if (!p) return false;
  *px = *p;
  return true;
}

// residual_norm (solver.rs:1405-1432): pixels, or the angle to the measured bearing
static bool residual_norm(const omvgba_problem& pr, size_t o, const omvgba_pose& pose, const omvgba_intrinsic& in,
                          const double* X, double* out) {
  Mat3 R = pose_R(pose);
  Vec3 C = pose_C(pose);
  Vec3 xc = rotate(R, {X[0] - C[0], X[1] - C[1], X[2] - C[2]});
  if (pr.residual_space == OMVGBA_RESIDUAL_ANGULAR) {
    auto b = camera_bearing(in, pr.observation_pixel[2 * o], pr.observation_pixel[2 * o + 1]);
    if (!b) return false;
    auto p = angular_projection(*b, xc);
    if (!p) return false;
    double n = std::hypot(p->residual[0], p->residual[1]);
    if (!std::isfinite(n)) return false;
    *out = n;
    return true;
  }
  Vec2 px;
  if (!camera_project_pixel(in, xc, &px)) return false;
  double n = std::hypot(px[0] - pr.observation_pixel[2 * o], px[1] - pr.observation_pixel[2 * o + 1]);
  if (!std::isfinite(n)) return false;
  *out = n;
  return true;
}

static Loss problem_loss(const omvgba_problem& pr) {
  Loss l;
  if (pr.loss_kind == OMVGBA_LOSS_HUBER) {
    l.kind = LossKind::Huber;
    l.scale = pr.loss_scale;
  } else if (pr.loss_kind == OMVGBA_LOSS_CAUCHY) {
    l.kind = LossKind::Cauchy;
    l.scale = pr.loss_scale / std::sqrt(2.0);
  }
  return l;
}

// active_objective_metrics (solver.rs:1052-1084) and inlier_metrics (solver.rs:1086-1106)
static bool active_metrics(const omvgba_problem& pr, const std::vector<uint8_t>& active, const Result* sol, double* cost,
                           double* rmse) {
  Loss loss = problem_loss(pr);
  double total = 0.0, rs = 0.0, ssr = 1.0;
  size_t count = 0;
  for (size_t o = 0; o < pr.observation_count; ++o) {
    size_t p = pr.observation_point[o];
    if (!active[p]) continue;
    const omvgba_pose& pose = sol ? sol->poses[pr.observation_pose[o]] : pr.poses[pr.observation_pose[o]];
    const omvgba_intrinsic& in = sol ? sol->intrinsics[pr.observation_intrinsic[o]] : pr.intrinsics[pr.observation_intrinsic[o]];
    const double* X = sol ? &sol->points[3 * p] : pr.points + 3 * p;
    double nrm;
    if (!residual_norm(pr, o, pose, in, X, &nrm)) return false;
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
  if (count == 0 || !std::isfinite(total) || total < 0.0) return false;
  double r = rs * std::sqrt(ssr / double(count));
  if (!std::isfinite(r)) return false;
  *cost = total;
  *rmse = r;
  return true;
}

static void refresh_inliers(const omvgba_problem& pr, const std::vector<uint8_t>& active, Result& res) {
  double limit = pr.loss_kind == OMVGBA_LOSS_SQUARED ? kInf : pr.loss_scale;
  uint64_t count = 0;
  double ss = 0.0;
  res.report.has_inlier_count = 0;
  res.report.has_final_inlier_rmse = 0;
  for (size_t o = 0; o < pr.observation_count; ++o) {
    size_t p = pr.observation_point[o];
    if (!active[p]) continue;
    double nrm;
    if (!residual_norm(pr, o, res.poses[pr.observation_pose[o]], res.intrinsics[pr.observation_intrinsic[o]],
                       &res.points[3 * p], &nrm))
      return;
    if (nrm <= limit) {
      count++;
      ss += nrm * nrm;
    }
  }
  res.report.has_inlier_count = 1;
  res.report.inlier_count = count;
  if (count > 0) {
    double r = std::sqrt(ss / double(count));
    if (std::isfinite(r)) {
      res.report.has_final_inlier_rmse = 1;
      res.report.final_inlier_rmse = r;
    }
  }
}

static Result solve_once(const omvgba_problem& pr, const omvgba_config& cfg);

static Result raise(const omvgba_problem& pr, const Native& n, const std::vector<NPose>& poses,
                    const std::vector<Vec3>& points, const std::vector<Radial>& groups, const NativeReport& nr,
                    bool iterative) {
  Result res;
  auto observed = observed_cameras(pr);
  res.poses.assign(pr.poses, pr.poses + pr.pose_count);
  for (size_t d = 0; d < n.camera_source_order.size(); ++d) {
    size_t s = n.camera_source_order[d];
    const omvgba_pose& in = pr.poses[s];
    if (in.variables == 0 || !observed[s]) continue;
    double R[9], C[3];
    pose_from_native(n, poses[d], R, C);
    if (in.variables & OMVGBA_POSE_ROTATION) std::memcpy(res.poses[s].rotation, R, sizeof(R));
    if (in.variables & OMVGBA_POSE_TRANSLATION) std::memcpy(res.poses[s].center, C, sizeof(C));
  }
  res.points.resize(3 * pr.point_count);
  for (size_t i = 0; i < pr.point_count; ++i) {
    Vec3 X = point_fixed(pr, i) ? point_at(pr, i) : point_from_native(n, points[i]);
    if (!all_finite(X.data(), 3)) fail(OMVGBA_NUMERICAL, "native BA returned a non-finite point");
    for (int k = 0; k < 3; ++k) res.points[3 * i + k] = X[k];
  }
  res.intrinsics.assign(pr.intrinsics, pr.intrinsics + pr.intrinsic_count);
  if (n.self_cal)
    for (size_t i = 0; i < pr.intrinsic_count; ++i) {  // with_radial_parameters (self_calibration.rs:455-481)
      auto& out = res.intrinsics[i];
      if (out.variables == 0) continue;
      out.fx = groups[i].focal;
      out.fy = groups[i].focal;
      if (out.model == OMVGBA_CAMERA_BROWN_CONRADY) {
        if (out.radial_kind >= 1) out.k1 = groups[i].k1;
        if (out.radial_kind >= 2) out.k2 = groups[i].k2;
      }
    }
  omvgba_report& r = res.report;
  std::memset(&r, 0, sizeof(r));
  r.status = nr.status == 0 ? OMVGBA_STATUS_CONVERGED
                            : (nr.status == 1 ? OMVGBA_STATUS_MAX_ITERATIONS
                                              : (nr.status == 2 ? OMVGBA_STATUS_STALLED : OMVGBA_STATUS_DEGENERATE));
  r.convergence_reason = nr.status == 0 ? (int)nr.reason : OMVGBA_REASON_NONE;
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
  if (r.observability != OMVGBA_OBS_NOT_ASSESSED) {
    r.has_observability_details = 1;
    r.details_pose_rank = r.observability == OMVGBA_OBS_FULL_RANK ? nr.D : 0;
    r.details_pose_dimension = nr.D;
    r.details_weak_point_count = nr.weak;
    if (nr.D == 0) r.has_observability_details = 0;
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
  // unobserved_free_intrinsics (native/mod.rs:379-391)
  std::vector<uint8_t> obs_i(pr.intrinsic_count, 0);
  for (size_t o = 0; o < pr.observation_count; ++o) obs_i[pr.observation_intrinsic[o]] = 1;
  return res;
}

// Solution::try_new_with_quarantined_points metrics (solver.rs:829-876)
static void finish_solution(const omvgba_problem& pr, Result& res) {
  std::vector<uint8_t> active(pr.point_count, 1);
  for (auto q : res.quarantined) active[q] = 0;
  uint64_t cnt = 0;
  for (size_t o = 0; o < pr.observation_count; ++o) cnt += active[pr.observation_point[o]];
  res.report.has_observation_count = 1;
  res.report.observation_count = cnt;
  res.report.quarantined_point_count = res.quarantined.size();
  if (!res.quarantined.empty()) {
    double c0, r0, c1, r1;
    if (!active_metrics(pr, active, nullptr, &c0, &r0) || !active_metrics(pr, active, &res, &c1, &r1))
      fail(OMVGBA_INTERNAL, "bundle-adjustment report is invalid");
    res.report.initial_objective = c0;
    res.report.initial_rmse = r0;
    res.report.final_objective = c1;
    res.report.final_rmse = r1;
  }
  refresh_inliers(pr, active, res);
}

// canonicalize_roundoff_non_descent (solver.rs:979-1046)
static void canonicalize(const omvgba_problem& pr, Result& res) {
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

// Entries of the lower triangle of the reduced pattern (diagonal blocks included) and the cross rows
// of the point caches (one per distinct free camera parameter a point touches).
static void pattern_counts(const Native& n, const Layout& L, uint64_t* nnz_lower, uint64_t* cross_rows) {
  const size_t nb = L.block_off.size();
  std::vector<std::vector<int>> lower(nb);
  std::vector<int> blocks;
  uint64_t rows = 0;
  for (size_t p = 0; p < n.points.size(); ++p) {
    blocks.clear();
    for (uint64_t o = n.pt_off[p]; o < n.pt_off[p + 1]; ++o) {
      const int c = n.obs_cam[o];
      if (L.pose_dim[c] > 0) {
        blocks.push_back(L.param_block[L.pose_off[c]]);
        rows += L.pose_dim[c];
      }
      if (n.self_cal) {
        const int g = n.cam_group[c];
        if (L.intr_dim[g] > 0) {
          const int b = L.param_block[L.intr_off[g]];
          if (std::find(blocks.begin(), blocks.end(), b) == blocks.end()) rows += L.intr_dim[g];
          blocks.push_back(b);
        }
      }
    }
    std::sort(blocks.begin(), blocks.end());
    blocks.erase(std::unique(blocks.begin(), blocks.end()), blocks.end());
    for (size_t i = 0; i < blocks.size(); ++i)
      for (size_t j = 0; j <= i; ++j) lower[blocks[i]].push_back(blocks[j]);
  }
  uint64_t nnz = 0;
  for (size_t X = 0; X < nb; ++X) {
    std::sort(lower[X].begin(), lower[X].end());
    lower[X].erase(std::unique(lower[X].begin(), lower[X].end()), lower[X].end());
    const uint64_t dX = L.block_dim[X];
    for (int Y : lower[X]) nnz += (size_t)Y == X ? dX * (dX + 1) / 2 : dX * (uint64_t)L.block_dim[Y];
  }
  *nnz_lower = nnz;
  *cross_rows = rows;
}

// Auto: the budget's choice between the direct and the iterative step (sparse/execution_policy.rs:
// 122-214 with SparseWorkspaceMemoryBudget::AUTO_BYTES = 1 GiB unless an explicit budget is given,
// api.rs:43-52): the direct estimate (four values per entry of the lower reduced pattern plus the
// point caches) must fit 4/5 of the budget; calibrated problems with at least 250,000 observations
// and D >= 768 take the retained PCG first when its estimate (the point caches and the camera-space
// vectors) fits the budget.
static bool auto_prefers_direct(const Native& n, const Layout& L, uint64_t budget, uint64_t* direct_out,
                                uint64_t* cached_out) {
  uint64_t nnz = 0, rows = 0;
  pattern_counts(n, L, &nnz, &rows);
  const uint64_t limit = budget ? budget : (uint64_t(1) << 30);
  const uint64_t points = n.points.size();
  const uint64_t point_cache = (points + 1) * 8 + points * (1 + 2 * 24) + rows * 24;
  const uint64_t direct = nnz * 8 * 4 + point_cache;
  const uint64_t cached = point_cache + (uint64_t)L.D * (5 * 8 + 8);
  *direct_out = direct;
  *cached_out = cached;
  const bool direct_fits = direct <= limit / 5 * 4 + limit % 5 * 4 / 5;
  if (n.self_cal) return direct_fits;
  if (n.obs_cam.size() >= 250000 && L.D >= 768 && cached <= limit) return false;
  return direct_fits;
}

static bool choose_iterative(const omvgba_config& cfg, const Native& n, const Layout& L) {
  if (cfg.linear_solver == OMVGBA_SOLVER_DIRECT) return false;
  if (cfg.linear_solver == OMVGBA_SOLVER_ITERATIVE) return true;
  // a translation-only solve resolves Auto to the direct solver, so its final rank is exact
  // (native/mod.rs:398-407)
  if (!n.self_cal && !n.angular && n.translation_only) return false;
  uint64_t de = 0, ce = 0;
  return !auto_prefers_direct(n, L, cfg.has_workspace_budget ? cfg.workspace_budget_bytes : 0, &de, &ce);
}

// Refuse, before the first iteration, a workspace over an explicit budget (native/mod.rs:557-570):
// the oracle's own storage for the solve -- point caches, the Hessian blocks (the dense S up to
// D = 2048) and the camera-space vectors.
static void check_workspace_budget(const omvgba_config& cfg, const Native& n, const Layout& L) {
  if (!cfg.has_workspace_budget) return;
  uint64_t nnz = 0, rows = 0;
  pattern_counts(n, L, &nnz, &rows);
  const uint64_t P = n.points.size(), D = (uint64_t)L.D;
  uint64_t bytes = P * (1 + 48 + 48 + 24 + 24) + (P + 1) * 8 + rows * (24 + 4) + D * 8 * 12;
  if (D <= (uint64_t)kDenseRankLimit) bytes += D * D * 8;
  for (int d : L.block_dim) bytes += (uint64_t)d * d * 8 * 2;
  if (bytes > cfg.workspace_budget_bytes)
    fail(OMVGBA_RESOURCE_EXHAUSTED, "workspace " + std::to_string(bytes) + " bytes exceeds the workspace budget " +
                                        std::to_string(cfg.workspace_budget_bytes));
}

// Eigenvalues of a small symmetric matrix (row-major D x D) by cyclic Jacobi rotations.
static std::vector<double> jacobi_eigenvalues(std::vector<double> A, int D) {
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, scale = 0.0;
    for (int i = 0; i < D; ++i) {
      scale = std::max(scale, std::fabs(A[(size_t)i * D + i]));
      for (int j = i + 1; j < D; ++j) off += A[(size_t)i * D + j] * A[(size_t)i * D + j];
    }
    if (!(off > 1e-32 * scale * scale)) break;
    for (int p = 0; p < D; ++p)
      for (int q = p + 1; q < D; ++q) {
        const double apq = A[(size_t)p * D + q];
        if (apq == 0.0) continue;
        const double app = A[(size_t)p * D + p], aqq = A[(size_t)q * D + q];
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
        for (int k = 0; k < D; ++k) {
          const double akp = A[(size_t)k * D + p], akq = A[(size_t)k * D + q];
          A[(size_t)k * D + p] = c * akp - sn * akq;
          A[(size_t)k * D + q] = sn * akp + c * akq;
        }
        for (int k = 0; k < D; ++k) {
          const double apk = A[(size_t)p * D + k], aqk = A[(size_t)q * D + k];
          A[(size_t)p * D + k] = c * apk - sn * aqk;
          A[(size_t)q * D + k] = sn * apk + c * aqk;
        }
      }
  }
  std::vector<double> ev(D);
  for (int i = 0; i < D; ++i) ev[i] = A[(size_t)i * D + i];
  return ev;
}

// unobserved_free_intrinsics (native/mod.rs:465-478): intrinsic blocks with free variables that no
// observation uses; the calibrated, angular and two-view solutions report them unconstrained
static std::vector<uint64_t> unobserved_free_intrinsics(const omvgba_problem& pr) {
  std::vector<uint8_t> seen(pr.intrinsic_count, 0);
  for (size_t o = 0; o < pr.observation_count; ++o) seen[pr.observation_intrinsic[o]] = 1;
  std::vector<uint64_t> out;
  for (size_t i = 0; i < pr.intrinsic_count; ++i)
    if (!seen[i] && pr.intrinsics[i].variables != 0) out.push_back(i);
  return out;
}

// ---- two-view bundle adjustment (native/two_view.rs, kernel/two_view/{optimizer,schur,residual}.rs) ----
// Two cameras, the anchor fixed and the other free, every point seen once by each: the free pose
// has 5 coordinates (rotation and the S^2 direction of a translation of fixed length, the baseline)
// and points move in baseline units. A dense LM over the 5 x 5 reduced camera system.

// has_repeated_pose_points (native/mod.rs:500-506)
static bool has_repeated_pose_points(const omvgba_problem& pr) {
  std::set<std::pair<uint32_t, uint32_t>> seen;
  for (size_t o = 0; o < pr.observation_count; ++o)
    if (!seen.insert({pr.observation_pose[o], pr.observation_point[o]}).second) return true;
  return false;
}
static bool undistorted_perspective(const omvgba_intrinsic& in) {  // pinhole() (native/mod.rs:523-541)
  return in.model == OMVGBA_CAMERA_PINHOLE || (in.model == OMVGBA_CAMERA_BROWN_CONRADY && in.radial_kind == 0 &&
                                               in.tangential_kind == 0);
}
// can_use_two_view (native/two_view.rs:14-48)
static bool can_use_two_view(const omvgba_problem& pr) {
  if (pr.pose_count != 2 || pr.observation_count != 2 * pr.point_count || has_free_intrinsics(pr) ||
      has_repeated_pose_points(pr))
    return false;
  for (size_t i = 0; i < pr.point_count; ++i)
    if (point_fixed(pr, i)) return false;
  std::vector<size_t> intr;
  if (!single_pose_intrinsics(pr, &intr)) return false;
  size_t anchor;
  if (pr.gauge_kind == OMVGBA_GAUGE_FIXED_BASELINE) {
    anchor = pr.gauge_first;
  } else {
    anchor = pr.poses[0].variables == 0 ? 0 : (pr.poses[1].variables == 0 ? 1 : 2);
    if (anchor == 2) return false;
  }
  if (pr.poses[anchor].variables != 0 || pr.poses[1 - anchor].variables != OMVGBA_POSE_FREE) return false;
  if (pr.residual_space == OMVGBA_RESIDUAL_ANGULAR) return true;
  for (size_t k : intr)
    if (!undistorted_perspective(pr.intrinsics[k])) return false;
  return true;
}

struct TwoView {
  bool angular = false;
  double cam[2][4];                      // pixel: fx, fy, cx, cy per view
  std::vector<Vec2> obs[2];              // pixel measurements per view
  std::vector<Vec3> bearing[2];          // angular measurements per view
  std::optional<Projection> project(int view, size_t index, const Vec3& X) const {
    if (angular) return angular_projection(bearing[view][index], X);
    const double* c = cam[view];
    return pixel_projection(c[0], c[1], c[2], c[3], obs[view][index], X);
  }
};
struct TvLocal {  // LocalLinearization (schur.rs:15-72)
  double Hpp[5][5] = {}, Hpx[5][3] = {}, Hxx[3][3] = {}, gp[5] = {}, gx[3] = {}, cost = 0.0, sq = 0.0;
  void accumulate(const double r[2], const double Jp[2][5], const double Jx[2][3], double sw) {
    for (int k = 0; k < 2; ++k) {
      const double wr = sw * r[k];
      double wp[5], wx[3];
      for (int a = 0; a < 5; ++a) wp[a] = sw * Jp[k][a];
      for (int a = 0; a < 3; ++a) wx[a] = sw * Jx[k][a];
      for (int a = 0; a < 5; ++a) {
        gp[a] += wp[a] * wr;
        for (int b = 0; b < 5; ++b) Hpp[a][b] += wp[a] * wp[b];
        for (int b = 0; b < 3; ++b) Hpx[a][b] += wp[a] * wx[b];
      }
      for (int a = 0; a < 3; ++a) {
        gx[a] += wx[a] * wr;
        for (int b = 0; b < 3; ++b) Hxx[a][b] += wx[a] * wx[b];
      }
    }
  }
};
static double tv_scaled_ginf(const double* g, const double* d, int n) {  // scaled_gradient_inf_norm (schur.rs:414-430)
  double scale = 0.0;
  for (int i = 0; i < n; ++i) scale = std::max(scale, d[i]);
  if (!(std::isfinite(scale) && scale > 0.0)) {
    for (int i = 0; i < n; ++i)
      if (g[i] != 0.0) return kInf;
    return 0.0;
  }
  const double floor = 64.0 * kEps * scale;
  double best = 0.0;
  for (int i = 0; i < n; ++i) best = std::max(best, std::fabs(g[i]) / std::sqrt(std::max(d[i], floor)));
  return best;
}
// linearize_point (schur.rs:223-271)
static bool tv_linearize(const TwoView& tv, const NPose& pose, const std::array<Vec3, 2>& basis, double baseline,
                         const Vec3& X, size_t index, const Loss& loss, TvLocal* out) {
  *out = TvLocal{};
  auto first = tv.project(0, index, X);
  if (!first) return false;
  const double n1 = std::sqrt(first->residual[0] * first->residual[0] + first->residual[1] * first->residual[1]);
  out->cost += loss.cost(n1);
  out->sq += n1 * n1;
  double Jp0[2][5] = {}, Jx0[2][3];
  for (int r = 0; r < 2; ++r)
    for (int c = 0; c < 3; ++c) Jx0[r][c] = first->jacobian[r][c] * baseline;
  out->accumulate(first->residual.data(), Jp0, Jx0, loss.sqrt_weight(n1));
  const Vec3 rot = rotate(pose.R, X);
  const Vec3 xc = {rot[0] + pose.t[0], rot[1] + pose.t[1], rot[2] + pose.t[2]};
  auto second = tv.project(1, index, xc);
  if (!second) return false;
  const double n2 = std::sqrt(second->residual[0] * second->residual[0] + second->residual[1] * second->residual[1]);
  out->cost += loss.cost(n2);
  out->sq += n2 * n2;
  double Jx1[2][3], Jp1[2][5];
  for (int r = 0; r < 2; ++r)
    for (int c = 0; c < 3; ++c)
      Jx1[r][c] = (second->jacobian[r][0] * pose.R[0][c] + second->jacobian[r][1] * pose.R[1][c] +
                   second->jacobian[r][2] * pose.R[2][c]) *
                  baseline;
  const double m[3][5] = {{0.0, rot[2], -rot[1], baseline * basis[0][0], baseline * basis[1][0]},
                          {-rot[2], 0.0, rot[0], baseline * basis[0][1], baseline * basis[1][1]},
                          {rot[1], -rot[0], 0.0, baseline * basis[0][2], baseline * basis[1][2]}};
  for (int r = 0; r < 2; ++r)
    for (int c = 0; c < 5; ++c)
      Jp1[r][c] = second->jacobian[r][0] * m[0][c] + second->jacobian[r][1] * m[1][c] + second->jacobian[r][2] * m[2][c];
  out->accumulate(second->residual.data(), Jp1, Jx1, loss.sqrt_weight(n2));
  return true;
}
struct TvSystem {  // ReducedSystem (schur.rs:74-221)
  double H[5][5] = {}, g[5] = {}, cost = 0.0, sq = 0.0, full_g[5] = {}, diag[5] = {}, point_red = 0.0,
         point_ginf = 0.0, min_rcond = 1.0;
  uint64_t weak = 0;
  bool valid = true;
  void add(const TvLocal& l, double damping) {
    cost += l.cost;
    sq += l.sq;
    for (int r = 0; r < 5; ++r) {
      full_g[r] += l.gp[r];
      diag[r] += l.Hpp[r][r];
    }
    const double dx[3] = {l.Hxx[0][0], l.Hxx[1][1], l.Hxx[2][2]};
    point_ginf = std::max(point_ginf, tv_scaled_ginf(l.gx, dx, 3));
    Mat3 V;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) V[a][b] = l.Hxx[a][b];
    auto f = point_block_factor(V, damping);
    if (!f) {
      valid = false;
      if (damping == 0.0) {
        weak++;
        min_rcond = 0.0;
      }
      return;
    }
    if (damping == 0.0) {
      const double rc = point_rcond(*f, V);
      min_rcond = std::min(min_rcond, rc);
      if (rc <= kPointBlockRcondThreshold) weak++;
    }
    const Vec3 ig = f->solve({l.gx[0], l.gx[1], l.gx[2]});
    point_red += 0.5 * (l.gx[0] * ig[0] + l.gx[1] * ig[1] + l.gx[2] * ig[2]);
    Vec3 ic[5];
    for (int r = 0; r < 5; ++r) ic[r] = f->solve({l.Hpx[r][0], l.Hpx[r][1], l.Hpx[r][2]});
    for (int r = 0; r < 5; ++r) {
      g[r] += l.gp[r] - (l.Hpx[r][0] * ig[0] + l.Hpx[r][1] * ig[1] + l.Hpx[r][2] * ig[2]);
      for (int c = 0; c < 5; ++c)
        H[r][c] += l.Hpp[r][c] - (l.Hpx[r][0] * ic[c][0] + l.Hpx[r][1] * ic[c][1] + l.Hpx[r][2] * ic[c][2]);
    }
  }
  double floor_() const {
    double sc = 0.0;
    for (double d : diag) sc = std::max(sc, d);
    return 64.0 * kEps * std::max(sc, kMinPositive);
  }
  void finish_damping(double damping) {
    const double fl = floor_();
    for (int i = 0; i < 5; ++i) H[i][i] += damping * std::max(diag[i], fl);
  }
  bool is_valid() const {
    if (!valid) return false;
    for (int i = 0; i < 5; ++i) {
      if (!std::isfinite(g[i])) return false;
      for (int j = 0; j < 5; ++j)
        if (!std::isfinite(H[i][j])) return false;
    }
    return true;
  }
  double scaled_ginf() const { return std::max(point_ginf, tv_scaled_ginf(full_g, diag, 5)); }
  double predicted(const double step[5], double damping, double point_dn) const {
    double quad = 0.0;
    for (int r = 0; r < 5; ++r) {
      double hs = 0.0;
      for (int c = 0; c < 5; ++c) hs += H[r][c] * step[c];
      quad += step[r] * hs;
    }
    double gs = 0.0;
    for (int r = 0; r < 5; ++r) gs += g[r] * step[r];
    const double damped = point_red - gs - 0.5 * quad;
    const double fl = floor_();
    double pdn = 0.0;
    for (int r = 0; r < 5; ++r) pdn += std::max(diag[r], fl) * step[r] * step[r];
    return damped + 0.5 * damping * (pdn + point_dn);
  }
  int rank() const {  // camera_hessian_diagnostics (schur.rs:338-370): spectral rank, tol 64 eps n lambda_max
    if (!is_valid()) return 0;
    std::vector<double> A(25);
    for (int i = 0; i < 5; ++i)
      for (int j = 0; j < 5; ++j) A[5 * i + j] = 0.5 * (H[i][j] + H[j][i]);
    std::vector<double> ev = jacobi_eigenvalues(A, 5);
    double largest = 0.0;
    for (double e : ev) largest = std::max(largest, std::fabs(e));
    if (!(std::isfinite(largest) && largest > 0.0)) return 0;
    const double tol = 64.0 * kEps * 5.0 * largest;
    int r = 0;
    for (double e : ev) r += (std::isfinite(e) && e > tol) ? 1 : 0;
    return r;
  }
};
// point_step_with_damping_norm (schur.rs:278-301)
static bool tv_point_step(const TvLocal& l, double damping, const double ps[5], Vec3* step, double* dn) {
  Mat3 V;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) V[a][b] = l.Hxx[a][b];
  auto f = point_block_factor(V, damping);
  if (!f) return false;
  Vec3 rhs;
  for (int c = 0; c < 3; ++c) {
    double s = 0.0;
    for (int p = 0; p < 5; ++p) s += l.Hpx[p][c] * ps[p];
    rhs[c] = l.gx[c] + s;
  }
  const Vec3 x = f->solve(rhs);
  *step = {-x[0], -x[1], -x[2]};
  auto d = damping_diagonal(V);
  if (!d) return false;
  *dn = (*d)[0] * (*step)[0] * (*step)[0] + (*d)[1] * (*step)[1] * (*step)[1] + (*d)[2] * (*step)[2] * (*step)[2];
  return true;
}
// solve_positive_definite (numerics/refine/solver.rs:281-335) for the 5 x 5 camera system
static bool tv_solve_spd(const double A[5][5], const double b[5], double x[5]) {
  for (int i = 0; i < 5; ++i) {
    if (!std::isfinite(b[i])) return false;
    for (int j = 0; j < 5; ++j)
      if (!std::isfinite(A[i][j])) return false;
  }
  double L[5][5] = {};
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j <= i; ++j) {
      double acc = 0.0;
      for (int k = 0; k < j; ++k) acc += L[i][k] * L[j][k];
      double sum = A[i][j] - acc;
      if (!std::isfinite(sum)) return false;
      if (i == j) {
        if (sum <= 0.0) return false;
        L[i][j] = std::sqrt(sum);
      } else {
        L[i][j] = sum / L[j][j];
      }
    }
  double y[5];
  for (int i = 0; i < 5; ++i) {
    double sum = b[i];
    for (int j = 0; j < i; ++j) sum -= L[i][j] * y[j];
    y[i] = sum / L[i][i];
  }
  for (int i = 4; i >= 0; --i) {
    double sum = y[i];
    for (int j = i + 1; j < 5; ++j) sum -= L[j][i] * x[j];
    x[i] = sum / L[i][i];
  }
  for (int i = 0; i < 5; ++i)
    if (!std::isfinite(x[i])) return false;
  return true;
}
static bool tv_metrics(const TwoView& tv, const NPose& pose, const std::vector<Vec3>& points, const Loss& loss,
                       double* cost, double* rmse) {  // metrics (schur.rs:303-330)
  double total = 0.0, sq = 0.0;
  for (size_t i = 0; i < points.size(); ++i) {
    const Vec3 rot = rotate(pose.R, points[i]);
    const Vec3 xc = {rot[0] + pose.t[0], rot[1] + pose.t[1], rot[2] + pose.t[2]};
    for (int v = 0; v < 2; ++v) {
      auto p = tv.project(v, i, v == 0 ? points[i] : xc);
      if (!p) {
        *cost = *rmse = kInf;
        return false;
      }
      const double nrm = std::sqrt(p->residual[0] * p->residual[0] + p->residual[1] * p->residual[1]);
      total += loss.cost(nrm);
      sq += nrm * nrm;
    }
  }
  *cost = total;
  *rmse = std::sqrt(sq / double(4 * points.size()));
  return true;
}
static bool tv_reduced(const TwoView& tv, const NPose& pose, const std::array<Vec3, 2>& basis, double baseline,
                       const std::vector<Vec3>& points, const Loss& loss, double damping, TvSystem* sys) {
  *sys = TvSystem{};
  for (size_t i = 0; i < points.size(); ++i) {
    TvLocal l;
    if (!tv_linearize(tv, pose, basis, baseline, points[i], i, loss, &l)) return false;
    sys->add(l, damping);
  }
  sys->finish_damping(damping);
  return true;
}

struct TvReport {
  NPose pose;
  int status;
  int reason;
  uint64_t iterations, accepted, rej[4];
  double initial_cost, final_cost, initial_rmse, final_rmse, grad_norm, final_damping;
  int rank;
  uint64_t weak;
};

// refine_ba_2view (kernel/two_view/optimizer.rs:16-240)
static TvReport refine_two_view(NPose pose, std::vector<Vec3>& points, const TwoView& tv, const Options& opt) {
  if (points.size() < 5) fail(OMVGBA_NUMERICAL, "two-view bundle adjustment needs at least 5 points");
  const double baseline = norm3(pose.t);
  if (!all_finite(pose.t.data(), 3) || !(std::isfinite(baseline) && baseline > 64.0 * kEps))
    fail(OMVGBA_NUMERICAL, "two-view bundle adjustment translation is invalid");
  for (size_t i = 0; i < points.size(); ++i) {  // validate_projection_domain (optimizer.rs:396-415)
    const Vec3 rot = rotate(pose.R, points[i]);
    const Vec3 xc = {rot[0] + pose.t[0], rot[1] + pose.t[1], rot[2] + pose.t[2]};
    if (!tv.project(0, i, points[i]) || !tv.project(1, i, xc))
      fail(OMVGBA_NUMERICAL, "two-view bundle adjustment point " + std::to_string(i) + " is not projectable");
  }
  TvReport rep{};
  tv_metrics(tv, pose, points, opt.loss, &rep.initial_cost, &rep.initial_rmse);
  const auto st = stages(opt.loss, opt.max_iterations);
  const int target = final_stage_index(st);
  RunState run(1e-4);
  bool done = false;
  for (int si = 0; si < 3 && !done; ++si) {
    for (uint64_t it = 0; it < st[si].max_iterations; ++it) {
      run.iterations++;
      const double lambda = run.damping.value;
      const Vec3 dir = {pose.t[0] / baseline, pose.t[1] / baseline, pose.t[2] / baseline};
      const auto basis = s2_tangent_basis(dir);
      TvSystem sys;
      if (!tv_reduced(tv, pose, basis, baseline, points, st[si].loss, lambda, &sys) || !sys.is_valid()) {
        run.rej_lin++;
        run.damping.reject();
        continue;
      }
      const double current = sys.cost;
      if (si == target && run.gradient_converged(sys.scaled_ginf(), current, opt.criteria)) {
        done = true;
        break;
      }
      double raw[5], step[5];
      if (!tv_solve_spd(sys.H, sys.g, raw)) {
        run.rej_solve++;
        run.damping.reject();
        continue;
      }
      for (int k = 0; k < 5; ++k) step[k] = -raw[k];
      {  // limit_pose_step (optimizer.rs:432-443)
        const double rn = std::sqrt(step[0] * step[0] + step[1] * step[1] + step[2] * step[2]);
        const double tn = std::sqrt(step[3] * step[3] + step[4] * step[4]);
        const double len = std::max(rn, tn);
        if (len > 0.5)
          for (double& v : step) v *= 0.5 / len;
      }
      NPose cand;  // retract_pose (optimizer.rs:365-381)
      cand.R = mat_mul(exp_so3({step[0], step[1], step[2]}), pose.R);
      const Vec3 nd = retract_s2(dir, basis, step[3], step[4]);
      cand.t = {baseline * nd[0], baseline * nd[1], baseline * nd[2]};
      // candidate_cost (optimizer.rs:270-305)
      double cand_cost = 0.0, pss = 0.0, pdn = 0.0;
      bool ok = true;
      std::vector<Vec3> moved(points.size());
      for (size_t i = 0; i < points.size() && ok; ++i) {
        TvLocal l;
        Vec3 dx;
        double dn;
        if (!tv_linearize(tv, pose, basis, baseline, points[i], i, st[si].loss, &l) ||
            !tv_point_step(l, lambda, step, &dx, &dn)) {
          ok = false;
          break;
        }
        moved[i] = {points[i][0] + baseline * dx[0], points[i][1] + baseline * dx[1], points[i][2] + baseline * dx[2]};
        const Vec3 rot = rotate(cand.R, moved[i]);
        const Vec3 xc = {rot[0] + cand.t[0], rot[1] + cand.t[1], rot[2] + cand.t[2]};
        auto p0 = tv.project(0, i, moved[i]);
        auto p1 = tv.project(1, i, xc);
        if (!p0 || !p1) {
          ok = false;
          break;
        }
        cand_cost += st[si].loss.cost(std::sqrt(p0->residual[0] * p0->residual[0] + p0->residual[1] * p0->residual[1]));
        cand_cost += st[si].loss.cost(std::sqrt(p1->residual[0] * p1->residual[0] + p1->residual[1] * p1->residual[1]));
        pss += dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
        pdn += dn;
      }
      if (!ok) {
        run.rej_cand++;
        run.damping.reject();
        continue;
      }
      const double point_rms = std::sqrt(pss / double(points.size()));
      const double reduction = current - cand_cost;
      const double predicted = sys.predicted(step, lambda, pdn);
      if (run.accept_gain(reduction, predicted)) {
        points = moved;  // commit_points: the same back-substitution at the same state
        pose = cand;
        double ss = 0.0;
        for (double v : step) ss += v * v;
        const double prms = std::sqrt(ss / 5.0);
        const double sn = std::sqrt(prms * prms + point_rms * point_rms);
        const bool is_target = si == target;
        Criterion cc = run.record_accepted(sn, reduction, current, is_target, opt.criteria);
        if (is_target && run.certify(cc)) {
          done = true;
          break;
        }
      }
    }
  }
  const double baseline2 = baseline;
  const Vec3 dir = {pose.t[0] / baseline2, pose.t[1] / baseline2, pose.t[2] / baseline2};
  TvSystem fin;
  const bool have = tv_reduced(tv, pose, s2_tangent_basis(dir), baseline, points, opt.loss, 0.0, &fin);
  rep.rank = have ? fin.rank() : 0;
  rep.weak = have ? fin.weak : points.size();
  rep.status = run.status(rep.rank == 5 && rep.weak == 0);
  rep.reason = (int)run.convergence;
  rep.grad_norm = (have && fin.is_valid()) ? fin.scaled_ginf() : kInf;
  if (have) {
    rep.final_cost = fin.cost;
    rep.final_rmse = std::sqrt(fin.sq / double(4 * points.size()));
  } else {
    tv_metrics(tv, pose, points, opt.loss, &rep.final_cost, &rep.final_rmse);
  }
  rep.pose = pose;
  rep.iterations = run.iterations;
  rep.accepted = run.accepted;
  rep.rej[0] = run.rej_lin;
  rep.rej[1] = run.rej_solve;
  rep.rej[2] = run.rej_cand;
  rep.rej[3] = run.rej_insuff;
  rep.final_damping = run.damping.value;
  return rep;
}

// solve_two_view (native/two_view.rs:50-185)
static Result solve_two_view(const omvgba_problem& pr, const omvgba_config& cfg) {
  std::vector<size_t> intr;
  if (!single_pose_intrinsics(pr, &intr))
    fail(OMVGBA_UNSUPPORTED, "two-view lowering requires one calibration per pose");
  GaugePlan plan = gauge_plan(pr);
  const size_t var = plan.anchor == 0 ? 1 : 0;
  if (pr.poses[var].variables != OMVGBA_POSE_FREE || pr.poses[plan.anchor].variables != 0)
    fail(OMVGBA_UNSUPPORTED, "direct two-view lowering requires one fixed anchor and one full-pose camera");
  Native n;
  set_anchor(pr, n, plan.anchor, plan.scale);
  NPose pose = pose_to_native(n, pr.poses[var]);
  std::vector<Vec3> points(pr.point_count);
  for (size_t i = 0; i < pr.point_count; ++i) points[i] = point_to_native(n, point_at(pr, i));
  TwoView tv;
  tv.angular = pr.residual_space == OMVGBA_RESIDUAL_ANGULAR;
  std::vector<int> have[2] = {std::vector<int>(pr.point_count, -1), std::vector<int>(pr.point_count, -1)};
  for (size_t o = 0; o < pr.observation_count; ++o) {
    const int view = pr.observation_pose[o] == plan.anchor ? 0 : 1;
    have[view][pr.observation_point[o]] = (int)o;
  }
  for (int v = 0; v < 2; ++v) {
    const omvgba_intrinsic& in = pr.intrinsics[intr[v == 0 ? plan.anchor : var]];
    tv.cam[v][0] = in.fx;
    tv.cam[v][1] = in.fy;
    tv.cam[v][2] = in.cx;
    tv.cam[v][3] = in.cy;
    if (!tv.angular && !(std::isfinite(in.fx) && std::isfinite(in.fy) && std::isfinite(in.cx) && std::isfinite(in.cy) &&
                         in.fx > 0.0 && in.fy > 0.0))
      fail(OMVGBA_NUMERICAL, "two-view bundle adjustment intrinsics are invalid");
    for (size_t i = 0; i < pr.point_count; ++i) {
      const int o = have[v][i];
      if (o < 0) fail(OMVGBA_UNSUPPORTED, "direct two-view lowering requires complete two-view tracks");
      const Vec2 px = {pr.observation_pixel[2 * o], pr.observation_pixel[2 * o + 1]};
      tv.obs[v].push_back(px);
      if (tv.angular) {
        auto b = camera_bearing(in, px[0], px[1]);
        if (!b) fail(OMVGBA_NUMERICAL, "a measured pixel does not define a bearing of its camera model");
        tv.bearing[v].push_back(*b);
      }
    }
  }
  Options opt;
  opt.max_iterations = cfg.max_iterations;
  opt.loss = problem_loss(pr);
  opt.criteria = {cfg.gradient_tolerance, cfg.parameter_tolerance, cfg.function_tolerance};
  TvReport tr = refine_two_view(pose, points, tv, opt);
  Result res;
  res.poses.assign(pr.poses, pr.poses + pr.pose_count);
  pose_from_native(n, tr.pose, res.poses[var].rotation, res.poses[var].center);
  res.points.resize(3 * pr.point_count);
  for (size_t i = 0; i < pr.point_count; ++i) {
    const Vec3 X = point_from_native(n, points[i]);
    for (int k = 0; k < 3; ++k) res.points[3 * i + k] = X[k];
  }
  res.intrinsics.assign(pr.intrinsics, pr.intrinsics + pr.intrinsic_count);
  omvgba_report& r = res.report;  // two_view_solve_report (native/reporting.rs:143-182)
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
  double vals[4] = {r.initial_objective, r.final_objective, r.initial_rmse, r.final_rmse};
  for (double v : vals)
    if (!std::isfinite(v) || v < 0.0) fail(OMVGBA_INTERNAL, "bundle-adjustment report is invalid");
  res.unconstrained = unobserved_free_intrinsics(pr);
  r.unconstrained_intrinsic_count = res.unconstrained.size();
  return res;
}

// The lowering solve_once chooses (native/mod.rs:352-367): angular residuals (fixed intrinsics
// only), self-calibration, or the calibrated pixel problem.
static Native lower_native(const omvgba_problem& pr) {
  if (pr.residual_space == OMVGBA_RESIDUAL_ANGULAR) {
    if (has_free_intrinsics(pr)) fail(OMVGBA_UNSUPPORTED, "angular BA requires fixed intrinsics");
    return lower_calibrated(pr, true);
  }
  return has_free_intrinsics(pr) ? lower_self_calibrating(pr) : lower_calibrated(pr);
}

// ---- translation-only observability (native/fixed_rotation.rs, native/mod.rs:184-230, 435-447,
// native/reporting.rs:24-134) ----------------------------------------------------------------------
struct Preflight {
  int status = OMVGBA_PREFLIGHT_PROCEED;
  bool has_counts = false;
  uint64_t pose_dimension = 0, covered = 0, weak = 0;
  bool escalation = false;
};

// common_pose_variables (native/gauge.rs:9-40): 1 translation-only, 0 rotation and translation, -1
// an unsupported mixture
static int common_pose_variables(const omvgba_problem& pr) {
  auto observed = observed_cameras(pr);
  int selected = -1;
  for (size_t i = 0; i < pr.pose_count; ++i) {
    uint32_t v = pr.poses[i].variables;
    if (!observed[i] || v == 0) continue;
    if (!(v & OMVGBA_POSE_TRANSLATION)) return -1;
    int cand = (v & OMVGBA_POSE_ROTATION) ? 0 : 1;
    if (selected >= 0 && selected != cand) return -1;
    selected = cand;
  }
  return selected < 0 ? 0 : selected;
}

// can_probe_scale_representative (native/mod.rs:510-521)
static bool can_probe_scale_representative(const omvgba_problem& pr) {
  if (pr.gauge_kind != OMVGBA_GAUGE_FIXED_BASELINE) return true;
  auto observed = observed_cameras(pr);
  Vec3 f = pose_C(pr.poses[pr.gauge_first]);
  for (size_t c = 0; c < pr.pose_count; ++c)
    if (c != pr.gauge_first && observed[c] && !(pr.poses[c].variables & OMVGBA_POSE_TRANSLATION) &&
        pose_C(pr.poses[c]) != f)
      return false;
  return true;
}

// probe_prepared (native/fixed_rotation.rs:50-165) on the native state poses / points
static Preflight probe_prepared(const omvgba_problem& pr, const Native& n, const std::vector<NPose>& poses,
                                const std::vector<Vec3>& points) {
  FrProblem q;
  std::vector<size_t> pose_intr;
  single_pose_intrinsics(pr, &pose_intr);
  auto observed = observed_cameras(pr);
  const size_t fallback = pr.observation_count ? pr.observation_intrinsic[0] : 0;
  for (int c = 0; c < n.ncam; ++c) {
    const NPose& P = poses[c];
    q.rotations.push_back(P.R);
    Vec3 C = rotate_transposed(P.R, P.t);
    q.centers.push_back({-C[0], -C[1], -C[2]});
    q.fixed_cameras.push_back(n.fixed_poses[c]);
    const size_t src = n.camera_source_order[c];
    FrIntrinsics k{0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (!observed[src] && n.pixel_model) {
      k.fx = k.fy = 1.0;
    } else {
      const omvgba_intrinsic& in = pr.intrinsics[observed[src] ? pose_intr[src] : fallback];
      k.fx = in.fx;
      k.fy = in.fy;
      k.cx = in.cx;
      k.cy = in.cy;
      if (!n.pixel_model && in.model == OMVGBA_CAMERA_BROWN_CONRADY) {
        k.k1 = in.radial_kind >= 1 ? in.k1 : 0.0;
        k.k2 = in.radial_kind >= 2 ? in.k2 : 0.0;
        k.k3 = in.radial_kind >= 3 ? in.k3 : 0.0;
        k.p1 = in.tangential_kind >= 1 ? in.p1 : 0.0;
        k.p2 = in.tangential_kind >= 2 ? in.p2 : 0.0;
      }
    }
    q.intrinsics.push_back(k);
  }
  q.points = points;
  q.tracks.resize(points.size());
  for (size_t p = 0; p < points.size(); ++p)
    for (uint64_t o = n.pt_off[p]; o < n.pt_off[p + 1]; ++o) q.tracks[p].push_back({n.obs_cam[o], n.obs_px[o][0], n.obs_px[o][1]});
  q.anchor = 0;
  q.scale_camera = (size_t)std::max(n.gauge_cam, 0);
  q.fixed_baseline = pr.gauge_kind == OMVGBA_GAUGE_FIXED_BASELINE;
  if (q.fixed_baseline) {
    const Vec3& a = q.centers[0];
    const Vec3& b = q.centers[q.scale_camera];
    q.distance = std::sqrt(sqdist(b, a));
  }
  FrReport rep;
  try {
    rep = fr_probe(q, problem_loss(pr), FrOptions{});
  } catch (const FrError& e) {
    fail(OMVGBA_NUMERICAL, e.message);
  }
  uint64_t required = 0;
  for (int c = 1; c < n.ncam; ++c) required += n.fixed_poses[c] ? 0 : 1;
  Preflight out;
  out.has_counts = true;
  out.pose_dimension = rep.pose_dimension;
  out.covered = rep.covered_free_cameras;
  out.weak = rep.weak_point_count;
  switch (rep.status) {  // native_preflight_from_probe (native/fixed_rotation.rs:167-202)
    case kFrCertified: out.status = OMVGBA_PREFLIGHT_PROCEED; break;
    case kFrCoverage: out.status = OMVGBA_PREFLIGHT_INSUFFICIENT_CAMERA_COVERAGE; break;
    case kFrResource: out.status = OMVGBA_PREFLIGHT_RESOURCE_LIMIT; break;
    case kFrWeak: out.status = OMVGBA_PREFLIGHT_WEAK_POINT_GEOMETRY; break;
    default:
      if (rep.weak_point_count == 0 && rep.covered_free_cameras >= required) {
        out.status = OMVGBA_PREFLIGHT_PROCEED;
        out.escalation = true;
      } else {
        out.status = OMVGBA_PREFLIGHT_OBSERVABILITY_NOT_CERTIFIED;
      }
  }
  return out;
}

// certified_observability and the probe's details (native/reporting.rs:24-134)
static void apply_preflight(const omvgba_problem& pr, const Preflight& pf, omvgba_report& r) {
  if (r.observability == OMVGBA_OBS_NOT_ASSESSED && pf.status == OMVGBA_PREFLIGHT_PROCEED && !pf.escalation &&
      pf.weak == 0)
    r.observability = pr.gauge_kind == OMVGBA_GAUGE_FIXED_BASELINE ? OMVGBA_OBS_FULL_RANK : OMVGBA_OBS_ONLY_EXPECTED_GAUGE;
  const bool ranked = pf.status == OMVGBA_PREFLIGHT_PROCEED &&
                      (!pf.escalation || r.observability == OMVGBA_OBS_FULL_RANK ||
                       r.observability == OMVGBA_OBS_ONLY_EXPECTED_GAUGE);
  if (pf.pose_dimension == 0) fail(OMVGBA_INTERNAL, "bundle-adjustment report is invalid");
  r.has_observability_details = 1;
  r.details_pose_rank = ranked ? pf.pose_dimension : 0;
  r.details_pose_dimension = pf.pose_dimension;
  r.details_weak_point_count = pf.weak;
}

static bool wants_post_solve_probe(const omvgba_problem& pr, const Native& n) {
  bool fixed_points = false;
  for (size_t i = 0; i < pr.point_count; ++i) fixed_points = fixed_points || point_fixed(pr, i);
  return !n.self_cal && !n.angular && n.translation_only && !fixed_points && n.pixel_model &&
         can_probe_scale_representative(pr) && n.gauge_cam >= 0;
}

// NativeBundleAdjuster::preflight (native/mod.rs:184-230)
static Preflight preflight(const omvgba_problem& pr, const omvgba_config& cfg) {
  validate_config(cfg);
  bool fixed_points = false;
  for (size_t i = 0; i < pr.point_count; ++i) fixed_points = fixed_points || point_fixed(pr, i);
  if (common_pose_variables(pr) != 1 || pr.residual_space == OMVGBA_RESIDUAL_ANGULAR || fixed_points) return {};
  if (has_free_intrinsics(pr)) fail(OMVGBA_UNSUPPORTED, "direct native lowering does not support self-calibration");
  Native n = lower_calibrated(pr);
  std::vector<size_t> pose_intr;
  if (n.gauge_cam < 0 || !single_pose_intrinsics(pr, &pose_intr) || !can_probe_scale_representative(pr)) return {};
  return probe_prepared(pr, n, n.poses, n.points);
}

static Result solve_once(const omvgba_problem& pr, const omvgba_config& cfg) {
  validate_config(cfg);
  if (!(pr.residual_space != OMVGBA_RESIDUAL_ANGULAR && has_free_intrinsics(pr)) && can_use_two_view(pr)) {
    Result res = solve_two_view(pr, cfg);
    finish_solution(pr, res);
    canonicalize(pr, res);
    return res;
  }
  double t0 = oracle_now();
  Native n = lower_native(pr);
  oracle_phase("lowering", t0);
  Layout L = make_layout(n);
  Options opt;
  opt.max_iterations = cfg.max_iterations;
  opt.loss = problem_loss(pr);
  opt.criteria = {cfg.gradient_tolerance, cfg.parameter_tolerance, cfg.function_tolerance};
  opt.iterative = choose_iterative(cfg, n, L);
  check_workspace_budget(cfg, n, L);
  opt.pcg_tol = cfg.pcg_relative_tolerance > 0.0 ? cfg.pcg_relative_tolerance : 1e-1;
  opt.pcg_max = cfg.pcg_max_iterations > 0 ? cfg.pcg_max_iterations : 600;
  std::vector<NPose> poses = n.poses;
  std::vector<Vec3> points = n.points;
  std::vector<Radial> groups = n.groups;
  t0 = oracle_now();
  NativeReport nr = refine(n, poses, points, groups, opt);
  oracle_phase("refine", t0);
  std::vector<uint64_t> held;
  if (n.self_cal && g_certificate) {
    held = unconstrained_groups(pr, n, groups, nr, opt.loss);
    if (!held.empty()) {
      // re-solve from the input state with the unconstrained groups fixed
      // (native/self_calibration.rs:236-249); the second solve is not certified again
      for (uint64_t g : held) n.group_dim[g] = 0;
      poses = n.poses;
      points = n.points;
      groups = n.groups;
      Options again = opt;
      again.iterative = choose_iterative(cfg, n, make_layout(n));
      again.certify_intrinsics = false;
      t0 = oracle_now();
      nr = refine(n, poses, points, groups, again);
      oracle_phase("refine (held intrinsics)", t0);
    }
  }
  t0 = oracle_now();
  Result res = raise(pr, n, poses, points, groups, nr, opt.iterative);
  res.unconstrained = n.self_cal ? held : unobserved_free_intrinsics(pr);
  res.report.unconstrained_intrinsic_count = res.unconstrained.size();
  if (wants_post_solve_probe(pr, n)) apply_preflight(pr, probe_prepared(pr, n, poses, points), res.report);
  finish_solution(pr, res);
  canonicalize(pr, res);
  oracle_phase("report", t0);
  return res;
}

// ------------------------------------------------------------------------------------------
// Quarantine (quarantine.rs:34-96, native/mod.rs:260-340).
// ------------------------------------------------------------------------------------------
static std::vector<size_t> degenerate_points(const omvgba_problem& pr, const omvgba_pose* poses, const double* points) {
  size_t N = pr.observation_count;
  std::vector<Vec3> off(N);
  std::vector<double> dist(N);
  for (size_t o = 0; o < N; ++o) {
    size_t p = pr.observation_point[o];
    const double* C = poses[pr.observation_pose[o]].center;
    off[o] = {points[3 * p] - C[0], points[3 * p + 1] - C[1], points[3 * p + 2] - C[2]};
    dist[o] = norm3(off[o]);
  }
  double scene = 0.0;
  if (N > 0) {
    std::vector<double> d = dist;
    std::nth_element(d.begin(), d.begin() + N / 2, d.end());
    scene = d[N / 2];
  }
  std::vector<TrackGeometry> geo(pr.point_count, TrackGeometry(scene));
  for (size_t o = 0; o < N; ++o) geo[pr.observation_point[o]].push(off[o]);
  std::vector<size_t> out;
  for (size_t p = 0; p < pr.point_count; ++p)
    if (geo[p].degenerate()) out.push_back(p);
  return out;
}

struct Restricted {
  std::vector<omvgba_pose> poses;
  std::vector<omvgba_intrinsic> intrinsics;
  std::vector<double> points;
  std::vector<uint8_t> fixed;
  std::vector<uint32_t> op, oi, opt;
  std::vector<double> px;
  omvgba_problem view;
  std::vector<size_t> kept;
};
// BundleProblem::without_points (problem.rs:650-701)
static void without_points(const omvgba_problem& pr, const Result* warm, const std::set<size_t>& dropped, Restricted& r) {
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
  std::vector<size_t> ni(pr.point_count, SIZE_MAX);
  r.kept.clear();
  r.points.clear();
  r.fixed.clear();
  for (size_t i = 0; i < pr.point_count; ++i) {
    if (dropped.count(i)) continue;
    ni[i] = r.kept.size();
    r.kept.push_back(i);
    for (int k = 0; k < 3; ++k) r.points.push_back(warm ? warm->points[3 * i + k] : pr.points[3 * i + k]);
    r.fixed.push_back(point_fixed(pr, i));
  }
  r.op.clear();
  r.oi.clear();
  r.opt.clear();
  r.px.clear();
  for (size_t o = 0; o < pr.observation_count; ++o) {
    if (ni[pr.observation_point[o]] == SIZE_MAX) continue;
    r.op.push_back(pr.observation_pose[o]);
    r.oi.push_back(pr.observation_intrinsic[o]);
    r.opt.push_back((uint32_t)ni[pr.observation_point[o]]);
    r.px.push_back(pr.observation_pixel[2 * o]);
    r.px.push_back(pr.observation_pixel[2 * o + 1]);
  }
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

// Solution::weak_points (solver.rs:1149-1226)
static std::vector<size_t> weak_points(const omvgba_problem& pr, const Result& sol) {
  Loss loss = problem_loss(pr);
  size_t P = pr.point_count;
  std::vector<Mat3> blocks(P, Mat3{});
  std::vector<uint8_t> ok(P, 1);
  for (size_t o = 0; o < pr.observation_count; ++o) {
    size_t p = pr.observation_point[o];
    if (!ok[p]) continue;
    const omvgba_pose& pose = sol.poses[pr.observation_pose[o]];
    Mat3 R = pose_R(pose);
    Vec3 C = pose_C(pose);
    Vec3 xc = rotate(R, {sol.points[3 * p] - C[0], sol.points[3 * p + 1] - C[1], sol.points[3 * p + 2] - C[2]});
    Vec2 obs = {pr.observation_pixel[2 * o], pr.observation_pixel[2 * o + 1]};
    std::optional<Projection> pj;
    if (pr.residual_space == OMVGBA_RESIDUAL_ANGULAR) {
      auto b = camera_bearing(sol.intrinsics[pr.observation_intrinsic[o]], obs[0], obs[1]);
      if (b) pj = angular_projection(*b, xc);
    } else {
      pj = to_model(sol.intrinsics[pr.observation_intrinsic[o]]).project_with_jacobian(obs, xc);
    }
    double rn = pj ? std::hypot(pj->residual[0], pj->residual[1]) : kInf;
    if (!pj || !std::isfinite(rn)) {
      ok[p] = 0;
      continue;
    }
    Mat23 J;
    for (int r = 0; r < 2; ++r)
      for (int c = 0; c < 3; ++c)
        J[r][c] = pj->jacobian[r][0] * R[0][c] + pj->jacobian[r][1] * R[1][c] + pj->jacobian[r][2] * R[2][c];
    double w = loss.sqrt_weight(rn);
    w *= w;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) blocks[p][i][j] += w * (J[0][i] * J[0][j] + J[1][i] * J[1][j]);
  }
  std::vector<uint8_t> deg(P, 0);
  for (auto q : sol.quarantined) deg[q] = 1;
  for (size_t p : degenerate_points(pr, sol.poses.data(), sol.points.data()))
    if (!point_fixed(pr, p)) deg[p] = 1;
  std::vector<size_t> out;
  for (size_t p = 0; p < P; ++p) {
    bool weak = deg[p];
    if (!weak && !point_fixed(pr, p)) {
      if (!ok[p])
        weak = true;
      else {
        // symmetric 3x3 eigenvalues by cyclic Jacobi
        std::vector<double> A(9);
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) A[i * 3 + j] = blocks[p][i][j];
        for (int sweep = 0; sweep < 50; ++sweep)
          for (int a = 0; a < 3; ++a)
            for (int b = a + 1; b < 3; ++b) {
              double apq = A[a * 3 + b];
              if (std::fabs(apq) < 1e-300) continue;
              double th = (A[b * 3 + b] - A[a * 3 + a]) / (2.0 * apq);
              double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
              double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
              for (int k = 0; k < 3; ++k) {
                double x = A[k * 3 + a], y = A[k * 3 + b];
                A[k * 3 + a] = c * x - s * y;
                A[k * 3 + b] = s * x + c * y;
              }
              for (int k = 0; k < 3; ++k) {
                double x = A[a * 3 + k], y = A[b * 3 + k];
                A[a * 3 + k] = c * x - s * y;
                A[b * 3 + k] = s * x + c * y;
              }
            }
        double mx = std::max({A[0], A[4], A[8]}), mn = std::min({A[0], A[4], A[8]});
        double thr = kPointBlockQuarantineRcond * mx;
        weak = !(mn > thr);
      }
    }
    if (weak) out.push_back(p);
  }
  return out;
}

static bool needs_resolve(const Result& r) {
  return (r.report.has_weak_point_count && r.report.weak_point_count > 0) ||
         r.report.observability == OMVGBA_OBS_RANK_DEFICIENT || r.report.status == OMVGBA_STATUS_DEGENERATE;
}

static Result solve_with_quarantine(const omvgba_problem& pr, const omvgba_config& cfg) {
  validate_config(cfg);
  std::vector<uint64_t> counts(pr.point_count, 0);
  for (size_t o = 0; o < pr.observation_count; ++o) counts[pr.observation_point[o]]++;
  std::vector<uint8_t> weak(pr.point_count, 0);
  for (size_t p = 0; p < pr.point_count; ++p) weak[p] = counts[p] < 2;
  double t0 = oracle_now();
  for (size_t p : degenerate_points(pr, pr.poses, pr.points)) weak[p] = 1;
  oracle_phase("degenerate points", t0);
  std::set<size_t> input_deg;
  for (size_t p = 0; p < pr.point_count; ++p)
    if (weak[p] && !point_fixed(pr, p)) input_deg.insert(p);
  if (input_deg.size() == pr.point_count)
    fail(OMVGBA_UNSUPPORTED, "no point can be adjusted: every point is seen fewer than twice or without parallax");
  Restricted first;
  const omvgba_problem* working = &pr;
  std::vector<size_t> kept(pr.point_count);
  std::iota(kept.begin(), kept.end(), 0);
  if (!input_deg.empty()) {
    without_points(pr, nullptr, input_deg, first);
    working = &first.view;
    kept = first.kept;
  }
  size_t quarantined = input_deg.size();
  bool changes_scale = false;
  if (pr.gauge_kind == OMVGBA_GAUGE_FIXED_BASELINE) changes_scale = std::fabs(gauge_plan(pr).scale - 1.0) > 1e-9;
  if (changes_scale && quarantined > 0)
    fail(OMVGBA_UNSUPPORTED, "native BA cannot change its physical baseline while holding out points");
  Result sol = solve_once(*working, cfg);
  omvgba_config retry = cfg;
  retry.max_iterations = std::min<uint64_t>(cfg.max_iterations, 8);
  std::vector<Restricted> chain;
  chain.reserve(4);
  const omvgba_problem* current = working;
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
      resolved = solve_once(next.view, retry);
    } catch (const SolveFailure&) {
      chain.pop_back();
      break;
    }
    std::vector<size_t> nk;
    for (size_t k : next.kept) nk.push_back(kept[k]);
    kept = nk;
    quarantined += wk.size();
    // SolveReport::continued_from (solver.rs:387-400)
    omvgba_report prev = sol.report;
    if (have_origin) {
      prev.initial_objective = origin.initial_objective;
      prev.initial_rmse = origin.initial_rmse;
      prev.iteration_count += origin.iteration_count;
      prev.accepted_step_count += origin.accepted_step_count;
      prev.rejected_step_count += origin.rejected_step_count;
      prev.rejected_linearization += origin.rejected_linearization;
      prev.rejected_step_solve += origin.rejected_step_solve;
      prev.rejected_candidate += origin.rejected_candidate;
      prev.rejected_insufficient_reduction += origin.rejected_insufficient_reduction;
    }
    origin = prev;
    have_origin = true;
    sol = resolved;
    current = &next.view;
  }
  if (changes_scale && quarantined > 0)
    fail(OMVGBA_UNSUPPORTED, "native BA cannot change its physical baseline while holding out points");
  if (quarantined == 0) return sol;
  // Solution::lifted (solver.rs:891-940)
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
  if (have_origin) {
    auto& r = out.report;
    r.initial_objective = origin.initial_objective;
    r.initial_rmse = origin.initial_rmse;
    r.iteration_count += origin.iteration_count;
    r.accepted_step_count += origin.accepted_step_count;
    r.rejected_step_count += origin.rejected_step_count;
    r.rejected_linearization += origin.rejected_linearization;
    r.rejected_step_solve += origin.rejected_step_solve;
    r.rejected_candidate += origin.rejected_candidate;
    r.rejected_insufficient_reduction += origin.rejected_insufficient_reduction;
  }
  finish_solution(pr, out);
  return out;
}

static int write_error(omvgba_error* e, int code, const std::string& msg) {
  if (e) {
    e->code = code;
    e->detail = -1;
    std::snprintf(e->message, sizeof(e->message), "%s", msg.c_str());
  }
  return code;
}

}  // namespace oracle

using namespace oracle;

extern "C" {

void omvgba_oracle_set_threads(int threads) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
}
// Forces the number of point shards (0 restores the topology rule). Changing it only regroups the
// floating-point sums, which measures the algorithm's own rounding sensitivity.
void omvgba_oracle_set_shards(int shards) { g_forced_shards = shards; }

// Timing runs of the bench switch off the final certificate's band factorization (the rank above
// D = 2048 and the self-calibration marginals); it does not run inside the LM loop they time.
void omvgba_oracle_set_certificate(int on) { oracle::g_certificate = on != 0; }

// Wall time of each LM iteration of the calling thread's last omvgba_oracle_solve, in order (the
// solve and, when the self-calibration certificate held groups, the re-solve); returns the count and
// writes at most cap values.
int omvgba_oracle_iteration_seconds(double* out, int cap) {
  const int n = (int)oracle::tl_iteration_seconds.size();
  for (int i = 0; i < n && i < cap; ++i) out[i] = oracle::tl_iteration_seconds[i];
  return n;
}

// The oracle's preflight (NativeBundleAdjuster::preflight) and its kernel-level probe.
int omvgba_oracle_preflight(const omvgba_problem* problem, const omvgba_config* config, omvgba_preflight* out,
                            omvgba_error* error) {
  try {
    oracle::validate_problem(*problem);
    oracle::Preflight pf = oracle::preflight(*problem, *config);
    std::memset(out, 0, sizeof(*out));
    out->status = pf.status;
    out->has_counts = pf.has_counts ? 1 : 0;
    out->pose_dimension = pf.pose_dimension;
    out->covered_free_pose_count = pf.covered;
    out->weak_point_count = pf.weak;
    out->dense_observability_escalation = pf.escalation ? 1 : 0;
    return OMVGBA_OK;
  } catch (const oracle::SolveFailure& f) {
    return write_error(error, f.code, f.message);
  }
}

int omvgba_oracle_probe_fixed_rotation(const omvgba_fixed_rotation_problem* fp, const omvgba_probe_options* opt,
                                       omvgba_probe_report* out, omvgba_error* error) {
  try {
    oracle::FrProblem q;
    for (uint64_t c = 0; c < fp->camera_count; ++c) {
      oracle::Mat3 R;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) R[i][j] = fp->rotations[9 * c + 3 * i + j];
      q.rotations.push_back(R);
      q.centers.push_back({fp->centers[3 * c], fp->centers[3 * c + 1], fp->centers[3 * c + 2]});
      const double* k = fp->intrinsics + 9 * c;
      q.intrinsics.push_back({k[0], k[1], k[2], k[3], k[4], k[5], k[6], k[7], k[8]});
      q.fixed_cameras.push_back(fp->fixed_cameras[c] ? 1 : 0);
    }
    for (uint64_t p = 0; p < fp->point_count; ++p) {
      q.points.push_back({fp->points[3 * p], fp->points[3 * p + 1], fp->points[3 * p + 2]});
      std::vector<oracle::FrObservation> t;
      for (uint64_t o = fp->track_offsets[p]; o < fp->track_offsets[p + 1]; ++o)
        t.push_back({fp->observation_camera[o], fp->observation_pixel[2 * o], fp->observation_pixel[2 * o + 1]});
      q.tracks.push_back(t);
    }
    q.fixed_baseline = fp->gauge_kind == OMVGBA_GAUGE_FIXED_BASELINE;
    q.anchor = fp->anchor;
    q.scale_camera = fp->scale_camera;
    q.distance = fp->distance;
    oracle::Loss loss;
    loss.kind = fp->loss_kind == OMVGBA_LOSS_HUBER ? oracle::LossKind::Huber
                                                    : (fp->loss_kind == OMVGBA_LOSS_CAUCHY ? oracle::LossKind::Cauchy
                                                                                            : oracle::LossKind::L2);
    loss.scale = fp->loss_scale;
    oracle::FrOptions o;
    o.max_tracks = opt->max_tracks;
    o.max_observations = opt->max_observations;
    o.max_observations_per_track = opt->max_observations_per_track;
    o.max_coverage_observations_per_track = opt->max_coverage_observations_per_track;
    o.max_reduced_nonzeros = opt->max_reduced_nonzeros;
    o.max_factor_nonzeros = opt->max_factor_nonzeros;
    o.max_symbolic_dense_nonzeros = opt->max_symbolic_dense_nonzeros;
    o.minimum_normalized_eigenvalue = opt->minimum_normalized_eigenvalue;
    oracle::FrReport r = oracle::fr_probe(q, loss, o);
    std::memset(out, 0, sizeof(*out));
    out->status = r.status;
    out->pose_dimension = r.pose_dimension;
    out->selected_tracks = r.selected_tracks;
    out->selected_observations = r.selected_observations;
    out->covered_free_cameras = r.covered_free_cameras;
    out->weak_point_count = r.weak_point_count;
    out->reduced_nonzeros = r.reduced_nonzeros;
    out->factor_nonzeros = r.factor_nonzeros;
    return OMVGBA_OK;
  } catch (const oracle::FrError& e) {
    return write_error(error, e.code, e.message);
  } catch (const oracle::SolveFailure& f) {
    return write_error(error, f.code, f.message);
  }
}

// The oracle's execution plan: the linear solver it would use (Auto resolved) and its estimates.
int omvgba_oracle_execution_plan(const omvgba_problem* problem, const omvgba_config* config, int32_t* iterative,
                                 uint64_t* direct_estimate, uint64_t* cached_estimate, omvgba_error* error) {
  try {
    oracle::validate_problem(*problem);
    oracle::validate_config(*config);
    // the solve's input quarantine first (quarantine.rs:34-96): points seen fewer than twice or
    // without parallax are held out before the lowering
    const omvgba_problem& pr = *problem;
    std::vector<uint64_t> counts(pr.point_count, 0);
    for (size_t o = 0; o < pr.observation_count; ++o) counts[pr.observation_point[o]]++;
    std::set<size_t> held;
    for (size_t p = 0; p < pr.point_count; ++p)
      if (counts[p] < 2 && !oracle::point_fixed(pr, p)) held.insert(p);
    for (size_t p : oracle::degenerate_points(pr, pr.poses, pr.points))
      if (!oracle::point_fixed(pr, p)) held.insert(p);
    oracle::Restricted first;
    const omvgba_problem* working = &pr;
    if (!held.empty()) {
      oracle::without_points(pr, nullptr, held, first);
      working = &first.view;
    }
    oracle::Native n = oracle::lower_native(*working);
    oracle::Layout L = oracle::make_layout(n);
    const bool direct = oracle::auto_prefers_direct(
        n, L, config->has_workspace_budget ? config->workspace_budget_bytes : 0, direct_estimate, cached_estimate);
    *iterative = oracle::choose_iterative(*config, n, L) ? 1 : 0;
    (void)direct;
    return OMVGBA_OK;
  } catch (const oracle::SolveFailure& f) {
    return write_error(error, f.code, f.message);
  }
}

int omvgba_oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int32_t omvgba_oracle_solve(const omvgba_problem* problem, const omvgba_config* config, omvgba_solution* solution,
                            omvgba_error* error) {
  if (error) {
    error->code = 0;
    error->detail = -1;
    error->message[0] = 0;
  }
  if (!problem || !config || !solution) return write_error(error, OMVGBA_INVALID_ARGUMENT, "null argument");
  try {
    validate_problem(*problem);
    oracle::tl_iteration_seconds.clear();
    Result r = solve_with_quarantine(*problem, *config);
    std::memcpy(solution->poses, r.poses.data(), sizeof(omvgba_pose) * problem->pose_count);
    std::memcpy(solution->intrinsics, r.intrinsics.data(), sizeof(omvgba_intrinsic) * problem->intrinsic_count);
    std::memcpy(solution->points, r.points.data(), sizeof(double) * 3 * problem->point_count);
    if (solution->quarantined_points)
      for (size_t i = 0; i < r.quarantined.size(); ++i) solution->quarantined_points[i] = r.quarantined[i];
    if (solution->unconstrained_intrinsics)
      for (size_t i = 0; i < r.unconstrained.size(); ++i) solution->unconstrained_intrinsics[i] = r.unconstrained[i];
    solution->report = r.report;
    return OMVGBA_OK;
  } catch (const SolveFailure& f) {
    return write_error(error, f.code, f.message);
  } catch (const std::exception& ex) {
    return write_error(error, OMVGBA_INTERNAL, ex.what());
  }
}

// First linearization of the lowered problem, per observation in point-major order.
int32_t omvgba_oracle_debug_linearize(const omvgba_problem* problem, const omvgba_config* config, double* residual,
                                      double* sqrt_weight, double* point_jacobian, double* camera_jacobian,
                                      uint64_t* source_index, omvgba_error* error) {
  try {
    validate_problem(*problem);
    validate_config(*config);
    Native n = lower_native(*problem);
    Layout L = make_layout(n);
    double scene = n.self_cal ? scene_scale_plain(n, n.poses, n.points) : scene_scale_observed(n, n.poses, n.points);
    GaugeState g = make_gauge(n, n.poses, scene);
    Loss loss = problem_loss(*problem);
    for (size_t p = 0; p < n.points.size(); ++p)
      for (uint64_t o = n.pt_off[p]; o < n.pt_off[p + 1]; ++o) {
        int cam = n.obs_cam[o];
        const NPose& P = n.poses[cam];
        Vec3 rot = rotate(P.R, n.points[p]);
        Vec3 xc = {rot[0] + P.t[0], rot[1] + P.t[1], rot[2] + P.t[2]};
        ObsLin ol;
        source_index[o] = n.obs_src[o];
        for (int k = 0; k < 18; ++k) camera_jacobian[18 * o + k] = 0.0;
        if (!project_obs(n, n.groups, o, xc, &ol)) {
          residual[2 * o] = residual[2 * o + 1] = std::nan("");
          sqrt_weight[o] = std::nan("");
          for (int k = 0; k < 6; ++k) point_jacobian[6 * o + k] = std::nan("");
          continue;
        }
        residual[2 * o] = ol.p.residual[0];
        residual[2 * o + 1] = ol.p.residual[1];
        sqrt_weight[o] = loss.sqrt_weight(std::sqrt(ol.p.residual[0] * ol.p.residual[0] + ol.p.residual[1] * ol.p.residual[1]));
        for (int r = 0; r < 2; ++r)
          for (int c = 0; c < 3; ++c)
            point_jacobian[6 * o + 3 * r + c] =
                (ol.p.jacobian[r][0] * P.R[0][c] + ol.p.jacobian[r][1] * P.R[1][c] + ol.p.jacobian[r][2] * P.R[2][c]) *
                g.scene_scale;
        int pd = L.pose_dim[cam];
        if (pd > 0) {
          double Jc[2][9] = {};
          pose_columns(n, L, g, cam, rot, xc, ol.p.jacobian, Jc);
          for (int r = 0; r < 2; ++r)
            for (int c = 0; c < pd; ++c) camera_jacobian[18 * o + 9 * r + c] = Jc[r][c];
        }
        if (n.self_cal) {
          int grp = n.cam_group[cam];
          for (int r = 0; r < 2; ++r)
            for (int c = 0; c < L.intr_dim[grp]; ++c) camera_jacobian[18 * o + 9 * r + pd + c] = ol.jint[r][c];
        }
      }
    return OMVGBA_OK;
  } catch (const SolveFailure& f) {
    return write_error(error, f.code, f.message);
  }
}

// Known-answer hooks for the oracle pins.
double omvgba_oracle_loss_cost(int kind, double scale, double r) {
  Loss l{(LossKind)kind, scale};
  return l.cost(r);
}
double omvgba_oracle_loss_sqrt_weight(int kind, double scale, double r) {
  Loss l{(LossKind)kind, scale};
  return l.sqrt_weight(r);
}
// Radial projection: out[0..2) residual, out[2..8) d pred / d camera point, out[8..14) intrinsic J.
int omvgba_oracle_radial_linearize(double f, double k1, double k2, const double* obs, const double* X, double* out) {
  Radial cam{f, k1, k2};
  auto t = radial_terms(cam, {X[0], X[1], X[2]});
  if (!t) return 0;
  auto p = radial_projection(cam, {obs[0], obs[1]}, *t);
  auto j = radial_intrinsic_jacobian(cam, *t);
  if (!p || !j) return 0;
  out[0] = p->residual[0];
  out[1] = p->residual[1];
  for (int r = 0; r < 2; ++r)
    for (int c = 0; c < 3; ++c) {
      out[2 + 3 * r + c] = p->jacobian[r][c];
      out[8 + 3 * r + c] = (*j)[r][c];
    }
  return 1;
}
// Brown–Conrady projection with Jacobian: out[0..2) pixel, out[2..8) Jacobian.
int omvgba_oracle_bc_project(const omvgba_intrinsic* in, const double* X, double* out) {
  BrownConrady m = to_model(*in);
  auto p = m.project_with_jacobian({0.0, 0.0}, {X[0], X[1], X[2]});
  if (!p) return 0;
  out[0] = p->residual[0];
  out[1] = p->residual[1];
  for (int r = 0; r < 2; ++r)
    for (int c = 0; c < 3; ++c) out[2 + 3 * r + c] = p->jacobian[r][c];
  return 1;
}
int omvgba_oracle_camera_bearing(const omvgba_intrinsic* in, double u, double v, double* out) {
  auto b = camera_bearing(*in, u, v);
  if (!b) return 0;
  for (int k = 0; k < 3; ++k) out[k] = (*b)[k];
  return 1;
}
int omvgba_oracle_angular_projection(const double* bearing, const double* X, double* out) {
  auto p = angular_projection({bearing[0], bearing[1], bearing[2]}, {X[0], X[1], X[2]});
  if (!p) return 0;
  out[0] = p->residual[0];
  out[1] = p->residual[1];
  for (int r = 0; r < 2; ++r)
    for (int c = 0; c < 3; ++c) out[2 + 3 * r + c] = p->jacobian[r][c];
  return 1;
}
int omvgba_oracle_bc_remove_distortion(const omvgba_intrinsic* in, double xd, double yd, double* xy) {
  BrownConrady m = to_model(*in);
  return m.remove_distortion(xd, yd, &xy[0], &xy[1]) ? 1 : 0;
}
// Nielsen controller trace: ops[i] = 0 reject, 1 accept(a[i], p[i]); writes damping after each op and the
// accept result (or -1 for rejects).
void omvgba_oracle_nielsen(int count, const int* ops, const double* actual, const double* predicted, double initial,
                           double* damping_out, int* accepted_out, double* gain_out, int* has_gain_out) {
  Nielsen n(initial);
  for (int i = 0; i < count; ++i) {
    if (ops[i] == 0) {
      n.reject();
      accepted_out[i] = -1;
    } else {
      accepted_out[i] = n.accept(actual[i], predicted[i]) ? 1 : 0;
    }
    damping_out[i] = n.value;
    gain_out[i] = n.gain;
    has_gain_out[i] = n.has_gain ? 1 : 0;
  }
}
void omvgba_oracle_exp_so3(const double* v, double* R) {
  Mat3 m = exp_so3({v[0], v[1], v[2]});
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) R[3 * i + j] = m[i][j];
}
int omvgba_oracle_point_block_inverse(const double* V, double lambda, double* inverse_packed, double* rcond) {
  Mat3 m;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) m[i][j] = V[3 * i + j];
  auto f = point_block_factor(m, lambda);
  if (!f) return 0;
  for (int i = 0; i < 6; ++i) inverse_packed[i] = f->inverse[i];
  *rcond = point_rcond(*f, m);
  return 1;
}
void omvgba_oracle_stages(int loss_kind, uint64_t max_iterations, uint64_t* budgets, int* kinds) {
  Loss l{(LossKind)loss_kind, 1.0};
  auto s = stages(l, max_iterations);
  for (int i = 0; i < 3; ++i) {
    budgets[i] = s[i].max_iterations;
    kinds[i] = (int)s[i].loss.kind;
  }
}
// Analytic reprojection residual and J^T v for the centred radial model over an unsorted list:
// the oracle for the GPU adjoint kernel. Cameras: rotvec, translation, intrinsics (f, k1, k2).
void omvgba_oracle_residual_vjp(uint64_t n, const uint32_t* cam, const uint32_t* pt, const double* px,
                                const double* rotvec, const double* trans, const double* intr, const double* points,
                                const double* grad, double* residual, double* g_rot, double* g_t, double* g_int,
                                double* g_pt) {
  for (uint64_t i = 0; i < n; ++i) {
    uint32_t c = cam[i], p = pt[i];
    Vec3 w = {rotvec[3 * c], rotvec[3 * c + 1], rotvec[3 * c + 2]};
    Mat3 R = exp_so3(w);
    Vec3 X = {points[3 * p], points[3 * p + 1], points[3 * p + 2]};
    Vec3 rx = rotate(R, X);
    Vec3 xc = {rx[0] + trans[3 * c], rx[1] + trans[3 * c + 1], rx[2] + trans[3 * c + 2]};
    Radial cm{intr[3 * c], intr[3 * c + 1], intr[3 * c + 2]};
    auto t = radial_terms(cm, xc);
    std::optional<Projection> pr;
    if (t) pr = radial_projection(cm, {px[2 * i], px[2 * i + 1]}, *t);
    if (!t || !pr) {
      residual[2 * i] = residual[2 * i + 1] = std::nan("");
      continue;
    }
    residual[2 * i] = pr->residual[0];
    residual[2 * i + 1] = pr->residual[1];
    if (!grad) continue;
    double g0 = grad[2 * i], g1 = grad[2 * i + 1];
    // d r / d xc = J (2x3); adjoint a = J^T g
    Vec3 a;
    for (int k = 0; k < 3; ++k) a[k] = pr->jacobian[0][k] * g0 + pr->jacobian[1][k] * g1;
    // translation: d xc / d t = I
    for (int k = 0; k < 3; ++k) g_t[3 * c + k] += a[k];
    // point: d xc / d X = R
    Vec3 ap = rotate_transposed(R, a);
    for (int k = 0; k < 3; ++k) g_pt[3 * p + k] += ap[k];
    // rotation vector: numeric-free analytic via left perturbation is not the rotvec derivative; use the
    // SO(3) right Jacobian: d(exp(w) X)/dw = -[R X]x Jl(w)
    double th = norm3(w);
    Mat3 Jl;
    if (th < 1e-8) {
      Mat3 k = skew(w);
      for (int r = 0; r < 3; ++r)
        for (int s = 0; s < 3; ++s) Jl[r][s] = (r == s ? 1.0 : 0.0) + 0.5 * k[r][s];
    } else {
      Mat3 k = skew(w);
      Mat3 k2 = mat_mul(k, k);
      double A = (1.0 - std::cos(th)) / (th * th), B = (th - std::sin(th)) / (th * th * th);
      for (int r = 0; r < 3; ++r)
        for (int s = 0; s < 3; ++s) Jl[r][s] = (r == s ? 1.0 : 0.0) + A * k[r][s] + B * k2[r][s];
    }
    // d xc / d w = -[rx]x Jl ; adjoint: Jl^T (-[rx]x)^T a = Jl^T ([rx]x a) = Jl^T (rx x a)
    Vec3 ca = cross3(rx, a);
    for (int s = 0; s < 3; ++s) g_rot[3 * c + s] += Jl[0][s] * ca[0] + Jl[1][s] * ca[1] + Jl[2][s] * ca[2];
    auto ji = radial_intrinsic_jacobian(cm, *t);
    if (ji) {
      // intrinsics are (f, k1, k2); the radial Jacobian column 0 is d/d log f = f * d/df
      g_int[3 * c] += ((*ji)[0][0] * g0 + (*ji)[1][0] * g1) / cm.focal;
      g_int[3 * c + 1] += (*ji)[0][1] * g0 + (*ji)[1][1] * g1;
      g_int[3 * c + 2] += (*ji)[0][2] * g0 + (*ji)[1][2] * g1;
    }
  }
}

}  // extern "C"
