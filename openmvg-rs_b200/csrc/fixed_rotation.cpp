// fixed_rotation.cpp — the observability probe of translation-only problems
// (probe_fixed_rotation_observability, crates/openmvg-ba/src/kernel/fixed_rotation/observability.rs:
// 24-262; options and outcome in kernel/fixed_rotation/api.rs, validation in
// kernel/fixed_rotation/validation.rs).
//
// With the rotations and intrinsics held, the unknowns are the free camera centres and the points. A
// capped subset of tracks (shortest first, covering every free camera) is linearized; each point is
// eliminated in square-root form, Z_a = (E_a - Q Q_a^T) J_a with Q the thin QR factor of the point's
// stacked whitened Jacobians, so its camera blocks Z_a^T Z_b are positive semidefinite by construction;
// the camera system is scaled to unit diagonal and shifted by minimum_normalized_eigenvalue, and it
// must factor. Success certifies the whole problem (omitted tracks only add positive semidefinite
// terms).
//
// Where it runs: the selection and the per-point elimination (bounded by max_observations, 1e5 by
// default) run on host threads, one fixed chunk of tracks each, merged in selection order, so the
// result does not depend on the thread count; the factorization, the only superlinear step, runs on
// the device as the banded tiled FP64 Cholesky of the explicit reduced camera system
// (device_certify_positive_definite). The reference factors with faer's simplicial sparse LLT after
// an AMD ordering; here the coordinates keep their camera order (a survey's band), the decision is
// the same away from rounding-level pivots, and factor_nonzeros counts the profile of that order.
#include "fixed_rotation.hpp"

#include <algorithm>
#include <cmath>
#include <string>
#include <thread>
#include <unordered_map>

#include "gpu_solver.hpp"

namespace omvgba {

void probe_options_default(omvgba_probe_options* o) {  // FixedRotationObservabilityProbeOptions::default
  o->max_tracks = 25000;
  o->max_observations = 100000;
  o->max_observations_per_track = 32;
  o->max_coverage_observations_per_track = 256;
  o->max_reduced_nonzeros = 1000000;
  o->max_factor_nonzeros = 4000000;
  o->max_symbolic_dense_nonzeros = 32000000;
  o->minimum_normalized_eigenvalue = 1e-10;
}

namespace {

[[noreturn]] void reject(int code, const char* message) { throw SolveFailure{code, message}; }

void validate(const ProbeProblem& p, const omvgba_probe_options& o) {
  // validate_problem (validation.rs:27-117), then validate_probe_options (validation.rs:6-25)
  const size_t n = p.cameras.size(), P = p.points.size() / 3;
  if (n < 2 || P == 0 || p.track_off.size() != P + 1)
    reject(OMVGBA_INVALID_PROBLEM, "fixed-rotation BA dimensions are inconsistent");
  bool finite = true;
  for (const ProbeCamera& c : p.cameras) {
    for (double v : c.R) finite = finite && std::isfinite(v);
    for (double v : c.C) finite = finite && std::isfinite(v);
    for (double v : c.intrinsics) finite = finite && std::isfinite(v);
  }
  for (double v : p.points) finite = finite && std::isfinite(v);
  for (double v : p.obs_px) finite = finite && std::isfinite(v);
  if (!finite) reject(OMVGBA_INVALID_PROBLEM, "fixed-rotation BA inputs must be finite");
  for (size_t k = 0; k < P; ++k) {
    if (p.track_off[k + 1] < p.track_off[k] + 2)
      reject(OMVGBA_INVALID_PROBLEM, "fixed-rotation BA requires valid two-view point tracks");
    for (uint64_t o2 = p.track_off[k]; o2 < p.track_off[k + 1]; ++o2)
      if (p.obs_cam[o2] >= n) reject(OMVGBA_INVALID_PROBLEM, "fixed-rotation BA requires valid two-view point tracks");
  }
  if (p.anchor == p.scale_camera || p.anchor >= n || p.scale_camera >= n)
    reject(OMVGBA_INVALID_PROBLEM, "fixed-rotation gauge endpoints are invalid");
  if (p.fixed_baseline && !(std::isfinite(p.distance) && p.distance > 0.0))
    reject(OMVGBA_INVALID_PROBLEM, "fixed baseline must be positive and finite");
  const double e = o.minimum_normalized_eigenvalue;
  if (o.max_tracks == 0 || o.max_observations < 2 || o.max_observations_per_track < 2 ||
      o.max_coverage_observations_per_track < o.max_observations_per_track || o.max_reduced_nonzeros == 0 ||
      o.max_factor_nonzeros == 0 || o.max_symbolic_dense_nonzeros == 0 || !(std::isfinite(e) && e > 0.0 && e < 1.0))
    reject(OMVGBA_INVALID_ARGUMENT, "invalid fixed-rotation observability probe limits");
}

// linearize (observability.rs:528-568): the whitened point Jacobian d pixel / d X of one observation,
// false when the camera cannot project the point (the track is then weak).
bool whitened_jacobian(const ProbeCamera& c, const double* X, double ox, double oy, const LossDev& loss,
                       double J[2][3]) {
  const double d[3] = {X[0] - c.C[0], X[1] - c.C[1], X[2] - c.C[2]};
  const double q[3] = {c.R[0] * d[0] + c.R[1] * d[1] + c.R[2] * d[2], c.R[3] * d[0] + c.R[4] * d[1] + c.R[5] * d[2],
                       c.R[6] * d[0] + c.R[7] * d[1] + c.R[8] * d[2]};
  if (!finite3(q[0], q[1], q[2]) || q[2] <= 0.0) return false;
  const double* k = c.intrinsics;
  if (!(k[0] > 0.0 && k[1] > 0.0 && std::isfinite(k[0]) && std::isfinite(k[1]))) return false;
  FixedCameraDev cam{};
  cam.fx = k[0];
  cam.fy = k[1];
  cam.cx = k[2];
  cam.cy = k[3];
  cam.k1 = k[4];
  cam.k2 = k[5];
  cam.k3 = k[6];
  cam.p1 = k[7];
  cam.p2 = k[8];
  cam.radial_kind = 3;
  cam.tangential_kind = 2;
  double t = 0.0;
  cam.has_turn = first_radial_turn_squared(cam.k1, cam.k2, &t) ? 1 : 0;
  cam.turn_squared = cam.has_turn ? t : INFINITY;
  double r[2], P[2][3];
  if (!cam.linearize(q[0], q[1], q[2], ox, oy, r, P)) return false;
  const double rn = std::sqrt(r[0] * r[0] + r[1] * r[1]);
  const double rel = loss.sqrt_weight(rn) / loss.sqrt_weight(0.0);  // relative_sqrt_weight (refine/api.rs:390)
  const double s = std::sqrt(rel * rel);
  for (int a = 0; a < 2; ++a)
    for (int j = 0; j < 3; ++j) J[a][j] = s * (P[a][0] * c.R[j] + P[a][1] * c.R[3 + j] + P[a][2] * c.R[6 + j]);
  return true;
}

struct Eliminated {
  bool weak = true;
  std::vector<uint32_t> cams;
  std::vector<double> J;      // 6 per observation (row-major 2 x 3)
  std::vector<double> blocks;  // 3L x 3L, row-major
};

// rank_point_schur (observability.rs:461-495) for one track.
void eliminate(const ProbeProblem& p, size_t point, Eliminated& out) {
  const uint64_t b = p.track_off[point], e = p.track_off[point + 1];
  const size_t L = (size_t)(e - b), rows = 2 * L, cols = 3 * L;
  out.weak = true;
  out.cams.resize(L);
  out.J.resize(6 * L);
  for (size_t a = 0; a < L; ++a) {
    double J[2][3];
    const uint32_t cam = p.obs_cam[b + a];
    if (!whitened_jacobian(p.cameras[cam], &p.points[3 * point], p.obs_px[2 * (b + a)], p.obs_px[2 * (b + a) + 1],
                           p.loss, J))
      return;
    out.cams[a] = cam;
    for (int r = 0; r < 2; ++r)
      for (int j = 0; j < 3; ++j) out.J[6 * a + 3 * r + j] = J[r][j];
  }
  // the point block sum J_a^T J_a and its weak test (observability.rs:449-455)
  double H[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (size_t a = 0; a < L; ++a) {
    const double* j = &out.J[6 * a];
    for (int u = 0; u < 3; ++u)
      for (int v = 0; v < 3; ++v) H[u][v] += j[u] * j[v] + j[3 + u] * j[3 + v];
  }
  const double V[6] = {H[0][0], H[1][0], H[1][1], H[2][0], H[2][1], H[2][2]};
  double damped[6], inv[6];
  const double rc = point_factor(V, 0.0, damped, inv) ? point_rcond(V, inv) : 0.0;
  const double det = H[0][0] * (H[1][1] * H[2][2] - H[1][2] * H[2][1]) - H[0][1] * (H[1][0] * H[2][2] - H[1][2] * H[2][0]) +
                     H[0][2] * (H[1][0] * H[2][1] - H[1][1] * H[2][0]);
  if (rc <= 64.0 * kEps * 3.0 || det == 0.0) return;
  // Householder thin QR of the stacked rows x 3 Jacobian; Q Q^T does not depend on the reflectors'
  // signs, so the blocks are those of any orthonormal basis of the column space, to rounding
  std::vector<double> A(rows * 3), Vh(rows * 3, 0.0), Q(rows * 3, 0.0);
  double beta[3] = {0, 0, 0};
  for (size_t a = 0; a < L; ++a)
    for (int r = 0; r < 2; ++r)
      for (int j = 0; j < 3; ++j) A[(2 * a + r) * 3 + j] = out.J[6 * a + 3 * r + j];
  for (int k = 0; k < 3; ++k) {
    double s2 = 0.0;
    for (size_t i = k; i < rows; ++i) s2 += A[i * 3 + k] * A[i * 3 + k];
    const double nrm = std::sqrt(s2);
    if (nrm == 0.0) continue;
    const double alpha = A[k * 3 + k] > 0.0 ? -nrm : nrm;
    double vv = 0.0;
    for (size_t i = k; i < rows; ++i) {
      Vh[i * 3 + k] = A[i * 3 + k] - (i == (size_t)k ? alpha : 0.0);
      vv += Vh[i * 3 + k] * Vh[i * 3 + k];
    }
    if (vv == 0.0) continue;
    beta[k] = 2.0 / vv;
    for (int c = k; c < 3; ++c) {
      double s = 0.0;
      for (size_t i = k; i < rows; ++i) s += Vh[i * 3 + k] * A[i * 3 + c];
      s *= beta[k];
      for (size_t i = k; i < rows; ++i) A[i * 3 + c] -= s * Vh[i * 3 + k];
    }
  }
  for (int c = 0; c < 3; ++c) Q[c * 3 + c] = 1.0;
  for (int k = 2; k >= 0; --k) {
    if (beta[k] == 0.0) continue;
    for (int c = 0; c < 3; ++c) {
      double s = 0.0;
      for (size_t i = k; i < rows; ++i) s += Vh[i * 3 + k] * Q[i * 3 + c];
      s *= beta[k];
      for (size_t i = k; i < rows; ++i) Q[i * 3 + c] -= s * Vh[i * 3 + k];
    }
  }
  // Z = blockdiag(J) - Q (Q_a^T J_a)_a, then Z^T Z
  std::vector<double> Z(rows * cols, 0.0);
  for (size_t a = 0; a < L; ++a) {
    const double* j = &out.J[6 * a];
    double M[3][3];
    for (int i = 0; i < 3; ++i)
      for (int c = 0; c < 3; ++c) M[i][c] = Q[(2 * a) * 3 + i] * j[c] + Q[(2 * a + 1) * 3 + i] * j[3 + c];
    for (size_t r = 0; r < rows; ++r)
      for (int c = 0; c < 3; ++c)
        Z[r * cols + 3 * a + c] = -(Q[r * 3] * M[0][c] + Q[r * 3 + 1] * M[1][c] + Q[r * 3 + 2] * M[2][c]);
    for (int r = 0; r < 2; ++r)
      for (int c = 0; c < 3; ++c) Z[(2 * a + r) * cols + 3 * a + c] += j[3 * r + c];
  }
  out.blocks.assign(cols * cols, 0.0);
  for (size_t u = 0; u < cols; ++u)
    for (size_t v = u; v < cols; ++v) {
      double s = 0.0;
      for (size_t r = 0; r < rows; ++r) s += Z[r * cols + u] * Z[r * cols + v];
      out.blocks[u * cols + v] = s;
      out.blocks[v * cols + u] = s;
    }
  out.weak = false;
}

// select_probe_tracks (observability.rs:294-389)
std::vector<size_t> select_tracks(const ProbeProblem& p, const std::vector<uint8_t>& free_cam,
                                  const omvgba_probe_options& o) {
  const size_t P = p.points.size() / 3;
  auto len = [&](size_t k) { return (size_t)(p.track_off[k + 1] - p.track_off[k]); };
  std::vector<std::pair<size_t, size_t>> cand;
  for (size_t k = 0; k < P; ++k) {
    bool sees_free = false;
    for (uint64_t q = p.track_off[k]; q < p.track_off[k + 1] && !sees_free; ++q) sees_free = free_cam[p.obs_cam[q]];
    if (len(k) <= o.max_coverage_observations_per_track && sees_free) cand.push_back({len(k), k});
  }
  std::sort(cand.begin(), cand.end());
  std::vector<uint8_t> chosen(P, 0), covered(free_cam.size(), 0);
  size_t tracks = 0, observations = 0;
  auto adds_coverage = [&](size_t k) {
    for (uint64_t q = p.track_off[k]; q < p.track_off[k + 1]; ++q)
      if (free_cam[p.obs_cam[q]] && !covered[p.obs_cam[q]]) return true;
    return false;
  };
  auto fits = [&](size_t k) { return tracks != o.max_tracks && observations + len(k) <= o.max_observations; };
  auto take = [&](size_t k, bool cover) {
    chosen[k] = 1;
    tracks++;
    observations += len(k);
    if (cover)
      for (uint64_t q = p.track_off[k]; q < p.track_off[k + 1]; ++q)
        if (free_cam[p.obs_cam[q]]) covered[p.obs_cam[q]] = 1;
  };
  auto all_covered = [&]() {
    for (size_t c = 0; c < free_cam.size(); ++c)
      if (free_cam[c] && !covered[c]) return false;
    return true;
  };
  for (const auto& c : cand)  // short tracks that add coverage
    if (len(c.second) <= o.max_observations_per_track && adds_coverage(c.second) && fits(c.second)) take(c.second, true);
  if (!all_covered())  // bounded long tracks that add coverage
    for (const auto& c : cand)
      if (len(c.second) > o.max_observations_per_track && !chosen[c.second] && adds_coverage(c.second) &&
          fits(c.second))
        take(c.second, true);
  if (all_covered())  // fill the caps with the remaining short tracks
    for (const auto& c : cand)
      if (!chosen[c.second] && len(c.second) <= o.max_observations_per_track && fits(c.second)) take(c.second, false);
  std::vector<size_t> out;
  for (size_t k = 0; k < P; ++k)
    if (chosen[k]) out.push_back(k);
  return out;
}

}  // namespace

omvgba_probe_report probe_fixed_rotation(Context* ctx, const ProbeProblem& p, const omvgba_probe_options& o) {
  validate(p, o);
  const size_t ncam = p.cameras.size();
  omvgba_probe_report rep{};
  rep.status = OMVGBA_PROBE_INSUFFICIENT_CAMERA_COVERAGE;
  // gauge_constraints (observability.rs:503-526): the anchor fixed, and the largest baseline
  // coordinate of the scale camera (the last of equal maxima)
  std::vector<uint8_t> fixed(3 * ncam);
  for (size_t c = 0; c < ncam; ++c)
    for (int k = 0; k < 3; ++k) fixed[3 * c + k] = p.cameras[c].fixed ? 1 : 0;
  for (int k = 0; k < 3; ++k) fixed[3 * p.anchor + k] = 1;
  const uint64_t s = p.scale_camera;
  if (!(fixed[3 * s] && fixed[3 * s + 1] && fixed[3 * s + 2])) {
    double m[3];
    for (int k = 0; k < 3; ++k) m[k] = std::fabs(p.cameras[s].C[k] - p.cameras[p.anchor].C[k]);
    int best = 0;
    for (int k = 1; k < 3; ++k)
      if (m[k] >= m[best]) best = k;
    if (!(std::isfinite(m[best]) && m[best] > 0.0))
      reject(OMVGBA_INVALID_PROBLEM, "fixed-rotation BA cannot fix scale from coincident camera centers");
    fixed[3 * s + best] = 1;
  }
  // free_coordinate_map (observability.rs:264-282): free coordinates in camera order
  std::vector<int> coord(3 * ncam, -1);
  int dim = 0;
  for (size_t q = 0; q < 3 * ncam; ++q)
    if (!fixed[q]) coord[q] = dim++;
  rep.pose_dimension = (uint64_t)dim;
  if (dim == 0) {
    rep.status = OMVGBA_PROBE_FULL_RANK_CERTIFIED;
    return rep;
  }
  std::vector<uint8_t> free_cam(ncam, 0);
  size_t required = 0;
  for (size_t c = 0; c < ncam; ++c) {
    free_cam[c] = !(fixed[3 * c] && fixed[3 * c + 1] && fixed[3 * c + 2]);
    required += free_cam[c];
  }
  const std::vector<size_t> sel = select_tracks(p, free_cam, o);
  uint64_t sel_obs = 0;
  for (size_t k : sel) sel_obs += p.track_off[k + 1] - p.track_off[k];
  rep.selected_tracks = sel.size();
  rep.selected_observations = sel_obs;
  if (sel.size() > o.max_tracks || sel_obs > o.max_observations || (uint64_t)dim > o.max_reduced_nonzeros) {
    rep.status = OMVGBA_PROBE_RESOURCE_LIMIT;
    return rep;
  }
  // eliminate every selected point on host threads (fixed chunks), then merge in selection order
  std::vector<Eliminated> elim(sel.size());
  {
    const size_t workers = std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(), 32));
    const size_t chunk = (sel.size() + workers - 1) / std::max<size_t>(workers, 1);
    std::vector<std::thread> pool;
    for (size_t w = 0; w < workers && w * chunk < sel.size(); ++w)
      pool.emplace_back([&, w]() {
        for (size_t i = w * chunk; i < std::min(sel.size(), (w + 1) * chunk); ++i) eliminate(p, sel[i], elim[i]);
      });
    for (auto& t : pool) t.join();
  }
  std::unordered_map<uint64_t, double> entries;  // key: column * dim + row, row >= column
  entries.reserve(std::min<uint64_t>(o.max_reduced_nonzeros, (uint64_t)dim * 64));
  for (int d = 0; d < dim; ++d) entries[(uint64_t)d * dim + d] = 0.0;
  std::vector<uint8_t> covered(ncam, 0);
  std::vector<double> raw(dim, 0.0);
  for (const Eliminated& t : elim) {
    if (t.weak) {
      rep.weak_point_count++;
      continue;
    }
    const size_t L = t.cams.size(), cols = 3 * L;
    for (uint32_t c : t.cams)
      if (free_cam[c]) covered[c] = 1;
    size_t free_scalars = 0;
    for (size_t a = 0; a < L; ++a)
      for (int l = 0; l < 3; ++l) {
        const int q = coord[3 * t.cams[a] + l];
        if (q < 0) continue;
        raw[q] += t.J[6 * a + l] * t.J[6 * a + l] + t.J[6 * a + 3 + l] * t.J[6 * a + 3 + l];
        free_scalars++;
      }
    if (entries.size() + free_scalars * (free_scalars + 1) / 2 > o.max_reduced_nonzeros) {
      rep.status = OMVGBA_PROBE_RESOURCE_LIMIT;
      for (size_t c = 0; c < ncam; ++c) rep.covered_free_cameras += covered[c];
      rep.reduced_nonzeros = entries.size();
      return rep;
    }
    for (size_t a = 0; a < L; ++a)  // add_sparse_free_block (observability.rs:391-411)
      for (size_t b = 0; b < L; ++b)
        for (int la = 0; la < 3; ++la) {
          const int row = coord[3 * t.cams[a] + la];
          if (row < 0) continue;
          for (int lb = 0; lb < 3; ++lb) {
            const int col = coord[3 * t.cams[b] + lb];
            if (col < 0 || row < col) continue;
            entries[(uint64_t)col * dim + row] += t.blocks[(3 * a + la) * cols + 3 * b + lb];
          }
        }
  }
  for (size_t c = 0; c < ncam; ++c) rep.covered_free_cameras += covered[c];
  rep.reduced_nonzeros = entries.size();
  if (rep.covered_free_cameras != required) {
    rep.status = OMVGBA_PROBE_INSUFFICIENT_CAMERA_COVERAGE;
    return rep;
  }
  if (rep.weak_point_count == rep.selected_tracks) {
    rep.status = OMVGBA_PROBE_WEAK_POINT_GEOMETRY;
    return rep;
  }
  // every free coordinate keeps a fraction of its information; equilibrate and shift
  std::vector<double> diag(dim);
  for (int d = 0; d < dim; ++d) diag[d] = entries[(uint64_t)d * dim + d];
  for (int d = 0; d < dim; ++d)
    if (!(std::isfinite(diag[d]) && diag[d] > kMinPositive) || diag[d] <= o.minimum_normalized_eigenvalue * raw[d]) {
      rep.status = OMVGBA_PROBE_WEAK_POINT_GEOMETRY;
      return rep;
    }
  std::vector<int> rows, cols;
  std::vector<double> vals;
  rows.reserve(entries.size());
  cols.reserve(entries.size());
  vals.reserve(entries.size());
  std::vector<int> first(dim);
  for (int d = 0; d < dim; ++d) first[d] = d;
  for (const auto& e : entries) {
    const int col = (int)(e.first / (uint64_t)dim), row = (int)(e.first % (uint64_t)dim);
    double v = e.second / std::sqrt(diag[row] * diag[col]);
    if (row == col) v -= o.minimum_normalized_eigenvalue;
    if (!std::isfinite(v)) {
      rep.status = OMVGBA_PROBE_WEAK_POINT_GEOMETRY;
      return rep;
    }
    rows.push_back(row);
    cols.push_back(col);
    vals.push_back(v);
    first[row] = std::min(first[row], col);
  }
  if ((uint64_t)dim * (uint64_t)(dim + 1) / 2 > o.max_symbolic_dense_nonzeros) {
    rep.status = OMVGBA_PROBE_RESOURCE_LIMIT;
    return rep;
  }
  uint64_t profile = 0;  // the factor's entries within each row's profile, in coordinate order
  for (int d = 0; d < dim; ++d) profile += (uint64_t)(d - first[d] + 1);
  rep.factor_nonzeros = profile;
  if (profile > o.max_factor_nonzeros) {
    rep.status = OMVGBA_PROBE_RESOURCE_LIMIT;
    return rep;
  }
  rep.status = device_certify_positive_definite(ctx, dim, rows, cols, vals) ? OMVGBA_PROBE_FULL_RANK_CERTIFIED
                                                                           : OMVGBA_PROBE_SPARSE_FACTORIZATION_FAILED;
  return rep;
}

}  // namespace omvgba
