// fixed_rotation_probe.hpp — TEST INFRASTRUCTURE ONLY (part of the CPU oracle): a restatement of the
// reference's bounded observability probe of translation-only problems, probe_fixed_rotation_
// observability (kernel/fixed_rotation/observability.rs:24-262, options and reasons in
// kernel/fixed_rotation/api.rs, validation in kernel/fixed_rotation/validation.rs).
//
// With the rotations and intrinsics held, the unknowns are the free camera centres and the points.
// A capped subset of tracks is selected (shortest first, covering every free camera), each point is
// eliminated in square-root form (the whitened Jacobians projected off the point's column space by a
// thin QR), the camera system is equilibrated to unit diagonal, shifted by the minimum normalized
// eigenvalue and factored: success certifies the whole problem, since omitted tracks only add
// positive semidefinite terms.
//
// Third-party arithmetic: the reference factors with faer's simplicial sparse Cholesky after an AMD
// ordering (numerics/sparse.rs). The factorization here is an envelope (skyline) Cholesky in the
// natural coordinate order; positive definiteness is decided the same way away from rounding-level
// pivots, and factor_nonzeros counts the envelope (the reference counts the AMD factor's entries), so
// the max_factor_nonzeros cap can differ at its boundary.
#pragma once

#include <map>
#include <utility>
#include <vector>

#include "oracle_core.hpp"

namespace oracle {

struct FrIntrinsics {
  double fx, fy, cx, cy, k1, k2, k3, p1, p2;
};
struct FrObservation {
  size_t camera;
  double x, y;
};
struct FrProblem {
  std::vector<Mat3> rotations;
  std::vector<Vec3> centers;
  std::vector<Vec3> points;
  std::vector<FrIntrinsics> intrinsics;
  std::vector<std::vector<FrObservation>> tracks;
  std::vector<uint8_t> fixed_cameras;
  bool fixed_baseline = false;
  size_t anchor = 0, scale_camera = 1;
  double distance = 0.0;
};
struct FrOptions {  // FixedRotationObservabilityProbeOptions::default (api.rs)
  size_t max_tracks = 25000, max_observations = 100000, max_observations_per_track = 32,
         max_coverage_observations_per_track = 256, max_reduced_nonzeros = 1000000, max_factor_nonzeros = 4000000,
         max_symbolic_dense_nonzeros = 32000000;
  double minimum_normalized_eigenvalue = 1e-10;
};
enum FrStatus { kFrCertified = 0, kFrCoverage = 1, kFrResource = 2, kFrWeak = 3, kFrFactorFailed = 4 };
struct FrReport {
  int status = kFrCoverage;
  size_t pose_dimension = 0, selected_tracks = 0, selected_observations = 0, covered_free_cameras = 0,
         weak_point_count = 0, reduced_nonzeros = 0, factor_nonzeros = 0;
};
struct FrError {
  int code;  // OMVGBA_INVALID_ARGUMENT (options) or OMVGBA_INVALID_PROBLEM
  std::string message;
};

// validate_probe_options (validation.rs:6-25)
inline void fr_validate_options(const FrOptions& o) {
  const double e = o.minimum_normalized_eigenvalue;
  if (o.max_tracks == 0 || o.max_observations < 2 || o.max_observations_per_track < 2 ||
      o.max_coverage_observations_per_track < o.max_observations_per_track || o.max_reduced_nonzeros == 0 ||
      o.max_factor_nonzeros == 0 || o.max_symbolic_dense_nonzeros == 0 || !(std::isfinite(e) && e > 0.0 && e < 1.0))
    throw FrError{OMVGBA_INVALID_ARGUMENT, "invalid fixed-rotation observability probe limits"};
}

// validate_problem (validation.rs:27-117)
inline void fr_validate_problem(const FrProblem& p) {
  const size_t n = p.centers.size();
  if (p.rotations.size() < 2 || p.rotations.size() != n || p.intrinsics.size() != n || p.fixed_cameras.size() != n ||
      p.points.empty() || p.points.size() != p.tracks.size())
    throw FrError{OMVGBA_INVALID_PROBLEM, "fixed-rotation BA dimensions are inconsistent"};
  bool finite = true;
  for (const Mat3& R : p.rotations)
    for (const auto& row : R) finite = finite && all_finite(row.data(), 3);
  for (const Vec3& c : p.centers) finite = finite && all_finite(c.data(), 3);
  for (const Vec3& x : p.points) finite = finite && all_finite(x.data(), 3);
  for (const auto& t : p.tracks)
    for (const auto& o : t) finite = finite && std::isfinite(o.x) && std::isfinite(o.y);
  for (const auto& k : p.intrinsics) {
    const double v[9] = {k.fx, k.fy, k.cx, k.cy, k.k1, k.k2, k.k3, k.p1, k.p2};
    finite = finite && all_finite(v, 9);
  }
  if (!finite) throw FrError{OMVGBA_INVALID_PROBLEM, "fixed-rotation BA inputs must be finite"};
  for (const auto& t : p.tracks) {
    if (t.size() < 2) throw FrError{OMVGBA_INVALID_PROBLEM, "fixed-rotation BA requires valid two-view point tracks"};
    for (const auto& o : t)
      if (o.camera >= n) throw FrError{OMVGBA_INVALID_PROBLEM, "fixed-rotation BA requires valid two-view point tracks"};
  }
  if (p.anchor == p.scale_camera || p.anchor >= n || p.scale_camera >= n)
    throw FrError{OMVGBA_INVALID_PROBLEM, "fixed-rotation gauge endpoints are invalid"};
  if (p.fixed_baseline && !(std::isfinite(p.distance) && p.distance > 0.0))
    throw FrError{OMVGBA_INVALID_PROBLEM, "fixed baseline must be positive and finite"};
}

// linearize (observability.rs:528-568): the whitened 2 x 3 point Jacobian of one observation, or
// nothing when the camera cannot project the point.
inline bool fr_linearize(const Mat3& R, const Vec3& C, const Vec3& X, const FrIntrinsics& k, double ox, double oy,
                         const Loss& loss, Mat23* out) {
  const Vec3 d = {X[0] - C[0], X[1] - C[1], X[2] - C[2]};
  const Vec3 q = rotate(R, d);
  if (!all_finite(q.data(), 3) || q[2] <= 0.0) return false;
  // PinholeCamera::try_new (pinhole.rs:195-240) and BrownConradyCamera::try_new (brown_conrady.rs:148-166)
  if (!(k.fx > 0.0 && k.fy > 0.0 && std::isfinite(k.fx) && std::isfinite(k.fy) && std::isfinite(k.cx) &&
        std::isfinite(k.cy)))
    return false;
  BrownConrady cam;
  cam.fx = k.fx;
  cam.fy = k.fy;
  cam.cx = k.cx;
  cam.cy = k.cy;
  cam.radial_kind = 3;
  cam.tangential_kind = 2;
  cam.k1 = k.k1;
  cam.k2 = k.k2;
  cam.k3 = k.k3;
  cam.p1 = k.p1;
  cam.p2 = k.p2;
  cam.turn_squared = first_radial_turn_squared(k.k1, k.k2);
  auto pr = cam.project_with_jacobian({ox, oy}, q);
  if (!pr) return false;
  const double rn = std::sqrt(pr->residual[0] * pr->residual[0] + pr->residual[1] * pr->residual[1]);
  const double rsw = loss.sqrt_weight(rn) / loss.sqrt_weight(0.0);  // relative_sqrt_weight (refine/api.rs:390)
  const double weight = rsw * rsw;
  const double s = std::sqrt(weight);
  for (int r = 0; r < 2; ++r)
    for (int c = 0; c < 3; ++c)
      (*out)[r][c] = s * (pr->jacobian[r][0] * R[0][c] + pr->jacobian[r][1] * R[1][c] + pr->jacobian[r][2] * R[2][c]);
  return true;
}

// rank_point_schur (observability.rs:461-495): Z^T Z with Z_a = (E_a - Q Q_a^T) J_a, Q the thin QR
// factor of the stacked Jacobians, or nothing when the point block is weak. Q Q^T is the projector
// onto the column space whatever the Householder sign convention, so any orthonormal basis gives the
// same blocks to rounding. Returns the 3L x 3L matrix row-major.
inline bool fr_point_schur(const std::vector<Mat23>& J, std::vector<double>* out) {
  const size_t L = J.size(), rows = 2 * L, cols = 3 * L;
  Mat3 H{};
  for (const Mat23& j : J)
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) H[a][b] += j[0][a] * j[0][b] + j[1][a] * j[1][b];
  // is_weak_point_block (observability.rs:449-455)
  auto f = point_block_factor(H, 0.0);
  const double rc = f ? point_rcond(*f, H) : 0.0;
  const double det = H[0][0] * (H[1][1] * H[2][2] - H[1][2] * H[2][1]) - H[0][1] * (H[1][0] * H[2][2] - H[1][2] * H[2][0]) +
                     H[0][2] * (H[1][0] * H[2][1] - H[1][1] * H[2][0]);
  if (rc <= kPointBlockRcondThreshold || det == 0.0) return false;
  // Householder QR of the stacked rows x 3 matrix A; Q = H1 H2 H3 applied to the first 3 columns of I
  std::vector<double> A(rows * 3), V(rows * 3, 0.0), beta(3, 0.0);
  for (size_t a = 0; a < L; ++a)
    for (int r = 0; r < 2; ++r)
      for (int c = 0; c < 3; ++c) A[(2 * a + r) * 3 + c] = J[a][r][c];
  for (int k = 0; k < 3 && (size_t)k < rows; ++k) {
    double nrm = 0.0;
    for (size_t i = k; i < rows; ++i) nrm += A[i * 3 + k] * A[i * 3 + k];
    nrm = std::sqrt(nrm);
    if (nrm == 0.0) continue;
    const double alpha = A[k * 3 + k] > 0.0 ? -nrm : nrm;
    for (size_t i = k; i < rows; ++i) V[i * 3 + k] = A[i * 3 + k];
    V[k * 3 + k] -= alpha;
    double vv = 0.0;
    for (size_t i = k; i < rows; ++i) vv += V[i * 3 + k] * V[i * 3 + k];
    if (vv == 0.0) continue;
    beta[k] = 2.0 / vv;
    for (int c = k; c < 3; ++c) {
      double s = 0.0;
      for (size_t i = k; i < rows; ++i) s += V[i * 3 + k] * A[i * 3 + c];
      s *= beta[k];
      for (size_t i = k; i < rows; ++i) A[i * 3 + c] -= s * V[i * 3 + k];
    }
  }
  std::vector<double> Q(rows * 3, 0.0);
  for (int c = 0; c < 3 && (size_t)c < rows; ++c) Q[c * 3 + c] = 1.0;
  for (int k = 2; k >= 0; --k) {
    if (beta[k] == 0.0) continue;
    for (int c = 0; c < 3; ++c) {
      double s = 0.0;
      for (size_t i = k; i < rows; ++i) s += V[i * 3 + k] * Q[i * 3 + c];
      s *= beta[k];
      for (size_t i = k; i < rows; ++i) Q[i * 3 + c] -= s * V[i * 3 + k];
    }
  }
  // Z (rows x cols)
  std::vector<double> Z(rows * cols, 0.0);
  for (size_t a = 0; a < L; ++a) {
    double M[3][3];  // Q_a^T J_a
    for (int i = 0; i < 3; ++i)
      for (int c = 0; c < 3; ++c) M[i][c] = Q[(2 * a) * 3 + i] * J[a][0][c] + Q[(2 * a + 1) * 3 + i] * J[a][1][c];
    for (size_t r = 0; r < rows; ++r)
      for (int c = 0; c < 3; ++c)
        Z[r * cols + 3 * a + c] = -(Q[r * 3 + 0] * M[0][c] + Q[r * 3 + 1] * M[1][c] + Q[r * 3 + 2] * M[2][c]);
    for (int r = 0; r < 2; ++r)
      for (int c = 0; c < 3; ++c) Z[(2 * a + r) * cols + 3 * a + c] += J[a][r][c];
  }
  out->assign(cols * cols, 0.0);
  for (size_t i = 0; i < cols; ++i)
    for (size_t j = 0; j < cols; ++j) {
      double s = 0.0;
      for (size_t r = 0; r < rows; ++r) s += Z[r * cols + i] * Z[r * cols + j];
      (*out)[i * cols + j] = s;
    }
  return true;
}

// select_probe_tracks (observability.rs:294-389)
inline std::vector<size_t> fr_select_tracks(const FrProblem& p, const std::vector<uint8_t>& free_cam,
                                            const FrOptions& o) {
  std::vector<std::pair<size_t, size_t>> cand;
  for (size_t k = 0; k < p.tracks.size(); ++k) {
    const auto& t = p.tracks[k];
    bool any = false;
    for (const auto& ob : t) any = any || free_cam[ob.camera];
    if (t.size() <= o.max_coverage_observations_per_track && any) cand.push_back({t.size(), k});
  }
  std::sort(cand.begin(), cand.end());
  std::vector<uint8_t> selected(p.tracks.size(), 0), covered(free_cam.size(), 0);
  size_t ntr = 0, nobs = 0;
  auto take = [&](size_t k) {
    selected[k] = 1;
    ntr++;
    nobs += p.tracks[k].size();
    for (const auto& ob : p.tracks[k])
      if (free_cam[ob.camera]) covered[ob.camera] = 1;
  };
  auto adds = [&](size_t k) {
    for (const auto& ob : p.tracks[k])
      if (free_cam[ob.camera] && !covered[ob.camera]) return true;
    return false;
  };
  auto uncovered = [&]() {
    for (size_t c = 0; c < free_cam.size(); ++c)
      if (free_cam[c] && !covered[c]) return true;
    return false;
  };
  for (const auto& e : cand) {
    const size_t k = e.second;
    if (p.tracks[k].size() > o.max_observations_per_track) continue;
    if (!adds(k) || ntr == o.max_tracks || nobs + p.tracks[k].size() > o.max_observations) continue;
    take(k);
  }
  if (uncovered())
    for (const auto& e : cand) {
      const size_t k = e.second;
      if (p.tracks[k].size() <= o.max_observations_per_track || selected[k]) continue;
      if (!adds(k) || ntr == o.max_tracks || nobs + p.tracks[k].size() > o.max_observations) continue;
      take(k);
    }
  if (!uncovered())
    for (const auto& e : cand) {
      const size_t k = e.second;
      if (selected[k] || p.tracks[k].size() > o.max_observations_per_track) continue;
      if (ntr == o.max_tracks || nobs + p.tracks[k].size() > o.max_observations) continue;
      selected[k] = 1;
      ntr++;
      nobs += p.tracks[k].size();
    }
  std::vector<size_t> out;
  for (size_t k = 0; k < selected.size(); ++k)
    if (selected[k]) out.push_back(k);
  return out;
}

// Envelope (skyline) Cholesky of the symmetric matrix whose lower triangle is `entries` ((column, row)
// keys, row >= column); true when it is positive definite. *nonzeros: the envelope size.
inline bool fr_envelope_cholesky(size_t n, const std::map<std::pair<size_t, size_t>, double>& entries,
                                 size_t max_nonzeros, size_t* nonzeros, bool* too_large) {
  std::vector<size_t> first(n);
  for (size_t i = 0; i < n; ++i) first[i] = i;
  for (const auto& e : entries) first[e.first.second] = std::min(first[e.first.second], e.first.first);
  std::vector<size_t> start(n + 1, 0);
  for (size_t i = 0; i < n; ++i) start[i + 1] = start[i] + (i - first[i] + 1);
  *nonzeros = start[n];
  *too_large = start[n] > max_nonzeros;
  if (*too_large) return false;
  std::vector<double> L(start[n], 0.0);
  for (const auto& e : entries) {
    const size_t c = e.first.first, r = e.first.second;
    L[start[r] + (c - first[r])] = e.second;
  }
  for (size_t i = 0; i < n; ++i) {
    double* Li = &L[start[i]];
    for (size_t j = first[i]; j < i; ++j) {
      const double* Lj = &L[start[j]];
      const size_t k0 = std::max(first[i], first[j]);
      double s = Li[j - first[i]];
      for (size_t k = k0; k < j; ++k) s -= Li[k - first[i]] * Lj[k - first[j]];
      Li[j - first[i]] = s / Lj[j - first[j]];
    }
    double d = Li[i - first[i]];
    for (size_t k = first[i]; k < i; ++k) d -= Li[k - first[i]] * Li[k - first[i]];
    if (!(d > 0.0) || !std::isfinite(d)) return false;
    Li[i - first[i]] = std::sqrt(d);
  }
  return true;
}

// probe_fixed_rotation_observability (observability.rs:24-262)
inline FrReport fr_probe(const FrProblem& p, const Loss& loss, const FrOptions& o) {
  fr_validate_problem(p);
  fr_validate_options(o);
  const size_t ncam = p.centers.size();
  // gauge_constraints (observability.rs:503-526): the anchor fully fixed, and the largest baseline
  // coordinate of the scale camera (the last of equal maxima)
  std::vector<std::array<bool, 3>> fixed(ncam);
  for (size_t c = 0; c < ncam; ++c) fixed[c] = {p.fixed_cameras[c] != 0, p.fixed_cameras[c] != 0, p.fixed_cameras[c] != 0};
  fixed[p.anchor] = {true, true, true};
  if (!(fixed[p.scale_camera][0] && fixed[p.scale_camera][1] && fixed[p.scale_camera][2])) {
    const Vec3& a = p.centers[p.anchor];
    const Vec3& s = p.centers[p.scale_camera];
    const double m[3] = {std::fabs(s[0] - a[0]), std::fabs(s[1] - a[1]), std::fabs(s[2] - a[2])};
    int best = 0;  // Iterator::max_by keeps the last of equal maxima
    for (int k = 1; k < 3; ++k)
      if (m[k] >= m[best]) best = k;
    if (!(std::isfinite(m[best]) && m[best] > 0.0))
      throw FrError{OMVGBA_INVALID_PROBLEM, "fixed-rotation BA cannot fix scale from coincident camera centers"};
    fixed[p.scale_camera][best] = true;
  }
  // free_coordinate_map (observability.rs:264-282)
  std::vector<long> coord(3 * ncam, -1);
  size_t dim = 0;
  for (size_t c = 0; c < ncam; ++c)
    for (int k = 0; k < 3; ++k)
      if (!fixed[c][k]) coord[3 * c + k] = (long)dim++;
  FrReport rep;
  rep.pose_dimension = dim;
  if (dim == 0) {
    rep.status = kFrCertified;
    return rep;
  }
  std::vector<uint8_t> free_cam(ncam, 0);
  size_t required = 0;
  for (size_t c = 0; c < ncam; ++c) {
    free_cam[c] = !(fixed[c][0] && fixed[c][1] && fixed[c][2]);
    required += free_cam[c];
  }
  const std::vector<size_t> sel = fr_select_tracks(p, free_cam, o);
  size_t sel_obs = 0;
  for (size_t k : sel) sel_obs += p.tracks[k].size();
  rep.selected_tracks = sel.size();
  rep.selected_observations = sel_obs;
  rep.status = kFrCoverage;
  if (sel.size() > o.max_tracks || sel_obs > o.max_observations || dim > o.max_reduced_nonzeros) {
    rep.status = kFrResource;
    return rep;
  }
  std::map<std::pair<size_t, size_t>, double> entries;
  for (size_t d = 0; d < dim; ++d) entries[{d, d}] = 0.0;
  std::vector<uint8_t> covered(ncam, 0);
  std::vector<double> raw(dim, 0.0);
  std::vector<double> schur;
  for (size_t k : sel) {
    const auto& track = p.tracks[k];
    std::vector<Mat23> J;
    std::vector<size_t> cams;
    bool weak = false;
    for (const auto& ob : track) {
      Mat23 j;
      if (!fr_linearize(p.rotations[ob.camera], p.centers[ob.camera], p.points[k], p.intrinsics[ob.camera], ob.x,
                        ob.y, loss, &j)) {
        weak = true;
        break;
      }
      J.push_back(j);
      cams.push_back(ob.camera);
    }
    if (weak || !fr_point_schur(J, &schur)) {
      rep.weak_point_count++;
      continue;
    }
    for (size_t c : cams)
      if (free_cam[c]) covered[c] = 1;
    for (size_t a = 0; a < cams.size(); ++a)
      for (int l = 0; l < 3; ++l) {
        const long q = coord[3 * cams[a] + l];
        if (q >= 0) raw[q] += J[a][0][l] * J[a][0][l] + J[a][1][l] * J[a][1][l];
      }
    size_t free_scalars = 0;
    for (size_t c : cams)
      for (int l = 0; l < 3; ++l) free_scalars += coord[3 * c + l] >= 0 ? 1 : 0;
    const size_t bound = free_scalars * (free_scalars + 1) / 2;
    if (entries.size() + bound > o.max_reduced_nonzeros) {
      rep.status = kFrResource;
      for (size_t c = 0; c < ncam; ++c) rep.covered_free_cameras += covered[c];
      rep.reduced_nonzeros = entries.size();
      return rep;
    }
    const size_t cols = 3 * cams.size();
    for (size_t a = 0; a < cams.size(); ++a)
      for (size_t b = 0; b < cams.size(); ++b)
        for (int la = 0; la < 3; ++la) {  // add_sparse_free_block (observability.rs:391-411)
          const long row = coord[3 * cams[a] + la];
          if (row < 0) continue;
          for (int lb = 0; lb < 3; ++lb) {
            const long col = coord[3 * cams[b] + lb];
            if (col < 0 || row < col) continue;
            entries[{(size_t)col, (size_t)row}] += schur[(3 * a + la) * cols + 3 * b + lb];
          }
        }
  }
  for (size_t c = 0; c < ncam; ++c) rep.covered_free_cameras += covered[c];
  rep.reduced_nonzeros = entries.size();
  if (rep.covered_free_cameras != required) {
    rep.status = kFrCoverage;
    return rep;
  }
  if (rep.weak_point_count == rep.selected_tracks) {
    rep.status = kFrWeak;
    return rep;
  }
  std::vector<double> diag(dim, 0.0);
  for (size_t d = 0; d < dim; ++d) diag[d] = entries[{d, d}];
  for (size_t d = 0; d < dim; ++d)
    if (!(std::isfinite(diag[d]) && diag[d] > kMinPositive) || diag[d] <= o.minimum_normalized_eigenvalue * raw[d]) {
      rep.status = kFrWeak;
      return rep;
    }
  for (auto& e : entries) {
    const size_t col = e.first.first, row = e.first.second;
    e.second /= std::sqrt(diag[row] * diag[col]);
    if (row == col) e.second -= o.minimum_normalized_eigenvalue;
    if (!std::isfinite(e.second)) {
      rep.status = kFrWeak;
      return rep;
    }
  }
  if (dim * (dim + 1) / 2 > o.max_symbolic_dense_nonzeros) {
    rep.status = kFrResource;
    return rep;
  }
  bool too_large = false;
  const bool pd = fr_envelope_cholesky(dim, entries, o.max_factor_nonzeros, &rep.factor_nonzeros, &too_large);
  if (too_large) {
    rep.status = kFrResource;
    return rep;
  }
  rep.status = pd ? kFrCertified : kFrFactorFailed;
  return rep;
}

}  // namespace oracle
