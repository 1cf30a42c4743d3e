// two_view.cuh — two-view bundle adjustment on the device (refine_ba_2view,
// crates/openmvg-ba/src/kernel/two_view/{optimizer,schur,residual}.rs).
//
// Two cameras: the first is the frame (identity), the second has 5 free coordinates (rotation and
// the S^2 direction of a translation whose length, the baseline, stays fixed); every point is seen
// once by each camera and moves in baseline units. Each LM iteration runs three kernels:
//   k_tv_linearize  one thread per point: both projections (pixel or angular), the point's local
//                   normal equations and its contribution to the 5 x 5 reduced camera system;
//   k_tv_reduce     one CTA: the fixed-order sums of those contributions (and the extrema);
//   k_tv_candidate  one thread per point: the damped point step for the camera step, the moved
//                   point and its robust cost at the candidate pose (the same local system the
//                   linearization stored, so the step equals the reference's re-linearized one).
// The 5 x 5 Cholesky solve, the Nielsen damping and the stop tests are scalar work on the host.
#pragma once

namespace omvgba {

struct TvDev {
  int P;
  int angular;
  double cam[2][4];         // pixel: fx, fy, cx, cy per view
  const double* obs;        // pixel: [view][point][2]
  const double* bearing;    // angular: [view][point][3]
};
struct TvPose {
  double R[9], t[3];
};
constexpr int kTvSums = 43;   // H (25), g (5), full gradient (5), pose diagonal (5), cost, sq, point reduction
constexpr int kTvLocal = 24;  // per point: V (6, packed 00 10 11 20 21 22), Hpx (15), g_x (3)
constexpr int kTvOut = kTvSums + 5;  // + max scaled point gradient, min rcond, weak, invalid, failed

__device__ __forceinline__ bool tv_project(const TvDev& d, int view, int i, const double X[3], double r[2],
                                           double J[2][3]) {
  if (d.angular) return angular_linearize(d.bearing + 3 * ((size_t)view * d.P + i), X, r, J);
  FixedCameraDev c{};
  c.fx = d.cam[view][0];
  c.fy = d.cam[view][1];
  c.cx = d.cam[view][2];
  c.cy = d.cam[view][3];
  const double* o = d.obs + 2 * ((size_t)view * d.P + i);
  return pixel_linearize(c, X[0], X[1], X[2], o[0], o[1], r, J);
}

// scaled_gradient_inf_norm (schur.rs:414-430)
__device__ __forceinline__ double tv_scaled_ginf(const double* g, const double* diag, int n) {
  double scale = 0.0;
  for (int i = 0; i < n; ++i) scale = fmax(scale, diag[i]);
  if (!(isfinite(scale) && scale > 0.0)) {
    for (int i = 0; i < n; ++i)
      if (g[i] != 0.0) return INFINITY;
    return 0.0;
  }
  const double floor = 64.0 * kEps * scale;
  double best = 0.0;
  for (int i = 0; i < n; ++i) best = fmax(best, fabs(g[i]) / sqrt(fmax(diag[i], floor)));
  return best;
}

// linearize_point + ReducedSystem::add (schur.rs:101-140, 223-271) for one point.
__global__ void __launch_bounds__(128) k_tv_linearize(TvDev d, const double* __restrict__ points, TvPose pose,
                                                      double b0x, double b0y, double b0z, double b1x, double b1y,
                                                      double b1z, double baseline, LossDev loss, double lambda,
                                                      double* __restrict__ out, double* __restrict__ local) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.P) return;
  double* o = out + (size_t)kTvOut * i;
  for (int k = 0; k < kTvOut; ++k) o[k] = 0.0;
  o[kTvSums + 1] = 1.0;  // min rcond
  const double X[3] = {points[3 * (size_t)i], points[3 * (size_t)i + 1], points[3 * (size_t)i + 2]};
  double Hpp[5][5] = {}, Hpx[5][3] = {}, Hxx[3][3] = {}, gp[5] = {}, gx[3] = {}, cost = 0.0, sq = 0.0;
  auto accumulate = [&](const double r[2], const double Jp[2][5], const double Jx[2][3], double sw) {
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
  };
  double r[2], J[2][3];
  if (!tv_project(d, 0, i, X, r, J)) {
    o[kTvSums + 4] = 1.0;
    return;
  }
  double n1 = sqrt(r[0] * r[0] + r[1] * r[1]);
  cost += loss.cost(n1);
  sq += n1 * n1;
  {
    const double Jp[2][5] = {};
    double Jx[2][3];
    for (int a = 0; a < 2; ++a)
      for (int c = 0; c < 3; ++c) Jx[a][c] = J[a][c] * baseline;
    accumulate(r, Jp, Jx, loss.sqrt_weight(n1));
  }
  const double rot[3] = {pose.R[0] * X[0] + pose.R[1] * X[1] + pose.R[2] * X[2],
                         pose.R[3] * X[0] + pose.R[4] * X[1] + pose.R[5] * X[2],
                         pose.R[6] * X[0] + pose.R[7] * X[1] + pose.R[8] * X[2]};
  const double xc[3] = {rot[0] + pose.t[0], rot[1] + pose.t[1], rot[2] + pose.t[2]};
  if (!tv_project(d, 1, i, xc, r, J)) {
    o[kTvSums + 4] = 1.0;
    return;
  }
  const double n2 = sqrt(r[0] * r[0] + r[1] * r[1]);
  cost += loss.cost(n2);
  sq += n2 * n2;
  {
    double Jx[2][3], Jp[2][5];
    for (int a = 0; a < 2; ++a)
      for (int c = 0; c < 3; ++c)
        Jx[a][c] = (J[a][0] * pose.R[c] + J[a][1] * pose.R[3 + c] + J[a][2] * pose.R[6 + c]) * baseline;
    const double m[3][5] = {{0.0, rot[2], -rot[1], baseline * b0x, baseline * b1x},
                            {-rot[2], 0.0, rot[0], baseline * b0y, baseline * b1y},
                            {rot[1], -rot[0], 0.0, baseline * b0z, baseline * b1z}};
    for (int a = 0; a < 2; ++a)
      for (int c = 0; c < 5; ++c) Jp[a][c] = J[a][0] * m[0][c] + J[a][1] * m[1][c] + J[a][2] * m[2][c];
    accumulate(r, Jp, Jx, loss.sqrt_weight(n2));
  }
  // the stored local system (for the candidate)
  double* l = local + (size_t)kTvLocal * i;
  const double V[6] = {Hxx[0][0], Hxx[1][0], Hxx[1][1], Hxx[2][0], Hxx[2][1], Hxx[2][2]};
  for (int k = 0; k < 6; ++k) l[k] = V[k];
  for (int a = 0; a < 5; ++a)
    for (int c = 0; c < 3; ++c) l[6 + 3 * a + c] = Hpx[a][c];
  for (int c = 0; c < 3; ++c) l[21 + c] = gx[c];
  // ReducedSystem::add
  double* H = o;
  double* g = o + 25;
  double* fg = o + 30;
  double* dg = o + 35;
  o[40] = cost;
  o[41] = sq;
  for (int a = 0; a < 5; ++a) {
    fg[a] = gp[a];
    dg[a] = Hpp[a][a];
  }
  const double dx[3] = {Hxx[0][0], Hxx[1][1], Hxx[2][2]};
  o[kTvSums] = tv_scaled_ginf(gx, dx, 3);
  double damped[6], inv[6];
  if (!point_factor(V, lambda, damped, inv)) {
    o[kTvSums + 3] = 1.0;
    if (lambda == 0.0) {
      o[kTvSums + 2] = 1.0;
      o[kTvSums + 1] = 0.0;
    }
    return;
  }
  if (lambda == 0.0) {
    const double rc = point_rcond(V, inv);
    o[kTvSums + 1] = rc;
    o[kTvSums + 2] = rc <= 64.0 * kEps * 3.0 ? 1.0 : 0.0;
  }
  double ig[3];
  sym3_apply(inv, gx, ig);
  o[42] = 0.5 * (gx[0] * ig[0] + gx[1] * ig[1] + gx[2] * ig[2]);
  double ic[5][3];
  for (int a = 0; a < 5; ++a) sym3_apply(inv, Hpx[a], ic[a]);
  for (int a = 0; a < 5; ++a) {
    g[a] = gp[a] - (Hpx[a][0] * ig[0] + Hpx[a][1] * ig[1] + Hpx[a][2] * ig[2]);
    for (int c = 0; c < 5; ++c)
      H[5 * a + c] = Hpp[a][c] - (Hpx[a][0] * ic[c][0] + Hpx[a][1] * ic[c][1] + Hpx[a][2] * ic[c][2]);
  }
}

// point_step_with_damping_norm (schur.rs:278-301) and the candidate cost (optimizer.rs:270-305):
// out per point: cost at the candidate pose, |step|^2, damping norm, failure flag.
__global__ void __launch_bounds__(128) k_tv_candidate(TvDev d, const double* __restrict__ points,
                                                      const double* __restrict__ local, double lambda,
                                                      const double* __restrict__ step, TvPose cand, double baseline,
                                                      LossDev loss, double* __restrict__ moved,
                                                      double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.P) return;
  double* o = out + 4 * (size_t)i;
  o[0] = o[1] = o[2] = 0.0;
  o[3] = 1.0;
  const double* l = local + (size_t)kTvLocal * i;
  const double V[6] = {l[0], l[1], l[2], l[3], l[4], l[5]};
  double damped[6], inv[6];
  if (!point_factor(V, lambda, damped, inv)) return;
  double rhs[3];
  for (int c = 0; c < 3; ++c) {
    double s = 0.0;
    for (int p = 0; p < 5; ++p) s += l[6 + 3 * p + c] * step[p];
    rhs[c] = l[21 + c] + s;
  }
  double x[3];
  sym3_apply(inv, rhs, x);
  const double dx[3] = {-x[0], -x[1], -x[2]};
  double dd[3];
  if (!point_damping_diagonal(V, dd)) return;
  const double dn = dd[0] * dx[0] * dx[0] + dd[1] * dx[1] * dx[1] + dd[2] * dx[2] * dx[2];
  const double X[3] = {points[3 * (size_t)i] + baseline * dx[0], points[3 * (size_t)i + 1] + baseline * dx[1],
                       points[3 * (size_t)i + 2] + baseline * dx[2]};
  for (int k = 0; k < 3; ++k) moved[3 * (size_t)i + k] = X[k];
  double r[2], J[2][3];
  if (!tv_project(d, 0, i, X, r, J)) return;
  double c0 = loss.cost(sqrt(r[0] * r[0] + r[1] * r[1]));
  const double xc[3] = {cand.R[0] * X[0] + cand.R[1] * X[1] + cand.R[2] * X[2] + cand.t[0],
                        cand.R[3] * X[0] + cand.R[4] * X[1] + cand.R[5] * X[2] + cand.t[1],
                        cand.R[6] * X[0] + cand.R[7] * X[1] + cand.R[8] * X[2] + cand.t[2]};
  if (!tv_project(d, 1, i, xc, r, J)) return;
  o[0] = c0 + loss.cost(sqrt(r[0] * r[0] + r[1] * r[1]));
  o[1] = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
  o[2] = dn;
  o[3] = 0.0;
}

// Fixed-order sums of per-point rows of `width` values over P points, one CTA: thread t takes points
// t, t + blockDim, ... in order, then a fixed shuffle tree and the warps in order. Columns in
// [sums, width) reduce by max (the first extra column), min (the second) and sum (the rest).
__global__ void __launch_bounds__(1024) k_tv_reduce(const double* __restrict__ in, int P, int width, int sums,
                                                    double* __restrict__ out) {
  __shared__ double part[32][kTvOut];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int c = 0; c < width; ++c) {
    const bool is_max = c == sums, is_min = c == sums + 1;
    double acc = is_max ? 0.0 : (is_min ? 1.0 : 0.0);
    for (int i = tid; i < P; i += blockDim.x) {
      const double v = in[(size_t)width * i + c];
      acc = is_max ? fmax(acc, v) : (is_min ? fmin(acc, v) : acc + v);
    }
    for (int off = 16; off > 0; off >>= 1) {
      const double w = __shfl_down_sync(0xffffffffu, acc, off);
      acc = is_max ? fmax(acc, w) : (is_min ? fmin(acc, w) : acc + w);
    }
    if (lane == 0) part[warp][c] = acc;
  }
  __syncthreads();
  if (tid < width) {
    const int c = tid;
    const bool is_max = c == sums, is_min = c == sums + 1;
    double acc = part[0][c];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
      acc = is_max ? fmax(acc, part[w][c]) : (is_min ? fmin(acc, part[w][c]) : acc + part[w][c]);
    out[c] = acc;
  }
}

}  // namespace omvgba
