// residual.cu — reprojection residual of the centred radial camera model over an unsorted
// observation list, and its hand-written vector-Jacobian product (adjoint).
//
// Model (crates/openmvg-ba/src/kernel/multi_view/self_calibration/model.rs:26-129): camera j has
// R_j = exp(rotvec_j), translation t_j and intrinsics (f, k1, k2); for observation i of camera j
// and point p, X_c = R_j X_p + t_j, n = (X_c.x / X_c.z, X_c.y / X_c.z), r^2 = |n|^2 and
//   residual_i = f (1 + k1 r^2 + k2 r^4) n - pixel_i            (pixels centred at the principal point)
// An observation is admissible when X_c.z > 64 eps max|X_c|, r^2 is inside the first radial turn
// (the first positive root of 1 + 3 k1 r^2 + 5 k2 r^4) and the distortion map has det > 1e-12
// (model.rs:26-75, 143-172); otherwise its residual is NaN and it adds nothing to the gradients.
//
// Adjoint of one observation with upstream gradient g (2 values) and J = d residual / d X_c:
//   a = J^T g;  d/dt += a;  d/dX_p += R^T a;  d/drotvec += Jl(rotvec)^T (R X_p x a)
//   d/df += (Jint[:,0] . g) / f;  d/dk1 += Jint[:,1] . g;  d/dk2 += Jint[:,2] . g
// where Jl is the left Jacobian of SO(3) (d exp(w) X / dw = -[exp(w) X]x Jl(w)) and Jint holds the
// model's intrinsic columns (log f, k1, k2) (model.rs:298-315).
//
// Determinism: observations arrive in any order, so gradients are reduced by key with integer
// atomics on per-output fixed-point values. A first pass records each output component's largest
// contribution magnitude (atomicMax on the float's bits, order independent); each component then
// gets a power-of-two scale that leaves ceil(log2 n) + 1 bits of headroom in a signed 64-bit
// accumulator; a second pass adds the scaled, rounded contributions (integer addition is
// associative, so the sum is the same in every run); a last pass converts and accumulates into the
// caller's gradient arrays. Resolution: 2^-(61 - ceil(log2 n)) of the component's largest term.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>

#include "../../include/ba_cuda.h"
#include "ba_device.cuh"

namespace omvgba {
namespace residual {

constexpr int kThreads = 256;

// Per-camera constants computed once per call.
template <typename T>
struct CamPre {
  T R[9];
  T Jl[9];  // left Jacobian of SO(3) at rotvec (VJP only)
  T f, k1, k2, turn;
  int has_turn;
  int pad[3];
};

template <typename T>
__device__ __forceinline__ void rodrigues(const T w[3], T R[9], T Jl[9]) {
  const T t2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  const T th = sqrt(t2);
  // a = sin(th)/th, b = (1 - cos th)/th^2 = 2 sin^2(th/2)/th^2, c = (th - sin th)/th^3
  T a, b, c;
  const T small = sizeof(T) == 4 ? T(0.1) : T(1e-3);
  if (th < small) {
    a = T(1) - t2 / T(6) + t2 * t2 / T(120);
    b = T(0.5) - t2 / T(24) + t2 * t2 / T(720);
    c = T(1) / T(6) - t2 / T(120) + t2 * t2 / T(5040);
  } else {
    const T s = sin(th), h = sin(T(0.5) * th);
    a = s / th;
    b = T(2) * h * h / t2;
    c = (th - s) / (t2 * th);
  }
  // K = [w]x, K^2 = w w^T - t2 I
  const T K[9] = {0, -w[2], w[1], w[2], 0, -w[0], -w[1], w[0], 0};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      const T k2 = w[i] * w[j] - (i == j ? t2 : T(0));
      const T id = i == j ? T(1) : T(0);
      R[3 * i + j] = id + a * K[3 * i + j] + b * k2;
      Jl[3 * i + j] = id + b * K[3 * i + j] + c * k2;
    }
}

template <typename T>
__device__ __forceinline__ CamPre<T> make_pre(const T* __restrict__ rotvec, const T* __restrict__ intr, uint64_t j) {
  CamPre<T> c;
  const T w[3] = {rotvec[3 * j], rotvec[3 * j + 1], rotvec[3 * j + 2]};
  rodrigues(w, c.R, c.Jl);
  c.f = intr[3 * j];
  c.k1 = intr[3 * j + 1];
  c.k2 = intr[3 * j + 2];
  double turn = 0.0;
  c.has_turn = first_radial_turn_squared((double)c.k1, (double)c.k2, &turn) ? 1 : 0;
  c.turn = (T)turn;
  return c;
}

template <typename T>
__global__ void k_cam_prepare(uint64_t ncam, const T* __restrict__ rotvec, const T* __restrict__ intr,
                              CamPre<T>* __restrict__ out) {
  const uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (j >= ncam) return;
  out[j] = make_pre(rotvec, intr, j);
}

// Residual, J = d residual / d X_c and the intrinsic columns (log f, k1, k2); false when the
// observation is inadmissible.
template <typename T>
__device__ __forceinline__ bool radial_eval(const CamPre<T>& c, T X, T Y, T Z, T ox, T oy, T r[2], T J[2][3],
                                            T Ji[2][3]) {
  const T s = fmax(fmax(fabs(X), fabs(Y)), fabs(Z));
  if (!(isfinite(X) && isfinite(Y) && isfinite(Z)) || !(Z > T(64.0 * kEps) * s)) return false;
  if (!(c.f > T(0) && isfinite(c.f) && isfinite(c.k1) && isfinite(c.k2))) return false;
  const T iz = T(1) / Z;
  const T n0 = X * iz, n1 = Y * iz;
  const T r2 = n0 * n0 + n1 * n1;
  if (c.has_turn && r2 >= c.turn) return false;
  const T r4 = r2 * r2;
  const T dist = T(1) + c.k1 * r2 + c.k2 * r4;
  const T rd = c.k1 + T(2) * (c.k2 * r2);
  const T slope = dist + T(2) * r2 * rd;
  const T det = dist * slope;
  if (!isfinite(det) || det <= T(1e-12)) return false;
  const T p0 = c.f * dist * n0, p1 = c.f * dist * n1;
  const T dx = T(2) * n0 * rd, dy = T(2) * n1 * rd;
  const T nj00 = c.f * (dist + n0 * dx), nj01 = c.f * n0 * dy;
  const T nj10 = c.f * n1 * dx, nj11 = c.f * (dist + n1 * dy);
  J[0][0] = nj00 * iz;
  J[0][1] = nj01 * iz;
  J[0][2] = -(nj00 * n0 + nj01 * n1) * iz;
  J[1][0] = nj10 * iz;
  J[1][1] = nj11 * iz;
  J[1][2] = -(nj10 * n0 + nj11 * n1) * iz;
  r[0] = p0 - ox;
  r[1] = p1 - oy;
  Ji[0][0] = p0;
  Ji[0][1] = c.f * r2 * n0;
  Ji[0][2] = c.f * r4 * n0;
  Ji[1][0] = p1;
  Ji[1][1] = c.f * r2 * n1;
  Ji[1][2] = c.f * r4 * n1;
  return isfinite(r[0]) && isfinite(r[1]) && isfinite(J[0][0] + J[0][1] + J[0][2] + J[1][0] + J[1][1] + J[1][2]);
}

template <typename T>
__device__ __forceinline__ void camera_point(const CamPre<T>& c, const T* t, const T* X, T xc[3], T rx[3]) {
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    rx[i] = c.R[3 * i] * X[0] + c.R[3 * i + 1] * X[1] + c.R[3 * i + 2] * X[2];
    xc[i] = rx[i] + t[i];
  }
}

// Forward pass: the camera constants are recomputed per observation, so the pass needs no scratch.
// An observation whose camera or point index is out of range (a negative int32 index reads as a
// large uint32) touches no camera or point and gets a NaN residual.
template <typename T>
__global__ void k_forward(uint64_t n, const uint32_t* __restrict__ cam, const uint32_t* __restrict__ pt,
                          const T* __restrict__ pixel, const T* __restrict__ rotvec, const T* __restrict__ intr,
                          const T* __restrict__ trans, const T* __restrict__ points, uint64_t ncam, uint64_t npts,
                          T* __restrict__ residual) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t j = cam[i], p = pt[i];
  if (j >= ncam || p >= npts) {
    residual[2 * i] = T(NAN);
    residual[2 * i + 1] = T(NAN);
    return;
  }
  const CamPre<T> c = make_pre(rotvec, intr, j);
  const T X[3] = {points[3 * (uint64_t)p], points[3 * (uint64_t)p + 1], points[3 * (uint64_t)p + 2]};
  const T t[3] = {trans[3 * (uint64_t)j], trans[3 * (uint64_t)j + 1], trans[3 * (uint64_t)j + 2]};
  T xc[3], rx[3], r[2], J[2][3], Ji[2][3];
  camera_point(c, t, X, xc, rx);
  const T nan = T(NAN);
  if (!radial_eval(c, xc[0], xc[1], xc[2], pixel[2 * i], pixel[2 * i + 1], r, J, Ji)) {
    residual[2 * i] = nan;
    residual[2 * i + 1] = nan;
    return;
  }
  residual[2 * i] = r[0];
  residual[2 * i + 1] = r[1];
}

// Fixed-point accumulation tables, one entry per output component (cameras: 9 = rotvec 3,
// translation 3, intrinsics 3; points: 3).
struct Accum {
  uint32_t* maxbits;  // pass 0: largest |contribution| (float bits); then the component's exponent
  unsigned long long* sum;
  uint64_t ncomp;
  uint32_t* bad_index;  // set when an observation's camera or point index is out of range
};

constexpr int kCamComps = 9;

__device__ __forceinline__ void record_max(uint32_t* slot, float v) {
  const float a = fabsf(v);
  if (a != 0.0f || isnan(v)) atomicMax(slot, isnan(v) ? 0x7fc00000u : __float_as_uint(a));
}

__device__ __forceinline__ void add_fixed(const Accum& acc, uint64_t k, float v) {
  if (v == 0.0f) return;
  const int e = (int)acc.maxbits[k];
  if (e == INT32_MIN) return;  // non-finite component: resolved in the finish pass
  const long long q = llrint(ldexp((double)v, e));
  atomicAdd(acc.sum + k, (unsigned long long)q);
}

// One observation's contributions; PASS 0 records maxima, PASS 1 adds fixed-point values. An
// observation whose camera or point index is out of range adds nothing anywhere and raises the
// bad-index word, which makes the finish pass write NaN into every gradient output.
template <int PASS>
__global__ void k_vjp(uint64_t n, const uint32_t* __restrict__ cam, const uint32_t* __restrict__ pt,
                      const float* __restrict__ pixel, const CamPre<float>* __restrict__ pre,
                      const float* __restrict__ trans, const float* __restrict__ points,
                      const float* __restrict__ grad, uint64_t ncam, uint64_t npts, Accum acc) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t j = cam[i], p = pt[i];
  if (j >= ncam || p >= npts) {
    if (PASS == 0) atomicOr(acc.bad_index, 1u);
    return;
  }
  const float g0 = grad[2 * i], g1 = grad[2 * i + 1];
  if (g0 == 0.0f && g1 == 0.0f) return;
  const CamPre<float> c = pre[j];
  const float X[3] = {points[3 * (uint64_t)p], points[3 * (uint64_t)p + 1], points[3 * (uint64_t)p + 2]};
  const float t[3] = {trans[3 * (uint64_t)j], trans[3 * (uint64_t)j + 1], trans[3 * (uint64_t)j + 2]};
  float xc[3], rx[3], r[2], J[2][3], Ji[2][3];
  camera_point(c, t, X, xc, rx);
  if (!radial_eval(c, xc[0], xc[1], xc[2], pixel[2 * i], pixel[2 * i + 1], r, J, Ji)) return;
  float v[12];
  float a[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) a[k] = J[0][k] * g0 + J[1][k] * g1;
  // rotation: Jl^T (rx x a)
  const float ca[3] = {rx[1] * a[2] - rx[2] * a[1], rx[2] * a[0] - rx[0] * a[2], rx[0] * a[1] - rx[1] * a[0]};
#pragma unroll
  for (int s = 0; s < 3; ++s) v[s] = c.Jl[s] * ca[0] + c.Jl[3 + s] * ca[1] + c.Jl[6 + s] * ca[2];
#pragma unroll
  for (int k = 0; k < 3; ++k) v[3 + k] = a[k];
  v[6] = (Ji[0][0] * g0 + Ji[1][0] * g1) / c.f;
  v[7] = Ji[0][1] * g0 + Ji[1][1] * g1;
  v[8] = Ji[0][2] * g0 + Ji[1][2] * g1;
  // point: R^T a
#pragma unroll
  for (int k = 0; k < 3; ++k) v[9 + k] = c.R[k] * a[0] + c.R[3 + k] * a[1] + c.R[6 + k] * a[2];
  const uint64_t cbase = (uint64_t)kCamComps * j, pbase = (uint64_t)kCamComps * ncam + 3 * (uint64_t)p;
  if (PASS == 0) {
#pragma unroll
    for (int k = 0; k < 9; ++k) record_max(acc.maxbits + cbase + k, v[k]);
#pragma unroll
    for (int k = 0; k < 3; ++k) record_max(acc.maxbits + pbase + k, v[9 + k]);
  } else {
#pragma unroll
    for (int k = 0; k < 9; ++k) add_fixed(acc, cbase + k, v[k]);
#pragma unroll
    for (int k = 0; k < 3; ++k) add_fixed(acc, pbase + k, v[9 + k]);
  }
}

// Converts each component's maximum into its scale exponent (in place).
__global__ void k_vjp_scales(Accum acc, int headroom) {
  const uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (k >= acc.ncomp) return;
  const uint32_t bits = acc.maxbits[k];
  if (bits == 0u) {
    acc.maxbits[k] = 0u;  // no contribution: exponent unused
    return;
  }
  if (bits >= 0x7f800000u) {
    acc.maxbits[k] = (uint32_t)INT32_MIN;
    return;
  }
  int E;
  frexp((double)__uint_as_float(bits), &E);  // max < 2^E
  acc.maxbits[k] = (uint32_t)(62 - headroom - E);
}

__global__ void k_vjp_finish(Accum acc, uint64_t ncam, float* __restrict__ g_rot, float* __restrict__ g_t,
                             float* __restrict__ g_int, float* __restrict__ g_pt) {
  const uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (k >= acc.ncomp) return;
  const int e = (int)acc.maxbits[k];
  float val;
  if (e == INT32_MIN || *acc.bad_index != 0u)
    val = NAN;
  else
    val = (float)ldexp((double)(long long)acc.sum[k], -e);
  if (k < kCamComps * ncam) {
    const uint64_t j = k / kCamComps, c = k - kCamComps * j;
    if (c < 3)
      g_rot[3 * j + c] += val;
    else if (c < 6)
      g_t[3 * j + c - 3] += val;
    else
      g_int[3 * j + c - 6] += val;
  } else {
    g_pt[k - kCamComps * ncam] += val;
  }
}

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Workspace: camera table, then the cleared region (maxima, sums, bad-index word).
struct VjpLayout {
  size_t pre, maxbits, sum, bad, total;
};
inline VjpLayout vjp_layout(uint64_t ncam, uint64_t npts) {
  VjpLayout l;
  const uint64_t ncomp = kCamComps * ncam + 3 * npts;
  l.pre = 0;
  l.maxbits = align256(sizeof(CamPre<float>) * ncam);
  l.sum = l.maxbits + align256(sizeof(uint32_t) * ncomp);
  l.bad = l.sum + align256(sizeof(unsigned long long) * ncomp);
  l.total = l.bad + 256;
  return l;
}

inline unsigned grid_for(uint64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

inline int ceil_log2(uint64_t n) {
  int b = 0;
  while ((1ull << b) < n && b < 63) ++b;
  return b;
}

int fail(omvgba_error* e, int code, const std::string& msg) {
  if (e) {
    e->code = code;
    e->detail = -1;
    std::strncpy(e->message, msg.c_str(), sizeof(e->message) - 1);
    e->message[sizeof(e->message) - 1] = 0;
  }
  return code;
}

int ok(omvgba_error* e) {
  if (e) {
    e->code = 0;
    e->detail = -1;
    e->message[0] = 0;
  }
  return OMVGBA_OK;
}

int cuda_status(omvgba_error* e) {
  cudaError_t st = cudaGetLastError();
  if (st != cudaSuccess) return fail(e, OMVGBA_CUDA_ERROR, std::string("CUDA error: ") + cudaGetErrorString(st));
  return ok(e);
}

template <typename T>
int forward(void* stream, uint64_t n, const uint32_t* cam, const uint32_t* pt, const T* pixel, uint64_t ncam,
            const T* rotvec, const T* trans, const T* intr, uint64_t npts, const T* points, T* residual,
            omvgba_error* err) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_forward<T><<<grid_for(n), kThreads, 0, st>>>(n, cam, pt, pixel, rotvec, intr, trans, points, ncam, npts,
                                                  residual);
  return cuda_status(err);
}

bool any_null(std::initializer_list<const void*> ptrs) {
  for (const void* p : ptrs)
    if (!p) return true;
  return false;
}

}  // namespace residual
}  // namespace omvgba

using namespace omvgba::residual;

extern "C" {

uint64_t omvgba_residual_vjp_workspace_bytes(uint64_t observation_count, uint64_t camera_count,
                                             uint64_t point_count) {
  (void)observation_count;
  return vjp_layout(camera_count, point_count).total;
}

int32_t omvgba_residual_forward_f32(void* stream, uint64_t observation_count, const uint32_t* camera_index,
                                    const uint32_t* point_index, const float* pixel, uint64_t camera_count,
                                    const float* rotvec, const float* translation, const float* intrinsics,
                                    uint64_t point_count, const float* points, float* residual,
                                    omvgba_error* error) {
  if (observation_count == 0) return ok(error);
  if (any_null({camera_index, point_index, pixel, rotvec, translation, intrinsics, points, residual}))
    return fail(error, OMVGBA_INVALID_ARGUMENT, "null argument");
  return forward<float>(stream, observation_count, camera_index, point_index, pixel, camera_count, rotvec,
                        translation, intrinsics, point_count, points, residual, error);
}

int32_t omvgba_residual_forward_f64(void* stream, uint64_t observation_count, const uint32_t* camera_index,
                                    const uint32_t* point_index, const double* pixel, uint64_t camera_count,
                                    const double* rotvec, const double* translation, const double* intrinsics,
                                    uint64_t point_count, const double* points, double* residual,
                                    omvgba_error* error) {
  if (observation_count == 0) return ok(error);
  if (any_null({camera_index, point_index, pixel, rotvec, translation, intrinsics, points, residual}))
    return fail(error, OMVGBA_INVALID_ARGUMENT, "null argument");
  return forward<double>(stream, observation_count, camera_index, point_index, pixel, camera_count, rotvec,
                         translation, intrinsics, point_count, points, residual, error);
}

int32_t omvgba_residual_vjp_f32(void* stream, uint64_t observation_count, const uint32_t* camera_index,
                                const uint32_t* point_index, const float* pixel, uint64_t camera_count,
                                const float* rotvec, const float* translation, const float* intrinsics,
                                uint64_t point_count, const float* points, const float* grad_residual,
                                float* grad_rotvec, float* grad_translation, float* grad_intrinsics,
                                float* grad_points, void* workspace, uint64_t workspace_bytes,
                                omvgba_error* error) {
  if (observation_count == 0) return ok(error);
  if (any_null({camera_index, point_index, pixel, rotvec, translation, intrinsics, points, grad_residual,
                grad_rotvec, grad_translation, grad_intrinsics, grad_points, workspace}))
    return fail(error, OMVGBA_INVALID_ARGUMENT, "null argument");
  const VjpLayout l = vjp_layout(camera_count, point_count);
  if (workspace_bytes < l.total)
    return fail(error, OMVGBA_INVALID_ARGUMENT,
                "workspace too small: " + std::to_string(workspace_bytes) + " < " + std::to_string(l.total));
  if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0)
    return fail(error, OMVGBA_INVALID_ARGUMENT, "workspace must be 256-byte aligned");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned char* ws = static_cast<unsigned char*>(workspace);
  CamPre<float>* pre = reinterpret_cast<CamPre<float>*>(ws + l.pre);
  Accum acc{reinterpret_cast<uint32_t*>(ws + l.maxbits), reinterpret_cast<unsigned long long*>(ws + l.sum),
            kCamComps * camera_count + 3 * point_count, reinterpret_cast<uint32_t*>(ws + l.bad)};
  if (cudaMemsetAsync(ws + l.maxbits, 0, l.total - l.maxbits, st) != cudaSuccess) return cuda_status(error);
  k_cam_prepare<float><<<grid_for(camera_count), kThreads, 0, st>>>(camera_count, rotvec, intrinsics, pre);
  k_vjp<0><<<grid_for(observation_count), kThreads, 0, st>>>(observation_count, camera_index, point_index, pixel, pre,
                                                             translation, points, grad_residual, camera_count,
                                                             point_count, acc);
  k_vjp_scales<<<grid_for(acc.ncomp), kThreads, 0, st>>>(acc, ceil_log2(observation_count) + 1);
  k_vjp<1><<<grid_for(observation_count), kThreads, 0, st>>>(observation_count, camera_index, point_index, pixel, pre,
                                                             translation, points, grad_residual, camera_count,
                                                             point_count, acc);
  k_vjp_finish<<<grid_for(acc.ncomp), kThreads, 0, st>>>(acc, camera_count, grad_rotvec, grad_translation,
                                                         grad_intrinsics, grad_points);
  return cuda_status(error);
}

}  // extern "C"
