// sfm_refresh.cu — the landmark reprojection-error refresh that openmvg-sfm runs after it commits a
// bundle adjustment (refresh_landmark_reprojection_errors_for, crates/openmvg-sfm/src/ops/
// reconstruction/bundle.rs:510-637), on the GPU.
//
// One thread per landmark walks the landmark's track in order: for each supporting observation whose
// view has a pose it evaluates the pixel-equivalent residual of the camera residual policy with no
// limit (camera_pixel_equivalent), keeps it when it exists and is finite, and sums the kept ones in
// track order, so the mean is the reference's sequential sum divided by the count. The camera point
// is R (X - C) for the world-to-camera rotation R and the camera centre C of the pose (the reference
// holds t = -R C and evaluates R X + t; the two agree to rounding). Fewer than two kept residuals
// reject the landmark; a landmark that kept every supporting residual keeps its support; otherwise
// the support shrinks to the kept observations.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "camera_models.cuh"
#include "gpu_solver.hpp"

namespace omvgba {

__global__ void __launch_bounds__(128)
    k_sfm_refresh(uint64_t landmarks, const double* __restrict__ rotation, const double* __restrict__ center,
                  const CameraDev* __restrict__ cameras, const double* __restrict__ points,
                  const uint8_t* __restrict__ active, const uint64_t* __restrict__ offset,
                  const uint32_t* __restrict__ track_pose, const uint32_t* __restrict__ track_intrinsic,
                  const double* __restrict__ track_pixel, const uint8_t* __restrict__ support_in,
                  uint8_t* __restrict__ support_out, uint8_t* __restrict__ update, double* __restrict__ error,
                  uint32_t* __restrict__ removed) {
  const uint64_t l = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= landmarks) return;
  const uint64_t a = offset[l], b = offset[l + 1];
  removed[l] = 0;
  if (!active[l]) {
    update[l] = OMVGBA_REFRESH_SKIPPED;
    for (uint64_t o = a; o < b; ++o) support_out[o] = support_in[o];
    return;
  }
  const double X[3] = {points[3 * l], points[3 * l + 1], points[3 * l + 2]};
  double sum = 0.0;
  uint32_t kept = 0, supporting = 0;
  for (uint64_t o = a; o < b; ++o) {
    uint8_t keep = 0;
    if (support_in[o]) {
      ++supporting;
      const uint32_t p = track_pose[o];
      if (p != OMVGBA_NO_POSE) {
        const double* R = rotation + 9 * (size_t)p;
        const double* C = center + 3 * (size_t)p;
        const double d0 = X[0] - C[0], d1 = X[1] - C[1], d2 = X[2] - C[2];
        const double xc[3] = {R[0] * d0 + R[1] * d1 + R[2] * d2, R[3] * d0 + R[4] * d1 + R[5] * d2,
                              R[6] * d0 + R[7] * d1 + R[8] * d2};
        double r;
        if (camera_pixel_equivalent(cameras[track_intrinsic[o]], xc, track_pixel[2 * o], track_pixel[2 * o + 1], &r)) {
          sum += r;
          ++kept;
          keep = 1;
        }
      }
    }
    support_out[o] = keep;
  }
  if (kept < 2 || kept == supporting) {  // rejected or unchanged: the support stays as it was
    for (uint64_t o = a; o < b; ++o) support_out[o] = support_in[o];
    update[l] = kept < 2 ? OMVGBA_REFRESH_REJECTED : OMVGBA_REFRESH_UNCHANGED;
    if (kept >= 2) error[l] = sum / (double)kept;
    return;
  }
  update[l] = OMVGBA_REFRESH_PRUNED;
  error[l] = sum / (double)kept;
  removed[l] = supporting - kept;
}

namespace {

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw SolveFailure{OMVGBA_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e)};
}

// Stream-ordered device buffer, freed on the stream when it goes out of scope.
struct StreamBuf {
  void* p = nullptr;
  cudaStream_t s;
  explicit StreamBuf(cudaStream_t stream) : s(stream) {}
  StreamBuf(const StreamBuf&) = delete;
  StreamBuf& operator=(const StreamBuf&) = delete;
  ~StreamBuf() {
    if (p) cudaFreeAsync(p, s);
  }
  template <typename T>
  T* alloc(size_t count) {
    check(cudaMallocAsync(&p, count ? sizeof(T) * count : 16, s), "cudaMallocAsync");
    return static_cast<T*>(p);
  }
  template <typename T>
  T* upload(const T* host, size_t count) {
    T* d = alloc<T>(count);
    if (count) check(cudaMemcpyAsync(d, host, sizeof(T) * count, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
    return d;
  }
};

}  // namespace

void gpu_sfm_refresh(Context* ctx, const SfmRefreshInput& in, SfmRefreshOutput& out) {
  check(cudaSetDevice(context_device(ctx)), "cudaSetDevice");
  cudaStream_t st = static_cast<cudaStream_t>(context_stream(ctx));
  const uint64_t L = in.landmark_count, N = in.track_count;
  std::vector<CameraDev> cams(in.intrinsic_count);
  const omvgba_intrinsic* intr = static_cast<const omvgba_intrinsic*>(in.intrinsics);
  for (uint64_t i = 0; i < in.intrinsic_count; ++i) cams[i] = make_camera_dev(intr[i]);
  StreamBuf b_rot(st), b_cen(st), b_cam(st), b_pts(st), b_act(st), b_off(st), b_tp(st), b_ti(st), b_px(st),
      b_sin(st), b_sout(st), b_upd(st), b_err(st), b_rem(st);
  const double* rot = b_rot.upload(in.rotation, 9 * in.pose_count);
  const double* cen = b_cen.upload(in.center, 3 * in.pose_count);
  const CameraDev* dcam = b_cam.upload(cams.data(), cams.size());
  const double* pts = b_pts.upload(in.points, 3 * L);
  const uint8_t* act = b_act.upload(in.active, L);
  const uint64_t* off = b_off.upload(in.track_offset, L + 1);
  const uint32_t* tp = b_tp.upload(in.track_pose, N);
  const uint32_t* ti = b_ti.upload(in.track_intrinsic, N);
  const double* px = b_px.upload(in.track_pixel, 2 * N);
  const uint8_t* sin_ = b_sin.upload(in.track_support, N);
  uint8_t* sout = b_sout.alloc<uint8_t>(N);
  uint8_t* upd = b_upd.alloc<uint8_t>(L);
  double* err = b_err.upload(out.reprojection_error, L);  // untouched entries come back as they were
  uint32_t* rem = b_rem.alloc<uint32_t>(L);
  if (L > 0) {
    k_sfm_refresh<<<(unsigned)((L + 127) / 128), 128, 0, st>>>(L, rot, cen, dcam, pts, act, off, tp, ti, px, sin_,
                                                                 sout, upd, err, rem);
    check(cudaGetLastError(), "k_sfm_refresh launch");
  }
  std::vector<uint32_t> removed(L);
  if (N) check(cudaMemcpyAsync(out.track_support, sout, N, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
  if (L) {
    check(cudaMemcpyAsync(out.landmark_update, upd, L, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    check(cudaMemcpyAsync(out.reprojection_error, err, sizeof(double) * L, cudaMemcpyDeviceToHost, st),
          "cudaMemcpyAsync");
    check(cudaMemcpyAsync(removed.data(), rem, sizeof(uint32_t) * L, cudaMemcpyDeviceToHost, st),
          "cudaMemcpyAsync");
  }
  check(cudaStreamSynchronize(st), "k_sfm_refresh");
  out.rejected_landmarks = 0;
  out.removed_observations = 0;
  for (uint64_t l = 0; l < L; ++l) {
    out.rejected_landmarks += out.landmark_update[l] == OMVGBA_REFRESH_REJECTED ? 1 : 0;
    out.removed_observations += removed[l];
  }
}

}  // namespace omvgba
