// gpu_solver.hpp — interface between the host-side lowering (host.cpp) and the GPU
// Levenberg–Marquardt driver (gpu_solver.cu).
#pragma once

#include <cstdint>
#include <string>
#include <memory>
#include <type_traits>
#include <utility>
#include <vector>

#include "ba_device.cuh"

namespace omvgba {

// Failure carrying an omvgba_code.
struct SolveFailure {
  int code;
  std::string message;
};

// The problem after native lowering (anchor frame, point-major observations, native camera order).
// Allocator whose value-less construct() default-initializes: resize() of a vector of a trivial
// type then leaves the new elements unwritten. For large host buffers that are filled completely
// right after allocation (by parallel loops), so that they are not first zeroed by one thread.
template <typename T>
struct DefaultInitAllocator : std::allocator<T> {
  template <typename U>
  struct rebind {
    using other = DefaultInitAllocator<U>;
  };
  DefaultInitAllocator() noexcept = default;
  template <typename U>
  DefaultInitAllocator(const DefaultInitAllocator<U>&) noexcept {}
  template <typename U>
  void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value) {
    ::new (static_cast<void*>(p)) U;
  }
  template <typename U, typename... Args>
  void construct(U* p, Args&&... args) {
    ::new (static_cast<void*>(p)) U(std::forward<Args>(args)...);
  }
};
template <typename T>
using FillVector = std::vector<T, DefaultInitAllocator<T>>;

struct NativeProblem {
  bool self_cal = false;
  int ncam = 0;
  std::vector<double> rotation;     // ncam x 9 (row-major, world -> camera in the anchor frame)
  std::vector<double> translation;  // ncam x 3
  FillVector<double> points;        // P x 3
  std::vector<uint8_t> fixed_points;
  std::vector<uint8_t> fixed_poses;
  FillVector<uint32_t> obs_cam;     // native camera per observation (point-major order)
  FillVector<double> obs_px;        // N x 2 (self-calibration: centred at the principal point)
  FillVector<uint64_t> obs_src;     // input observation index
  FillVector<uint32_t> obs_model;   // calibrated: fixed camera model per observation
  FillVector<uint64_t> pt_off;      // P + 1
  FillVector<uint64_t> point_source;  // native point -> input point (points are regrouped for locality)
  bool pixel_model = true;          // pinhole pixel projection (no distortion anywhere)
  std::vector<FixedCameraDev> models;
  std::vector<double> groups;       // self-calibration: ng x 3 (focal, k1, k2)
  std::vector<uint32_t> cam_group;  // per native camera
  std::vector<int> group_dim;       // free (log f, k1, k2) prefix per group, 0 when fixed
  int gauge_cam = -1;               // FixedBaseline camera on the S^2 chart, -1 when free
  // Calibrated solves carry explicit per-camera pose masks (bit 0 rotation, bit 1 translation, 0
  // fixed; workspace/topology.rs:305-347): camera 0 is free when its mask is, a rotation-only block
  // turns the camera about its fixed centre and a translation-only block moves only the centre.
  // Self-calibration keeps the legacy layout (camera 0 fixed, the others full or fixed).
  bool explicit_masks = false;
  std::vector<uint8_t> pose_mask;   // per native camera
  bool translation_only = false;    // no free mask moves a rotation (CameraPoseVariables)
  // Angular residuals (kernel/projection.rs:89-149): each observation's unit bearing in the camera
  // frame, point-major like obs_px
  bool angular = false;
  FillVector<double> obs_bearing;   // N x 3
};

// Free pose coordinates of native camera c (ReducedLayout, workspace/topology.rs:263-347).
inline int pose_block_dim(const NativeProblem& n, int c) {
  if (n.explicit_masks) {
    const int m = n.pose_mask[c];
    if (n.fixed_poses[c] || m == 0) return 0;
    return 3 * (m & 1) + ((m & 2) ? (c == n.gauge_cam ? 2 : 3) : 0);
  }
  return (c == 0 || n.fixed_poses[c]) ? 0 : (c == n.gauge_cam ? 5 : 6);
}

struct LmOptions {
  uint64_t max_iterations = 50;
  LossDev loss{kLossL2, 0.0};
  double gradient_tolerance = 1e-10, step_tolerance = 1e-8, relative_cost_tolerance = 1e-6;
  bool iterative = false;           // the linear solver in use (resolved from Auto by the solver)
  int linear_solver = 1;            // the configuration's choice: 0 Auto, 1 Direct, 2 Iterative
  uint64_t workspace_budget = 0;    // explicit workspace budget in bytes, 0 when none
  double pcg_tolerance = 1e-1;
  uint64_t pcg_max_iterations = 600;
  int precision = 0;  // 0 FP64, 1 mixed
  int matvec = 0;     // 0 auto, 1 explicit, 2 implicit
  int dense_rank_limit = 2048;
  bool certify_intrinsics = true;  // self-calibration: compute the intrinsic marginal covariances
  void* stream = nullptr;  // cudaStream_t the solve runs on; null: the context's own stream
};

struct NativeReport {
  int status = 1;      // 0 converged, 1 max iterations, 2 stalled, 3 degenerate
  int reason = -1;     // 0 cost, 1 gradient, 2 step
  uint64_t iterations = 0, accepted = 0, rejected = 0;
  uint64_t rej[4] = {0, 0, 0, 0};
  double initial_cost = 0, initial_rmse = 0, final_cost = 0, final_rmse = 0;
  double gradient_inf_norm = 0;
  int rank = 3;        // 0 full, 2 deficient, 3 not assessed
  uint64_t weak = 0;
  uint64_t noninvertible = 0;
  uint64_t pcg_terms = 0;
  double final_damping = 0;
  int D = 0;
  // self-calibration certificate: (S^-1)_gg of each intrinsic group at the final state, 9 values per
  // group (row-major, the free dim x dim corner used); marginals_ok = 0 when S does not factor
  std::vector<double> marginals;
  int marginals_ok = 0;
  int iterative = 0;  // the linear solver the solve used (Auto resolved)
};

// The execution plan a solve would use, computed on the host without a GPU: Auto resolved against
// the budget (sparse/execution_policy.rs:122-253 restated with this solver's estimates) and the
// device workspace it needs.
struct ExecutionPlan {
  bool iterative = false;
  uint64_t direct_estimate = 0, cached_estimate = 0, workspace_bytes = 0;
};
ExecutionPlan execution_plan(const NativeProblem& problem, const LmOptions& options);

// Two-view bundle adjustment (native/two_view.rs, kernel/two_view/*): the first camera is the frame,
// the second's native pose and the points (native frame) are refined; pixel or angular measurements.
struct TwoViewProblem {
  bool angular = false;
  double cam[2][4] = {};          // pixel: fx, fy, cx, cy per view
  std::vector<double> obs;        // pixel: [view][point][2]
  std::vector<double> bearing;    // angular: [view][point][3]
  double R[9] = {}, t[3] = {};    // the second camera's native pose
  std::vector<double> points;     // P x 3, native frame
};
struct TwoViewReport {
  double R[9] = {}, t[3] = {};
  int status = 1, reason = -1;    // as NativeReport
  uint64_t iterations = 0, accepted = 0, rej[4] = {0, 0, 0, 0};
  double initial_cost = 0, final_cost = 0, initial_rmse = 0, final_rmse = 0, grad_norm = 0, final_damping = 0;
  int rank = 0;                   // of the final 5 x 5 reduced camera system
  uint64_t weak = 0;
};

struct Context;  // device, stream, pinned scratch

int device_count();
Context* context_create(int device, std::string* error);
int context_device(const Context* ctx);
void* context_stream(const Context* ctx);  // the context's cudaStream_t

// refresh_landmark_reprojection_errors_for (openmvg-sfm ops/reconstruction/bundle.rs:510-637) on the
// context's device, inputs and outputs in host memory (see omvgba_sfm_refresh_reprojection). The
// caller has checked every index. Throws SolveFailure on a CUDA error.
struct SfmRefreshInput {
  uint64_t pose_count, intrinsic_count, landmark_count, track_count;
  const double* rotation;      // 9 per pose, world to camera, row-major
  const double* center;        // 3 per pose
  const void* intrinsics;      // omvgba_intrinsic[intrinsic_count]
  const double* points;        // 3 per landmark
  const uint8_t* active;
  const uint64_t* track_offset;
  const uint32_t* track_pose, * track_intrinsic;
  const double* track_pixel;
  const uint8_t* track_support;
};
struct SfmRefreshOutput {
  uint8_t* landmark_update;
  double* reprojection_error;
  uint8_t* track_support;
  uint64_t rejected_landmarks = 0, removed_observations = 0;
};
void gpu_sfm_refresh(Context* ctx, const SfmRefreshInput& in, SfmRefreshOutput& out);
void context_destroy(Context* ctx);

// Runs the LM refinement on the GPU; on return points/rotation/translation/groups hold the refined
// native state. Throws SolveFailure.
// refine_ba_2view on the device; on return `problem.points` holds the refined points. Throws
// SolveFailure (OMVGBA_NUMERICAL for the kernel's own input errors).
TwoViewReport gpu_two_view(Context* ctx, TwoViewProblem& problem, const LmOptions& options);

NativeReport gpu_refine(Context* ctx, const NativeProblem& problem, const LmOptions& options,
                        std::vector<double>& rotation, std::vector<double>& translation,
                        std::vector<double>& points, std::vector<double>& groups);

// First linearization, per observation (point-major): see omvgba_debug_linearize.
void gpu_debug_linearize(Context* ctx, const NativeProblem& problem, const LmOptions& options, double* residual,
                         double* sqrt_weight, double* point_jacobian, double* camera_jacobian);

// Matrix-free S x versus the explicit dense S x at the first linearization (operator parity).
void gpu_debug_schur_product(Context* ctx, const NativeProblem& problem, const LmOptions& options, double lambda,
                             const double* x, double* y_mv, double* y_dense, int* dimension);

// A lowered problem kept resident in device memory for repeated solves from its initial state.
// The NativeProblem must outlive the Resident.
struct Resident;
struct ResidentInfo {
  uint64_t observations = 0, points = 0, cameras = 0, dimension = 0;
  uint64_t jacobian_entries = 0;  // sum over observations of 2 x (free camera dim + free point dim)
  uint64_t tiles64 = 0, tiles32 = 0;
  uint64_t record_bytes64 = 0, record_bytes32 = 0, metadata_bytes64 = 0, metadata_bytes32 = 0;
  int iterative = 0, mixed = 0;
};
Resident* resident_create(Context* ctx, const NativeProblem& problem, const LmOptions& options);
void resident_destroy(Resident* resident);
NativeReport resident_refine(Resident* resident, std::vector<double>& rotation, std::vector<double>& translation,
                             std::vector<double>& points, std::vector<double>& groups);
ResidentInfo resident_info(const Resident* resident);
// S_lambda x at the initial state's linearization; x and y are device pointers. stage 0: the
// whole product; stage 1: the tile pass alone (y is not written).
void resident_schur_product(Resident* resident, double lambda, bool fp32, int stage, const double* x, double* y);

// Kernels launched and host<->device bytes copied by the calling thread so far.
void telemetry_read(uint64_t* launches, uint64_t* h2d, uint64_t* d2h);

// Host threads that the set-up run by the calling thread may use (0: hardware_concurrency). Every
// parallel host loop writes disjoint outputs or combines per-chunk results in chunk order, so the
// result does not depend on this; it exists so that this can be tested.
void set_host_thread_limit(unsigned threads);
unsigned host_thread_limit();
// FNV-1a digest of the host-built device set-up of a lowered problem: the block tables and the
// matvec tiles in the precision the options select. Uses no GPU.
uint64_t setup_digest(const NativeProblem& problem, const LmOptions& options);
// FNV-1a over bytes, continuing from h.
uint64_t fnv1a(const void* data, size_t bytes, uint64_t h);

// Residual norms of an input problem's observations with a world-frame state, for the Solution
// metrics (solver.rs:1052-1131). active: per point flag. Returns false when a projection fails.
struct WorldMetrics {
  double cost = 0, rmse = 0;
  uint64_t count = 0;
  uint64_t inliers = 0;
  double inlier_sq = 0;
  bool ok = false;
};

}  // namespace omvgba
