/*
 * ba_cuda.h — C ABI of the B200-native bundle-adjustment solver.
 *
 * This header is the drop-in boundary for openmvg-ba's bundle-adjustment
 * hot path. Every entry point takes plain pointers and sizes; no C++ or
 * torch types cross it. All input buffers are caller-owned and read-only;
 * all output buffers are caller-allocated with the shapes stated below.
 *
 * Reference interfaces this boundary replaces (paths inside openmvg-rs):
 *   - BundleAdjuster::solve          crates/openmvg-ba/src/solver.rs:1562-1573
 *   - BundleProblem (+ builder)      crates/openmvg-ba/src/problem.rs:447-577
 *   - SolveConfig / validate         crates/openmvg-ba/src/solver.rs:74-155
 *   - SolveReport / SolveDiagnostics crates/openmvg-ba/src/solver.rs:294-624
 *   - Solution                       crates/openmvg-ba/src/solver.rs:788-1314
 *   - SolveError                     crates/openmvg-ba/src/solver.rs:1474-1493
 *   - ProblemError                   crates/openmvg-ba/src/problem.rs:731-779
 *
 * Return codes map one to one onto SolveError / ProblemError variants; the
 * UTF-8 message is written into omvgba_error.message.
 */
#ifndef OMVGBA_BA_CUDA_H
#define OMVGBA_BA_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OMVGBA_ABI_VERSION 3u

/* ---- return codes (SolveError, solver.rs:1474-1493; ProblemError, problem.rs:731) ---- */
enum omvgba_code {
  OMVGBA_OK = 0,
  OMVGBA_INVALID_CONFIG = 1,      /* SolveError::InvalidConfig */
  OMVGBA_UNSUPPORTED = 2,         /* SolveError::Unsupported: hand the problem on unchanged */
  OMVGBA_RESOURCE_EXHAUSTED = 3,  /* SolveError::ResourceExhausted */
  OMVGBA_NUMERICAL = 4,           /* SolveError::Numerical */
  OMVGBA_INTERNAL = 5,            /* SolveError::Internal */
  OMVGBA_INVALID_PROBLEM = 6,     /* ProblemError (BundleProblemBuilder::build) */
  OMVGBA_INVALID_ARGUMENT = 7,    /* null pointer, short output buffer, bad enum */
  OMVGBA_CUDA_ERROR = 8           /* a CUDA runtime call failed (reported as Internal upstream) */
};

typedef struct omvgba_error {
  int32_t code;
  int32_t detail; /* ProblemError variant index or offending element index, -1 if none */
  char message[480];
} omvgba_error;

/* ---- camera models (openmvg-core camera::Camera, brown_conrady.rs, distortion.rs) ---- */
enum omvgba_camera_model {
  OMVGBA_CAMERA_PINHOLE = 0,
  OMVGBA_CAMERA_BROWN_CONRADY = 1,
  OMVGBA_CAMERA_FISHEYE = 2,   /* accepted by the contract, rejected as Unsupported for pixel BA */
  OMVGBA_CAMERA_SPHERICAL = 3  /* idem */
};
/* RadialDistortion discriminant: None, K1, K1K2, K1K2K3 (distortion.rs:183-241) */
/* Brown-Conrady RadialDistortion, or the fisheye's FisheyeDistortion (K1K2K3K4 is fisheye only). */
enum omvgba_radial_kind {
  OMVGBA_RADIAL_NONE = 0,
  OMVGBA_RADIAL_K1 = 1,
  OMVGBA_RADIAL_K1K2 = 2,
  OMVGBA_RADIAL_K1K2K3 = 3,
  OMVGBA_RADIAL_K1K2K3K4 = 4
};
/* TangentialDistortion discriminant: None, P1, P1P2 (distortion.rs:459-527) */
enum omvgba_tangential_kind { OMVGBA_TANGENTIAL_NONE = 0, OMVGBA_TANGENTIAL_P1 = 1, OMVGBA_TANGENTIAL_P1P2 = 2 };

/* IntrinsicVariables bits (problem.rs:42-70) */
#define OMVGBA_INTRINSIC_FOCAL (1u << 0)
#define OMVGBA_INTRINSIC_PRINCIPAL_POINT (1u << 1)
#define OMVGBA_INTRINSIC_RADIAL (1u << 2)
#define OMVGBA_INTRINSIC_TANGENTIAL (1u << 3)
/* PoseVariables bits (problem.rs:15-40) */
#define OMVGBA_POSE_ROTATION (1u << 0)
#define OMVGBA_POSE_TRANSLATION (1u << 1)
#define OMVGBA_POSE_FREE (OMVGBA_POSE_ROTATION | OMVGBA_POSE_TRANSLATION)

/* BundlePose: WorldToCameraPose (rotation R world->camera, row-major; center C) + variables. */
typedef struct omvgba_pose {
  double rotation[9];
  double center[3];
  uint32_t variables;
  uint32_t reserved;
} omvgba_pose;

/* BundleIntrinsic: CameraIntrinsics + IntrinsicVariables + IntrinsicCertification. */
typedef struct omvgba_intrinsic {
  int32_t model;            /* omvgba_camera_model */
  int32_t radial_kind;      /* omvgba_radial_kind (Brown-Conrady and fisheye) */
  int32_t tangential_kind;  /* omvgba_tangential_kind (Brown-Conrady only) */
  uint32_t variables;       /* OMVGBA_INTRINSIC_* bits */
  int32_t certification;    /* 0 Required, 1 Waived */
  int32_t fixed_model;      /* CameraIntrinsics::is_fixed(): 1 forbids variable coordinates */
  double fx, fy, cx, cy;
  double k1, k2, k3, p1, p2;
  uint32_t width, height;   /* spherical: width (even), height = width / 2 */
  double k4;                /* fisheye K1K2K3K4 only */
} omvgba_intrinsic;

enum omvgba_residual_space { OMVGBA_RESIDUAL_PIXELS = 0, OMVGBA_RESIDUAL_ANGULAR = 1 };
/* RobustLoss (problem.rs:267-300). The scale carries its own residual space. */
enum omvgba_loss_kind { OMVGBA_LOSS_SQUARED = 0, OMVGBA_LOSS_HUBER = 1, OMVGBA_LOSS_CAUCHY = 2 };
/* Gauge (problem.rs:302-312) */
enum omvgba_gauge_kind { OMVGBA_GAUGE_FREE = 0, OMVGBA_GAUGE_FIXED_BASELINE = 1 };

/* BundleProblem (problem.rs:447-577) as structure-of-arrays. */
typedef struct omvgba_problem {
  uint64_t pose_count;
  const omvgba_pose* poses;
  uint64_t intrinsic_count;
  const omvgba_intrinsic* intrinsics;
  uint64_t point_count;
  const double* points;        /* point_count x 3, interleaved xyz */
  const uint8_t* point_fixed;  /* point_count flags, or NULL for all free */
  uint64_t observation_count;
  const uint32_t* observation_pose;
  const uint32_t* observation_intrinsic;
  const uint32_t* observation_point;
  const double* observation_pixel; /* observation_count x 2, interleaved */
  int32_t residual_space;      /* omvgba_residual_space */
  int32_t loss_kind;           /* omvgba_loss_kind */
  double loss_scale;           /* delta (Huber) or scale (Cauchy), in loss_scale_space units */
  int32_t loss_scale_space;    /* omvgba_residual_space of the loss scale */
  int32_t gauge_kind;          /* omvgba_gauge_kind */
  uint64_t gauge_first, gauge_second;
  double gauge_distance;
} omvgba_problem;

/* LinearSolver (solver.rs:11-18) */
enum omvgba_linear_solver { OMVGBA_SOLVER_AUTO = 0, OMVGBA_SOLVER_DIRECT = 1, OMVGBA_SOLVER_ITERATIVE = 2 };
/* Build-private precision policy (not in the reference API). */
enum omvgba_precision {
  OMVGBA_PRECISION_FP64 = 0,  /* every kernel in FP64 */
  OMVGBA_PRECISION_MIXED = 1  /* FP32 Jacobians and matvecs; FP64 point inverses, factorizations,
                                 dot products, cost and LM test; FP64 refinement of the step */
};
/* Build-private reduced-camera-system operator. */
enum omvgba_matvec { OMVGBA_MATVEC_AUTO = 0, OMVGBA_MATVEC_EXPLICIT = 1, OMVGBA_MATVEC_IMPLICIT = 2 };

/* SolveConfig (solver.rs:74-155) plus build-private execution options. */
typedef struct omvgba_config {
  uint64_t max_iterations;        /* default 50 */
  double function_tolerance;      /* default 1e-6 */
  double gradient_tolerance;      /* default 1e-10 */
  double parameter_tolerance;     /* default 1e-8 */
  int32_t linear_solver;          /* omvgba_linear_solver, default Auto */
  int32_t has_workspace_budget;   /* 0: None */
  uint64_t workspace_budget_bytes;
  /* build-private */
  int32_t precision;              /* omvgba_precision */
  int32_t matvec;                 /* omvgba_matvec */
  double pcg_relative_tolerance;  /* 0: native default 1e-1 (native/mod.rs:597-603) */
  uint32_t pcg_max_iterations;    /* 0: 600 (sparse/api.rs:395) */
  int32_t device;                 /* CUDA device ordinal */
  void* stream;                   /* cudaStream_t or NULL for a context-owned stream */
} omvgba_config;

/* Fill *config with SolveConfig::default() and the build-private defaults. */
void omvgba_config_default(omvgba_config* config);

/* SolveStatus / ConvergenceReason (solver.rs:87-105) */
enum omvgba_solve_status {
  OMVGBA_STATUS_CONVERGED = 0,
  OMVGBA_STATUS_MAX_ITERATIONS = 1,
  OMVGBA_STATUS_STALLED = 2,
  OMVGBA_STATUS_DEGENERATE = 3,
  OMVGBA_STATUS_SKIPPED = 4
};
enum omvgba_convergence_reason { OMVGBA_REASON_NONE = -1, OMVGBA_REASON_OBJECTIVE = 0, OMVGBA_REASON_GRADIENT = 1, OMVGBA_REASON_STEP = 2 };
/* Observability (solver.rs:107-115) */
enum omvgba_observability {
  OMVGBA_OBS_FULL_RANK = 0,
  OMVGBA_OBS_ONLY_EXPECTED_GAUGE = 1,
  OMVGBA_OBS_RANK_DEFICIENT = 2,
  OMVGBA_OBS_NOT_ASSESSED = 3
};

/* SolveReport + SolveDiagnostics (solver.rs:294-624). Optional fields carry a has_ flag. */
typedef struct omvgba_report {
  int32_t status;                 /* omvgba_solve_status */
  int32_t convergence_reason;     /* omvgba_convergence_reason */
  uint64_t iteration_count;
  double initial_objective, final_objective;
  double initial_rmse, final_rmse;
  uint64_t accepted_step_count, rejected_step_count;
  uint64_t rejected_linearization, rejected_step_solve, rejected_candidate, rejected_insufficient_reduction;
  int32_t has_stationarity;
  double scaled_gradient_inf_norm;
  int32_t observability;          /* omvgba_observability */
  int32_t has_weak_point_count;
  uint64_t weak_point_count;
  uint64_t quarantined_point_count;
  int32_t has_noninvertible_observation_count;
  uint64_t noninvertible_observation_count;
  int32_t has_observability_details;
  uint64_t details_pose_rank, details_pose_dimension, details_weak_point_count;
  int32_t has_linear_solver;
  int32_t linear_solver;          /* omvgba_linear_solver actually used */
  int32_t has_observation_count;
  uint64_t observation_count;
  int32_t has_inlier_count;
  uint64_t inlier_count;
  int32_t has_final_inlier_rmse;
  double final_inlier_rmse;
  uint64_t unconstrained_intrinsic_count; /* indices in omvgba_solution.unconstrained_intrinsics */
  /* build telemetry (not part of the reference report) */
  uint64_t pcg_iteration_count;
  uint64_t reduced_dimension;
  double final_damping;
  double solve_seconds;           /* wall time inside omvgba_solve */
  double upload_seconds;          /* host->device problem upload inside that time */
  uint64_t kernel_launches;       /* GPU kernels the call launched (graph-launched ones included) */
  uint64_t h2d_bytes, d2h_bytes;  /* host<->device bytes the call copied */
} omvgba_report;

/* Solution (solver.rs:788-1314). Every array is caller-allocated. */
typedef struct omvgba_solution {
  omvgba_pose* poses;              /* pose_count */
  omvgba_intrinsic* intrinsics;    /* intrinsic_count */
  double* points;                  /* point_count x 3 */
  uint64_t* quarantined_points;    /* capacity point_count; count = report.quarantined_point_count */
  uint64_t* unconstrained_intrinsics; /* capacity intrinsic_count */
  omvgba_report report;
} omvgba_solution;

/* One solver context per thread or stream: device workspaces, streams, no global state. */
typedef struct omvgba_context omvgba_context;

/* Number of CUDA devices visible to this process (0 when none or when the driver is missing). */
int32_t omvgba_device_count(void);

omvgba_context* omvgba_context_create(int32_t device, omvgba_error* error);
void omvgba_context_destroy(omvgba_context* context);
uint32_t omvgba_abi_version(void);

/* BundleAdjuster::solve (solver.rs:1562-1573) on the GPU. Never mutates the problem. */
int32_t omvgba_solve(omvgba_context* context, const omvgba_problem* problem, const omvgba_config* config,
                     omvgba_solution* solution, omvgba_error* error);

/* BundleAdjuster::name (solver.rs:1566). */
const char* omvgba_adjuster_name(void);

/*
 * A problem prepared once for repeated solves: validation, the quarantine of input points that
 * cannot be adjusted (quarantine.rs:34-96), lowering (native/mod.rs:260-367) and the upload to
 * device memory happen in omvgba_plan_create; every omvgba_plan_solve then starts from the
 * problem's initial state with everything already in device memory, and returns what omvgba_solve
 * would return for the same problem and config. The problem's arrays must stay alive and unchanged
 * until omvgba_plan_destroy. A plan runs on config->stream (or the context's stream) and, like its
 * context, is used by one thread at a time. No reference counterpart: the reference lowers and
 * solves in one call (native/mod.rs:117-367).
 */
typedef struct omvgba_plan omvgba_plan;

typedef struct omvgba_plan_info {
  uint64_t observation_count;     /* observations in the solved problem (after input quarantine) */
  uint64_t point_count;
  uint64_t camera_count;
  uint64_t reduced_dimension;     /* D, schur/layout.rs:143-205 */
  uint64_t jacobian_entries;      /* sum over observations of 2 x (free camera dim + free point dim) */
  uint64_t tile_count_fp64, tile_count_fp32;
  uint64_t record_bytes_fp64, record_bytes_fp32;      /* per-observation Jacobian records in device memory */
  uint64_t metadata_bytes_fp64, metadata_bytes_fp32;  /* per-tile segment tables of the matrix-free product */
  int32_t iterative;              /* 1: PCG steps; 0: dense Cholesky steps */
  int32_t mixed;                  /* 1: FP32 products with FP64 refinement */
} omvgba_plan_info;

int32_t omvgba_plan_create(omvgba_context* context, const omvgba_problem* problem, const omvgba_config* config,
                           omvgba_plan** plan, omvgba_error* error);
int32_t omvgba_plan_solve(omvgba_plan* plan, omvgba_solution* solution, omvgba_error* error);
int32_t omvgba_plan_info_get(const omvgba_plan* plan, omvgba_plan_info* info, omvgba_error* error);
/*
 * The reduced camera system product y = S_lambda x of a PCG plan at its initial state's
 * linearization (the first call, and the first after a solve or a new lambda, re-linearizes).
 * x and y are DEVICE pointers of reduced_dimension doubles. fp32 selects the FP32 records of a
 * mixed plan. stage 0 computes the whole product; stage 1 launches only the tile pass (the
 * per-point coupling partials, y untouched), for timing the kernel by itself; stage 2 builds only the
 * explicit S of the linearization by block rows (x and y untouched), for timing that kernel; stage 3
 * runs only the camera-side sums of the linearization's assembly (U blocks, gradients, damping
 * diagonal, pose/intrinsic edges and point coupling per block; x and y untouched). Runs on
 * the plan's stream without synchronizing. Operator: retained/operator.rs:137-227.
 */
int32_t omvgba_plan_schur_product(omvgba_plan* plan, double lambda, int32_t fp32, int32_t stage, const double* x,
                                  double* y, omvgba_error* error);
void omvgba_plan_destroy(omvgba_plan* plan);

/*
 * First linearization of the lowered problem, per observation in the solver's
 * point-major order (observations stably sorted by point, native/calibrated.rs:371-375).
 * Outputs: residual (n x 2, prediction minus pixel), sqrt_weight (n), point Jacobian
 * J_proj * R * s (n x 6, row-major 2x3), camera Jacobian (n x 2 x 9, row-major; columns
 * beyond the camera's free dimension are zero), source_index (n, the input observation).
 * Reference: schur/point.rs:176-355, kernel/projection.rs:47-87, self_calibration/model.rs:26-324.
 */
int32_t omvgba_debug_linearize(omvgba_context* context, const omvgba_problem* problem,
                               const omvgba_config* config, double* residual, double* sqrt_weight,
                               double* point_jacobian, double* camera_jacobian, uint64_t* source_index,
                               omvgba_error* error);

/*
 * Digest (64-bit FNV-1a) of the host side of a solve's set-up: the quarantine preparation (points
 * held out before the solve, native/mod.rs:260-340, quarantine.rs:34-96), the lowering
 * (native/self_calibration.rs:47-198, native/calibrated.rs:200-494) and the block tables and
 * matvec tiles the solver uploads, built with at most `threads` host threads (0: all of them).
 * Uses no GPU and needs no context. The set-up's result does not depend on the thread count (the
 * reference's reproducibility rule); this entry point exists to test that.
 */
int32_t omvgba_debug_setup_digest(const omvgba_problem* problem, const omvgba_config* config, uint32_t threads,
                                  uint64_t* digest, omvgba_error* error);

/*
 * The linear solver a solve of this problem and config would use, without a GPU: an explicit
 * Direct or Iterative choice as given; Auto resolved by the budget (the explicit
 * workspace_budget_bytes, else 1 GiB): the direct step when its estimate fits 4/5 of the budget, the
 * retained PCG first for calibrated problems with at least 250,000 observations and D >= 768
 * (crates/openmvg-ba/src/kernel/multi_view/sparse/execution_policy.rs:122-253). Also reports both
 * estimates in bytes. For tests of the policy.
 */
int32_t omvgba_debug_execution_plan(const omvgba_problem* problem, const omvgba_config* config, int32_t* iterative,
                                    uint64_t* direct_estimate, uint64_t* cached_estimate, omvgba_error* error);

/*
 * Reduced camera system product S_lambda x at the first linearization of the lowered problem,
 * computed twice: by the matrix-free kernel the PCG uses (y_matvec) and from the explicit dense
 * Schur complement (y_dense). With x == NULL only *dimension is written. FP64; for operator
 * parity tests. Reference operator: crates/openmvg-ba/src/kernel/multi_view/sparse/retained/operator.rs:137-227.
 */
int32_t omvgba_debug_schur_product(omvgba_context* context, const omvgba_problem* problem,
                                   const omvgba_config* config, double lambda, const double* x, double* y_matvec,
                                   double* y_dense, int32_t* dimension, omvgba_error* error);

/*
 * Reprojection residual of the centred radial model (self_calibration/model.rs:26-129) over an
 * unsorted observation list, and its vector-Jacobian product. Camera j has rotation vector
 * rotvec[3j..3j+3] (R = exp(rotvec)), translation t[3j..], intrinsics intr[3j..] = (f, k1, k2);
 * residual_i = f (1 + k1 r^2 + k2 r^4) n_i - pixel_i with n_i the normalized camera point.
 * Inadmissible observations produce NaN residuals and zero gradients. An observation whose camera
 * index is >= camera_count or point index >= point_count (a negative int32 index reads as a large
 * uint32) reads no camera or point: the forward writes a NaN residual for it, and the VJP then writes
 * NaN into every gradient output of the call.
 * The VJP accumulates into grad_* (caller zeroes them): for each input the adjoint sum over
 * observations of J^T grad_residual, in a fixed order (deterministic run to run).
 * Pointers are DEVICE pointers; stream is a cudaStream_t (NULL = legacy default stream).
 */
int32_t omvgba_residual_forward_f32(void* stream, uint64_t observation_count, const uint32_t* camera_index,
                                    const uint32_t* point_index, const float* pixel, uint64_t camera_count,
                                    const float* rotvec, const float* translation, const float* intrinsics,
                                    uint64_t point_count, const float* points, float* residual,
                                    omvgba_error* error);
int32_t omvgba_residual_vjp_f32(void* stream, uint64_t observation_count, const uint32_t* camera_index,
                                const uint32_t* point_index, const float* pixel, uint64_t camera_count,
                                const float* rotvec, const float* translation, const float* intrinsics,
                                uint64_t point_count, const float* points, const float* grad_residual,
                                float* grad_rotvec, float* grad_translation, float* grad_intrinsics,
                                float* grad_points, void* workspace, uint64_t workspace_bytes,
                                omvgba_error* error);
/* Bytes of device workspace omvgba_residual_vjp_f32 needs for these sizes. */
uint64_t omvgba_residual_vjp_workspace_bytes(uint64_t observation_count, uint64_t camera_count,
                                             uint64_t point_count);
int32_t omvgba_residual_forward_f64(void* stream, uint64_t observation_count, const uint32_t* camera_index,
                                    const uint32_t* point_index, const double* pixel, uint64_t camera_count,
                                    const double* rotvec, const double* translation, const double* intrinsics,
                                    uint64_t point_count, const double* points, double* residual,
                                    omvgba_error* error);

/*
 * omvgba_residual_vjp_f32 for callers that cannot allocate device memory: hosts whose GPU memory
 * is reserved up front by another allocator, or loops that allow no driver allocation (nor the
 * synchronisation a cudaMalloc / cudaFree may cause) after start-up. No counterpart in the
 * reference. The scratch is a static device array of OMVGBA_RESIDUAL_STATIC_SCRATCH_BYTES that
 * every GPU loading this library holds until exit; sizes whose omvgba_residual_vjp_workspace_bytes
 * exceed it (about 440,000 points with 3,000 cameras) are rejected with OMVGBA_INVALID_ARGUMENT
 * before any device work. It allocates nothing itself, but CUDA loads the library's modules
 * lazily by default: the first call on a device loads the module that holds the array, which is
 * when the driver reserves its 16 MiB. Callers that allow no driver allocation after start-up make
 * one warm-up call at start-up (or run with CUDA_MODULE_LOADING=EAGER). Every call resolves the
 * array's device address on the current device with cudaGetSymbolAddress (no allocation), so make
 * the first call before any stream capture.
 * Runs on the current device; arguments and results as omvgba_residual_vjp_f32. All calls share the
 * one array: calls that overlap on the GPU race, so order them on one stream.
 */
#define OMVGBA_RESIDUAL_STATIC_SCRATCH_BYTES (16u * 1024u * 1024u)
int32_t omvgba_residual_vjp_f32_static(void* stream, uint64_t observation_count, const uint32_t* camera_index,
                                       const uint32_t* point_index, const float* pixel, uint64_t camera_count,
                                       const float* rotvec, const float* translation, const float* intrinsics,
                                       uint64_t point_count, const float* points, const float* grad_residual,
                                       float* grad_rotvec, float* grad_translation, float* grad_intrinsics,
                                       float* grad_points, omvgba_error* error);

/*
 * Many independent problems (local-BA windows) in one call: solutions[i] receives window i, which is
 * solved exactly as omvgba_solve would solve it alone (so each window carries its own status and
 * convergence reason in its report). The windows run concurrently on a pool of host workers (16,
 * or the OMVGBA_BATCH_WORKERS environment variable), each with its own stream on the context's
 * device; config->stream is not used. Returns OMVGBA_OK
 * when every window succeeded, else the code of the lowest-numbered failing window with its index in
 * error->detail (the other windows' solutions are still written). No reference counterpart: the
 * reference solves one problem per call (crates/openmvg-ba/src/solver.rs:1562).
 */
int32_t omvgba_solve_batched(omvgba_context* context, uint64_t window_count, const omvgba_problem* windows,
                             const omvgba_config* config, omvgba_solution* solutions, omvgba_error* error);

/*
 * Observability probe of a translation-and-structure problem with fixed rotations
 * (probe_fixed_rotation_observability, kernel/fixed_rotation/observability.rs:24-262; the problem,
 * options and outcome of kernel/fixed_rotation/api.rs). A capped subset of tracks (shortest first,
 * covering every free camera) is linearized, each point is eliminated in square-root form, and the
 * camera system, scaled to unit diagonal and shifted by minimum_normalized_eigenvalue, must factor:
 * FULL_RANK_CERTIFIED certifies the whole problem; any other status is not evidence of deficiency.
 * Track selection and the per-point elimination run on the host (bounded by the options: at most
 * max_observations observations); the factorization runs on the context's device.
 */
typedef struct omvgba_fixed_rotation_problem {
  uint64_t camera_count;               /* >= 2 */
  const double* rotations;             /* camera_count x 9, world-to-camera, row-major */
  const double* centers;               /* camera_count x 3 */
  const double* intrinsics;            /* camera_count x 9: fx, fy, cx, cy, k1, k2, k3, p1, p2 */
  const uint8_t* fixed_cameras;        /* camera_count */
  uint64_t point_count;                /* >= 1 */
  const double* points;                /* point_count x 3 */
  const uint64_t* track_offsets;       /* point_count + 1: each point's observations */
  const uint32_t* observation_camera;  /* track_offsets[point_count] */
  const double* observation_pixel;     /* track_offsets[point_count] x 2 */
  int32_t gauge_kind;                  /* omvgba_gauge_kind: Free or FixedBaseline */
  uint64_t anchor, scale_camera;
  double distance;                     /* FixedBaseline: the baseline length */
  int32_t loss_kind;                   /* omvgba_loss_kind; the weights are relative to the loss at 0 */
  double loss_scale;                   /* Huber delta / Cauchy scale of the numerics loss */
} omvgba_fixed_rotation_problem;

typedef struct omvgba_probe_options {  /* FixedRotationObservabilityProbeOptions (api.rs) */
  uint64_t max_tracks, max_observations, max_observations_per_track, max_coverage_observations_per_track;
  uint64_t max_reduced_nonzeros, max_factor_nonzeros, max_symbolic_dense_nonzeros;
  double minimum_normalized_eigenvalue;
} omvgba_probe_options;

enum omvgba_probe_status {
  OMVGBA_PROBE_FULL_RANK_CERTIFIED = 0,
  OMVGBA_PROBE_INSUFFICIENT_CAMERA_COVERAGE = 1,
  OMVGBA_PROBE_RESOURCE_LIMIT = 2,
  OMVGBA_PROBE_WEAK_POINT_GEOMETRY = 3,
  OMVGBA_PROBE_SPARSE_FACTORIZATION_FAILED = 4
};

typedef struct omvgba_probe_report {  /* FixedRotationObservabilityProbe (api.rs) */
  int32_t status;                     /* omvgba_probe_status */
  int32_t reserved;
  uint64_t pose_dimension, selected_tracks, selected_observations, covered_free_cameras, weak_point_count;
  uint64_t reduced_nonzeros;          /* stored lower-triangle entries of the camera system */
  uint64_t factor_nonzeros;           /* entries of the factor's profile (envelope) in coordinate order */
} omvgba_probe_report;

/* FixedRotationObservabilityProbeOptions::default. */
void omvgba_probe_options_default(omvgba_probe_options* options);

/* Invalid options: OMVGBA_INVALID_ARGUMENT; an inconsistent problem: OMVGBA_INVALID_PROBLEM
   (FixedRotationError, api.rs). A point a camera cannot project counts as weak. */
int32_t omvgba_probe_fixed_rotation(omvgba_context* context, const omvgba_fixed_rotation_problem* problem,
                                    const omvgba_probe_options* options, omvgba_probe_report* report,
                                    omvgba_error* error);

/* NativeBundleAdjuster::preflight (native/mod.rs:120-230): a problem whose observed free poses all
   move only their centres, with pixel residuals, no fixed point, an explicit scale camera and one
   camera model per pose, runs the probe on its prepared (rebased) frame; every other problem
   reports PROCEED with has_counts = 0. Errors of the preparation are returned as by omvgba_solve;
   a probe error is OMVGBA_NUMERICAL. */
enum omvgba_preflight_status {
  OMVGBA_PREFLIGHT_PROCEED = 0,
  OMVGBA_PREFLIGHT_INSUFFICIENT_CAMERA_COVERAGE = 1,
  OMVGBA_PREFLIGHT_RESOURCE_LIMIT = 2,
  OMVGBA_PREFLIGHT_WEAK_POINT_GEOMETRY = 3,
  OMVGBA_PREFLIGHT_OBSERVABILITY_NOT_CERTIFIED = 4
};
typedef struct omvgba_preflight {      /* NativePreflight (native/mod.rs:143-165) */
  int32_t status;                      /* omvgba_preflight_status */
  int32_t has_counts;                  /* 0: the probe did not run (the counts are None) */
  uint64_t pose_dimension, covered_free_pose_count, weak_point_count;
  int32_t dense_observability_escalation;
  int32_t reserved;
} omvgba_preflight;

int32_t omvgba_preflight_check(omvgba_context* context, const omvgba_problem* problem, const omvgba_config* config,
                               omvgba_preflight* preflight, omvgba_error* error);

/* ---- the SfM side of a bundle adjustment: refreshing the landmarks' reprojection errors ----------
 *
 * After openmvg-sfm commits a bundle adjustment it measures every supporting observation of every
 * active landmark again (refresh_landmark_reprojection_errors_for, crates/openmvg-sfm/src/ops/
 * reconstruction/bundle.rs:510-637): the observation's pixel-equivalent residual under the camera
 * residual policy with no limit (ops/reconstruction/residual.rs:37-90) -- the pixel distance of the
 * projection for pinhole and Brown-Conrady cameras, the bearing angle times the nominal pixels per
 * radian for fisheye and spherical ones -- is kept when it exists and is finite; the landmark's
 * reprojection error becomes the mean of the kept residuals in track order; a landmark with fewer
 * than two is rejected, one that lost some has its support pruned to the kept observations. */
#define OMVGBA_NO_POSE 0xFFFFFFFFu
typedef struct omvgba_landmark_tracks {
  uint64_t landmark_count;
  const double* points;            /* 3 per landmark, world frame */
  const uint8_t* active;           /* 1 for LandmarkStatus::Active; other landmarks are left as they are */
  const uint64_t* track_offset;    /* landmark_count + 1: each landmark's track observations below */
  const uint32_t* track_pose;      /* pose of the observing view, or OMVGBA_NO_POSE when it has none */
  const uint32_t* track_intrinsic; /* intrinsic of the observing view */
  const double* track_pixel;       /* 2 per track observation */
  const uint8_t* track_support;    /* 1 when the observation is in the landmark's support */
} omvgba_landmark_tracks;

typedef enum omvgba_refresh_update {
  OMVGBA_REFRESH_SKIPPED = 0,   /* not active: nothing changes */
  OMVGBA_REFRESH_REJECTED = 1,  /* fewer than two supporting residuals: LandmarkStatus::Rejected */
  OMVGBA_REFRESH_UNCHANGED = 2, /* every supporting residual kept: new reprojection error only */
  OMVGBA_REFRESH_PRUNED = 3     /* some dropped: new support and reprojection error */
} omvgba_refresh_update;

typedef struct omvgba_refresh_result {
  uint8_t* landmark_update;     /* landmark_count: omvgba_refresh_update */
  double* reprojection_error;   /* landmark_count: mean residual (pixels) of kept landmarks, else untouched */
  uint8_t* track_support;       /* track observations: the support after the refresh */
  uint64_t rejected_landmarks;  /* LandmarkSupportCleanupReport */
  uint64_t removed_observations;
} omvgba_refresh_result;

/* Refresh of refresh_landmark_reprojection_errors_for (bundle.rs:510-637) on the context's device:
 * one thread per landmark evaluates its track in order. Poses are world-to-camera rotations with
 * camera centres (as omvgba_pose); intrinsics as omvgba_intrinsic. Returns OMVGBA_INVALID_PROBLEM
 * for an index out of range or a fisheye or spherical camera without a positive finite pixel scale
 * (the residual policy's own error), before any device work. */
int32_t omvgba_sfm_refresh_reprojection(omvgba_context* context, uint64_t pose_count, const omvgba_pose* poses,
                                        uint64_t intrinsic_count, const omvgba_intrinsic* intrinsics,
                                        const omvgba_landmark_tracks* tracks, omvgba_refresh_result* result,
                                        omvgba_error* error);

/* ---- the SfM side of a bundle adjustment: building the problem from a reconstruction -----------
 *
 * prepare_bundle_adjustment_problem (crates/openmvg-sfm/src/ops/reconstruction/bundle.rs:707-989):
 * the poses of the registered views (ascending pose id; fixed when a fixed view maps to them, or by
 * the scope), the intrinsic groups those views use (ascending id; free focal and radial terms only
 * under self-calibration and never for fisheye or spherical cameras; certification waived for a
 * placeholder focal), the active landmarks not excluded (fixed when listed or under the poses-only
 * scope) and, landmark by landmark in track order, their supporting observations seen from a
 * registered view. The residuals are angular when any group is fisheye or spherical, and a pixel
 * loss scale is then converted with the mean angle one pixel subtends (canonical_robust_loss,
 * :1006-1032). Unlike the reference this works on flat tables, so the caller resolves view and
 * landmark ids to table rows, and one reconstruction component per problem is the caller's check. */
typedef enum omvgba_scope {
  OMVGBA_SCOPE_FULL = 0,                 /* poses and points */
  OMVGBA_SCOPE_POINTS_ONLY = 1,
  OMVGBA_SCOPE_POSES_ONLY = 2,
  OMVGBA_SCOPE_TRANSLATIONS_AND_POINTS = 3,
  OMVGBA_SCOPE_SELF_CALIBRATION = 4
} omvgba_scope;

typedef struct omvgba_sfm_workspace {
  uint64_t view_count;
  const uint32_t* view_pose;        /* pose row of each view, OMVGBA_NO_POSE when it is not registered */
  const uint32_t* view_intrinsic;   /* intrinsic row of each view */
  const uint32_t* view_size;        /* width, height of each view's image */
  uint64_t pose_count;
  const omvgba_pose* poses;         /* rotation and centre; variables are set by the preparation */
  uint64_t intrinsic_count;
  const omvgba_intrinsic* intrinsics;
  const uint8_t* intrinsic_guess;   /* 1 when the group's focal is a placeholder (IntrinsicPrior::Guess) */
  omvgba_landmark_tracks landmarks; /* track_pose holds the observing VIEW row here */
} omvgba_sfm_workspace;

typedef struct omvgba_sfm_prepare_config {
  int32_t scope;                    /* omvgba_scope */
  uint64_t fixed_view_count;
  const uint32_t* fixed_views;      /* view rows whose poses stay fixed */
  uint64_t fixed_landmark_count;
  const uint32_t* fixed_landmarks;  /* landmark rows held fixed */
  uint64_t excluded_landmark_count;
  const uint32_t* excluded_landmarks;
  int32_t loss_kind;                /* omvgba_loss_kind, scale and its space as in omvgba_problem */
  double loss_scale;
  int32_t loss_scale_space;
  int32_t gauge_kind;               /* omvgba_gauge_kind; the fixed baseline's ends are view rows */
  uint32_t gauge_first_view, gauge_second_view;
  double gauge_distance;
} omvgba_sfm_prepare_config;

typedef struct omvgba_sfm_prepared {
  omvgba_problem problem;           /* arrays caller-allocated with the counts of the sizing call */
  uint32_t* pose_rows;              /* pose_count: workspace pose row of each problem pose */
  uint32_t* intrinsic_rows;         /* intrinsic_count */
  uint32_t* landmark_rows;          /* point_count */
} omvgba_sfm_prepared;

/* Call once with prepared->problem's array pointers null to receive the counts (pose, intrinsic,
 * point and observation), allocate, then call again to fill. OMVGBA_INVALID_PROBLEM for a row out of
 * range, an intrinsic shared by images of different sizes, a missing fixed-baseline view or a loss
 * scale whose units cannot be converted; OMVGBA_INVALID_CONFIG for an invalid scope or loss. */
int32_t omvgba_sfm_prepare_problem(const omvgba_sfm_workspace* workspace, const omvgba_sfm_prepare_config* config,
                                   omvgba_sfm_prepared* prepared, omvgba_error* error);

#ifdef __cplusplus
}
#endif

#endif /* OMVGBA_BA_CUDA_H */
