//! Raw bindings of include/ba_cuda.h. Every struct is `#[repr(C)]` and mirrors the C declaration
//! field for field; `check_layout` compares the sizes with what the library was compiled with
//! (`omvgba_struct_sizes`) before the first solve.

#![allow(non_camel_case_types)]

use std::ffi::{c_char, c_void};

pub const OMVGBA_ABI_VERSION: u32 = 3;

// omvgba_code
pub const OMVGBA_OK: i32 = 0;
pub const OMVGBA_INVALID_CONFIG: i32 = 1;
pub const OMVGBA_UNSUPPORTED: i32 = 2;
pub const OMVGBA_RESOURCE_EXHAUSTED: i32 = 3;
pub const OMVGBA_NUMERICAL: i32 = 4;
pub const OMVGBA_INTERNAL: i32 = 5;
pub const OMVGBA_INVALID_PROBLEM: i32 = 6;
pub const OMVGBA_INVALID_ARGUMENT: i32 = 7;
pub const OMVGBA_CUDA_ERROR: i32 = 8;

// omvgba_camera_model, radial and tangential kinds
pub const OMVGBA_CAMERA_PINHOLE: i32 = 0;
pub const OMVGBA_CAMERA_BROWN_CONRADY: i32 = 1;
pub const OMVGBA_CAMERA_FISHEYE: i32 = 2;
pub const OMVGBA_CAMERA_SPHERICAL: i32 = 3;
pub const OMVGBA_RADIAL_NONE: i32 = 0;
pub const OMVGBA_RADIAL_K1: i32 = 1;
pub const OMVGBA_RADIAL_K1K2: i32 = 2;
pub const OMVGBA_RADIAL_K1K2K3: i32 = 3;
pub const OMVGBA_RADIAL_K1K2K3K4: i32 = 4;
pub const OMVGBA_TANGENTIAL_NONE: i32 = 0;
pub const OMVGBA_TANGENTIAL_P1: i32 = 1;
pub const OMVGBA_TANGENTIAL_P1P2: i32 = 2;

// variable bits
pub const OMVGBA_INTRINSIC_FOCAL: u32 = 1 << 0;
pub const OMVGBA_INTRINSIC_PRINCIPAL_POINT: u32 = 1 << 1;
pub const OMVGBA_INTRINSIC_RADIAL: u32 = 1 << 2;
pub const OMVGBA_INTRINSIC_TANGENTIAL: u32 = 1 << 3;
pub const OMVGBA_POSE_ROTATION: u32 = 1 << 0;
pub const OMVGBA_POSE_TRANSLATION: u32 = 1 << 1;

// residual space, loss, gauge, solver, precision
pub const OMVGBA_RESIDUAL_PIXELS: i32 = 0;
pub const OMVGBA_RESIDUAL_ANGULAR: i32 = 1;
pub const OMVGBA_LOSS_SQUARED: i32 = 0;
pub const OMVGBA_LOSS_HUBER: i32 = 1;
pub const OMVGBA_LOSS_CAUCHY: i32 = 2;
pub const OMVGBA_GAUGE_FREE: i32 = 0;
pub const OMVGBA_GAUGE_FIXED_BASELINE: i32 = 1;
pub const OMVGBA_SOLVER_AUTO: i32 = 0;
pub const OMVGBA_SOLVER_DIRECT: i32 = 1;
pub const OMVGBA_SOLVER_ITERATIVE: i32 = 2;
pub const OMVGBA_PRECISION_FP64: i32 = 0;
pub const OMVGBA_PRECISION_MIXED: i32 = 1;

// omvgba_solve_status, omvgba_convergence_reason, omvgba_observability
pub const OMVGBA_STATUS_CONVERGED: i32 = 0;
pub const OMVGBA_STATUS_MAX_ITERATIONS: i32 = 1;
pub const OMVGBA_STATUS_STALLED: i32 = 2;
pub const OMVGBA_STATUS_DEGENERATE: i32 = 3;
pub const OMVGBA_STATUS_SKIPPED: i32 = 4;
pub const OMVGBA_REASON_NONE: i32 = -1;
pub const OMVGBA_REASON_OBJECTIVE: i32 = 0;
pub const OMVGBA_REASON_GRADIENT: i32 = 1;
pub const OMVGBA_REASON_STEP: i32 = 2;
pub const OMVGBA_OBS_FULL_RANK: i32 = 0;
pub const OMVGBA_OBS_ONLY_EXPECTED_GAUGE: i32 = 1;
pub const OMVGBA_OBS_RANK_DEFICIENT: i32 = 2;
pub const OMVGBA_OBS_NOT_ASSESSED: i32 = 3;

#[repr(C)]
pub struct omvgba_error {
    pub code: i32,
    pub detail: i32,
    pub message: [c_char; 480],
}

impl omvgba_error {
    pub fn zeroed() -> Self {
        Self { code: 0, detail: -1, message: [0; 480] }
    }

    /// The UTF-8 message (lossy), up to the first NUL.
    pub fn text(&self) -> String {
        let bytes: Vec<u8> = self.message.iter().take_while(|&&c| c != 0).map(|&c| c as u8).collect();
        String::from_utf8_lossy(&bytes).into_owned()
    }
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct omvgba_pose {
    pub rotation: [f64; 9],
    pub center: [f64; 3],
    pub variables: u32,
    pub reserved: u32,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct omvgba_intrinsic {
    pub model: i32,
    pub radial_kind: i32,
    pub tangential_kind: i32,
    pub variables: u32,
    pub certification: i32,
    pub fixed_model: i32,
    pub fx: f64,
    pub fy: f64,
    pub cx: f64,
    pub cy: f64,
    pub k1: f64,
    pub k2: f64,
    pub k3: f64,
    pub p1: f64,
    pub p2: f64,
    pub width: u32,
    pub height: u32,
    pub k4: f64,
}

#[repr(C)]
pub struct omvgba_problem {
    pub pose_count: u64,
    pub poses: *const omvgba_pose,
    pub intrinsic_count: u64,
    pub intrinsics: *const omvgba_intrinsic,
    pub point_count: u64,
    pub points: *const f64,
    pub point_fixed: *const u8,
    pub observation_count: u64,
    pub observation_pose: *const u32,
    pub observation_intrinsic: *const u32,
    pub observation_point: *const u32,
    pub observation_pixel: *const f64,
    pub residual_space: i32,
    pub loss_kind: i32,
    pub loss_scale: f64,
    pub loss_scale_space: i32,
    pub gauge_kind: i32,
    pub gauge_first: u64,
    pub gauge_second: u64,
    pub gauge_distance: f64,
}

#[repr(C)]
pub struct omvgba_config {
    pub max_iterations: u64,
    pub function_tolerance: f64,
    pub gradient_tolerance: f64,
    pub parameter_tolerance: f64,
    pub linear_solver: i32,
    pub has_workspace_budget: i32,
    pub workspace_budget_bytes: u64,
    pub precision: i32,
    pub matvec: i32,
    pub pcg_relative_tolerance: f64,
    pub pcg_max_iterations: u32,
    pub device: i32,
    pub stream: *mut c_void,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct omvgba_report {
    pub status: i32,
    pub convergence_reason: i32,
    pub iteration_count: u64,
    pub initial_objective: f64,
    pub final_objective: f64,
    pub initial_rmse: f64,
    pub final_rmse: f64,
    pub accepted_step_count: u64,
    pub rejected_step_count: u64,
    pub rejected_linearization: u64,
    pub rejected_step_solve: u64,
    pub rejected_candidate: u64,
    pub rejected_insufficient_reduction: u64,
    pub has_stationarity: i32,
    pub scaled_gradient_inf_norm: f64,
    pub observability: i32,
    pub has_weak_point_count: i32,
    pub weak_point_count: u64,
    pub quarantined_point_count: u64,
    pub has_noninvertible_observation_count: i32,
    pub noninvertible_observation_count: u64,
    pub has_observability_details: i32,
    pub details_pose_rank: u64,
    pub details_pose_dimension: u64,
    pub details_weak_point_count: u64,
    pub has_linear_solver: i32,
    pub linear_solver: i32,
    pub has_observation_count: i32,
    pub observation_count: u64,
    pub has_inlier_count: i32,
    pub inlier_count: u64,
    pub has_final_inlier_rmse: i32,
    pub final_inlier_rmse: f64,
    pub unconstrained_intrinsic_count: u64,
    pub pcg_iteration_count: u64,
    pub reduced_dimension: u64,
    pub final_damping: f64,
    pub solve_seconds: f64,
    pub upload_seconds: f64,
    pub kernel_launches: u64,
    pub h2d_bytes: u64,
    pub d2h_bytes: u64,
}

#[repr(C)]
pub struct omvgba_solution {
    pub poses: *mut omvgba_pose,
    pub intrinsics: *mut omvgba_intrinsic,
    pub points: *mut f64,
    pub quarantined_points: *mut u64,
    pub unconstrained_intrinsics: *mut u64,
    pub report: omvgba_report,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct omvgba_preflight {
    pub status: i32,
    pub has_counts: i32,
    pub pose_dimension: u64,
    pub covered_free_pose_count: u64,
    pub weak_point_count: u64,
    pub dense_observability_escalation: i32,
    pub reserved: i32,
}

// omvgba_preflight_status
pub const OMVGBA_PREFLIGHT_PROCEED: i32 = 0;
pub const OMVGBA_PREFLIGHT_INSUFFICIENT_CAMERA_COVERAGE: i32 = 1;
pub const OMVGBA_PREFLIGHT_RESOURCE_LIMIT: i32 = 2;
pub const OMVGBA_PREFLIGHT_WEAK_POINT_GEOMETRY: i32 = 3;
pub const OMVGBA_PREFLIGHT_OBSERVABILITY_NOT_CERTIFIED: i32 = 4;

// ---- the SfM side of a bundle adjustment (openmvg-sfm ops/reconstruction/bundle.rs) ----
pub const OMVGBA_NO_POSE: u32 = 0xFFFF_FFFF;

#[repr(C)]
#[derive(Clone, Copy)]
pub struct omvgba_landmark_tracks {
    pub landmark_count: u64,
    pub points: *const f64,
    pub active: *const u8,
    pub track_offset: *const u64,
    pub track_pose: *const u32,
    pub track_intrinsic: *const u32,
    pub track_pixel: *const f64,
    pub track_support: *const u8,
}

// omvgba_refresh_update
pub const OMVGBA_REFRESH_SKIPPED: u8 = 0;
pub const OMVGBA_REFRESH_REJECTED: u8 = 1;
pub const OMVGBA_REFRESH_UNCHANGED: u8 = 2;
pub const OMVGBA_REFRESH_PRUNED: u8 = 3;

#[repr(C)]
pub struct omvgba_refresh_result {
    pub landmark_update: *mut u8,
    pub reprojection_error: *mut f64,
    pub track_support: *mut u8,
    pub rejected_landmarks: u64,
    pub removed_observations: u64,
}

// omvgba_scope
pub const OMVGBA_SCOPE_FULL: i32 = 0;
pub const OMVGBA_SCOPE_POINTS_ONLY: i32 = 1;
pub const OMVGBA_SCOPE_POSES_ONLY: i32 = 2;
pub const OMVGBA_SCOPE_TRANSLATIONS_AND_POINTS: i32 = 3;
pub const OMVGBA_SCOPE_SELF_CALIBRATION: i32 = 4;

#[repr(C)]
pub struct omvgba_sfm_workspace {
    pub view_count: u64,
    pub view_pose: *const u32,
    pub view_intrinsic: *const u32,
    pub view_size: *const u32,
    pub pose_count: u64,
    pub poses: *const omvgba_pose,
    pub intrinsic_count: u64,
    pub intrinsics: *const omvgba_intrinsic,
    pub intrinsic_guess: *const u8,
    pub landmarks: omvgba_landmark_tracks,
}

#[repr(C)]
pub struct omvgba_sfm_prepare_config {
    pub scope: i32,
    pub fixed_view_count: u64,
    pub fixed_views: *const u32,
    pub fixed_landmark_count: u64,
    pub fixed_landmarks: *const u32,
    pub excluded_landmark_count: u64,
    pub excluded_landmarks: *const u32,
    pub loss_kind: i32,
    pub loss_scale: f64,
    pub loss_scale_space: i32,
    pub gauge_kind: i32,
    pub gauge_first_view: u32,
    pub gauge_second_view: u32,
    pub gauge_distance: f64,
}

#[repr(C)]
pub struct omvgba_sfm_prepared {
    pub problem: omvgba_problem,
    pub pose_rows: *mut u32,
    pub intrinsic_rows: *mut u32,
    pub landmark_rows: *mut u32,
}

/// Opaque per-thread solver context.
#[repr(C)]
pub struct omvgba_context {
    _private: [u8; 0],
}

unsafe extern "C" {
    pub fn omvgba_abi_version() -> u32;
    pub fn omvgba_struct_sizes(out: *mut u64);
    pub fn omvgba_device_count() -> i32;
    pub fn omvgba_adjuster_name() -> *const c_char;
    pub fn omvgba_config_default(config: *mut omvgba_config);
    pub fn omvgba_context_create(device: i32, error: *mut omvgba_error) -> *mut omvgba_context;
    pub fn omvgba_context_destroy(context: *mut omvgba_context);
    pub fn omvgba_solve(
        context: *mut omvgba_context,
        problem: *const omvgba_problem,
        config: *const omvgba_config,
        solution: *mut omvgba_solution,
        error: *mut omvgba_error,
    ) -> i32;
    pub fn omvgba_preflight_check(
        context: *mut omvgba_context,
        problem: *const omvgba_problem,
        config: *const omvgba_config,
        preflight: *mut omvgba_preflight,
        error: *mut omvgba_error,
    ) -> i32;
    pub fn omvgba_sfm_prepare_problem(
        workspace: *const omvgba_sfm_workspace,
        config: *const omvgba_sfm_prepare_config,
        prepared: *mut omvgba_sfm_prepared,
        error: *mut omvgba_error,
    ) -> i32;
    pub fn omvgba_sfm_refresh_reprojection(
        context: *mut omvgba_context,
        pose_count: u64,
        poses: *const omvgba_pose,
        intrinsic_count: u64,
        intrinsics: *const omvgba_intrinsic,
        tracks: *const omvgba_landmark_tracks,
        result: *mut omvgba_refresh_result,
        error: *mut omvgba_error,
    ) -> i32;
}

/// Sizes of the ABI structs in the order `omvgba_struct_sizes` reports them.
pub fn rust_struct_sizes() -> [u64; 7] {
    use std::mem::size_of;
    [
        size_of::<omvgba_error>() as u64,
        size_of::<omvgba_pose>() as u64,
        size_of::<omvgba_intrinsic>() as u64,
        size_of::<omvgba_problem>() as u64,
        size_of::<omvgba_config>() as u64,
        size_of::<omvgba_report>() as u64,
        size_of::<omvgba_solution>() as u64,
    ]
}

/// Compares the Rust struct layout with the library's; false on any mismatch.
pub fn check_layout() -> bool {
    let mut sizes = [0u64; 16];
    // SAFETY: the library writes seven sizes into a buffer of sixteen.
    unsafe { omvgba_struct_sizes(sizes.as_mut_ptr()) };
    // SAFETY: a plain call without arguments.
    let version = unsafe { omvgba_abi_version() };
    version == OMVGBA_ABI_VERSION && sizes[..7] == rust_struct_sizes()
}
