//! `CudaBundleAdjuster`: openmvg-ba's [`BundleAdjuster`] on a B200 GPU, through the C ABI of
//! libomvgba_cuda.so (include/ba_cuda.h).
//!
//! This crate holds all of the workspace's `unsafe` code for the GPU solver: the library crates
//! (openmvg-ba, openmvg-sfm, openmvg-core) keep `#![forbid(unsafe_code)]`. A solve copies the
//! borrowed [`BundleProblem`] into structure-of-arrays buffers, calls `omvgba_solve` with
//! caller-allocated outputs of the problem's shapes, maps the return code onto [`SolveError`]
//! (`solver.rs:1474-1493`) and rebuilds the [`Solution`] through
//! `Solution::try_new_with_quarantined_points` (`solver.rs:829-876`), so the same shape,
//! fixed-block, mask and baseline checks that guard the native adjuster guard this one. Problems the
//! GPU solver does not take (angular residuals, partial pose masks) come back as
//! `SolveError::Unsupported`, which the contract defines as "hand the problem to another adjuster
//! unchanged".
//!
//! Not compiled in this repository (no Rust toolchain in its build environment); written against
//! `crates/openmvg-ba/src/{problem.rs,solver.rs}` and `crates/openmvg-core/src/{camera,model}` of
//! openmvg-rs as read.

pub mod ffi;

use std::ptr;

use nalgebra::{Matrix3, Point3};
use openmvg_ba::{
    BundleAdjuster, BundleIntrinsic, BundleProblem, ConvergenceReason, Gauge, IntrinsicCertification,
    LinearSolver, Observability, ObservabilityDiagnostics, ResidualSpace, RobustLoss, Solution, SolveConfig,
    SolveDiagnostics, SolveError, SolveReport, SolveStatus, StationarityAudit, StepRejections,
};
use openmvg_core::camera::{Camera, FisheyeDistortion, RadialDistortion, TangentialDistortion};
use openmvg_core::model::{CameraIntrinsics, WorldToCameraPose};

/// Execution options of the GPU solver that `SolveConfig` does not carry.
#[derive(Clone, Copy, Debug)]
pub struct CudaOptions {
    /// `ffi::OMVGBA_PRECISION_FP64` or `ffi::OMVGBA_PRECISION_MIXED`.
    pub precision: i32,
    /// PCG forcing tolerance; 0 keeps the native default (1e-1, native/mod.rs:596-603).
    pub pcg_relative_tolerance: f64,
    /// PCG iteration cap; 0 keeps 600 (sparse/api.rs:395).
    pub pcg_max_iterations: u32,
}

impl Default for CudaOptions {
    fn default() -> Self {
        Self { precision: ffi::OMVGBA_PRECISION_FP64, pcg_relative_tolerance: 0.0, pcg_max_iterations: 0 }
    }
}

/// `NativePreflightStatus` (crates/openmvg-ba/src/native/mod.rs:120-141).
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub enum CudaPreflightStatus {
    Proceed,
    InsufficientCameraCoverage,
    ResourceLimit,
    WeakPointGeometry,
    ObservabilityNotCertified,
}

/// `NativePreflight` (crates/openmvg-ba/src/native/mod.rs:143-165); the counts are `None` when the
/// check did not run.
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub struct CudaPreflight {
    pub status: CudaPreflightStatus,
    pub pose_dimension: Option<usize>,
    pub covered_free_pose_count: Option<usize>,
    pub weak_point_count: Option<usize>,
    pub dense_observability_escalation: bool,
}

/// One solver context on one CUDA device. `Send` but not `Sync`: the context is used through
/// `&mut self` only, one solve at a time, as the trait requires.
pub struct CudaBundleAdjuster {
    context: *mut ffi::omvgba_context,
    device: i32,
    options: CudaOptions,
}

// SAFETY: the context is owned by this value and only touched through `&mut self`; the library
// keeps no thread-affine state in it (every call makes its device current).
unsafe impl Send for CudaBundleAdjuster {}

impl CudaBundleAdjuster {
    /// A context on `device`. Fails when the library's struct layout differs from this crate's or
    /// the device cannot be initialised.
    pub fn new(device: i32, options: CudaOptions) -> Result<Self, SolveError> {
        if !ffi::check_layout() {
            return Err(SolveError::Internal(
                "libomvgba_cuda ABI version or struct layout differs from openmvg-ba-cuda".to_owned(),
            ));
        }
        let mut error = ffi::omvgba_error::zeroed();
        // SAFETY: `error` is a valid out-pointer for the duration of the call.
        let context = unsafe { ffi::omvgba_context_create(device, &mut error) };
        if context.is_null() {
            return Err(SolveError::Internal(format!("CUDA context on device {device}: {}", error.text())));
        }
        Ok(Self { context, device, options })
    }

    /// The translation-only observability check openmvg-sfm runs before a bundle adjustment of
    /// camera positions with fixed rotations (`NativeBundleAdjuster::preflight`,
    /// crates/openmvg-ba/src/native/mod.rs:184-230). `NativePreflight` cannot be built outside
    /// openmvg-ba, so the outcome comes back as this crate's `CudaPreflight` with the same fields.
    pub fn preflight(&mut self, problem: &BundleProblem, config: &SolveConfig) -> Result<CudaPreflight, SolveError> {
        config.validate()?;
        let marshalled = marshal(problem)?;
        let view = problem_view(problem, &marshalled);
        let cfg = config_view(config, self.device, &self.options);
        // SAFETY: an all-zero preflight is a valid value of this plain C struct; the call overwrites it.
        let mut out: ffi::omvgba_preflight = unsafe { std::mem::zeroed() };
        let mut error = ffi::omvgba_error::zeroed();
        // SAFETY: `view` points into `marshalled`, which outlives the call; `out` and `error` are
        // valid out-pointers; the context is ours.
        let code = unsafe { ffi::omvgba_preflight_check(self.context, &view, &cfg, &mut out, &mut error) };
        if code != ffi::OMVGBA_OK {
            return Err(to_solve_error(code, &error));
        }
        let count = |value: u64| (out.has_counts != 0).then_some(value as usize);
        Ok(CudaPreflight {
            status: match out.status {
                ffi::OMVGBA_PREFLIGHT_PROCEED => CudaPreflightStatus::Proceed,
                ffi::OMVGBA_PREFLIGHT_INSUFFICIENT_CAMERA_COVERAGE => CudaPreflightStatus::InsufficientCameraCoverage,
                ffi::OMVGBA_PREFLIGHT_RESOURCE_LIMIT => CudaPreflightStatus::ResourceLimit,
                ffi::OMVGBA_PREFLIGHT_WEAK_POINT_GEOMETRY => CudaPreflightStatus::WeakPointGeometry,
                _ => CudaPreflightStatus::ObservabilityNotCertified,
            },
            pose_dimension: count(out.pose_dimension),
            covered_free_pose_count: count(out.covered_free_pose_count),
            weak_point_count: count(out.weak_point_count),
            dense_observability_escalation: out.dense_observability_escalation != 0,
        })
    }

    /// CUDA devices visible to this process.
    pub fn device_count() -> usize {
        // SAFETY: a plain call without arguments.
        usize::try_from(unsafe { ffi::omvgba_device_count() }).unwrap_or(0)
    }
}

impl Drop for CudaBundleAdjuster {
    fn drop(&mut self) {
        // SAFETY: the context came from omvgba_context_create and is destroyed once.
        unsafe { ffi::omvgba_context_destroy(self.context) };
    }
}

/// The problem as the C ABI's structure of arrays; the vectors own the storage the raw view
/// points into, so they live as long as the view.
struct Marshalled {
    poses: Vec<ffi::omvgba_pose>,
    intrinsics: Vec<ffi::omvgba_intrinsic>,
    points: Vec<f64>,
    point_fixed: Vec<u8>,
    observation_pose: Vec<u32>,
    observation_intrinsic: Vec<u32>,
    observation_point: Vec<u32>,
    observation_pixel: Vec<f64>,
}

fn index_u32(index: usize) -> Result<u32, SolveError> {
    u32::try_from(index)
        .map_err(|_| SolveError::Unsupported("an index exceeds the 32-bit range of the GPU solver".to_owned()))
}

fn intrinsic_to_ffi(block: &BundleIntrinsic) -> ffi::omvgba_intrinsic {
    let data = block.intrinsics();
    let (width, height) = data.dimensions();
    let variables = block.variables();
    let principal = data.camera().principal_point();
    let mut out = ffi::omvgba_intrinsic {
        model: ffi::OMVGBA_CAMERA_PINHOLE,
        radial_kind: ffi::OMVGBA_RADIAL_NONE,
        tangential_kind: ffi::OMVGBA_TANGENTIAL_NONE,
        variables: (u32::from(variables.focal()) * ffi::OMVGBA_INTRINSIC_FOCAL)
            | (u32::from(variables.principal_point()) * ffi::OMVGBA_INTRINSIC_PRINCIPAL_POINT)
            | (u32::from(variables.radial()) * ffi::OMVGBA_INTRINSIC_RADIAL)
            | (u32::from(variables.tangential()) * ffi::OMVGBA_INTRINSIC_TANGENTIAL),
        certification: i32::from(block.certification() == IntrinsicCertification::Waived),
        fixed_model: i32::from(data.is_fixed()),
        fx: 0.0,
        fy: 0.0,
        cx: principal.x,
        cy: principal.y,
        k1: 0.0,
        k2: 0.0,
        k3: 0.0,
        p1: 0.0,
        p2: 0.0,
        width,
        height,
        k4: 0.0,
    };
    match data.camera() {
        Camera::Pinhole(camera) => {
            out.fx = camera.focal_x();
            out.fy = camera.focal_y();
        }
        Camera::BrownConrady(camera) => {
            out.model = ffi::OMVGBA_CAMERA_BROWN_CONRADY;
            out.fx = camera.focal_x();
            out.fy = camera.focal_y();
            match *camera.radial_distortion() {
                RadialDistortion::None => {}
                RadialDistortion::K1(k1) => {
                    out.radial_kind = ffi::OMVGBA_RADIAL_K1;
                    out.k1 = k1;
                }
                RadialDistortion::K1K2(k1, k2) => {
                    out.radial_kind = ffi::OMVGBA_RADIAL_K1K2;
                    (out.k1, out.k2) = (k1, k2);
                }
                RadialDistortion::K1K2K3(k1, k2, k3) => {
                    out.radial_kind = ffi::OMVGBA_RADIAL_K1K2K3;
                    (out.k1, out.k2, out.k3) = (k1, k2, k3);
                }
            }
            match *camera.tangential_distortion() {
                TangentialDistortion::None => {}
                TangentialDistortion::P1(p1) => {
                    out.tangential_kind = ffi::OMVGBA_TANGENTIAL_P1;
                    out.p1 = p1;
                }
                TangentialDistortion::P1P2(p1, p2) => {
                    out.tangential_kind = ffi::OMVGBA_TANGENTIAL_P1P2;
                    (out.p1, out.p2) = (p1, p2);
                }
            }
        }
        // wide-angle models serve angular residuals (their bearings); the GPU solver answers
        // Unsupported for them in pixel residuals
        Camera::Fisheye(camera) => {
            out.model = ffi::OMVGBA_CAMERA_FISHEYE;
            out.fx = camera.focal_x();
            out.fy = camera.focal_y();
            match *camera.fisheye_distortion() {
                FisheyeDistortion::None => {}
                FisheyeDistortion::K1(k1) => {
                    out.radial_kind = ffi::OMVGBA_RADIAL_K1;
                    out.k1 = k1;
                }
                FisheyeDistortion::K1K2(k1, k2) => {
                    out.radial_kind = ffi::OMVGBA_RADIAL_K1K2;
                    (out.k1, out.k2) = (k1, k2);
                }
                FisheyeDistortion::K1K2K3(k1, k2, k3) => {
                    out.radial_kind = ffi::OMVGBA_RADIAL_K1K2K3;
                    (out.k1, out.k2, out.k3) = (k1, k2, k3);
                }
                FisheyeDistortion::K1K2K3K4(k1, k2, k3, k4) => {
                    out.radial_kind = ffi::OMVGBA_RADIAL_K1K2K3K4;
                    (out.k1, out.k2, out.k3, out.k4) = (k1, k2, k3, k4);
                }
            }
        }
        Camera::Spherical(_) => out.model = ffi::OMVGBA_CAMERA_SPHERICAL,
    }
    out
}

fn marshal(problem: &BundleProblem) -> Result<Marshalled, SolveError> {
    let poses = problem
        .poses()
        .iter()
        .map(|block| {
            let r = block.pose().rotation_matrix();
            let c = block.pose().center();
            let v = block.variables();
            ffi::omvgba_pose {
                rotation: [r[(0, 0)], r[(0, 1)], r[(0, 2)], r[(1, 0)], r[(1, 1)], r[(1, 2)], r[(2, 0)], r[(2, 1)], r[(2, 2)]],
                center: [c.x, c.y, c.z],
                variables: (u32::from(v.rotation()) * ffi::OMVGBA_POSE_ROTATION)
                    | (u32::from(v.translation()) * ffi::OMVGBA_POSE_TRANSLATION),
                reserved: 0,
            }
        })
        .collect();
    let intrinsics = problem.intrinsics().iter().map(intrinsic_to_ffi).collect();
    let mut points = Vec::with_capacity(3 * problem.points().len());
    let mut point_fixed = Vec::with_capacity(problem.points().len());
    for point in problem.points() {
        let p = point.position();
        points.extend_from_slice(&[p.x, p.y, p.z]);
        point_fixed.push(u8::from(point.is_fixed()));
    }
    let n = problem.observations().len();
    let (mut observation_pose, mut observation_intrinsic, mut observation_point) =
        (Vec::with_capacity(n), Vec::with_capacity(n), Vec::with_capacity(n));
    let mut observation_pixel = Vec::with_capacity(2 * n);
    for observation in problem.observations() {
        observation_pose.push(index_u32(observation.pose())?);
        observation_intrinsic.push(index_u32(observation.intrinsic())?);
        observation_point.push(index_u32(observation.point())?);
        observation_pixel.extend_from_slice(&[observation.pixel().x, observation.pixel().y]);
    }
    Ok(Marshalled {
        poses,
        intrinsics,
        points,
        point_fixed,
        observation_pose,
        observation_intrinsic,
        observation_point,
        observation_pixel,
    })
}

fn residual_space_code(space: ResidualSpace) -> i32 {
    match space {
        ResidualSpace::Angular => ffi::OMVGBA_RESIDUAL_ANGULAR,
        _ => ffi::OMVGBA_RESIDUAL_PIXELS,
    }
}

fn problem_view(problem: &BundleProblem, m: &Marshalled) -> ffi::omvgba_problem {
    let (loss_kind, loss_scale, loss_scale_space) = match problem.robust_loss() {
        RobustLoss::Huber(scale) => (ffi::OMVGBA_LOSS_HUBER, scale.value(), residual_space_code(scale.space())),
        RobustLoss::Cauchy(scale) => (ffi::OMVGBA_LOSS_CAUCHY, scale.value(), residual_space_code(scale.space())),
        _ => (ffi::OMVGBA_LOSS_SQUARED, 0.0, ffi::OMVGBA_RESIDUAL_PIXELS),
    };
    let (gauge_kind, gauge_first, gauge_second, gauge_distance) = match problem.gauge() {
        Gauge::FixedBaseline { first, second, distance } => {
            (ffi::OMVGBA_GAUGE_FIXED_BASELINE, first as u64, second as u64, distance)
        }
        _ => (ffi::OMVGBA_GAUGE_FREE, 0, 0, 0.0),
    };
    ffi::omvgba_problem {
        pose_count: m.poses.len() as u64,
        poses: m.poses.as_ptr(),
        intrinsic_count: m.intrinsics.len() as u64,
        intrinsics: m.intrinsics.as_ptr(),
        point_count: m.point_fixed.len() as u64,
        points: m.points.as_ptr(),
        point_fixed: m.point_fixed.as_ptr(),
        observation_count: m.observation_pose.len() as u64,
        observation_pose: m.observation_pose.as_ptr(),
        observation_intrinsic: m.observation_intrinsic.as_ptr(),
        observation_point: m.observation_point.as_ptr(),
        observation_pixel: m.observation_pixel.as_ptr(),
        residual_space: residual_space_code(problem.residual_space()),
        loss_kind,
        loss_scale,
        loss_scale_space,
        gauge_kind,
        gauge_first,
        gauge_second,
        gauge_distance,
    }
}

fn config_view(config: &SolveConfig, device: i32, options: &CudaOptions) -> ffi::omvgba_config {
    let mut out = ffi::omvgba_config {
        max_iterations: 0,
        function_tolerance: 0.0,
        gradient_tolerance: 0.0,
        parameter_tolerance: 0.0,
        linear_solver: 0,
        has_workspace_budget: 0,
        workspace_budget_bytes: 0,
        precision: 0,
        matvec: 0,
        pcg_relative_tolerance: 0.0,
        pcg_max_iterations: 0,
        device: 0,
        stream: ptr::null_mut(),
    };
    // SAFETY: `out` is a valid, writable config.
    unsafe { ffi::omvgba_config_default(&mut out) };
    out.max_iterations = config.max_iterations() as u64;
    out.function_tolerance = config.function_tolerance();
    out.gradient_tolerance = config.gradient_tolerance();
    out.parameter_tolerance = config.parameter_tolerance();
    out.linear_solver = match config.linear_solver() {
        LinearSolver::Direct => ffi::OMVGBA_SOLVER_DIRECT,
        LinearSolver::Iterative => ffi::OMVGBA_SOLVER_ITERATIVE,
        _ => ffi::OMVGBA_SOLVER_AUTO,
    };
    if let Some(budget) = config.workspace_budget_bytes() {
        out.has_workspace_budget = 1;
        out.workspace_budget_bytes = u64::try_from(budget).unwrap_or(u64::MAX);
    }
    out.precision = options.precision;
    out.pcg_relative_tolerance = options.pcg_relative_tolerance;
    out.pcg_max_iterations = options.pcg_max_iterations;
    out.device = device;
    out
}

fn to_solve_error(code: i32, error: &ffi::omvgba_error) -> SolveError {
    let text = error.text();
    match code {
        ffi::OMVGBA_INVALID_CONFIG => SolveError::InvalidConfig(invalid_config_message(&text)),
        ffi::OMVGBA_UNSUPPORTED => SolveError::Unsupported(text),
        ffi::OMVGBA_RESOURCE_EXHAUSTED => SolveError::ResourceExhausted(text),
        ffi::OMVGBA_NUMERICAL => SolveError::Numerical(text),
        _ => SolveError::Internal(text),
    }
}

/// `SolveError::InvalidConfig` carries a `&'static str`; the library's messages for it restate the
/// fixed texts of `SolveConfig::validate` (solver.rs:122-141).
fn invalid_config_message(text: &str) -> &'static str {
    const KNOWN: [&str; 5] = [
        "max_iterations must be positive",
        "function_tolerance must be finite and non-negative",
        "gradient_tolerance must be finite and non-negative",
        "parameter_tolerance must be finite and non-negative",
        "workspace_budget_bytes must be positive",
    ];
    KNOWN.iter().copied().find(|known| text.contains(known)).unwrap_or("invalid solve configuration")
}

fn pose_from_ffi(p: &ffi::omvgba_pose) -> Result<WorldToCameraPose, SolveError> {
    WorldToCameraPose::from_matrix(Matrix3::from_row_slice(&p.rotation), Point3::new(p.center[0], p.center[1], p.center[2]))
        .map_err(|e| SolveError::Internal(format!("GPU solver returned an invalid pose: {e}")))
}

/// The refined intrinsics: blocks the solve cannot change keep the input's own values; a
/// self-calibrated block gets its refined focal length and radial terms.
fn intrinsic_from_ffi(input: &BundleIntrinsic, out: &ffi::omvgba_intrinsic) -> Result<CameraIntrinsics, SolveError> {
    let data = input.intrinsics();
    if input.variables().is_fixed() {
        return Ok(data.clone());
    }
    let (width, height) = data.dimensions();
    let camera = match out.model {
        ffi::OMVGBA_CAMERA_PINHOLE => Camera::try_pinhole(out.fx, out.fy, out.cx, out.cy),
        ffi::OMVGBA_CAMERA_BROWN_CONRADY => {
            let radial = match out.radial_kind {
                ffi::OMVGBA_RADIAL_K1 => RadialDistortion::K1(out.k1),
                ffi::OMVGBA_RADIAL_K1K2 => RadialDistortion::K1K2(out.k1, out.k2),
                ffi::OMVGBA_RADIAL_K1K2K3 => RadialDistortion::K1K2K3(out.k1, out.k2, out.k3),
                _ => RadialDistortion::None,
            };
            let tangential = match out.tangential_kind {
                ffi::OMVGBA_TANGENTIAL_P1 => TangentialDistortion::P1(out.p1),
                ffi::OMVGBA_TANGENTIAL_P1P2 => TangentialDistortion::P1P2(out.p1, out.p2),
                _ => TangentialDistortion::None,
            };
            Camera::try_brown_conrady(out.fx, out.fy, out.cx, out.cy, radial, tangential)
        }
        _ => return Ok(data.clone()),
    }
    .map_err(|e| SolveError::Internal(format!("GPU solver returned an invalid camera: {e}")))?;
    CameraIntrinsics::try_new(camera, width, height)
        .map_err(|e| SolveError::Internal(format!("GPU solver returned invalid intrinsics: {e}")))
}

fn report_from_ffi(r: &ffi::omvgba_report, unconstrained: Vec<usize>) -> Result<SolveReport, SolveError> {
    let internal = |what: &str| SolveError::Internal(format!("GPU solver report: {what}"));
    let status = match r.status {
        ffi::OMVGBA_STATUS_CONVERGED => SolveStatus::Converged(match r.convergence_reason {
            ffi::OMVGBA_REASON_GRADIENT => ConvergenceReason::Gradient,
            ffi::OMVGBA_REASON_STEP => ConvergenceReason::Step,
            _ => ConvergenceReason::Objective,
        }),
        ffi::OMVGBA_STATUS_MAX_ITERATIONS => SolveStatus::MaxIterations,
        ffi::OMVGBA_STATUS_STALLED => SolveStatus::Stalled,
        ffi::OMVGBA_STATUS_DEGENERATE => SolveStatus::Degenerate,
        _ => SolveStatus::Skipped,
    };
    let observability = match r.observability {
        ffi::OMVGBA_OBS_FULL_RANK => Observability::FullRank,
        ffi::OMVGBA_OBS_ONLY_EXPECTED_GAUGE => Observability::OnlyExpectedGauge,
        ffi::OMVGBA_OBS_RANK_DEFICIENT => Observability::RankDeficient,
        _ => Observability::NotAssessed,
    };
    let stationarity = StationarityAudit::try_from_fresh_zero_damping(r.scaled_gradient_inf_norm)
        .map_err(|_| internal("non-finite stationarity audit"))?;
    let mut diagnostics = SolveDiagnostics::new(
        r.accepted_step_count as usize,
        r.rejected_step_count as usize,
        stationarity,
        observability,
        r.weak_point_count as usize,
        r.noninvertible_observation_count as usize,
    )
    .with_step_rejections(StepRejections {
        linearization: r.rejected_linearization as usize,
        step_solve: r.rejected_step_solve as usize,
        candidate: r.rejected_candidate as usize,
        insufficient_reduction: r.rejected_insufficient_reduction as usize,
    })
    .with_quarantined_point_count(r.quarantined_point_count as usize);
    if r.has_observability_details != 0 {
        let details = ObservabilityDiagnostics::try_new(
            r.details_pose_rank as usize,
            r.details_pose_dimension as usize,
            r.details_weak_point_count as usize,
        )
        .map_err(|_| internal("invalid observability details"))?;
        diagnostics = diagnostics.with_observability_details(details);
    }
    if r.has_linear_solver != 0 {
        diagnostics = diagnostics.with_linear_solver(match r.linear_solver {
            ffi::OMVGBA_SOLVER_DIRECT => LinearSolver::Direct,
            ffi::OMVGBA_SOLVER_ITERATIVE => LinearSolver::Iterative,
            _ => LinearSolver::Auto,
        });
    }
    SolveReport::try_new(
        status,
        r.iteration_count as usize,
        r.initial_objective,
        r.final_objective,
        r.initial_rmse,
        r.final_rmse,
        diagnostics,
    )
    .map(|report| report.with_unconstrained_intrinsics(unconstrained))
    .map_err(|_| internal("non-finite or inconsistent report"))
}

impl BundleAdjuster for CudaBundleAdjuster {
    fn name(&self) -> &'static str {
        "openmvg-ba-cuda-b200"
    }

    fn solve(&mut self, problem: &BundleProblem, config: SolveConfig) -> Result<Solution, SolveError> {
        config.validate()?;
        let marshalled = marshal(problem)?;
        let view = problem_view(problem, &marshalled);
        let cfg = config_view(&config, self.device, &self.options);
        let mut poses = marshalled.poses.clone();
        let mut intrinsics = marshalled.intrinsics.clone();
        let mut points = vec![0.0; marshalled.points.len()];
        let mut quarantined = vec![0u64; problem.points().len().max(1)];
        let mut unconstrained = vec![0u64; problem.intrinsics().len().max(1)];
        let mut solution = ffi::omvgba_solution {
            poses: poses.as_mut_ptr(),
            intrinsics: intrinsics.as_mut_ptr(),
            points: points.as_mut_ptr(),
            quarantined_points: quarantined.as_mut_ptr(),
            unconstrained_intrinsics: unconstrained.as_mut_ptr(),
            // SAFETY: an all-zero report is a valid value of this plain C struct; the call overwrites it.
            report: unsafe { std::mem::zeroed() },
        };
        let mut error = ffi::omvgba_error::zeroed();
        // SAFETY: every pointer in `view` and `solution` refers to live buffers of the shapes the
        // header requires (the problem's counts), which outlive the call; the context is ours.
        let code = unsafe { ffi::omvgba_solve(self.context, &view, &cfg, &mut solution, &mut error) };
        if code != ffi::OMVGBA_OK {
            return Err(to_solve_error(code, &error));
        }
        let report = &solution.report;
        let poses = poses.iter().map(pose_from_ffi).collect::<Result<Vec<_>, _>>()?;
        let intrinsics = problem
            .intrinsics()
            .iter()
            .zip(&intrinsics)
            .map(|(input, out)| intrinsic_from_ffi(input, out))
            .collect::<Result<Vec<_>, _>>()?;
        let points = points.chunks_exact(3).map(|p| Point3::new(p[0], p[1], p[2])).collect();
        let held = unconstrained[..report.unconstrained_intrinsic_count as usize].iter().map(|&g| g as usize).collect();
        let quarantined = quarantined[..report.quarantined_point_count as usize].iter().map(|&p| p as usize).collect();
        let report = report_from_ffi(report, held)?;
        Solution::try_new_with_quarantined_points(problem, poses, intrinsics, points, report, quarantined)
            .map_err(|e| SolveError::Internal(format!("GPU solution failed the solution checks: {e}")))
    }
}
