"""ctypes mirror of ``include/ba_cuda.h`` and marshalling between numpy arrays and the C structs.

Every struct here must match the header byte for byte; ``tests/test_abi.py`` checks the sizes and
field offsets against the compiled library's own ``sizeof`` report.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

OMVGBA_OK = 0
OMVGBA_INVALID_CONFIG = 1
OMVGBA_UNSUPPORTED = 2
OMVGBA_RESOURCE_EXHAUSTED = 3
OMVGBA_NUMERICAL = 4
OMVGBA_INTERNAL = 5
OMVGBA_INVALID_PROBLEM = 6
OMVGBA_INVALID_ARGUMENT = 7
OMVGBA_CUDA_ERROR = 8

CAMERA_PINHOLE, CAMERA_BROWN_CONRADY, CAMERA_FISHEYE, CAMERA_SPHERICAL = 0, 1, 2, 3
RADIAL_NONE, RADIAL_K1, RADIAL_K1K2, RADIAL_K1K2K3, RADIAL_K1K2K3K4 = 0, 1, 2, 3, 4
TANGENTIAL_NONE, TANGENTIAL_P1, TANGENTIAL_P1P2 = 0, 1, 2
INTRINSIC_FOCAL, INTRINSIC_PRINCIPAL_POINT, INTRINSIC_RADIAL, INTRINSIC_TANGENTIAL = 1, 2, 4, 8
POSE_ROTATION, POSE_TRANSLATION = 1, 2
POSE_FREE = 3
RESIDUAL_PIXELS, RESIDUAL_ANGULAR = 0, 1
LOSS_SQUARED, LOSS_HUBER, LOSS_CAUCHY = 0, 1, 2
GAUGE_FREE, GAUGE_FIXED_BASELINE = 0, 1
SOLVER_AUTO, SOLVER_DIRECT, SOLVER_ITERATIVE = 0, 1, 2
PRECISION_FP64, PRECISION_MIXED = 0, 1
MATVEC_AUTO, MATVEC_EXPLICIT, MATVEC_IMPLICIT = 0, 1, 2
STATUS_CONVERGED, STATUS_MAX_ITERATIONS, STATUS_STALLED, STATUS_DEGENERATE, STATUS_SKIPPED = 0, 1, 2, 3, 4
REASON_NONE, REASON_OBJECTIVE, REASON_GRADIENT, REASON_STEP = -1, 0, 1, 2
OBS_FULL_RANK, OBS_ONLY_EXPECTED_GAUGE, OBS_RANK_DEFICIENT, OBS_NOT_ASSESSED = 0, 1, 2, 3


class Error(C.Structure):
    _fields_ = [("code", C.c_int32), ("detail", C.c_int32), ("message", C.c_char * 480)]


class Pose(C.Structure):
    _fields_ = [
        ("rotation", C.c_double * 9),
        ("center", C.c_double * 3),
        ("variables", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


class Intrinsic(C.Structure):
    _fields_ = [
        ("model", C.c_int32),
        ("radial_kind", C.c_int32),
        ("tangential_kind", C.c_int32),
        ("variables", C.c_uint32),
        ("certification", C.c_int32),
        ("fixed_model", C.c_int32),
        ("fx", C.c_double),
        ("fy", C.c_double),
        ("cx", C.c_double),
        ("cy", C.c_double),
        ("k1", C.c_double),
        ("k2", C.c_double),
        ("k3", C.c_double),
        ("p1", C.c_double),
        ("p2", C.c_double),
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("k4", C.c_double),
    ]


class Problem(C.Structure):
    _fields_ = [
        ("pose_count", C.c_uint64),
        ("poses", C.POINTER(Pose)),
        ("intrinsic_count", C.c_uint64),
        ("intrinsics", C.POINTER(Intrinsic)),
        ("point_count", C.c_uint64),
        ("points", C.POINTER(C.c_double)),
        ("point_fixed", C.POINTER(C.c_uint8)),
        ("observation_count", C.c_uint64),
        ("observation_pose", C.POINTER(C.c_uint32)),
        ("observation_intrinsic", C.POINTER(C.c_uint32)),
        ("observation_point", C.POINTER(C.c_uint32)),
        ("observation_pixel", C.POINTER(C.c_double)),
        ("residual_space", C.c_int32),
        ("loss_kind", C.c_int32),
        ("loss_scale", C.c_double),
        ("loss_scale_space", C.c_int32),
        ("gauge_kind", C.c_int32),
        ("gauge_first", C.c_uint64),
        ("gauge_second", C.c_uint64),
        ("gauge_distance", C.c_double),
    ]


class Config(C.Structure):
    _fields_ = [
        ("max_iterations", C.c_uint64),
        ("function_tolerance", C.c_double),
        ("gradient_tolerance", C.c_double),
        ("parameter_tolerance", C.c_double),
        ("linear_solver", C.c_int32),
        ("has_workspace_budget", C.c_int32),
        ("workspace_budget_bytes", C.c_uint64),
        ("precision", C.c_int32),
        ("matvec", C.c_int32),
        ("pcg_relative_tolerance", C.c_double),
        ("pcg_max_iterations", C.c_uint32),
        ("device", C.c_int32),
        ("stream", C.c_void_p),
    ]


class Report(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("convergence_reason", C.c_int32),
        ("iteration_count", C.c_uint64),
        ("initial_objective", C.c_double),
        ("final_objective", C.c_double),
        ("initial_rmse", C.c_double),
        ("final_rmse", C.c_double),
        ("accepted_step_count", C.c_uint64),
        ("rejected_step_count", C.c_uint64),
        ("rejected_linearization", C.c_uint64),
        ("rejected_step_solve", C.c_uint64),
        ("rejected_candidate", C.c_uint64),
        ("rejected_insufficient_reduction", C.c_uint64),
        ("has_stationarity", C.c_int32),
        ("scaled_gradient_inf_norm", C.c_double),
        ("observability", C.c_int32),
        ("has_weak_point_count", C.c_int32),
        ("weak_point_count", C.c_uint64),
        ("quarantined_point_count", C.c_uint64),
        ("has_noninvertible_observation_count", C.c_int32),
        ("noninvertible_observation_count", C.c_uint64),
        ("has_observability_details", C.c_int32),
        ("details_pose_rank", C.c_uint64),
        ("details_pose_dimension", C.c_uint64),
        ("details_weak_point_count", C.c_uint64),
        ("has_linear_solver", C.c_int32),
        ("linear_solver", C.c_int32),
        ("has_observation_count", C.c_int32),
        ("observation_count", C.c_uint64),
        ("has_inlier_count", C.c_int32),
        ("inlier_count", C.c_uint64),
        ("has_final_inlier_rmse", C.c_int32),
        ("final_inlier_rmse", C.c_double),
        ("unconstrained_intrinsic_count", C.c_uint64),
        ("pcg_iteration_count", C.c_uint64),
        ("reduced_dimension", C.c_uint64),
        ("final_damping", C.c_double),
        ("solve_seconds", C.c_double),
        ("upload_seconds", C.c_double),
        ("kernel_launches", C.c_uint64),
        ("h2d_bytes", C.c_uint64),
        ("d2h_bytes", C.c_uint64),
    ]


class Solution(C.Structure):
    _fields_ = [
        ("poses", C.POINTER(Pose)),
        ("intrinsics", C.POINTER(Intrinsic)),
        ("points", C.POINTER(C.c_double)),
        ("quarantined_points", C.POINTER(C.c_uint64)),
        ("unconstrained_intrinsics", C.POINTER(C.c_uint64)),
        ("report", Report),
    ]


def _ptr(array: np.ndarray, ctype):
    return array.ctypes.data_as(C.POINTER(ctype))


class MarshalledProblem:
    """Holds the numpy buffers a ``Problem`` struct points into, so they outlive the call."""

    def __init__(self, problem):
        n_poses = len(problem.rotations)
        self.poses = (Pose * n_poses)()
        rot = np.ascontiguousarray(problem.rotations, dtype=np.float64).reshape(n_poses, 9)
        cen = np.ascontiguousarray(problem.centers, dtype=np.float64).reshape(n_poses, 3)
        var = np.asarray(problem.pose_variables, dtype=np.uint32)
        raw = np.frombuffer(self.poses, dtype=np.uint8).reshape(n_poses, C.sizeof(Pose))
        view = raw.view(np.dtype([("rotation", "<f8", 9), ("center", "<f8", 3), ("variables", "<u4"), ("reserved", "<u4")]))
        view["rotation"][:, 0] = rot
        view["center"][:, 0] = cen
        view["variables"][:, 0] = var
        self.intrinsics = (Intrinsic * len(problem.intrinsics))()
        for i, intr in enumerate(problem.intrinsics):
            intr.fill(self.intrinsics[i])
        self.points = np.ascontiguousarray(problem.points, dtype=np.float64).reshape(-1)
        self.point_fixed = np.ascontiguousarray(problem.point_fixed, dtype=np.uint8)
        self.obs_pose = np.ascontiguousarray(problem.observation_pose, dtype=np.uint32)
        self.obs_intr = np.ascontiguousarray(problem.observation_intrinsic, dtype=np.uint32)
        self.obs_point = np.ascontiguousarray(problem.observation_point, dtype=np.uint32)
        self.obs_pixel = np.ascontiguousarray(problem.observation_pixel, dtype=np.float64).reshape(-1)
        s = Problem()
        s.pose_count = n_poses
        s.poses = C.cast(self.poses, C.POINTER(Pose))
        s.intrinsic_count = len(problem.intrinsics)
        s.intrinsics = C.cast(self.intrinsics, C.POINTER(Intrinsic))
        s.point_count = len(self.points) // 3
        s.points = _ptr(self.points, C.c_double)
        s.point_fixed = _ptr(self.point_fixed, C.c_uint8)
        s.observation_count = len(self.obs_pose)
        s.observation_pose = _ptr(self.obs_pose, C.c_uint32)
        s.observation_intrinsic = _ptr(self.obs_intr, C.c_uint32)
        s.observation_point = _ptr(self.obs_point, C.c_uint32)
        s.observation_pixel = _ptr(self.obs_pixel, C.c_double)
        s.residual_space = problem.residual_space
        loss = problem.robust_loss
        s.loss_kind = loss.kind
        s.loss_scale = loss.scale
        s.loss_scale_space = loss.space
        g = problem.gauge
        s.gauge_kind = g.kind
        s.gauge_first = g.first
        s.gauge_second = g.second
        s.gauge_distance = g.distance
        self.struct = s


class SolutionBuffers:
    """Caller-allocated output buffers of one solve."""

    def __init__(self, problem):
        n_poses = len(problem.rotations)
        self.poses = (Pose * n_poses)()
        self.intrinsics = (Intrinsic * len(problem.intrinsics))()
        n_points = int(np.asarray(problem.points).shape[0])
        self.points = np.zeros(n_points * 3, dtype=np.float64)
        self.quarantined = np.zeros(max(n_points, 1), dtype=np.uint64)
        self.unconstrained = np.zeros(max(len(problem.intrinsics), 1), dtype=np.uint64)
        s = Solution()
        s.poses = C.cast(self.poses, C.POINTER(Pose))
        s.intrinsics = C.cast(self.intrinsics, C.POINTER(Intrinsic))
        s.points = _ptr(self.points, C.c_double)
        s.quarantined_points = _ptr(self.quarantined, C.c_uint64)
        s.unconstrained_intrinsics = _ptr(self.unconstrained, C.c_uint64)
        self.struct = s

    def pose_arrays(self):
        n = len(self.poses)
        raw = np.frombuffer(self.poses, dtype=np.uint8).reshape(n, C.sizeof(Pose))
        view = raw.view(np.dtype([("rotation", "<f8", 9), ("center", "<f8", 3), ("variables", "<u4"), ("reserved", "<u4")]))
        return view["rotation"][:, 0].reshape(n, 3, 3).copy(), view["center"][:, 0].copy()


def report_to_dict(r: Report) -> dict:
    return {name: getattr(r, name) for name, _ in Report._fields_}


class PlanInfo(C.Structure):
    """omvgba_plan_info."""
    _fields_ = [
        ("observation_count", C.c_uint64),
        ("point_count", C.c_uint64),
        ("camera_count", C.c_uint64),
        ("reduced_dimension", C.c_uint64),
        ("jacobian_entries", C.c_uint64),
        ("tile_count_fp64", C.c_uint64),
        ("tile_count_fp32", C.c_uint64),
        ("record_bytes_fp64", C.c_uint64),
        ("record_bytes_fp32", C.c_uint64),
        ("metadata_bytes_fp64", C.c_uint64),
        ("metadata_bytes_fp32", C.c_uint64),
        ("iterative", C.c_int32),
        ("mixed", C.c_int32),
    ]

    def to_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class FixedRotationProblem(C.Structure):
    """omvgba_fixed_rotation_problem (kernel/fixed_rotation/api.rs FixedRotationProblem)."""
    _fields_ = [
        ("camera_count", C.c_uint64),
        ("rotations", C.POINTER(C.c_double)),
        ("centers", C.POINTER(C.c_double)),
        ("intrinsics", C.POINTER(C.c_double)),
        ("fixed_cameras", C.POINTER(C.c_uint8)),
        ("point_count", C.c_uint64),
        ("points", C.POINTER(C.c_double)),
        ("track_offsets", C.POINTER(C.c_uint64)),
        ("observation_camera", C.POINTER(C.c_uint32)),
        ("observation_pixel", C.POINTER(C.c_double)),
        ("gauge_kind", C.c_int32),
        ("anchor", C.c_uint64),
        ("scale_camera", C.c_uint64),
        ("distance", C.c_double),
        ("loss_kind", C.c_int32),
        ("loss_scale", C.c_double),
    ]


class ProbeOptions(C.Structure):
    """omvgba_probe_options (FixedRotationObservabilityProbeOptions)."""
    _fields_ = [
        ("max_tracks", C.c_uint64),
        ("max_observations", C.c_uint64),
        ("max_observations_per_track", C.c_uint64),
        ("max_coverage_observations_per_track", C.c_uint64),
        ("max_reduced_nonzeros", C.c_uint64),
        ("max_factor_nonzeros", C.c_uint64),
        ("max_symbolic_dense_nonzeros", C.c_uint64),
        ("minimum_normalized_eigenvalue", C.c_double),
    ]


class ProbeReport(C.Structure):
    """omvgba_probe_report (FixedRotationObservabilityProbe)."""
    _fields_ = [
        ("status", C.c_int32),
        ("reserved", C.c_int32),
        ("pose_dimension", C.c_uint64),
        ("selected_tracks", C.c_uint64),
        ("selected_observations", C.c_uint64),
        ("covered_free_cameras", C.c_uint64),
        ("weak_point_count", C.c_uint64),
        ("reduced_nonzeros", C.c_uint64),
        ("factor_nonzeros", C.c_uint64),
    ]

    def to_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved"}


class Preflight(C.Structure):
    """omvgba_preflight (NativePreflight)."""
    _fields_ = [
        ("status", C.c_int32),
        ("has_counts", C.c_int32),
        ("pose_dimension", C.c_uint64),
        ("covered_free_pose_count", C.c_uint64),
        ("weak_point_count", C.c_uint64),
        ("dense_observability_escalation", C.c_int32),
        ("reserved", C.c_int32),
    ]

    def to_dict(self) -> dict:
        d = {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved"}
        if not d["has_counts"]:  # None in the reference's NativePreflight
            d["pose_dimension"] = d["covered_free_pose_count"] = d["weak_point_count"] = None
        return d


PROBE_FULL_RANK_CERTIFIED, PROBE_INSUFFICIENT_CAMERA_COVERAGE, PROBE_RESOURCE_LIMIT = 0, 1, 2
PROBE_WEAK_POINT_GEOMETRY, PROBE_SPARSE_FACTORIZATION_FAILED = 3, 4
PREFLIGHT_PROCEED, PREFLIGHT_INSUFFICIENT_CAMERA_COVERAGE, PREFLIGHT_RESOURCE_LIMIT = 0, 1, 2
PREFLIGHT_WEAK_POINT_GEOMETRY, PREFLIGHT_OBSERVABILITY_NOT_CERTIFIED = 3, 4


# ---- the SfM-side reprojection-error refresh (omvgba_sfm_refresh_reprojection) ----
NO_POSE = 0xFFFFFFFF
REFRESH_SKIPPED, REFRESH_REJECTED, REFRESH_UNCHANGED, REFRESH_PRUNED = 0, 1, 2, 3


class LandmarkTracks(C.Structure):
    _fields_ = [
        ("landmark_count", C.c_uint64),
        ("points", C.POINTER(C.c_double)),
        ("active", C.POINTER(C.c_uint8)),
        ("track_offset", C.POINTER(C.c_uint64)),
        ("track_pose", C.POINTER(C.c_uint32)),
        ("track_intrinsic", C.POINTER(C.c_uint32)),
        ("track_pixel", C.POINTER(C.c_double)),
        ("track_support", C.POINTER(C.c_uint8)),
    ]


class RefreshResult(C.Structure):
    _fields_ = [
        ("landmark_update", C.POINTER(C.c_uint8)),
        ("reprojection_error", C.POINTER(C.c_double)),
        ("track_support", C.POINTER(C.c_uint8)),
        ("rejected_landmarks", C.c_uint64),
        ("removed_observations", C.c_uint64),
    ]


def marshal_poses(rotations, centers):
    """(Pose array, keep-alive) for world-to-camera rotations (n, 3, 3) and camera centres (n, 3)."""
    n = len(rotations)
    poses = (Pose * n)()
    raw = np.frombuffer(poses, dtype=np.uint8).reshape(n, C.sizeof(Pose)) if n else None
    if n:
        view = raw.view(np.dtype([("rotation", "<f8", 9), ("center", "<f8", 3), ("variables", "<u4"), ("reserved", "<u4")]))
        view["rotation"][:, 0] = np.ascontiguousarray(rotations, dtype=np.float64).reshape(n, 9)
        view["center"][:, 0] = np.ascontiguousarray(centers, dtype=np.float64).reshape(n, 3)
    return poses


# ---- building the problem from a reconstruction (omvgba_sfm_prepare_problem) ----
SCOPE_FULL, SCOPE_POINTS_ONLY, SCOPE_POSES_ONLY, SCOPE_TRANSLATIONS_AND_POINTS, SCOPE_SELF_CALIBRATION = 0, 1, 2, 3, 4


class SfmWorkspace(C.Structure):
    _fields_ = [
        ("view_count", C.c_uint64),
        ("view_pose", C.POINTER(C.c_uint32)),
        ("view_intrinsic", C.POINTER(C.c_uint32)),
        ("view_size", C.POINTER(C.c_uint32)),
        ("pose_count", C.c_uint64),
        ("poses", C.POINTER(Pose)),
        ("intrinsic_count", C.c_uint64),
        ("intrinsics", C.POINTER(Intrinsic)),
        ("intrinsic_guess", C.POINTER(C.c_uint8)),
        ("landmarks", LandmarkTracks),
    ]


class SfmPrepareConfig(C.Structure):
    _fields_ = [
        ("scope", C.c_int32),
        ("fixed_view_count", C.c_uint64),
        ("fixed_views", C.POINTER(C.c_uint32)),
        ("fixed_landmark_count", C.c_uint64),
        ("fixed_landmarks", C.POINTER(C.c_uint32)),
        ("excluded_landmark_count", C.c_uint64),
        ("excluded_landmarks", C.POINTER(C.c_uint32)),
        ("loss_kind", C.c_int32),
        ("loss_scale", C.c_double),
        ("loss_scale_space", C.c_int32),
        ("gauge_kind", C.c_int32),
        ("gauge_first_view", C.c_uint32),
        ("gauge_second_view", C.c_uint32),
        ("gauge_distance", C.c_double),
    ]


class SfmPrepared(C.Structure):
    _fields_ = [
        ("problem", Problem),
        ("pose_rows", C.POINTER(C.c_uint32)),
        ("intrinsic_rows", C.POINTER(C.c_uint32)),
        ("landmark_rows", C.POINTER(C.c_uint32)),
    ]
