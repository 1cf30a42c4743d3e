"""Python mirror of openmvg-ba's problem / config / solution contract.

Names and meanings follow ``crates/openmvg-ba/src/problem.rs`` (``BundleProblem``, ``BundlePose``,
``BundleIntrinsic``, ``RobustLoss``, ``Gauge``) and ``crates/openmvg-ba/src/solver.rs``
(``SolveConfig``, ``SolveReport``, ``Solution``, ``SolveError``), stored as numpy arrays so that a
problem with millions of observations marshals into the C ABI without per-element Python work.
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field

import numpy as np

from . import abi


# ---- errors: SolveError (solver.rs:1474-1493) and ProblemError (problem.rs:731) -----------------
class SolveError(Exception):
    code = abi.OMVGBA_INTERNAL


class InvalidConfig(SolveError):
    code = abi.OMVGBA_INVALID_CONFIG


class Unsupported(SolveError):
    """The adjuster declines the problem; hand it unchanged to another adjuster."""

    code = abi.OMVGBA_UNSUPPORTED


class ResourceExhausted(SolveError):
    code = abi.OMVGBA_RESOURCE_EXHAUSTED


class Numerical(SolveError):
    code = abi.OMVGBA_NUMERICAL


class Internal(SolveError):
    code = abi.OMVGBA_INTERNAL


class ProblemError(SolveError):
    code = abi.OMVGBA_INVALID_PROBLEM


class CudaError(Internal):
    code = abi.OMVGBA_CUDA_ERROR


_ERRORS = {
    abi.OMVGBA_INVALID_CONFIG: InvalidConfig,
    abi.OMVGBA_UNSUPPORTED: Unsupported,
    abi.OMVGBA_RESOURCE_EXHAUSTED: ResourceExhausted,
    abi.OMVGBA_NUMERICAL: Numerical,
    abi.OMVGBA_INTERNAL: Internal,
    abi.OMVGBA_INVALID_PROBLEM: ProblemError,
    abi.OMVGBA_INVALID_ARGUMENT: ValueError,
    abi.OMVGBA_CUDA_ERROR: CudaError,
}


def raise_for(code: int, error: abi.Error) -> None:
    if code == abi.OMVGBA_OK:
        return
    cls = _ERRORS.get(code, Internal)
    raise cls(error.message.decode("utf-8", "replace"))


# ---- problem contract -------------------------------------------------------------------------
@dataclass
class CameraIntrinsics:
    """``BundleIntrinsic``: camera model, variable mask and certification (problem.rs:98-176)."""

    model: int = abi.CAMERA_PINHOLE
    fx: float = 1.0
    fy: float = 1.0
    cx: float = 0.0
    cy: float = 0.0
    radial_kind: int = abi.RADIAL_NONE
    k1: float = 0.0
    k2: float = 0.0
    k3: float = 0.0
    tangential_kind: int = abi.TANGENTIAL_NONE
    p1: float = 0.0
    p2: float = 0.0
    width: int = 640
    height: int = 480
    k4: float = 0.0  # fisheye K1K2K3K4 only
    variables: int = 0
    certification: int = 0
    fixed_model: int = 0

    def fill(self, s: abi.Intrinsic) -> None:
        for name in ("model", "radial_kind", "tangential_kind", "variables", "certification", "fixed_model",
                     "fx", "fy", "cx", "cy", "k1", "k2", "k3", "p1", "p2", "width", "height", "k4"):
            setattr(s, name, getattr(self, name))

    @classmethod
    def from_struct(cls, s: abi.Intrinsic) -> "CameraIntrinsics":
        return cls(**{f.name: getattr(s, f.name) for f in dataclasses.fields(cls)})


@dataclass(frozen=True)
class RobustLoss:
    """``RobustLoss`` (problem.rs:267-300): Squared, Huber(scale) or Cauchy(scale)."""

    kind: int = abi.LOSS_SQUARED
    scale: float = 0.0
    space: int = abi.RESIDUAL_PIXELS

    @classmethod
    def squared(cls):
        return cls()

    @classmethod
    def huber(cls, pixels: float):
        return cls(abi.LOSS_HUBER, float(pixels), abi.RESIDUAL_PIXELS)

    @classmethod
    def cauchy(cls, pixels: float):
        return cls(abi.LOSS_CAUCHY, float(pixels), abi.RESIDUAL_PIXELS)


@dataclass(frozen=True)
class Gauge:
    """``Gauge`` (problem.rs:302-312): Free or FixedBaseline {first, second, distance}."""

    kind: int = abi.GAUGE_FREE
    first: int = 0
    second: int = 0
    distance: float = 0.0

    @classmethod
    def fixed_baseline(cls, first: int, second: int, distance: float):
        return cls(abi.GAUGE_FIXED_BASELINE, int(first), int(second), float(distance))


@dataclass
class BundleProblem:
    """``BundleProblem`` (problem.rs:447-577) in structure-of-arrays form.

    rotations: (n_poses, 3, 3) world-to-camera rotations; centers: (n_poses, 3) camera centres;
    pose_variables: (n_poses,) ``POSE_*`` bits; points: (n_points, 3); point_fixed: (n_points,);
    observation_pose / _intrinsic / _point: (n_obs,) indices; observation_pixel: (n_obs, 2).
    """

    rotations: np.ndarray
    centers: np.ndarray
    pose_variables: np.ndarray
    intrinsics: list
    points: np.ndarray
    point_fixed: np.ndarray
    observation_pose: np.ndarray
    observation_intrinsic: np.ndarray
    observation_point: np.ndarray
    observation_pixel: np.ndarray
    residual_space: int = abi.RESIDUAL_PIXELS
    robust_loss: RobustLoss = field(default_factory=RobustLoss)
    gauge: Gauge = field(default_factory=Gauge)

    @property
    def observation_count(self) -> int:
        return int(len(self.observation_pose))

    @property
    def point_count(self) -> int:
        return int(np.asarray(self.points).shape[0])

    @property
    def pose_count(self) -> int:
        return int(np.asarray(self.rotations).shape[0])


@dataclass
class SolveConfig:
    """``SolveConfig`` (solver.rs:74-155) plus build-private execution options."""

    max_iterations: int = 50
    function_tolerance: float = 1.0e-6
    gradient_tolerance: float = 1.0e-10
    parameter_tolerance: float = 1.0e-8
    linear_solver: int = abi.SOLVER_AUTO
    workspace_budget_bytes: int | None = None
    precision: int = abi.PRECISION_FP64
    matvec: int = abi.MATVEC_AUTO
    pcg_relative_tolerance: float = 0.0
    pcg_max_iterations: int = 0
    device: int = 0
    stream: int = 0  # cudaStream_t handle (e.g. torch.cuda.current_stream().cuda_stream); 0: the context's

    def with_(self, **kwargs) -> "SolveConfig":
        return dataclasses.replace(self, **kwargs)

    def to_struct(self) -> abi.Config:
        c = abi.Config()
        c.max_iterations = self.max_iterations
        c.function_tolerance = self.function_tolerance
        c.gradient_tolerance = self.gradient_tolerance
        c.parameter_tolerance = self.parameter_tolerance
        c.linear_solver = self.linear_solver
        c.has_workspace_budget = 0 if self.workspace_budget_bytes is None else 1
        c.workspace_budget_bytes = 0 if self.workspace_budget_bytes is None else int(self.workspace_budget_bytes)
        c.precision = self.precision
        c.matvec = self.matvec
        c.pcg_relative_tolerance = self.pcg_relative_tolerance
        c.pcg_max_iterations = self.pcg_max_iterations
        c.device = self.device
        c.stream = self.stream or None
        return c


@dataclass
class Solution:
    """``Solution`` (solver.rs:788-1314): refined state, report and quarantined points."""

    rotations: np.ndarray
    centers: np.ndarray
    intrinsics: list
    points: np.ndarray
    quarantined_points: np.ndarray
    report: dict
    unconstrained_intrinsics: np.ndarray = None  # groups the self-calibration certificate held

    @classmethod
    def from_buffers(cls, buffers: abi.SolutionBuffers) -> "Solution":
        rot, cen = buffers.pose_arrays()
        report = abi.report_to_dict(buffers.struct.report)
        q = buffers.quarantined[: report["quarantined_point_count"]].copy()
        u = buffers.unconstrained[: report["unconstrained_intrinsic_count"]].copy()
        return cls(
            rotations=rot,
            centers=cen,
            intrinsics=[CameraIntrinsics.from_struct(s) for s in buffers.intrinsics],
            points=buffers.points.reshape(-1, 3).copy(),
            quarantined_points=q,
            report=report,
            unconstrained_intrinsics=u,
        )
