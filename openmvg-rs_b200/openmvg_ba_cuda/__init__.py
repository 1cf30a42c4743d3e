"""openmvg_ba_cuda — B200-native bundle adjustment behind openmvg-ba's BundleAdjuster contract."""
from . import abi
from .problem import (BundleProblem, CameraIntrinsics, Gauge, RobustLoss, Solution, SolveConfig, SolveError,
                      InvalidConfig, Unsupported, ResourceExhausted, Numerical, Internal, ProblemError, CudaError)

__all__ = ["abi", "BundleProblem", "CameraIntrinsics", "Gauge", "RobustLoss", "Solution", "SolveConfig",
           "SolveError", "InvalidConfig", "Unsupported", "ResourceExhausted", "Numerical", "Internal",
           "ProblemError", "CudaError"]
