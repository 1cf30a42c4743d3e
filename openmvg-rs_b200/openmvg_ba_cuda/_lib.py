"""Loader for the in-tree libomvgba_cuda.so. There is no fallback: if the library is missing the
import fails loudly, so a CPU or pure-Python path can never stand in for the GPU solver."""
from __future__ import annotations

import ctypes as C
import os

from . import abi

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libomvgba_cuda.so")
_lib = None


class NativeLibraryMissing(ImportError):
    pass


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise NativeLibraryMissing(
            f"{LIB_PATH} is not built; run `python openmvg-rs_b200/build.py` (nvcc, sm_100a) first")
    L = C.CDLL(LIB_PATH)
    L.omvgba_abi_version.restype = C.c_uint32
    L.omvgba_adjuster_name.restype = C.c_char_p
    L.omvgba_config_default.argtypes = [C.POINTER(abi.Config)]
    L.omvgba_struct_sizes.argtypes = [C.POINTER(C.c_uint64)]
    L.omvgba_context_create.argtypes = [C.c_int32, C.POINTER(abi.Error)]
    L.omvgba_context_create.restype = C.c_void_p
    L.omvgba_context_destroy.argtypes = [C.c_void_p]
    L.omvgba_solve.argtypes = [C.c_void_p, C.POINTER(abi.Problem), C.POINTER(abi.Config), C.POINTER(abi.Solution),
                               C.POINTER(abi.Error)]
    L.omvgba_solve.restype = C.c_int32
    dp = C.POINTER(C.c_double)
    L.omvgba_debug_linearize.argtypes = [C.c_void_p, C.POINTER(abi.Problem), C.POINTER(abi.Config), dp, dp, dp, dp,
                                         C.POINTER(C.c_uint64), C.POINTER(abi.Error)]
    L.omvgba_debug_linearize.restype = C.c_int32
    L.omvgba_debug_schur_product.argtypes = [C.c_void_p, C.POINTER(abi.Problem), C.POINTER(abi.Config), C.c_double,
                                             dp, dp, dp, C.POINTER(C.c_int32), C.POINTER(abi.Error)]
    L.omvgba_debug_schur_product.restype = C.c_int32
    L.omvgba_debug_setup_digest.argtypes = [C.POINTER(abi.Problem), C.POINTER(abi.Config), C.c_uint32,
                                             C.POINTER(C.c_uint64), C.POINTER(abi.Error)]
    L.omvgba_debug_setup_digest.restype = C.c_int32
    L.omvgba_debug_execution_plan.argtypes = [C.POINTER(abi.Problem), C.POINTER(abi.Config), C.POINTER(C.c_int32),
                                              C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(abi.Error)]
    L.omvgba_debug_execution_plan.restype = C.c_int32
    L.omvgba_solve_batched.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(abi.Problem), C.POINTER(abi.Config),
                                       C.POINTER(abi.Solution), C.POINTER(abi.Error)]
    L.omvgba_solve_batched.restype = C.c_int32
    L.omvgba_plan_create.argtypes = [C.c_void_p, C.POINTER(abi.Problem), C.POINTER(abi.Config),
                                     C.POINTER(C.c_void_p), C.POINTER(abi.Error)]
    L.omvgba_plan_create.restype = C.c_int32
    L.omvgba_plan_solve.argtypes = [C.c_void_p, C.POINTER(abi.Solution), C.POINTER(abi.Error)]
    L.omvgba_plan_solve.restype = C.c_int32
    L.omvgba_plan_info_get.argtypes = [C.c_void_p, C.POINTER(abi.PlanInfo), C.POINTER(abi.Error)]
    L.omvgba_plan_info_get.restype = C.c_int32
    L.omvgba_plan_schur_product.argtypes = [C.c_void_p, C.c_double, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                            C.POINTER(abi.Error)]
    L.omvgba_plan_schur_product.restype = C.c_int32
    L.omvgba_plan_destroy.argtypes = [C.c_void_p]
    L.omvgba_device_count.restype = C.c_int32
    L.omvgba_probe_options_default.argtypes = [C.POINTER(abi.ProbeOptions)]
    L.omvgba_probe_fixed_rotation.argtypes = [C.c_void_p, C.POINTER(abi.FixedRotationProblem),
                                              C.POINTER(abi.ProbeOptions), C.POINTER(abi.ProbeReport),
                                              C.POINTER(abi.Error)]
    L.omvgba_probe_fixed_rotation.restype = C.c_int32
    L.omvgba_preflight_check.argtypes = [C.c_void_p, C.POINTER(abi.Problem), C.POINTER(abi.Config),
                                         C.POINTER(abi.Preflight), C.POINTER(abi.Error)]
    L.omvgba_preflight_check.restype = C.c_int32
    L.omvgba_sfm_refresh_reprojection.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(abi.Pose), C.c_uint64,
                                                  C.POINTER(abi.Intrinsic), C.POINTER(abi.LandmarkTracks),
                                                  C.POINTER(abi.RefreshResult), C.POINTER(abi.Error)]
    L.omvgba_sfm_refresh_reprojection.restype = C.c_int32
    L.omvgba_sfm_prepare_problem.argtypes = [C.POINTER(abi.SfmWorkspace), C.POINTER(abi.SfmPrepareConfig),
                                             C.POINTER(abi.SfmPrepared), C.POINTER(abi.Error)]
    L.omvgba_sfm_prepare_problem.restype = C.c_int32
    vp, u64 = C.c_void_p, C.c_uint64
    L.omvgba_residual_forward_f32.argtypes = [vp, u64, vp, vp, vp, u64, vp, vp, vp, u64, vp, vp, C.POINTER(abi.Error)]
    L.omvgba_residual_forward_f32.restype = C.c_int32
    L.omvgba_residual_forward_f64.argtypes = [vp, u64, vp, vp, vp, u64, vp, vp, vp, u64, vp, vp, C.POINTER(abi.Error)]
    L.omvgba_residual_forward_f64.restype = C.c_int32
    L.omvgba_residual_vjp_f32.argtypes = [vp, u64, vp, vp, vp, u64, vp, vp, vp, u64, vp, vp, vp, vp, vp, vp, vp, u64,
                                          C.POINTER(abi.Error)]
    L.omvgba_residual_vjp_f32.restype = C.c_int32
    L.omvgba_residual_vjp_f32_static.argtypes = [vp, u64, vp, vp, vp, u64, vp, vp, vp, u64, vp, vp, vp, vp, vp, vp,
                                                 C.POINTER(abi.Error)]
    L.omvgba_residual_vjp_f32_static.restype = C.c_int32
    L.omvgba_residual_vjp_workspace_bytes.argtypes = [u64, u64, u64]
    L.omvgba_residual_vjp_workspace_bytes.restype = u64
    _lib = L
    return L


def struct_sizes() -> dict:
    out = (C.c_uint64 * 7)()
    lib().omvgba_struct_sizes(out)
    names = ["error", "pose", "intrinsic", "problem", "config", "report", "solution"]
    return dict(zip(names, list(out)))


def device_count() -> int:
    return int(lib().omvgba_device_count())
