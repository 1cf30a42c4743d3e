"""TEST INFRASTRUCTURE ONLY: ctypes loader for the CPU oracle (oracle/_build/liboracle.so).

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference legs as the checker.
The shipped solver never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
_lib = None


def build() -> None:
    subprocess.run(["make", "-C", HERE], check=True, capture_output=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        from openmvg_ba_cuda import abi
        L = C.CDLL(LIB_PATH)
        L.omvgba_oracle_solve.argtypes = [C.POINTER(abi.Problem), C.POINTER(abi.Config), C.POINTER(abi.Solution),
                                          C.POINTER(abi.Error)]
        L.omvgba_oracle_solve.restype = C.c_int32
        dp = C.POINTER(C.c_double)
        L.omvgba_oracle_debug_linearize.argtypes = [C.POINTER(abi.Problem), C.POINTER(abi.Config), dp, dp, dp, dp,
                                                    C.POINTER(C.c_uint64), C.POINTER(abi.Error)]
        L.omvgba_oracle_debug_linearize.restype = C.c_int32
        L.omvgba_oracle_set_threads.argtypes = [C.c_int]
        L.omvgba_oracle_set_shards.argtypes = [C.c_int]
        L.omvgba_oracle_set_certificate.argtypes = [C.c_int]
        L.omvgba_oracle_execution_plan.argtypes = [C.POINTER(abi.Problem), C.POINTER(abi.Config),
                                                   C.POINTER(C.c_int32), C.POINTER(C.c_uint64),
                                                   C.POINTER(C.c_uint64), C.POINTER(abi.Error)]
        L.omvgba_oracle_execution_plan.restype = C.c_int32
        L.omvgba_oracle_iteration_seconds.argtypes = [C.POINTER(C.c_double), C.c_int]
        L.omvgba_oracle_iteration_seconds.restype = C.c_int
        L.omvgba_oracle_max_threads.restype = C.c_int
        L.omvgba_oracle_loss_cost.argtypes = [C.c_int, C.c_double, C.c_double]
        L.omvgba_oracle_loss_cost.restype = C.c_double
        L.omvgba_oracle_loss_sqrt_weight.argtypes = [C.c_int, C.c_double, C.c_double]
        L.omvgba_oracle_loss_sqrt_weight.restype = C.c_double
        L.omvgba_oracle_radial_linearize.argtypes = [C.c_double, C.c_double, C.c_double, dp, dp, dp]
        L.omvgba_oracle_radial_linearize.restype = C.c_int
        L.omvgba_oracle_bc_project.argtypes = [C.POINTER(abi.Intrinsic), dp, dp]
        L.omvgba_oracle_bc_project.restype = C.c_int
        L.omvgba_oracle_camera_bearing.argtypes = [C.POINTER(abi.Intrinsic), C.c_double, C.c_double, dp]
        L.omvgba_oracle_camera_bearing.restype = C.c_int
        L.omvgba_oracle_angular_projection.argtypes = [dp, dp, dp]
        L.omvgba_oracle_angular_projection.restype = C.c_int
        L.omvgba_oracle_bc_remove_distortion.argtypes = [C.POINTER(abi.Intrinsic), C.c_double, C.c_double, dp]
        L.omvgba_oracle_bc_remove_distortion.restype = C.c_int
        ip = C.POINTER(C.c_int)
        L.omvgba_oracle_nielsen.argtypes = [C.c_int, ip, dp, dp, C.c_double, dp, ip, dp, ip]
        L.omvgba_oracle_exp_so3.argtypes = [dp, dp]
        L.omvgba_oracle_point_block_inverse.argtypes = [dp, C.c_double, dp, dp]
        L.omvgba_oracle_point_block_inverse.restype = C.c_int
        L.omvgba_oracle_stages.argtypes = [C.c_int, C.c_uint64, C.POINTER(C.c_uint64), ip]
        L.omvgba_oracle_preflight.argtypes = [C.POINTER(abi.Problem), C.POINTER(abi.Config), C.POINTER(abi.Preflight),
                                              C.POINTER(abi.Error)]
        L.omvgba_oracle_preflight.restype = C.c_int
        L.omvgba_oracle_probe_fixed_rotation.argtypes = [C.POINTER(abi.FixedRotationProblem),
                                                         C.POINTER(abi.ProbeOptions), C.POINTER(abi.ProbeReport),
                                                         C.POINTER(abi.Error)]
        L.omvgba_oracle_probe_fixed_rotation.restype = C.c_int
        u32p = C.POINTER(C.c_uint32)
        L.omvgba_oracle_residual_vjp.argtypes = [C.c_uint64, u32p, u32p, dp, dp, dp, dp, dp, dp, dp, dp, dp, dp, dp]
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().omvgba_oracle_set_threads(int(n))


def set_shards(n: int) -> None:
    lib().omvgba_oracle_set_shards(int(n))


def set_certificate(on: bool) -> None:
    """Timing runs only: skip the final certificate's band factorization (rank above D = 2048 and
    the self-calibration marginals), which runs after the LM loop."""
    lib().omvgba_oracle_set_certificate(int(bool(on)))


def iteration_seconds() -> list:
    """Wall time of each LM iteration of this thread's last solve."""
    buf = (C.c_double * 4096)()
    n = lib().omvgba_oracle_iteration_seconds(buf, 4096)
    return [buf[i] for i in range(min(n, 4096))]


def max_threads() -> int:
    return int(lib().omvgba_oracle_max_threads())


def solve(problem, config):
    """Run the oracle's BundleAdjuster::solve; returns openmvg_ba_cuda.problem.Solution."""
    from openmvg_ba_cuda import abi
    from openmvg_ba_cuda.problem import Solution, raise_for
    mp = abi.MarshalledProblem(problem)
    out = abi.SolutionBuffers(problem)
    cfg = config.to_struct()
    err = abi.Error()
    code = lib().omvgba_oracle_solve(C.byref(mp.struct), C.byref(cfg), C.byref(out.struct), C.byref(err))
    raise_for(code, err)
    return Solution.from_buffers(out)


def debug_linearize(problem, config):
    from openmvg_ba_cuda import abi
    from openmvg_ba_cuda.problem import raise_for
    mp = abi.MarshalledProblem(problem)
    n = problem.observation_count
    res = np.zeros((n, 2)); sw = np.zeros(n); jp = np.zeros((n, 2, 3)); jc = np.zeros((n, 2, 9))
    src = np.zeros(n, dtype=np.uint64)
    err = abi.Error()
    cfg = config.to_struct()
    dp = C.POINTER(C.c_double)
    code = lib().omvgba_oracle_debug_linearize(C.byref(mp.struct), C.byref(cfg), res.ctypes.data_as(dp),
                                               sw.ctypes.data_as(dp), jp.ctypes.data_as(dp), jc.ctypes.data_as(dp),
                                               src.ctypes.data_as(C.POINTER(C.c_uint64)), C.byref(err))
    raise_for(code, err)
    return {"residual": res, "sqrt_weight": sw, "point_jacobian": jp, "camera_jacobian": jc, "source_index": src}


def residual_vjp(inputs: dict, grad=None):
    """Analytic residual and J^T grad (float64) for the centred radial model."""
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    cam = np.ascontiguousarray(inputs["camera_index"], dtype=np.uint32)
    pt = np.ascontiguousarray(inputs["point_index"], dtype=np.uint32)
    px, rv, t, it, X = (f64(inputs[k]) for k in ("pixel", "rotvec", "translation", "intrinsics", "points"))
    n = len(cam)
    res = np.zeros((n, 2))
    g = f64(grad) if grad is not None else None
    gr, gt, gi, gp = np.zeros_like(rv), np.zeros_like(t), np.zeros_like(it), np.zeros_like(X)
    dp = C.POINTER(C.c_double)
    P = lambda a: a.ctypes.data_as(dp) if a is not None else None
    u32p = C.POINTER(C.c_uint32)
    lib().omvgba_oracle_residual_vjp(n, cam.ctypes.data_as(u32p), pt.ctypes.data_as(u32p), P(px), P(rv), P(t), P(it),
                                     P(X), P(g), P(res), P(gr), P(gt), P(gi), P(gp))
    return res, {"rotvec": gr, "translation": gt, "intrinsics": gi, "points": gp}


def execution_plan(problem, config):
    """(iterative, direct estimate, cached estimate) the oracle would use for this problem and config."""
    from openmvg_ba_cuda import abi
    from openmvg_ba_cuda.problem import raise_for
    mp = abi.MarshalledProblem(problem)
    cfg = config.to_struct()
    it, de, ce, err = C.c_int32(), C.c_uint64(), C.c_uint64(), abi.Error()
    code = lib().omvgba_oracle_execution_plan(C.byref(mp.struct), C.byref(cfg), C.byref(it), C.byref(de),
                                              C.byref(ce), C.byref(err))
    raise_for(code, err)
    return bool(it.value), int(de.value), int(ce.value)


def preflight(problem, config):
    """The oracle's NativeBundleAdjuster::preflight (dict of the NativePreflight fields)."""
    from openmvg_ba_cuda import abi
    from openmvg_ba_cuda.problem import raise_for
    mp = abi.MarshalledProblem(problem)
    cfg = config.to_struct()
    out, err = abi.Preflight(), abi.Error()
    raise_for(lib().omvgba_oracle_preflight(C.byref(mp.struct), C.byref(cfg), C.byref(out), C.byref(err)), err)
    return out.to_dict()


def probe_fixed_rotation(problem, options=None):
    """The oracle's probe_fixed_rotation_observability of a fixed_rotation.FixedRotationProblem."""
    from openmvg_ba_cuda import abi
    from openmvg_ba_cuda.fixed_rotation import ProbeOptions
    from openmvg_ba_cuda.problem import raise_for
    opts = (options or ProbeOptions()).to_struct()
    fp = problem.to_struct()
    out, err = abi.ProbeReport(), abi.Error()
    raise_for(lib().omvgba_oracle_probe_fixed_rotation(C.byref(fp), C.byref(opts), C.byref(out), C.byref(err)), err)
    return out.to_dict()


def camera_bearing(intrinsic, u: float, v: float):
    """The oracle's Camera::bearing of pixel (u, v) (unit vector) or None outside the model's domain."""
    from openmvg_ba_cuda import abi
    st = abi.Intrinsic()
    intrinsic.fill(st)
    out = np.zeros(3)
    ok = lib().omvgba_oracle_camera_bearing(C.byref(st), float(u), float(v), out.ctypes.data_as(C.POINTER(C.c_double)))
    return out if ok else None


def angular_projection(bearing, X):
    """(residual (2,), jacobian (2, 3)) of angular_projection, or None."""
    b = np.ascontiguousarray(bearing, dtype=np.float64)
    x = np.ascontiguousarray(X, dtype=np.float64)
    out = np.zeros(8)
    dp = C.POINTER(C.c_double)
    ok = lib().omvgba_oracle_angular_projection(b.ctypes.data_as(dp), x.ctypes.data_as(dp), out.ctypes.data_as(dp))
    return (out[:2], out[2:].reshape(2, 3)) if ok else None
