"""``CudaBundleAdjuster``: the ``BundleAdjuster`` trait (crates/openmvg-ba/src/solver.rs:1562-1573)
implemented by the B200 solver through the C ABI."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from ._lib import lib
from .problem import BundleProblem, Solution, SolveConfig, raise_for


class CudaBundleAdjuster:
    """One GPU solver context (device workspaces and stream). ``solve`` never mutates the problem."""

    def __init__(self, device: int = 0):
        err = abi.Error()
        self._ctx = lib().omvgba_context_create(device, C.byref(err))
        if not self._ctx:
            raise_for(err.code or abi.OMVGBA_CUDA_ERROR, err)
        self.device = device

    def name(self) -> str:
        return lib().omvgba_adjuster_name().decode()

    def solve(self, problem: BundleProblem, config: SolveConfig | None = None) -> Solution:
        config = config or SolveConfig()
        mp = abi.MarshalledProblem(problem)
        out = abi.SolutionBuffers(problem)
        cfg = config.to_struct()
        err = abi.Error()
        code = lib().omvgba_solve(self._ctx, C.byref(mp.struct), C.byref(cfg), C.byref(out.struct), C.byref(err))
        raise_for(code, err)
        return Solution.from_buffers(out)

    def preflight(self, problem: BundleProblem, config: SolveConfig | None = None) -> dict:
        """``NativeBundleAdjuster::preflight`` (native/mod.rs:184-230): the translation-only
        observability probe on the prepared problem, or PROCEED with no counts for other problems."""
        config = config or SolveConfig()
        mp = abi.MarshalledProblem(problem)
        cfg = config.to_struct()
        out, err = abi.Preflight(), abi.Error()
        code = lib().omvgba_preflight_check(self._ctx, C.byref(mp.struct), C.byref(cfg), C.byref(out), C.byref(err))
        raise_for(code, err)
        return out.to_dict()

    def probe_fixed_rotation(self, problem, options=None) -> dict:
        """``probe_fixed_rotation_observability`` (kernel/fixed_rotation/observability.rs:24-262) of a
        ``fixed_rotation.FixedRotationProblem``."""
        from .fixed_rotation import ProbeOptions
        opts = (options or ProbeOptions()).to_struct()
        fp = problem.to_struct()
        out, err = abi.ProbeReport(), abi.Error()
        code = lib().omvgba_probe_fixed_rotation(self._ctx, C.byref(fp), C.byref(opts), C.byref(out), C.byref(err))
        raise_for(code, err)
        return out.to_dict()

    def debug_linearize(self, problem: BundleProblem, config: SolveConfig | None = None) -> dict:
        config = config or SolveConfig()
        mp = abi.MarshalledProblem(problem)
        n = problem.observation_count
        res = np.zeros((n, 2)); sw = np.zeros(n); jp = np.zeros((n, 2, 3)); jc = np.zeros((n, 2, 9))
        src = np.zeros(n, dtype=np.uint64)
        cfg = config.to_struct()
        err = abi.Error()
        dp = C.POINTER(C.c_double)
        code = lib().omvgba_debug_linearize(self._ctx, C.byref(mp.struct), C.byref(cfg), res.ctypes.data_as(dp),
                                            sw.ctypes.data_as(dp), jp.ctypes.data_as(dp), jc.ctypes.data_as(dp),
                                            src.ctypes.data_as(C.POINTER(C.c_uint64)), C.byref(err))
        raise_for(code, err)
        return {"residual": res, "sqrt_weight": sw, "point_jacobian": jp, "camera_jacobian": jc, "source_index": src}

    def debug_schur_product(self, problem: BundleProblem, x: np.ndarray | None, damping: float = 0.0,
                            config: SolveConfig | None = None):
        """(y_matvec, y_dense) = S_lambda x by the matrix-free kernel and by the dense Schur complement."""
        config = config or SolveConfig()
        mp = abi.MarshalledProblem(problem)
        cfg = config.to_struct()
        err = abi.Error()
        dim = C.c_int32(0)
        dp = C.POINTER(C.c_double)
        code = lib().omvgba_debug_schur_product(self._ctx, C.byref(mp.struct), C.byref(cfg), damping, None, None, None,
                                                C.byref(dim), C.byref(err))
        raise_for(code, err)
        if x is None:
            return dim.value
        x = np.ascontiguousarray(x, dtype=np.float64)
        assert x.shape == (dim.value,)
        ym, yd = np.zeros(dim.value), np.zeros(dim.value)
        code = lib().omvgba_debug_schur_product(self._ctx, C.byref(mp.struct), C.byref(cfg), damping,
                                                x.ctypes.data_as(dp), ym.ctypes.data_as(dp), yd.ctypes.data_as(dp),
                                                C.byref(dim), C.byref(err))
        raise_for(code, err)
        return ym, yd

    def solve_batched(self, problems: list, config: SolveConfig | None = None) -> list:
        """Solve independent windows in one call; window i's solution is what ``solve`` returns for it."""
        config = config or SolveConfig()
        marshalled = [abi.MarshalledProblem(p) for p in problems]
        outs = [abi.SolutionBuffers(p) for p in problems]
        n = len(problems)
        probs = (abi.Problem * max(n, 1))(*[m.struct for m in marshalled])
        sols = (abi.Solution * max(n, 1))(*[o.struct for o in outs])
        cfg = config.to_struct()
        err = abi.Error()
        code = lib().omvgba_solve_batched(self._ctx, n, probs, C.byref(cfg), sols, C.byref(err))
        raise_for(code, err)
        results = []
        for o, s in zip(outs, sols):
            o.struct = s  # the report was written into the array copy of the struct
            results.append(Solution.from_buffers(o))
        return results

    def plan(self, problem: BundleProblem, config: SolveConfig | None = None) -> "Plan":
        """Prepare ``problem`` once (lowering, upload) for repeated solves from its initial state."""
        return Plan(self, problem, config or SolveConfig())

    def close(self) -> None:
        if getattr(self, "_ctx", None):
            lib().omvgba_context_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Plan:
    """A problem resident in device memory: ``solve`` returns what ``CudaBundleAdjuster.solve``
    returns, without the per-call lowering and upload. Keeps the marshalled problem alive."""

    def __init__(self, adjuster: CudaBundleAdjuster, problem: BundleProblem, config: SolveConfig):
        self._adjuster = adjuster
        self._problem = problem
        self._mp = abi.MarshalledProblem(problem)
        self._cfg = config.to_struct()
        self._out = abi.SolutionBuffers(problem)
        handle = C.c_void_p()
        err = abi.Error()
        code = lib().omvgba_plan_create(adjuster._ctx, C.byref(self._mp.struct), C.byref(self._cfg),
                                        C.byref(handle), C.byref(err))
        raise_for(code, err)
        self._plan = handle

    def solve(self) -> Solution:
        err = abi.Error()
        code = lib().omvgba_plan_solve(self._plan, C.byref(self._out.struct), C.byref(err))
        raise_for(code, err)
        return Solution.from_buffers(self._out)

    def info(self) -> dict:
        info = abi.PlanInfo()
        err = abi.Error()
        raise_for(lib().omvgba_plan_info_get(self._plan, C.byref(info), C.byref(err)), err)
        return info.to_dict()

    def schur_product(self, x_ptr: int, y_ptr: int, damping: float, fp32: bool = False, stage: int = 0) -> None:
        """y = S_lambda x on device pointers (stage 1: the tile pass alone; stage 2: the explicit S
        rows alone; stage 3: the camera-side assembly sums alone), on the plan's stream."""
        err = abi.Error()
        code = lib().omvgba_plan_schur_product(self._plan, damping, int(fp32), stage, C.c_void_p(x_ptr),
                                               C.c_void_p(y_ptr), C.byref(err))
        raise_for(code, err)

    def close(self) -> None:
        if getattr(self, "_plan", None):
            lib().omvgba_plan_destroy(self._plan)
            self._plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
