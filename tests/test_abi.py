"""The C ABI library (no GPU needed): it loads, exports every function include/ba_cuda.h declares,
its struct layouts match the Python mirrors, and host-side argument checks fail cleanly."""
import ctypes as C
import os
import re

import pytest

from openmvg_ba_cuda import SolveConfig, abi, synthetic
from openmvg_ba_cuda import _lib

HEADER = os.path.join(os.path.dirname(__file__), "..", "include", "ba_cuda.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(omvgba_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_reports_version():
    L = _lib.lib()
    assert L.omvgba_abi_version() == 3
    assert L.omvgba_adjuster_name().decode() == "openmvg-ba-cuda-b200"


def test_every_declared_function_is_exported():
    L = _lib.lib()
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_struct_layouts_match_the_mirrors():
    sizes = _lib.struct_sizes()
    assert sizes == {
        "error": C.sizeof(abi.Error), "pose": C.sizeof(abi.Pose), "intrinsic": C.sizeof(abi.Intrinsic),
        "problem": C.sizeof(abi.Problem), "config": C.sizeof(abi.Config), "report": C.sizeof(abi.Report),
        "solution": C.sizeof(abi.Solution),
    }


def test_config_default_is_solveconfig_default():
    c = abi.Config()
    _lib.lib().omvgba_config_default(C.byref(c))
    # SolveConfig::default (crates/openmvg-ba/src/solver.rs:112-120)
    assert c.max_iterations == 50
    assert c.function_tolerance == 1e-6
    assert c.gradient_tolerance == 1e-10
    assert c.parameter_tolerance == 1e-8
    assert c.linear_solver == abi.SOLVER_AUTO
    assert c.has_workspace_budget == 0
    assert c.precision == abi.PRECISION_FP64


def test_null_arguments_are_rejected_without_a_device():
    L = _lib.lib()
    err = abi.Error()
    assert L.omvgba_solve(None, None, None, None, C.byref(err)) == abi.OMVGBA_INVALID_ARGUMENT
    assert b"null" in err.message
    handle = C.c_void_p()
    assert L.omvgba_plan_create(None, None, None, C.byref(handle), C.byref(err)) == abi.OMVGBA_INVALID_ARGUMENT
    assert L.omvgba_plan_solve(None, None, C.byref(err)) == abi.OMVGBA_INVALID_ARGUMENT
    L.omvgba_plan_destroy(None)
    L.omvgba_context_destroy(None)


def test_residual_entry_points_check_arguments_on_the_host():
    L = _lib.lib()
    err = abi.Error()
    # a null pointer with a non-zero count is rejected before any device work
    code = L.omvgba_residual_forward_f32(None, 4, None, None, None, 1, None, None, None, 1, None, None, C.byref(err))
    assert code == abi.OMVGBA_INVALID_ARGUMENT
    # zero observations is a no-op
    code = L.omvgba_residual_forward_f32(None, 0, None, None, None, 0, None, None, None, 0, None, None, C.byref(err))
    assert code == abi.OMVGBA_OK
    assert L.omvgba_residual_vjp_workspace_bytes(1000, 10, 100) > 0


@pytest.mark.skipif(_lib.device_count() > 0, reason="a device is present")
def test_context_creation_fails_cleanly_without_a_device():
    err = abi.Error()
    ctx = _lib.lib().omvgba_context_create(0, C.byref(err))
    assert not ctx
    assert err.code == abi.OMVGBA_CUDA_ERROR


def test_solve_config_marshals():
    cfg = SolveConfig(linear_solver=abi.SOLVER_ITERATIVE, precision=abi.PRECISION_MIXED,
                      pcg_relative_tolerance=1e-6).to_struct()
    assert cfg.linear_solver == abi.SOLVER_ITERATIVE and cfg.precision == abi.PRECISION_MIXED
    assert cfg.pcg_relative_tolerance == 1e-6 and cfg.stream is None


def test_problem_marshalling_round_trips():
    p = synthetic.ring_problem(seed=1, points=50)
    mp = abi.MarshalledProblem(p)
    s = mp.struct
    assert s.pose_count == 20 and s.point_count == 50 and s.observation_count == p.observation_count
    assert s.observation_point[p.observation_count - 1] == p.observation_point[-1]
    assert s.points[3] == p.points[1, 0]
