"""The linear solver a solve uses and the workspace budget (sparse/execution_policy.rs:122-253,
native/mod.rs:544-570): Auto resolved by the budget in the library (host side, no GPU) and in the
oracle from the same estimates, and a workspace over an explicit budget refused with
ResourceExhausted before the first iteration."""
import ctypes as C

import pytest

import oracle as O
from openmvg_ba_cuda import SolveConfig, abi, synthetic
from openmvg_ba_cuda._lib import lib
from openmvg_ba_cuda.problem import ResourceExhausted, raise_for


def library_plan(problem, config):
    mp = abi.MarshalledProblem(problem)
    cfg = config.to_struct()
    it, de, ce, err = C.c_int32(), C.c_uint64(), C.c_uint64(), abi.Error()
    code = lib().omvgba_debug_execution_plan(C.byref(mp.struct), C.byref(cfg), C.byref(it), C.byref(de),
                                             C.byref(ce), C.byref(err))
    raise_for(code, err)
    return bool(it.value), int(de.value), int(ce.value)


CASES = {
    "ring": lambda: synthetic.ring_problem(seed=3),
    "ring_self_cal": lambda: synthetic.ring_problem(seed=3, self_calibrating=True),
    "plane_self_cal": lambda: synthetic.plane_problem(seed=11, cameras=200, points=15_000, mean_track=6.5,
                                                      extent=60.0),
    "plane_calibrated_large": lambda: synthetic.plane_problem(seed=12, cameras=200, points=45_000, mean_track=6.5,
                                                              extent=60.0, per_camera_intrinsics=False,
                                                              free_intrinsics=False),
}


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request):
    return request.param, CASES[request.param]()


def test_auto_choice_and_estimates_match_the_oracle(case):
    name, p = case
    for budget in (None, 10**12, 1 << 20):
        cfg = SolveConfig(linear_solver=abi.SOLVER_AUTO, workspace_budget_bytes=budget)
        got, want = library_plan(p, cfg), O.execution_plan(p, cfg)
        assert got == want, (name, budget, got, want)


def test_auto_follows_the_policy(case):
    name, p = case
    iterative, direct, cached = library_plan(p, SolveConfig(linear_solver=abi.SOLVER_AUTO))
    if name == "plane_calibrated_large":  # >= 250,000 observations and D >= 768: retained PCG first
        assert p.observation_count >= 250_000 and iterative
    else:
        assert not iterative and direct <= (1 << 30) * 4 // 5
    # a budget below the direct estimate sends every problem to PCG
    tight = SolveConfig(linear_solver=abi.SOLVER_AUTO, workspace_budget_bytes=direct // 2)
    assert library_plan(p, tight)[0] is True
    # an explicit choice is kept
    for solver, want in ((abi.SOLVER_DIRECT, False), (abi.SOLVER_ITERATIVE, True)):
        assert library_plan(p, SolveConfig(linear_solver=solver))[0] is want


def test_oracle_refuses_a_workspace_over_the_budget():
    p = synthetic.ring_problem(seed=3)
    with pytest.raises(ResourceExhausted, match="exceeds the workspace budget"):
        O.solve(p, SolveConfig(workspace_budget_bytes=1024))
    O.solve(p, SolveConfig(workspace_budget_bytes=1 << 40, max_iterations=3))


@pytest.mark.gpu
def test_library_refuses_a_workspace_over_the_budget(adjuster):
    p = synthetic.ring_problem(seed=3)
    with pytest.raises(ResourceExhausted, match="exceeds the workspace budget"):
        adjuster.solve(p, SolveConfig(workspace_budget_bytes=1024))
    sol = adjuster.solve(p, SolveConfig(workspace_budget_bytes=1 << 40, max_iterations=3))
    assert sol.report["iteration_count"] == 3
