"""Batched local-BA windows (omvgba_solve_batched): every window's solution equals the single-problem
solve of that window bit for bit, and matches the oracle at the parity tolerances; a failing window
is reported with its index while the others are still solved."""
import dataclasses

import numpy as np
import pytest

import oracle
from openmvg_ba_cuda import ProblemError, SolveConfig, abi, synthetic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def windows():
    return synthetic.window_problems(seed=31, windows=12, total_observations=60_000, min_points=300,
                                     max_points=3000, max_cameras=24)


def test_batched_windows_equal_single_solves_and_the_oracle(adjuster, windows):
    cfg = SolveConfig(max_iterations=30)
    batched = adjuster.solve_batched(windows, cfg)
    assert len(batched) == len(windows)
    for w, got in zip(windows, batched):
        single = adjuster.solve(w, cfg)
        assert np.array_equal(got.points, single.points)
        assert np.array_equal(got.rotations, single.rotations)
        assert got.report["final_objective"] == single.report["final_objective"]
        assert got.report["iteration_count"] == single.report["iteration_count"]
        ref = oracle.solve(w, cfg)
        assert got.report["iteration_count"] == ref.report["iteration_count"]
        rel = abs(got.report["final_objective"] - ref.report["final_objective"]) / ref.report["final_objective"]
        assert rel <= 1e-9
        assert got.report["kernel_launches"] > 0


def test_a_failing_window_is_reported_by_index(adjuster, windows):
    # an angular residual space with a pixel loss scale fails the problem's validation
    bad = dataclasses.replace(windows[2], residual_space=abi.RESIDUAL_ANGULAR)
    batch = [windows[0], windows[1], bad, windows[3]]
    with pytest.raises(ProblemError, match="window 2"):
        adjuster.solve_batched(batch, SolveConfig(max_iterations=5))
