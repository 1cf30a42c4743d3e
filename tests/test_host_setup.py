"""The host side of a solve's set-up (quarantine preparation, lowering, block tables, matvec tiles)
runs on several host threads; like the reference's own solver, its result must not depend on how
many. omvgba_debug_setup_digest builds the set-up on the CPU alone (no GPU, no context) with a given
thread limit and returns a digest of everything it builds, so these tests run without a GPU."""
import ctypes as C
import dataclasses

import numpy as np
import pytest

from openmvg_ba_cuda import SolveConfig, abi, synthetic
from openmvg_ba_cuda._lib import lib


def _digest(problem, cfg, threads):
    m = abi.MarshalledProblem(problem)
    c = cfg.to_struct()
    out = C.c_uint64(0)
    err = abi.Error()
    code = lib().omvgba_debug_setup_digest(C.byref(m.struct), C.byref(c), threads, C.byref(out), C.byref(err))
    assert code == 0, err.message
    return out.value


def _with_held_out(problem, every=97):
    """Every `every`-th point keeps only its first observation, so preparation holds it out."""
    pt = np.asarray(problem.observation_point)
    first = np.zeros(len(pt), dtype=bool)
    first[np.unique(pt, return_index=True)[1]] = True
    keep = (pt % every != 0) | first
    return dataclasses.replace(
        problem,
        observation_pose=np.asarray(problem.observation_pose)[keep],
        observation_intrinsic=np.asarray(problem.observation_intrinsic)[keep],
        observation_point=pt[keep],
        observation_pixel=np.asarray(problem.observation_pixel)[keep],
    )


@pytest.fixture(scope="module")
def plane():
    # ~180k observations: above the size at which the set-up's loops split across threads
    return synthetic.plane_problem(seed=3, cameras=120, points=30_000)


@pytest.mark.parametrize("precision", [abi.PRECISION_MIXED, abi.PRECISION_FP64])
def test_setup_does_not_depend_on_thread_count(plane, precision):
    cfg = SolveConfig(linear_solver=abi.SOLVER_ITERATIVE, precision=precision)
    digests = [_digest(plane, cfg, threads) for threads in (1, 3, 0)]
    assert digests[0] == digests[1] == digests[2]


def test_setup_with_held_out_points_does_not_depend_on_thread_count(plane):
    cfg = SolveConfig(linear_solver=abi.SOLVER_ITERATIVE, precision=abi.PRECISION_MIXED)
    held = _with_held_out(plane)
    digests = [_digest(held, cfg, threads) for threads in (1, 4, 0)]
    assert digests[0] == digests[1] == digests[2]
    # the digest covers the inputs: holding points out changes it
    assert digests[0] != _digest(plane, cfg, 0)


def test_setup_digest_rejects_null_arguments(plane):
    cfg = SolveConfig().to_struct()
    out = C.c_uint64(0)
    err = abi.Error()
    code = lib().omvgba_debug_setup_digest(None, C.byref(cfg), 0, C.byref(out), C.byref(err))
    assert code == abi.OMVGBA_INVALID_ARGUMENT
