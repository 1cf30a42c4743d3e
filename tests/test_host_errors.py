"""Problem validation and the lowering's unsupported cases run on the host before any device work,
so their error behaviour is checked on the CPU: for each malformed or unsupported problem, and each
invalid configuration, the library, through omvgba_debug_setup_digest (validation, quarantine
preparation and lowering without a GPU), returns the same error code as the oracle's solve
(problem.rs:470-577, solver.rs:122-155, native/mod.rs:235-367, quarantine.rs:34-96), and a valid
problem passes both."""
import ctypes as C
import dataclasses

import numpy as np
import pytest

import oracle as O
from openmvg_ba_cuda import SolveConfig, abi, synthetic
from openmvg_ba_cuda import problem as P
from openmvg_ba_cuda._lib import lib

_CODE_OF = {cls: code for code, cls in P._ERRORS.items()}


def _lib_code(problem, cfg):
    m = abi.MarshalledProblem(problem)
    c = cfg.to_struct()
    out = C.c_uint64(0)
    err = abi.Error()
    return lib().omvgba_debug_setup_digest(C.byref(m.struct), C.byref(c), 0, C.byref(out), C.byref(err))


def _oracle_code(problem, cfg):
    try:
        O.solve(problem, cfg)
    except P.SolveError as e:
        return _CODE_OF[type(e)]
    except ValueError:
        return abi.OMVGBA_INVALID_ARGUMENT
    return abi.OMVGBA_OK


@pytest.fixture(scope="module")
def ring():
    return synthetic.ring_problem(seed=7)


def _copy(p, **changes):
    arrays = {f.name: (np.array(getattr(p, f.name), copy=True) if isinstance(getattr(p, f.name), np.ndarray)
                       else getattr(p, f.name)) for f in dataclasses.fields(p)}
    arrays.update(changes)
    return P.BundleProblem(**arrays)


def _set(p, name, index, value):
    a = np.array(getattr(p, name), copy=True)
    a[index] = value
    return _copy(p, **{name: a})


def _single_observation_tracks(p):
    pt = np.asarray(p.observation_point)
    keep = np.zeros(len(pt), dtype=bool)
    keep[np.unique(pt, return_index=True)[1]] = True
    return _copy(p, observation_pose=np.asarray(p.observation_pose)[keep],
                 observation_intrinsic=np.asarray(p.observation_intrinsic)[keep], observation_point=pt[keep],
                 observation_pixel=np.asarray(p.observation_pixel)[keep])


def _no_observations(p):
    return _copy(p, observation_pose=np.zeros(0, np.uint32), observation_intrinsic=np.zeros(0, np.uint32),
                 observation_point=np.zeros(0, np.uint32), observation_pixel=np.zeros((0, 2)))


CASES = {
    "pose index out of range": (lambda p: _set(p, "observation_pose", 5, len(p.rotations)), abi.OMVGBA_INVALID_PROBLEM),
    "point index out of range": (lambda p: _set(p, "observation_point", 7, len(p.points)), abi.OMVGBA_INVALID_PROBLEM),
    "intrinsic index out of range": (lambda p: _set(p, "observation_intrinsic", 3, len(p.intrinsics)),
                                     abi.OMVGBA_INVALID_PROBLEM),
    "non-finite pixel": (lambda p: _set(p, "observation_pixel", (3, 0), np.nan), abi.OMVGBA_INVALID_PROBLEM),
    "non-finite point": (lambda p: _set(p, "points", (11, 2), np.inf), abi.OMVGBA_INVALID_PROBLEM),
    "scaled rotation": (lambda p: _set(p, "rotations", 2, 1.01 * np.asarray(p.rotations)[2]),
                        abi.OMVGBA_INVALID_PROBLEM),
    "reflection": (lambda p: _set(p, "rotations", 4, -np.asarray(p.rotations)[4]), abi.OMVGBA_INVALID_PROBLEM),
    "fixed baseline to itself": (lambda p: _copy(p, gauge=P.Gauge.fixed_baseline(1, 1, 2.0)),
                                 abi.OMVGBA_INVALID_PROBLEM),
    "loss units differ from residuals": (
        lambda p: _copy(p, residual_space=abi.RESIDUAL_ANGULAR, robust_loss=P.RobustLoss.huber(1.0)),
        abi.OMVGBA_INVALID_PROBLEM),
    "angular residuals with free intrinsics": (
        lambda p: _copy(p, residual_space=abi.RESIDUAL_ANGULAR, robust_loss=P.RobustLoss.squared(),
                        intrinsics=[dataclasses.replace(p.intrinsics[0], variables=abi.INTRINSIC_FOCAL)]),
        abi.OMVGBA_UNSUPPORTED),
    "angular residuals of a pixel outside a spherical camera": (
        lambda p: _copy(p, residual_space=abi.RESIDUAL_ANGULAR, robust_loss=P.RobustLoss.squared(),
                        intrinsics=[P.CameraIntrinsics(model=abi.CAMERA_SPHERICAL, width=64, height=32)]),
        abi.OMVGBA_NUMERICAL),
    "every track a single observation": (_single_observation_tracks, abi.OMVGBA_UNSUPPORTED),
    "no observations": (_no_observations, abi.OMVGBA_INVALID_PROBLEM),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_invalid_problem_gets_the_oracles_error(ring, name):
    mutate, expected = CASES[name]
    p = mutate(ring)
    cfg = SolveConfig()
    assert _oracle_code(p, cfg) == expected
    assert _lib_code(p, cfg) == expected


def test_valid_problem_passes_the_host_checks(ring):
    assert _lib_code(ring, SolveConfig()) == abi.OMVGBA_OK


CONFIG_CASES = {
    "no iterations": dict(max_iterations=0),
    "zero function tolerance": dict(function_tolerance=0.0),
    "non-finite gradient tolerance": dict(gradient_tolerance=float("nan")),
    "negative parameter tolerance": dict(parameter_tolerance=-1.0),
    "zero workspace budget": dict(workspace_budget_bytes=0),
}


@pytest.mark.parametrize("name", sorted(CONFIG_CASES))
def test_invalid_config_gets_the_oracles_error(ring, name):
    cfg = dataclasses.replace(SolveConfig(), **CONFIG_CASES[name])
    assert _oracle_code(ring, cfg) == abi.OMVGBA_INVALID_CONFIG
    assert _lib_code(ring, cfg) == abi.OMVGBA_INVALID_CONFIG
