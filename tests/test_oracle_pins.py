"""Pins of the oracle against the reference's own known-answer tests (CPU only).

The reference (Rust) cannot be built here, so the oracle's arithmetic is pinned to the assertions
the reference's unit tests make, restated with the same inputs and tolerances:
  robust losses ............ crates/openmvg-ba/src/numerics/robust.rs:50-131
  Nielsen damping .......... crates/openmvg-ba/src/numerics/refine/nonlinear/controller.rs:97-114,
                             run_state.rs:216-245
  stage schedule ........... crates/openmvg-ba/src/numerics/refine/nonlinear/continuation.rs:82-112
  radial Jacobians ......... crates/openmvg-ba/src/kernel/multi_view/self_calibration/model.rs:357-467
  Brown-Conrady k3 ......... crates/openmvg-ba/src/kernel/multi_view/camera_kernel.rs:274-293
"""
import math

import numpy as np
import pytest

import oracle
from openmvg_ba_cuda import abi

EPS = np.finfo(np.float64).eps


def cost(kind, scale, r):
    return oracle.lib().omvgba_oracle_loss_cost(kind, scale, r)


def sqrt_weight(kind, scale, r):
    return oracle.lib().omvgba_oracle_loss_sqrt_weight(kind, scale, r)


# ---- robust.rs ---------------------------------------------------------------------------------
def test_cauchy_downweights_large_residuals():
    assert sqrt_weight(abi.LOSS_CAUCHY, 0.01, 0.5) < 0.1 * sqrt_weight(abi.LOSS_CAUCHY, 0.01, 0.001)


def test_cauchy_weight_matches_cost_derivative_across_decades():
    scale = 0.01
    for exponent in range(-4, 5):
        r = scale * 10.0 ** exponent
        h = 1e-6 * r
        numerical = (cost(abi.LOSS_CAUCHY, scale, r + h) - cost(abi.LOSS_CAUCHY, scale, r - h)) / (2 * h)
        w = sqrt_weight(abi.LOSS_CAUCHY, scale, r)
        analytic = w * w * r
        rounding = 4.0 * EPS * cost(abi.LOSS_CAUCHY, scale, r) / h
        assert abs(numerical - analytic) <= 1e-6 * abs(analytic) + rounding


def test_cauchy_far_tail_is_not_floored():
    w = sqrt_weight(abi.LOSS_CAUCHY, 0.01, 1e18)
    assert w * w < 1e-14


def test_huber_weight_matches_cost_derivative_on_both_branches():
    delta, h = 0.01, 1e-8
    for r in (0.004, 0.04, -0.04):
        numerical = (cost(abi.LOSS_HUBER, delta, r + h) - cost(abi.LOSS_HUBER, delta, r - h)) / (2 * h)
        w = sqrt_weight(abi.LOSS_HUBER, delta, r)
        assert abs(numerical - w * w * r) < 1e-10


def test_losses_zero_at_zero_even_nondecreasing():
    scale = 0.01
    for kind in (abi.LOSS_HUBER, abi.LOSS_CAUCHY):
        assert cost(kind, scale, 0.0) == 0.0
        prev = 0.0
        for exponent in range(-8, 9):
            r = scale * 10.0 ** exponent
            assert cost(kind, scale, r) == cost(kind, scale, -r)
            assert cost(kind, scale, r) >= prev
            prev = cost(kind, scale, r)


def test_cauchy_cost_keeps_precision_for_tiny_residuals():
    for r in (1e-5, 1e-9, 1e-150):
        expected = 0.5 * r * r
        assert abs(cost(abi.LOSS_CAUCHY, 1.0, r) - expected) <= 1e-9 * expected


def test_huber_is_c1_at_transition():
    delta, h = 0.01, 1e-12
    below, above = cost(abi.LOSS_HUBER, delta, delta - h), cost(abi.LOSS_HUBER, delta, delta + h)
    assert abs(above - below - 2 * h * delta) <= 1e-20
    assert sqrt_weight(abi.LOSS_HUBER, delta, delta) == 1.0
    assert abs(sqrt_weight(abi.LOSS_HUBER, delta, delta + h) - 1.0) <= 1e-9


# ---- Nielsen controller and run state -----------------------------------------------------------
def nielsen(ops, initial):
    import ctypes as C
    n = len(ops)
    kinds = (C.c_int * n)(*[0 if o is None else 1 for o in ops])
    actual = (C.c_double * n)(*[0.0 if o is None else o[0] for o in ops])
    predicted = (C.c_double * n)(*[0.0 if o is None else o[1] for o in ops])
    damping, gain = (C.c_double * n)(), (C.c_double * n)()
    accepted, has_gain = (C.c_int * n)(), (C.c_int * n)()
    oracle.lib().omvgba_oracle_nielsen(n, kinds, actual, predicted, initial, damping, accepted, gain, has_gain)
    return [(damping[i], accepted[i], gain[i] if has_gain[i] else None) for i in range(n)]


def test_nielsen_uses_gain_and_rejection_history():
    d0 = 1e-4
    t = nielsen([(2.0, 2.0), None, None, (-1.0, 1.0), (1.0, -1.0)], d0)
    assert t[0][1] == 1 and t[0][2] == 1.0
    assert abs(t[0][0] - d0 / 3.0) < 1e-15
    assert t[1][2] is None
    assert abs(t[1][0] - 2.0 * d0 / 3.0) < 1e-15
    assert abs(t[2][0] - 8.0 * d0 / 3.0) < 1e-15
    assert t[3][1] == 0 and t[3][2] == -1.0
    assert t[4][1] == 0 and t[4][2] is None


def test_rejection_table_preserves_history():
    def near(a, b):
        assert abs(a - b) <= 8.0 * EPS * max(abs(b), 1.0)
    t = nielsen([None, None, (-1.0, 1.0), (1.0, -1.0)], 1e-4)
    near(t[0][0], 2e-4)
    near(t[1][0], 8e-4)
    near(t[2][0], 6.4e-3)
    assert t[2][2] == -1.0
    near(t[3][0], 0.1024)
    assert t[3][2] is None


def test_accepted_gain_resets_rejection_history():
    t = nielsen([None, (1.0, 1.0), None], 1e-4)
    accepted = 2e-4 / 3.0
    assert abs(t[1][0] - accepted) <= 8.0 * EPS
    assert abs(t[2][0] - 2.0 * accepted) <= 8.0 * EPS


# ---- continuation stages ------------------------------------------------------------------------
def test_stage_schedule_preserves_budget_and_reaches_target_loss():
    import ctypes as C
    for iterations in range(20):
        for kind in (abi.LOSS_SQUARED, abi.LOSS_HUBER, abi.LOSS_CAUCHY):
            budgets, kinds = (C.c_uint64 * 3)(), (C.c_int * 3)()
            oracle.lib().omvgba_oracle_stages(kind, iterations, budgets, kinds)
            assert sum(budgets) == iterations
            if iterations > 0:
                assert any(budgets[i] > 0 and kinds[i] == kind for i in range(3))


# ---- radial self-calibration model --------------------------------------------------------------
def radial(f, k1, k2, obs, X):
    import ctypes as C
    out = np.zeros(14)
    dp = C.POINTER(C.c_double)
    ok = oracle.lib().omvgba_oracle_radial_linearize(f, k1, k2, np.asarray(obs, float).ctypes.data_as(dp),
                                                     np.asarray(X, float).ctypes.data_as(dp), out.ctypes.data_as(dp))
    assert ok
    return out[:2], out[2:8].reshape(2, 3), out[8:14].reshape(2, 3)


def close(actual, expected, tol):
    assert abs(actual - expected) <= tol * (1.0 + abs(expected)), (actual, expected)


def test_radial_point_jacobian_matches_central_differences():
    f, k1, k2 = 730.0, 0.08, -0.025
    obs, X = [17.0, -23.0], np.array([0.71, -0.43, 2.4])
    _, J, _ = radial(f, k1, k2, obs, X)
    h = 1e-6
    for c in range(3):
        plus, minus = X.copy(), X.copy()
        plus[c] += h
        minus[c] -= h
        rp, rm = radial(f, k1, k2, obs, plus)[0], radial(f, k1, k2, obs, minus)[0]
        for row in range(2):
            close(J[row, c], (rp[row] - rm[row]) / (2 * h), 2e-8)


def test_radial_intrinsic_jacobian_matches_log_focal_retraction():
    f, k1, k2 = 730.0, 0.08, -0.025
    obs, X = [0.0, 0.0], [0.71, -0.43, 2.4]
    _, _, Ji = radial(f, k1, k2, obs, X)
    h = 1e-6
    perturb = [
        ((f * math.exp(h), k1, k2), (f * math.exp(-h), k1, k2)),
        ((f, k1 + h, k2), (f, k1 - h, k2)),
        ((f, k1, k2 + h), (f, k1, k2 - h)),
    ]
    for col, (p, m) in enumerate(perturb):
        rp, rm = radial(*p, obs, X)[0], radial(*m, obs, X)[0]
        for row in range(2):
            close(Ji[row, col], (rp[row] - rm[row]) / (2 * h), 2e-8)


# ---- Brown-Conrady k3 one-axis derivative -------------------------------------------------------
def test_brown_conrady_k3_one_axis_derivative():
    import ctypes as C
    s = abi.Intrinsic()
    s.model, s.radial_kind, s.tangential_kind = abi.CAMERA_BROWN_CONRADY, abi.RADIAL_K1K2K3, abi.TANGENTIAL_NONE
    s.fx, s.fy, s.cx, s.cy = 800.0, 600.0, 0.0, 0.0
    s.k1, s.k2, s.k3 = -0.08, 0.012, -0.001
    s.width, s.height = 640, 480
    x = 0.4
    q = x * x
    out = np.zeros(8)
    dp = C.POINTER(C.c_double)
    X = np.array([x, 0.0, 1.0])
    assert oracle.lib().omvgba_oracle_bc_project(C.byref(s), X.ctypes.data_as(dp), out.ctypes.data_as(dp))
    factor = 1.0 - 0.08 * q + 0.012 * q * q - 0.001 * q * q * q
    slope = 1.0 - 3.0 * 0.08 * q + 5.0 * 0.012 * q * q - 7.0 * 0.001 * q * q * q
    J = out[2:8].reshape(2, 3)
    assert abs(out[0] - 800.0 * x * factor) < 1e-12
    assert abs(J[0, 0] - 800.0 * slope) < 1e-12
    assert abs(J[1, 1] - 600.0 * factor) < 1e-12


# ---- SO(3) exponential and the point-block inverse ------------------------------------------------
def exp_so3(v):
    import ctypes as C
    R = np.zeros(9)
    dp = C.POINTER(C.c_double)
    oracle.lib().omvgba_oracle_exp_so3(np.asarray(v, float).ctypes.data_as(dp), R.ctypes.data_as(dp))
    return R.reshape(3, 3)


def test_exp_so3_is_rodrigues():
    R = exp_so3([0.0, 0.0, math.pi / 2])
    assert np.allclose(R, [[0, -1, 0], [1, 0, 0], [0, 0, 1]], atol=1e-15)
    rng = np.random.default_rng(5)
    for _ in range(20):
        v = rng.normal(size=3) * rng.uniform(1e-9, 3.0)
        R = exp_so3(v)
        assert np.allclose(R @ R.T, np.eye(3), atol=1e-14)
        assert abs(np.linalg.det(R) - 1.0) < 1e-14
        assert np.allclose(R @ v, v, atol=1e-14 * max(1.0, np.linalg.norm(v)))  # the axis is fixed


def test_point_block_inverse_is_the_damped_inverse():
    import ctypes as C
    rng = np.random.default_rng(9)
    A = rng.normal(size=(3, 3))
    V = A @ A.T + 0.5 * np.eye(3)
    lam = 1e-3
    packed, rc = np.zeros(6), C.c_double()
    dp = C.POINTER(C.c_double)
    assert oracle.lib().omvgba_oracle_point_block_inverse(np.ascontiguousarray(V).ctypes.data_as(dp), lam,
                                                           packed.ctypes.data_as(dp), C.byref(rc))
    # damped_matrix (point_block.rs:90-97): V + lambda * diag(max(V_ii, 64 eps max V_ii))
    d = np.diag(V)
    Vd = V + lam * np.diag(np.maximum(d, 64 * EPS * d.max()))
    inv = np.linalg.inv(Vd)
    # packed lower triangle: (0,0) (1,0) (1,1) (2,0) (2,1) (2,2)
    expect = [inv[0, 0], inv[1, 0], inv[1, 1], inv[2, 0], inv[2, 1], inv[2, 2]]
    assert np.allclose(packed, expect, rtol=1e-12, atol=0)
    assert 0.0 < rc.value <= 1.0
