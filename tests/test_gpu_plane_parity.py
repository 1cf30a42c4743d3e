"""GPU FP64 solve vs the CPU oracle at the measured workloads' own sizes, and mixed precision vs FP64.

plane500 is the 500-camera, 200,000-point ground-plane survey with per-camera (f, k1, k2) (about 1.1M
observations, D = 4,493), solved here for 4 LM iterations with a tight PCG tolerance so that the
GPU and oracle trajectories can be compared step for step (the Auto operator switches to the
explicit S inside this run). plane3000_200k keeps the 3,000-camera geometry of the 12M-observation
workload with 200,000 points and the cameras' intrinsics held (D = 18,000), so that the oracle's LM
iterations and its final rank certificate finish within seconds; with free intrinsics and only ~70
points per camera most (f, k1, k2) groups come out unconstrained and the reference re-solves with
them held, which the oracle would take minutes to repeat at D = 27,000.

The mixed-precision pin restates the reference's F32 retained-cross-cache test
(crates/openmvg-ba/tests/sparse_bundle_adjustment/iterative_schur.rs:173-262, fixture main.rs:66-135):
four pinhole cameras, 24 points, camera 3 missing every third point, a fixed baseline between
cameras 0 and 1, L2 loss, 12 iterations of the iterative solver; FP32 Jacobian records and products
must take the same accepted and rejected steps as FP64 and end within 1e-7 of its cost.
"""
import numpy as np
import pytest

import oracle as O
from openmvg_ba_cuda import BundleProblem, CameraIntrinsics, Gauge, RobustLoss, SolveConfig, abi, synthetic

pytestmark = pytest.mark.gpu

LM_KEYS = ("status", "iteration_count", "accepted_step_count", "rejected_step_count", "quarantined_point_count",
           "inlier_count", "linear_solver", "reduced_dimension")


def _compare(g, o, tag):
    for k in LM_KEYS:
        assert g.report[k] == o.report[k], (tag, k, g.report[k], o.report[k])
    fo = o.report["final_objective"]
    assert abs(g.report["final_objective"] - fo) <= 1e-9 * fo, (tag, g.report["final_objective"], fo)
    assert abs(g.report["initial_objective"] - o.report["initial_objective"]) <= 1e-12 * o.report["initial_objective"]
    dr = np.max(np.abs(g.rotations - o.rotations))
    dc = np.max(np.abs(g.centers - o.centers))
    assert dr < 1e-7 and dc < 1e-7, (tag, dr, dc)
    for ia, ib in zip(g.intrinsics, o.intrinsics):
        assert abs(ia.fx - ib.fx) / abs(ib.fx) < 1e-9, (tag, ia.fx, ib.fx)
        assert abs(ia.k1 - ib.k1) < 1e-7 and abs(ia.k2 - ib.k2) < 1e-7, tag
    dp = np.abs(g.points - o.points).max(axis=1)
    assert np.quantile(dp, 0.999) < 1e-7 and dp.max() < 1e-6, (tag, np.quantile(dp, 0.999), dp.max())


def _check_pcg_count(g, o):
    """PCG products within one per LM iteration: a run whose relative residual lands at the tolerance
    on some iteration can stop one product earlier or later under a different summation order."""
    assert abs(g.report["pcg_iteration_count"] - o.report["pcg_iteration_count"]) <= o.report["iteration_count"]


def test_plane500_fp64_matches_oracle(adjuster):
    p = synthetic.plane_problem()
    cfg = SolveConfig(max_iterations=4, linear_solver=abi.SOLVER_ITERATIVE, precision=abi.PRECISION_FP64,
                      pcg_relative_tolerance=1e-10)
    g, o = adjuster.solve(p, cfg), O.solve(p, cfg)
    _compare(g, o, "plane500")
    assert g.report["observability"] == o.report["observability"]
    _check_pcg_count(g, o)


def test_plane3000_geometry_fp64_matches_oracle(adjuster):
    p = synthetic.plane_problem(seed=5, cameras=3000, points=200_000, mean_track=6.5, extent=245.0,
                                free_intrinsics=False)
    cfg = SolveConfig(max_iterations=3, linear_solver=abi.SOLVER_ITERATIVE, precision=abi.PRECISION_FP64,
                      pcg_relative_tolerance=1e-10)
    g, o = adjuster.solve(p, cfg), O.solve(p, cfg)
    _compare(g, o, "plane3000_200k")
    assert g.report["observability"] == o.report["observability"]
    _check_pcg_count(g, o)


def _rot_y(a):
    c, s = np.cos(a), np.sin(a)
    return np.array([[c, 0.0, s], [0.0, 1.0, 0.0], [-s, 0.0, c]])


def f32_cache_fixture():
    """fixture() and perturbed() of the reference's sparse tests (main.rs:66-135) at the native API:
    world-to-camera poses (R, t) with centres -R^T t."""
    R = [np.eye(3), _rot_y(0.04), _rot_y(-0.05), _rot_y(0.07)]
    t = [np.zeros(3), np.array([0.62, 0.02, 0.05]), np.array([-0.51, 0.04, 0.09]), np.array([0.14, -0.37, 0.08])]
    idx = np.arange(24)
    X = np.stack([-1.0 + 0.4 * (idx % 6), -0.65 + 0.42 * (idx // 6), 4.0 + 0.16 * (idx % 5)], axis=1)
    fx, fy, cx, cy = 720.0, 710.0, 320.0, 240.0
    op, oc, pix = [], [], []
    for i, x in enumerate(X):
        for c in range(4):
            if c == 3 and i % 3 == 0:
                continue
            v = R[c] @ x + t[c]
            op.append(i)
            oc.append(c)
            pix.append([fx * v[0] / v[2] + cx, fy * v[1] / v[2] + cy])
    tp = [t[0]] + [t[c] + np.array([0.025 * c, -0.012 * c, 0.018]) for c in range(1, 4)]
    Xp = X + np.stack([0.018 * np.sin(idx), -0.015 * np.cos(0.7 * idx), 0.025 * np.sin(0.4 * idx)], axis=1)
    cam = CameraIntrinsics(model=abi.CAMERA_PINHOLE, fx=fx, fy=fy, cx=cx, cy=cy)
    n = len(op)
    return BundleProblem(
        rotations=np.array(R), centers=np.array([-Ri.T @ ti for Ri, ti in zip(R, tp)]),
        pose_variables=np.array([0, abi.POSE_FREE, abi.POSE_FREE, abi.POSE_FREE], dtype=np.uint32),
        intrinsics=[cam], points=Xp, point_fixed=np.zeros(24, dtype=np.uint8),
        observation_pose=np.array(oc, dtype=np.uint32), observation_intrinsic=np.zeros(n, dtype=np.uint32),
        observation_point=np.array(op, dtype=np.uint32), observation_pixel=np.array(pix),
        robust_loss=RobustLoss(abi.LOSS_SQUARED, 0.0, abi.RESIDUAL_PIXELS),
        gauge=Gauge.fixed_baseline(0, 1, float(np.linalg.norm(tp[1]))))


def test_fp32_records_preserve_the_bounded_solve(adjuster):
    """opt_in_f32_retained_cross_cache_preserves_the_bounded_solve (iterative_schur.rs:173-262)"""
    p = f32_cache_fixture()
    base = dict(max_iterations=12, linear_solver=abi.SOLVER_ITERATIVE)
    f64 = adjuster.solve(p, SolveConfig(precision=abi.PRECISION_FP64, **base))
    f32 = adjuster.solve(p, SolveConfig(precision=abi.PRECISION_MIXED, **base))
    assert f64.report["linear_solver"] == abi.SOLVER_ITERATIVE == f32.report["linear_solver"]
    assert f32.report["accepted_step_count"] == f64.report["accepted_step_count"]
    assert f32.report["rejected_step_count"] == f64.report["rejected_step_count"]
    drift = abs(f32.report["final_objective"] - f64.report["final_objective"]) / max(abs(f64.report["final_objective"]), 1.0)
    assert drift <= 1e-7, drift
    assert f64.report["final_objective"] < f64.report["initial_objective"]
    o = O.solve(p, SolveConfig(**base))
    assert f64.report["accepted_step_count"] == o.report["accepted_step_count"]
    assert abs(f64.report["final_objective"] - o.report["final_objective"]) <= 1e-9 * max(o.report["final_objective"], 1.0)
