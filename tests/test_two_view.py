"""Two-view bundle adjustment (native/two_view.rs, kernel/two_view/*): a problem with two poses, the
anchor fixed and the other free, every point seen once by each camera, goes to the dedicated two-view
LM over the 5 coordinates of the free pose (rotation and the direction of a fixed-length baseline).

The fixtures restate the reference's two-view tests (crates/openmvg-ba/tests/bundle_adjustment.rs:
44-291) at the native API: a 30-point scene with a true relative pose, a perturbed initial pose of the
same baseline and perturbed points, pinhole pixels (the second camera's skew dropped: the ABI carries
none) or angular bearings of the same pixels. Checks: the cost falls, the final RMSE is below 5% of
the initial, the pose has full rank with no weak point and keeps its baseline to 1e-12
(assert_report_improves, :86-113); point-only errors still take accepted steps (:208-248); a Cauchy
loss keeps the pose closer to the truth than squared loss under 20% outliers (:250-290). The tests
marked gpu run the same problems through the CUDA library and compare them with the oracle.
"""
import numpy as np
import pytest

import oracle as O
from openmvg_ba_cuda import BundleProblem, CameraIntrinsics, Gauge, RobustLoss, SolveConfig, abi


def exp_so3(w):
    w = np.asarray(w, dtype=float)
    th = np.linalg.norm(w)
    K = np.array([[0, -w[2], w[1]], [w[2], 0, -w[0]], [-w[1], w[0], 0]]) / th
    return np.eye(3) + np.sin(th) * K + (1 - np.cos(th)) * K @ K


def fixture():
    """fixture (bundle_adjustment.rs:44-84): truth (R, t), initial (R, t), truth points, initial points."""
    R_t, t_t = exp_so3([0.04, -0.08, 0.025]), np.array([0.8, 0.1, 0.15])
    idx = np.arange(30)
    pts = np.stack([(idx % 6) * 0.22 - 0.55, (idx // 6) * 0.18 - 0.36, 3.0 + 0.07 * idx], axis=1)
    baseline = np.linalg.norm(t_t)
    raw = np.array([0.79, 0.125, 0.12])
    R_i, t_i = exp_so3([0.025, -0.018, 0.012]) @ R_t, baseline * raw / np.linalg.norm(raw)
    ph = idx.astype(float)
    init = pts + np.stack([0.025 * np.sin(ph), 0.02 * np.cos(0.7 * ph), 0.04 * np.sin(0.3 * ph)], axis=1)
    return (R_t, t_t), (R_i, t_i), pts, init


CAM1 = dict(fx=500.0, fy=510.0, cx=320.0, cy=240.0)
CAM2 = dict(fx=520.0, fy=515.0, cx=315.0, cy=238.0)


def pix(cam, X):
    return np.array([cam["fx"] * X[0] / X[2] + cam["cx"], cam["fy"] * X[1] / X[2] + cam["cy"]])


def two_view_problem(angular=False, loss=None, outliers=False, point_only=False, same_camera=False):
    (R_t, t_t), (R_i, t_i), truth, init = fixture()
    c1, c2 = (CAM1, CAM1) if same_camera else (CAM1, CAM2)
    obs1 = np.array([pix(c1, X) for X in truth])
    obs2 = np.array([pix(c2, R_t @ X + t_t) for X in truth])
    if outliers:
        obs2[::5] += [120.0, -80.0]
    if point_only:
        R_i, t_i = R_t, t_t
        ph = np.arange(30, dtype=float)
        init = truth + np.stack([1e-3 * np.sin(ph), 8e-4 * np.cos(0.7 * ph), 1.2e-3 * np.sin(0.3 * ph)], axis=1)
    P = len(truth)
    intr = [CameraIntrinsics(model=abi.CAMERA_PINHOLE, **c1), CameraIntrinsics(model=abi.CAMERA_PINHOLE, **c2)]
    baseline = float(np.linalg.norm(t_i))
    if loss is None:
        loss = RobustLoss(abi.LOSS_SQUARED, 0.0, abi.RESIDUAL_ANGULAR if angular else abi.RESIDUAL_PIXELS)
    return BundleProblem(
        rotations=np.array([np.eye(3), R_i]), centers=np.array([np.zeros(3), -R_i.T @ t_i]),
        pose_variables=np.array([0, abi.POSE_FREE], dtype=np.uint32), intrinsics=intr, points=init,
        point_fixed=np.zeros(P, dtype=np.uint8),
        observation_pose=np.concatenate([np.zeros(P), np.ones(P)]).astype(np.uint32),
        observation_intrinsic=np.concatenate([np.zeros(P), np.ones(P)]).astype(np.uint32),
        observation_point=np.concatenate([np.arange(P), np.arange(P)]).astype(np.uint32),
        observation_pixel=np.vstack([obs1, obs2]),
        residual_space=abi.RESIDUAL_ANGULAR if angular else abi.RESIDUAL_PIXELS, robust_loss=loss,
        gauge=Gauge.fixed_baseline(0, 1, baseline)), (R_t, t_t)


def check_improves(problem, sol):
    """assert_report_improves (bundle_adjustment.rs:86-113) on the native report."""
    r = sol.report
    assert r["final_objective"] < r["initial_objective"]
    assert r["final_rmse"] < 0.05 * r["initial_rmse"]
    assert r["final_damping"] > 0.0 and np.isfinite(r["final_damping"])
    assert r["status"] != abi.STATUS_DEGENERATE
    assert r["observability"] == abi.OBS_FULL_RANK
    assert r["weak_point_count"] == 0
    assert r["linear_solver"] == abi.SOLVER_DIRECT
    assert r["reduced_dimension"] == 5
    b0 = np.linalg.norm(problem.centers[1] - problem.centers[0])
    assert abs(np.linalg.norm(sol.centers[1] - sol.centers[0]) - b0) < 1e-12
    assert np.array_equal(sol.rotations[0], problem.rotations[0]) and np.array_equal(sol.centers[0], problem.centers[0])


def pose_error(sol, truth):
    R_t, t_t = truth
    R, C = sol.rotations[1], sol.centers[1]
    t = -R @ C
    rot = np.arccos(np.clip((np.trace(R @ R_t.T) - 1) / 2, -1, 1))
    return rot + np.arccos(np.clip(t @ t_t / np.linalg.norm(t) / np.linalg.norm(t_t), -1, 1))


@pytest.mark.parametrize("angular", [False, True])
def test_oracle_two_view_refines_pose_and_points(angular):
    p, _ = two_view_problem(angular)
    check_improves(p, O.solve(p, SolveConfig(max_iterations=40)))


def test_oracle_two_view_point_only_error_takes_steps():
    p, _ = two_view_problem(point_only=True, same_camera=True)
    sol = O.solve(p, SolveConfig(max_iterations=10, gradient_tolerance=1e-2, parameter_tolerance=1e-14,
                                 function_tolerance=1e-14))
    assert sol.report["accepted_step_count"] > 0
    assert sol.report["final_objective"] < sol.report["initial_objective"]


def test_oracle_two_view_cauchy_protects_the_pose_from_outliers():
    cfg = SolveConfig(max_iterations=35)
    l2, truth = two_view_problem(outliers=True, same_camera=True)
    robust, _ = two_view_problem(outliers=True, same_camera=True, loss=RobustLoss.cauchy(2.0))
    assert pose_error(O.solve(robust, cfg), truth) < pose_error(O.solve(l2, cfg), truth)


def test_a_third_camera_leaves_the_two_view_path():
    """With an unobserved third camera the problem is no longer two-view: the multi-view path solves
    it (the FixedBaseline camera has the same 5 coordinates there) and reaches the two-view optimum."""
    p, _ = two_view_problem()
    two = O.solve(p, SolveConfig(max_iterations=40))
    p.rotations = np.vstack([p.rotations, p.rotations[:1]])
    p.centers = np.vstack([p.centers, [[0.0, 0.5, 0.0]]])
    p.pose_variables = np.array([0, abi.POSE_FREE, 0], dtype=np.uint32)
    multi = O.solve(p, SolveConfig(max_iterations=40))
    assert multi.report["reduced_dimension"] == 5
    assert abs(multi.report["final_objective"] - two.report["final_objective"]) <= 1e-6 * two.report["initial_objective"]
    assert np.max(np.abs(multi.centers[:2] - two.centers)) < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["pixel", "angular", "point_only", "cauchy_outliers"])
def test_gpu_two_view_matches_oracle(adjuster, case):
    if case == "pixel":
        p, _ = two_view_problem()
        cfg = SolveConfig(max_iterations=40)
    elif case == "angular":
        p, _ = two_view_problem(angular=True)
        cfg = SolveConfig(max_iterations=40)
    elif case == "point_only":
        p, _ = two_view_problem(point_only=True, same_camera=True)
        cfg = SolveConfig(max_iterations=10, gradient_tolerance=1e-2, parameter_tolerance=1e-14,
                          function_tolerance=1e-14)
    else:
        p, _ = two_view_problem(outliers=True, same_camera=True, loss=RobustLoss.cauchy(2.0))
        cfg = SolveConfig(max_iterations=35)
    g, o = adjuster.solve(p, cfg), O.solve(p, cfg)
    for k in ("status", "iteration_count", "accepted_step_count", "observability", "weak_point_count",
              "linear_solver", "reduced_dimension", "inlier_count"):
        assert g.report[k] == o.report[k], k
    # 1e-9 relative, with a rounding floor for a cost near zero (noise-free pixels): residuals
    # computed a few ulps apart (1e-13 px on 640-px coordinates) move the cost by at most
    # sqrt(2 f m) * 1e-13 for m residual components
    f = o.report["final_objective"]
    floor = np.sqrt(2.0 * f * 2 * p.observation_count) * 1e-13
    assert abs(g.report["final_objective"] - f) <= 1e-9 * f + floor
    assert np.max(np.abs(g.rotations - o.rotations)) < 1e-9
    assert np.max(np.abs(g.centers - o.centers)) < 1e-9
    assert np.max(np.abs(g.points - o.points)) < 1e-8
    if case in ("pixel", "angular"):
        check_improves(p, g)
