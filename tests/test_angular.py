"""Angular residuals: the measured pixel's bearing against the camera point, for pinhole,
Brown-Conrady, fisheye and spherical cameras.

Pins, each against an independent restatement written here in numpy:
  * angular_projection (kernel/projection.rs:89-149): the residual is the angle between bearing and
    point times the unit direction in the bearing's tangent plane; the Jacobian matches central
    differences;
  * Camera::bearing of each model (openmvg-core camera/*.rs unproject): pixels projected by the
    model's forward equations come back as the point's direction;
  * the reference's capability fixture angular_controls_support_mixed_pose_masks
    (crates/openmvg-ba/tests/native_capabilities.rs:705-731): with fixed world controls and masks
    (free, translation-only, rotation-only) the angular solve recovers the true geometry, keeps held
    rotations and centres bit for bit, and reports the RMSE and objective of the independent angles.
The tests marked gpu solve the same problems through the CUDA library and compare with the oracle.
"""
import numpy as np
import pytest

import oracle as O
from openmvg_ba_cuda import BundleProblem, CameraIntrinsics, Gauge, RobustLoss, SolveConfig, abi

import test_pose_masks as M


def _angle(a, b):
    a = a / np.linalg.norm(a)
    b = b / np.linalg.norm(b)
    return np.arctan2(np.linalg.norm(np.cross(a, b)), a @ b)


def test_angular_projection_residual_and_jacobian():
    rng = np.random.Generator(np.random.PCG64(1))
    for _ in range(50):
        b = rng.normal(size=3)
        X = b / np.linalg.norm(b) * rng.uniform(1, 5) + rng.normal(scale=0.05, size=3)
        r, J = O.angular_projection(b, X)
        assert abs(np.hypot(*r) - _angle(b, X)) < 1e-12
        h = 1e-6
        for c in range(3):
            e = np.zeros(3)
            e[c] = h
            fd = (O.angular_projection(b, X + e)[0] - O.angular_projection(b, X - e)[0]) / (2 * h)
            assert np.max(np.abs(fd - J[:, c])) < 1e-7 * max(1.0, np.max(np.abs(J)))
    assert O.angular_projection([0.0, 0.0, 1.0], [0.0, 0.0, -2.0]) is None  # the antipode


def _fisheye_pixel(k, fx, fy, cx, cy, X):
    r = np.hypot(X[0], X[1])
    t = np.arctan2(r, X[2])
    td = t * (1 + k[0] * t ** 2 + k[1] * t ** 4 + k[2] * t ** 6 + k[3] * t ** 8)
    return np.array([fx * td * X[0] / r + cx, fy * td * X[1] / r + cy])


def _spherical_pixel(width, X):
    d = X / np.linalg.norm(X)
    lon, lat = np.arctan2(d[0], d[2]), np.arctan2(d[1], np.hypot(d[0], d[2]))
    h = width // 2
    return np.array([((lon + np.pi) * width / (2 * np.pi)) % width - 0.5, (lat + np.pi / 2) * h / np.pi - 0.5])


@pytest.mark.parametrize("model", ["pinhole", "brown", "fisheye", "spherical"])
def test_camera_bearing_inverts_the_projection(model):
    rng = np.random.Generator(np.random.PCG64(2))
    if model == "pinhole":
        cam = CameraIntrinsics(model=abi.CAMERA_PINHOLE, fx=620.0, fy=710.0, cx=320.0, cy=240.0)
        fwd = lambda X: np.array([620.0 * X[0] / X[2] + 320.0, 710.0 * X[1] / X[2] + 240.0])
    elif model == "brown":
        cal = M.BROWN
        cam = CameraIntrinsics(model=abi.CAMERA_BROWN_CONRADY, fx=cal["fx"], fy=cal["fy"], cx=cal["cx"], cy=cal["cy"],
                               radial_kind=abi.RADIAL_K1K2K3, k1=cal["k1"], k2=cal["k2"], k3=cal["k3"],
                               tangential_kind=abi.TANGENTIAL_P1P2, p1=cal["p1"], p2=cal["p2"])
        fwd = lambda X: M.project(cal, (np.eye(3), np.zeros(3)), X)
    elif model == "fisheye":
        k = (0.03, -0.01, 0.002, -0.0003)
        cam = CameraIntrinsics(model=abi.CAMERA_FISHEYE, fx=300.0, fy=300.0, cx=320.0, cy=240.0,
                               radial_kind=abi.RADIAL_K1K2K3K4, k1=k[0], k2=k[1], k3=k[2], k4=k[3])
        fwd = lambda X: _fisheye_pixel(k, 300.0, 300.0, 320.0, 240.0, X)
    else:
        cam = CameraIntrinsics(model=abi.CAMERA_SPHERICAL, width=1024, height=512)
        fwd = lambda X: _spherical_pixel(1024, X)
    for _ in range(40):
        if model == "spherical":
            X = rng.normal(size=3)
        elif model == "fisheye":
            X = np.array([*rng.uniform(-1.5, 1.5, size=2), rng.uniform(0.3, 1.0)])
        else:
            X = np.array([*rng.uniform(-0.4, 0.4, size=2), 1.0])
        b = O.camera_bearing(cam, *fwd(X))
        assert b is not None
        assert abs(np.linalg.norm(b) - 1.0) < 1e-14
        assert _angle(b, X) < 1e-9, (model, X, b)


def angular_controls_problem():
    """angular_controls_support_mixed_pose_masks (native_capabilities.rs:705-731)"""
    p = M.controls_problem(M.PINHOLE, False, [M.FREE, M.TRANSLATION, M.ROTATION])
    p.residual_space = abi.RESIDUAL_ANGULAR
    p.robust_loss = RobustLoss.squared()
    p.gauge = Gauge()
    return p


def check_angular_controls(problem, sol):
    truth, points = M.truth_poses(), M.truth_points()
    cal = M.PINHOLE
    sq = 0.0
    for o in range(problem.observation_count):  # the independent pinhole bearing equation
        v, p = int(problem.observation_pose[o]), int(problem.observation_point[o])
        u, w = problem.observation_pixel[o]
        m = np.array([(u - cal["cx"]) / cal["fx"], (w - cal["cy"]) / cal["fy"], 1.0])
        q = sol.rotations[v] @ (sol.points[p] - sol.centers[v])
        sq += _angle(m, q) ** 2
    rmse = np.sqrt(sq / problem.observation_count)
    assert rmse < 2e-7, rmse
    assert abs(sol.report["final_rmse"] - rmse) < 1e-10
    assert abs(sol.report["final_objective"] - 0.5 * sq) < 1e-9
    for v in range(3):
        M.assert_pose_recovered(sol.rotations[v], sol.centers[v], truth[v])
    assert np.array_equal(sol.points, points[:8])
    assert np.array_equal(sol.rotations[1], problem.rotations[1])
    assert np.array_equal(sol.centers[2], problem.centers[2])


def test_oracle_angular_controls_with_mixed_masks():
    p = angular_controls_problem()
    check_angular_controls(p, O.solve(p, M.config()))


def angular_ring(model: str, seed: int = 4):
    """A 12-camera ring seeing 600 points with 3-6 observations each, measured through the given
    camera model with 0.3 px noise; angular residuals with a Huber loss of 1e-3 rad."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n, P = 12, 600
    ang = 2 * np.pi * np.arange(n) / n
    C = np.stack([3.0 * np.cos(ang), 3.0 * np.sin(ang), 0.2 * np.sin(3 * ang)], axis=1)
    R = []
    for c in C:
        z = -c / np.linalg.norm(c)
        x = np.cross([0.0, 0.0, 1.0], z)
        x /= np.linalg.norm(x)
        R.append(np.stack([x, np.cross(z, x), z]))
    R = np.array(R)
    X = rng.uniform(-0.8, 0.8, size=(P, 3))
    if model == "fisheye":
        k = (0.02, -0.005, 0.001, 0.0)
        cam = CameraIntrinsics(model=abi.CAMERA_FISHEYE, fx=280.0, fy=280.0, cx=320.0, cy=240.0,
                               radial_kind=abi.RADIAL_K1K2K3, k1=k[0], k2=k[1], k3=k[2])
        fwd = lambda q: _fisheye_pixel(k, 280.0, 280.0, 320.0, 240.0, q)
    elif model == "spherical":
        cam = CameraIntrinsics(model=abi.CAMERA_SPHERICAL, width=2048, height=1024)
        fwd = lambda q: _spherical_pixel(2048, q)
    else:
        cal = M.BROWN
        cam = CameraIntrinsics(model=abi.CAMERA_BROWN_CONRADY, fx=cal["fx"], fy=cal["fy"], cx=cal["cx"], cy=cal["cy"],
                               radial_kind=abi.RADIAL_K1K2K3, k1=cal["k1"], k2=cal["k2"], k3=cal["k3"],
                               tangential_kind=abi.TANGENTIAL_P1P2, p1=cal["p1"], p2=cal["p2"])
        fwd = lambda q: M.project(cal, (np.eye(3), np.zeros(3)), q)
    obs_pt, obs_cam = [], []
    for p in range(P):
        for c in rng.choice(n, size=int(rng.integers(3, 7)), replace=False):
            obs_pt.append(p)
            obs_cam.append(int(c))
    pix = np.array([fwd(R[c] @ (X[p] - C[c])) for p, c in zip(obs_pt, obs_cam)])
    pix += rng.normal(0.0, 0.3, size=pix.shape)
    Rp = np.array([M.euler(*rng.normal(0.0, 0.005, size=3)) @ r for r in R])
    return BundleProblem(
        rotations=Rp, centers=C + rng.normal(0.0, 0.02, size=C.shape),
        pose_variables=np.full(n, abi.POSE_FREE, dtype=np.uint32), intrinsics=[cam],
        points=X + rng.normal(0.0, 0.01, size=X.shape), point_fixed=np.zeros(P, dtype=np.uint8),
        observation_pose=np.array(obs_cam, dtype=np.uint32), observation_intrinsic=np.zeros(len(obs_cam), dtype=np.uint32),
        observation_point=np.array(obs_pt, dtype=np.uint32), observation_pixel=pix,
        residual_space=abi.RESIDUAL_ANGULAR,
        robust_loss=RobustLoss(abi.LOSS_HUBER, 1e-3, abi.RESIDUAL_ANGULAR), gauge=Gauge())


@pytest.mark.parametrize("model", ["brown", "fisheye", "spherical"])
def test_oracle_angular_ring_converges(model):
    p = angular_ring(model)
    sol = O.solve(p, SolveConfig(max_iterations=50))
    r = sol.report
    assert r["status"] == abi.STATUS_CONVERGED, r["status"]
    assert r["final_objective"] < 0.5 * r["initial_objective"]
    assert r["final_rmse"] < 5e-3  # radians, with 0.3 px of pixel noise


def test_angular_problems_refuse_free_intrinsics():
    p = angular_ring("brown")
    p.intrinsics[0].variables = abi.INTRINSIC_FOCAL
    p.intrinsics[0].radial_kind = abi.RADIAL_K1K2
    with pytest.raises(Exception, match="angular BA requires fixed intrinsics"):
        O.solve(p, SolveConfig(max_iterations=5))


@pytest.mark.gpu
def test_gpu_angular_controls_with_mixed_masks(adjuster):
    p = angular_controls_problem()
    g = adjuster.solve(p, M.config())
    check_angular_controls(p, g)
    o = O.solve(p, M.config())
    assert np.max(np.abs(g.rotations - o.rotations)) < 1e-9 and np.max(np.abs(g.centers - o.centers)) < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("model", ["brown", "fisheye", "spherical"])
@pytest.mark.parametrize("solver", [abi.SOLVER_DIRECT, abi.SOLVER_ITERATIVE])
def test_gpu_angular_ring_matches_oracle(adjuster, model, solver):
    p = angular_ring(model)
    cfg = SolveConfig(max_iterations=50, linear_solver=solver, pcg_relative_tolerance=1e-10)
    g, o = adjuster.solve(p, cfg), O.solve(p, cfg)
    assert g.report["iteration_count"] == o.report["iteration_count"]
    assert abs(g.report["final_objective"] - o.report["final_objective"]) <= 1e-9 * o.report["final_objective"]
    for k in ("status", "observability", "inlier_count", "weak_point_count", "quarantined_point_count"):
        assert g.report[k] == o.report[k], k
    assert np.max(np.abs(g.rotations - o.rotations)) < 1e-7
    assert np.max(np.abs(g.centers - o.centers)) < 1e-7
