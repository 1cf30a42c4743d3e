"""Per-pose variable masks in calibrated solves: rotation-only, translation-only, full and fixed poses
in any mixture, and fixed world control points that leave every pose free (camera 0 included).

The scenes restate the reference's capability fixtures (crates/openmvg-ba/tests/native_capabilities.rs:
22-160: three cameras looking at twelve points, an independent pinhole / Brown-Conrady projection,
deterministic pose and point perturbations) and their assertions: noise-free measurements must be
recovered to 2e-5 in world units and 5e-6 in rotation-matrix norm, the reported RMSE and objective
must describe the independently projected residuals, held rotations and held centres must come back
bit for bit, and world controls must move camera 0 (native_capabilities.rs:426-660, 912-1017).

The oracle runs on the CPU; the same fixtures go through the CUDA library in the tests marked gpu,
which also compare it with the oracle.
"""
import numpy as np
import pytest

import oracle as O
from openmvg_ba_cuda import BundleProblem, CameraIntrinsics, Gauge, RobustLoss, SolveConfig, abi

WORLD_TOLERANCE = 2.0e-5
ROTATION_TOLERANCE = 5.0e-6
FREE, FIXED = abi.POSE_FREE, 0
TRANSLATION, ROTATION = abi.POSE_TRANSLATION, abi.POSE_ROTATION

PINHOLE = dict(fx=620.0, fy=710.0, cx=320.0, cy=240.0, k1=0.0, k2=0.0, k3=0.0, p1=0.0, p2=0.0)
BROWN = dict(PINHOLE, k1=-0.055, k2=0.008, k3=0.018, p1=0.0012, p2=-0.0008)


def euler(rx, ry, rz):
    """nalgebra's Rotation3::from_euler_angles(roll, pitch, yaw) = Rz(yaw) Ry(pitch) Rx(roll)."""
    cx, sx, cy, sy, cz, sz = np.cos(rx), np.sin(rx), np.cos(ry), np.sin(ry), np.cos(rz), np.sin(rz)
    Rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    return Rz @ Ry @ Rx


def truth_poses():
    spec = [((0.35, -0.20, 0.15), (0.03, -0.05, 0.02)),
            ((1.45, 0.12, 0.32), (-0.02, 0.07, -0.03)),
            ((-0.50, 0.90, -0.08), (0.04, 0.02, 0.05))]
    return [(euler(*r), np.array(c, dtype=float)) for c, r in spec]


def truth_points():
    i = np.arange(12, dtype=float)
    return np.stack([1.30 * np.sin(0.83 * i + 0.2), 0.85 * np.cos(1.17 * i - 0.3),
                     4.4 + 0.12 * i + 0.35 * np.sin(0.51 * i)], axis=1)


def perturb_pose(pose, mask, index):
    R, C = pose
    i = index + 1.0
    if mask & ROTATION:
        R = euler(0.009 * i, -0.007 * i, 0.006 * i) @ R
    if mask & TRANSLATION:
        C = C + np.array([0.035 * i, -0.022 * i, 0.018 * i])
    return R, C


def perturb_points(points):
    i = np.arange(len(points), dtype=float)
    return points + np.stack([0.028 * np.sin(i + 0.4), -0.022 * np.cos(i + 0.7), np.full_like(i, 0.035)], axis=1)


def project(cal, pose, X):
    """Independent normalized-coordinate Brown-Conrady projection in pixels."""
    R, C = pose
    q = R @ (X - C)
    assert q[2] > 0.0
    x, y = q[0] / q[2], q[1] / q[2]
    r2 = x * x + y * y
    radial = 1.0 + cal["k1"] * r2 + cal["k2"] * r2 * r2 + cal["k3"] * r2 * r2 * r2
    dx = x * radial + 2.0 * cal["p1"] * x * y + cal["p2"] * (r2 + 2.0 * x * x)
    dy = y * radial + cal["p1"] * (r2 + 2.0 * y * y) + 2.0 * cal["p2"] * x * y
    return np.array([cal["fx"] * dx + cal["cx"], cal["fy"] * dy + cal["cy"]])


def make_problem(cal, brown, poses, masks, points, fixed_points, measured_poses, measured_points, gauge=None,
                 observations=None):
    """BundleProblem with one fixed camera model, squared loss; observations (pose, point) default to
    every pose seeing every point, measured from the true geometry."""
    if observations is None:
        observations = [(v, p) for p in range(len(measured_points)) for v in range(len(measured_poses))]
    pix = np.array([project(cal, measured_poses[v], measured_points[p]) for v, p in observations])
    intr = CameraIntrinsics(model=abi.CAMERA_BROWN_CONRADY if brown else abi.CAMERA_PINHOLE,
                            fx=cal["fx"], fy=cal["fy"], cx=cal["cx"], cy=cal["cy"], width=640, height=480)
    if brown:
        intr.radial_kind, intr.k1, intr.k2, intr.k3 = abi.RADIAL_K1K2K3, cal["k1"], cal["k2"], cal["k3"]
        intr.tangential_kind, intr.p1, intr.p2 = abi.TANGENTIAL_P1P2, cal["p1"], cal["p2"]
    return BundleProblem(
        rotations=np.array([R for R, _ in poses]), centers=np.array([C for _, C in poses]),
        pose_variables=np.array(masks, dtype=np.uint32), intrinsics=[intr], points=np.array(points, dtype=float),
        point_fixed=np.full(len(points), 1 if fixed_points else 0, dtype=np.uint8),
        observation_pose=np.array([v for v, _ in observations], dtype=np.uint32),
        observation_intrinsic=np.zeros(len(observations), dtype=np.uint32),
        observation_point=np.array([p for _, p in observations], dtype=np.uint32), observation_pixel=pix,
        robust_loss=RobustLoss.squared(), gauge=gauge or Gauge())


def controls_problem(cal, brown, masks):
    """controls_problem (native_capabilities.rs:353-378): eight fixed world points, perturbed poses."""
    truth = truth_poses()[: len(masks)]
    points = truth_points()[:8]
    initial = [perturb_pose(p, m, i) for i, (p, m) in enumerate(zip(truth, masks))]
    return make_problem(cal, brown, initial, masks, points, True, truth, points)


def config(linear_solver=abi.SOLVER_DIRECT):
    return SolveConfig(max_iterations=100, function_tolerance=1e-12, gradient_tolerance=1e-11,
                       parameter_tolerance=1e-11, linear_solver=linear_solver)


def check_solution(problem, sol, cal):
    """The checks of solve_with_linear_solver (native_capabilities.rs:225-300): nothing held out, the
    intrinsics unchanged, an independent RMSE < 2e-5 px that the report restates, and the objective
    = 0.5 * sum of squared residuals."""
    assert len(sol.quarantined_points) == 0
    assert sol.report["observation_count"] == problem.observation_count
    sq = 0.0
    for o in range(problem.observation_count):
        v, p = int(problem.observation_pose[o]), int(problem.observation_point[o])
        r = project(cal, (sol.rotations[v], sol.centers[v]), sol.points[p]) - problem.observation_pixel[o]
        sq += float(r @ r)
    rmse = np.sqrt(sq / problem.observation_count)
    assert rmse < 2e-5, rmse
    assert abs(sol.report["final_rmse"] - rmse) < 1e-10
    assert abs(sol.report["final_objective"] - 0.5 * sq) < 1e-9


def assert_pose_recovered(R, C, truth):
    assert np.linalg.norm(C - truth[1]) < WORLD_TOLERANCE
    assert np.linalg.norm(R - truth[0]) < ROTATION_TOLERANCE


# ---- the fixtures: (name, problem builder, checks) ----------------------------------------------
def case_controls_free():
    """fixed_world_controls_optimize_every_free_pose (native_capabilities.rs:425-441)"""
    masks = [FREE] * 3
    return controls_problem(PINHOLE, False, masks), PINHOLE


def case_mixed_masks():
    """mixed_pose_masks_preserve_rotations_and_camera_centers (native_capabilities.rs:513-532)"""
    masks = [FREE, TRANSLATION, ROTATION]
    return controls_problem(PINHOLE, False, masks), PINHOLE


def case_known_rotations_brown():
    """fixed_brown_controls_with_known_rotations_keep_world_frame (native_capabilities.rs:569-579)"""
    masks = [TRANSLATION] * 3
    return controls_problem(BROWN, True, masks), BROWN


def case_known_rotation_one_camera():
    """known_rotation_does_not_lock_another_free_camera_rotation (native_capabilities.rs:581-657)"""
    truth, points = truth_poses(), truth_points()
    masks = [FREE, TRANSLATION, FREE]
    initial = [perturb_pose(p, m, i) for i, (p, m) in enumerate(zip(truth, masks))]
    return make_problem(PINHOLE, False, initial, masks, perturb_points(points), False, truth, points), PINHOLE


def case_single_camera():
    """single_camera_world_controls_recover_the_free_pose (native_capabilities.rs:936-967)"""
    truth, points = truth_poses()[:1], truth_points()[:6]
    initial = [perturb_pose(truth[0], FREE, 0)]
    return make_problem(PINHOLE, False, initial, [FREE], points, True, truth, points), PINHOLE


def case_fixed_baseline_brown():
    """fixed_brown_pixels_recover_metric_geometry_without_changing_calibration (native_capabilities.rs:
    380-423)"""
    truth, points = truth_poses(), truth_points()
    masks = [FIXED, FREE, FREE]
    initial = [perturb_pose(p, m, i) for i, (p, m) in enumerate(zip(truth, masks))]
    initial[1] = (initial[1][0], truth[1][1].copy())
    distance = float(np.linalg.norm(truth[1][1] - truth[0][1]))
    return make_problem(BROWN, True, initial, masks, perturb_points(points), False, truth, points,
                        gauge=Gauge.fixed_baseline(0, 1, distance)), BROWN


def _check_case(name, problem, sol, cal):
    check_solution(problem, sol, cal)
    truth, points = truth_poses(), truth_points()
    R_in, C_in = problem.rotations, problem.centers
    if name == "controls_free":
        for v in range(3):
            assert_pose_recovered(sol.rotations[v], sol.centers[v], truth[v])
        assert np.array_equal(sol.points, points[:8])
        # world controls must not make camera 0 an implicit fixed camera
        assert np.linalg.norm(sol.centers[0] - C_in[0]) > 0.02
        assert np.linalg.norm(sol.rotations[0] - R_in[0]) > 0.005
    elif name == "mixed_masks":
        for v in range(3):
            assert_pose_recovered(sol.rotations[v], sol.centers[v], truth[v])
        assert np.array_equal(sol.points, points[:8])
        assert np.array_equal(sol.rotations[1], R_in[1])  # held rotation, bit for bit
        assert np.array_equal(sol.centers[2], C_in[2])    # held centre, bit for bit
        # rotation-only refinement holds C, so t = -R C changes
        t_out = -sol.rotations[2] @ sol.centers[2]
        t_in = -R_in[2] @ C_in[2]
        assert np.linalg.norm(t_out - t_in) > 0.005
    elif name == "known_rotations_brown":
        for v in range(3):
            assert_pose_recovered(sol.rotations[v], sol.centers[v], truth[v])
            assert np.array_equal(sol.rotations[v], R_in[v])
        assert np.array_equal(sol.points, points[:8])
    elif name == "known_rotation_one_camera":
        assert np.array_equal(sol.rotations[1], R_in[1])
        for v in range(3):
            assert np.linalg.norm(sol.rotations[v] - truth[v][0]) < ROTATION_TOLERANCE
        # similarity up to scale and translation (the known rotation removes the rotational gauge)
        est, tru = sol.centers, np.array([c for _, c in truth])
        em, tm = est.mean(axis=0), tru.mean(axis=0)
        scale = float(np.sum((est - em) * (tru - tm)) / np.sum((est - em) ** 2))
        assert np.isfinite(scale) and scale > 0.0
        shift = tm - scale * em
        assert np.all(np.linalg.norm(scale * est + shift - tru, axis=1) < WORLD_TOLERANCE)
        assert np.all(np.linalg.norm(scale * sol.points + shift - points, axis=1) < WORLD_TOLERANCE)
    elif name == "single_camera":
        assert_pose_recovered(sol.rotations[0], sol.centers[0], truth[0])
        assert np.array_equal(sol.points, points[:6])
        assert sol.report["observability"] == abi.OBS_FULL_RANK
        assert np.linalg.norm(sol.centers[0] - C_in[0]) > 0.02
        assert np.linalg.norm(sol.rotations[0] - R_in[0]) > 0.005
    elif name == "fixed_baseline_brown":
        for v in range(3):
            assert_pose_recovered(sol.rotations[v], sol.centers[v], truth[v])
        assert np.all(np.linalg.norm(sol.points - points, axis=1) < WORLD_TOLERANCE)
        assert np.array_equal(sol.rotations[0], R_in[0])
        assert np.array_equal(sol.centers[0], C_in[0])
        d = np.linalg.norm(sol.centers[1] - sol.centers[0])
        assert abs(d - problem.gauge.distance) < 1e-10
    else:
        raise AssertionError(name)


CASES = {
    "controls_free": case_controls_free,
    "mixed_masks": case_mixed_masks,
    "known_rotations_brown": case_known_rotations_brown,
    "known_rotation_one_camera": case_known_rotation_one_camera,
    "single_camera": case_single_camera,
    "fixed_baseline_brown": case_fixed_baseline_brown,
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_recovers_masked_fixtures(name):
    problem, cal = CASES[name]()
    sol = O.solve(problem, config())
    _check_case(name, problem, sol, cal)


def test_oracle_direct_and_iterative_agree_with_mixed_masks():
    """mixed_controls_direct_and_iterative_agree_on_geometry (native_capabilities.rs:911-934)"""
    problem, cal = case_mixed_masks()
    d = O.solve(problem, config(abi.SOLVER_DIRECT))
    it = O.solve(problem, config(abi.SOLVER_ITERATIVE))
    _check_case("mixed_masks", problem, it, cal)
    assert np.max(np.linalg.norm(it.centers - d.centers, axis=1)) < 1e-6
    assert np.max(np.abs(it.rotations - d.rotations)) < 1e-6
    assert np.array_equal(it.points, d.points)
    assert d.report["linear_solver"] == abi.SOLVER_DIRECT and it.report["linear_solver"] == abi.SOLVER_ITERATIVE


def test_translation_only_resolves_auto_to_direct():
    """A translation-only solve resolves Auto to the direct solver (native/mod.rs:398-407)."""
    problem, _ = case_known_rotations_brown()
    iterative, _, _ = O.execution_plan(problem, config(abi.SOLVER_AUTO))
    assert not iterative
    sol = O.solve(problem, config(abi.SOLVER_AUTO))
    assert sol.report["linear_solver"] == abi.SOLVER_DIRECT


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_recovers_masked_fixtures_like_the_oracle(adjuster, name):
    problem, cal = CASES[name]()
    g = adjuster.solve(problem, config())
    _check_case(name, problem, g, cal)
    o = O.solve(problem, config())
    assert np.max(np.abs(g.rotations - o.rotations)) < 1e-9
    assert np.max(np.abs(g.centers - o.centers)) < 1e-9
    assert np.max(np.abs(g.points - o.points)) < 1e-9
    assert g.report["iteration_count"] == o.report["iteration_count"]
    assert g.report["observability"] == o.report["observability"]


@pytest.mark.gpu
@pytest.mark.parametrize("solver,matvec", [(abi.SOLVER_DIRECT, abi.MATVEC_AUTO), (abi.SOLVER_ITERATIVE, abi.MATVEC_AUTO),
                                           (abi.SOLVER_ITERATIVE, abi.MATVEC_IMPLICIT),
                                           (abi.SOLVER_ITERATIVE, abi.MATVEC_EXPLICIT)])
def test_gpu_masked_ring_matches_oracle(adjuster, solver, matvec):
    """A 20-camera ring with every mask kind (full, rotation-only, translation-only, fixed), 5% gross
    outliers and Huber loss, direct and iterative (matrix-free and explicit S), against the oracle at
    the solve-parity tolerances. Along this trajectory a track-2 point is pulled within 3e-4 of a
    camera centre (cond(V) about 1e9): the point coupling must go through the point block's factor,
    as the reference's cached solves do, for the products to stay accurate there."""
    from openmvg_ba_cuda import synthetic
    kinds = [FREE, ROTATION, TRANSLATION, FREE, FIXED]
    p = synthetic.ring_problem(seed=5, radius=3.0,
                               pose_variables=np.array([kinds[i % len(kinds)] for i in range(20)]))
    cfg = SolveConfig(max_iterations=30, linear_solver=solver, matvec=matvec, pcg_relative_tolerance=1e-10)
    g = adjuster.solve(p, cfg)
    o = O.solve(p, cfg)
    assert abs(g.report["final_objective"] - o.report["final_objective"]) <= 1e-9 * abs(o.report["final_objective"])
    assert g.report["iteration_count"] == o.report["iteration_count"]
    # poses within 1e-7, or within 10x the oracle's own spread under a different (fixed) grouping of
    # its sums where the iterative trajectory amplifies rounding
    O.set_shards(7)
    try:
        o2 = O.solve(p, cfg)
    finally:
        O.set_shards(0)
    for a, b, c in ((g.rotations, o.rotations, o2.rotations), (g.centers, o.centers, o2.centers)):
        assert np.max(np.abs(a - b)) <= max(1e-7, 10.0 * np.max(np.abs(c - b))), (np.max(np.abs(a - b)),
                                                                                np.max(np.abs(c - b)))
    held_rot = p.pose_variables == TRANSLATION
    held_cen = p.pose_variables == ROTATION
    assert np.array_equal(g.rotations[held_rot], p.rotations[held_rot])
    assert np.array_equal(g.centers[held_cen], p.centers[held_cen])


@pytest.mark.gpu
def test_gpu_tile_product_is_linear_and_symmetric_at_an_ill_conditioned_point(adjuster):
    """The masked ring's state after 14 oracle iterations holds a track-2 point within 3e-4 of a
    camera centre (cond(V) about 1.7e9). There the matrix-free tile product, which applies the point
    block through its inverse factor (N^T N b), stays linear and symmetric to 1e-9 of its size; a
    product with the explicit inverse carried rounding noise near 3e-5 of its size that changed with
    the vector, which slowed PCG and moved the LM trajectory off the reference's."""
    import copy
    from openmvg_ba_cuda import synthetic
    kinds = [FREE, ROTATION, TRANSLATION, FREE, FIXED]
    p = synthetic.ring_problem(seed=5, radius=3.0,
                               pose_variables=np.array([kinds[i % len(kinds)] for i in range(20)]))
    cfg = SolveConfig(max_iterations=14, linear_solver=abi.SOLVER_ITERATIVE, pcg_relative_tolerance=1e-10)
    o = O.solve(p, cfg)
    q = copy.deepcopy(p)
    q.rotations, q.centers, q.points = o.rotations.copy(), o.centers.copy(), o.points.copy()
    D = adjuster.debug_schur_product(q, None)
    rng = np.random.default_rng(1)
    for lam in (0.0, o.report["final_damping"]):
        x1, x2 = rng.normal(size=D), rng.normal(size=D)
        y1, _ = adjuster.debug_schur_product(q, x1, lam)
        y2, _ = adjuster.debug_schur_product(q, x2, lam)
        y12, _ = adjuster.debug_schur_product(q, x1 + x2, lam)
        size = max(np.max(np.abs(y1)), np.max(np.abs(y2)))
        assert np.max(np.abs(y12 - y1 - y2)) <= 1e-9 * size, (lam, np.max(np.abs(y12 - y1 - y2)) / size)
        asym = abs(x2 @ y1 - x1 @ y2)
        assert asym <= 1e-9 * np.linalg.norm(x1) * np.linalg.norm(y2), (lam, asym)
