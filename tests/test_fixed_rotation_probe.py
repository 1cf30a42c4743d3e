"""The translation-only observability probe (probe_fixed_rotation_observability) and the native
preflight built on it.

The cases restate the reference's unit tests (crates/openmvg-ba/src/kernel/fixed_rotation/tests.rs:
40-531) with their fixtures and assertions: a four-camera, 24-point synthetic scene with identity
rotations, capped selections, long-track coverage, unprojectable and numerically singular points, a
point collapsed onto a camera centre, a distant camera, two-view links that leave a baseline length
free, a camera without tracks, invalid limits, and long chains of two-view tracks. The oracle runs them
on the CPU; the tests marked gpu run the same cases through the CUDA library (host selection and
elimination, device factorization) and compare every field with the oracle.
"""
import numpy as np
import pytest

import oracle as O
from openmvg_ba_cuda import abi
from openmvg_ba_cuda.fixed_rotation import FixedRotationProblem, ProbeOptions

CERTIFIED = abi.PROBE_FULL_RANK_CERTIFIED
COVERAGE = abi.PROBE_INSUFFICIENT_CAMERA_COVERAGE
WEAK = abi.PROBE_WEAK_POINT_GEOMETRY
FACTOR = abi.PROBE_SPARSE_FACTORIZATION_FAILED


def _observe(camera, point, center):
    depth = point[2] - center[2]
    return (camera, 800.0 * (point[0] - center[0]) / depth, 800.0 * (point[1] - center[1]) / depth)


def synthetic_problem():
    """synthetic_problem (tests.rs:40-100)"""
    centers = [[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [1.0, 1.0, 0.0]]
    points = [[-0.5 + 0.35 * (i % 6), -0.4 + 0.3 * (i // 6), 4.0 + 0.15 * ((i * 7) % 5)] for i in range(24)]
    tracks = [[_observe(c, p, centers[c]) for c in range(len(centers))] for p in points]
    n = len(centers)
    return FixedRotationProblem(rotations=np.tile(np.eye(3), (n, 1, 1)), centers=np.array(centers),
                                points=np.array(points), intrinsics=np.tile([800.0, 800.0, 0, 0, 0, 0, 0, 0, 0], (n, 1)),
                                tracks=tracks, fixed_cameras=np.zeros(n, dtype=np.uint8), anchor=0, scale_camera=1)


def chain_problem(camera_count):
    """The two-view chains of tests.rs:382-531: each adjacent pair of cameras on a line shares three
    tracks, which fix each baseline's direction but not its length."""
    centers = [[float(c), 0.0, 0.0] for c in range(camera_count)]
    points, tracks = [], []
    for c in range(camera_count - 1):
        for s in range(3):
            p = [c + 0.25 + 0.2 * s, -0.3 + 0.3 * s, 5.0 + 0.2 * s]
            points.append(p)
            tracks.append([(v, 800.0 * (p[0] - centers[v][0]) / p[2], 800.0 * p[1] / p[2]) for v in (c, c + 1)])
    n = camera_count
    return FixedRotationProblem(rotations=np.tile(np.eye(3), (n, 1, 1)), centers=np.array(centers),
                                points=np.array(points), intrinsics=np.tile([800.0, 800.0, 0, 0, 0, 0, 0, 0, 0], (n, 1)),
                                tracks=tracks, fixed_cameras=np.zeros(n, dtype=np.uint8), anchor=0, scale_camera=1)


def case_capped_subset():
    """capped_sparse_probe_certifies_a_well_constrained_subset (tests.rs:101-121)"""
    return synthetic_problem(), ProbeOptions(max_tracks=8, max_observations=32)


def check_capped_subset(r):
    assert r["status"] == CERTIFIED
    assert r["pose_dimension"] == 8
    assert r["selected_tracks"] == 8
    assert r["covered_free_cameras"] == 3
    assert r["reduced_nonzeros"] > 0 and r["factor_nonzeros"] > 0


def case_incomplete_cap():
    """an_incomplete_cap_is_not_mislabeled_rank_deficient (tests.rs:123-143)"""
    return synthetic_problem(), ProbeOptions(max_observations=2)


def check_incomplete_cap(r):
    assert r["status"] == COVERAGE
    assert r["selected_tracks"] == 0


def case_long_tracks():
    """bounded_long_track_exception_covers_free_cameras (tests.rs:145-169)"""
    return synthetic_problem(), ProbeOptions(max_observations_per_track=3, max_coverage_observations_per_track=4,
                                             max_tracks=8, max_observations=32)


def check_long_tracks(r):
    assert r["covered_free_cameras"] == 3
    assert r["selected_tracks"] > 0
    assert r["status"] != COVERAGE


def case_unprojectable():
    """an_unprojectable_point_is_weak_instead_of_aborting_the_probe (tests.rs:171-185)"""
    p = synthetic_problem()
    p.points[0] = p.centers[0]
    return p, ProbeOptions()


def check_unprojectable(r):
    assert r["weak_point_count"] == 1
    assert r["covered_free_cameras"] == 3


def case_singular_point():
    """a_numerically_singular_point_is_weak_instead_of_corrupting_the_rank (tests.rs:187-222)"""
    p = synthetic_problem()
    p.centers[3] = [0.0, 0.0, 1.0]
    for track, point in zip(p.tracks, p.points):
        track[3] = _observe(3, point, p.centers[3])
    point = np.array([1e-7, 0.0, 5.0])
    p.points = np.vstack([p.points, point])
    p.tracks.append([_observe(0, point, p.centers[0]), _observe(3, point, p.centers[3])])
    return p, ProbeOptions()


def check_singular_point(r):
    assert r["weak_point_count"] == 1
    assert r["status"] == CERTIFIED


def collapsed_point_problem(step):
    """the_probe_certifies_through_a_point_collapsed_onto_a_camera_centre (tests.rs:224-266)"""
    p = synthetic_problem()
    p.centers[3] = [0.5, 0.5, -0.1]
    for track, point in zip(p.tracks, p.points):
        depth = point[2] + 0.1
        track[3] = (3, 800.0 * (point[0] - 0.5) / depth, 800.0 * (point[1] - 0.5) / depth)
    p.points = np.vstack([p.points, [1e-7, 1e-7, 1e-7 * (1.0 + 0.01 * step)]])
    p.tracks.append([(0, 40.0, -30.0), (3, -60.0, 20.0)])
    return p


def case_distant_camera():
    """a_distant_camera_is_not_mislabeled_rank_deficient (tests.rs:268-292)"""
    p = synthetic_problem()
    distance = 1.0e4
    p.centers[3] = [0.5, 0.5, -distance]
    for track, point in zip(p.tracks, p.points):
        depth = point[2] + distance
        track[3] = (3, 800.0 * (point[0] - 0.5) / depth, 800.0 * (point[1] - 0.5) / depth)
    return p, ProbeOptions()


def check_distant_camera(r):
    assert r["weak_point_count"] == 0
    assert r["status"] == CERTIFIED


def case_two_view_link():
    """a_camera_linked_by_two_view_tracks_to_one_neighbour_is_not_certified (tests.rs:294-339)"""
    p = synthetic_problem()
    p.tracks = [[o for o in t if o[0] != 3] for t in p.tracks]
    extra = []
    for i in range(6):
        point = [0.2 + 0.1 * i, 0.3 - 0.05 * i, 3.0 + 0.2 * (i % 3)]
        extra.append(point)
        p.tracks.append([_observe(c, point, p.centers[c]) for c in (2, 3)])
    p.points = np.vstack([p.points, extra])
    return p, ProbeOptions()


def check_two_view_link(r):
    assert r["weak_point_count"] == 0
    assert r["status"] != CERTIFIED


def case_camera_without_tracks():
    """a_camera_without_any_track_fails_closed (tests.rs:341-360)"""
    p = synthetic_problem()
    p.tracks = [[o for o in t if o[0] != 3] for t in p.tracks]
    return p, ProbeOptions()


def check_camera_without_tracks(r):
    assert r["status"] == COVERAGE


def case_large_chain():
    """large_sparse_chain_is_bounded_and_fails_closed (tests.rs:381-455)"""
    return chain_problem(2307), ProbeOptions()


def check_large_chain(r):
    assert r["pose_dimension"] == 3 * 2307 - 4
    assert r["status"] in (FACTOR, WEAK)
    assert r["reduced_nonzeros"] < 100_000
    assert r["factor_nonzeros"] < 100_000


CASES = {
    "capped_subset": (case_capped_subset, check_capped_subset),
    "incomplete_cap": (case_incomplete_cap, check_incomplete_cap),
    "long_tracks": (case_long_tracks, check_long_tracks),
    "unprojectable": (case_unprojectable, check_unprojectable),
    "singular_point": (case_singular_point, check_singular_point),
    "distant_camera": (case_distant_camera, check_distant_camera),
    "two_view_link": (case_two_view_link, check_two_view_link),
    "camera_without_tracks": (case_camera_without_tracks, check_camera_without_tracks),
    "large_chain": (case_large_chain, check_large_chain),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_probe_matches_the_reference_cases(name):
    make, check = CASES[name]
    problem, options = make()
    check(O.probe_fixed_rotation(problem, options))


def test_oracle_probe_certifies_through_a_collapsed_point():
    for step in range(20):
        r = O.probe_fixed_rotation(collapsed_point_problem(step), ProbeOptions())
        assert r["status"] == CERTIFIED, step


@pytest.mark.parametrize("cameras", [3, 4, 8, 40])
def test_oracle_probe_never_certifies_a_two_view_chain(cameras):
    """a_chain_of_two_view_tracks_is_not_certified_at_any_length (tests.rs:457-531)"""
    assert O.probe_fixed_rotation(chain_problem(cameras))["status"] != CERTIFIED


def test_oracle_probe_rejects_invalid_limits():
    """invalid_probe_limits_are_rejected (tests.rs:362-379)"""
    with pytest.raises(ValueError, match="invalid fixed-rotation observability probe limits"):
        O.probe_fixed_rotation(synthetic_problem(), ProbeOptions(max_factor_nonzeros=0))


# ---- the native preflight ----------------------------------------------------------------------
def translation_only_problem(gauge_fixed_baseline=True, fixed_points=False, masks=None):
    """A ring of 8 pinhole cameras with known rotations (translation-only masks) seeing 300 points."""
    from openmvg_ba_cuda import BundleProblem, CameraIntrinsics, Gauge, RobustLoss
    rng = np.random.Generator(np.random.PCG64(3))
    n, P = 8, 300
    ang = 2 * np.pi * np.arange(n) / n
    C = np.stack([4.0 * np.cos(ang), 4.0 * np.sin(ang), 0.3 * np.sin(2 * ang)], axis=1)
    R = []
    for c in C:  # look at the origin
        z = -c / np.linalg.norm(c)
        x = np.cross([0.0, 0.0, 1.0], z)
        x /= np.linalg.norm(x)
        R.append(np.stack([x, np.cross(z, x), z]))
    R = np.array(R)
    X = rng.uniform(-1.0, 1.0, size=(P, 3))
    obs_pt, obs_cam = [], []
    for p in range(P):
        for c in rng.choice(n, size=int(rng.integers(2, 6)), replace=False):
            obs_pt.append(p)
            obs_cam.append(int(c))
    obs_pt, obs_cam = np.array(obs_pt, dtype=np.uint32), np.array(obs_cam, dtype=np.uint32)
    q = np.einsum("nij,nj->ni", R[obs_cam], X[obs_pt] - C[obs_cam])
    pix = np.stack([600.0 * q[:, 0] / q[:, 2] + 320.0, 600.0 * q[:, 1] / q[:, 2] + 240.0], axis=1)
    pix += rng.normal(0.0, 0.3, size=pix.shape)
    masks = np.full(n, abi.POSE_TRANSLATION, dtype=np.uint32) if masks is None else np.asarray(masks, dtype=np.uint32)
    Cp = C + rng.normal(0.0, 0.02, size=C.shape)
    gauge = Gauge.fixed_baseline(0, 4, float(np.linalg.norm(Cp[4] - Cp[0]))) if gauge_fixed_baseline else Gauge()
    return BundleProblem(
        rotations=R, centers=Cp, pose_variables=masks,
        intrinsics=[CameraIntrinsics(model=abi.CAMERA_PINHOLE, fx=600.0, fy=600.0, cx=320.0, cy=240.0)],
        points=X + rng.normal(0.0, 0.01, size=X.shape),
        point_fixed=np.full(P, 1 if fixed_points else 0, dtype=np.uint8), observation_pose=obs_cam,
        observation_intrinsic=np.zeros(len(obs_cam), dtype=np.uint32), observation_point=obs_pt,
        observation_pixel=pix, robust_loss=RobustLoss.huber(1.0), gauge=gauge)


@pytest.mark.parametrize("fixed_baseline", [True, False])
def test_oracle_preflight_certifies_a_translation_only_ring(fixed_baseline):
    from openmvg_ba_cuda import SolveConfig
    pf = O.preflight(translation_only_problem(fixed_baseline), SolveConfig())
    assert pf["status"] == abi.PREFLIGHT_PROCEED and pf["has_counts"] == 1
    assert pf["dense_observability_escalation"] == 0
    assert pf["covered_free_pose_count"] == 7  # every camera but the anchor
    assert pf["pose_dimension"] == 3 * 8 - 4
    assert pf["weak_point_count"] == 0


def test_oracle_preflight_skips_problems_it_does_not_cover():
    from openmvg_ba_cuda import SolveConfig
    for p in (translation_only_problem(masks=[abi.POSE_FREE] * 8), translation_only_problem(fixed_points=True)):
        pf = O.preflight(p, SolveConfig())
        assert pf["status"] == abi.PREFLIGHT_PROCEED and pf["has_counts"] == 0 and pf["pose_dimension"] is None


def test_oracle_translation_only_solve_reports_the_probe():
    """A translation-only solve runs the probe on its accepted geometry (native/mod.rs:435-447): the
    observability details come from it."""
    from openmvg_ba_cuda import SolveConfig
    sol = O.solve(translation_only_problem(), SolveConfig(max_iterations=30))
    r = sol.report
    assert r["linear_solver"] == abi.SOLVER_DIRECT
    assert r["observability"] == abi.OBS_FULL_RANK
    assert r["has_observability_details"] == 1
    assert r["details_pose_dimension"] == 3 * 8 - 4 and r["details_pose_rank"] == 3 * 8 - 4


# ---- the CUDA library ----------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_probe_matches_the_oracle(adjuster, name):
    make, check = CASES[name]
    problem, options = make()
    g = adjuster.probe_fixed_rotation(problem, options)
    check(g)
    assert g == O.probe_fixed_rotation(problem, options)


@pytest.mark.gpu
def test_gpu_probe_collapsed_point_and_chains(adjuster):
    for step in range(0, 20, 4):
        assert adjuster.probe_fixed_rotation(collapsed_point_problem(step))["status"] == CERTIFIED
    for cameras in (3, 4, 8, 40):
        assert adjuster.probe_fixed_rotation(chain_problem(cameras))["status"] != CERTIFIED
    with pytest.raises(ValueError):
        adjuster.probe_fixed_rotation(synthetic_problem(), ProbeOptions(max_factor_nonzeros=0))


@pytest.mark.gpu
@pytest.mark.parametrize("fixed_baseline", [True, False])
def test_gpu_preflight_and_translation_only_solve_match_the_oracle(adjuster, fixed_baseline):
    from openmvg_ba_cuda import SolveConfig
    p = translation_only_problem(fixed_baseline)
    assert adjuster.preflight(p, SolveConfig()) == O.preflight(p, SolveConfig())
    cfg = SolveConfig(max_iterations=30)
    g, o = adjuster.solve(p, cfg), O.solve(p, cfg)
    for k in ("observability", "has_observability_details", "details_pose_rank", "details_pose_dimension",
              "details_weak_point_count", "linear_solver", "iteration_count"):
        assert g.report[k] == o.report[k], k
    assert abs(g.report["final_objective"] - o.report["final_objective"]) <= 1e-9 * o.report["final_objective"]
    assert np.array_equal(g.rotations, p.rotations)  # held rotations, bit for bit
    assert np.max(np.abs(g.centers - o.centers)) < 1e-7
