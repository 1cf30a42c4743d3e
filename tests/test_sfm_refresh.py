"""The landmark reprojection-error refresh openmvg-sfm runs after a bundle adjustment
(refresh_landmark_reprojection_errors_for, crates/openmvg-sfm/src/ops/reconstruction/bundle.rs:
510-637) on the GPU (omvgba_sfm_refresh_reprojection) against the oracle's restatement.

The CPU tests pin the oracle's residual policy to the reference's own tests
(ops/reconstruction/tests/residual.rs:19-70): the bearing error of an exact projection is zero, and
the policy measures perspective cameras in pixels and fisheye and spherical cameras in bearing angle
scaled by the nominal pixels per radian (600 px/rad for a 600 px fisheye focal, 1024/2pi for a
1024-px-wide spherical image). The GPU tests refresh a synthetic workspace of pinhole,
Brown-Conrady, fisheye and spherical views (views without a pose, observations outside the support,
inactive landmarks, landmarks behind some cameras, gross outliers) and compare every landmark's
update, reprojection error and support, and the cleanup counts, with the oracle.
"""
import math

import numpy as np
import pytest

import sfm_oracle as S
from openmvg_ba_cuda import CameraIntrinsics, abi
from openmvg_ba_cuda.sfm import LandmarkTracks


def test_oracle_bearing_error_of_an_exact_projection_is_zero():
    """camera_bearing_error_matches_exact_projection (tests/residual.rs:19-27)"""
    cam = CameraIntrinsics(model=abi.CAMERA_PINHOLE, fx=100.0, fy=100.0, cx=32.0, cy=24.0)
    X = [0.25, -0.1, 2.0]
    assert abs(S.bearing_error_rad(cam, X, S.project(cam, X))) < 1e-12
    assert S.pixel_equivalent(cam, X, S.project(cam, X)) == 0.0


def test_oracle_policy_units_follow_the_camera_family():
    """residual_policy_uses_pixels_for_perspective_and_angles_for_spherical (tests/residual.rs:29-70)"""
    pin = CameraIntrinsics(model=abi.CAMERA_PINHOLE, fx=800.0, fy=600.0, cx=32.0, cy=24.0)
    brown = CameraIntrinsics(model=abi.CAMERA_BROWN_CONRADY, fx=800.0, fy=600.0, cx=32.0, cy=24.0,
                             radial_kind=abi.RADIAL_K1K2K3, k1=-0.1, k2=0.01, k3=0.0)
    fish = CameraIntrinsics(model=abi.CAMERA_FISHEYE, fx=600.0, fy=600.0, cx=32.0, cy=24.0)
    sph = CameraIntrinsics(model=abi.CAMERA_SPHERICAL, width=1024, height=512)
    assert not S.is_generalized(pin) and not S.is_generalized(brown)
    assert S.is_generalized(fish) and S.is_generalized(sph)
    assert abs(4.0 / S.pixels_per_radian(fish) - 4.0 / 600.0) < 1e-12
    assert abs(4.0 / S.pixels_per_radian(sph) - 4.0 * 2.0 * math.pi / 1024.0) < 1e-12
    # a perspective residual is the pixel distance of the projection
    X = [0.1, 0.05, 3.0]
    u, v = S.project(pin, X)
    assert abs(S.pixel_equivalent(pin, X, (u + 3.0, v - 4.0)) - 5.0) < 1e-12
    # behind the camera there is no residual; a spherical camera sees every direction
    assert S.pixel_equivalent(pin, [0.1, 0.05, -3.0], (u, v)) is None
    assert S.pixel_equivalent(sph, [0.1, 0.05, -3.0], S.project(sph, [0.1, 0.05, -3.0])) < 1e-9


def _look_at(C):
    z = -C / np.linalg.norm(C)
    x = np.cross([0.0, 1.0, 0.0], z)
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    return np.stack([x, y, z])


def workspace(seed=3, landmarks=1500, views=24):
    """A ring of views of four camera models around points near the origin, with the cases the
    refresh distinguishes: views without a pose, observations outside the support, inactive
    landmarks, points behind some cameras, gross outliers."""
    rng = np.random.default_rng(seed)
    intr = [CameraIntrinsics(model=abi.CAMERA_PINHOLE, fx=700.0, fy=690.0, cx=320.0, cy=240.0),
            CameraIntrinsics(model=abi.CAMERA_BROWN_CONRADY, fx=650.0, fy=650.0, cx=330.0, cy=245.0,
                             radial_kind=abi.RADIAL_K1K2K3, k1=-0.08, k2=0.01, k3=0.001,
                             tangential_kind=abi.TANGENTIAL_P1P2, p1=1e-3, p2=-5e-4),
            CameraIntrinsics(model=abi.CAMERA_FISHEYE, fx=300.0, fy=300.0, cx=320.0, cy=240.0,
                             radial_kind=abi.RADIAL_K1K2, k1=-0.02, k2=0.001),
            CameraIntrinsics(model=abi.CAMERA_SPHERICAL, width=2048, height=1024)]
    ang = 2 * np.pi * np.arange(views) / views
    C = np.stack([4.0 * np.cos(ang), 0.3 * np.sin(2 * ang), 4.0 * np.sin(ang)], axis=1)
    R = np.stack([_look_at(c) for c in C])
    view_intr = np.arange(views) % 4
    posed = np.ones(views, dtype=bool)
    posed[[5, 13]] = False
    X = rng.uniform(-1.0, 1.0, size=(landmarks, 3))
    far = rng.random(landmarks) < 0.05
    X[far] *= 6.0  # outside the ring: behind some cameras
    offset, tpose, tintr, tpix, tsup = [0], [], [], [], []
    for l in range(landmarks):
        k = int(rng.integers(1, 7))
        for v in rng.choice(views, size=k, replace=False):
            cam = intr[view_intr[v]]
            xc = S.camera_point(R[v], C[v], X[l])
            px = S.project(cam, xc)
            if px is None:
                px = (float(rng.uniform(0, 600)), float(rng.uniform(0, 400)))
            px = np.array(px) + rng.normal(0.0, 0.7, size=2)
            if rng.random() < 0.03:
                px += rng.uniform(-200, 200, size=2)
            tpose.append(int(v) if posed[v] else abi.NO_POSE)
            tintr.append(int(view_intr[v]))
            tpix.append(px)
            tsup.append(0 if rng.random() < 0.08 else 1)
        offset.append(len(tpose))
    active = (rng.random(landmarks) > 0.05).astype(np.uint8)
    tracks = LandmarkTracks(points=X, active=active, track_offset=np.array(offset, dtype=np.uint64),
                            track_pose=np.array(tpose, dtype=np.uint32), track_intrinsic=np.array(tintr, dtype=np.uint32),
                            track_pixel=np.array(tpix), track_support=np.array(tsup, dtype=np.uint8))
    return R, C, intr, tracks


def test_oracle_workspace_covers_every_update_kind():
    R, C, intr, tracks = workspace(landmarks=600)
    update, _, _, rejected, removed = S.refresh(R, C, intr, tracks, np.zeros(600))
    kinds = set(update)
    assert kinds == {abi.REFRESH_SKIPPED, abi.REFRESH_REJECTED, abi.REFRESH_UNCHANGED, abi.REFRESH_PRUNED}
    assert rejected == sum(1 for u in update if u == abi.REFRESH_REJECTED) and removed > 0


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [3, 8])
def test_gpu_refresh_matches_oracle(adjuster, seed):
    from openmvg_ba_cuda.sfm import refresh_reprojection
    R, C, intr, tracks = workspace(seed=seed)
    L = len(tracks.points)
    before = np.full(L, 7.5)
    g = refresh_reprojection(adjuster, R, C, intr, tracks, before)
    update, error, support, rejected, removed = S.refresh(R, C, intr, tracks, before)
    assert np.array_equal(g.landmark_update, np.array(update, dtype=np.uint8))
    assert np.array_equal(g.track_support, np.array(support, dtype=np.uint8))
    assert (g.rejected_landmarks, g.removed_observations) == (rejected, removed)
    error = np.array(error)
    kept = (g.landmark_update == abi.REFRESH_UNCHANGED) | (g.landmark_update == abi.REFRESH_PRUNED)
    # 1e-9 relative, plus rounding of the pixels the residuals are differences of: a point far off a
    # distorted camera's axis projects to pixels near 1e9, where one ulp is ~1e-7 px
    mag = np.array([np.max(np.abs(tracks.track_pixel[int(tracks.track_offset[l]):int(tracks.track_offset[l + 1])]),
                           initial=0.0) for l in range(L)])
    tol = 1e-9 * np.maximum(error, 1.0) + 16 * np.finfo(float).eps * mag
    assert np.all(np.abs(g.reprojection_error[kept] - error[kept]) <= tol[kept])
    assert np.array_equal(g.reprojection_error[~kept], before[~kept])  # skipped and rejected keep theirs
    assert np.array_equal(refresh_reprojection(adjuster, R, C, intr, tracks, before).reprojection_error,
                          g.reprojection_error)  # run to run the same bits


@pytest.mark.gpu
def test_gpu_refresh_rejects_bad_indices(adjuster):
    from openmvg_ba_cuda.problem import ProblemError
    from openmvg_ba_cuda.sfm import refresh_reprojection
    R, C, intr, tracks = workspace(landmarks=20)
    tracks.track_intrinsic = tracks.track_intrinsic.copy()
    tracks.track_intrinsic[3] = 9
    with pytest.raises(ProblemError):
        refresh_reprojection(adjuster, R, C, intr, tracks)


@pytest.mark.gpu
def test_gpu_prepare_solve_refresh_round_trip(adjuster):
    """The SfM side around one solve: the workspace tables of a ring survey are prepared into a
    problem, solved on the GPU and the landmarks refreshed with the solved state; the refresh equals
    the oracle's, and on the solved state the landmarks' errors fall."""
    from openmvg_ba_cuda import SolveConfig, synthetic
    from openmvg_ba_cuda.sfm import PrepareConfig, SfmWorkspace, prepare_problem, refresh_reprojection
    src = synthetic.ring_problem(seed=4)
    P = len(src.points)
    order = np.argsort(src.observation_point, kind="stable")
    offset = np.concatenate([[0], np.cumsum(np.bincount(src.observation_point, minlength=P))]).astype(np.uint64)
    tracks = LandmarkTracks(points=src.points, active=np.ones(P, np.uint8), track_offset=offset,
                            track_pose=src.observation_pose[order].astype(np.uint32),
                            track_intrinsic=src.observation_intrinsic[order].astype(np.uint32),
                            track_pixel=src.observation_pixel[order], track_support=np.ones(len(order), np.uint8))
    ws = SfmWorkspace(view_pose=np.arange(len(src.rotations), dtype=np.uint32),
                      view_intrinsic=np.zeros(len(src.rotations), dtype=np.uint32),
                      view_size=np.tile([640, 480], (len(src.rotations), 1)).astype(np.uint32),
                      rotations=src.rotations, centers=src.centers, intrinsics=src.intrinsics,
                      intrinsic_guess=np.zeros(1, np.uint8), landmarks=tracks)
    problem, pose_rows, _, lm_rows = prepare_problem(ws, PrepareConfig(loss_kind=abi.LOSS_HUBER, loss_scale=1.0))
    assert problem.observation_count == src.observation_count and list(lm_rows) == list(range(P))
    sol = adjuster.solve(problem, SolveConfig(max_iterations=20))
    before = refresh_reprojection(adjuster, src.rotations, src.centers, src.intrinsics, tracks)
    tracks.points = sol.points  # the commit writes the refined points and poses back
    after = refresh_reprojection(adjuster, sol.rotations, sol.centers, sol.intrinsics, tracks)
    update, error, support, rejected, removed = S.refresh(sol.rotations, sol.centers, sol.intrinsics, tracks, np.zeros(P))
    assert np.array_equal(after.landmark_update, np.array(update, dtype=np.uint8))
    assert np.array_equal(after.track_support, np.array(support, dtype=np.uint8))
    assert (after.rejected_landmarks, after.removed_observations) == (rejected, removed)
    ok = after.landmark_update == abi.REFRESH_UNCHANGED
    assert np.all(np.abs(after.reprojection_error[ok] - np.array(error)[ok]) <= 1e-9 * np.maximum(np.array(error)[ok], 1.0))
    assert np.median(after.reprojection_error[ok]) < np.median(before.reprojection_error[ok])
