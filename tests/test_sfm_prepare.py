"""Building the bundle-adjustment problem from a reconstruction's tables (omvgba_sfm_prepare_problem,
prepare_bundle_adjustment_problem in crates/openmvg-sfm/src/ops/reconstruction/bundle.rs:707-989)
against the oracle's restatement: pose, intrinsic and landmark order and rows, pose and point
variables under each optimization scope, intrinsic variables and certification, the observation
gather (supporting observations from registered views, landmark by landmark in track order), the
gauge's pose rows, the residual space and the robust loss in the residual's units; and the
reference's own pin of the loss conversion (bundle.rs:1039-1063): a 2 px Cauchy scale over angular
residuals at 0.001 rad per pixel becomes 0.002 rad. Host code only: no GPU.
"""
import numpy as np
import pytest

import sfm_oracle as S
from openmvg_ba_cuda import CameraIntrinsics, abi
from openmvg_ba_cuda.problem import ProblemError
from openmvg_ba_cuda.sfm import LandmarkTracks, PrepareConfig, SfmWorkspace, prepare_problem


def make_workspace(seed=2, views=30, poses=26, landmarks=400, wide=False):
    rng = np.random.default_rng(seed)
    intr = [CameraIntrinsics(model=abi.CAMERA_PINHOLE, fx=700.0, fy=690.0, cx=320.0, cy=240.0),
            CameraIntrinsics(model=abi.CAMERA_BROWN_CONRADY, fx=650.0, fy=650.0, cx=330.0, cy=245.0,
                             radial_kind=abi.RADIAL_K1K2, k1=-0.08, k2=0.01),
            CameraIntrinsics(model=abi.CAMERA_PINHOLE, fx=900.0, fy=900.0, cx=400.0, cy=300.0)]
    if wide:
        intr.append(CameraIntrinsics(model=abi.CAMERA_FISHEYE, fx=1000.0, fy=1000.0, cx=320.0, cy=240.0))
    view_intr = np.arange(views) % len(intr)
    sizes = {0: (640, 480), 1: (660, 490), 2: (800, 600), 3: (640, 480)}
    view_size = np.array([sizes[int(i)] for i in view_intr], dtype=np.uint32)
    view_pose = rng.permutation(views)[:views].astype(np.uint32) % poses  # some views share a pose row
    view_pose[rng.random(views) < 0.15] = abi.NO_POSE
    offset, tv, tpix, tsup = [0], [], [], []
    for _ in range(landmarks):
        for v in rng.choice(views, size=int(rng.integers(1, 8)), replace=False):
            tv.append(int(v))
            tpix.append(rng.uniform(0, 600, size=2))
            tsup.append(0 if rng.random() < 0.1 else 1)
        offset.append(len(tv))
    tracks = LandmarkTracks(points=rng.normal(size=(landmarks, 3)), active=(rng.random(landmarks) > 0.1).astype(np.uint8),
                            track_offset=np.array(offset, dtype=np.uint64), track_pose=np.array(tv, dtype=np.uint32),
                            track_intrinsic=np.zeros(len(tv), dtype=np.uint32), track_pixel=np.array(tpix),
                            track_support=np.array(tsup, dtype=np.uint8))
    R = np.stack([np.eye(3)] * poses) + rng.normal(scale=1e-3, size=(poses, 3, 3))
    return SfmWorkspace(view_pose=view_pose, view_intrinsic=view_intr.astype(np.uint32), view_size=view_size,
                        rotations=R, centers=rng.normal(size=(poses, 3)), intrinsics=intr,
                        intrinsic_guess=np.array([0, 1, 0, 0][:len(intr)], dtype=np.uint8), landmarks=tracks)


def registered_views(ws):
    return [v for v in range(len(ws.view_pose)) if ws.view_pose[v] != abi.NO_POSE]


def check(ws, cfg):
    p, pose_rows, intr_rows, lm_rows = prepare_problem(ws, cfg)
    o = S.prepare(ws.view_pose, ws.view_intrinsic, ws.view_size, ws.intrinsics, ws.intrinsic_guess, ws.landmarks,
                  cfg.scope, cfg.fixed_views, cfg.fixed_landmarks, cfg.excluded_landmarks,
                  (cfg.loss_kind, cfg.loss_scale, cfg.loss_scale_space),
                  (cfg.gauge_kind, cfg.gauge_first_view, cfg.gauge_second_view, cfg.gauge_distance))
    assert list(pose_rows) == o["pose_rows"] and list(p.pose_variables) == o["pose_vars"]
    assert np.array_equal(p.rotations, ws.rotations[o["pose_rows"]]) and np.array_equal(p.centers, ws.centers[o["pose_rows"]])
    assert list(intr_rows) == [d["row"] for d in o["intrinsics"]]
    for c, d in zip(p.intrinsics, o["intrinsics"]):
        src = ws.intrinsics[d["row"]]
        assert (c.model, c.fx, c.fy, c.cx, c.cy, c.k1) == (src.model, src.fx, src.fy, src.cx, src.cy, src.k1)
        assert (c.width, c.height, c.variables, c.certification) == (d["width"], d["height"], d["variables"], d["certification"])
    assert list(lm_rows) == o["landmark_rows"] and list(p.point_fixed) == o["point_fixed"]
    assert np.array_equal(p.points, ws.landmarks.points[o["landmark_rows"]])
    obs = o["observations"]
    assert p.observation_count == len(obs)
    assert list(p.observation_pose) == [x[0] for x in obs] and list(p.observation_intrinsic) == [x[1] for x in obs]
    assert list(p.observation_point) == [x[2] for x in obs]
    assert np.array_equal(p.observation_pixel, np.array([[x[3], x[4]] for x in obs]).reshape(-1, 2))
    assert (p.gauge.kind, p.gauge.first, p.gauge.second) == o["gauge"][:3]
    assert p.residual_space == o["residual_space"]
    assert (p.robust_loss.kind, p.robust_loss.scale, p.robust_loss.space) == o["loss"]
    return p


@pytest.mark.parametrize("scope", [abi.SCOPE_FULL, abi.SCOPE_POINTS_ONLY, abi.SCOPE_POSES_ONLY,
                                   abi.SCOPE_TRANSLATIONS_AND_POINTS, abi.SCOPE_SELF_CALIBRATION])
def test_prepare_matches_oracle_under_every_scope(scope):
    ws = make_workspace()
    reg = registered_views(ws)
    cfg = PrepareConfig(scope=scope, fixed_views=(reg[0],), fixed_landmarks=(3, 17), excluded_landmarks=(5, 6, 40),
                        loss_kind=abi.LOSS_HUBER, loss_scale=1.5, loss_scale_space=abi.RESIDUAL_PIXELS,
                        gauge_kind=abi.GAUGE_FIXED_BASELINE, gauge_first_view=reg[1], gauge_second_view=reg[2],
                        gauge_distance=1.25)
    p = check(ws, cfg)
    assert p.residual_space == abi.RESIDUAL_PIXELS and p.robust_loss.scale == 1.5


def test_wide_angle_group_makes_the_residuals_angular_and_converts_the_loss():
    """a_pixel_loss_over_angular_residuals_is_converted_with_the_angle_of_a_pixel (bundle.rs:1039-1063)"""
    ws = make_workspace(wide=True)
    ws.intrinsics = [ws.intrinsics[3]] * 4  # every group a 1000 px fisheye: 0.001 rad per pixel
    p = check(ws, PrepareConfig(loss_kind=abi.LOSS_CAUCHY, loss_scale=2.0, loss_scale_space=abi.RESIDUAL_PIXELS))
    assert p.residual_space == abi.RESIDUAL_ANGULAR
    assert p.robust_loss.space == abi.RESIDUAL_ANGULAR and abs(p.robust_loss.scale - 0.002) < 1e-15
    assert all(c.variables == 0 for c in p.intrinsics)  # never estimated, even under self-calibration
    p = check(ws, PrepareConfig(scope=abi.SCOPE_SELF_CALIBRATION))
    assert all(c.variables == 0 for c in p.intrinsics)


def test_prepare_errors_like_the_reference():
    ws = make_workspace()
    ws.view_size = ws.view_size.copy()
    ws.view_size[0] = (1, 1)  # a group shared by images of different sizes
    with pytest.raises(ProblemError):
        prepare_problem(ws, PrepareConfig())
    ws = make_workspace()
    unregistered = [v for v in range(len(ws.view_pose)) if ws.view_pose[v] == abi.NO_POSE][0]
    with pytest.raises(ProblemError):  # fixed-baseline anchor without a pose
        prepare_problem(ws, PrepareConfig(gauge_kind=abi.GAUGE_FIXED_BASELINE, gauge_first_view=unregistered,
                                          gauge_second_view=registered_views(ws)[0], gauge_distance=1.0))
    with pytest.raises(ProblemError):  # an angular loss scale over pixel residuals
        prepare_problem(ws, PrepareConfig(loss_kind=abi.LOSS_HUBER, loss_scale=0.01, loss_scale_space=abi.RESIDUAL_ANGULAR))
