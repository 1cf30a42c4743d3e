"""The SfM side of a bundle adjustment: the landmark reprojection-error refresh openmvg-sfm runs after
it commits a solve (refresh_landmark_reprojection_errors_for, crates/openmvg-sfm/src/ops/
reconstruction/bundle.rs:510-637), through omvgba_sfm_refresh_reprojection.

A workspace's landmarks arrive as flat arrays: each landmark's point and active flag, and its track
(CSR by landmark) with the observing view's pose (abi.NO_POSE when the view has none), intrinsic,
pixel and whether the observation supports the landmark.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import abi
from ._lib import lib
from .problem import raise_for


@dataclass
class LandmarkTracks:
    points: np.ndarray          # (L, 3) world frame
    active: np.ndarray          # (L,) uint8: 1 for an active landmark
    track_offset: np.ndarray    # (L + 1,) uint64
    track_pose: np.ndarray      # (N,) uint32, abi.NO_POSE for a view without a pose
    track_intrinsic: np.ndarray  # (N,) uint32
    track_pixel: np.ndarray     # (N, 2)
    track_support: np.ndarray   # (N,) uint8


@dataclass
class RefreshOutcome:
    landmark_update: np.ndarray     # (L,) abi.REFRESH_*
    reprojection_error: np.ndarray  # (L,) mean pixel-equivalent residual of kept landmarks
    track_support: np.ndarray       # (N,) the support after the refresh
    rejected_landmarks: int
    removed_observations: int


def refresh_reprojection(adjuster, rotations, centers, intrinsics, tracks: LandmarkTracks,
                         reprojection_error=None) -> RefreshOutcome:
    """Refresh every active landmark's reprojection error and support on the adjuster's device.

    rotations (P, 3, 3) world to camera and centers (P, 3) are the poses; intrinsics is a list of
    CameraIntrinsics. reprojection_error (L,), when given, is the current error kept for landmarks
    that are skipped or rejected (zeros otherwise)."""
    L = int(np.asarray(tracks.points).reshape(-1, 3).shape[0])
    poses = abi.marshal_poses(np.asarray(rotations), np.asarray(centers))
    intr = (abi.Intrinsic * len(intrinsics))()
    for i, c in enumerate(intrinsics):
        c.fill(intr[i])
    keep = dict(
        points=np.ascontiguousarray(tracks.points, dtype=np.float64).reshape(-1),
        active=np.ascontiguousarray(tracks.active, dtype=np.uint8),
        offset=np.ascontiguousarray(tracks.track_offset, dtype=np.uint64),
        pose=np.ascontiguousarray(tracks.track_pose, dtype=np.uint32),
        intrinsic=np.ascontiguousarray(tracks.track_intrinsic, dtype=np.uint32),
        pixel=np.ascontiguousarray(tracks.track_pixel, dtype=np.float64).reshape(-1),
        support=np.ascontiguousarray(tracks.track_support, dtype=np.uint8),
    )
    N = int(keep["offset"][-1]) if len(keep["offset"]) else 0
    t = abi.LandmarkTracks()
    t.landmark_count = L
    t.points = keep["points"].ctypes.data_as(C.POINTER(C.c_double))
    t.active = keep["active"].ctypes.data_as(C.POINTER(C.c_uint8))
    t.track_offset = keep["offset"].ctypes.data_as(C.POINTER(C.c_uint64))
    t.track_pose = keep["pose"].ctypes.data_as(C.POINTER(C.c_uint32))
    t.track_intrinsic = keep["intrinsic"].ctypes.data_as(C.POINTER(C.c_uint32))
    t.track_pixel = keep["pixel"].ctypes.data_as(C.POINTER(C.c_double))
    t.track_support = keep["support"].ctypes.data_as(C.POINTER(C.c_uint8))
    update = np.zeros(L, dtype=np.uint8)
    err = np.zeros(L) if reprojection_error is None else np.array(reprojection_error, dtype=np.float64)
    support = np.zeros(N, dtype=np.uint8)
    r = abi.RefreshResult()
    r.landmark_update = update.ctypes.data_as(C.POINTER(C.c_uint8))
    r.reprojection_error = err.ctypes.data_as(C.POINTER(C.c_double))
    r.track_support = support.ctypes.data_as(C.POINTER(C.c_uint8))
    e = abi.Error()
    code = lib().omvgba_sfm_refresh_reprojection(adjuster._ctx, len(poses), C.cast(poses, C.POINTER(abi.Pose)),
                                                 len(intrinsics), C.cast(intr, C.POINTER(abi.Intrinsic)),
                                                 C.byref(t), C.byref(r), C.byref(e))
    raise_for(code, e)
    return RefreshOutcome(update, err, support, int(r.rejected_landmarks), int(r.removed_observations))


@dataclass
class SfmWorkspace:
    """The reconstruction tables the preparation reads (rows, not the reference's ids)."""
    view_pose: np.ndarray       # (V,) uint32 pose row, abi.NO_POSE for an unregistered view
    view_intrinsic: np.ndarray  # (V,) uint32
    view_size: np.ndarray       # (V, 2) uint32 width, height
    rotations: np.ndarray       # (P, 3, 3) world to camera
    centers: np.ndarray         # (P, 3)
    intrinsics: list            # CameraIntrinsics per intrinsic row
    intrinsic_guess: np.ndarray  # (I,) uint8
    landmarks: LandmarkTracks   # track_pose holds the observing view row


@dataclass
class PrepareConfig:
    scope: int = abi.SCOPE_FULL
    fixed_views: tuple = ()
    fixed_landmarks: tuple = ()
    excluded_landmarks: tuple = ()
    loss_kind: int = abi.LOSS_SQUARED
    loss_scale: float = 0.0
    loss_scale_space: int = abi.RESIDUAL_PIXELS
    gauge_kind: int = abi.GAUGE_FREE
    gauge_first_view: int = 0
    gauge_second_view: int = 0
    gauge_distance: float = 0.0


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def prepare_problem(ws: SfmWorkspace, cfg: PrepareConfig):
    """omvgba_sfm_prepare_problem: (BundleProblem, pose_rows, intrinsic_rows, landmark_rows)."""
    from .problem import BundleProblem, CameraIntrinsics, Gauge, RobustLoss
    keep = dict(vp=_u32(ws.view_pose), vi=_u32(ws.view_intrinsic), vs=_u32(ws.view_size).reshape(-1),
                guess=np.ascontiguousarray(ws.intrinsic_guess, dtype=np.uint8),
                pts=np.ascontiguousarray(ws.landmarks.points, dtype=np.float64).reshape(-1),
                act=np.ascontiguousarray(ws.landmarks.active, dtype=np.uint8),
                off=np.ascontiguousarray(ws.landmarks.track_offset, dtype=np.uint64),
                tv=_u32(ws.landmarks.track_pose), ti=_u32(ws.landmarks.track_intrinsic),
                px=np.ascontiguousarray(ws.landmarks.track_pixel, dtype=np.float64).reshape(-1),
                sup=np.ascontiguousarray(ws.landmarks.track_support, dtype=np.uint8),
                fv=_u32(cfg.fixed_views), fl=_u32(cfg.fixed_landmarks), xl=_u32(cfg.excluded_landmarks))
    ptr = lambda a, t: a.ctypes.data_as(C.POINTER(t))
    poses = abi.marshal_poses(np.asarray(ws.rotations), np.asarray(ws.centers))
    intr = (abi.Intrinsic * len(ws.intrinsics))()
    for i, c in enumerate(ws.intrinsics):
        c.fill(intr[i])
    w = abi.SfmWorkspace()
    w.view_count = len(keep["vp"])
    w.view_pose, w.view_intrinsic, w.view_size = ptr(keep["vp"], C.c_uint32), ptr(keep["vi"], C.c_uint32), ptr(keep["vs"], C.c_uint32)
    w.pose_count, w.poses = len(poses), C.cast(poses, C.POINTER(abi.Pose))
    w.intrinsic_count, w.intrinsics = len(ws.intrinsics), C.cast(intr, C.POINTER(abi.Intrinsic))
    w.intrinsic_guess = ptr(keep["guess"], C.c_uint8)
    lt = w.landmarks
    lt.landmark_count = len(keep["act"])
    lt.points, lt.active, lt.track_offset = ptr(keep["pts"], C.c_double), ptr(keep["act"], C.c_uint8), ptr(keep["off"], C.c_uint64)
    lt.track_pose, lt.track_intrinsic = ptr(keep["tv"], C.c_uint32), ptr(keep["ti"], C.c_uint32)
    lt.track_pixel, lt.track_support = ptr(keep["px"], C.c_double), ptr(keep["sup"], C.c_uint8)
    c = abi.SfmPrepareConfig(cfg.scope, len(keep["fv"]), ptr(keep["fv"], C.c_uint32), len(keep["fl"]), ptr(keep["fl"], C.c_uint32),
                             len(keep["xl"]), ptr(keep["xl"], C.c_uint32), cfg.loss_kind, cfg.loss_scale, cfg.loss_scale_space,
                             cfg.gauge_kind, cfg.gauge_first_view, cfg.gauge_second_view, cfg.gauge_distance)
    out = abi.SfmPrepared()
    e = abi.Error()
    raise_for(lib().omvgba_sfm_prepare_problem(C.byref(w), C.byref(c), C.byref(out), C.byref(e)), e)
    pr = out.problem
    P, I, K, N = pr.pose_count, pr.intrinsic_count, pr.point_count, pr.observation_count
    o_poses = (abi.Pose * max(P, 1))()
    o_intr = (abi.Intrinsic * max(I, 1))()
    o = dict(pts=np.zeros(3 * K), pf=np.zeros(K, np.uint8), op=np.zeros(N, np.uint32), oi=np.zeros(N, np.uint32),
             ot=np.zeros(N, np.uint32), ox=np.zeros(2 * N), pr=np.zeros(P, np.uint32), ir=np.zeros(I, np.uint32),
             lr=np.zeros(K, np.uint32))
    pr.poses, pr.intrinsics = C.cast(o_poses, C.POINTER(abi.Pose)), C.cast(o_intr, C.POINTER(abi.Intrinsic))
    pr.points, pr.point_fixed = ptr(o["pts"], C.c_double), ptr(o["pf"], C.c_uint8)
    pr.observation_pose, pr.observation_intrinsic = ptr(o["op"], C.c_uint32), ptr(o["oi"], C.c_uint32)
    pr.observation_point, pr.observation_pixel = ptr(o["ot"], C.c_uint32), ptr(o["ox"], C.c_double)
    out.pose_rows, out.intrinsic_rows, out.landmark_rows = ptr(o["pr"], C.c_uint32), ptr(o["ir"], C.c_uint32), ptr(o["lr"], C.c_uint32)
    raise_for(lib().omvgba_sfm_prepare_problem(C.byref(w), C.byref(c), C.byref(out), C.byref(e)), e)
    raw = np.frombuffer(o_poses, dtype=np.uint8).reshape(-1, C.sizeof(abi.Pose))[:P]
    view = raw.view(np.dtype([("rotation", "<f8", 9), ("center", "<f8", 3), ("variables", "<u4"), ("reserved", "<u4")]))
    problem = BundleProblem(
        rotations=view["rotation"][:, 0].reshape(P, 3, 3).copy(), centers=view["center"][:, 0].copy(),
        pose_variables=view["variables"][:, 0].copy(), intrinsics=[CameraIntrinsics.from_struct(o_intr[i]) for i in range(I)],
        points=o["pts"].reshape(K, 3), point_fixed=o["pf"], observation_pose=o["op"], observation_intrinsic=o["oi"],
        observation_point=o["ot"], observation_pixel=o["ox"].reshape(N, 2), residual_space=pr.residual_space,
        robust_loss=RobustLoss(pr.loss_kind, pr.loss_scale, pr.loss_scale_space),
        gauge=Gauge(pr.gauge_kind, pr.gauge_first, pr.gauge_second, pr.gauge_distance))
    return problem, o["pr"], o["ir"], o["lr"]
