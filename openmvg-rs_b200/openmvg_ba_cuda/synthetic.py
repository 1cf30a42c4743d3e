"""Seeded synthetic bundle-adjustment problems with the shapes, sizes and noise model of the
workloads this solver is measured on. No public dataset is used: every input is generated here
from a recorded seed (numpy PCG64).

Workloads
---------
ring_problem      20 radial3 cameras on a ring of radius 10 around 2,000 points in [-1, 1]^3
                  (~8k observations); fixed intrinsics, or one shared free (f, k1, k2) group.
plane_problem     cameras on a 2-D grid of trajectories over a 100 x 100 ground plane looking down,
                  points on the plane, geometric track lengths: 500 cameras / 200k points / ~1.2M
                  observations, or 3,000 cameras / 2M points / ~12M observations; per-camera
                  (f, k1, k2) intrinsics.
window_problems   uneven local-BA windows (5-40 cameras, 500-20k points, tracks 2-10).
residual_inputs   random poses, points and radial intrinsics for the residual / adjoint kernels.

Noise model (all BA workloads): pixel noise N(0, 0.5 px), 5% of observations replaced by outliers
uniform in the image, initial state perturbed by rotations of 0.01 rad, camera-centre offsets of
0.05 and point offsets of 0.02 (per-axis standard deviations).
"""
from __future__ import annotations

import numpy as np

from . import abi
from .problem import BundleProblem, CameraIntrinsics, Gauge, RobustLoss

WIDTH, HEIGHT = 640, 480


def _exp_so3(w: np.ndarray) -> np.ndarray:
    """Rodrigues rotation for an (n, 3) array of rotation vectors."""
    w = np.atleast_2d(w)
    th = np.linalg.norm(w, axis=1)
    k = np.zeros((len(w), 3, 3))
    k[:, 0, 1], k[:, 0, 2] = -w[:, 2], w[:, 1]
    k[:, 1, 0], k[:, 1, 2] = w[:, 2], -w[:, 0]
    k[:, 2, 0], k[:, 2, 1] = -w[:, 1], w[:, 0]
    safe = np.where(th > 1e-12, th, 1.0)
    a = np.where(th > 1e-12, np.sin(th) / safe, 1.0)
    b = np.where(th > 1e-12, (1 - np.cos(th)) / safe**2, 0.5)
    return np.eye(3)[None] + a[:, None, None] * k + b[:, None, None] * (k @ k)


def _look_at(centers: np.ndarray, targets: np.ndarray, up=(0.0, 0.0, 1.0)) -> np.ndarray:
    z = targets - centers
    z /= np.linalg.norm(z, axis=1, keepdims=True)
    upv = np.broadcast_to(np.asarray(up, dtype=np.float64), z.shape)
    x = np.cross(upv, z)
    bad = np.linalg.norm(x, axis=1) < 1e-9
    x[bad] = np.cross(np.array([0.0, 1.0, 0.0]), z[bad])
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    y = np.cross(z, x)
    return np.stack([x, y, z], axis=1)  # rows: camera axes in world -> world-to-camera rotation


def _distort(xn, yn, k1, k2, k3):
    r2 = xn * xn + yn * yn
    f = 1.0 + k1 * r2 + k2 * r2 * r2 + k3 * r2 * r2 * r2
    return xn * f, yn * f


def _project(R, C, X, f, cx, cy, k1, k2, k3):
    """Pixels and depths; points whose normalized radius leaves the undistorted field of view
    (where the radial polynomial would fold back into the image) get depth -1 so they never count
    as visible."""
    xc = np.einsum("nij,nj->ni", R, X - C)
    xn, yn = xc[:, 0] / xc[:, 2], xc[:, 1] / xc[:, 2]
    xd, yd = _distort(xn, yn, k1, k2, k3)
    depth = np.where(xn * xn + yn * yn < 0.81, xc[:, 2], -1.0)
    return np.stack([f * xd + cx, f * yd + cy], axis=1), depth


def _noisy(rng, pixels, outlier_fraction=0.05, sigma=0.5):
    obs = pixels + rng.normal(0.0, sigma, size=pixels.shape)
    out = rng.random(len(obs)) < outlier_fraction
    obs[out, 0] = rng.uniform(0, WIDTH, out.sum())
    obs[out, 1] = rng.uniform(0, HEIGHT, out.sum())
    return obs


def _perturb(rng, R, C, X, rot=0.01, trans=0.05, pts=0.02):
    Rp = _exp_so3(rng.normal(0.0, rot, size=(len(R), 3))) @ R
    Cp = C + rng.normal(0.0, trans, size=C.shape)
    Xp = X + rng.normal(0.0, pts, size=X.shape)
    return Rp, Cp, Xp


def ring_problem(seed: int = 7, cameras: int = 20, points: int = 2000, self_calibrating: bool = False,
                 loss: RobustLoss | None = None, radius: float = 10.0,
                 pose_variables: np.ndarray | None = None) -> BundleProblem:
    """20 radial3 cameras on a ring of radius 10 looking at points uniform in [-1, 1]^3.

    At radius 10 the cube spans about +-50 px, where radial distortion is barely observable; a
    smaller ``radius`` spreads the points over the image.

    ``self_calibrating=False``: fixed Brown-Conrady (k1, k2, k3) intrinsics.
    ``self_calibrating=True``: one shared Brown-Conrady K1K2 group with free (f, k1, k2) and a fixed
    principal point (the reference rejects free cx, cy or k3).

    ``pose_variables``: per-pose ``POSE_*`` bits; the parts of a pose that a mask holds (the rotation
    without ``POSE_ROTATION``, the centre without ``POSE_TRANSLATION``) keep their true values, so a
    masked solve is consistent with the observations.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    ang = 2 * np.pi * np.arange(cameras) / cameras
    C = np.stack([radius * np.cos(ang), radius * np.sin(ang), 0.05 * radius * np.sin(3 * ang)], axis=1)
    R = _look_at(C, np.zeros_like(C))
    X = rng.uniform(-1.0, 1.0, size=(points, 3))
    f, cx, cy = 500.0, 320.0, 240.0
    k1, k2, k3 = (-0.1, 0.01, -0.001) if not self_calibrating else (-0.1, 0.01, 0.0)
    counts = rng.integers(2, 9, size=points)
    cam_lists = [rng.choice(cameras, size=c, replace=False) for c in counts]
    obs_point = np.repeat(np.arange(points), counts).astype(np.uint32)
    obs_pose = np.concatenate(cam_lists).astype(np.uint32)
    pix, _ = _project(R[obs_pose], C[obs_pose], X[obs_point], f, cx, cy, k1, k2, k3)
    obs = _noisy(rng, pix)
    Rp, Cp, Xp = _perturb(rng, R, C, X)
    masks = np.full(cameras, abi.POSE_FREE, dtype=np.uint32)
    if pose_variables is not None:
        masks = np.asarray(pose_variables, dtype=np.uint32)
        Rp = np.where(((masks & abi.POSE_ROTATION) == 0)[:, None, None], R, Rp)
        Cp = np.where(((masks & abi.POSE_TRANSLATION) == 0)[:, None], C, Cp)
    if self_calibrating:
        intr = CameraIntrinsics(model=abi.CAMERA_BROWN_CONRADY, fx=505.0, fy=505.0, cx=cx, cy=cy,
                                radial_kind=abi.RADIAL_K1K2, k1=-0.09, k2=0.0,
                                variables=abi.INTRINSIC_FOCAL | abi.INTRINSIC_RADIAL)
    else:
        intr = CameraIntrinsics(model=abi.CAMERA_BROWN_CONRADY, fx=f, fy=f, cx=cx, cy=cy,
                                radial_kind=abi.RADIAL_K1K2K3, k1=k1, k2=k2, k3=k3)
    return BundleProblem(
        rotations=Rp, centers=Cp, pose_variables=masks, intrinsics=[intr], points=Xp,
        point_fixed=np.zeros(points, dtype=np.uint8),
        observation_pose=obs_pose, observation_intrinsic=np.zeros(len(obs_pose), dtype=np.uint32),
        observation_point=obs_point, observation_pixel=obs,
        robust_loss=loss if loss is not None else RobustLoss.huber(1.0), gauge=Gauge(),
    )


def plane_problem(seed: int = 11, cameras: int = 500, points: int = 200_000, mean_track: float = 6.0,
                  altitude: float = 16.0, extent: float = 100.0, per_camera_intrinsics: bool = True,
                  free_intrinsics: bool = True, loss: RobustLoss | None = None,
                  chunk: int = 250_000) -> BundleProblem:
    """Cameras on a grid of trajectories over an ``extent`` x ``extent`` ground plane.

    Cameras fly serpentine rows at ``altitude`` looking down (small random tilt); points lie on the
    plane with up to 2 units of relief. Track length is 2 + Geometric(mean ``mean_track`` - 2),
    capped by the number of cameras that see the point. Each camera has its own Brown-Conrady K1K2
    intrinsic group (free f, k1, k2 and fixed principal point when ``free_intrinsics``).
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    rows = int(round(np.sqrt(cameras * 0.8)))
    cols = int(np.ceil(cameras / rows))
    gx = (np.arange(cols) + 0.5) * extent / cols
    gy = (np.arange(rows) + 0.5) * extent / rows
    cx_grid, cy_grid = np.meshgrid(gx, gy)
    cx_grid[1::2] = cx_grid[1::2, ::-1]  # serpentine trajectories
    C = np.stack([cx_grid.ravel(), cy_grid.ravel(), np.full(rows * cols, altitude)], axis=1)[:cameras]
    C[:, :2] += rng.normal(0.0, 0.1, size=(cameras, 2))
    C[:, 2] += rng.normal(0.0, 0.3, size=cameras)
    heading = np.where((np.arange(cameras) // cols) % 2 == 0, 0.0, np.pi)
    down = np.array([[1.0, 0.0, 0.0], [0.0, -1.0, 0.0], [0.0, 0.0, -1.0]])  # camera z -> world -z
    yaw = _exp_so3(np.stack([np.zeros(cameras), np.zeros(cameras), heading], axis=1))
    tilt = _exp_so3(rng.normal(0.0, 0.03, size=(cameras, 3)))
    R = tilt @ down[None] @ np.transpose(yaw, (0, 2, 1))
    f0, ppx, ppy = 500.0, WIDTH / 2, HEIGHT / 2
    k1s = rng.uniform(-0.12, -0.06, size=cameras)
    k2s = rng.uniform(0.0, 0.02, size=cameras)
    fs = f0 * rng.uniform(0.97, 1.03, size=cameras)
    X = np.stack([rng.uniform(0, extent, points), rng.uniform(0, extent, points), rng.uniform(0, 2.0, points)], axis=1)
    # candidate cameras: grid cells around the point
    cell_w, cell_h = extent / cols, extent / rows
    half_x = altitude * (WIDTH / 2) / f0 * 1.3
    half_y = altitude * (HEIGHT / 2) / f0 * 1.3
    rad = max(half_x, half_y)
    kx, ky = int(np.ceil(rad / cell_w)) + 1, int(np.ceil(rad / cell_h)) + 1
    offs = np.array([(dx, dy) for dy in range(-ky, ky + 1) for dx in range(-kx, kx + 1)])
    cam_at = -np.ones((rows, cols), dtype=np.int64)
    for idx in range(cameras):
        r, c = divmod(idx, cols)
        cc = c if r % 2 == 0 else cols - 1 - c
        cam_at[r, cc] = idx
    extra = rng.geometric(1.0 / max(mean_track - 1.0, 1.0), size=points) - 1  # mean mean_track - 2
    want = 2 + extra
    obs_pose_parts, obs_point_parts, pix_parts = [], [], []
    for start in range(0, points, chunk):
        stop = min(points, start + chunk)
        Xc = X[start:stop]
        col = np.clip((Xc[:, 0] / cell_w).astype(np.int64), 0, cols - 1)
        row = np.clip((Xc[:, 1] / cell_h).astype(np.int64), 0, rows - 1)
        cc = col[:, None] + offs[None, :, 0]
        rr = row[:, None] + offs[None, :, 1]
        inside = (cc >= 0) & (cc < cols) & (rr >= 0) & (rr < rows)
        cand = np.where(inside, cam_at[np.clip(rr, 0, rows - 1), np.clip(cc, 0, cols - 1)], -1)
        valid = cand >= 0
        ci = np.where(valid, cand, 0)
        n, m = ci.shape
        pi = np.repeat(np.arange(n), m)
        pix, depth = _project(R[ci.ravel()], C[ci.ravel()], np.repeat(Xc, m, axis=0), fs[ci.ravel()],
                              ppx, ppy, k1s[ci.ravel()], k2s[ci.ravel()], 0.0)
        vis = valid.ravel() & (depth > 0.5) & (pix[:, 0] > 8) & (pix[:, 0] < WIDTH - 8) & \
            (pix[:, 1] > 8) & (pix[:, 1] < HEIGHT - 8)
        vis = vis.reshape(n, m)
        key = np.where(vis, rng.random((n, m)), 2.0)
        order = np.argsort(key, axis=1)
        nvis = vis.sum(axis=1)
        take = np.minimum(want[start:stop], nvis)
        rank = np.argsort(order, axis=1)
        chosen = rank < take[:, None]
        sel_p, sel_k = np.nonzero(chosen)
        obs_point_parts.append((sel_p + start).astype(np.uint32))
        obs_pose_parts.append(cand[sel_p, sel_k].astype(np.uint32))
        pix_parts.append(pix.reshape(n, m, 2)[sel_p, sel_k])
    obs_point = np.concatenate(obs_point_parts)
    obs_pose = np.concatenate(obs_pose_parts)
    obs = _noisy(rng, np.concatenate(pix_parts))
    Rp, Cp, Xp = _perturb(rng, R, C, X)
    intrinsics = []
    if per_camera_intrinsics:
        for i in range(cameras):
            var = (abi.INTRINSIC_FOCAL | abi.INTRINSIC_RADIAL) if free_intrinsics else 0
            f_init = fs[i] * (1.0 + 0.005 * rng.standard_normal()) if free_intrinsics else fs[i]
            k1_init = k1s[i] + (0.005 * rng.standard_normal() if free_intrinsics else 0.0)
            intrinsics.append(CameraIntrinsics(model=abi.CAMERA_BROWN_CONRADY, fx=f_init, fy=f_init, cx=ppx, cy=ppy,
                                               radial_kind=abi.RADIAL_K1K2, k1=k1_init, k2=k2s[i], variables=var))
        obs_intr = obs_pose.copy()
    else:
        intrinsics.append(CameraIntrinsics(model=abi.CAMERA_BROWN_CONRADY, fx=f0, fy=f0, cx=ppx, cy=ppy,
                                           radial_kind=abi.RADIAL_K1K2, k1=-0.09, k2=0.01))
        obs_intr = np.zeros_like(obs_pose)
    return BundleProblem(
        rotations=Rp, centers=Cp, pose_variables=np.full(cameras, abi.POSE_FREE, dtype=np.uint32),
        intrinsics=intrinsics, points=Xp, point_fixed=np.zeros(points, dtype=np.uint8),
        observation_pose=obs_pose, observation_intrinsic=obs_intr.astype(np.uint32),
        observation_point=obs_point, observation_pixel=obs,
        robust_loss=loss if loss is not None else RobustLoss.huber(1.0), gauge=Gauge(),
    )


def window_problems(seed: int = 23, windows: int = 256, total_observations: int = 1_500_000,
                    min_cameras: int = 5, max_cameras: int = 40, min_points: int = 500,
                    max_points: int = 20_000) -> list:
    """Uneven local-BA windows: cameras uniform in [min_cameras, max_cameras], point counts
    log-uniform in [min_points, max_points] and then scaled together so that the windows hold about
    ``total_observations`` observations (tracks 2-10, capped by the cameras that see a point). The
    scale is set from a first draw's observation count and the windows are drawn again with it."""
    rng = np.random.Generator(np.random.PCG64(seed))
    cams = rng.integers(min_cameras, max_cameras + 1, size=windows)
    raw = np.exp(rng.uniform(np.log(min_points), np.log(max_points), size=windows))
    seeds = rng.integers(1 << 31, size=windows)

    def draw(scale):
        pts = np.clip(np.round(raw * scale), min_points, max_points).astype(int)
        return [plane_problem(seed=int(seeds[w]), cameras=int(cams[w]), points=int(pts[w]), mean_track=6.0,
                              altitude=16.0, extent=30.0, per_camera_intrinsics=False, free_intrinsics=False)
                for w in range(windows)]

    scale = min(1.0, total_observations / (raw.sum() * 6.0))
    first = draw(scale)
    got = sum(p.observation_count for p in first)
    if got == 0 or abs(got - total_observations) < 0.02 * total_observations:
        return first
    return draw(scale * total_observations / got)


def residual_inputs(seed: int = 5, observations: int = 10_000_000, cameras: int = 3000, points: int = 2_000_000,
                    dtype=np.float32):
    """Random radial-camera residual inputs: rotations from random rotation vectors, translations in
    the unit box, points at depths 2-50 in front of their camera, intrinsics (f, k1, k2).

    Each point is placed in front of an owning camera and observed from the owner's 16 cameras with
    the closest viewing directions (the owner included), so a point's gradient sums contributions
    from several cameras, as it does in a real track."""
    rng = np.random.Generator(np.random.PCG64(seed))
    rotvec = rng.normal(0.0, 1.0, size=(cameras, 3))
    rotvec *= (rng.uniform(0, np.pi, size=cameras) / np.linalg.norm(rotvec, axis=1))[:, None]
    t = rng.uniform(0.0, 1.0, size=(cameras, 3))
    intr = np.stack([rng.uniform(400, 600, cameras), rng.uniform(-0.1, 0.0, cameras),
                     rng.uniform(0.0, 0.01, cameras)], axis=1)
    cam = rng.integers(0, cameras, size=observations).astype(np.uint32)
    pt = rng.integers(0, points, size=observations).astype(np.uint32)
    # place each point in front of one of its cameras: camera-frame point at depth 2-50
    owner = rng.integers(0, cameras, size=points)
    depth = rng.uniform(2.0, 50.0, size=points)
    xy = rng.uniform(-0.4, 0.4, size=(points, 2)) * depth[:, None]
    pc = np.concatenate([xy, depth[:, None]], axis=1)
    R = _exp_so3(rotvec)
    X = np.einsum("nji,nj->ni", R[owner], pc - t[owner])  # R^T (pc - t)
    # the 16 cameras whose optical axes (third rows of R) are closest to each camera's, itself first
    axis = R[:, 2, :]
    near = np.argsort(-(axis @ axis.T), axis=1, kind="stable")[:, :16]
    cam = near[owner[pt], rng.integers(0, near.shape[1], size=observations)].astype(np.uint32)
    pix = rng.uniform(-200, 200, size=(observations, 2))
    return {
        "camera_index": cam, "point_index": pt, "pixel": pix.astype(dtype), "rotvec": rotvec.astype(dtype),
        "translation": t.astype(dtype), "intrinsics": intr.astype(dtype), "points": X.astype(dtype),
    }
