"""Oracle (test infrastructure): a CPU restatement of the landmark reprojection-error refresh that
openmvg-sfm runs after a bundle adjustment, for the parity tests only.

refresh_landmark_reprojection_errors_for (crates/openmvg-sfm/src/ops/reconstruction/bundle.rs:510-637)
with the camera residual policy (ops/reconstruction/residual.rs:37-151) and openmvg-core's camera
projection (camera/pinhole.rs:276-298, brown_conrady.rs:240-332, fisheye.rs:182-210, spherical.rs:
147-209) and bearing error (camera_model.rs:238-269). Plain Python loops: small cases only. The
unprojection of a measured pixel comes from the oracle's C++ restatement (oracle.camera_bearing).
Pinned by tests/test_sfm_refresh.py against the reference's own tests of the residual policy
(ops/reconstruction/tests/residual.rs).
"""
import math
from fractions import Fraction

import oracle as O

PINHOLE, BROWN, FISHEYE, SPHERICAL = 0, 1, 2, 3
EPS = 2.220446049250313e-16
MAX_INCIDENT_ANGLE = math.pi - 1e-10  # camera/fisheye.rs:32


def _finite(*v):
    return all(math.isfinite(x) for x in v)


def _fma(a, b, c):
    """a * b + c rounded once (f64::mul_add), exactly through rationals."""
    if not _finite(a, b, c):
        return a * b + c
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def first_radial_turn_squared(k1, k2):
    """distortion.rs:553-574"""
    scale = max(abs(k1), abs(k2), 1.0)
    a, b, c = 5.0 * (k2 / scale), 3.0 * (k1 / scale), 1.0 / scale
    if a == 0.0:
        if b == 0.0:
            return None
        root = -c / b
        return root if (b < 0.0 and math.isfinite(root) and root > 0.0) else None
    disc = b * b - 4.0 * a * c
    if disc < 0.0 or not math.isfinite(disc):
        return None
    q = -0.5 * (b + math.copysign(math.sqrt(disc), b))
    roots = [-b / (2.0 * a)] if q == 0.0 else [q / a, c / q]
    roots = [r for r in roots if math.isfinite(r) and r > 0.0]
    return min(roots) if roots else None


def _coeffs(cam):
    rk, tk = cam.radial_kind, cam.tangential_kind
    return (cam.k1 if rk >= 1 else 0.0, cam.k2 if rk >= 2 else 0.0, cam.k3 if rk >= 3 else 0.0,
            cam.p1 if tk >= 1 else 0.0, cam.p2 if tk >= 2 else 0.0)


def _radial(cam, r2):  # distortion.rs:227-240
    k1, k2, k3, _, _ = _coeffs(cam)
    rk = cam.radial_kind
    if rk == 0:
        return 1.0
    if rk == 1:
        return 1.0 + k1 * r2
    r4 = r2 * r2
    if rk == 2:
        return 1.0 + k1 * r2 + k2 * r4
    return 1.0 + k1 * r2 + k2 * r4 + k3 * (r4 * r2)


def _tangential(cam, x, y, r2):  # distortion.rs:493-506
    _, _, _, p1, p2 = _coeffs(cam)
    if cam.tangential_kind == 0:
        return 0.0, 0.0
    if cam.tangential_kind == 1:
        return 2.0 * p1 * x * y, p1 * (r2 + 2.0 * y * y)
    return (2.0 * p1 * x * y + p2 * (r2 + 2.0 * x * x), p1 * (r2 + 2.0 * y * y) + 2.0 * p2 * x * y)


def _jacobian_det(cam, x, y):  # distortion.rs:613-635
    k1, k2, k3, p1, p2 = _coeffs(cam)
    r2 = _fma(x, x, y * y)
    rf = _radial(cam, r2)
    rd = k1 + 2.0 * (k2 * r2) + 3.0 * (k3 * r2 * r2)
    j11 = rf + 2.0 * x * x * rd + 2.0 * p1 * y + 6.0 * p2 * x
    j12 = 2.0 * x * y * rd + 2.0 * p1 * x + 2.0 * p2 * y
    j22 = rf + 2.0 * y * y * rd + 6.0 * p1 * y + 2.0 * p2 * x
    det = _fma(j11, j22, -j12 * j12)
    return det if _finite(j11, j12, j22, det) else None


def _forward_domain(cam, x, y):  # brown_conrady.rs:240-267, distortion.rs:580-602
    if not _finite(x, y):
        return False
    if cam.radial_kind == 0 and cam.tangential_kind == 0:
        return True
    k1, k2, k3, p1, p2 = _coeffs(cam)
    if k3 == 0.0 and p1 == 0.0 and p2 == 0.0:
        r2 = _fma(x, x, y * y)
        if not math.isfinite(r2):
            return False
        turn = first_radial_turn_squared(k1, k2)
        if turn is not None and r2 >= turn:
            return False
        d = _jacobian_det(cam, x, y)
        return d is not None and d > 1e-12
    for i in range(33):
        s = i / 32.0
        d = _jacobian_det(cam, x * s, y * s)
        if d is None or not d > 1e-12:
            return False
    return True


def _normalize(d):  # camera_model.rs:91-109
    if not _finite(*d):
        return None
    s = max(abs(d[0]), abs(d[1]), abs(d[2]))
    if s == 0.0:
        return None
    x = [v / s for v in d]
    n = math.sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2])
    if not math.isfinite(n) or n == 0.0:
        return None
    return [v / n for v in x]


def _fisheye_apply(cam, t):  # distortion.rs:319-330
    ks = [cam.k1, cam.k2, cam.k3, cam.k4][:cam.radial_kind]
    t2 = t * t
    t4 = t2 * t2
    terms = [t2, t4, t4 * t2, t4 * t4]
    acc = 1.0
    for k, p in zip(ks, terms):
        acc += k * p
    return t * acc


def project(cam, X):
    """Camera::project: the pixel, or None outside the model's domain."""
    if cam.model in (PINHOLE, BROWN):
        if not _finite(*X) or X[2] <= 0.0:
            return None
        if cam.model == PINHOLE:  # pinhole.rs:276-298
            inv = 1.0 / X[2]
            u, v = _fma(cam.fx, X[0] * inv, cam.cx), _fma(cam.fy, X[1] * inv, cam.cy)
            return (u, v) if _finite(u, v) else None
        x, y = X[0] / X[2], X[1] / X[2]  # brown_conrady.rs:310-332
        if not _forward_domain(cam, x, y):
            return None
        r2 = x * x + y * y
        rf = _radial(cam, r2)
        dx, dy = _tangential(cam, x, y, r2)
        xd, yd = x * rf + dx, y * rf + dy
        u, v = _fma(cam.fx, xd * 1.0, cam.cx), _fma(cam.fy, yd * 1.0, cam.cy)
        return (u, v) if _finite(u, v) else None
    d = _normalize(X)
    if d is None:
        return None
    if cam.model == FISHEYE:  # fisheye.rs:182-210
        radial = math.hypot(d[0], d[1])
        if radial == 0.0:
            return (cam.cx, cam.cy) if d[2] > 0.0 else None
        theta = math.atan2(radial, d[2])
        if theta > fisheye_max_angle(cam) + 1e-12:
            return None
        scale = _fisheye_apply(cam, theta) / radial
        u, v = _fma(cam.fx, d[0] * scale, cam.cx), _fma(cam.fy, d[1] * scale, cam.cy)
        return (u, v) if _finite(u, v) else None
    lon, lat = math.atan2(d[0], d[2]), math.atan2(d[1], math.hypot(d[0], d[2]))  # spherical.rs:147-209
    w, h = float(cam.width), float(cam.width // 2)
    return (((lon + math.pi) * w / (2.0 * math.pi)) % w - 0.5, (lat + math.pi / 2.0) * h / math.pi - 0.5)


def _fisheye_derivative(cam, t):
    k = [cam.k1, cam.k2, cam.k3, cam.k4][:cam.radial_kind] + [0.0] * (4 - cam.radial_kind)
    t2 = t * t
    t4 = t2 * t2
    return 1.0 + 3.0 * k[0] * t2 + 5.0 * k[1] * t4 + 7.0 * k[2] * (t4 * t2) + 9.0 * k[3] * (t4 * t4)


def fisheye_max_angle(cam, max_theta=MAX_INCIDENT_ANGLE):
    """FisheyeDistortion::max_invertible_angle (distortion.rs:416-456)"""
    k = [cam.k1, cam.k2, cam.k3, cam.k4][:cam.radial_kind] + [0.0] * (4 - cam.radial_kind)
    if k[2] == 0.0 and k[3] == 0.0:
        q = first_radial_turn_squared(k[0], k[1])
        return max_theta if q is None else min(math.sqrt(q), max_theta)
    if all(v >= 0.0 for v in k):
        return max_theta
    previous = 0.0
    for i in range(1, 1025):
        t = max_theta * i / 1024.0
        if _fisheye_derivative(cam, t) <= 0.0:
            lo, hi = previous, t
            for _ in range(64):
                mid = 0.5 * (lo + hi)
                if _fisheye_derivative(cam, mid) > 0.0:
                    lo = mid
                else:
                    hi = mid
            return lo
        previous = t
    return max_theta


def is_generalized(cam):  # residual.rs:149-151
    return cam.model in (FISHEYE, SPHERICAL)


def pixels_per_radian(cam):
    """nominal_pixels_per_radian (residual.rs:96-115); None where the policy would fail."""
    s = cam.width / (2.0 * math.pi) if cam.model == SPHERICAL else min(abs(cam.fx), abs(cam.fy))
    return s if (math.isfinite(s) and s > 0.0) else None


def pixel_equivalent(cam, xc, pixel):
    """CameraResidualPolicy::from_pixel_limit(camera, inf).evaluate(...).pixel_equivalent
    (residual.rs:37-90); None when it does not exist or is not finite."""
    projected = project(cam, xc)
    if projected is None:
        return None
    if not is_generalized(cam):  # camera_pixel_residual (residual.rs:117-138)
        if not _finite(*projected, *pixel):
            return None
        r = math.hypot(projected[0] - pixel[0], projected[1] - pixel[1])
    else:  # Camera::bearing_error_rad (camera_model.rs:238-269)
        observed = O.camera_bearing(cam, pixel[0], pixel[1])
        predicted = _normalize(xc)
        if observed is None or predicted is None:
            return None
        chord2 = sum((a - b) * (a - b) for a, b in zip(predicted, observed))
        if not math.isfinite(chord2):
            return None
        chord2 = min(max(chord2, 0.0), 4.0)
        r = 2.0 * math.asin(min(max(0.5 * math.sqrt(chord2), 0.0), 1.0)) * pixels_per_radian(cam)
    return r if math.isfinite(r) else None


def camera_point(R, C, X):
    d = [X[k] - C[k] for k in range(3)]
    return [R[r][0] * d[0] + R[r][1] * d[1] + R[r][2] * d[2] for r in range(3)]


def refresh(rotations, centers, intrinsics, tracks, reprojection_error):
    """refresh_landmark_reprojection_errors_for (bundle.rs:510-637) over every landmark.
    Returns (update, error, support, rejected, removed) with the abi.REFRESH_* codes."""
    L = len(tracks.points)
    update, error = [0] * L, list(reprojection_error)
    support = [int(v) for v in tracks.track_support]
    rejected = removed = 0
    for l in range(L):
        if not tracks.active[l]:
            continue
        a, b = int(tracks.track_offset[l]), int(tracks.track_offset[l + 1])
        total, kept, supporting, keep = 0.0, 0, 0, []
        for o in range(a, b):
            if not tracks.track_support[o]:
                continue
            supporting += 1
            p = int(tracks.track_pose[o])
            if p == 0xFFFFFFFF:  # the view has no pose
                continue
            cam = intrinsics[int(tracks.track_intrinsic[o])]
            r = pixel_equivalent(cam, camera_point(rotations[p], centers[p], tracks.points[l]),
                                 tracks.track_pixel[o])
            if r is not None:
                total += r
                kept += 1
                keep.append(o)
        if kept < 2:
            update[l] = 1
            rejected += 1
        elif kept == supporting:
            update[l] = 2
            error[l] = total / kept
        else:
            update[l] = 3
            error[l] = total / kept
            removed += supporting - kept
            for o in range(a, b):
                support[o] = 1 if o in keep else 0
    return update, error, support, rejected, removed


def bearing_error_rad(cam, xc, pixel):
    """Camera::bearing_error_rad (camera_model.rs:238-269), or None outside the model's domain."""
    if project(cam, xc) is None:
        return None
    observed = O.camera_bearing(cam, pixel[0], pixel[1])
    predicted = _normalize(xc)
    if observed is None or predicted is None:
        return None
    chord2 = sum((a - b) * (a - b) for a, b in zip(predicted, observed))
    if not math.isfinite(chord2):
        return None
    return 2.0 * math.asin(min(max(0.5 * math.sqrt(min(max(chord2, 0.0), 4.0)), 0.0), 1.0))


def prepare(view_pose, view_intrinsic, view_size, intrinsics, guess, tracks, scope=0, fixed_views=(),
            fixed_landmarks=(), excluded_landmarks=(), loss=(0, 0.0, 0), gauge=(0, 0, 0, 0.0)):
    """prepare_bundle_adjustment_problem (bundle.rs:707-989) on row tables. Returns a dict of the
    problem's arrays and the row maps; raises ValueError where the reference returns an error."""
    NO = 0xFFFFFFFF
    V = len(view_pose)
    pose_rows = sorted({int(view_pose[v]) for v in range(V) if view_pose[v] != NO})
    intr_rows = sorted({int(view_intrinsic[v]) for v in range(V) if view_pose[v] != NO})
    fixed_poses = set()
    for v in fixed_views:
        if view_pose[v] == NO:
            raise ValueError("a fixed view has no pose")
        fixed_poses.add(int(view_pose[v]))
    pose_index = {p: i for i, p in enumerate(pose_rows)}
    intr_index = {r: i for i, r in enumerate(intr_rows)}
    pose_vars = []
    for p in pose_rows:  # bundle.rs:764-772
        if p in fixed_poses or scope == 1:
            pose_vars.append(0)
        elif scope == 3:
            pose_vars.append(2)
        else:
            pose_vars.append(3)
    out_intr = []
    for r in intr_rows:  # bundle.rs:784-846
        sizes = {(int(view_size[v][0]), int(view_size[v][1])) for v in range(V) if view_intrinsic[v] == r}
        if len(sizes) != 1:
            raise ValueError("intrinsic shared by images with different dimensions")
        w, h = sizes.pop()
        cam = intrinsics[r]
        fixed = scope != 4 or is_generalized(cam)
        out_intr.append(dict(row=r, width=w, height=h, fixed_model=int(fixed), variables=0 if fixed else (1 | 4),
                             certification=int(bool(guess[r]))))
    excluded, fixed_l = set(excluded_landmarks), set(fixed_landmarks)
    rows = [l for l in range(len(tracks.points)) if tracks.active[l] and l not in excluded]
    point_fixed = [int(l in fixed_l or scope == 2) for l in rows]
    obs = []
    for k, l in enumerate(rows):  # bundle.rs:871-920
        for o in range(int(tracks.track_offset[l]), int(tracks.track_offset[l + 1])):
            v = int(tracks.track_pose[o])
            if tracks.track_support[o] and view_pose[v] != NO:
                obs.append((pose_index[int(view_pose[v])], intr_index[int(view_intrinsic[v])], k,
                            float(tracks.track_pixel[o][0]), float(tracks.track_pixel[o][1])))
    gk, g0, g1, gd = gauge  # bundle.rs:937-963
    first = second = 0
    if gk == 1:
        for v in (g0, g1):
            if v >= V or view_pose[v] == NO or int(view_pose[v]) not in pose_index:
                raise ValueError("fixed-baseline anchor is missing")
        first, second = pose_index[int(view_pose[g0])], pose_index[int(view_pose[g1])]
    space = 1 if any(is_generalized(intrinsics[r]) for r in intr_rows) else 0  # :964-973
    steps = [2.0 * math.pi / out_intr[i]["width"] if intrinsics[r].model == SPHERICAL else 1.0 / intrinsics[r].fx
             for i, r in enumerate(intr_rows)]
    total = 0.0
    for s_ in steps:
        total += s_
    rpp = total / max(len(steps), 1)  # mean_radians_per_pixel (:991-1004)
    kind, scale, scale_space = loss  # canonical_robust_loss (:1006-1032)
    if kind != 0 and scale_space != space:
        if scale_space != 0:
            raise ValueError("robust-loss units do not match the BA residual domain")
        scale, scale_space = scale * rpp, 1
    return dict(pose_rows=pose_rows, pose_vars=pose_vars, intrinsics=out_intr, landmark_rows=rows,
                point_fixed=point_fixed, observations=obs, gauge=(gk, first, second, gd if gk == 1 else 0.0),
                residual_space=space, loss=(kind, scale, scale_space))
