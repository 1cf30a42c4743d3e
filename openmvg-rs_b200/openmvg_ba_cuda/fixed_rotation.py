"""The observability probe of translation-only problems, in numpy form.

Mirrors ``FixedRotationProblem`` / ``FixedRotationObservabilityProbeOptions``
(``crates/openmvg-ba/src/kernel/fixed_rotation/api.rs``): fixed rotations and intrinsics per camera,
camera centres, points and their tracks, a gauge (anchor and scale camera) and a robust loss.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import abi


@dataclass
class ProbeOptions:
    """FixedRotationObservabilityProbeOptions::default (api.rs)."""

    max_tracks: int = 25_000
    max_observations: int = 100_000
    max_observations_per_track: int = 32
    max_coverage_observations_per_track: int = 256
    max_reduced_nonzeros: int = 1_000_000
    max_factor_nonzeros: int = 4_000_000
    max_symbolic_dense_nonzeros: int = 32_000_000
    minimum_normalized_eigenvalue: float = 1e-10

    def to_struct(self) -> abi.ProbeOptions:
        s = abi.ProbeOptions()
        for name, _ in abi.ProbeOptions._fields_:
            setattr(s, name, getattr(self, name))
        return s


@dataclass
class FixedRotationProblem:
    """rotations (n, 3, 3) world-to-camera; centers (n, 3); intrinsics (n, 9): fx, fy, cx, cy, k1, k2,
    k3, p1, p2; tracks: one list of (camera, x, y) per point."""

    rotations: np.ndarray
    centers: np.ndarray
    points: np.ndarray
    intrinsics: np.ndarray
    tracks: list
    fixed_cameras: np.ndarray = None
    gauge_kind: int = abi.GAUGE_FREE
    anchor: int = 0
    scale_camera: int = 1
    distance: float = 0.0
    loss_kind: int = abi.LOSS_SQUARED
    loss_scale: float = 0.0
    _keep: list = field(default_factory=list, repr=False)

    def to_struct(self) -> abi.FixedRotationProblem:
        n = len(self.centers)
        rot = np.ascontiguousarray(np.asarray(self.rotations, dtype=np.float64).reshape(n, 9))
        cen = np.ascontiguousarray(np.asarray(self.centers, dtype=np.float64).reshape(n, 3))
        intr = np.ascontiguousarray(np.asarray(self.intrinsics, dtype=np.float64).reshape(n, 9))
        fixed = np.zeros(n, dtype=np.uint8) if self.fixed_cameras is None else \
            np.ascontiguousarray(np.asarray(self.fixed_cameras, dtype=np.uint8))
        pts = np.ascontiguousarray(np.asarray(self.points, dtype=np.float64).reshape(-1, 3))
        off = np.zeros(len(self.tracks) + 1, dtype=np.uint64)
        off[1:] = np.cumsum([len(t) for t in self.tracks])
        cams = np.array([o[0] for t in self.tracks for o in t], dtype=np.uint32)
        pix = np.array([[o[1], o[2]] for t in self.tracks for o in t], dtype=np.float64).reshape(-1, 2)
        self._keep = [rot, cen, intr, fixed, pts, off, cams, pix]
        s = abi.FixedRotationProblem()
        dp = C.POINTER(C.c_double)
        s.camera_count = n
        s.rotations = rot.ctypes.data_as(dp)
        s.centers = cen.ctypes.data_as(dp)
        s.intrinsics = intr.ctypes.data_as(dp)
        s.fixed_cameras = fixed.ctypes.data_as(C.POINTER(C.c_uint8))
        s.point_count = len(self.tracks)
        s.points = pts.ctypes.data_as(dp)
        s.track_offsets = off.ctypes.data_as(C.POINTER(C.c_uint64))
        s.observation_camera = cams.ctypes.data_as(C.POINTER(C.c_uint32))
        s.observation_pixel = pix.ctypes.data_as(dp)
        s.gauge_kind = self.gauge_kind
        s.anchor = self.anchor
        s.scale_camera = self.scale_camera
        s.distance = self.distance
        s.loss_kind = self.loss_kind
        s.loss_scale = self.loss_scale
        return s
