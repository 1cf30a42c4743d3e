"""``ReprojectionResidual``: the radial-camera reprojection residual as a torch.autograd.Function.

Forward and backward call the library's CUDA kernels through the C ABI
(``omvgba_residual_forward_f32`` / ``omvgba_residual_vjp_f32``) on torch's current stream; the
backward is the hand-written adjoint kernel, deterministic run to run. There is no CPU path: the
tensors must live on a CUDA device and the library must be built.

Model (crates/openmvg-ba/src/kernel/multi_view/self_calibration/model.rs:26-129): for observation i
of camera j and point p, X_c = exp(rotvec_j) X_p + t_j, n = X_c.xy / X_c.z and
residual_i = f_j (1 + k1_j |n|^2 + k2_j |n|^4) n - pixel_i. Inadmissible observations give NaN
residuals and no gradient. Indices are checked on the device: an out-of-range camera or point index
gives that observation a NaN residual and makes the backward's gradients NaN (no memory outside the
inputs is read or written).
"""
from __future__ import annotations

import ctypes as C

import torch

from . import abi
from ._lib import lib
from .problem import raise_for


def _check(t: torch.Tensor, name: str, dtype, shape_tail=None, device=None) -> torch.Tensor:
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if device is not None and t.device != device:
        raise ValueError(f"{name} is on {t.device}, the other inputs on {device}")
    if t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
    if shape_tail is not None and tuple(t.shape[1:]) != shape_tail:
        raise ValueError(f"{name} must have shape (n, {', '.join(map(str, shape_tail))})")
    return t.contiguous()


class ReprojectionResidual(torch.autograd.Function):
    """residual = ReprojectionResidual.apply(camera_index, point_index, pixel, rotvec, translation,
    intrinsics, points); indices int32 (n,), pixel (n, 2), rotvec / translation / intrinsics
    (cameras, 3), points (points, 3), all float32 on one CUDA device."""

    @staticmethod
    def forward(ctx, camera_index, point_index, pixel, rotvec, translation, intrinsics, points):
        px = _check(pixel, "pixel", torch.float32, (2,))
        dev = px.device
        cam = _check(camera_index, "camera_index", torch.int32, device=dev)
        pt = _check(point_index, "point_index", torch.int32, device=dev)
        rv = _check(rotvec, "rotvec", torch.float32, (3,), dev)
        tr = _check(translation, "translation", torch.float32, (3,), dev)
        it = _check(intrinsics, "intrinsics", torch.float32, (3,), dev)
        X = _check(points, "points", torch.float32, (3,), dev)
        if cam.shape[0] != px.shape[0] or pt.shape[0] != px.shape[0]:
            raise ValueError("camera_index, point_index and pixel must have one row per observation")
        n = cam.shape[0]
        residual = torch.empty((n, 2), dtype=torch.float32, device=px.device)
        err = abi.Error()
        stream = torch.cuda.current_stream(px.device).cuda_stream
        code = lib().omvgba_residual_forward_f32(stream, n, cam.data_ptr(), pt.data_ptr(), px.data_ptr(),
                                                 rv.shape[0], rv.data_ptr(), tr.data_ptr(), it.data_ptr(),
                                                 X.shape[0], X.data_ptr(), residual.data_ptr(), C.byref(err))
        raise_for(code, err)
        ctx.save_for_backward(cam, pt, px, rv, tr, it, X)
        return residual

    @staticmethod
    def backward(ctx, grad_residual):
        cam, pt, px, rv, tr, it, X = ctx.saved_tensors
        g = grad_residual.contiguous().to(torch.float32)
        grads = vjp(cam, pt, px, rv, tr, it, X, g)
        return (None, None, None) + grads


def vjp(cam, pt, px, rv, tr, it, X, grad_residual):
    """(d rotvec, d translation, d intrinsics, d points) = J^T grad_residual by the adjoint kernel.
    An out-of-range camera or point index makes every returned gradient NaN."""
    dev = px.device
    for t, name in ((cam, "camera_index"), (pt, "point_index"), (rv, "rotvec"), (tr, "translation"),
                    (it, "intrinsics"), (X, "points"), (grad_residual, "grad_residual")):
        if t.device != dev:
            raise ValueError(f"{name} is on {t.device}, the other inputs on {dev}")
        if not t.is_contiguous():
            raise ValueError(f"{name} must be contiguous")
    if grad_residual.dtype != torch.float32 or tuple(grad_residual.shape) != (cam.shape[0], 2):
        raise ValueError("grad_residual must be float32 with shape (n, 2)")
    n = cam.shape[0]
    g_rot, g_t, g_int, g_pt = (torch.zeros_like(a) for a in (rv, tr, it, X))
    ws_bytes = int(lib().omvgba_residual_vjp_workspace_bytes(n, rv.shape[0], X.shape[0]))
    workspace = torch.empty(max(ws_bytes, 256), dtype=torch.uint8, device=px.device)
    err = abi.Error()
    stream = torch.cuda.current_stream(px.device).cuda_stream
    code = lib().omvgba_residual_vjp_f32(stream, n, cam.data_ptr(), pt.data_ptr(), px.data_ptr(), rv.shape[0],
                                         rv.data_ptr(), tr.data_ptr(), it.data_ptr(), X.shape[0], X.data_ptr(),
                                         grad_residual.data_ptr(), g_rot.data_ptr(), g_t.data_ptr(),
                                         g_int.data_ptr(), g_pt.data_ptr(), workspace.data_ptr(), workspace.numel(),
                                         C.byref(err))
    raise_for(code, err)
    return g_rot, g_t, g_int, g_pt


def reprojection_residual(camera_index, point_index, pixel, rotvec, translation, intrinsics, points):
    return ReprojectionResidual.apply(camera_index, point_index, pixel, rotvec, translation, intrinsics, points)


def residual_f64(camera_index, point_index, pixel, rotvec, translation, intrinsics, points) -> torch.Tensor:
    """FP64 forward (no autograd), for finite-difference checks of the adjoint."""
    px = _check(pixel, "pixel", torch.float64, (2,))
    dev = px.device
    cam = _check(camera_index, "camera_index", torch.int32, device=dev)
    pt = _check(point_index, "point_index", torch.int32, device=dev)
    rv, tr, it, X = (_check(a, nm, torch.float64, (3,), dev) for a, nm in
                     ((rotvec, "rotvec"), (translation, "translation"), (intrinsics, "intrinsics"),
                      (points, "points")))
    if cam.shape[0] != px.shape[0] or pt.shape[0] != px.shape[0]:
        raise ValueError("camera_index, point_index and pixel must have one row per observation")
    residual = torch.empty((cam.shape[0], 2), dtype=torch.float64, device=px.device)
    err = abi.Error()
    stream = torch.cuda.current_stream(px.device).cuda_stream
    code = lib().omvgba_residual_forward_f64(stream, cam.shape[0], cam.data_ptr(), pt.data_ptr(), px.data_ptr(),
                                             rv.shape[0], rv.data_ptr(), tr.data_ptr(), it.data_ptr(), X.shape[0],
                                             X.data_ptr(), residual.data_ptr(), C.byref(err))
    raise_for(code, err)
    return residual
