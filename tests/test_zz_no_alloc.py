"""omvgba_residual_vjp_f32_static (no device allocation, static scratch) against the workspace entry
point omvgba_residual_vjp_f32, through the C ABI, on two calls in a row."""
import ctypes as C

import numpy as np
import pytest

from openmvg_ba_cuda import abi, synthetic
from openmvg_ba_cuda._lib import lib

N_OBS, N_CAM, N_PTS = 200_000, 300, 40_000


def _call_static(stream, n, ptrs, ncam, npts, grads):
    err = abi.Error()
    code = lib().omvgba_residual_vjp_f32_static(stream, n, ptrs["cam"], ptrs["pt"], ptrs["px"], ncam, ptrs["rv"],
                                                ptrs["tr"], ptrs["it"], npts, ptrs["X"], ptrs["g"], *grads,
                                                C.byref(err))
    return code, err


def test_sizes_beyond_the_static_scratch_are_rejected_before_device_work():
    limit = 16 * 1024 * 1024
    need = lib().omvgba_residual_vjp_workspace_bytes(10, 3000, 2_000_000)
    assert need > limit
    ptrs = {k: None for k in ("cam", "pt", "px", "rv", "tr", "it", "X", "g")}
    code, err = _call_static(None, 10, ptrs, 3000, 2_000_000, [None] * 4)
    assert code == abi.OMVGBA_INVALID_ARGUMENT
    assert b"static scratch" in err.message and str(limit).encode() in err.message


@pytest.mark.gpu
def test_static_scratch_vjp_matches_the_workspace_vjp_on_two_calls():
    import torch
    d = synthetic.residual_inputs(seed=33, observations=N_OBS, cameras=N_CAM, points=N_PTS, dtype=np.float32)
    dev = "cuda"
    cam = torch.as_tensor(d["camera_index"].astype(np.int32), device=dev)
    pt = torch.as_tensor(d["point_index"].astype(np.int32), device=dev)
    px, rv, tr, it, X = (torch.as_tensor(d[k], device=dev) for k in
                         ("pixel", "rotvec", "translation", "intrinsics", "points"))
    g = torch.randn(N_OBS, 2, device=dev, generator=torch.Generator(dev).manual_seed(5))
    ptrs = {"cam": cam.data_ptr(), "pt": pt.data_ptr(), "px": px.data_ptr(), "rv": rv.data_ptr(),
            "tr": tr.data_ptr(), "it": it.data_ptr(), "X": X.data_ptr(), "g": g.data_ptr()}
    stream = torch.cuda.current_stream().cuda_stream

    # the existing entry point, with a caller-provided workspace
    ref = [torch.zeros_like(a) for a in (rv, tr, it, X)]
    ws_bytes = int(lib().omvgba_residual_vjp_workspace_bytes(N_OBS, N_CAM, N_PTS))
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    err = abi.Error()
    code = lib().omvgba_residual_vjp_f32(stream, N_OBS, ptrs["cam"], ptrs["pt"], ptrs["px"], N_CAM, ptrs["rv"],
                                         ptrs["tr"], ptrs["it"], N_PTS, ptrs["X"], ptrs["g"],
                                         *[a.data_ptr() for a in ref], ws.data_ptr(), ws_bytes, C.byref(err))
    assert code == abi.OMVGBA_OK, err.message
    torch.cuda.synchronize()

    for call in range(2):  # two calls in a row share the static scratch
        out = [torch.zeros_like(a) for a in (rv, tr, it, X)]
        torch.cuda.synchronize()
        # the first call may load the module that holds the array (lazy module loading); from the
        # second call on, neither torch's allocator nor the device's free memory may change
        allocated, (free, _) = torch.cuda.memory_allocated(), torch.cuda.mem_get_info()
        code, err = _call_static(stream, N_OBS, ptrs, N_CAM, N_PTS, [a.data_ptr() for a in out])
        assert code == abi.OMVGBA_OK, err.message
        torch.cuda.synchronize()
        if call == 1:
            assert torch.cuda.memory_allocated() == allocated
            assert torch.cuda.mem_get_info()[0] == free
        for got, want in zip(out, ref):
            # the tolerance of the adjoint's parity tests (relative norm 2e-4) ...
            rel = float(torch.linalg.vector_norm((got - want).double()) / torch.linalg.vector_norm(want.double()))
            assert rel < 2e-4
            # ... and, since both run the same deterministic kernels, the same bits
            assert torch.equal(got, want)
