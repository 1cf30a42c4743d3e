"""Residual kernel and its adjoint (VJP) against the oracle's analytic Jacobian and against central
finite differences of the FP64 forward (h = 1e-4), through the C ABI and the autograd Function."""
import numpy as np
import pytest

import oracle
from openmvg_ba_cuda import synthetic

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

N_OBS, N_CAM, N_PTS = 200_000, 300, 40_000


@pytest.fixture(scope="module")
def inputs():
    d = synthetic.residual_inputs(seed=21, observations=N_OBS, cameras=N_CAM, points=N_PTS, dtype=np.float64)
    # a few inadmissible observations: points moved behind the camera that observes them
    R = synthetic._exp_so3(d["rotvec"])
    for p in range(50):
        obs = np.nonzero(d["point_index"] == p)[0]
        if len(obs):
            j = d["camera_index"][obs[0]]
            d["points"][p] = R[j].T @ (np.array([0.3, -0.2, -5.0]) - d["translation"][j])
    return d


def to_dev(d, dtype):
    dev = "cuda"
    return (torch.as_tensor(d["camera_index"].astype(np.int32), device=dev),
            torch.as_tensor(d["point_index"].astype(np.int32), device=dev),
            *(torch.as_tensor(d[k], dtype=dtype, device=dev)
              for k in ("pixel", "rotvec", "translation", "intrinsics", "points")))


def test_forward_f64_matches_oracle(inputs):
    from openmvg_ba_cuda.autograd import residual_f64
    ref, _ = oracle.residual_vjp(inputs)
    got = residual_f64(*to_dev(inputs, torch.float64)).cpu().numpy()
    nan_ref, nan_got = np.isnan(ref), np.isnan(got)
    assert np.array_equal(nan_ref, nan_got)
    ok = ~nan_ref
    assert np.max(np.abs(got[ok] - ref[ok]) / (1.0 + np.abs(ref[ok]))) < 1e-10


def test_forward_f32_matches_oracle(inputs):
    from openmvg_ba_cuda.autograd import reprojection_residual
    ref, _ = oracle.residual_vjp(inputs)
    got = reprojection_residual(*to_dev(inputs, torch.float32)).cpu().numpy().astype(np.float64)
    ok = ~np.isnan(ref)
    assert np.array_equal(np.isnan(got), ~ok)
    # FP32 arithmetic on pixel-scale predictions: absolute tolerance in pixels
    assert np.max(np.abs(got[ok] - ref[ok])) < 2e-3


def test_vjp_matches_oracle_analytic_jacobian(inputs):
    from openmvg_ba_cuda.autograd import vjp
    rng = np.random.default_rng(4)
    g = rng.normal(size=(N_OBS, 2))
    _, ref = oracle.residual_vjp(inputs, g)
    t = to_dev(inputs, torch.float32)
    got = vjp(*t, torch.as_tensor(g, dtype=torch.float32, device="cuda"))
    for name, val in zip(("rotvec", "translation", "intrinsics", "points"), got):
        v = val.cpu().numpy().astype(np.float64)
        r = ref[name]
        rel = np.linalg.norm(v - r) / np.linalg.norm(r)
        assert rel < 2e-4, (name, rel)


def test_vjp_matches_central_differences_of_the_f64_forward(inputs):
    """<J^T g, v> against (r(x + h v) - r(x - h v)) . g / 2h, h = 1e-4, per input block."""
    from openmvg_ba_cuda.autograd import residual_f64, vjp
    rng = np.random.default_rng(8)
    g = rng.normal(size=(N_OBS, 2))
    t64 = list(to_dev(inputs, torch.float64))
    base_nan = torch.isnan(residual_f64(*t64)).any(dim=1)
    g[base_nan.cpu().numpy()] = 0.0
    gt = torch.as_tensor(g, device="cuda")
    grads = vjp(*to_dev(inputs, torch.float32), gt.to(torch.float32))
    h = 1e-4
    for slot, grad in zip(range(3, 7), grads):
        v = torch.as_tensor(rng.normal(size=tuple(t64[slot].shape)), device="cuda")
        plus, minus = list(t64), list(t64)
        plus[slot] = t64[slot] + h * v
        minus[slot] = t64[slot] - h * v
        rp, rm = residual_f64(*plus), residual_f64(*minus)
        fd = torch.nan_to_num((rp - rm) / (2 * h)) * gt
        fd = float(fd.sum())
        an = float((grad.to(torch.float64) * v).sum())
        assert abs(fd - an) <= 1e-3 * abs(fd) + 1e-6, (slot, fd, an)


def test_vjp_is_deterministic(inputs):
    from openmvg_ba_cuda.autograd import vjp
    t = to_dev(inputs, torch.float32)
    g = torch.randn(N_OBS, 2, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    a = vjp(*t, g)
    b = vjp(*t, g)
    for x, y in zip(a, b):
        assert torch.equal(x, y)


def test_autograd_function_backward_is_the_vjp(inputs):
    from openmvg_ba_cuda.autograd import reprojection_residual, vjp
    cam, pt, px, rv, tr, it, X = to_dev(inputs, torch.float32)
    leaves = [a.clone().requires_grad_(True) for a in (rv, tr, it, X)]
    res = reprojection_residual(cam, pt, px, *leaves)
    g = torch.randn_like(res)
    g[torch.isnan(res)] = 0.0
    res_ok = torch.nan_to_num(res)
    (res_ok * g).sum().backward()
    direct = vjp(cam, pt, px, rv, tr, it, X, g)
    for leaf, d in zip(leaves, direct):
        assert torch.equal(leaf.grad, d)


def test_inadmissible_observations_are_nan_without_gradient(inputs):
    from openmvg_ba_cuda.autograd import reprojection_residual, vjp
    cam, pt, px, rv, tr, it, X = to_dev(inputs, torch.float32)
    res = reprojection_residual(cam, pt, px, rv, tr, it, X)
    bad = torch.isnan(res).any(dim=1)
    assert int(bad.sum()) > 0
    g = torch.zeros_like(res)
    g[bad] = 1.0  # upstream gradient only on inadmissible observations
    for x in vjp(cam, pt, px, rv, tr, it, X, g):
        assert float(x.abs().max()) == 0.0


def test_out_of_range_indices_give_nan_not_a_fault(inputs):
    """A camera index past the camera count and a negative point index are caught on the device: the
    forward gives those observations NaN residuals and the adjoint returns NaN gradients; the rest of
    the forward is unchanged and later calls on the same context still work."""
    from openmvg_ba_cuda.autograd import reprojection_residual, vjp
    cam, pt, px, rv, tr, it, X = to_dev(inputs, torch.float32)
    good = reprojection_residual(cam, pt, px, rv, tr, it, X)
    bad_cam, bad_pt = cam.clone(), pt.clone()
    bad_cam[5] = N_CAM
    bad_pt[7] = -1
    res = reprojection_residual(bad_cam, bad_pt, px, rv, tr, it, X)
    assert bool(torch.isnan(res[5]).all()) and bool(torch.isnan(res[7]).all())
    keep = torch.ones(N_OBS, dtype=torch.bool, device="cuda")
    keep[5] = keep[7] = False
    assert torch.equal(torch.isnan(res[keep]), torch.isnan(good[keep]))
    assert torch.equal(torch.nan_to_num(res[keep]), torch.nan_to_num(good[keep]))
    g = torch.ones(N_OBS, 2, device="cuda")
    for x in vjp(bad_cam, bad_pt, px, rv, tr, it, X, g):
        assert bool(torch.isnan(x).all())
    torch.cuda.synchronize()
    for x in vjp(cam, pt, px, rv, tr, it, X, g):  # the context is still usable
        assert bool(torch.isfinite(x).any())
