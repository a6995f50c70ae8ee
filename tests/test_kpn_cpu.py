"""The oracle's restatement of the kernel-predicting denoiser path (modules/kpn_module/src/Kernel.cu
and the libtorch ops PyTorchDenoiser composes it with) against torch's own CPU implementations of
those ops and an independent torch formulation of the per-pixel kernel."""
import numpy as np
import pytest
import torch
import torch.nn.functional as F

from oracle import bridge


def rnd(*shape, seed=0, scale=1.0):
    return (np.random.default_rng(seed).standard_normal(shape) * scale).astype(np.float32)


def test_softmax_matches_torch():
    x = rnd(2, 25, 9, 13, seed=1, scale=3.0)
    ref = torch.softmax(torch.from_numpy(x), 1).numpy()
    assert np.allclose(bridge.softmax_channels(x), ref, rtol=1e-6, atol=1e-7)


def test_avg_pool_matches_torch():
    x = rnd(2, 4, 17, 22, seed=2)
    ref = F.avg_pool2d(torch.from_numpy(x), 2, 2).numpy()
    assert np.allclose(bridge.avg_pool2(x), ref, rtol=1e-6, atol=1e-7)


def test_grid_sample_matches_torch():
    prev = rnd(2, 4, 20, 24, seed=3)
    uv = np.random.default_rng(4).uniform(-0.1, 1.1, (2, 2, 20, 24)).astype(np.float32)
    ref = F.grid_sample(torch.from_numpy(prev), torch.from_numpy(uv).permute(0, 2, 3, 1) * 2 - 1, mode="bilinear",
                        padding_mode="zeros", align_corners=False).numpy()
    assert np.allclose(bridge.grid_sample(prev, uv), ref, rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("k", [3, 5])
def test_kpn_apply_matches_unfold_formulation(k):
    img = rnd(2, 3, 15, 19, seed=5)
    logits = rnd(2, k * k, 15, 19, seed=6)
    w = torch.softmax(torch.from_numpy(logits), 1)
    cols = F.unfold(torch.from_numpy(img), k, padding=k // 2).view(2, 3, k * k, 15, 19)
    ref = (cols * w[:, None]).sum(2).numpy()
    assert np.allclose(bridge.kpn_apply(img, logits, k, softmax=True), ref, rtol=1e-5, atol=1e-6)


def test_inv_iter_blend_by_hand():
    """One pixel of getInvIterBaseKernel written out, and the double-precision previous-frame blend."""
    k = 3
    x_hi, pred, x_lo, prev = rnd(1, 1, 4, 4, seed=7), rnd(1, 1, 2, 2, seed=8), rnd(1, 1, 2, 2, seed=9), rnd(1, 1, 4, 4, seed=10)
    fused = rnd(1, k * k + 3, 4, 4, seed=11)
    sig = lambda v: np.float32(1.0) / (np.float32(1.0) + np.exp(-v, dtype=np.float32))  # noqa: E731
    lf_w, hf_w, pv_w = sig(fused[0, 9, 3, 2]), sig(fused[0, 10, 3, 2]), sig(fused[0, 11, 3, 2])
    lf = np.float32(lf_w * pred[0, 0, 1, 1] + (np.float32(1) - lf_w) * x_lo[0, 0, 1, 1])
    lf = np.float32(float(lf) * (1.0 - float(pv_w)) + float(np.float32(prev[0, 0, 3, 2] * pv_w)))
    base = hf_w * (x_hi[0, 0, 3, 2] - x_lo[0, 0, 1, 1] + lf) + (np.float32(1) - hf_w) * lf
    # with a one-hot kernel on the centre tap the output is the base itself
    fused2 = fused.copy()
    fused2[:, :k * k] = -40.0
    fused2[:, (k * k) // 2] = 40.0
    out = bridge.kpn_inv_iter(x_hi, pred, x_lo, prev, fused2, k, True)
    assert np.isclose(out[0, 0, 3, 2], base, rtol=1e-6, atol=1e-7)
