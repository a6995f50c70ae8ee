"""The kernel-predicting denoiser kernels of the CUDA core (vpt_kpn_*) against the oracle's
restatement of modules/kpn_module/src/Kernel.cu and the libtorch ops around it.  Float work:
rtol 1e-5 (the fused softmax sums its taps in another order than the oracle)."""
import numpy as np
import pytest
import torch

from cloudrendering_b200 import kpn
from oracle import bridge

pytestmark = pytest.mark.gpu
RTOL, ATOL = 1e-5, 1e-6


def rnd(*shape, seed=0, scale=1.0):
    return (np.random.default_rng(seed).standard_normal(shape) * scale).astype(np.float32)


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("k,shape", [(3, (1, 3, 17, 23)), (5, (2, 4, 32, 40)), (5, (1, 4, 9, 7))])
def test_apply_matches_oracle(k, shape):
    n, c, h, w = shape
    img, logits = rnd(*shape, seed=1), rnd(n, k * k, h, w, seed=2, scale=2.0)
    got = kpn.apply_kernels(cuda(img), cuda(logits), k).cpu().numpy()
    assert np.allclose(got, bridge.kpn_apply(img, logits, k, softmax=True), rtol=RTOL, atol=ATOL)


def test_apply_output_size_is_min_of_image_and_weights():
    img, logits = rnd(1, 3, 20, 18, seed=3), rnd(1, 9, 16, 22, seed=4)
    got = kpn.apply_kernels(cuda(img), cuda(logits), 3).cpu().numpy()
    ref = bridge.kpn_apply(img, logits, 3, softmax=True)
    assert got.shape == ref.shape == (1, 3, 16, 18)
    assert np.allclose(got, ref, rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("use_prev", [False, True])
@pytest.mark.parametrize("n,k", [(1, 5), (2, 3)])
def test_inv_iter_matches_oracle(use_prev, n, k):
    c, h, w = 4, 26, 30
    x_hi, prev = rnd(n, c, h, w, seed=5), rnd(n, c, h, w, seed=6)
    x_lo, pred = rnd(n, c, h // 2, w // 2, seed=7), rnd(n, c, h // 2, w // 2, seed=8)
    fused = rnd(n, k * k + 3, h, w, seed=9, scale=2.0)
    got = kpn.inv_iter(cuda(x_hi), cuda(pred), cuda(x_lo), cuda(prev) if use_prev else None, cuda(fused), k)
    ref = bridge.kpn_inv_iter(x_hi, pred, x_lo, prev if use_prev else None, fused, k, use_prev)
    assert np.allclose(got.cpu().numpy(), ref, rtol=RTOL, atol=ATOL)


def test_pool_and_reproject_match_oracle():
    x = rnd(2, 4, 33, 26, seed=10)
    assert np.allclose(kpn.avg_pool2(cuda(x)).cpu().numpy(), bridge.avg_pool2(x), rtol=RTOL, atol=ATOL)
    prev = rnd(2, 4, 24, 28, seed=11)
    uv = np.random.default_rng(12).uniform(-0.1, 1.1, (2, 2, 24, 28)).astype(np.float32)
    assert np.allclose(kpn.reproject(cuda(prev), cuda(uv)).cpu().numpy(), bridge.grid_sample(prev, uv),
                       rtol=RTOL, atol=ATOL)


def test_three_scale_reconstruction_matches_oracle():
    n, h, w, k = 1, 64, 48, 5
    x0 = rnd(n, 4, h, w, seed=13)
    l0, l1, l2 = rnd(n, k * k + 3, h, w, seed=14), rnd(n, k * k + 3, h // 2, w // 2, seed=15), rnd(n, k * k, h // 4, w // 4, seed=16)
    lprev, prev = rnd(n, k * k, h, w, seed=17), rnd(n, 4, h, w, seed=18)
    uv = np.random.default_rng(19).uniform(0.0, 1.0, (n, 2, h, w)).astype(np.float32)
    got = kpn.inv_iter_denoise(cuda(x0), cuda(l0), cuda(l1), cuda(l2), cuda(lprev), cuda(prev), cuda(uv)).cpu().numpy()
    x1 = bridge.avg_pool2(x0)
    x2 = bridge.avg_pool2(x1)
    r0 = bridge.kpn_apply(bridge.grid_sample(prev, uv), lprev, k, softmax=True)
    r1 = bridge.avg_pool2(r0)
    kp2 = bridge.kpn_apply(x2, l2, k, softmax=True)
    kp1 = bridge.kpn_inv_iter(x1, kp2, x2, r1, l1, k, True)
    ref = bridge.kpn_inv_iter(x0, kp1, x1, r0, l0, k, True)
    assert np.allclose(got, ref, rtol=1e-4, atol=1e-5)
