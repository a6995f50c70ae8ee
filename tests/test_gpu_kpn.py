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


# ---- against the reference's own extension (modules/kpn_module/src/Kernel.cu and perPixelKernel.cpp,
# compiled unmodified for sm_100a into oracle/_ref/libref_kpn.so) ----
REF_KPN = __import__("os").path.join(__import__("os").path.dirname(__import__("os").path.dirname(
    __import__("os").path.abspath(__file__))), "oracle", "_ref", "libref_kpn.so")


@pytest.fixture(scope="module")
def ref_ops():
    if not __import__("os").path.exists(REF_KPN):
        pytest.skip("the reference's KPN extension was not built (no reference tree where the build ran)")
    torch.ops.load_library(REF_KPN)
    return torch.ops


@pytest.mark.parametrize("k,shape", [(3, (1, 3, 17, 23)), (5, (2, 4, 32, 40)), (5, (1, 4, 9, 7))])
def test_apply_matches_reference_extension(ref_ops, k, shape):
    """perPixelKernelForward on softmaxed weights, as PyTorchDenoiser.cpp:425-431 calls it."""
    n, c, h, w = shape
    img, logits = cuda(rnd(*shape, seed=21)), cuda(rnd(n, k * k, h, w, seed=22, scale=2.0))
    want = ref_ops.per_pixel_kernel.forward(img, torch.softmax(logits, 1), k)
    got = kpn.apply_kernels(img, logits, k)
    torch.cuda.synchronize()
    assert got.shape == want.shape
    assert torch.allclose(got, want, rtol=RTOL, atol=ATOL)


def test_apply_output_size_matches_reference_extension(ref_ops):
    img, logits = cuda(rnd(1, 3, 20, 18, seed=23)), cuda(rnd(1, 9, 16, 22, seed=24))
    want = ref_ops.per_pixel_kernel.forward(img, torch.softmax(logits, 1), 3)
    got = kpn.apply_kernels(img, logits, 3)
    assert got.shape == want.shape == (1, 3, 16, 18)
    assert torch.allclose(got, want, rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("use_prev", [False, True])
@pytest.mark.parametrize("k", [3, 5])
def test_inv_iter_matches_reference_extension(ref_ops, use_prev, k):
    """inv_iter_kernel (PyTorchDenoiser.cpp:174-179): getInvIterBaseCuda, then the per-pixel kernel of
    the softmaxed first k*k channels.  One image: the reference indexes the fused weights of batch b
    with a stride of k*k channels instead of k*k + 3 (Kernel.cu:166-168), which the core corrects."""
    c, h, w = 4, 26, 30
    x_hi, prev = cuda(rnd(1, c, h, w, seed=25)), cuda(rnd(1, c, h, w, seed=26))
    x_lo, pred = cuda(rnd(1, c, h // 2, w // 2, seed=27)), cuda(rnd(1, c, h // 2, w // 2, seed=28))
    fused = cuda(rnd(1, k * k + 3, h, w, seed=29, scale=2.0))
    base = ref_ops.ref_kpn.inv_iter_base(x_hi, pred, x_lo, prev, fused, use_prev, k)
    want = ref_ops.per_pixel_kernel.forward(base, torch.softmax(fused[:, :k * k], 1).contiguous(), k)
    got = kpn.inv_iter(x_hi, pred, x_lo, prev if use_prev else None, fused, k)
    assert torch.allclose(got, want, rtol=RTOL, atol=ATOL)


def test_three_scale_reconstruction_matches_reference_composition(ref_ops):
    """PyTorchDenoiser::denoise with blend inv_iter (PyTorchDenoiser.cpp:411-440), composed from the
    reference's extension and the libtorch operators it calls, against the core's inv_iter_denoise."""
    k, c, h, w = 5, 4, 32, 36
    x0 = cuda(rnd(1, 6, h, w, seed=30))
    l0, l1, l2 = (cuda(rnd(1, k * k + 3, h >> s, w >> s, seed=31 + s, scale=2.0)) for s in range(3))
    l2 = l2[:, :k * k].contiguous()
    lprev = cuda(rnd(1, k * k, h, w, seed=35, scale=2.0))
    prev = cuda(rnd(1, c, h, w, seed=36))
    uv = torch.rand((1, 2, h, w), device="cuda", generator=torch.Generator(device="cuda").manual_seed(37))
    xs0 = x0[:, :4].contiguous()
    xs1 = torch.nn.functional.avg_pool2d(xs0, 2, 2)
    xs2 = torch.nn.functional.avg_pool2d(xs1, 2, 2)
    reproj0 = torch.grid_sampler_2d(prev, uv.permute(0, 2, 3, 1) * 2 - 1, 0, 0, False)
    reproj0 = ref_ops.per_pixel_kernel.forward(reproj0.contiguous(), torch.softmax(lprev, 1), k)
    reproj1 = torch.nn.functional.avg_pool2d(reproj0, 2, 2)

    def inv_iter_ref(x, kp, xl, rp, lw):
        base = ref_ops.ref_kpn.inv_iter_base(x, kp, xl, rp, lw, True, k)
        return ref_ops.per_pixel_kernel.forward(base, torch.softmax(lw[:, :k * k], 1).contiguous(), k)

    kp2 = ref_ops.per_pixel_kernel.forward(xs2, torch.softmax(l2, 1), k)
    kp1 = inv_iter_ref(xs1, kp2, xs2, reproj1, l1)
    want = inv_iter_ref(xs0, kp1, xs1, reproj0, l0)
    got = kpn.inv_iter_denoise(x0, l0, l1, l2, lprev=lprev, prev=prev, reproj_uv=uv)
    assert got.shape == want.shape
    assert torch.allclose(got, want, rtol=1e-4, atol=1e-5)
