"""The learned denoiser's network kernels (csrc/vpt_unet.cu, tcgen05 tensor cores) against the CPU
oracle (oracle/unet_oracle.py, float64 on the same bf16-rounded inputs), through the C ABI.

Tolerances: fp32 outputs of bf16 x bf16 -> fp32 products: |gpu - ref| <= 1e-5 * (|ref| + rms(ref))
(fp32 accumulation over K <= 2592 terms); bf16 outputs: one bf16 rounding, |gpu - ref| <=
2^-8 * |ref| + 1e-6 * rms(ref)."""
import ctypes

import numpy as np
import pytest
import torch

from cloudrendering_b200 import _lib
from oracle import unet_oracle as uo

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    torch.cuda.init()
    return _lib.load()


def dev_bf16(a):
    return torch.from_numpy(uo.bf16(np.asarray(a, np.float32))).to(torch.bfloat16).cuda().contiguous()


def dev_f32(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def host(t):
    return t.float().cpu().numpy().astype(np.float64)


def close_f32(got, ref):
    scale = np.sqrt(np.mean(ref ** 2)) + 1e-30
    err = np.abs(got - ref) / (np.abs(ref) + scale)
    assert err.max() <= 1e-5, f"max scaled error {err.max():.3g}"


def close_bf16(got, ref):
    scale = np.sqrt(np.mean(ref ** 2)) + 1e-30
    ok = np.abs(got - ref) <= 2.0 ** -8 * np.abs(ref) + 1e-6 * scale
    assert ok.mean() == 1.0, f"{(~ok).sum()} of {ok.size} beyond one bf16 rounding; max {np.abs(got - ref).max():.3g}"


def run(lib, name, *args):
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = getattr(lib, name)(*args, ptr(err), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert st == 0, name
    assert int(err.item()) == 0, f"{name}: device error {int(err.item())}"


def rng_data(seed, *shape, scale=1.0):
    return (np.random.default_rng(seed).standard_normal(shape) * scale).astype(np.float32)


CONV_CASES = [
    # n, h, w, cin, cout
    (2, 9, 13, 16, 32),     # ragged pixel count (234)
    (1, 16, 16, 32, 64),
    (1, 8, 8, 288, 128),    # decoder concat width
    (1, 6, 10, 160, 160),
    (1, 6, 10, 128, 288),   # two output-channel tiles (input gradient of a 288-channel concat)
    (3, 5, 7, 96, 96),
]


@pytest.fixture(params=[0, 1, 8], ids=["ksplit_auto", "ksplit_off", "ksplit_8"])
def ksplit(lib, request):
    """K splits of the gather convolution: by grid size (most cases here split), none, and 8 forced
    (more splits than some cases have K stages per split: empty splits contribute zeros)."""
    assert lib.vpt_unet_set_conv_ksplit(request.param) == 0
    yield request.param
    assert lib.vpt_unet_set_conv_ksplit(0) == 0


@pytest.mark.parametrize("case", CONV_CASES)
@pytest.mark.parametrize("epilogue", ["f32", "bias_relu_bf16", "mask_bf16"])
def test_conv_forward(lib, case, epilogue, ksplit):
    n, h, w, cin, cout = case
    x = uo.bf16(rng_data(1, n, h, w, cin))
    wt = uo.bf16(rng_data(2, cout, 9, cin, scale=1.0 / np.sqrt(9 * cin)))
    bias = rng_data(3, cout, scale=0.1)
    mask = uo.bf16(rng_data(4, n, h, w, cout))
    dx, dw = dev_bf16(x), dev_bf16(wt)
    if epilogue == "f32":
        y = torch.empty((n, h, w, cout), dtype=torch.float32, device="cuda")
        run(lib, "vpt_unet_conv3x3", ptr(dx), ptr(dw), None, None, ptr(y), n, h, w, cin, cout, 0, 1)
        close_f32(host(y), uo.conv3x3(x, wt))
    elif epilogue == "bias_relu_bf16":
        y = torch.empty((n, h, w, cout), dtype=torch.bfloat16, device="cuda")
        b = dev_f32(bias)
        run(lib, "vpt_unet_conv3x3", ptr(dx), ptr(dw), ptr(b), None, ptr(y), n, h, w, cin, cout, 1, 0)
        close_bf16(host(y), uo.conv3x3(x, wt, bias=bias, relu=True))
    else:
        y = torch.empty((n, h, w, cout), dtype=torch.bfloat16, device="cuda")
        m = dev_bf16(mask)
        run(lib, "vpt_unet_conv3x3", ptr(dx), ptr(dw), None, ptr(m), ptr(y), n, h, w, cin, cout, 0, 0)
        close_bf16(host(y), uo.conv3x3(x, wt, mask=mask))


@pytest.mark.parametrize("case", CONV_CASES)
def test_conv_input_grad(lib, case, ksplit):
    n, h, w, cin, cout = case
    dy = uo.bf16(rng_data(5, n, h, w, cout))
    wt = uo.bf16(rng_data(6, cout, 9, cin, scale=1.0 / np.sqrt(9 * cout)))
    x = uo.bf16(rng_data(7, n, h, w, cin))  # forward input: ReLU-derivative mask
    d_dy, d_w, d_x = dev_bf16(dy), dev_bf16(wt), dev_bf16(x)
    wrot = torch.empty((cin, 9, cout), dtype=torch.bfloat16, device="cuda")
    st = lib.vpt_unet_rotate_weights(ptr(d_w), ptr(wrot), cin, cout, None)
    assert st == 0
    torch.cuda.synchronize()
    assert np.array_equal(host(wrot), uo.rotate_weights(wt))
    out = torch.empty((n, h, w, cin), dtype=torch.float32, device="cuda")
    run(lib, "vpt_unet_conv3x3", ptr(d_dy), ptr(wrot), None, None, ptr(out), n, h, w, cout, cin, 0, 1)
    close_f32(host(out), uo.conv3x3_input_grad(dy, wt))
    out_b = torch.empty((n, h, w, cin), dtype=torch.bfloat16, device="cuda")
    run(lib, "vpt_unet_conv3x3", ptr(d_dy), ptr(wrot), None, ptr(d_x), ptr(out_b), n, h, w, cout, cin, 0, 0)
    close_bf16(host(out_b), uo.conv3x3_input_grad(dy, wt, mask=x))


STRIP_CASES = [
    # n, h, w, cin, cout: images at least 128 pixels wide take the row-strip kernel
    (1, 5, 130, 32, 32),    # ragged second tile (2 of 128 pixels valid)
    (2, 9, 256, 16, 32),
    (1, 3, 128, 96, 32),
    (1, 4, 200, 32, 176),   # 13x13 kernel head
    (1, 37, 128, 64, 64),   # many rows: several segments per column
    (1, 6, 128, 160, 64),   # input channels in two groups (fp32 partial between the passes)
    (3, 20, 384, 32, 32),   # three columns, several segments each: the input ring wraps across segments
]


@pytest.mark.parametrize("kind", [0, 1], ids=["warp_specialised", "cp_async"])
@pytest.mark.parametrize("case", STRIP_CASES)
def test_strip_conv_forward_and_input_grad(lib, case, kind):
    n, h, w, cin, cout = case
    assert lib.vpt_unet_set_strip_kernel(kind) == 0
    assert lib.vpt_unet_set_conv_path(2) == 0
    x = uo.bf16(rng_data(21, n, h, w, cin))
    wt = uo.bf16(rng_data(22, cout, 9, cin, scale=1.0 / np.sqrt(9 * cin)))
    bias = rng_data(23, cout, scale=0.1)
    dx, dw, b = dev_bf16(x), dev_bf16(wt), dev_f32(bias)
    y = torch.empty((n, h, w, cout), dtype=torch.float32, device="cuda")
    run(lib, "vpt_unet_conv3x3", ptr(dx), ptr(dw), ptr(b), None, ptr(y), n, h, w, cin, cout, 0, 1)
    close_f32(host(y), uo.conv3x3(x, wt, bias=bias))
    yb = torch.empty((n, h, w, cout), dtype=torch.bfloat16, device="cuda")
    run(lib, "vpt_unet_conv3x3", ptr(dx), ptr(dw), ptr(b), None, ptr(yb), n, h, w, cin, cout, 1, 0)
    close_bf16(host(yb), uo.conv3x3(x, wt, bias=bias, relu=True))
    # the gather kernel gives the same result up to the summation order
    assert lib.vpt_unet_set_conv_path(1) == 0
    y2 = torch.empty_like(y)
    run(lib, "vpt_unet_conv3x3", ptr(dx), ptr(dw), ptr(b), None, ptr(y2), n, h, w, cin, cout, 0, 1)
    assert lib.vpt_unet_set_conv_path(2) == 0
    close_f32(host(y2), host(y))
    # input gradient with the ReLU-derivative mask (rotated weights: cout -> cin; 176 input channels
    # of the head's gradient take two channel groups)
    dy = uo.bf16(rng_data(24, n, h, w, cout))
    wrot = torch.empty((cin, 9, cout), dtype=torch.bfloat16, device="cuda")
    assert lib.vpt_unet_rotate_weights(ptr(dw), ptr(wrot), cin, cout, None) == 0
    g = torch.empty((n, h, w, cin), dtype=torch.bfloat16, device="cuda")
    d_dy = dev_bf16(dy)  # kept alive: a temporary's memory may be reused by the next allocation
    run(lib, "vpt_unet_conv3x3", ptr(d_dy), ptr(wrot), None, ptr(dx), ptr(g), n, h, w, cout, cin, 0, 0)
    close_bf16(host(g), uo.conv3x3_input_grad(dy, wt, mask=x))
    assert lib.vpt_unet_set_conv_path(0) == 0
    assert lib.vpt_unet_set_strip_kernel(0) == 0


WGRAD_CASES = [
    # n, h, w, cin, cout, pixels per split (images narrower than 128 pixels: the gather kernel)
    (2, 9, 13, 16, 32, 64),
    (1, 16, 16, 96, 160, 128),
    (1, 8, 8, 288, 128, 64),
    (2, 6, 10, 32, 288, 192),
    (1, 32, 32, 64, 64, 1024),
    # row-strip weight gradient (>= 128 pixels wide): input channels as M (padded to 64 / 128),
    # output channels as M (two chunks), tap groups, several segments per column
    (1, 5, 130, 32, 32, 64),
    (2, 7, 256, 16, 32, 64),
    (1, 4, 128, 96, 32, 64),
    (1, 5, 200, 32, 176, 64),
    (1, 6, 128, 64, 64, 64),
    (1, 4, 128, 160, 64, 64),
    (1, 37, 128, 32, 32, 64),
]


@pytest.mark.parametrize("case", WGRAD_CASES)
def test_conv_weight_grad(lib, case):
    n, h, w, cin, cout, pps = case
    x = uo.bf16(rng_data(8, n, h, w, cin))
    dy = uo.bf16(rng_data(9, n, h, w, cout))
    P = n * h * w
    assert lib.vpt_unet_set_conv_path(2 if w >= 128 else 0) == 0  # the strip kernel on every wide case
    splits = lib.vpt_unet_wgrad_splits(n, h, w, cin, cout, pps)
    assert splits >= 1
    rows = lib.vpt_unet_wgrad_rows(cin)
    assert rows % 128 == 0 and rows >= 9 * cin
    part = torch.full((splits, rows, cout), float("nan"), dtype=torch.float32, device="cuda")
    d_x, d_dy = dev_bf16(x), dev_bf16(dy)
    run(lib, "vpt_unet_conv3x3_wgrad", ptr(d_x), ptr(d_dy), ptr(part), n, h, w, cin, cout, pps)
    bblocks = 7
    bpart = torch.empty((bblocks, cout), dtype=torch.float32, device="cuda")
    assert lib.vpt_unet_bias_grad(ptr(d_dy), ptr(bpart), P, cout, bblocks, None) == 0
    gw = torch.empty((cout, 9, cin), dtype=torch.float32, device="cuda")
    gb = torch.empty((cout,), dtype=torch.float32, device="cuda")
    assert lib.vpt_unet_reduce_grads(ptr(part), splits, cin, cout, ptr(bpart), bblocks, ptr(gw), ptr(gb), None) == 0
    torch.cuda.synchronize()
    assert lib.vpt_unet_set_conv_path(0) == 0
    close_f32(host(gw), uo.conv3x3_weight_grad(x, dy))
    close_f32(host(gb), uo.bias_grad(dy))


def test_pool_upcat_and_gradients(lib):
    n, h, w, ca, cs = 2, 10, 14, 32, 16
    e = uo.bf16(rng_data(10, n, h, w, cs))
    lo = uo.bf16(rng_data(11, n, h // 2, w // 2, ca))
    d_e, d_lo = dev_bf16(e), dev_bf16(lo)
    pooled = torch.empty((n, h // 2, w // 2, cs), dtype=torch.bfloat16, device="cuda")
    assert lib.vpt_unet_pool2(ptr(d_e), ptr(pooled), n, h, w, cs, None) == 0
    cat = torch.empty((n, h, w, ca + cs), dtype=torch.bfloat16, device="cuda")
    assert lib.vpt_unet_upcat(ptr(d_lo), ptr(d_e), ptr(cat), n, h, w, ca, cs, None) == 0
    d_cat = uo.bf16(rng_data(12, n, h, w, ca + cs))
    d_pool = uo.bf16(rng_data(13, n, h // 2, w // 2, cs))
    t_dcat, t_dpool = dev_bf16(d_cat), dev_bf16(d_pool)
    dlo = torch.empty_like(d_lo)
    assert lib.vpt_unet_upcat_grad_lo(ptr(t_dcat), ptr(d_lo), ptr(dlo), n, h, w, ca, cs, None) == 0
    de = torch.empty_like(d_e)
    assert lib.vpt_unet_encoder_grad(ptr(t_dcat), ca + cs, ca, ptr(t_dpool), ptr(d_e), ptr(de), n, h, w, cs,
                                     None) == 0
    torch.cuda.synchronize()
    close_bf16(host(pooled), uo.pool2(e))
    assert np.array_equal(host(cat), uo.upcat(lo, e))
    close_bf16(host(dlo), uo.upcat_grad_lo(d_cat, lo))
    close_bf16(host(de), uo.encoder_grad(d_cat, ca, d_pool, e))


def test_pack_input_and_kpn_head(lib):
    n, h, w = 2, 12, 17
    g = np.random.default_rng(14)
    rad = (g.exponential(1.0, (n, 3, h, w)) * (g.random((n, 3, h, w)) < 0.7)).astype(np.float32)
    alb = g.random((n, 3, h, w)).astype(np.float32)
    nrm = g.standard_normal((n, 3, h, w)).astype(np.float32)
    dep = g.random((n, h, w)).astype(np.float32)
    trn = g.random((n, h, w)).astype(np.float32)
    noise = np.array([1.0, 0.125], np.float32)
    m2 = (rad * rad * (1.0 + g.random((n, 3, h, w)))).astype(np.float32)
    packed = torch.empty((n, h, w, 16), dtype=torch.bfloat16, device="cuda")
    t = [dev_f32(a) for a in (rad, alb, nrm, dep, trn, noise, m2)]
    assert lib.vpt_unet_pack_input(*[ptr(a) for a in t], ptr(packed), n, h, w, None) == 0
    torch.cuda.synchronize()
    ref = uo.pack_input(rad, alb, nrm, dep, trn, noise, m2)
    close_bf16(host(packed), ref.astype(np.float64))


@pytest.mark.parametrize("shape", [(2, 12, 17), (1, 5, 150), (3, 70, 9), (1, 3, 128)],
                         ids=["narrow", "ragged_segments", "tall", "two_segments"])
def test_kpn_head(lib, shape):
    """Kernel application, loss and logit gradient; rows of 64-pixel segments with ragged ends and
    images narrower than one segment."""
    n, h, w = shape
    g = np.random.default_rng(14)
    rad = (g.exponential(1.0, (n, 3, h, w)) * (g.random((n, 3, h, w)) < 0.7)).astype(np.float32)
    target = g.exponential(1.0, (n, 3, h, w)).astype(np.float32)
    d_rad, d_target = dev_f32(rad), dev_f32(target)
    blocks = lib.vpt_unet_head_blocks(n, h, w)
    for ks, hc in ((5, 32), (9, 96), (11, 128), (3, 16), (13, 176), (1, 8), (7, 56), (15, 232)):
        logits = rng_data(15 + ks, n, h, w, hc, scale=2.0)
        out = torch.empty((n, 3, h, w), dtype=torch.float32, device="cuda")
        dl = torch.empty((n, h, w, hc), dtype=torch.bfloat16, device="cuda")
        lp = torch.empty((blocks,), dtype=torch.float32, device="cuda")
        d_logits = dev_f32(logits)
        assert lib.vpt_unet_kpn_head(ptr(d_logits), hc, ks, ptr(d_rad), ptr(d_target), ptr(out), ptr(dl), ptr(lp), n,
                                     h, w, ctypes.c_float(1e-2), None) == 0
        torch.cuda.synchronize()
        d, loss, dlog = uo.kpn_head(logits, rad, target, ks=ks)
        close_f32(host(out), d)
        assert abs(float(lp.double().sum()) - loss) <= 1e-5 * loss
        close_bf16(host(dl), dlog)
        # inference: the image alone
        out2 = torch.full((n, 3, h, w), -1.0, dtype=torch.float32, device="cuda")
        assert lib.vpt_unet_kpn_head(ptr(d_logits), hc, ks, ptr(d_rad), None, ptr(out2), None, None, n, h, w,
                                     ctypes.c_float(1e-2), None) == 0
        torch.cuda.synchronize()
        assert torch.equal(out2, out)


def test_adam(lib):
    count = 10000
    g = np.random.default_rng(16)
    p = g.standard_normal(count).astype(np.float32)
    m1 = (g.standard_normal(count) * 0.01).astype(np.float32)
    m2 = (g.random(count) * 0.01).astype(np.float32)
    gr = g.standard_normal(count).astype(np.float32)
    tp, tm1, tm2, tg = dev_f32(p), dev_f32(m1), dev_f32(m2), dev_f32(gr)
    pb = torch.empty(count, dtype=torch.bfloat16, device="cuda")
    assert lib.vpt_unet_adam(ptr(tp), ptr(pb), ptr(tm1), ptr(tm2), ptr(tg), count, ctypes.c_float(1e-3),
                             ctypes.c_float(0.9), ctypes.c_float(0.999), ctypes.c_float(1e-8), 7, ctypes.c_float(1.0),
                             None) == 0
    torch.cuda.synchronize()
    f32 = lambda v: float(np.float32(v))  # the kernel receives float hyperparameters
    rp, rm1, rm2 = uo.adam(*(a.astype(np.float64) for a in (p, m1, m2, gr)), 7, lr=f32(1e-3), beta1=f32(0.9),
                           beta2=f32(0.999), eps=f32(1e-8))
    # fp32 arithmetic with contracted multiply-adds: a few ulps of the largest term
    for got, ref in ((host(tp), rp), (host(tm1), rm1), (host(tm2), rm2)):
        assert np.all(np.abs(got - ref) <= 1e-6 * np.abs(ref) + 4 * 2.0 ** -23 * np.abs(ref).max())
    assert np.array_equal(host(pb), uo.bf16(host(tp).astype(np.float32)))
