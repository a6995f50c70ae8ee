"""CPU oracle of the learned denoiser's network operations (test infrastructure only).

Restates, in float64 numpy, what the CUDA kernels of cloudrendering_b200/csrc/vpt_unet.cu compute:
3x3 convolutions (stride 1, zero padding 1) on NHWC tensors with weights [cout][9][cin]
(tap = (dy + 1) * 3 + (dx + 1)), their input and weight gradients, 2x2 average pooling, nearest
upsampling + concatenation, the encoder gradient combine, the per-pixel 5x5 kernel head with the
relative-MSE loss and its logit gradient, and Adam (Kingma & Ba 2015, Algorithm 1).

The reference (chrismile/CloudRendering) has no training code: its learned denoiser is a TorchScript
forward (src/Denoiser/PyTorchDenoiser.cpp:637-800) and the kernel application of
modules/kpn_module/src/Kernel.cu:38-135 (softmax over the taps, taps outside the image skipped),
which kpn_head follows.  The convolution semantics are pinned to torch.nn.functional.conv2d and the
gradients to torch.autograd in float64 (tests/test_unet_cpu.py).

Inputs the GPU reads as bf16 are rounded to bf16 first (bf16()), so the oracle sees the same values.
"""
from __future__ import annotations

import numpy as np


def bf16(a) -> np.ndarray:
    """Round float32 values to bfloat16 (round to nearest even), returned as float32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).copy()
    nan = np.isnan(a)
    out[nan] = np.nan
    return out


def _shift(x: np.ndarray, dy: int, dx: int) -> np.ndarray:
    """x[n, y + dy, x + dx, c] with zeros outside the image."""
    n, h, w, c = x.shape
    out = np.zeros_like(x)
    ys, ye = max(0, -dy), min(h, h - dy)
    xs, xe = max(0, -dx), min(w, w - dx)
    if ys < ye and xs < xe:
        out[:, ys:ye, xs:xe, :] = x[:, ys + dy:ye + dy, xs + dx:xe + dx, :]
    return out


def conv3x3(x, w, bias=None, relu=False, mask=None) -> np.ndarray:
    """y[p][co] = act(bias[co] + sum_{t,ci} x[p + off(t)][ci] * w[co][t][ci]); x [n,h,w,cin], w [cout,9,cin].
    mask (same shape as y): y *= (mask > 0)."""
    x = np.asarray(x, np.float64)
    w = np.asarray(w, np.float64)
    n, h, wd, cin = x.shape
    cout = w.shape[0]
    y = np.zeros((n, h, wd, cout))
    for t in range(9):
        y += _shift(x, t // 3 - 1, t % 3 - 1) @ w[:, t, :].T
    if bias is not None:
        y += np.asarray(bias, np.float64)
    if relu:
        y = np.maximum(y, 0.0)
    if mask is not None:
        y = np.where(np.asarray(mask) > 0, y, 0.0)
    return y


def rotate_weights(w) -> np.ndarray:
    """wrot[ci][t][co] = w[co][8 - t][ci]."""
    w = np.asarray(w)
    return np.ascontiguousarray(w[:, ::-1, :].transpose(2, 1, 0))


def conv3x3_input_grad(dy, w, mask=None) -> np.ndarray:
    """dx[p][ci] = sum_{t,co} dy[p - off(t)][co] * w[co][t][ci], optionally times (mask > 0)."""
    return conv3x3(dy, rotate_weights(w), mask=mask)


def conv3x3_weight_grad(x, dy) -> np.ndarray:
    """dw[co][t][ci] = sum_p dy[p][co] * x[p + off(t)][ci]."""
    x = np.asarray(x, np.float64)
    dy = np.asarray(dy, np.float64)
    cin, cout = x.shape[-1], dy.shape[-1]
    d2 = dy.reshape(-1, cout)
    dw = np.zeros((cout, 9, cin))
    for t in range(9):
        dw[:, t, :] = d2.T @ _shift(x, t // 3 - 1, t % 3 - 1).reshape(-1, cin)
    return dw


def bias_grad(dy) -> np.ndarray:
    dy = np.asarray(dy, np.float64)
    return dy.reshape(-1, dy.shape[-1]).sum(axis=0)


def pool2(x) -> np.ndarray:
    x = np.asarray(x, np.float64)
    n, h, w, c = x.shape
    return x.reshape(n, h // 2, 2, w // 2, 2, c).mean(axis=(2, 4))


def upcat(lo, skip) -> np.ndarray:
    lo = np.asarray(lo, np.float64)
    up = lo.repeat(2, axis=1).repeat(2, axis=2)
    return np.concatenate([up, np.asarray(skip, np.float64)], axis=-1)


def upcat_grad_lo(d, lo) -> np.ndarray:
    """Gradient at the coarse ReLU output lo: (lo > 0) * 2x2 sum of d[..., :ca]."""
    lo = np.asarray(lo)
    n, h2, w2, ca = lo.shape
    s = np.asarray(d, np.float64)[..., :ca].reshape(n, h2, 2, w2, 2, ca).sum(axis=(2, 4))
    return np.where(lo > 0, s, 0.0)


def encoder_grad(d_cat, cat_off, d_pool, e) -> np.ndarray:
    """(e > 0) * (d_cat[..., cat_off:cat_off + c] + upsampled d_pool / 4)."""
    e = np.asarray(e)
    c = e.shape[-1]
    acc = np.zeros(e.shape)
    if d_cat is not None:
        acc += np.asarray(d_cat, np.float64)[..., cat_off:cat_off + c]
    if d_pool is not None:
        acc += 0.25 * np.asarray(d_pool, np.float64).repeat(2, axis=1).repeat(2, axis=2)
    return np.where(e > 0, acc, 0.0)


def pack_input(radiance, albedo=None, normal=None, depth=None, transmittance=None, noise_level=None,
               second_moment=None) -> np.ndarray:
    """Network input [n,h,w,16]: log1p(max(radiance, 0)) 3, albedo 3, normal 3, depth 1,
    transmittance 1, noise level (per image) 1, log1p(sqrt(max(0, m2 - mean^2)) * noise level) 3,
    zero 1 (planes [n][c][h][w])."""
    r = np.asarray(radiance, np.float32)
    n, _, h, w = r.shape
    out = np.zeros((n, h, w, 16), np.float32)
    out[..., 0:3] = np.log1p(np.maximum(r, 0)).transpose(0, 2, 3, 1)
    if albedo is not None:
        out[..., 3:6] = np.asarray(albedo, np.float32).transpose(0, 2, 3, 1)
    if normal is not None:
        out[..., 6:9] = np.asarray(normal, np.float32).transpose(0, 2, 3, 1)
    if depth is not None:
        out[..., 9] = np.asarray(depth, np.float32)
    if transmittance is not None:
        out[..., 10] = np.asarray(transmittance, np.float32)
    if noise_level is not None:
        nl = np.asarray(noise_level, np.float32)
        out[..., 11] = nl[:, None, None]
        if second_moment is not None:
            m2 = np.asarray(second_moment, np.float32)
            se = np.sqrt(np.maximum(0, m2 - r * r)) * nl[:, None, None, None]
            out[..., 12:15] = np.log1p(se).transpose(0, 2, 3, 1)
    return out


def kpn_head(logits, x, target=None, eps=1e-2, ks=5):
    """Softmax over the ks*ks logits of each pixel (channels 0..ks*ks-1 of logits [n,h,w,hc]), the
    ks x ks kernel applied to x [n,3,h,w] with taps outside the image skipped; with a target, the
    relative MSE loss sum (d - t)^2 / (t^2 + eps) / count and its gradient with respect to the
    logits.  Returns (d, loss, dlogits)."""
    taps, rad = ks * ks, ks // 2
    lg = np.asarray(logits, np.float64)[..., :taps]
    x = np.asarray(x, np.float64)
    n, _, h, w = x.shape
    s = np.exp(lg - lg.max(axis=-1, keepdims=True))
    s /= s.sum(axis=-1, keepdims=True)
    xs = []  # x at each tap, [n,3,h,w], zero outside
    for j in range(taps):
        dy, dx = j // ks - rad, j % ks - rad
        xs.append(_shift(x.transpose(0, 2, 3, 1), dy, dx).transpose(0, 3, 1, 2))
    xs = np.stack(xs, axis=-1)  # [n,3,h,w,taps]
    d = (xs * s[:, None, :, :, :]).sum(axis=-1)
    if target is None:
        return d, None, None
    t = np.asarray(target, np.float64)
    count = d.size
    den = t * t + eps
    loss = float(((d - t) ** 2 / den).sum() / count)
    g = 2.0 * (d - t) / den / count  # [n,3,h,w]
    gx = (g[..., None] * xs).sum(axis=1)  # [n,h,w,taps]
    gd = (g * d).sum(axis=1)[..., None]
    dl = np.zeros(np.asarray(logits).shape)
    dl[..., :taps] = s * (gx - gd)
    return d, loss, dl


def adam(param, m1, m2, grad, step, lr=1e-4, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam step; returns (param, m1, m2)."""
    m1 = beta1 * m1 + (1 - beta1) * grad
    m2 = beta2 * m2 + (1 - beta2) * grad * grad
    mhat = m1 / (1 - beta1 ** step)
    vhat = m2 / (1 - beta2 ** step)
    return param - lr * mhat / (np.sqrt(vhat) + eps), m1, m2


# ---------------------------------------------------------------------------------------------
# the whole network (cloudrendering_b200/learned_denoiser.py: KpnUNet.forward / backward)
# ---------------------------------------------------------------------------------------------
def layer_table(widths, head_channels=32, coarse_heads=()):
    """coarse_heads: head channel counts of the level 1 and 2 kernel heads (multi-scale), or ()."""
    w = list(widths)
    t = []
    for l in range(4):
        t.append((f"enc{l}a", 16 if l == 0 else w[l - 1], w[l]))
        t.append((f"enc{l}b", w[l], w[l]))
    t.append(("mida", w[3], w[4]))
    t.append(("midb", w[4], w[4]))
    for l in (3, 2, 1, 0):
        t.append((f"dec{l}a", w[l + 1] + w[l], w[l]))
        t.append((f"dec{l}b", w[l], w[l]))
    t.append(("head", w[0], head_channels))
    for l, hc in enumerate(coarse_heads, start=1):
        t.append((f"head{l}", w[l], hc))
    return t


def split_params(flat, widths, head_channels=32, coarse_heads=()):
    """Flat parameter vector -> {name: (w [cout][9][cin], b [cout])} (weights then bias per layer)."""
    out, off = {}, 0
    for name, cin, cout in layer_table(widths, head_channels, coarse_heads):
        w = np.asarray(flat[off:off + cout * 9 * cin]).reshape(cout, 9, cin)
        off += cout * 9 * cin
        out[name] = (w, np.asarray(flat[off:off + cout]))
        off += cout
    return out


def head_channels_for(ks, blend):
    return (ks * ks + (1 if blend else 0) + 15) // 16 * 16


def network_loss_and_grad(flat, widths, x0, radiance, target, round_bf16=True, eps=1e-2, ks=5, coarse_ks=()):
    """Forward, relative-MSE loss of the kernel head and the gradient with respect to every
    parameter (flat, same layout).  With round_bf16 the weights, activations and backward
    gradients are rounded to bf16 where the GPU stores them in bf16; without, all float64."""
    rnd = (lambda a: bf16(np.asarray(a, np.float32)).astype(np.float64)) if round_bf16 else (lambda a: a)
    multi = len(coarse_ks) > 0
    hc = head_channels_for(ks, multi)
    coarse_hc = tuple(head_channels_for(k, l < len(coarse_ks)) for l, k in enumerate(coarse_ks, start=1))
    P = split_params(flat, widths, hc, coarse_hc)
    Wt = {k: rnd(v[0]) for k, v in P.items()}
    Bs = {k: np.asarray(v[1], np.float64) for k, v in P.items()}
    A = {}
    cur = rnd(x0)
    for l in range(4):
        A[f"in{l}"] = cur
        A[f"enc{l}a"] = rnd(conv3x3(cur, Wt[f"enc{l}a"], Bs[f"enc{l}a"], relu=True))
        A[f"enc{l}b"] = rnd(conv3x3(A[f"enc{l}a"], Wt[f"enc{l}b"], Bs[f"enc{l}b"], relu=True))
        cur = rnd(pool2(A[f"enc{l}b"]))
    A["in4"] = cur
    A["mida"] = rnd(conv3x3(cur, Wt["mida"], Bs["mida"], relu=True))
    cur = A["midb"] = rnd(conv3x3(A["mida"], Wt["midb"], Bs["midb"], relu=True))
    for l in (3, 2, 1, 0):
        A[f"cat{l}"] = upcat(cur, A[f"enc{l}b"])
        A[f"dec{l}a"] = rnd(conv3x3(A[f"cat{l}"], Wt[f"dec{l}a"], Bs[f"dec{l}a"], relu=True))
        cur = A[f"dec{l}b"] = rnd(conv3x3(A[f"dec{l}a"], Wt[f"dec{l}b"], Bs[f"dec{l}b"], relu=True))
    f32 = (lambda a: a.astype(np.float32).astype(np.float64)) if round_bf16 else (lambda a: a)
    logits = f32(conv3x3(cur, Wt["head"], Bs["head"]))
    if multi:
        lgs = [logits] + [f32(conv3x3(A[f"dec{l}b"], Wt[f"head{l}"], Bs[f"head{l}"]))
                          for l in range(1, len(coarse_ks) + 1)]
        loss, dls, d = multiscale_loss_and_grad(lgs, radiance, target, (ks,) + tuple(coarse_ks), eps)
        dl = dls[0]
    else:
        d, loss, dl = kpn_head(logits, radiance, target, eps, ks)
    G = {}

    def grads(name, x, dy):
        G[name] = (conv3x3_weight_grad(x, dy), bias_grad(dy))

    g = rnd(dl)
    grads("head", A["dec0b"], g)
    g = rnd(conv3x3_input_grad(g, Wt["head"], mask=A["dec0b"]))
    dcat = {}
    for l in (0, 1, 2, 3):
        grads(f"dec{l}b", A[f"dec{l}a"], g)
        ga = rnd(conv3x3_input_grad(g, Wt[f"dec{l}b"], mask=A[f"dec{l}a"]))
        grads(f"dec{l}a", A[f"cat{l}"], ga)
        dcat[l] = rnd(conv3x3_input_grad(ga, Wt[f"dec{l}a"]))
        lo = A["midb"] if l == 3 else A[f"dec{l + 1}b"]
        g = rnd(upcat_grad_lo(dcat[l], lo))
        if multi and l + 1 <= len(coarse_ks):
            hl = f"head{l + 1}"
            dlh = rnd(dls[l + 1])
            grads(hl, A[f"dec{l + 1}b"], dlh)
            g = rnd(g + rnd(conv3x3_input_grad(dlh, Wt[hl], mask=A[f"dec{l + 1}b"])))
    grads("midb", A["mida"], g)
    ga = rnd(conv3x3_input_grad(g, Wt["midb"], mask=A["mida"]))
    grads("mida", A["in4"], ga)
    dpool = rnd(conv3x3_input_grad(ga, Wt["mida"]))
    w = list(widths)
    for l in (3, 2, 1, 0):
        ge = rnd(encoder_grad(dcat[l], w[l + 1], dpool, A[f"enc{l}b"]))
        grads(f"enc{l}b", A[f"enc{l}a"], ge)
        ga = rnd(conv3x3_input_grad(ge, Wt[f"enc{l}b"], mask=A[f"enc{l}a"]))
        grads(f"enc{l}a", A[f"in{l}"], ga)
        if l > 0:
            dpool = rnd(conv3x3_input_grad(ga, Wt[f"enc{l}a"]))
    flat_g = []
    for name, _, _ in layer_table(widths, hc, coarse_hc):
        flat_g += [G[name][0].reshape(-1), G[name][1]]
    return loss, np.concatenate(flat_g), logits, d


# ---------------------------------------------------------------------------------------------
# multi-scale reconstruction (cloudrendering_b200/csrc/vpt_unet.cu: kpn_combine_kernel,
# kpn_level_grad_kernel)
# ---------------------------------------------------------------------------------------------
def pool2_planar(x):
    x = np.asarray(x, np.float64)
    n, c, h, w = x.shape
    return x.reshape(n, c, h // 2, 2, w // 2, 2).mean(axis=(3, 5))


def up2_planar(x):
    return np.asarray(x, np.float64).repeat(2, axis=2).repeat(2, axis=3)


def _sigmoid(v):
    return 1.0 / (1.0 + np.exp(-v))


def multiscale_reconstruct(logits, x0, ks):
    """logits: per level l (l = 0 full resolution) NHWC [n, h_l, w_l, hc_l]; ks: kernel size per level.
    Levels below the coarsest carry a blend logit at channel ks_l^2.  Returns (c0, per-level d, c)."""
    L = len(logits)
    xs = [np.asarray(x0, np.float64)]
    for _ in range(L - 1):
        xs.append(pool2_planar(xs[-1]))
    ds = [kpn_head(logits[l], xs[l], ks=ks[l])[0] for l in range(L)]
    cs = [None] * L
    cs[L - 1] = ds[L - 1]
    for l in range(L - 2, -1, -1):
        a = _sigmoid(np.asarray(logits[l], np.float64)[..., ks[l] * ks[l]])[:, None, :, :]
        cs[l] = ds[l] + a * (up2_planar(cs[l + 1]) - up2_planar(pool2_planar(ds[l])))
    return cs[0], xs, ds, cs


def multiscale_loss_and_grad(logits, x0, target, ks, eps=1e-2):
    """Relative-MSE loss of the reconstruction and its gradient with respect to every level's logits."""
    L = len(logits)
    c0, xs, ds, cs = multiscale_reconstruct(logits, x0, ks)
    t = np.asarray(target, np.float64)
    count = c0.size
    loss = float(((c0 - t) ** 2 / (t * t + eps)).sum() / count)
    g = 2.0 * (c0 - t) / (t * t + eps) / count
    grads = [None] * L
    for l in range(L):
        lg = np.asarray(logits[l], np.float64)
        taps = ks[l] * ks[l]
        if l < L - 1:
            a = _sigmoid(lg[..., taps])[:, None, :, :]
            ag = a * g
            s = up2_planar(pool2_planar(ag) * 4.0)  # family sums of a g, on each child
            gd = g - 0.25 * s
            diff = up2_planar(cs[l + 1]) - up2_planar(pool2_planar(ds[l]))
            dalpha = (g * diff).sum(axis=1) * (a[:, 0] * (1 - a[:, 0]))
            g_next = pool2_planar(ag) * 4.0
        else:
            gd, dalpha, g_next = g, None, None
        # kernel application backward (kpn_head's formula with an upstream gradient)
        taps_lg = lg[..., :taps]
        sm = np.exp(taps_lg - taps_lg.max(axis=-1, keepdims=True))
        sm /= sm.sum(axis=-1, keepdims=True)
        rad = ks[l] // 2
        xt = xs[l].transpose(0, 2, 3, 1)
        gx = np.zeros(taps_lg.shape)
        for j in range(taps):
            xs_j = _shift(xt, j // ks[l] - rad, j % ks[l] - rad)  # [n,h,w,3]
            gx[..., j] = (gd.transpose(0, 2, 3, 1) * xs_j).sum(axis=-1)
        gdd = (gd * ds[l]).sum(axis=1)[..., None]
        dl = np.zeros(lg.shape)
        dl[..., :taps] = sm * (gx - gdd)
        if dalpha is not None:
            dl[..., taps] = dalpha
        grads[l] = dl
        g = g_next
    return loss, grads, c0
