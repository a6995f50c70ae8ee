"""Pins the learned denoiser's CPU oracle (oracle/unet_oracle.py) to torch on the CPU in float64:
convolution semantics to torch.nn.functional.conv2d (weights [cout][9][cin] <-> [cout][cin][3][3]),
every backward formula to torch.autograd, Adam to torch.optim.Adam, pooling / upsampling to
torch's avg_pool2d / interpolate(nearest).  The GPU kernels are then compared with this oracle
(tests/test_gpu_unet_kernels.py)."""
import numpy as np
import torch
import torch.nn.functional as F

from oracle import unet_oracle as uo


def t64(a, grad=False):
    return torch.tensor(np.asarray(a, np.float64), requires_grad=grad)


def to_torch_w(w):  # [cout][9][cin] -> [cout][cin][3][3]
    cout, _, cin = w.shape
    return w.reshape(cout, 3, 3, cin).transpose(0, 3, 1, 2)


def test_bf16_rounding():
    a = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5e-3, 3.3e38, 1e-40], np.float32)
    assert np.array_equal(uo.bf16(a), torch.tensor(a).to(torch.bfloat16).float().numpy())
    r = np.random.default_rng(0).standard_normal(100000).astype(np.float32) * 1e3
    assert np.array_equal(uo.bf16(r), torch.tensor(r).to(torch.bfloat16).float().numpy())


def test_conv_and_gradients_match_torch():
    g = np.random.default_rng(1)
    n, h, w, cin, cout = 2, 7, 9, 16, 32
    x = g.standard_normal((n, h, w, cin))
    wt = g.standard_normal((cout, 9, cin)) * 0.1
    b = g.standard_normal(cout) * 0.1
    tx, tw, tb = t64(x.transpose(0, 3, 1, 2), True), t64(to_torch_w(wt), True), t64(b, True)
    ty = F.relu(F.conv2d(tx, tw, tb, padding=1))
    y = uo.conv3x3(x, wt, bias=b, relu=True)
    assert np.allclose(y, ty.detach().numpy().transpose(0, 2, 3, 1), rtol=1e-12, atol=1e-12)
    dy = g.standard_normal(y.shape)
    ty.backward(t64(dy.transpose(0, 3, 1, 2)))
    dpre = np.where(y > 0, dy, 0.0)  # gradient at the pre-activation
    assert np.allclose(uo.conv3x3_input_grad(dpre, wt), tx.grad.numpy().transpose(0, 2, 3, 1), atol=1e-12)
    assert np.allclose(to_torch_w(uo.conv3x3_weight_grad(x, dpre)), tw.grad.numpy(), atol=1e-10)
    assert np.allclose(uo.bias_grad(dpre), tb.grad.numpy(), atol=1e-12)


def test_pool_upcat_encoder_grad_match_torch():
    g = np.random.default_rng(2)
    n, h, w, ca, cs = 2, 6, 8, 8, 16
    e = g.standard_normal((n, h, w, cs))
    lo = np.maximum(g.standard_normal((n, h // 2, w // 2, ca)), 0)
    te, tlo = t64(e.transpose(0, 3, 1, 2), True), t64(lo.transpose(0, 3, 1, 2), True)
    tp = F.avg_pool2d(F.relu(te), 2)
    tcat = torch.cat([F.interpolate(tlo, scale_factor=2, mode="nearest"), F.relu(te)], dim=1)
    e_relu = np.maximum(e, 0)
    assert np.allclose(uo.pool2(e_relu), tp.detach().numpy().transpose(0, 2, 3, 1), atol=1e-14)
    assert np.allclose(uo.upcat(lo, e_relu), tcat.detach().numpy().transpose(0, 2, 3, 1), atol=0)
    d_cat = g.standard_normal(tcat.shape)
    d_pool = g.standard_normal(tp.shape)
    (tcat * t64(d_cat)).sum().add((tp * t64(d_pool)).sum()).backward()
    d_cat_nhwc, d_pool_nhwc = d_cat.transpose(0, 2, 3, 1), d_pool.transpose(0, 2, 3, 1)
    got_e = uo.encoder_grad(d_cat_nhwc, ca, d_pool_nhwc, e_relu)
    assert np.allclose(got_e, te.grad.numpy().transpose(0, 2, 3, 1), atol=1e-12)
    # the coarse input's gradient (masked by its own ReLU output, as the coarse level's conv output)
    got_lo = uo.upcat_grad_lo(d_cat_nhwc, lo)
    assert np.allclose(got_lo, np.where(lo > 0, tlo.grad.numpy().transpose(0, 2, 3, 1), 0), atol=1e-12)


def test_kpn_head_loss_gradient_matches_autograd():
    g = np.random.default_rng(3)
    n, h, w = 2, 7, 6
    logits = g.standard_normal((n, h, w, 32)) * 2
    x = g.exponential(1.0, (n, 3, h, w))
    t = g.exponential(1.0, (n, 3, h, w))
    d, loss, dl = uo.kpn_head(logits, x, t)
    tl = t64(logits[..., :25], True)
    s = torch.softmax(tl, dim=-1)
    tx = t64(x)
    xp = F.pad(tx, (2, 2, 2, 2))
    out = torch.zeros_like(tx)
    for j in range(25):
        dy, dx = j // 5, j % 5
        out = out + s[..., j][:, None] * xp[:, :, dy:dy + h, dx:dx + w]
    tt = t64(t)
    tloss = ((out - tt) ** 2 / (tt * tt + 1e-2)).sum() / out.numel()
    tloss.backward()
    assert np.allclose(d, out.detach().numpy(), rtol=1e-12)
    assert abs(loss - tloss.item()) <= 1e-12 * abs(loss)
    assert np.allclose(dl[..., :25], tl.grad.numpy(), atol=1e-14)
    assert np.all(dl[..., 25:] == 0)
    # other kernel sizes: finite differences of the oracle's own loss
    for ks in (3, 7):
        lg = g.standard_normal((1, 5, 6, 64))
        xx = g.exponential(1.0, (1, 3, 5, 6))
        tt2 = g.exponential(1.0, (1, 3, 5, 6))
        _, l0, dl2 = uo.kpn_head(lg, xx, tt2, ks=ks)
        for idx in [(0, 2, 3, 0), (0, 4, 5, ks * ks - 1), (0, 0, 0, ks * ks // 2)]:
            lp, lm = lg.copy(), lg.copy()
            lp[idx] += 1e-6
            lm[idx] -= 1e-6
            fd = (uo.kpn_head(lp, xx, tt2, ks=ks)[1] - uo.kpn_head(lm, xx, tt2, ks=ks)[1]) / 2e-6
            assert abs(fd - dl2[idx]) <= 1e-6 * (abs(fd) + 1e-6)
        assert np.all(dl2[..., ks * ks:] == 0)


def test_adam_matches_torch():
    g = np.random.default_rng(4)
    p0 = g.standard_normal(50)
    tp = torch.nn.Parameter(t64(p0))
    opt = torch.optim.Adam([tp], lr=1e-3, betas=(0.9, 0.999), eps=1e-8)
    p, m1, m2 = p0.copy(), np.zeros(50), np.zeros(50)
    for step in range(1, 6):
        gr = g.standard_normal(50)
        tp.grad = t64(gr)
        opt.step()
        p, m1, m2 = uo.adam(p, m1, m2, gr, step, lr=1e-3)
    assert np.allclose(p, tp.detach().numpy(), rtol=1e-12, atol=1e-14)


def test_oracle_network_gradient_matches_finite_differences():
    """The oracle's whole-network backward (float64, no rounding) against central differences of
    its own forward loss."""
    widths = (16, 16, 16, 16, 32)
    g = np.random.default_rng(5)
    table = uo.layer_table(widths)
    flat = []
    for name, cin, cout in table:
        flat += [g.standard_normal(cout * 9 * cin) * np.sqrt(2.0 / (9 * cin)) * (0.3 if name == "head" else 1.0),
                 g.standard_normal(cout) * 0.05]
    flat = np.concatenate(flat)
    n, h, w = 1, 16, 16
    x0 = np.zeros((n, h, w, 16))
    x0[..., :12] = g.standard_normal((n, h, w, 12))
    rad = g.exponential(1.0, (n, 3, h, w))
    tgt = g.exponential(1.0, (n, 3, h, w))
    loss, grad, _, _ = uo.network_loss_and_grad(flat, widths, x0, rad, tgt, round_bf16=False)
    # indices spread over all layers (weights and biases)
    idx = np.unique(g.integers(0, flat.size, 40))
    hstep = 1e-6
    for i in idx:
        fp, fm = flat.copy(), flat.copy()
        fp[i] += hstep
        fm[i] -= hstep
        lp = uo.network_loss_and_grad(fp, widths, x0, rad, tgt, round_bf16=False)[0]
        lm = uo.network_loss_and_grad(fm, widths, x0, rad, tgt, round_bf16=False)[0]
        fd = (lp - lm) / (2 * hstep)
        assert abs(fd - grad[i]) <= 1e-5 * (abs(fd) + np.abs(grad).max() * 1e-3), (i, fd, grad[i])


def test_multiscale_reconstruction_gradient_matches_autograd():
    g = np.random.default_rng(6)
    n, h, w = 2, 8, 12
    ks = (5, 3, 3)
    hcs = (32, 16, 16)
    logits = [g.standard_normal((n, h >> l, w >> l, hcs[l])) for l in range(3)]
    x0 = g.exponential(1.0, (n, 3, h, w))
    t = g.exponential(1.0, (n, 3, h, w))
    loss, grads, c0 = uo.multiscale_loss_and_grad(logits, x0, t, ks)

    tl = [t64(lg, True) for lg in logits]
    xs = [t64(x0)]
    for _ in range(2):
        xs.append(F.avg_pool2d(xs[-1], 2))

    def apply(x, lg, k):
        s = torch.softmax(lg[..., :k * k], dim=-1)
        hh, ww = x.shape[2], x.shape[3]
        xp = F.pad(x, (k // 2,) * 4)
        out = torch.zeros_like(x)
        for j in range(k * k):
            out = out + s[..., j][:, None] * xp[:, :, j // k:j // k + hh, j % k:j % k + ww]
        return out

    ds = [apply(xs[l], tl[l], ks[l]) for l in range(3)]
    c = ds[2]
    for l in (1, 0):
        a = torch.sigmoid(tl[l][..., ks[l] * ks[l]])[:, None]
        up = lambda v: F.interpolate(v, scale_factor=2, mode="nearest")
        c = ds[l] + a * (up(c) - up(F.avg_pool2d(ds[l], 2)))
    tt = t64(t)
    tloss = ((c - tt) ** 2 / (tt * tt + 1e-2)).sum() / c.numel()
    tloss.backward()
    assert np.allclose(c0, c.detach().numpy(), rtol=1e-12, atol=1e-14)
    assert abs(loss - tloss.item()) <= 1e-12 * loss
    for l in range(3):
        used = ks[l] * ks[l] + (1 if l < 2 else 0)
        assert np.allclose(grads[l][..., :used], tl[l].grad.numpy()[..., :used], atol=1e-14), l
        assert np.all(grads[l][..., used:] == 0)


def test_oracle_multiscale_network_gradient_matches_finite_differences():
    widths = (16, 16, 16, 16, 32)
    coarse_ks = (3, 3)
    g = np.random.default_rng(8)
    hc0 = uo.head_channels_for(5, True)
    chc = (uo.head_channels_for(3, True), uo.head_channels_for(3, False))
    flat = []
    for name, cin, cout in uo.layer_table(widths, hc0, chc):
        flat += [g.standard_normal(cout * 9 * cin) * np.sqrt(2.0 / (9 * cin)) * (0.3 if "head" in name else 1.0),
                 g.standard_normal(cout) * 0.05]
    flat = np.concatenate(flat)
    n, h, w = 1, 16, 16
    x0 = np.zeros((n, h, w, 16))
    x0[..., :12] = g.standard_normal((n, h, w, 12))
    rad = g.exponential(1.0, (n, 3, h, w))
    tgt = g.exponential(1.0, (n, 3, h, w))
    kw = dict(round_bf16=False, ks=5, coarse_ks=coarse_ks)
    loss, grad, _, _ = uo.network_loss_and_grad(flat, widths, x0, rad, tgt, **kw)
    names = [n_ for n_, _, _ in uo.layer_table(widths, hc0, chc)]
    # indices in the coarse heads and the decoder levels they feed, plus random ones
    offs, off = {}, 0
    for name, cin, cout in uo.layer_table(widths, hc0, chc):
        offs[name] = off
        off += cout * 9 * cin + cout
    idx = [offs["head1"] + 5, offs["head2"] + 17, offs["dec1b"] + 3, offs["dec2b"] + 40, offs["head"] + 9]
    idx += list(g.integers(0, flat.size, 15))
    for i in idx:
        fp, fm = flat.copy(), flat.copy()
        fp[i] += 1e-6
        fm[i] -= 1e-6
        fd = (uo.network_loss_and_grad(fp, widths, x0, rad, tgt, **kw)[0] -
              uo.network_loss_and_grad(fm, widths, x0, rad, tgt, **kw)[0]) / 2e-6
        assert abs(fd - grad[i]) <= 1e-5 * (abs(fd) + np.abs(grad).max() * 1e-3), (i, fd, grad[i])
    assert "head2" in names
