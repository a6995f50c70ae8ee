"""The learned kernel-predicting denoiser (cloudrendering_b200/learned_denoiser.py) on the GPU:

* the whole network's loss and parameter gradient (tcgen05 forward and backward kernels) against
  the CPU oracle's network (oracle/unet_oracle.py, the same bf16 rounding points, float64
  arithmetic), whose own gradient is pinned by finite differences in tests/test_unet_cpu.py;
* training on tracer-generated pairs lowers the relative MSE of held-out noisy renders against
  their many-sample targets: what the trained network gains over the noisy input it starts from;
* the saved model (weights.npz + model_info.json) loads back to the same network.
"""
import json

import numpy as np
import pytest
import torch

from cloudrendering_b200 import learned_denoiser as ld
from cloudrendering_b200 import vpt
from oracle import unet_oracle as uo

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def module():
    vpt.initialize()
    yield
    vpt.cleanup()


def random_flat(widths, seed, head_scale=0.3, hc=32, coarse_hc=()):
    g = np.random.default_rng(seed)
    flat = []
    for name, cin, cout in uo.layer_table(widths, hc, coarse_hc):
        std = np.sqrt(2.0 / (9 * cin)) * (head_scale if name.startswith("head") else 1.0)
        flat += [g.standard_normal(cout * 9 * cin) * std, g.standard_normal(cout) * 0.05]
    return np.concatenate(flat).astype(np.float32)


@pytest.mark.parametrize("coarse", [(), (3, 3)])
def test_network_gradient_matches_oracle(coarse):
    widths = (16, 32, 32, 48, 64)
    net = ld.KpnUNet(widths, kernel_size=5, coarse_kernels=coarse)
    hc = uo.head_channels_for(5, len(coarse) > 0)
    chc = tuple(uo.head_channels_for(k, l < len(coarse)) for l, k in enumerate(coarse, start=1))
    flat = random_flat(widths, 1, hc=hc, coarse_hc=chc)
    net.set_parameters(flat)
    g = np.random.default_rng(2)
    n, h, w = 2, 32, 32
    x0 = np.zeros((n, h, w, 16), np.float32)
    x0[..., :12] = g.standard_normal((n, h, w, 12))
    x0 = uo.bf16(x0)
    rad = g.exponential(1.0, (n, 3, h, w)).astype(np.float32)
    tgt = g.exponential(1.0, (n, 3, h, w)).astype(np.float32)
    d_x0 = torch.from_numpy(x0).to(torch.bfloat16).cuda()
    d_rad, d_tgt = torch.from_numpy(rad).cuda(), torch.from_numpy(tgt).cuda()
    logits = net.forward(d_x0)
    _, loss, dls = net.reconstruct(d_rad, d_tgt)
    net.backward(dls)
    torch.cuda.synchronize()
    net.check_errors()
    ref_loss, ref_grad, ref_logits, _ = uo.network_loss_and_grad(flat.astype(np.float64), widths, x0, rad, tgt,
                                                                 coarse_ks=coarse)
    got_logits = logits.cpu().numpy().astype(np.float64)
    assert np.abs(got_logits - ref_logits).max() <= 2e-2 * np.abs(ref_logits).max()
    assert abs(float(loss) - ref_loss) <= 1e-3 * ref_loss
    got = net.grad.cpu().numpy().astype(np.float64)
    cos = got @ ref_grad / (np.linalg.norm(got) * np.linalg.norm(ref_grad))
    print(f"loss {float(loss):.6g} vs {ref_loss:.6g}; gradient cosine {cos:.6f}")
    assert cos >= 0.999
    for L in net.layers:
        a, b = L["w_off"], L["b_off"] + L["cout"]
        rel = np.linalg.norm(got[a:b] - ref_grad[a:b]) / (np.linalg.norm(ref_grad[a:b]) + 1e-30)
        assert rel <= 5e-2, (L["name"], rel)


def test_training_on_tracer_pairs_beats_the_noisy_input(tmp_path):
    data = ld.TrainingSet(vpt, num_scenes=12, size=64, spp_levels=(1, 4, 16), target_spp=512, seed0=500, grid=64)
    net = ld.KpnUNet(seed=3, coarse_kernels=(5, 5))
    hist = ld.train(net, data, steps=400, batch_size=8, lr=5e-4, seed=4)
    assert np.all(np.isfinite(hist["loss_curve"]))
    # held-out scenes
    gains = []
    for s in range(3):
        r = ld.render_scene_levels(vpt, ld.sample_scene(9000 + s), 64, (4,), 512, grid=64)
        lv = r["levels"][0]
        noise = torch.tensor([0.5], device="cuda")
        out = net.denoise(lv["radiance"][None], lv["albedo"][None], lv["normal"][None], lv["depth"][None],
                          lv["transmittance"][None], noise)[0]
        before = ld.relmse(lv["radiance"], r["target"])
        after = ld.relmse(out, r["target"])
        gains.append(before / after)
        print(f"held-out scene {s}: relMSE noisy {before:.4g} -> denoised {after:.4g}")
    print("loss curve", hist["loss_curve"])
    assert np.mean(gains) > 1.5

    net.save(str(tmp_path / "model"))
    info = json.load(open(tmp_path / "model" / "model_info.json"))
    assert info["input_feature_maps"][0] == "Result" and info["blend"] == "kpn"
    back = ld.KpnUNet.load(str(tmp_path / "model"))
    assert back.coarse_kernels == (5, 5)
    assert torch.equal(back.param, net.param) and torch.equal(back.param_bf16, net.param_bf16)


def test_denoise_graph_equals_eager_denoise():
    """The captured denoise (one graph launch) gives the eager result for new inputs."""
    net = ld.KpnUNet(seed=5, coarse_kernels=(5, 5))
    g = torch.Generator(device="cuda").manual_seed(1)
    n, h, w = 1, 64, 128
    mk = lambda c: torch.rand((n, c, h, w), device="cuda", generator=g)  # noqa: E731
    graph = net.graph(n, h, w)
    for _ in range(2):
        args = (mk(3) * 2, mk(3), mk(3), mk(1), mk(1), torch.tensor([0.5], device="cuda"))
        got = graph(*args).clone()
        ref = net.denoise(*args)
        assert torch.allclose(got, ref, rtol=1e-6, atol=1e-6)


def test_fused_feature_read_and_graph_from_renderer():
    """vpt.read_denoiser_features writes the same planes as the per-map reads (identical arithmetic),
    and DenoiseGraph.from_renderer gives the eager denoise of those planes."""
    ld.setup_scene(vpt, ld.sample_scene(4242), grid=64, max_bounces=16)
    vpt.set_use_feature_maps(["Albedo", "Normal", "Depth", "Transmittance"])
    img = torch.zeros((3, 48, 64), device="cuda")
    vpt.set_frame_index(0)
    out = vpt.render_frame(img, 3)
    f = ld.read_features(vpt, img)
    for key, name, planes in (("albedo", "Albedo", 3), ("normal", "Normal", 3), ("depth", "Depth", 1),
                              ("transmittance", "Transmittance", 1)):
        assert torch.equal(f[key], vpt.get_feature_map_from_string(img, name)[:planes]), key
    net = ld.KpnUNet(seed=6)
    graph = net.graph(1, 48, 64)
    noise = torch.tensor([0.5], device="cuda")
    got = graph.from_renderer(vpt, out, noise).clone()
    ref = net.denoise(out[None], f["albedo"][None], f["normal"][None], f["depth"][None], f["transmittance"][None],
                      noise)
    assert torch.allclose(got, ref, rtol=1e-6, atol=1e-6)
    vpt.set_use_feature_maps([])
