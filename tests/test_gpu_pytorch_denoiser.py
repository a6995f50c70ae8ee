"""The "PyTorch Denoiser Module" through the vpt module surface (set_denoiser,
set_pytorch_denoiser_model_file, render_frame; Module.cpp:1070 and PyTorchDenoiser.cpp:182-460):
the model receives the feature maps in its model_info.json order, its image output is returned,
and for blend "inv_iter" its kernel logits are composed by the KPN kernels (whose own parity with
the reference's Kernel.cu restatement is tests/test_gpu_kpn.py), with the previous frame on the
second call."""
import pytest
import torch

from cloudrendering_b200 import kpn, vpt
from cloudrendering_b200.pytorch_denoiser import save_model
from tests.test_pytorch_denoiser_cpu import InvIter

pytestmark = pytest.mark.gpu


class AlbedoOut(torch.nn.Module):
    def forward(self, x):
        return x[:, 4:8] * 1.0


@pytest.fixture(scope="module", autouse=True)
def module():
    vpt.initialize()
    vpt.set_vpt_mode_from_name("Delta Tracking")
    yield
    vpt.set_denoiser("None")
    vpt.cleanup()


def test_image_output_model_gets_the_feature_maps(tmp_path):
    p = str(tmp_path / "albedo.pt")
    save_model(AlbedoOut(), p, ["Color", "Albedo"], use_batch_dimension=True)
    vpt.set_denoiser("PyTorch Denoiser Module")
    vpt.set_pytorch_denoiser_model_file(p)
    t = torch.zeros((4, 48, 64), device="cuda")
    out = vpt.render_frame(t, 3)
    alb = vpt.get_feature_map_from_string(t, "Albedo")
    assert out.shape == (4, 48, 64)
    assert torch.equal(out, alb)
    cpu = vpt.render_frame(torch.zeros((3, 48, 64)), 1)
    assert cpu.device.type == "cpu" and cpu.shape == (3, 48, 64)
    vpt.set_denoiser("None")


def test_inv_iter_model_is_composed_by_the_kpn_kernels(tmp_path):
    torch.manual_seed(0)
    model = InvIter(4 + 2 + 4).cuda()
    p = str(tmp_path / "inv.pt")
    save_model(model, p, ["Color", "Reproj_UV", "Albedo"], blend="inv_iter", use_previous_frame=True)
    vpt.set_denoiser("PyTorch Denoiser Module")
    vpt.set_pytorch_denoiser_model_file(p)
    den = vpt.S.torch_denoiser
    t = torch.zeros((4, 64, 64), device="cuda")
    outs, expected = [], []
    prev = None
    for _ in range(2):
        out = vpt.render_frame(t, 2)
        color = vpt.get_feature_map(t, 0)  # the accumulated result before denoising
        x = den.pack_input(color, lambda n: vpt.get_feature_map_from_string(t, n))
        with torch.no_grad():
            lprev, l2, l1, l0 = model(x, prev if prev is not None else torch.zeros_like(x[:, :4]))
        ref = kpn.inv_iter_denoise(x, l0.contiguous(), l1.contiguous(), l2.contiguous(),
                                   lprev.contiguous() if prev is not None else None, prev,
                                   x[:, 4:6] if prev is not None else None)[0]
        prev = ref[None].clone()
        outs.append(out)
        expected.append(ref)
    for o, r in zip(outs, expected):
        assert torch.isfinite(o).all()
        assert torch.allclose(o, r, rtol=1e-4, atol=1e-5)
    assert not torch.allclose(outs[0], outs[1])  # the second frame used the previous output
    vpt.set_denoiser("None")
