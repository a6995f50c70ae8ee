"""The reference's model contract (PyTorchDenoiser::loadModelFromFile, src/Denoiser/PyTorchDenoiser.cpp:
637-800) as restated in cloudrendering_b200/pytorch_denoiser.py: model_info.json keys, defaults and
error messages, and the packing of the input feature maps (FEATURE_MAP_NUM_CHANNELS order), on the
CPU."""
import json

import pytest
import torch
import torch.nn.functional as F

from cloudrendering_b200.pytorch_denoiser import DENOISER_FEATURE_MAPS, PyTorchDenoiser, save_model


class ColorOut(torch.nn.Module):
    def __init__(self, cin):
        super().__init__()
        self.conv = torch.nn.Conv2d(cin, 4, 3, padding=1)

    def forward(self, x):
        return self.conv(x)


class InvIter(torch.nn.Module):
    def __init__(self, cin, ks: int = 5):
        super().__init__()
        self.c0 = torch.nn.Conv2d(cin, ks * ks + 3, 3, padding=1)
        self.c1 = torch.nn.Conv2d(cin, ks * ks + 3, 3, padding=1)
        self.c2 = torch.nn.Conv2d(cin, ks * ks, 3, padding=1)
        self.cp = torch.nn.Conv2d(cin, ks * ks, 3, padding=1)

    def forward(self, x, prev):
        x1 = F.avg_pool2d(x, 2)
        x2 = F.avg_pool2d(x1, 2)
        return self.cp(x), self.c2(x2), self.c1(x1), self.c0(x)


def test_feature_map_table_matches_the_reference_order():
    names = [n for n, _ in DENOISER_FEATURE_MAPS]
    assert names[:6] == ["Color", "Albedo", "Flow", "Flow Reverse", "Position", "Normal"]
    assert dict(DENOISER_FEATURE_MAPS)["Depth"] == 2 and dict(DENOISER_FEATURE_MAPS)["Position"] == 3
    assert len(names) == 18


def test_model_info_keys_and_defaults(tmp_path):
    p = str(tmp_path / "inv.pt")
    save_model(InvIter(12), p, ["color", "Reproj_UV", "ALBEDO", "Depth"], blend="inv_iter", use_previous_frame=True)
    d = PyTorchDenoiser(device="cpu")
    d.load_model_from_file(p)
    assert d.blend_inv_iter and d.use_previous_frame and not d.use_fp16
    assert d.use_batch_dimension  # the first parameter is a 4-d conv weight
    assert d.input_feature_maps == ["Color", "Reproj_UV", "Albedo", "Depth"] and d.num_channels == 12
    assert d.renderer_feature_maps() == ["Albedo", "Depth"]
    p2 = str(tmp_path / "c.pt")
    save_model(ColorOut(4), p2, ["Color"], use_batch_dimension=False, use_fp16=True)
    d.load_model_from_file(p2)
    assert not d.blend_inv_iter and not d.use_previous_frame and not d.use_batch_dimension and d.use_fp16


@pytest.mark.parametrize("info, message", [
    ({"blend": 3, "input_feature_maps": ["Color"]}, "Element 'blendtype' should be a string"),
    ({"use_previous_frame": 1, "input_feature_maps": ["Color"]}, "'use_previous_frame' should be a bool"),
    ({"use_batch_dimension": "yes", "input_feature_maps": ["Color"]}, "'use_batch_dimension' should be a bool"),
    ({"use_fp16": 0, "input_feature_maps": ["Color"]}, "'use_fp16' should be a bool"),
    ({}, "Array 'input_feature_maps' could not be found"),
    ({"input_feature_maps": "Color"}, "'input_feature_maps' is not an array"),
    ({"input_feature_maps": [1]}, "is not a string"),
    ({"input_feature_maps": ["Colour"]}, "Invalid feature map name 'colour'"),
    ({"input_feature_maps": ["Color", "nabla(z)"]}, "'nabla\\(z\\)' used by"),
])
def test_model_info_errors(tmp_path, info, message):
    p = str(tmp_path / "m.pt")
    torch.jit.save(torch.jit.script(ColorOut(4)), p, _extra_files={"model_info.json": json.dumps(info)})
    d = PyTorchDenoiser(device="cpu")
    with pytest.raises(RuntimeError, match=message):
        d.load_model_from_file(p)
    assert d.module is None


def test_missing_model_info_and_bad_file(tmp_path):
    p = str(tmp_path / "m.pt")
    torch.jit.save(torch.jit.script(ColorOut(4)), p)
    d = PyTorchDenoiser(device="cpu")
    with pytest.raises(RuntimeError, match="Couldn't find model_info.json"):
        d.load_model_from_file(p)
    (tmp_path / "junk.pt").write_bytes(b"not a model")
    with pytest.raises(RuntimeError, match="Couldn't load the PyTorch module"):
        d.load_model_from_file(str(tmp_path / "junk.pt"))


def test_pack_input_order_and_channels(tmp_path):
    p = str(tmp_path / "m.pt")
    maps = ["Color", "Reproj_UV", "Normal (Length 1)", "Depth", "Flow", "Position"]
    save_model(ColorOut(4 + 2 + 3 + 2 + 2 + 3), p, maps)
    d = PyTorchDenoiser(device="cpu")
    d.load_model_from_file(p)
    h, w = 4, 6
    color = torch.arange(4 * h * w, dtype=torch.float32).reshape(4, h, w)
    feats = {"Normal (Length 1)": torch.full((4, h, w), 3 ** -0.5), "Depth": torch.full((2, h, w), 7.0),
             "First X": torch.full((4, h, w), -1.0)}  # the renderer's maps (Normal (Length 1) normalised there)
    x = d.pack_input(color, lambda n: feats[n])
    assert x.shape == (1, 16, h, w)
    assert torch.equal(x[0, :4], color)
    assert torch.allclose(x[0, 4, 0, :], (torch.arange(w) + 0.5) / w) and torch.allclose(x[0, 5, :, 0], (torch.arange(h) + 0.5) / h)
    assert torch.allclose(x[0, 6:9], torch.full((3, h, w), 3 ** -0.5))
    assert torch.equal(x[0, 9:11], torch.full((2, h, w), 7.0)) and torch.equal(x[0, 11:13], torch.zeros(2, h, w))
    assert torch.equal(x[0, 13:16], torch.full((3, h, w), -1.0))
