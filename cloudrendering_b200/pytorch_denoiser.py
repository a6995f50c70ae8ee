"""The reference's learned-denoiser model contract ("PyTorch Denoiser Module").

Restates PyTorchDenoiser::loadModelFromFile (src/Denoiser/PyTorchDenoiser.cpp:637-800) and the
model-input / output handling of PyTorchDenoiser::denoise (:182-460):

* a model file is a TorchScript archive with an extra file ``model_info.json``: ``input_feature_maps``
  (names of FEATURE_MAP_NAMES, src/Denoiser/Denoiser.hpp:83-101, compared case-insensitively),
  ``blend`` (``"inv_iter"``: the module returns (lprev, l2, l1, l0) kernel logits, composed by the
  kernel-predicting reconstruction; anything else: the module returns the image), ``use_previous_frame``,
  ``use_batch_dimension`` (default: whether the first parameter has 4 dimensions) and ``use_fp16``;
* the input is the concatenation of the feature maps in that order, each with its
  FEATURE_MAP_NUM_CHANNELS channels, as (1,) C x H x W float (half with use_fp16);
* with use_previous_frame the previous output (zeros first) is the second input.

The module's forward runs through torch.jit (as the reference runs it through libtorch); the
inv_iter reconstruction and the previous-frame reprojection run on this package's CUDA kernels
(kpn.py).  Feature maps this renderer does not produce raise an error naming them.
"""
from __future__ import annotations

import json
import os
from typing import Callable, Dict, List, Optional

import torch

from . import kpn

# FEATURE_MAPS of src/Denoiser/Denoiser.hpp:83-101: name, channels
DENOISER_FEATURE_MAPS = [
    ("Color", 4), ("Albedo", 4), ("Flow", 2), ("Flow Reverse", 2), ("Position", 3), ("Normal", 3),
    ("Normal (Length 1)", 3), ("CloudOnly", 4), ("Depth", 2), ("Depth Far", 1), ("Density", 2), ("Background", 4),
    ("Reproj_UV", 2), ("Depth Blended", 2), ("Depth Nearest Opaque", 2), ("nabla(z)", 2), ("fwidth(z)", 1),
    ("Unused", 2),
]
_CHANNELS = {n: c for n, c in DENOISER_FEATURE_MAPS}
_BY_LOWER = {n.lower(): n for n, _ in DENOISER_FEATURE_MAPS}

# denoiser feature map -> (renderer feature map name of vpt.VPT_FEATURE_MAP_NAMES, channels taken);
# "Color" is the accumulated result
RENDERER_FEATURES = {
    "Albedo": ("Albedo", 4), "Position": ("First X", 3), "Normal": ("Normal", 3),
    "Normal (Length 1)": ("Normal (Length 1)", 3), "CloudOnly": ("Cloud Only", 4), "Depth": ("Depth", 2),
    "Depth Far": ("Depth Far", 1), "Density": ("Density", 2), "Background": ("Background", 4),
    "Depth Blended": ("Depth Blended", 2), "Depth Nearest Opaque": ("Depth Nearest Opaque", 2),
}
# maps the renderer provides without a feature pass (static camera: no motion between frames)
SYNTHESISED = {"Flow", "Flow Reverse", "Reproj_UV", "Unused"}


class PyTorchDenoiser:
    def __init__(self, device: Optional[torch.device] = None):
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.module = None
        self.model_path = ""
        self.blend_inv_iter = False
        self.use_previous_frame = False
        self.use_batch_dimension = False
        self.use_fp16 = False
        self.input_feature_maps: List[str] = []
        self.previous: Optional[torch.Tensor] = None
        self.zero_out_previous_frame = False

    # ---- loadModelFromFile ----
    def load_model_from_file(self, model_path: str) -> None:
        extra = {"model_info.json": ""}
        try:
            module = torch.jit.load(model_path, map_location=self.device, _extra_files=extra)
        except Exception as e:  # c10::Error / torch::jit::ErrorReport in the reference
            raise RuntimeError(f"Error: Couldn't load the PyTorch module from \"{model_path}\"! What: {e}") from None
        text = extra.get("model_info.json", "")
        if not text:
            raise RuntimeError(
                f"Error: Couldn't find model_info.json in the PyTorch module loaded from \"{model_path}\"!")
        try:
            root = json.loads(text)
        except ValueError as e:
            raise RuntimeError(f"Error in PyTorchDenoiser::loadModelFromFile: {e}") from None
        blend = False
        if "blend" in root:
            if not isinstance(root["blend"], str):
                raise RuntimeError(f"Error: Element 'blendtype' should be a string in \"{model_path}\"!")
            blend = root["blend"].lower() == "inv_iter"
        use_prev = False
        if "use_previous_frame" in root:
            if not isinstance(root["use_previous_frame"], bool):
                raise RuntimeError(f"Error: Element 'use_previous_frame' should be a bool in \"{model_path}\"!")
            use_prev = root["use_previous_frame"]
        params = list(module.parameters())
        use_batch = len(params) > 0 and params[0].dim() == 4
        if "use_batch_dimension" in root:
            if not isinstance(root["use_batch_dimension"], bool):
                raise RuntimeError(f"Error: Element 'use_batch_dimension' should be a bool in \"{model_path}\"!")
            use_batch = root["use_batch_dimension"]
        use_fp16 = self.use_fp16
        if "use_fp16" in root:
            if not isinstance(root["use_fp16"], bool):
                raise RuntimeError(f"Error: Element 'use_fp16' should be a bool in \"{model_path}\"!")
            use_fp16 = root["use_fp16"]
        if "input_feature_maps" not in root:
            raise RuntimeError("Error: Array 'input_feature_maps' could not be found in the model_info.json file of "
                               f"the PyTorch module loaded from \"{model_path}\"!")
        node = root["input_feature_maps"]
        if not isinstance(node, list):
            raise RuntimeError("Error: 'input_feature_maps' is not an array in the model_info.json file of the "
                               f"PyTorch module loaded from \"{model_path}\"!")
        maps = []
        for child in node:
            if not isinstance(child, str):
                raise RuntimeError("Error: A child of the array 'input_feature_maps' in the model_info.json file of "
                                   f"the PyTorch module loaded from \"{model_path}\" is not a string!")
            name = _BY_LOWER.get(child.lower())
            if name is None:
                raise RuntimeError(f"Error: Invalid feature map name '{child.lower()}' found in the model_info.json "
                                   f"file of the PyTorch module loaded from \"{model_path}\"!")
            if name != "Color" and name not in RENDERER_FEATURES and name not in SYNTHESISED:
                raise RuntimeError(f"Error: Feature map '{name}' used by \"{model_path}\" is not produced by this "
                                   "renderer.")
            maps.append(name)
        self.module = module
        self.model_path = model_path
        self.blend_inv_iter = blend
        self.use_previous_frame = use_prev
        self.use_batch_dimension = use_batch
        self.use_fp16 = use_fp16
        self.input_feature_maps = maps
        self.previous = None

    @property
    def num_channels(self) -> int:
        return sum(_CHANNELS[n] for n in self.input_feature_maps)

    def renderer_feature_maps(self) -> List[str]:
        """Feature maps of the renderer this model needs accumulated."""
        return sorted({RENDERER_FEATURES[n][0] for n in self.input_feature_maps if n in RENDERER_FEATURES})

    def reset_previous_frame(self) -> None:
        self.previous = None

    # ---- denoise ----
    def pack_input(self, color: torch.Tensor, feature: Callable[[str], torch.Tensor]) -> torch.Tensor:
        """1 x C x H x W float input: the feature maps in model order.  color: 4 x H x W accumulated
        result; feature(name) returns a renderer feature map [c, H, W]."""
        _, h, w = color.shape
        parts = []
        for name in self.input_feature_maps:
            c = _CHANNELS[name]
            if name == "Color":
                t = color[:4]
            elif name in RENDERER_FEATURES:
                t = feature(RENDERER_FEATURES[name][0])[:c]
            elif name == "Reproj_UV":  # static camera: each pixel maps to itself
                ys = (torch.arange(h, device=color.device, dtype=torch.float32) + 0.5) / h
                xs = (torch.arange(w, device=color.device, dtype=torch.float32) + 0.5) / w
                t = torch.stack([xs[None, :].expand(h, w), ys[:, None].expand(h, w)])
            else:  # Flow, Flow Reverse, Unused: no motion
                t = torch.zeros((c, h, w), device=color.device)
            parts.append(t.float())
        return torch.cat(parts, dim=0)[None].contiguous()

    def denoise(self, color: torch.Tensor, feature: Callable[[str], torch.Tensor]) -> torch.Tensor:
        """Denoised 4 x H x W float image."""
        if self.module is None:
            raise RuntimeError("Error in PyTorchDenoiser::denoise: no model loaded.")
        _, h, w = color.shape
        x = self.pack_input(color.to(self.device), feature)
        inp = x if self.use_batch_dimension else x[0]
        if self.use_fp16:
            inp = inp.half()
        inputs = [inp]
        has_prev = True
        if self.use_previous_frame:
            if self.previous is None or self.zero_out_previous_frame:
                has_prev = False
                self.previous = torch.zeros((1, 4, h, w), device=self.device)
            prev = self.previous if self.use_batch_dimension else self.previous[0]
            inputs.append(prev.half() if self.use_fp16 else prev.float())
        self.module.to(torch.float16 if self.use_fp16 else torch.float32)
        with torch.no_grad():
            result = self.module.forward(*inputs)
        if self.blend_inv_iter:
            lprev, l2, l1, l0 = (t.float() for t in result)
            if not self.use_batch_dimension:
                lprev, l2, l1, l0 = (t[None] if t.dim() == 3 else t for t in (lprev, l2, l1, l0))
            prev = self.previous if (self.use_previous_frame and has_prev) else None
            uv = x[:, 4:6] if prev is not None else None
            out = kpn.inv_iter_denoise(x, l0.contiguous(), l1.contiguous(), l2.contiguous(),
                                       lprev.contiguous() if prev is not None else None, prev, uv)
        else:
            out = result.float()
            if out.dim() == 3:
                out = out[None]
            if out.dim() != 4 or out.shape[0] != 1:
                raise RuntimeError("Error in PyTorchDenoiser::denoise: Expected a batch dimension of 1, but got "
                                   f"{out.shape[0] if out.dim() == 4 else out.dim()}.")
        self.previous = out.detach().clone()
        o = out[0]
        if o.shape[0] < 4:  # RGB output: alpha 1
            o = torch.cat([o, torch.ones((4 - o.shape[0], h, w), device=o.device)], dim=0)
        return o[:4].contiguous()


def save_model(module: torch.nn.Module, path: str, input_feature_maps: List[str], blend: Optional[str] = None,
               use_previous_frame: Optional[bool] = None, use_batch_dimension: Optional[bool] = None,
               use_fp16: Optional[bool] = None) -> None:
    """Writes a TorchScript archive with model_info.json in the layout loadModelFromFile reads."""
    info: Dict[str, object] = {"input_feature_maps": list(input_feature_maps)}
    if blend is not None:
        info["blend"] = blend
    if use_previous_frame is not None:
        info["use_previous_frame"] = use_previous_frame
    if use_batch_dimension is not None:
        info["use_batch_dimension"] = use_batch_dimension
    if use_fp16 is not None:
        info["use_fp16"] = use_fp16
    scripted = module if isinstance(module, torch.jit.ScriptModule) else torch.jit.script(module)
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    torch.jit.save(scripted, path, _extra_files={"model_info.json": json.dumps(info)})
