"""Learned kernel-predicting denoiser, trained and run on the GPU by this package's own kernels.

The reference's learned path (src/Denoiser/PyTorchDenoiser.cpp:637-800) loads a TorchScript model
and a ``model_info.json`` and runs it through libtorch; it has no network and no training code of its
own.  Here the network is a 5-level U-Net of 3x3 convolutions (widths 32-64-96-128-160 by default,
2x2 average pooling down, nearest upsampling + skip concatenation up, ReLU) whose head predicts a
k x k kernel per pixel (k*k logits, softmaxed; k = 13 by default); the kernel is applied to the noisy radiance
(perPixelKernelCuda semantics, modules/kpn_module/src/Kernel.cu:38-135).  Every convolution,
forward and backward, runs on the tcgen05 tensor cores (csrc/vpt_unet.cu); torch only allocates
device memory and orders the launches on its current stream.

Training pairs come from the tracer itself: a noisy render of a seeded cloud scene at a few sample
counts (radiance plus albedo / normal / depth / primary-ray transmittance features averaged over the
same frames; optionally the per-pixel second moment of the frames' radiance, from which the network
input carries the standard error of each pixel's mean) against a many-sample render of the same scene from a disjoint frame range.  The loss
is the relative MSE sum (d - t)^2 / (t^2 + 0.01) / count the evaluation uses.

Parameters are saved as ``<dir>/weights.npz`` (fp32) with ``<dir>/model_info.json`` in the
reference's key style (``input_feature_maps``, ``blend``, ...; see load()).
"""
from __future__ import annotations

import ctypes
import json
import math
import os
import time
from typing import Dict, List, Optional, Sequence

import numpy as np
import torch
import torch.distributed as dist

from . import _lib

WIDTHS = (32, 64, 96, 128, 160)
IN_CHANNELS = 16
KERNEL_SIZE = 13
COARSE_KERNELS = ()  # kernel sizes of the half / quarter-resolution heads (multi-scale reconstruction)
LOSS_EPS = 1e-2
# feature maps the network reads (names of VolumetricPathTracingPass.hpp:74-80, plus the 2D
# primary-ray transmittance of this package)
INPUT_FEATURE_MAPS = ["Result", "Albedo", "Normal", "Depth", "Transmittance"]


def _p(t: Optional[torch.Tensor], offset_elems: int = 0):
    if t is None:
        return None
    return ctypes.c_void_p(t.data_ptr() + offset_elems * t.element_size())


def head_channels(kernel_size: int, blend: bool = False) -> int:
    """Channels of a kernel head: k*k tap logits (+ 1 blend logit), rounded up to 16."""
    return (kernel_size * kernel_size + (1 if blend else 0) + 15) // 16 * 16


def layer_table(widths: Sequence[int], kernel_size: int = KERNEL_SIZE, coarse_kernels: Sequence[int] = ()) -> List[dict]:
    """Convolution layers in forward order: name, cin, cout, level.  coarse_kernels: kernel sizes of the
    half- and quarter-resolution heads of the multi-scale reconstruction (empty: one full-resolution
    kernel)."""
    w = list(widths)
    if len(w) != 5 or any(c % 16 for c in w):
        raise ValueError("widths: five multiples of 16")
    t = []
    for l in range(4):
        t.append(dict(name=f"enc{l}a", cin=IN_CHANNELS if l == 0 else w[l - 1], cout=w[l], level=l))
        t.append(dict(name=f"enc{l}b", cin=w[l], cout=w[l], level=l))
    t.append(dict(name="mida", cin=w[3], cout=w[4], level=4))
    t.append(dict(name="midb", cin=w[4], cout=w[4], level=4))
    for l in (3, 2, 1, 0):
        t.append(dict(name=f"dec{l}a", cin=w[l + 1] + w[l], cout=w[l], level=l))
        t.append(dict(name=f"dec{l}b", cin=w[l], cout=w[l], level=l))
    multi = len(coarse_kernels) > 0
    t.append(dict(name="head", cin=w[0], cout=head_channels(kernel_size, multi), level=0))
    for l, k in enumerate(coarse_kernels, start=1):
        t.append(dict(name=f"head{l}", cin=w[l], cout=head_channels(k, l < len(coarse_kernels)), level=l))
    return t


class KpnUNet:
    """The network, its fp32 master parameters, Adam state and activation buffers (one device)."""

    def __init__(self, widths: Sequence[int] = WIDTHS, seed: int = 0, device: Optional[torch.device] = None,
                 kernel_size: int = KERNEL_SIZE, coarse_kernels: Sequence[int] = COARSE_KERNELS):
        self.lib = _lib.load()
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.widths = tuple(int(c) for c in widths)
        for k in (kernel_size, *coarse_kernels):
            if k % 2 == 0 or not 1 <= k <= 15:
                raise ValueError("kernel sizes: odd, 1..15")
        if len(coarse_kernels) > 2:
            raise ValueError("at most two coarse levels (half and quarter resolution)")
        self.kernel_size = int(kernel_size)
        self.coarse_kernels = tuple(int(k) for k in coarse_kernels)
        self.kernels = (self.kernel_size,) + self.coarse_kernels
        self.head_channels = head_channels(self.kernel_size, len(self.coarse_kernels) > 0)
        self.layers = layer_table(self.widths, self.kernel_size, self.coarse_kernels)
        self.by_name = {L["name"]: L for L in self.layers}
        off = 0
        for L in self.layers:
            L["w_off"] = off
            off += L["cout"] * 9 * L["cin"]
            L["b_off"] = off
            off += L["cout"]
        self.count = off
        self.param = torch.zeros(self.count, dtype=torch.float32, device=self.device)
        self.param_bf16 = torch.zeros(self.count, dtype=torch.bfloat16, device=self.device)
        self.m1 = torch.zeros_like(self.param)
        self.m2 = torch.zeros_like(self.param)
        self.grad = torch.zeros_like(self.param)
        self.wrot = {L["name"]: torch.zeros((L["cin"], 9, L["cout"]), dtype=torch.bfloat16, device=self.device)
                     for L in self.layers}
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.steps = 0
        self._buf: Dict[str, torch.Tensor] = {}
        self.init_parameters(seed)

    # ---- parameters ----
    def init_parameters(self, seed: int) -> None:
        """He-normal weights (std sqrt(2 / fan_in), fan_in over the used input channels), zero
        biases; the head starts small so the first kernels are close to a k x k box filter."""
        g = np.random.default_rng(seed)
        host = np.zeros(self.count, np.float32)
        for L in self.layers:
            cin_used = 15 if L["name"] == "enc0a" else L["cin"]
            std = math.sqrt(2.0 / (9 * cin_used)) if not L["name"].startswith("head") else 1e-3
            w = (g.standard_normal((L["cout"], 9, L["cin"])) * std).astype(np.float32)
            if L["name"] == "enc0a":
                w[:, :, 15:] = 0.0
            host[L["w_off"]:L["w_off"] + w.size] = w.reshape(-1)
        self.set_parameters(host)

    def set_parameters(self, host: np.ndarray) -> None:
        if host.size != self.count:
            raise ValueError(f"expected {self.count} parameters, got {host.size}")
        self.param.copy_(torch.from_numpy(np.ascontiguousarray(host, np.float32)))
        self._call("vpt_unet_to_bf16", _p(self.param), _p(self.param_bf16), self.count, self._stream())
        self._rotate_all()

    def parameters_host(self) -> np.ndarray:
        return self.param.cpu().numpy()

    def _rotate_all(self) -> None:
        for L in self.layers:
            self._call("vpt_unet_rotate_weights", _p(self.param_bf16, L["w_off"]), _p(self.wrot[L["name"]]),
                       L["cin"], L["cout"], self._stream())

    # ---- plumbing ----
    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _call(self, name: str, *args) -> None:
        st = getattr(self.lib, name)(*args)
        if st != 0:
            raise RuntimeError(f"{name} failed: {self.lib.vpt_status_string(st).decode()}")

    def check_errors(self) -> None:
        """Raises if a kernel's bounded wait expired since the last check."""
        e = int(self.err.item())
        if e:
            self.err.zero_()
            raise RuntimeError(f"device error in the denoiser network: {self.lib.vpt_status_string(e).decode()}")

    def buf(self, name: str, shape, dtype=torch.bfloat16) -> torch.Tensor:
        t = self._buf.get(name)
        if t is None or tuple(t.shape) != tuple(shape) or t.dtype != dtype:
            t = torch.empty(shape, dtype=dtype, device=self.device)
            self._buf[name] = t
        return t

    def _conv(self, L: dict, x: torch.Tensor, out: torch.Tensor, n: int, h: int, w: int, relu: int,
              out_f32: int = 0) -> torch.Tensor:
        self._call("vpt_unet_conv3x3", _p(x), _p(self.param_bf16, L["w_off"]), _p(self.param, L["b_off"]), None,
                   _p(out), n, h, w, L["cin"], L["cout"], relu, out_f32, _p(self.err), self._stream())
        return out

    def _input_grad(self, L: dict, dy: torch.Tensor, mask: Optional[torch.Tensor], out: torch.Tensor, n: int, h: int,
                    w: int) -> torch.Tensor:
        self._call("vpt_unet_conv3x3", _p(dy), _p(self.wrot[L["name"]]), None, _p(mask), _p(out), n, h, w,
                   L["cout"], L["cin"], 0, 0, _p(self.err), self._stream())
        return out

    def _weight_grad(self, L: dict, x: torch.Tensor, dy: torch.Tensor, n: int, h: int, w: int) -> None:
        P = n * h * w
        rows = self.lib.vpt_unet_wgrad_rows(L["cin"])
        mtiles = rows // 128
        splits = max(1, min((P + 63) // 64, (2 * 148 + mtiles - 1) // mtiles))
        pps = ((P + splits - 1) // splits + 63) // 64 * 64
        splits = self.lib.vpt_unet_wgrad_splits(n, h, w, L["cin"], L["cout"], pps)
        part = self.buf("wgrad_partial", (splits * rows * L["cout"],), torch.float32)
        self._call("vpt_unet_conv3x3_wgrad", _p(x), _p(dy), _p(part), n, h, w, L["cin"], L["cout"], pps,
                   _p(self.err), self._stream())
        bblocks = max(1, min(296, (P + 255) // 256))
        bpart = self.buf("bias_partial", (bblocks * L["cout"],), torch.float32)
        self._call("vpt_unet_bias_grad", _p(dy), _p(bpart), P, L["cout"], bblocks, self._stream())
        self._call("vpt_unet_reduce_grads", _p(part), splits, L["cin"], L["cout"], _p(bpart), bblocks,
                   _p(self.grad, L["w_off"]), _p(self.grad, L["b_off"]), self._stream())

    # ---- network ----
    def forward(self, x0: torch.Tensor) -> torch.Tensor:
        """x0: packed input [n, h, w, 16] bf16 (h, w multiples of 16).  Returns the head's logits
        [n, h, w, head channels] fp32; the activations stay in this object for backward()."""
        n, h, w, c = x0.shape
        if c != IN_CHANNELS or h % 16 or w % 16:
            raise ValueError("input must be [n, h, w, 16] with h, w multiples of 16")
        self.shape = (n, h, w)
        W = self.widths
        dims = [(h >> l, w >> l) for l in range(5)]
        cur = x0
        for l in range(4):
            hh, ww = dims[l]
            a = self._conv(self.by_name[f"enc{l}a"], cur, self.buf(f"enc{l}a", (n, hh, ww, W[l])), n, hh, ww, 1)
            e = self._conv(self.by_name[f"enc{l}b"], a, self.buf(f"enc{l}b", (n, hh, ww, W[l])), n, hh, ww, 1)
            pooled = self.buf(f"pool{l}", (n, hh // 2, ww // 2, W[l]))
            self._call("vpt_unet_pool2", _p(e), _p(pooled), n, hh, ww, W[l], self._stream())
            cur = pooled
        hh, ww = dims[4]
        a = self._conv(self.by_name["mida"], cur, self.buf("mida", (n, hh, ww, W[4])), n, hh, ww, 1)
        cur = self._conv(self.by_name["midb"], a, self.buf("midb", (n, hh, ww, W[4])), n, hh, ww, 1)
        for l in (3, 2, 1, 0):
            hh, ww = dims[l]
            ca, cs = W[l + 1], W[l]
            u = self.buf(f"cat{l}", (n, hh, ww, ca + cs))
            self._call("vpt_unet_upcat", _p(cur), _p(self._buf[f"enc{l}b"]), _p(u), n, hh, ww, ca, cs, self._stream())
            a = self._conv(self.by_name[f"dec{l}a"], u, self.buf(f"dec{l}a", (n, hh, ww, W[l])), n, hh, ww, 1)
            cur = self._conv(self.by_name[f"dec{l}b"], a, self.buf(f"dec{l}b", (n, hh, ww, W[l])), n, hh, ww, 1)
        hh, ww = dims[0]
        self._x0 = x0
        self.logits = [self._conv(self.by_name["head"], cur,
                                  self.buf("logits", (n, hh, ww, self.head_channels), torch.float32), n, hh, ww, 0, 1)]
        for l in range(1, len(self.kernels)):
            L = self.by_name[f"head{l}"]
            h2, w2 = dims[l]
            self.logits.append(self._conv(L, self._buf[f"dec{l}b"], self.buf(f"logits{l}", (n, h2, w2, L["cout"]),
                                                                          torch.float32), n, h2, w2, 0, 1))
        return self.logits[0]

    def backward(self, dlogits) -> None:
        """dlogits: bf16 gradient of the loss at the heads' outputs, [n, h, w, head channels] (or one per
        level of the multi-scale reconstruction).  Fills self.grad (flat, same layout as the parameters)."""
        n, h, w = self.shape
        W = self.widths
        B = self._buf
        dls = list(dlogits) if isinstance(dlogits, (list, tuple)) else [dlogits]
        dlogits = dls[0]
        dims = [(h >> l, w >> l) for l in range(5)]
        hh, ww = dims[0]
        L = self.by_name["head"]
        self._weight_grad(L, B["dec0b"], dlogits, n, hh, ww)
        g = self._input_grad(L, dlogits, B["dec0b"], self.buf("g0", (n, hh, ww, W[0])), n, hh, ww)
        dcat = {}
        for l in (0, 1, 2, 3):
            hh, ww = dims[l]
            Lb, La = self.by_name[f"dec{l}b"], self.by_name[f"dec{l}a"]
            self._weight_grad(Lb, B[f"dec{l}a"], g, n, hh, ww)
            ga = self._input_grad(Lb, g, B[f"dec{l}a"], self.buf(f"gdec{l}a", (n, hh, ww, W[l])), n, hh, ww)
            self._weight_grad(La, B[f"cat{l}"], ga, n, hh, ww)
            ca, cs = W[l + 1], W[l]
            du = self._input_grad(La, ga, None, self.buf(f"gcat{l}", (n, hh, ww, ca + cs)), n, hh, ww)
            dcat[l] = du
            lo = B["midb"] if l == 3 else B[f"dec{l + 1}b"]
            h2, w2 = dims[l + 1]
            g = self.buf(f"glo{l + 1}", (n, h2, w2, ca))
            self._call("vpt_unet_upcat_grad_lo", _p(du), _p(lo), _p(g), n, hh, ww, ca, cs, self._stream())
            if l + 1 < len(dls):  # the coarse kernel head on this decoder level
                Lh = self.by_name[f"head{l + 1}"]
                self._weight_grad(Lh, lo, dls[l + 1], n, h2, w2)
                hg = self._input_grad(Lh, dls[l + 1], lo, self.buf(f"ghead{l + 1}", (n, h2, w2, ca)), n, h2, w2)
                self._call("vpt_unet_add", _p(g), _p(hg), _p(g), g.numel(), self._stream())
        hh, ww = dims[4]
        self._weight_grad(self.by_name["midb"], B["mida"], g, n, hh, ww)
        ga = self._input_grad(self.by_name["midb"], g, B["mida"], self.buf("gmida", (n, hh, ww, W[4])), n, hh, ww)
        self._weight_grad(self.by_name["mida"], B["pool3"], ga, n, hh, ww)
        dpool = self._input_grad(self.by_name["mida"], ga, None, self.buf("gpool3", (n, hh, ww, W[3])), n, hh, ww)
        for l in (3, 2, 1, 0):
            hh, ww = dims[l]
            ca, cs = W[l + 1], W[l]
            ge = self.buf(f"genc{l}b", (n, hh, ww, W[l]))
            self._call("vpt_unet_encoder_grad", _p(dcat[l]), ca + cs, ca, _p(dpool), _p(B[f"enc{l}b"]), _p(ge), n,
                       hh, ww, W[l], self._stream())
            Lb, La = self.by_name[f"enc{l}b"], self.by_name[f"enc{l}a"]
            self._weight_grad(Lb, B[f"enc{l}a"], ge, n, hh, ww)
            ga = self._input_grad(Lb, ge, B[f"enc{l}a"], self.buf(f"genc{l}a", (n, hh, ww, W[l])), n, hh, ww)
            xin = self._x0 if l == 0 else B[f"pool{l - 1}"]
            self._weight_grad(La, xin, ga, n, hh, ww)
            if l > 0:
                dpool = self._input_grad(La, ga, None, self.buf(f"gpool{l - 1}", (n, hh, ww, W[l - 1])), n, hh, ww)

    def adam_step(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8) -> None:
        self.steps += 1
        self._call("vpt_unet_adam", _p(self.param), _p(self.param_bf16), _p(self.m1), _p(self.m2), _p(self.grad),
                   self.count, lr, beta1, beta2, eps, self.steps, 1.0, self._stream())
        self._rotate_all()

    # ---- the kernel-prediction head ----
    def pack(self, radiance, albedo=None, normal=None, depth=None, transmittance=None, noise_level=None,
             second_moment=None):
        n, _, h, w = radiance.shape
        x0 = self.buf("input", (n, h, w, IN_CHANNELS))
        self._call("vpt_unet_pack_input", _p(radiance), _p(albedo), _p(normal), _p(depth), _p(transmittance),
                   _p(noise_level), _p(second_moment), _p(x0), n, h, w, self._stream())
        return x0

    def reconstruct(self, radiance, target=None, out=None):
        """Applies the predicted kernels (multi-scale: at full, half and quarter resolution, blended);
        with a target also the loss (device scalar) and the gradients at the heads' logits.  Returns
        (out, loss, dlogits per level)."""
        if len(self.kernels) == 1:
            o, loss, dl = self.head(self.logits[0], radiance, target, out)
            return o, loss, [dl]
        n, _, h, w = radiance.shape
        L = len(self.kernels)
        xs, ds, cs = [radiance], [], [None] * L
        for l in range(1, L):
            hl, wl = h >> l, w >> l
            x = self.buf(f"x{l}", (n, 3, hl, wl), torch.float32)
            self._call("vpt_kpn_avg_pool2", _p(xs[-1]), n, 3, hl * 2, wl * 2, _p(x), self._stream())
            xs.append(x)
        for l in range(L):
            hl, wl = h >> l, w >> l
            d = self.buf(f"d{l}", (n, 3, hl, wl), torch.float32)
            hc = self.logits[l].shape[-1]
            self._call("vpt_unet_kpn_head", _p(self.logits[l]), hc, self.kernels[l], _p(xs[l]), None, _p(d), None,
                       None, n, hl, wl, LOSS_EPS, self._stream())
            ds.append(d)
        cs[L - 1] = ds[L - 1]
        for l in range(L - 2, -1, -1):
            hl, wl = h >> l, w >> l
            c = out if (l == 0 and out is not None) else self.buf(f"c{l}", (n, 3, hl, wl), torch.float32)
            hc = self.logits[l].shape[-1]
            k = self.kernels[l]
            self._call("vpt_unet_kpn_combine", _p(ds[l]), _p(cs[l + 1]), _p(self.logits[l]), hc, k * k, _p(c), n,
                       hl, wl, self._stream())
            cs[l] = c
        if target is None:
            return cs[0], None, None
        blocks = self.lib.vpt_unet_head_blocks(n, h, w)
        lp = self.buf("loss_partial", (blocks,), torch.float32)
        dls = []
        g_in = None
        for l in range(L):
            hl, wl = h >> l, w >> l
            hc = self.logits[l].shape[-1]
            k = self.kernels[l]
            dl = self.buf(f"dlogits{l}", (n, hl, wl, hc))
            blend = l < L - 1
            g_next = self.buf(f"gc{l + 1}", (n, 3, hl // 2, wl // 2), torch.float32) if blend else None
            self._call("vpt_unet_kpn_level_grad", _p(self.logits[l]), hc, k, k * k if blend else -1, _p(xs[l]),
                       _p(ds[l]), _p(cs[l + 1]) if blend else None, _p(g_in), _p(cs[0]) if l == 0 else None,
                       _p(target) if l == 0 else None, LOSS_EPS, _p(dl), _p(g_next), _p(lp) if l == 0 else None, n,
                       hl, wl, self._stream())
            dls.append(dl)
            g_in = g_next
        return cs[0], lp.sum(), dls

    def head(self, logits, radiance, target=None, out=None):
        """Applies the predicted kernels; with a target also the loss (device scalar) and the
        gradient at the logits (returned as (out, loss, dlogits))."""
        n, _, h, w = radiance.shape
        blocks = self.lib.vpt_unet_head_blocks(n, h, w)
        dl = lp = None
        if target is not None:
            dl = self.buf("dlogits", (n, h, w, self.head_channels))
            lp = self.buf("loss_partial", (blocks,), torch.float32)
        self._call("vpt_unet_kpn_head", _p(logits), self.head_channels, self.kernel_size, _p(radiance), _p(target),
                   _p(out), _p(dl), _p(lp), n, h, w, LOSS_EPS, self._stream())
        return out, (lp.sum() if lp is not None else None), dl

    def train_step(self, batch: dict, lr: float, group=None) -> torch.Tensor:
        """One Adam step on `batch`.  With a process group (data-parallel training, one rank per GPU),
        the ranks' gradients are averaged before the step, so every rank's parameters stay equal."""
        x0 = self.pack(batch["radiance"], batch.get("albedo"), batch.get("normal"), batch.get("depth"),
                       batch.get("transmittance"), batch.get("noise_level"), batch.get("second_moment"))
        self.forward(x0)
        _, loss, dls = self.reconstruct(batch["radiance"], batch["target"])
        self.backward(dls)
        if group is not None:
            average_gradients(self.grad, group)
        self.adam_step(lr)
        return loss

    def denoise(self, radiance, albedo=None, normal=None, depth=None, transmittance=None, noise_level=None,
                second_moment=None):
        """Denoised radiance [n, 3, h, w] fp32 (h, w multiples of 16)."""
        x0 = self.pack(radiance, albedo, normal, depth, transmittance, noise_level, second_moment)
        self.forward(x0)
        out = torch.empty_like(radiance)
        self.reconstruct(radiance, None, out)
        return out

    def graph(self, n: int, h: int, w: int) -> "DenoiseGraph":
        """A CUDA-graph replay of denoise() for inputs of this shape (one launch from the host)."""
        return DenoiseGraph(self, n, h, w)

    # ---- the model contract ----
    def save(self, directory: str) -> None:
        os.makedirs(directory, exist_ok=True)
        np.savez(os.path.join(directory, "weights.npz"), params=self.parameters_host())
        info = {"input_feature_maps": INPUT_FEATURE_MAPS, "blend": "kpn", "kernel_size": self.kernel_size,
                "coarse_kernel_sizes": list(self.coarse_kernels),
                "use_previous_frame": False, "use_batch_dimension": True, "use_fp16": False,
                "network": "unet", "widths": list(self.widths), "input_channels": IN_CHANNELS,
                "head_channels": self.head_channels, "loss": "relmse", "loss_eps": LOSS_EPS, "steps": self.steps}
        with open(os.path.join(directory, "model_info.json"), "w") as f:
            json.dump(info, f, indent=1)

    @classmethod
    def load(cls, directory: str, device=None) -> "KpnUNet":
        with open(os.path.join(directory, "model_info.json")) as f:
            info = json.load(f)
        if info.get("network") != "unet" or info.get("blend") != "kpn":
            raise RuntimeError(f"unsupported model_info.json in {directory}: network {info.get('network')}, "
                               f"blend {info.get('blend')}")
        net = cls(info["widths"], device=device, kernel_size=int(info.get("kernel_size", KERNEL_SIZE)),
                  coarse_kernels=tuple(info.get("coarse_kernel_sizes", ())))
        net.set_parameters(np.load(os.path.join(directory, "weights.npz"))["params"])
        net.steps = int(info.get("steps", 0))
        return net


class DenoiseGraph:
    """denoise() captured once for a fixed input shape and replayed: the input packing, every
    convolution of the U-Net and the kernel reconstruction are one graph launch (the per-kernel host
    calls dominate a single 512^2 image otherwise).  Inputs are copied into the graph's own tensors."""

    def __init__(self, net: KpnUNet, n: int, h: int, w: int):
        dev = net.device
        self.net = net
        self.inputs = {"radiance": torch.zeros((n, 3, h, w), device=dev), "albedo": torch.zeros((n, 3, h, w), device=dev),
                       "normal": torch.zeros((n, 3, h, w), device=dev), "depth": torch.zeros((n, 1, h, w), device=dev),
                       "transmittance": torch.zeros((n, 1, h, w), device=dev),
                       "noise_level": torch.zeros((n,), device=dev)}
        stream = torch.cuda.Stream(dev)
        stream.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(stream):
            self._run()  # warm-up: allocates every buffer outside the capture
        torch.cuda.current_stream(dev).wait_stream(stream)
        torch.cuda.synchronize(dev)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.out = self._run()
        net.check_errors()

    def _run(self):
        i = self.inputs
        return self.net.denoise(i["radiance"], i["albedo"], i["normal"], i["depth"], i["transmittance"],
                                i["noise_level"])

    def from_renderer(self, vpt, radiance, noise_level):
        """Denoises the renderer's current accumulation: its feature planes are written straight into
        the graph's inputs (one launch), then the graph is replayed.  radiance [3, H, W] (or [1, 3, H, W]),
        noise_level [1]; batch 1."""
        i = self.inputs
        vpt.read_denoiser_features(i["albedo"], i["normal"], i["depth"], i["transmittance"])
        i["radiance"].copy_(radiance.reshape(i["radiance"].shape))
        i["noise_level"].copy_(noise_level.reshape(i["noise_level"].shape))
        self.graph.replay()
        return self.out

    def __call__(self, radiance, albedo=None, normal=None, depth=None, transmittance=None, noise_level=None):
        for k, v in (("radiance", radiance), ("albedo", albedo), ("normal", normal), ("depth", depth),
                     ("transmittance", transmittance), ("noise_level", noise_level)):
            if v is None:
                self.inputs[k].zero_()
            else:
                self.inputs[k].copy_(v.reshape(self.inputs[k].shape))
        self.graph.replay()
        return self.out


# ---------------------------------------------------------------------------------------------
# training pairs from the tracer
# ---------------------------------------------------------------------------------------------
def relmse(x: torch.Tensor, ref: torch.Tensor, eps: float = LOSS_EPS) -> float:
    """mean over pixels and channels of (x - ref)^2 / (ref^2 + eps)."""
    x = x.double()
    ref = ref.double()
    return float(((x - ref) ** 2 / (ref * ref + eps)).mean())


def sample_scene(seed: int) -> dict:
    """A seeded cloud scene of the training / evaluation family (fBm cloud, sun + constant sky)."""
    g = np.random.default_rng(seed)
    sun = g.normal(size=3)
    sun[1] = abs(sun[1]) + 0.5
    a = g.uniform(0, 2 * math.pi)
    elev = g.uniform(-0.2, 0.8)
    return dict(seed=int(seed), extinction=float(math.exp(g.uniform(math.log(100.0), math.log(1000.0)))),
                g=float(g.uniform(0.6, 0.9)), sun=(sun / np.linalg.norm(sun)).tolist(),
                camera=[2.0 * math.sin(a), elev, 2.0 * math.cos(a)], threshold=float(g.uniform(0.25, 0.4)))


def setup_scene(vpt, sc: dict, grid: int = 128, max_bounces: int = 64) -> None:
    vpt.set_max_grid_extent(0.5)
    vpt.generate_fbm_cloud(grid, seed=sc["seed"], threshold=sc["threshold"])
    vpt.set_extinction_scale(sc["extinction"])
    vpt.set_scattering_albedo([0.99, 0.99, 0.99])
    vpt.set_phase_g(sc["g"])
    vpt.set_use_builtin_environment_map("Constant Sky + Sun")
    vpt.set_sky_color([0.2, 0.2, 0.2])
    vpt.set_sun(sc["sun"], [5.0, 5.0, 5.0])
    vpt.set_camera_position(sc["camera"])
    vpt.set_camera_target([0.0, 0.0, 0.0])
    vpt.set_camera_fovy(60.0)
    vpt.set_max_bounces(max_bounces)
    vpt.set_grid_interpolation("Stochastic")
    vpt.set_denoiser("None")
    vpt.set_vpt_mode_from_name("Delta Tracking")


def read_features(vpt, img: torch.Tensor) -> dict:
    """Feature planes of the current accumulation: albedo [3], normal [3], depth [1], transmittance [1]
    (one launch: vpt.read_denoiser_features)."""
    _, h, w = img.shape
    f = {"albedo": torch.empty((3, h, w), device=img.device), "normal": torch.empty((3, h, w), device=img.device),
         "depth": torch.empty((1, h, w), device=img.device), "transmittance": torch.empty((1, h, w), device=img.device)}
    vpt.read_denoiser_features(f["albedo"], f["normal"], f["depth"], f["transmittance"])
    return f


def target_seed_offset(width: int, height: int) -> int:
    """Seed offset of target renders: the seed of a path is (frame * W * H + pixel + offset) mod 2^32
    (Clouds.glsl:80-84), so frame indices alone repeat every 2^32 / (W * H) frames.  Half the pixel
    count is not a multiple of W * H, so the targets' seeds of a pixel (frames 0 .. 2^32 / (W * H) - 1)
    differ from every seed the noisy inputs use at offset 0."""
    return (width * height) // 2


FEATURE_FRAMES = 2  # feature maps are accumulated over the first 2 frames (first-hit features converge fast)


def render_scene_levels(vpt, sc: dict, size: int, spp_levels: Sequence[int], target_spp: int, grid: int = 128,
                        max_bounces: int = 64, second_moment: bool = False) -> dict:
    """Noisy renders of one scene after each sample count in spp_levels (nested: the frames of a
    level include the previous level's) with their features (and, with second_moment, the mean
    square of the frames' radiance), and the target (target_spp frames whose seeds differ from the
    inputs', see target_seed_offset), all on the GPU."""
    setup_scene(vpt, sc, grid, max_bounces)
    vpt.set_use_feature_maps(["Albedo", "Normal", "Depth", "Transmittance"])
    vpt.set_feature_frame_limit(FEATURE_FRAMES)
    vpt.set_collect_statistics(second_moment)
    img = torch.zeros((3, size, size), dtype=torch.float32, device="cuda")
    vpt.set_frame_index(0)
    levels = []
    done = 0
    for spp in spp_levels:
        rad = vpt.render_frame(img, spp - done).clone()
        done = spp
        m2 = vpt.get_film_moments(size, size, spp)[1] if second_moment else None
        levels.append(dict(spp=spp, radiance=rad, second_moment=m2, **read_features(vpt, img)))
    vpt.set_use_feature_maps([])
    vpt.set_feature_frame_limit(0)
    vpt.set_collect_statistics(False)
    if target_spp * size * size > (1 << 32):
        raise ValueError("target_spp exceeds the distinct seeds of one seed offset at this size")
    vpt.set_seed_offset(target_seed_offset(size, size))
    vpt.set_frame_index(0)
    left = target_spp
    tgt = None
    while left > 0:
        k = min(left, 256)
        tgt = vpt.render_frame(img, k)
        left -= k
    target = tgt.clone()
    vpt.set_seed_offset(0)
    vpt.set_frame_index(0)
    return dict(levels=levels, target=target)


class TrainingSet:
    """Tracer-generated training pairs held on the GPU: for each scene and sample count, the noisy
    radiance and features, and the scene's target."""

    def __init__(self, vpt, num_scenes: int, size: int = 256, spp_levels=(1, 4, 16, 64), target_spp: int = 1024,
                 seed0: int = 1000, grid: int = 128, second_moment: bool = False):
        t0 = time.perf_counter()
        self.size = size
        self.spp_levels = tuple(spp_levels)
        S, L = num_scenes, len(self.spp_levels)
        dev = torch.device("cuda")
        self.radiance = torch.empty((S, L, 3, size, size), device=dev)
        self.albedo = torch.empty((S, L, 3, size, size), device=dev)
        self.normal = torch.empty((S, L, 3, size, size), device=dev)
        self.depth = torch.empty((S, L, 1, size, size), device=dev)
        self.transmittance = torch.empty((S, L, 1, size, size), device=dev)
        self.second_moment = torch.empty((S, L, 3, size, size), device=dev) if second_moment else None
        self.target = torch.empty((S, 3, size, size), device=dev)
        for s in range(S):
            r = render_scene_levels(vpt, sample_scene(seed0 + s), size, self.spp_levels, target_spp, grid,
                                    second_moment=second_moment)
            for j, lv in enumerate(r["levels"]):
                self.radiance[s, j] = lv["radiance"]
                self.albedo[s, j] = lv["albedo"]
                self.normal[s, j] = lv["normal"]
                self.depth[s, j] = lv["depth"]
                self.transmittance[s, j] = lv["transmittance"]
                if second_moment:
                    self.second_moment[s, j] = lv["second_moment"]
            self.target[s] = r["target"]
        torch.cuda.synchronize()
        self.seconds = time.perf_counter() - t0
        self.paths = S * size * size * (max(self.spp_levels) + target_spp)

    def batch(self, rng: np.random.Generator, batch_size: int) -> dict:
        """A random batch of (scene, sample count) pairs with random flips / transposes.  The pair
        indices are drawn on the GPU (a generator seeded from rng on first use): no host round trip,
        so the host queues the next training step while the GPU runs the current one."""
        S, L = self.radiance.shape[:2]
        if getattr(self, "_gen", None) is None:
            self._gen = torch.Generator(device="cuda")
            self._gen.manual_seed(int(rng.integers(0, 2**62)))
        si = torch.randint(0, S, (batch_size,), device="cuda", generator=self._gen)
        li = torch.randint(0, L, (batch_size,), device="cuda", generator=self._gen)
        keys = ["radiance", "albedo", "normal", "depth", "transmittance"]
        if self.second_moment is not None:
            keys.append("second_moment")
        out = {k: getattr(self, k)[si, li] for k in keys}
        out["target"] = self.target[si]
        if getattr(self, "_inv_sqrt_spp", None) is None:  # one upload: a copy per batch would wait for the GPU
            self._inv_sqrt_spp = 1.0 / torch.tensor(self.spp_levels, dtype=torch.float32, device="cuda").sqrt()
        out["noise_level"] = self._inv_sqrt_spp[li]
        flip = rng.integers(0, 8)
        for k in list(out.keys()):
            if k == "noise_level":
                continue
            t = out[k]
            if flip & 1:
                t = t.flip(-1)
            if flip & 2:
                t = t.flip(-2)
            if flip & 4:
                t = t.transpose(-1, -2)
            out[k] = t.contiguous()
        for k in ("depth", "transmittance"):
            out[k] = out[k][:, 0].contiguous()
        return out


def average_gradients(grad: torch.Tensor, group=None) -> None:
    """Data-parallel training: replaces the flat fp32 gradient by the mean over the ranks of `group`
    (one all_reduce of the whole vector: 7.6 MB for the 1.9 M-parameter network, a few microseconds of
    NVLink time against a multi-millisecond step)."""
    world = dist.get_world_size(group)
    if world > 1:
        dist.all_reduce(grad, op=dist.ReduceOp.SUM, group=group)
        grad.div_(float(world))


def train(net: KpnUNet, data: TrainingSet, steps: int, batch_size: int = 8, lr: float = 1e-4, seed: int = 0,
          log_every: int = 0, lr_end: Optional[float] = None, group=None) -> dict:
    """Adam training (learning rate constant, or cosine-annealed from lr to lr_end); returns timing and
    the loss curve (mean loss per logging window).  With a process group the training is data parallel:
    each rank draws its own batches (its rank offsets the seed) from its own training set and the
    gradients are averaged every step (networks built with the same seed start equal and stay equal)."""
    if group is not None:
        seed = seed + 7919 * dist.get_rank(group)
    rng = np.random.default_rng(seed)
    losses = []
    acc = torch.zeros((), dtype=torch.float32, device=net.device)
    window = max(1, log_every or steps // 10)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(steps):
        step_lr = lr if lr_end is None else lr_end + 0.5 * (lr - lr_end) * (1.0 + math.cos(math.pi * i / steps))
        loss = net.train_step(data.batch(rng, batch_size), step_lr, group)
        acc += loss
        if (i + 1) % window == 0:
            losses.append(float(acc.item()) / window)
            acc.zero_()
    torch.cuda.synchronize()
    net.check_errors()
    return {"steps": steps, "seconds": time.perf_counter() - t0, "loss_curve": losses}


def layer_timings(net: KpnUNet, batch: int = 8, size: int = 256, reps: int = 20) -> Dict[str, dict]:
    """Device time of every convolution of a training step at batch x size^2 (forward, input gradient,
    weight gradient; random activations), with the flops of each.  The repetitions are captured in a
    CUDA graph, so that host-side launch cost does not hide the device time of small layers."""
    def timed(fn):
        fn()
        torch.cuda.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            for _ in range(reps):
                fn()
        graph.replay()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        graph.replay()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    out = {}
    for L in net.layers:
        hh, ww = size >> L["level"], size >> L["level"]
        x = torch.randn((batch, hh, ww, L["cin"]), device=net.device).to(torch.bfloat16)
        y = torch.empty((batch, hh, ww, L["cout"]), dtype=torch.bfloat16, device=net.device)
        dy = torch.randn((batch, hh, ww, L["cout"]), device=net.device).to(torch.bfloat16)
        dx = torch.empty_like(x)
        flop = 2.0 * 9 * L["cin"] * L["cout"] * batch * hh * ww
        t_f = timed(lambda: net._conv(L, x, y, batch, hh, ww, 1))
        t_d = timed(lambda: net._input_grad(L, dy, x, dx, batch, hh, ww))
        t_w = timed(lambda: net._weight_grad(L, x, dy, batch, hh, ww))
        out[L["name"]] = {"forward_ms": t_f, "input_grad_ms": t_d, "weight_grad_ms": t_w, "gflop": flop / 1e9}
    net.check_errors()
    return out


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser(description="learned denoiser network: kernel timings and profiling launches")
    ap.add_argument("--layers", action="store_true", help="time every convolution of a training step")
    ap.add_argument("--profile-launches", action="store_true",
                    help="one forward and one weight-gradient launch of two level-0 layers (32->32, 96->32) at "
                         "8x256^2, for a profiler")
    ap.add_argument("--profile-layer", default="",
                    help="one forward launch of the named layer (e.g. dec3a) at batch x size^2, for a profiler")
    ap.add_argument("--profile-denoise", action="store_true",
                    help="one denoise of a batch x size^2 image (every inference launch), for a profiler")
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--batch", type=int, default=8)
    args = ap.parse_args()
    net = KpnUNet(seed=0)
    if args.layers:
        print(json.dumps(layer_timings(net, args.batch, args.size), indent=1))
    if args.profile_layer:
        L = net.by_name[args.profile_layer]
        n, hh, ww = args.batch, args.size >> L["level"], args.size >> L["level"]
        x = torch.randn((n, hh, ww, L["cin"]), device=net.device).to(torch.bfloat16)
        y = torch.empty((n, hh, ww, L["cout"]), dtype=torch.bfloat16, device=net.device)
        net._conv(L, x, y, n, hh, ww, 1)
        torch.cuda.synchronize()
        net.check_errors()
        print("ok")
    if args.profile_denoise:
        g = torch.Generator(device=net.device).manual_seed(1)
        mk = lambda c: torch.rand((args.batch, c, args.size, args.size), device=net.device, generator=g)  # noqa: E731
        out = net.denoise(mk(3) * 2, mk(3), mk(3), mk(1), mk(1), torch.full((args.batch,), 0.5, device=net.device))
        torch.cuda.synchronize()
        net.check_errors()
        print("ok", float(out.mean()))
    if args.profile_launches:
        for name in ("enc0b", "dec0a"):
            L = net.by_name[name]
            n, hh, ww = args.batch, args.size, args.size
            x = torch.randn((n, hh, ww, L["cin"]), device=net.device).to(torch.bfloat16)
            y = torch.empty((n, hh, ww, L["cout"]), dtype=torch.bfloat16, device=net.device)
            dy = torch.randn((n, hh, ww, L["cout"]), device=net.device).to(torch.bfloat16)
            net._conv(L, x, y, n, hh, ww, 1)
            net._weight_grad(L, x, dy, n, hh, ww)
        torch.cuda.synchronize()
        net.check_errors()
        print("ok")
