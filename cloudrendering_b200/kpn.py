"""Kernel-predicting denoiser reconstruction on the CUDA core (the "inv_iter" blend of the
reference's PyTorch denoiser, src/Denoiser/PyTorchDenoiser.cpp:411-440).

A learned model predicts, per pixel, kernel logits at three scales (l2, l1, l0: k*k channels, plus 3
blend channels for l1 and l0) and for the reprojected previous frame (lprev).  The reconstruction
filters the quarter-resolution input with l2, then goes up one scale at a time: the inv_iter kernel
blends the upsampled prediction with the finer input's high frequencies (and the previous frame) and
filters the result with the scale's kernels.  All steps run in this library's kernels
(vpt_kpn_apply / vpt_kpn_inv_iter / vpt_kpn_avg_pool2 / vpt_kpn_reproject); torch only holds the
buffers.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import torch

from . import _lib


def _p(t: torch.Tensor):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _check(st, where):
    _lib.check(st, where)


def _cuda(t: torch.Tensor) -> torch.Tensor:
    if not t.is_cuda:
        raise RuntimeError("kpn: tensors must be on a CUDA device")
    return t.detach().to(torch.float32).contiguous()


def avg_pool2(x: torch.Tensor) -> torch.Tensor:
    x = _cuda(x)
    n, c, h, w = x.shape
    out = torch.empty((n, c, h // 2, w // 2), dtype=torch.float32, device=x.device)
    _check(_lib.load().vpt_kpn_avg_pool2(_p(x), n, c, h, w, _p(out), _stream()), "vpt_kpn_avg_pool2")
    return out


def apply_kernels(image: torch.Tensor, logits: torch.Tensor, kernel_size: int, softmax: bool = True) -> torch.Tensor:
    """per_pixel_kernel::forward with the softmax over the taps fused in."""
    image, logits = _cuda(image), _cuda(logits)
    n, c, h, w = image.shape
    wh, ww = logits.shape[2:]
    out = torch.empty((n, c, min(h, wh), min(w, ww)), dtype=torch.float32, device=image.device)
    _check(_lib.load().vpt_kpn_apply(_p(image), _p(logits), n, c, h, w, wh, ww, kernel_size, 1 if softmax else 0,
                                     _p(out), _stream()), "vpt_kpn_apply")
    return out


def inv_iter(x_hi, pred_lo, x_lo, prev: Optional[torch.Tensor], fused, kernel_size: int) -> torch.Tensor:
    x_hi, pred_lo, x_lo, fused = _cuda(x_hi), _cuda(pred_lo), _cuda(x_lo), _cuda(fused)
    n, c, h, w = x_hi.shape
    lh, lw = x_lo.shape[2:]
    wh, ww = fused.shape[2:]
    use_prev = prev is not None
    prev_t = _cuda(prev) if use_prev else x_hi
    out = torch.empty((n, c, min(h, wh), min(w, ww)), dtype=torch.float32, device=x_hi.device)
    _check(_lib.load().vpt_kpn_inv_iter(_p(x_hi), _p(pred_lo), _p(x_lo), _p(prev_t), _p(fused), n, c, h, w, lh, lw, wh,
                                        ww, kernel_size, 1 if use_prev else 0, _p(out), _stream()), "vpt_kpn_inv_iter")
    return out


def reproject(prev: torch.Tensor, uv: torch.Tensor) -> torch.Tensor:
    prev, uv = _cuda(prev), _cuda(uv)
    n, c, ph, pw = prev.shape
    h, w = uv.shape[2:]
    out = torch.empty((n, c, h, w), dtype=torch.float32, device=prev.device)
    _check(_lib.load().vpt_kpn_reproject(_p(prev), _p(uv), n, c, ph, pw, h, w, _p(out), _stream()),
           "vpt_kpn_reproject")
    return out


def inv_iter_denoise(x0: torch.Tensor, l0: torch.Tensor, l1: torch.Tensor, l2: torch.Tensor,
                     lprev: Optional[torch.Tensor] = None, prev: Optional[torch.Tensor] = None,
                     reproj_uv: Optional[torch.Tensor] = None) -> torch.Tensor:
    """The reconstruction of PyTorchDenoiser::denoise for blend "inv_iter" (PyTorchDenoiser.cpp:411-440).
    x0: N x C x H x W noisy input (its first 4 channels); l2 / l1 / l0: model outputs at 1/4, 1/2 and
    full resolution; lprev, prev, reproj_uv: previous-frame kernels, previous output and its
    reprojection texture coordinates (all None without a previous frame)."""
    kernel_size = 5 if l0.shape[1] >= 25 else 3
    x0 = _cuda(x0[:, :4])
    x1 = avg_pool2(x0)
    x2 = avg_pool2(x1)
    reproj0 = reproj1 = None
    if prev is not None:
        reproj0 = apply_kernels(reproject(prev, reproj_uv), lprev, kernel_size)
        reproj1 = avg_pool2(reproj0)
    kp2 = apply_kernels(x2, l2, kernel_size)
    kp1 = inv_iter(x1, kp2, x2, reproj1, l1, kernel_size)
    return inv_iter(x0, kp1, x1, reproj0, l0, kernel_size)
