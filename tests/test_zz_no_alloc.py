"""vpt_eaw_denoise_rgba_noalloc (the EAW entry point whose ping-pong image is a fixed array inside the
library) against vpt_eaw_denoise_rgba (which allocates its ping-pong image), through the C ABI.

Calls in a row with different sizes and iteration counts: the first fills the whole shared array (the
largest image it holds), and the later ones, with odd iteration counts, find that call's contents in
the array and must still give the same image.  Tolerance as in the EAW parity test
(rtol 1e-5, atol 1e-6); both entry points run the same kernel, so the images are expected to be equal.
"""
import ctypes

import numpy as np
import pytest
import torch

from cloudrendering_b200 import _lib

pytestmark = pytest.mark.gpu

VPT_OK = 0
VPT_ERR_ARG = 1
MAX_PIXELS = 1024 * 1024


def dptr(t):
    return ctypes.c_void_p(t.data_ptr())


def images(seed, h, w):
    g = torch.Generator(device="cpu").manual_seed(seed)
    color = torch.rand((h, w, 4), generator=g) * 2.0
    pos = torch.rand((h, w, 4), generator=g) * 0.2
    nrm = torch.rand((h, w, 4), generator=g)
    return [t.cuda() for t in (color, pos, nrm)]


def run(lib, fn, color, pos, nrm, iterations, quirk):
    h, w = color.shape[:2]
    out = torch.full_like(color, float("nan"))
    st = getattr(lib, fn)(dptr(color), dptr(pos), dptr(nrm), w, h, iterations, 5.0, 0.1, 0.1, quirk, dptr(out), None)
    torch.cuda.synchronize()
    assert st == VPT_OK, _lib.load().vpt_status_string(st)
    return out.cpu().numpy()


def test_noalloc_eaw_matches_allocating_eaw_on_two_calls_in_a_row():
    lib = _lib.load()
    torch.cuda.set_device(0)
    # (h, w), iterations, quirk, seed: the maximum image first, so that stale contents of the array
    # would show across the whole of the later images
    calls = [((1024, 1024), 4, 1, 12), ((96, 160), 5, 0, 11), ((1000, 1048), 3, 0, 13)]
    for (h, w), iterations, quirk, seed in calls:
        color, pos, nrm = images(seed, h, w)
        want = run(lib, "vpt_eaw_denoise_rgba", color, pos, nrm, iterations, quirk)
        got = run(lib, "vpt_eaw_denoise_rgba_noalloc", color, pos, nrm, iterations, quirk)
        assert np.isfinite(got).all()
        assert np.allclose(got, want, rtol=1e-5, atol=1e-6)


def test_noalloc_eaw_rejects_images_above_its_maximum():
    lib = _lib.load()
    buf = torch.zeros(16, device="cuda")  # a valid pointer; the size check returns before any use
    for w, h in [(MAX_PIXELS + 1, 1), (2048, 1024), (1025, 1024)]:
        st = lib.vpt_eaw_denoise_rgba_noalloc(dptr(buf), None, None, w, h, 1, 5.0, 0.1, 0.1, 0, dptr(buf), None)
        assert st == VPT_ERR_ARG
    torch.cuda.synchronize()


def test_noalloc_eaw_rejects_an_output_that_overlaps_an_input():
    lib = _lib.load()
    color, pos, nrm = images(3, 16, 16)
    for out in (color, pos, nrm, color[4:]):
        st = lib.vpt_eaw_denoise_rgba_noalloc(dptr(color), dptr(pos), dptr(nrm), 16, 16, 3, 5.0, 0.1, 0.1, 0,
                                              dptr(out), None)
        assert st == VPT_ERR_ARG
    torch.cuda.synchronize()
