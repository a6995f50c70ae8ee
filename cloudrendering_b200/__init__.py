"""B200-native volumetric path-tracing core (CUDA sm_100a) behind the reference's `vpt` module API.

`cloudrendering_b200.vpt` mirrors the reference PyTorch module; the CUDA core itself is
`libvpt_b200.so` with the C ABI of include/vpt_b200.h.
"""
from . import vpt  # noqa: F401

__all__ = ["vpt"]
