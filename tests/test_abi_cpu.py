"""CPU tests of the C-ABI boundary: the library loads and exports every declared entry point."""
import ctypes

import pytest
import os
import re

from cloudrendering_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for hdr in os.listdir(os.path.join(ROOT, "include")):
        if not hdr.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", hdr)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(vpt_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


@pytest.mark.parametrize("path", [_lib.LIB_PATH, _lib.LIB_PATH_DR])
def test_library_exports_every_declared_symbol(path):
    lib = ctypes.CDLL(path)
    names = declared_functions()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    assert set(declared_functions()) == set(_lib.SIGNATURES)


def test_status_strings_and_abi_version_without_gpu():
    lib = _lib.load()
    assert lib.vpt_abi_version() == 1
    assert lib.vpt_status_string(0) == b"ok"
    assert lib.vpt_status_string(4) == b"iteration guard reached"


def test_null_context_is_rejected_without_gpu():
    lib = _lib.load()
    assert lib.vpt_set_phase_g(None, 0.5) == 1
    assert lib.vpt_render_frames(None, 1, None) == 1
    assert lib.vpt_last_error(None) == b"null context"


def test_stateless_entry_points_reject_bad_arguments_without_gpu():
    lib = _lib.load()
    assert lib.vpt_build_supervoxel_grid(None, 8, 8, 8, 8, 0, None, None, None, None, None) == 1
    assert lib.vpt_build_occupancy_grid(None, 8, 8, 8, 8, 0, 0.0, None, None) == 1
    assert lib.vpt_eaw_denoise_rgba(None, None, None, 4, 4, 1, 5.0, 0.1, 0.1, 0, None, None) == 1
    assert lib.vpt_build_environment_pyramid(None, 4, 4, 3, None, None) == 1
