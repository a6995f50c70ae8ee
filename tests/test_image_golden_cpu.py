"""The oracle's environment importance map and EAW filter against the reference's own shaders run on
the CPU (OctahedralMapper.glsl; the compute stage of EAWDenoise.glsl; fixture
tests/golden/image_filters.npz).  The map is bit-exact.  EAW agrees to rtol 1e-5 / atol 2e-5: the
shader reads its neighbours through a linear-filtering sampler at texel centres computed in float
((x + 0.5) / width + offset * step), which on images whose width is not a power of two lands up to
~1e-6 of a texel away from the centre and blends that much of the next texel in (the CPU stand-in
filters in float; a GPU's fixed-point filter weights would round it away)."""
import numpy as np
import pytest

from oracle import bridge
from tests.harness import image_golden

OCTA, EAW = image_golden()


@pytest.mark.parametrize("key", sorted(OCTA))
def test_octahedral_map_matches_reference(key):
    env, ref = OCTA[key]
    res = ref.shape[0]
    levels = int(np.log2(res))
    got = bridge.env_pyramid(env, levels)[:res * res].reshape(res, res)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("key", sorted(EAW))
def test_eaw_compute_path_matches_reference(key):
    color, pos, nrm, it, phi, ref = EAW[key]
    got = bridge.eaw(color, pos, nrm, it, *phi, 1)  # the compute path's colour weight (ref_compute_quirk)
    assert np.allclose(got, ref, rtol=1e-5, atol=2e-5)
