"""The oracle's SVGF frame (oracle_svgf_frame) against the reference's own SVGF compute shaders run on the
CPU over five frames (fixture tests/golden/svgf_frames.npz): filtered image, colour history and moments
history.  Float sums in other orders: at least 99.9 % of the pixels agree to rtol 1e-4 on every channel
and every value to 1e-5 absolute."""
import numpy as np
import pytest

from oracle import bridge
from tests.harness import svgf_close, svgf_golden

META, INPUTS, OUTPUTS = svgf_golden()


@pytest.mark.parametrize("iterations", META["iterations"])
def test_oracle_svgf_matches_reference_shaders(iterations):
    h, w = META["h"], META["w"]
    hist = {"color": np.zeros((h, w, 4), np.float32), "moments": np.zeros((h, w, 4), np.float32),
            "normal": np.zeros((h, w, 4), np.float32), "depth": np.zeros((h, w), np.float32)}
    for f, (noisy, nrm, depth, fw, motion) in enumerate(INPUTS):
        out = bridge.svgf_frame(noisy, nrm, depth, fw, motion, hist, META["z_threshold"], META["normal_threshold"],
                                iterations)
        ref_out, ref_color, ref_moments = OUTPUTS[(iterations, f)]
        for name, got, exp in (("out", out, ref_out), ("color", hist["color"], ref_color),
                               ("moments", hist["moments"], ref_moments)):
            assert svgf_close(got, exp) >= 0.999, (f, name)
            assert np.abs(got - exp).max() <= 1e-5, (f, name)
