"""Pins the CPU oracle to the reference's own tracer shaders: tests/golden/ref_paths.npz holds the
outputs of Data/Shaders/VPT/Clouds.glsl (+ tracker includes) compiled for the CPU
(tests/golden/make_golden.py).  Every camera path of frame 0 must match bit for bit or to float
rounding, and the 8-frame running mean must agree to fp32 accumulation error."""
import numpy as np
import pytest

from tests.harness import golden_cases, oracle_scene, path_agreement

CASES = golden_cases()


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_shader_paths(name):
    sp, inv, paths, mean8 = CASES[name]
    sc = oracle_scene(None, sp, 1)  # nee_ess runs with ess_ref_compat (the reference's behaviour)
    sc.set("inv_view_proj", inv)
    ys, xs = np.mgrid[0:sp.height, 0:sp.width]
    got = sc.trace_paths(xs.reshape(-1), ys.reshape(-1), np.zeros(xs.size, np.uint32)).reshape(paths.shape)
    agree = path_agreement(got, paths, rtol=1e-5, atol=1e-6)
    exact = float(np.mean(np.all(got == paths, axis=-1)))
    print(f"{name}: agreement {agree:.4f}, bit-exact {exact:.4f}")
    assert agree >= 0.995
    sc.set("num_frames", 8)
    film, _, _ = sc.render()
    m = film.reshape(paths.shape) / 8.0
    close = np.all(np.abs(m - mean8) <= 1e-5 + 1e-4 * np.abs(mean8), axis=-1)
    assert close.mean() >= 0.99
