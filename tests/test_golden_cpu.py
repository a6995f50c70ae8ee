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


def test_last_frame_maps_fixture_is_consistent():
    """tests/golden/ref_last_frame_maps.npz (the reference's First W, Flow, Flow Reverse and Reprojected
    UV images): where the last frame scattered (first W pdf > 0), Flow is the pixel minus the
    reprojected uv in pixels (Clouds.glsl:240-246 and 319-327 project the same point); where it had no
    event, Flow and First W are zero."""
    import json
    import os

    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_last_frame_maps.npz"))
    meta = json.loads(str(z["meta"]))
    assert set(meta) == {"fbm_lastframe_delta", "fbm_lastframe_nee"}
    for name, m in meta.items():
        h, w = m["height"], m["width"]
        first_w, flow, uv = z[name + "__first_w"], z[name + "__flow"], z[name + "__reproj_uv"]
        event = first_w[..., 3] > 0
        assert 0.3 < event.mean() < 1.0
        ys, xs = np.mgrid[0:h, 0:w]
        fx = xs - (uv[..., 0] * w - 0.5)
        fy = ys - (uv[..., 1] * h - 0.5)
        assert np.allclose(flow[..., 0][event], fx[event], atol=2e-3)
        assert np.allclose(flow[..., 1][event], fy[event], atol=2e-3)
        # no event on the last frame: zero flow and zero first W (an absorbed first event has a flow but
        # no scatter direction, so the converse does not hold)
        none = np.all(flow[..., :2] == 0.0, axis=-1)
        assert none.any() and np.all(first_w[none] == 0.0)
        # unit directions after the first scatter
        assert np.allclose(np.linalg.norm(first_w[..., :3][event], axis=-1), 1.0, atol=1e-4)
