"""Generates tests/golden/ref_paths.npz from the reference's own tracer shaders
(Data/Shaders/VPT/Clouds.glsl and the tracker includes, compiled for the CPU by oracle/ref_build.py).

For every case the fixture stores the inputs (grid, scene parameters, camera matrix) and the
reference's output: the radiance of each camera path of frame 0 (1 spp; accImage after one frame is
the path radiance itself) and the reference's fp32 running mean after 8 frames.

With the argument ``depth_maps`` it writes tests/golden/ref_depth_maps.npz instead: the reference's
Depth Blended and Depth Nearest Opaque images (Clouds.glsl:367-383) after 4 frames; with
``last_frame_maps``, tests/golden/ref_last_frame_maps.npz: the First W, Flow, Flow Reverse and
Reprojected UV images, which hold the last frame's values, after 4 frames; with ``depth_deriv_maps``,
tests/golden/ref_depth_deriv_maps.npz: the Normal, Depth (nabla) and Depth (fwidth) images after 4 frames.

Run in a container that has the reference tree:  python tests/golden/make_golden.py [depth_maps]
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import bridge, ref_build  # noqa: E402
from tests.harness import (SceneSpec, camera_inv_view_proj, camera_view_proj, cloud_block, gradient_magnitude,  # noqa: E402
                           reference_scene)

W = H = 32


def env_image():
    rng = np.random.default_rng(9)
    rgba = np.ones((32, 64, 4), np.float32)
    rgba[..., :3] = 0.2 + rng.random((32, 64, 3)).astype(np.float32) * 0.05
    rgba[5:8, 20:24, :3] = 40.0
    return rgba


def cases():
    fbm = bridge.fbm(24, 2, base_frequency=3.0, contrast=3.5)
    base = dict(extinction=120.0, albedo=0.99, g=0.85, width=W, height=H, env="default", linear_rgb=1,
                cam_pos=(0.3, 0.4, 1.4), max_grid_extent=0.5)
    out = {
        # the reference test suite's fixtures (test/VolumetricPathTracingTestData.cpp) and settings
        "block1_delta": SceneSpec(grid=cloud_block(1, 1, 1), mode="delta", width=W, height=H),
        "block1_ratio": SceneSpec(grid=cloud_block(1, 1, 1), mode="ratio", width=W, height=H),
        "block8_decomposition_nearest": SceneSpec(grid=cloud_block(8, 8, 8), mode="decomposition",
                                                  interp="nearest", width=W, height=H),
        "block8b_nee": SceneSpec(grid=cloud_block(8, 8, 8, empty_boundary=True), mode="nee", width=W, height=H),
    }
    for name, kw in {"delta_stochastic": dict(mode="delta"), "delta_nearest": dict(mode="delta", interp="nearest"),
                     "delta_trilinear": dict(mode="delta", interp="trilinear"), "ratio": dict(mode="ratio"),
                     "nee": dict(mode="nee"), "nee_ess": dict(mode="nee", use_ess=True, ess_ref_compat=True),
                     "decomposition": dict(mode="decomposition"), "rrt": dict(mode="rrt"),
                     "nee_env_image": dict(mode="nee", env="image", env_rgba=env_image()),
                     "delta_black": dict(mode="delta", env="black"),
                     "delta_single_color": dict(mode="delta", env="single"),
                     # lights of the light editor (NEE only): a spot light in view space beside the
                     # camera plus a world-space point light; a directional light alone under a black sky
                     "nee_lights2": dict(mode="nee", lights=[
                         dict(type="Spotlight", space="View", position=(0.05, 0.1, 0.0), spot_direction=(0.0, -0.1, -1.0),
                              spot_total_width=0.6, spot_falloff_start=0.3, intensity=3.0),
                         dict(type="Point Light", space="World", position=(0.6, 0.8, 0.3), intensity=0.8,
                              color=(1.0, 0.8, 0.6))]),
                     "nee_light_directional_black": dict(mode="nee", env="black", lights=[
                         dict(type="Directional Light", space="World", position=(0.4, 0.9, 0.2), intensity=2.0,
                              use_distance=0)])}.items():
        kw2 = dict(base)
        kw2.update(kw)
        out["fbm_" + name] = SceneSpec(grid=fbm, **kw2)
    # spectral trackers: chromatic extinction and albedo, each collision-probability mode
    chroma = dict(extinction_base=(1.0, 0.55, 0.3), albedo_rgb=(0.99, 0.9, 0.8))
    for name, kw in {"sdt_max": dict(mode="spectral_delta", sdt_prob=0),
                     "sdt_avg": dict(mode="spectral_delta", sdt_prob=1),
                     "sdt_hist": dict(mode="spectral_delta", sdt_prob=2),
                     "sdt_hist_trilinear": dict(mode="spectral_delta", sdt_prob=2, interp="trilinear"),
                     "nees_max": dict(mode="spectral_nee", sdt_prob=0),
                     "nees_hist": dict(mode="spectral_nee", sdt_prob=2)}.items():
        kw2 = dict(base)
        kw2.update(chroma)
        kw2.update(kw)
        out["fbm_" + name] = SceneSpec(grid=fbm, **kw2)
    # emission grid (USE_EMISSION, next event tracking): a second fbm field on its own (smaller) box
    emission = bridge.fbm(20, 7, base_frequency=2.0, contrast=3.0)
    for name, kw in {"nee_emission": dict(mode="nee"),
                     "nee_emission_trilinear": dict(mode="nee", interp="trilinear"),
                     "nees_hist_emission": dict(mode="spectral_nee", sdt_prob=2, **chroma)}.items():
        kw2 = dict(base)
        kw2.update(kw)
        out["fbm_" + name] = SceneSpec(grid=fbm, emission=emission, emission_cap=1.6, emission_strength=3.0, **kw2)
    # transfer function (USE_TRANSFER_FUNCTION): a 64-entry table, transparent below 0.2, a warm ramp
    for name, kw in {"delta_tf": dict(mode="delta"), "delta_tf_trilinear": dict(mode="delta", interp="trilinear"),
                     "nee_tf": dict(mode="nee"), "nee_tf_trilinear": dict(mode="nee", interp="trilinear"),
                     "sdt_hist_tf": dict(mode="spectral_delta", sdt_prob=2, **chroma),
                     "nees_hist_tf": dict(mode="spectral_nee", sdt_prob=2, **chroma)}.items():
        kw2 = dict(base)
        kw2.update(kw)
        out["fbm_" + name] = SceneSpec(grid=fbm, tf=transfer_function_table(), emission_strength=2.5, **kw2)
    # the table's colour as scattering albedo of spectral tracking (USE_TRANSFER_FUNCTION_SCATTERING_ALBEDO)
    for name, kw in {"sdt_hist_tf_albedo": dict(mode="spectral_delta", sdt_prob=2, **chroma),
                     "nees_hist_tf_albedo": dict(mode="spectral_nee", sdt_prob=2, **chroma)}.items():
        kw2 = dict(base)
        kw2.update(kw)
        out["fbm_" + name] = SceneSpec(grid=fbm, tf=transfer_function_table(), emission_strength=2.5,
                                       tf_albedo_strength=0.6, **kw2)
    # environment-image rotation (USE_ENV_MAP_ROTATION): envMapDirRot = glm::eulerAngleYXZ(0.7, -0.4, 0.25)
    for name, kw in {"delta_env_image_rot": dict(mode="delta"), "nee_env_image_rot": dict(mode="nee")}.items():
        kw2 = dict(base)
        kw2.update(kw)
        kw2.update(env="image", env_rgba=env_image(), env_rot=env_rotation())
        out["fbm_" + name] = SceneSpec(grid=fbm, **kw2)
    # isosurfaces inside the volume (USE_ISOSURFACES, density field, Lambertian surfaces, delta tracking
    # with trilinear lookups): the reference's default surface, and a thinner medium with a coloured one
    for name, kw in {"delta_iso": dict(iso_value=0.5),
                     "delta_iso_coloured": dict(iso_value=0.3, iso_color=(0.9, 0.6, 0.3), extinction=40.0,
                                                albedo=0.9, g=0.2)}.items():
        kw2 = dict(base)
        kw2.update(kw)
        out["fbm_" + name] = SceneSpec(grid=fbm, mode="delta", interp="trilinear", iso=True, **kw2)
    # the other surface BRDFs built here: Blinn-Phong (exponent 10) and constant lighting ("Ambient")
    for name, brdf in {"delta_iso_blinn": "Blinn Phong", "delta_iso_ambient": "Ambient"}.items():
        kw2 = dict(base)
        kw2.update(iso_value=0.3, iso_color=(0.9, 0.6, 0.3), extinction=40.0, albedo=0.9, g=0.2)
        out["fbm_" + name] = SceneSpec(grid=fbm, mode="delta", interp="trilinear", iso=True, iso_brdf=brdf, **kw2)
    # Cook-Torrance with the pass's default parameters and with a glossier, partly metallic surface
    for name, params in {"delta_iso_cook": None,
                         "delta_iso_cook_metal": {"metallic": 0.6, "specular": 0.8, "roughness": 0.25}}.items():
        kw2 = dict(base)
        kw2.update(iso_value=0.3, iso_color=(0.9, 0.6, 0.3), extinction=40.0, albedo=0.9, g=0.2)
        out["fbm_" + name] = SceneSpec(grid=fbm, mode="delta", interp="trilinear", iso=True, iso_brdf="Cook Torrance",
                                       brdf_params=params, **kw2)
    # Disney (2012) with the pass's default parameters and with every lobe and parameter in use
    for name, params in {"delta_iso_disney": None,
                         "delta_iso_disney_all": {"subsurface": 0.3, "metallic": 0.3, "specular": 0.7,
                                                  "specular_tint": 0.4, "roughness": 0.4, "anisotropic": 0.5,
                                                  "sheen": 0.5, "sheen_tint": 0.3, "clearcoat": 0.7,
                                                  "clearcoat_gloss": 0.6}}.items():
        kw2 = dict(base)
        kw2.update(iso_value=0.3, iso_color=(0.9, 0.6, 0.3), extinction=40.0, albedo=0.9, g=0.2)
        out["fbm_" + name] = SceneSpec(grid=fbm, mode="delta", interp="trilinear", iso=True, iso_brdf="Disney (2012)",
                                       brdf_params=params, **kw2)
    # the clip plane (USE_CLIP_PLANE): an oblique plane through the cloud, camera on its positive side
    for name, kw in {"delta_clip": dict(mode="delta"), "nee_clip": dict(mode="nee"),
                     "sdt_hist_clip": dict(mode="spectral_delta", sdt_prob=2, **chroma)}.items():
        kw2 = dict(base)
        kw2.update(kw)
        out["fbm_" + name] = SceneSpec(grid=fbm, clip_plane=(0.3, 0.5, 0.8, -0.02), **kw2)
    # isosurfaces closed by the box faces and the clip plane (CLOSE_ISOSURFACES): a low iso value, so that
    # many camera rays enter the box inside a surface, and the plane through the cloud
    for name, mode in (("delta_iso_clip_close", "delta"), ("nee_iso_clip_close", "nee")):
        kw2 = dict(base)
        kw2.update(iso_value=0.05, iso_color=(0.9, 0.6, 0.3), extinction=40.0, albedo=0.9, g=0.2)
        out["fbm_" + name] = SceneSpec(grid=fbm, mode=mode, interp="trilinear", iso=True, clip_plane=(0.3, 0.5, 0.8, -0.02),
                                       close_iso=True, **kw2)
    # next event tracking with isosurfaces and surface next-event estimation, every BRDF (MIS for the
    # specular samples of Cook-Torrance and Disney)
    for name, brdf, params in (("nee_iso", "Lambertian", None), ("nee_iso_blinn", "Blinn Phong", None),
                               ("nee_iso_ambient", "Ambient", None),
                               ("nee_iso_cook", "Cook Torrance", {"metallic": 0.6, "specular": 0.8, "roughness": 0.25}),
                               ("nee_iso_disney", "Disney (2012)", {"metallic": 0.3, "roughness": 0.4,
                                                                    "clearcoat": 0.7, "sheen": 0.5})):
        kw2 = dict(base)
        kw2.update(iso_value=0.3, iso_color=(0.9, 0.6, 0.3), extinction=40.0, albedo=0.9, g=0.2)
        out["fbm_" + name] = SceneSpec(grid=fbm, mode="nee", interp="trilinear", iso=True, iso_brdf=brdf,
                                       brdf_params=params, **kw2)
    # spectral next event tracking with isosurfaces (path-history probabilities, chromatic medium)
    for name, brdf, params in (("nees_hist_iso", "Lambertian", None),
                               ("nees_hist_iso_cook", "Cook Torrance", {"metallic": 0.6, "specular": 0.8,
                                                                        "roughness": 0.25})):
        kw2 = dict(base)
        kw2.update(iso_value=0.3, iso_color=(0.9, 0.6, 0.3), extinction=40.0, g=0.2,
                   extinction_base=(1.0, 0.7, 0.4), albedo_rgb=(0.95, 0.8, 0.9))
        out["fbm_" + name] = SceneSpec(grid=fbm, mode="spectral_nee", sdt_prob=2, interp="trilinear", iso=True,
                                       iso_brdf=brdf, brdf_params=params, **kw2)
    # spectral delta tracking with isosurfaces: a chromatic medium around the coloured density surface
    for name, prob in {"sdt_hist_iso": 2, "sdt_max_iso": 0}.items():
        kw2 = dict(base)
        kw2.update(iso_value=0.3, iso_color=(0.9, 0.6, 0.3), extinction=40.0, g=0.2,
                   extinction_base=(1.0, 0.7, 0.4), albedo_rgb=(0.95, 0.8, 0.9))
        out["fbm_" + name] = SceneSpec(grid=fbm, mode="spectral_delta", sdt_prob=prob, interp="trilinear", iso=True,
                                       **kw2)
    # isosurfaces of the gradient magnitude (ISOSURFACE_TYPE_GRADIENT) at its upper quartile inside the cloud
    gm = gradient_magnitude(fbm)
    kw2 = dict(base)
    kw2.update(iso_value=float(np.float32(np.quantile(gm[gm > 0], 0.75))), iso_color=(0.9, 0.6, 0.3), extinction=40.0,
               albedo=0.9, g=0.2)
    out["fbm_delta_isograd"] = SceneSpec(grid=fbm, mode="delta", interp="trilinear", iso=True, iso_type="Gradient", **kw2)
    return out


def env_rotation():
    """glm::eulerAngleYXZ(0.7, -0.4, 0.25) as 9 floats, column-major (R = Ry(0.7) Rx(-0.4) Rz(0.25))."""
    def ry(a):
        return np.array([[np.cos(a), 0, np.sin(a)], [0, 1, 0], [-np.sin(a), 0, np.cos(a)]])

    def rx(a):
        return np.array([[1, 0, 0], [0, np.cos(a), -np.sin(a)], [0, np.sin(a), np.cos(a)]])

    def rz(a):
        return np.array([[np.cos(a), -np.sin(a), 0], [np.sin(a), np.cos(a), 0], [0, 0, 1]])

    m = ry(0.7) @ rx(-0.4) @ rz(0.25)
    return tuple(float(v) for v in m.T.reshape(-1).astype(np.float32))


def transfer_function_table(n=64):
    u = (np.arange(n, dtype=np.float64) + 0.5) / n
    rgba = np.stack([np.clip(1.5 * u, 0, 1), u ** 2, 0.3 * (1 - u), np.clip((u - 0.2) / 0.8, 0, 1) ** 1.5], axis=1)
    return rgba.astype(np.float32)


FIELDS = ["mode", "interp", "extinction", "albedo", "g", "width", "height", "seed_offset", "env", "linear_rgb",
          "sun_dir", "sun_intensity", "cam_pos", "cam_target", "fovy", "near", "far", "max_grid_extent", "use_ess",
          "env_intensity", "max_bounces", "ess_ref_compat", "lights", "extinction_base", "albedo_rgb", "sdt_prob",
          "emission_cap", "emission_strength", "iso", "iso_value", "iso_color", "env_rot", "tf_albedo_strength",
          "iso_brdf", "brdf_params", "iso_type", "clip_plane", "close_iso"]


def depth_map_cases():
    """Depth Blended / Depth Nearest Opaque (Clouds.glsl:367-383): the fbm cloud, delta tracking,
    nearest and trilinear lookups (deterministic: the marches consume no random numbers)."""
    fbm = bridge.fbm(24, 2, base_frequency=3.0, contrast=3.5)
    base = dict(mode="delta", extinction=120.0, albedo=0.99, g=0.85, width=W, height=H, env="default", linear_rgb=1,
                cam_pos=(0.3, 0.4, 1.4), max_grid_extent=0.5)
    return {f"fbm_depthmaps_{i}": SceneSpec(grid=fbm, interp=i, **base) for i in ("nearest", "trilinear")}


DEPTH_FRAMES = 4


def main_depth_maps():
    """tests/golden/ref_depth_maps.npz: the reference's depthBlendedImage and depthNearestOpaqueImage
    (fp32 running means, H x W x 4) after 4 frames."""
    from oracle import ref_bridge

    data, meta = {}, {}
    for name, sp in depth_map_cases().items():
        inv = camera_inv_view_proj(sp)
        sc, _ = reference_scene(sp, DEPTH_FRAMES, inv=inv)
        variant = f"depthmaps__{sp.interp}__default__linear"
        sc.render(variant)
        data[name + "__blended"] = ref_bridge.Scene.depth_feature(0, sp.height, sp.width)
        data[name + "__nearest"] = ref_bridge.Scene.depth_feature(1, sp.height, sp.width)
        data[name + "__grid"] = np.ascontiguousarray(sp.grid, np.float32)
        meta[name] = {"variant": variant, "frames": DEPTH_FRAMES,
                      **{f: (list(getattr(sp, f)) if isinstance(getattr(sp, f), tuple) else getattr(sp, f))
                         for f in FIELDS}}
        print(name, variant, float(data[name + "__blended"][..., 1].mean()), float(data[name + "__nearest"][..., 0].mean()))
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_depth_maps.npz")
    np.savez_compressed(out, meta=json.dumps(meta), **data)
    print("wrote", out, os.path.getsize(out), "bytes")


LAST_FRAMES = 4


def last_frame_cases():
    """First W / Flow / Flow Reverse / Reprojected UV (Clouds.glsl:239-246, 286-343): the fbm cloud seen
    from cam_pos, the previous view-projection that of a camera a little to the side; delta tracking and
    next event tracking, stochastic lookups."""
    fbm = bridge.fbm(24, 2, base_frequency=3.0, contrast=3.5)
    base = dict(extinction=60.0, albedo=0.99, g=0.85, width=W, height=H, env="default", linear_rgb=1,
                cam_pos=(0.3, 0.4, 1.4), max_grid_extent=0.5)
    prev = SceneSpec(grid=fbm, **dict(base, cam_pos=(0.36, 0.37, 1.41)))
    return {f"fbm_lastframe_{t}": (SceneSpec(grid=fbm, mode=t, **base), camera_view_proj(prev)) for t in ("delta", "nee")}


def main_last_frame_maps():
    """tests/golden/ref_last_frame_maps.npz: the reference's firstW, flowImage, flowReverseImage and
    reprojUVImage (H x W x 4) after LAST_FRAMES frames, with parameters.previousViewProjMatrix set."""
    from oracle import ref_bridge

    data, meta = {}, {}
    for name, (sp, prev_vp) in last_frame_cases().items():
        inv = camera_inv_view_proj(sp)
        sc, _ = reference_scene(sp, LAST_FRAMES, inv=inv)
        sc.set("prev_view_proj", prev_vp)
        variant = f"lastframe_{sp.mode}__stochastic__default__linear"
        sc.render(variant)
        for k, key in enumerate(("first_w", "flow", "flow_reverse", "reproj_uv")):
            data[f"{name}__{key}"] = ref_bridge.Scene.last_frame_feature(k, sp.height, sp.width)
        data[name + "__grid"] = np.ascontiguousarray(sp.grid, np.float32)
        data[name + "__prev_view_proj"] = np.array(prev_vp, np.float32)
        data[name + "__inv_view_proj"] = np.array(inv, np.float32)
        meta[name] = {"variant": variant, "frames": LAST_FRAMES,
                      **{f: (list(getattr(sp, f)) if isinstance(getattr(sp, f), tuple) else getattr(sp, f))
                         for f in FIELDS}}
        print(name, variant, float(np.abs(data[name + "__flow"]).mean()), float((data[name + "__reproj_uv"] >= 0).mean()))
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_last_frame_maps.npz")
    np.savez_compressed(out, meta=json.dumps(meta), **data)
    print("wrote", out, os.path.getsize(out), "bytes")


DERIV_FRAMES = 4


def main_depth_deriv_maps():
    """tests/golden/ref_depth_deriv_maps.npz: the reference's normalImage, depthNablaImage and
    depthFwidthImage (H x W x 4) after DERIV_FRAMES frames (the last-frame scenes, current camera)."""
    from oracle import ref_bridge

    data, meta = {}, {}
    for name, (sp, _) in last_frame_cases().items():
        name = name.replace("lastframe", "depthderiv")
        inv = camera_inv_view_proj(sp)
        sc, _ = reference_scene(sp, DERIV_FRAMES, inv=inv)
        variant = f"depthderiv_{sp.mode}__stochastic__default__linear"
        sc.render(variant)
        for k, key in ((4, "normal"), (5, "nabla"), (6, "fwidth")):
            data[f"{name}__{key}"] = ref_bridge.Scene.last_frame_feature(k, sp.height, sp.width)
        if sp.mode == "delta":  # the fwidth map alone (Clouds.glsl:356-364 then reads this frame's nabla)
            sc2, _ = reference_scene(sp, DERIV_FRAMES, inv=inv)
            sc2.render("depthfwidth_delta__stochastic__default__linear")
            data[f"{name}__fwidth_only"] = ref_bridge.Scene.last_frame_feature(6, sp.height, sp.width)
        data[name + "__grid"] = np.ascontiguousarray(sp.grid, np.float32)
        data[name + "__inv_view_proj"] = np.array(inv, np.float32)
        meta[name] = {"variant": variant, "frames": DERIV_FRAMES,
                      **{f: (list(getattr(sp, f)) if isinstance(getattr(sp, f), tuple) else getattr(sp, f))
                         for f in FIELDS}}
        nab = data[name + "__nabla"]
        print(name, variant, "nan fraction", float(np.isnan(nab[..., 0]).mean()),
              "mean |nabla|", float(np.nanmean(np.abs(nab[..., :2]))))
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_depth_deriv_maps.npz")
    np.savez_compressed(out, meta=json.dumps(meta), **data)
    print("wrote", out, os.path.getsize(out), "bytes")


def main():
    ref_build.build()
    data = {}
    meta = {}
    grids = []
    for name, sp in cases().items():
        inv = camera_inv_view_proj(sp)
        sc, variant = reference_scene(sp, 1, inv=inv)
        paths = sc.render(variant)[..., :3].copy()
        sc.set("num_frames", 8)
        mean8 = sc.render(variant)[..., :3].copy()
        g = np.ascontiguousarray(sp.grid, np.float32)
        key = next((k for k, a in grids if a.shape == g.shape and np.array_equal(a, g)), None)
        if key is None:
            key = f"grid{len(grids)}"
            grids.append((key, g))
            data[key] = g
        data[name + "__paths"] = paths
        data[name + "__mean8"] = mean8
        data[name + "__inv_view_proj"] = np.array(inv, np.float32)
        if sp.env == "image":
            data[name + "__env_rgba"] = np.ascontiguousarray(sp.env_rgba, np.float32)
        if sp.emission is not None:
            data[name + "__emission"] = np.ascontiguousarray(sp.emission, np.float32)
        if sp.tf is not None:
            data[name + "__tf"] = np.ascontiguousarray(sp.tf, np.float32)
        meta[name] = {"variant": variant, "grid": key, **{f: (list(getattr(sp, f)) if isinstance(getattr(sp, f), tuple)
                                                 else getattr(sp, f)) for f in FIELDS}}
        print(name, variant, float(paths.mean()))
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_paths.npz")
    np.savez_compressed(out, meta=json.dumps(meta), **data)
    print("wrote", out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "depth_maps":
        ref_build.build()
        main_depth_maps()
        sys.exit(0)
    if len(sys.argv) > 1 and sys.argv[1] == "last_frame_maps":
        ref_build.build()
        main_last_frame_maps()
        sys.exit(0)
    if len(sys.argv) > 1 and sys.argv[1] == "depth_deriv_maps":
        ref_build.build()
        main_depth_deriv_maps()
        sys.exit(0)
    main()
