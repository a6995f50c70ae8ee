"""Builds the reference's own code for the CPU (TEST INFRASTRUCTURE ONLY; outputs in oracle/_ref/).

1. ``libref_vpt.so``: the reference tracer shaders (Data/Shaders/VPT/Clouds.glsl and everything it
   includes) compiled as C++ on top of ``ref_shim.h``.  The GLSL text is rewritten mechanically
   (comments dropped, ``in/out/inout`` parameter qualifiers -> C++ values/references, float
   literals -> ``f`` suffix, the RNG state made thread-local, ``main`` renamed); nothing else is
   changed.  One variant per (tracker, interpolation, environment, colour space) define set, as the
   reference's loadShader() would select (VolumetricPathTracingPass.cpp:1558-1782).
3. ``libref_pnanovdb.so``: Data/Shaders/VPT/PNanoVDB.glsl compiled in its own C99 mode
   (-DPNANOVDB_C -DPNANOVDB_HDDA) with ``ref_pnanovdb_driver.c``: the reference's NanoVDB read
   accessor, map and HDDA.
4. ``libref_nanovdb_builder.so``: the reference's vendored NanoVDB GridBuilder
   (src/nanovdb/util/GridBuilder.h) driven as CloudData::getSparseDensityField drives it
   (``ref_nanovdb_builder.cpp``).
6. ``libref_kpn.so``: the reference's PyTorch KPN extension (modules/kpn_module/src/Kernel.cu with
   perPixelKernel.cpp, CUDA for sm_100a) and ``ref_kpn_driver.cpp``; GPU tests load it with
   torch.ops.load_library and compare the core's KPN kernels with the reference's.
5. ``libref_supervoxel.so``: the reference's supervoxel grid builders and density-field normalisation
   (src/PathTracer/SuperVoxelGrid.cpp, src/DensityField.cpp) compiled unmodified against the small
   glm / sgl / Vulkan stand-ins of ``ref_cpp_shim/`` (``ref_supervoxel_driver.cpp``).

The reference tree is read from $VPT_REFERENCE_ROOT, else from a directory named ``reference`` beside
this repository's root; when it is absent the build is skipped (the prebuilt libraries under
oracle/_ref are used as they are).
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
GEN = os.path.join(OUT, "gen")
REF = os.environ.get("VPT_REFERENCE_ROOT") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
SHADERS = os.path.join(REF, "Data", "Shaders", "VPT")
BRDFS = os.path.join(REF, "Data", "Shaders", "BRDF")

# (name, defines) of the tracer variants; the C driver indexes them in this order.
TRACKERS = {
    "delta": ["USE_DELTA_TRACKING"],
    "ratio": ["USE_RATIO_TRACKING"],
    "decomposition": ["USE_DECOMPOSITION_TRACKING"],
    "rrt": ["USE_RESIDUAL_RATIO_TRACKING"],
    "nee": ["USE_NEXT_EVENT_TRACKING"],
    "nee_ess": ["USE_NEXT_EVENT_TRACKING", "USE_OCCUPANCY_GRID"],
}
INTERPS = {"nearest": "GRID_INTERPOLATION_NEAREST", "stochastic": "GRID_INTERPOLATION_STOCHASTIC",
           "trilinear": "GRID_INTERPOLATION_TRILINEAR"}
# environment x colour space combinations that are built
ENVS = {
    "default__srgb": ["USE_ENVIRONMENT_MAP_DEFAULT"],
    "default__linear": ["USE_ENVIRONMENT_MAP_DEFAULT", "USE_LINEAR_RGB"],
    "black__linear": ["USE_ENVIRONMENT_MAP_BLACK", "USE_LINEAR_RGB"],
    "single__linear": ["USE_ENVIRONMENT_MAP_SINGLE_COLOR", "USE_LINEAR_RGB"],
    "image__linear": ["USE_ENVIRONMENT_MAP_IMAGE", "ENV_MAP_IMAGE_USES_LINEAR_RGB", "USE_LINEAR_RGB"],
}


# NEE with lights (NUM_LIGHTS > 0): stochastic lookups, default and black environments
LIGHT_VARIANTS = {"nee_l1": 1, "nee_l2": 2}
# spectral trackers, one variant per collision-probability mode (VolumetricPathTracingPass.cpp:1566-1584)
SDT_PROB = {"max": "MAX_BASED_PROBABILITY", "avg": "AVG_BASED_PROBABILITY",
            "hist": "PATH_HISTORY_AVG_BASED_PROBABILITY"}
SPECTRAL = {"sdt": "USE_SPECTRAL_DELTA_TRACKING", "nees": "USE_NEXT_EVENT_TRACKING_SPECTRAL"}
# the Depth Blended / Depth Nearest Opaque feature maps (Clouds.glsl:367-383), deterministic lookups
DEPTH_MAPS = ["WRITE_DEPTH_BLENDED_MAP", "WRITE_DEPTH_NEAREST_OPAQUE_MAP"]
# the maps overwritten every frame (Clouds.glsl:239-246, 286-343)
LAST_FRAME_MAPS = ["WRITE_FIRST_W_MAP", "WRITE_FLOW_MAP", "WRITE_FLOW_REVERSE_MAP", "WRITE_REPROJ_UV_MAP"]
# the normal map's running mean and the depth derivative maps computed from it (Clouds.glsl:258-297, 344-364)
DEPTH_DERIV_MAPS = ["WRITE_NORMAL_MAP", "WRITE_DEPTH_NABLA_MAP", "WRITE_DEPTH_FWIDTH_MAP"]
ISO = ["USE_ISOSURFACES", "NUM_ISOSURFACE_SUBDIVISIONS=2", "SURFACE_BRDF_LAMBERTIAN", "ISOSURFACE_TYPE_DENSITY"]


def variants():
    """(name, defines, NUM_LIGHTS)"""
    out = []
    for t, tdefs in TRACKERS.items():
        for i, idef in INTERPS.items():
            for e, edefs in ENVS.items():
                out.append((f"{t}__{i}__{e}", tdefs + [idef] + edefs, 0))
    for t, n in LIGHT_VARIANTS.items():
        for e in ("default__linear", "black__linear"):
            out.append((f"{t}__stochastic__{e}", TRACKERS["nee"] + [INTERPS["stochastic"]] + ENVS[e], n))
    for t, tdef in SPECTRAL.items():
        for p, pdef in SDT_PROB.items():
            for i in ("stochastic", "trilinear"):
                out.append((f"{t}_{p}__{i}__default__linear", [tdef, pdef, INTERPS[i]] + ENVS["default__linear"], 0))
    for i in ("nearest", "trilinear"):
        out.append((f"depthmaps__{i}__default__linear", TRACKERS["delta"] + [INTERPS[i]] + ENVS["default__linear"]
                    + DEPTH_MAPS, 0))
    for t in ("delta", "nee"):
        out.append((f"lastframe_{t}__stochastic__default__linear", TRACKERS[t] + [INTERPS["stochastic"]]
                    + ENVS["default__linear"] + LAST_FRAME_MAPS, 0))
        out.append((f"depthderiv_{t}__stochastic__default__linear", TRACKERS[t] + [INTERPS["stochastic"]]
                    + ENVS["default__linear"] + DEPTH_DERIV_MAPS, 0))
    # Depth (fwidth) without the nabla map: it then averages each frame's own nabla
    out.append(("depthfwidth_delta__stochastic__default__linear", TRACKERS["delta"] + [INTERPS["stochastic"]]
                + ENVS["default__linear"] + ["WRITE_NORMAL_MAP", "WRITE_DEPTH_FWIDTH_MAP"], 0))
    # emission grid (USE_EMISSION) with next event tracking, grey and spectral
    for i in ("stochastic", "trilinear"):
        out.append((f"nee_emission__{i}__default__linear", TRACKERS["nee"] + [INTERPS[i]] + ENVS["default__linear"]
                    + ["USE_EMISSION"], 0))
    out.append(("nees_hist_emission__stochastic__default__linear",
                [SPECTRAL["nees"], SDT_PROB["hist"], INTERPS["stochastic"], "USE_EMISSION"] + ENVS["default__linear"], 0))
    # transfer-function appearance (USE_TRANSFER_FUNCTION): density = TF(value).a, absorption emission
    for t in ("delta", "nee"):
        for i in ("stochastic", "trilinear"):
            out.append((f"{t}_tf__{i}__default__linear", TRACKERS[t] + [INTERPS[i]] + ENVS["default__linear"]
                        + ["USE_TRANSFER_FUNCTION"], 0))
    for t, tdef in SPECTRAL.items():
        out.append((f"{t}_hist_tf__stochastic__default__linear",
                    [tdef, SDT_PROB["hist"], INTERPS["stochastic"], "USE_TRANSFER_FUNCTION"] + ENVS["default__linear"], 0))
        # the transfer function's colour as scattering albedo (setTfScatteringAlbedoStrength > 0)
        out.append((f"{t}_hist_tf_albedo__stochastic__default__linear",
                    [tdef, SDT_PROB["hist"], INTERPS["stochastic"], "USE_TRANSFER_FUNCTION",
                     "USE_TRANSFER_FUNCTION_SCATTERING_ALBEDO"] + ENVS["default__linear"], 0))
    # environment-image rotation (USE_ENV_MAP_ROTATION, VolumetricPathTracingPass.cpp:1708-1710)
    for t in ("delta", "nee"):
        out.append((f"{t}_rot__stochastic__image__linear", TRACKERS[t] + [INTERPS["stochastic"]] + ENVS["image__linear"]
                    + ["USE_ENV_MAP_ROTATION"], 0))
    # isosurfaces inside the volume (USE_ISOSURFACES; VolumetricPathTracingPass.cpp:1737-1768): density
    # isosurfaces, Lambertian surfaces, 2 subdivisions per free-flight segment, trilinear lookups forced
    # (VolumetricPathTracingPass.cpp:117-120)
    out.append(("delta_iso__trilinear__default__linear", TRACKERS["delta"] + [INTERPS["trilinear"]]
                + ENVS["default__linear"] + ISO, 0))
    # the Blinn-Phong, Cook-Torrance, Disney (2012) and constant-lighting surface BRDFs
    # (Data/Shaders/BRDF/BlinnPhong.glsl, CookTorrance.glsl, Disney2012.glsl, ConstantLighting.glsl)
    for tag, define in (("blinn", "SURFACE_BRDF_BLINN_PHONG"), ("ambient", "SURFACE_BRDF_AMBIENT"),
                        ("cook", "SURFACE_BRDF_COOK_TORRANCE"), ("disney", "SURFACE_BRDF_DISNEY")):
        out.append((f"delta_iso_{tag}__trilinear__default__linear", TRACKERS["delta"] + [INTERPS["trilinear"]]
                    + ENVS["default__linear"] + [define if d == "SURFACE_BRDF_LAMBERTIAN" else d for d in ISO], 0))
    # the clip plane (USE_CLIP_PLANE, VolumetricPathTracingPass.cpp:1774-1776): delta and next event tracking
    for t in ("delta", "nee"):
        out.append((f"{t}_clip__stochastic__default__linear", TRACKERS[t] + [INTERPS["stochastic"]]
                    + ENVS["default__linear"] + ["USE_CLIP_PLANE"], 0))
    out.append(("sdt_hist_clip__stochastic__default__linear", [SPECTRAL["sdt"], SDT_PROB["hist"],
                INTERPS["stochastic"]] + ENVS["default__linear"] + ["USE_CLIP_PLANE"], 0))
    # isosurfaces closed by the box and the clip plane (CLOSE_ISOSURFACES, VolumetricPathTracingPass.cpp:1777-1779)
    out.append(("delta_iso_clip_close__trilinear__default__linear", TRACKERS["delta"] + [INTERPS["trilinear"]]
                + ENVS["default__linear"] + ISO + ["USE_CLIP_PLANE", "CLOSE_ISOSURFACES"], 0))
    out.append(("nee_iso_clip_close__trilinear__default__linear", TRACKERS["nee"] + [INTERPS["trilinear"]]
                + ENVS["default__linear"] + ISO + ["USE_ISOSURFACE_NEE", "USE_CLIP_PLANE", "CLOSE_ISOSURFACES"], 0))
    # next event tracking with isosurfaces (USE_ISOSURFACE_NEE, VolumetricPathTracingPass.cpp:1761-1763) for
    # every surface BRDF
    for tag, define in (("", "SURFACE_BRDF_LAMBERTIAN"), ("_blinn", "SURFACE_BRDF_BLINN_PHONG"),
                        ("_ambient", "SURFACE_BRDF_AMBIENT"), ("_cook", "SURFACE_BRDF_COOK_TORRANCE"),
                        ("_disney", "SURFACE_BRDF_DISNEY")):
        out.append((f"nee_iso{tag}__trilinear__default__linear", TRACKERS["nee"] + [INTERPS["trilinear"]]
                    + ENVS["default__linear"] + [define if d == "SURFACE_BRDF_LAMBERTIAN" else d for d in ISO]
                    + ["USE_ISOSURFACE_NEE"], 0))
    # spectral next event tracking with isosurfaces and surface next-event estimation (Lambertian, Cook-Torrance)
    for tag, define in (("", "SURFACE_BRDF_LAMBERTIAN"), ("_cook", "SURFACE_BRDF_COOK_TORRANCE")):
        out.append((f"nees_hist_iso{tag}__trilinear__default__linear", [SPECTRAL["nees"], SDT_PROB["hist"],
                    INTERPS["trilinear"]] + ENVS["default__linear"]
                    + [define if d == "SURFACE_BRDF_LAMBERTIAN" else d for d in ISO] + ["USE_ISOSURFACE_NEE"], 0))
    # spectral delta tracking with isosurfaces (DeltaTracking.glsl:37-63), path-history and max probabilities
    for p in ("hist", "max"):
        out.append((f"sdt_{p}_iso__trilinear__default__linear", [SPECTRAL["sdt"], SDT_PROB[p], INTERPS["trilinear"]]
                    + ENVS["default__linear"] + ISO, 0))
    # isosurfaces of the gradient magnitude (ISOSURFACE_TYPE_GRADIENT: gradientImage, VptUtils.glsl:687-707)
    out.append(("delta_isograd__trilinear__default__linear", TRACKERS["delta"] + [INTERPS["trilinear"]]
                + ENVS["default__linear"] + ["ISOSURFACE_TYPE_GRADIENT" if d == "ISOSURFACE_TYPE_DENSITY" else d
                                             for d in ISO], 0))
    return out


FLOAT_LIT = re.compile(r"(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)(?![\w.])")
QUAL_REF = re.compile(r"\b(?:inout|out)\s+(\w+)\s+(\w+)")
QUAL_IN = re.compile(r"\bin\s+(\w+)\s+(\w+)")
MULTI_RANDOM = re.compile(r"\b(vec[234])\(((?:[^()]|\(\))*random\(\)(?:[^()]|\(\))*random\(\)(?:[^()]|\(\))*)\)")


def strip_comments(text: str) -> str:
    text = re.sub(r"/\*.*?\*/", lambda m: "\n" * m.group(0).count("\n"), text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def transform(text: str) -> str:
    text = strip_comments(text)
    lines = []
    for ln in text.split("\n"):
        s = ln.strip()
        if s.startswith("--") or s.startswith("#version") or s.startswith("#extension"):
            lines.append("")
            continue
        m = re.match(r'\s*#include\s+"([\w.]+)"', ln)
        if m:
            name = m.group(1)
            lines.append(f'#include "{name}.inc"' if name != "VptHeader.glsl" else "")
            continue
        if s.startswith("#define"):
            lines.append(FLOAT_LIT.sub(lambda m: m.group(1) + "f", ln))
            continue
        if s.startswith("#"):
            lines.append(ln)
            continue
        ln = QUAL_REF.sub(r"\1& \2", ln)
        ln = QUAL_IN.sub(r"\1 \2", ln)
        ln = FLOAT_LIT.sub(lambda m: m.group(1) + "f", ln)
        ln = re.sub(r"^uvec4 rngState", "thread_local uvec4 rngState", ln)
        # GLSL evaluates constructor arguments left to right; C++ does so only in braced lists.
        ln = MULTI_RANDOM.sub(lambda m: m.group(1) + "{" + m.group(2) + "}", ln)
        lines.append(ln)
    return "\n".join(lines)


UNIFORM_BLOCK = re.compile(r"layout\s*\([^)]*\)\s*uniform\s+\w+\s*\{(.*?)\}\s*;", re.S)
UNIFORM_VAR = re.compile(r"layout\s*\([^)]*\)\s*uniform\s+(?:writeonly\s+|readonly\s+)?(\w+)\s+(\w+)\s*;")
LOCAL_SIZE = re.compile(r"layout\s*\([^)]*\)\s*in\s*;")


def image_shader_section(path: str, section: str) -> str:
    """One ``-- <section>`` stage of a shader file, with its resource declarations turned into plain
    declarations: uniform blocks lose their wrapper (members become variables), samplers and images
    become variables, the work-group size line and ``shared`` qualifiers are dropped; then the
    transform of the tracer shaders."""
    with open(path, encoding="utf-8") as fh:
        text = fh.read()
    parts = re.split(r"^-- (.+)$", text, flags=re.M)
    body = dict(zip(parts[1::2], parts[2::2]))[section]
    body = strip_comments(body)
    body = UNIFORM_BLOCK.sub(lambda m: m.group(1), body)
    body = UNIFORM_VAR.sub(lambda m: f"{m.group(1)} {m.group(2)};", body)
    body = LOCAL_SIZE.sub("", body)
    body = re.sub(r"^\s*shared\s+", "", body, flags=re.M)
    # swizzles that name the whole vector: .rgba of a vec4, .rg of a vec2
    body = body.replace(".rgba", "")
    vec2_names = sorted(set(re.findall(r"\bvec2\s+(\w+)", body)))
    if vec2_names:
        body = re.sub(r"\b(" + "|".join(vec2_names) + r")\.rg\b", r"\1", body)
    return transform(body)


def build_image_shaders(force=False, verbose=False) -> None:
    """libref_image.so: OctahedralMapper.glsl, the compute stage of EAWDenoise.glsl and the three compute
    stages of SVGF.glsl on the CPU (ref_image_driver.cpp)."""
    drv = os.path.join(HERE, "ref_image_driver.cpp")
    shim = os.path.join(HERE, "ref_shim.h")
    lib = os.path.join(OUT, "libref_image.so")
    if not _stale(lib, [drv, shim, __file__], force):
        return
    gen = os.path.join(GEN, "img")
    os.makedirs(gen, exist_ok=True)
    den = os.path.join(REF, "Data", "Shaders", "Denoiser")
    svgf = os.path.join(den, "SVGF", "SVGF.glsl")
    for src, section, name in (
            (os.path.join(SHADERS, "OctahedralMapper.glsl"), "Compute", "OctahedralMapper.compute.inc"),
            (os.path.join(den, "EAWDenoise.glsl"), "Compute", "EAWDenoise.compute.inc"),
            (svgf, "Compute-Reproject", "SVGF.reproject.inc"),
            (svgf, "Compute-Filter-Moments", "SVGF.filter_moments.inc"),
            (svgf, "Compute-ATrous", "SVGF.atrous.inc")):
        with open(os.path.join(gen, name), "w") as fh:
            fh.write(image_shader_section(src, section))
    with open(os.path.join(den, "SVGF", "svgf_common.glsl"), encoding="utf-8") as fi, \
            open(os.path.join(gen, "svgf_common.glsl.inc"), "w") as fo:
        fo.write(transform(fi.read()))
    _run(["g++", "-O2", "-std=c++20", "-fPIC", "-shared", "-ffp-contract=off", "-w", "-I", gen, "-I", HERE, "-o", lib,
          drv], verbose)


def generate() -> None:
    os.makedirs(GEN, exist_ok=True)
    # the tracer shaders and the surface BRDFs (Data/Shaders/BRDF, included by the isosurface code)
    for d in (SHADERS, BRDFS):
        for f in os.listdir(d):
            if f.endswith(".glsl"):
                with open(os.path.join(d, f), encoding="utf-8") as fh:
                    text = fh.read()
                with open(os.path.join(GEN, f + ".inc"), "w") as fh:
                    fh.write(transform(text))


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr[-6000:]}")


def build_tracer(force=False, verbose=False) -> str:
    lib = os.path.join(OUT, "libref_vpt.so")
    driver = os.path.join(HERE, "ref_driver.cpp")
    shim = os.path.join(HERE, "ref_shim.h")
    if not force and os.path.exists(lib) and os.path.getmtime(lib) > max(os.path.getmtime(driver),
                                                                         os.path.getmtime(shim),
                                                                         os.path.getmtime(__file__)):
        return lib
    generate()
    objs, jobs = [], []
    vs = variants()
    flags = ["g++", "-O2", "-std=c++20", "-fPIC", "-fopenmp", "-ffp-contract=off", "-w", "-I", GEN, "-I", HERE]
    for idx, (name, defs, nlights) in enumerate(vs):
        obj = os.path.join(GEN, f"v_{name}.o")
        objs.append(obj)
        dflags = [f"-D{d}" for d in defs] + [f"-DREF_VARIANT_NS=v_{name}", f"-DNUM_LIGHTS={nlights}",
                                             "-DCUSTOM_SEED_OFFSET=ref_seed_offset", "-DREF_VARIANT_BODY"]
        jobs.append(flags + dflags + ["-c", driver, "-o", obj])
    reg = os.path.join(GEN, "registry.cpp")
    with open(reg, "w") as fh:
        fh.write('#include "ref_shim.h"\n#include "ref_driver_api.h"\n')
        for name, _, _ in vs:
            fh.write(f"namespace glslref {{ namespace v_{name} {{ void run_pixel(int x, int y); }} }}\n")
        fh.write("const RefVariant ref_variants[] = {\n")
        for name, _, _ in vs:
            fh.write(f'    {{"{name}", &glslref::v_{name}::run_pixel}},\n')
        fh.write("};\nconst int ref_num_variants = %d;\n" % len(vs))
    jobs.append(flags + ["-c", reg, "-o", os.path.join(GEN, "registry.o")])
    jobs.append(flags + ["-DREF_DRIVER_COMMON", "-c", driver, "-o", os.path.join(GEN, "driver_common.o")])
    objs += [os.path.join(GEN, "registry.o"), os.path.join(GEN, "driver_common.o")]
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        list(ex.map(lambda c: _run(c, verbose), jobs))
    _run(["g++", "-shared", "-fopenmp", "-o", lib] + objs, verbose)
    return lib


def _stale(lib, deps, force):
    return force or not os.path.exists(lib) or os.path.getmtime(lib) < max(os.path.getmtime(d) for d in deps)


def build_nanovdb(force=False, verbose=False) -> None:
    drv = os.path.join(HERE, "ref_pnanovdb_driver.c")
    lib = os.path.join(OUT, "libref_pnanovdb.so")
    if _stale(lib, [drv, __file__], force):
        _run(["gcc", "-O2", "-std=c99", "-fPIC", "-shared", "-ffp-contract=off", "-w", "-I", SHADERS, "-o", lib, drv,
              "-lm"], verbose)
    src = os.path.join(HERE, "ref_nanovdb_builder.cpp")
    lib = os.path.join(OUT, "libref_nanovdb_builder.so")
    if _stale(lib, [src, __file__], force):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-w", "-I", os.path.join(REF, "src"), "-o", lib, src,
              "-lpthread"], verbose)


def build_supervoxel(force=False, verbose=False) -> None:
    """libref_supervoxel.so: src/PathTracer/SuperVoxelGrid.cpp and src/DensityField.cpp copied unmodified
    into oracle/_ref/gen/cpp (their quoted includes then resolve to oracle/ref_cpp_shim) and compiled
    with ref_supervoxel_driver.cpp."""
    srcs = [os.path.join(REF, "src", "PathTracer", "SuperVoxelGrid.cpp"),
            os.path.join(REF, "src", "PathTracer", "SuperVoxelGrid.hpp"),
            os.path.join(REF, "src", "DensityField.cpp"), os.path.join(REF, "src", "DensityField.hpp")]
    drv = os.path.join(HERE, "ref_supervoxel_driver.cpp")
    shim = os.path.join(HERE, "ref_cpp_shim")
    lib = os.path.join(OUT, "libref_supervoxel.so")
    if not _stale(lib, [drv, os.path.join(shim, "ref_cpp_shim.h"), __file__], force):
        return
    gen = os.path.join(GEN, "cpp")
    os.makedirs(gen, exist_ok=True)
    for src in srcs:
        with open(src, "rb") as fi, open(os.path.join(gen, os.path.basename(src)), "wb") as fo:
            fo.write(fi.read())
    _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-w", "-I", shim, "-I", gen, "-o", lib,
          os.path.join(gen, "SuperVoxelGrid.cpp"), os.path.join(gen, "DensityField.cpp"), drv], verbose)


def build_kpn(force=False, verbose=False) -> None:
    """libref_kpn.so: the reference's PyTorch KPN extension (modules/kpn_module/src/Kernel.cu and
    perPixelKernel.cpp, unmodified; CUDA kernels for sm_100a) with ref_kpn_driver.cpp.  Loaded with
    torch.ops.load_library on a GPU, it provides torch.ops.per_pixel_kernel.forward and
    torch.ops.ref_kpn.inv_iter_base."""
    import torch

    src = os.path.join(REF, "modules", "kpn_module", "src")
    drv = os.path.join(HERE, "ref_kpn_driver.cpp")
    lib = os.path.join(OUT, "libref_kpn.so")
    if not _stale(lib, [drv, __file__], force):
        return
    tdir = os.path.dirname(torch.__file__)
    inc = ["-I", os.path.join(tdir, "include"), "-I", os.path.join(tdir, "include", "torch", "csrc", "api", "include"),
           "-I", src, "-I", "/usr/local/cuda/include"]
    defs = ["-DKPN_MODULE_OP_API=", f"-D_GLIBCXX_USE_CXX11_ABI={int(torch._C._GLIBCXX_USE_CXX11_ABI)}"]
    gen = os.path.join(GEN, "kpn")
    os.makedirs(gen, exist_ok=True)
    objs = [os.path.join(gen, n) for n in ("Kernel.o", "perPixelKernel.o", "driver.o")]
    nvcc = "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else "nvcc"
    jobs = [[nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17", "-Xcompiler", "-fPIC", "-w",
             *defs, *inc, "-c", os.path.join(src, "Kernel.cu"), "-o", objs[0]],
            ["g++", "-O2", "-std=c++17", "-fPIC", "-w", *defs, *inc, "-c", os.path.join(src, "perPixelKernel.cpp"),
             "-o", objs[1]],
            ["g++", "-O2", "-std=c++17", "-fPIC", "-w", *defs, *inc, "-c", drv, "-o", objs[2]]]
    with ThreadPoolExecutor(max_workers=3) as ex:
        list(ex.map(lambda c: _run(c, verbose), jobs))
    tlib = os.path.join(tdir, "lib")
    _run(["g++", "-shared", "-o", lib, *objs, "-L", tlib, "-Wl,-rpath," + tlib, "-ltorch", "-ltorch_cpu", "-ltorch_cuda",
          "-lc10", "-lc10_cuda", "-L", "/usr/local/cuda/lib64", "-lcudart"], verbose)


def build(force=False, verbose=False) -> None:
    if not os.path.isdir(SHADERS):
        return
    os.makedirs(OUT, exist_ok=True)
    build_tracer(force, verbose)
    build_nanovdb(force, verbose)
    build_supervoxel(force, verbose)
    build_image_shaders(force, verbose)
    build_kpn(force, verbose)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
