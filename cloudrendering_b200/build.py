"""Builds the CUDA core ``libvpt_b200.so`` in-tree with nvcc for sm_100a.

Run ``python -m cloudrendering_b200.build`` (or ``__graft_entry__.build()``).  Each ``.cu`` file of
``csrc/`` is compiled in parallel; objects go to ``cloudrendering_b200/_build/`` and the shared library
next to this file, where ``cloudrendering_b200._lib`` loads it.  The CUDA runtime is linked statically,
so the library only needs the NVIDIA driver at run time.

A second library, ``libvpt_b200_dr.so``, is the same core with the tracer's transcendental functions
evaluated in double precision and rounded once to float and without FMA contraction (``-DVPT_DOUBLE_ROUNDED_MATH`` on
the tracer units ``vpt_kernels.cu`` and ``vpt_trace_*.cu``).  The parity tests use it to compare paths one by one with the CPU oracle in the
same mode; the default library is the product.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libvpt_b200.so")
LIB_DR = os.path.join(HERE, "libvpt_b200_dr.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC]
# The tracer is compiled without FMA contraction so that its arithmetic matches the CPU oracle
# operation by operation (see the conventions at the top of vpt_device.cuh).
NO_FMA = {"vpt_kpn.cu", "vpt_denoise.cu"}
# The product's per-family tracer units use the special-function unit's log / exp / sin / cos / pow
# and approximate division and square root (VPT_FAST_MATH in vpt_device.cuh).
FAST_MATH = True


def _is_tracer(src: str) -> bool:
    """The tracer's units: the launchers and the per-family kernel instantiations (vpt_trace_*.cu)."""
    return src == "vpt_kernels.cu" or src.startswith("vpt_trace_")


def _per_file(src: str, double_rounded: bool = False) -> list[str]:
    """The product's per-family kernel units (vpt_trace_*.cu) are compiled with FMA contraction (3 %
    faster on the headline launch, A/B on one B200: 789 vs 763 M path samples/s); the parity build
    (double_rounded) keeps every multiply and add separate, operation for operation like the CPU
    oracle.  vpt_kernels.cu (grid generators, environment pyramid, film readout) never contracts: its
    outputs are bit-exact against the oracle and the reference's shaders in both builds."""
    if src in NO_FMA or src == "vpt_kernels.cu" or (double_rounded and _is_tracer(src)):
        return ["--fmad=false"]
    if FAST_MATH and src.startswith("vpt_trace_"):
        return ["-DVPT_FAST_MATH", "--prec-div=false", "--prec-sqrt=false"]
    return []


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _sources() -> list[str]:
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _needs_rebuild(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "vpt_b200.h"))
    jobs = []
    objs, objs_dr = [], []

    def add(src, obj, extra):
        deps = [os.path.join(CSRC, src)] + headers
        if force or _needs_rebuild(obj, deps + [__file__]):
            jobs.append([nvcc, *ARCH, *COMMON, *_per_file(src, "-DVPT_DOUBLE_ROUNDED_MATH" in extra), *extra, "-c",
                         os.path.join(CSRC, src), "-o", obj])

    for src in _sources():
        obj = os.path.join(BUILD, src[:-3] + ".o")
        add(src, obj, [])
        objs.append(obj)
        if _is_tracer(src):  # the sources that hold the tracer's transcendental calls (built twice)
            obj_dr = os.path.join(BUILD, src[:-3] + "_dr.o")
            add(src, obj_dr, ["-DVPT_DOUBLE_ROUNDED_MATH"])
            objs_dr.append(obj_dr)
        else:
            objs_dr.append(obj)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed ({' '.join(cmd)}):\n{r.stdout}\n{r.stderr}")
        return r

    if jobs:
        with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            list(ex.map(run, jobs))
    for lib, lib_objs in ((LIB, objs), (LIB_DR, objs_dr)):
        if jobs or not os.path.exists(lib) or force:
            run([nvcc, *ARCH, "-shared", "-o", lib, *lib_objs])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="--force" in sys.argv))
