"""Build recipe for the CPU oracle (test infrastructure).

* ``liboracle_vpt.so``: this project's C++ restatement of the reference shaders (vpt_oracle.cpp).
* ``_ref/``: code compiled from the reference's own sources when the reference tree is present
  (see ref_build.py); outputs only go to ``oracle/_ref``.

Compiled for the baseline x86-64 ISA (the .so travels to other hosts) with FMA contraction off so
that float operations round exactly like the CUDA core's.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle_vpt.so")
FLAGS = ["-O3", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-mtune=generic"]


def build(force: bool = False, verbose: bool = False) -> str:
    src = os.path.join(HERE, "vpt_oracle.cpp")
    hdr = os.path.join(HERE, "vpt_oracle.h")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(src), os.path.getmtime(hdr)):
        cmd = ["g++", *FLAGS, src, "-o", LIB]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    # the reference's own code for the CPU (optional: needs the reference tree; a no-op without it)
    sys.path.insert(0, os.path.dirname(HERE))
    from oracle import ref_build
    ref_build.build(force=force, verbose=verbose)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
