"""Build libgbgpu.so in-tree for sm_100a (nvcc, no JIT cache).

    python -m gb_b200.build        # or gb_b200.build.build()

The library is a plain shared object with a C ABI (include/gbgpu.h); it links
the CUDA runtime statically so it does not depend on which libcudart another
module of the process loaded first.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgbgpu.so")
LIFT_LIB = os.path.join(HERE, "libgblift.so")  # host-only helper of gb_b200/multimod.py
SYNTH_LIB = os.path.join(HERE, "libgbsynth.so")  # host-only generator of gb_b200/synth.py
OBJDIR = os.path.join(REPO, "_build", "gbgpu")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "--expt-relaxed-constexpr", "-I" + os.path.join(REPO, "include")]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale(obj: str, deps) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(REPO, "include", "*.h"))
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            cmd = [NVCC] + ARCH + FLAGS + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                                stderr=subprocess.STDOUT)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((src, out.decode(errors="replace")))
        elif verbose and out:
            print(out.decode(errors="replace"))
    if failed:
        msg = "\n".join(f"{s}:\n{o}" for s, o in failed)
        raise RuntimeError(f"nvcc failed:\n{msg}")
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    build_lift(verbose=verbose, force=force)
    build_synth(verbose=verbose, force=force)
    return LIB


def build_lift(verbose: bool = False, force: bool = False) -> str:
    """libgblift.so: the host-side Chinese remaindering of the multi-modular
    driver (plain C++, g++)."""
    src = os.path.join(CSRC, "lift.cpp")
    if force or _stale(LIFT_LIB, [src]):
        cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-pthread", src, "-o", LIFT_LIB]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIFT_LIB


def build_synth(verbose: bool = False, force: bool = False) -> str:
    """libgbsynth.so: the host generator of the large synthetic staircase
    matrices (plain C++, g++)."""
    src = os.path.join(CSRC, "synth.cpp")
    if force or _stale(SYNTH_LIB, [src]):
        cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-pthread", src, "-o", SYNTH_LIB]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return SYNTH_LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
