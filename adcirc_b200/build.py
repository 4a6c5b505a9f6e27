"""Build libadcgpu.so in-tree for sm_100a (B200).

    python -m adcirc_b200.build [--verbose]

Every translation unit is compiled with ``--fmad=false``: the FP64 path
reproduces the reference's serial arithmetic only if no multiply-add is
contracted, and the kernels are bandwidth bound so nothing is lost.
"""
from __future__ import annotations

import os
import pathlib
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "lib" / "libadcgpu.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-ffp-contract=off"]


def sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def build(verbose: bool = False, force: bool = False) -> pathlib.Path:
    srcs = sources()
    deps = srcs + sorted(CSRC.glob("*.cuh")) + [HERE.parent / "include" / "adcgpu.h"]
    if OUT.exists() and not force:
        t = OUT.stat().st_mtime
        if all(p.stat().st_mtime <= t for p in deps):
            return OUT
    OUT.parent.mkdir(parents=True, exist_ok=True)
    objdir = HERE / "lib" / "_build"
    objdir.mkdir(parents=True, exist_ok=True)
    objs = []
    for s in srcs:
        o = objdir / (s.stem + ".o")
        cmd = [NVCC, *ARCH, *FLAGS, "-rdc=false", "-c", str(s), "-o", str(o)]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {s.name}")
        if verbose and r.stderr:
            sys.stderr.write(r.stderr)
        objs.append(str(o))
    cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(OUT), *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    return OUT


if __name__ == "__main__":
    p = build(verbose="--verbose" in sys.argv, force=True)
    print(p)
