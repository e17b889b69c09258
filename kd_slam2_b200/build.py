"""Builds libkds.so (CUDA, sm_100a) and libkds_synth.so in-tree.

    python -m kd_slam2_b200.build          # or kd_slam2_b200.build.build()

The tree build, the tree operations and the alignment kernels are compiled with
-fmad=false: they round every multiply and add separately so that they reproduce the
CPU oracle bit for bit (the alignment kernels also spell their per-leaf and pose
arithmetic with explicit __fmul_rn/__fadd_rn and __dmul_rn/__dadd_rn).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
                      "-I", os.path.join(ROOT, "include"), "--expt-relaxed-constexpr"]

UNITS = [
    ("kds_tree.cu", ["-fmad=false"]),
    ("kds_build.cu", ["-fmad=false"]),
    ("kds_align.cu", ["-fmad=false"]),
    ("kds_api.cu", []),
    ("kds_serve.cu", ["-fmad=false"]),
    ("kds_factor.cu", []),
    ("kds_voxel.cu", []),
    ("kds_tracker.cu", []),
]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("command failed: " + " ".join(cmd))
    if r.stderr.strip():
        sys.stderr.write(r.stderr)


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "kds.h"))
    objs = []
    for src, extra in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if _stale(o, [s] + headers) or ptxas_info:
            cmd = [nvcc] + NVCC_COMMON + extra + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
    lib = os.path.join(HERE, "libkds.so")
    if _stale(lib, objs):
        _run([nvcc] + ARCH + ["-shared", "-o", lib] + objs + ["-lpthread"])
    synth_src = os.path.join(CSRC, "kds_synth.cpp")
    synth = os.path.join(HERE, "libkds_synth.so")
    if _stale(synth, [synth_src]):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", synth, synth_src, "-lpthread"])
    return lib


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv)
    print("built", os.path.join(HERE, "libkds.so"))
