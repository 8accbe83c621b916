"""Build libpfb200.so in-tree with nvcc for sm_100a.

    python -m photonfdtd_b200.build [--debug]

The library lands next to this file, where photonfdtd_b200._native loads it.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def build(debug: bool = False, verbose: bool = False) -> str:
    out = os.path.join(HERE, "libpfb200.so")
    src = [os.path.join(CSRC, f) for f in ("engine.cu", "flux_noalloc.cu", "batch2d.cu",
                                           "surrogate.cu", "smoothing.cu", "design.cu",
                                           "modesolver.cu")]
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + \
        [os.path.join(os.path.dirname(HERE), "include", "pfb200.h")]
    if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps):
        return out
    cmd = [nvcc(), *ARCH, "-lineinfo", "-std=c++17", "-O3", "-Xcompiler", "-fPIC", "-shared",
           "-o", out + ".tmp", *src]
    if debug:
        cmd.insert(1, "-DPF_CHECK=1")
    if verbose:
        cmd.append("-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    print(build(debug="--debug" in sys.argv, verbose="-v" in sys.argv))
