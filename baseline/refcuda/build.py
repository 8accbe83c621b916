"""Compile the reference's own CUDA stepping kernels for sm_100a.

    python -m baseline.refcuda.build [REFERENCE_ROOT]

The reference keeps its Yee+CPML kernels as CUDA C source text inside
rust/src/cuda.rs (the KERNEL_SRC raw string, compiled at run time by NVRTC
with -DREAL=float|double). This recipe reads that text from the reference
tree (located by baseline.locate: argument, PHOTONFDTD_REFERENCE, or a
``reference`` directory beside the repository), writes it to a temporary directory outside
the repository, and compiles it together with this project's host harness
(launch.cu) into baseline/_ref/librefcuda_f32.so and librefcuda_f64.so,
which are git-ignored. Nothing is built when the reference tree is absent.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(os.path.dirname(HERE), "_ref")
START = 'const KERNEL_SRC: &str = r#"'
END = '"#;'


def kernel_source(ref_root: str) -> str:
    with open(os.path.join(ref_root, "rust", "src", "cuda.rs")) as f:
        text = f.read()
    i = text.index(START) + len(START)
    return text[i:text.index(END, i)]


def build(ref_root: str = None, force: bool = False) -> list:
    from baseline.locate import reference_root
    ref_root = reference_root(ref_root)
    if ref_root is None:
        return []
    src_file = os.path.join(ref_root, "rust", "src", "cuda.rs")
    if not os.path.exists(src_file):
        return []
    os.makedirs(OUT, exist_ok=True)
    outs = [os.path.join(OUT, f"librefcuda_{tag}.so") for tag in ("f32", "f64")]
    deps = [src_file, os.path.join(HERE, "launch.cu"), os.path.abspath(__file__)]
    if not force and all(os.path.exists(o) and
                         all(os.path.getmtime(o) >= os.path.getmtime(d) for d in deps)
                         for o in outs):
        return outs
    from photonfdtd_b200.build import ARCH, nvcc
    tmp = tempfile.mkdtemp(prefix="refcuda_")
    try:
        kpath = os.path.join(tmp, "ref_kernels.cuh")
        with open(kpath, "w") as f:
            f.write(kernel_source(ref_root))
        for real, out in zip(("float", "double"), outs):
            cmd = [nvcc(), *ARCH, "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
                   f"-DREAL={real}", f'-DREF_KERNEL_SRC="{kpath}"',
                   os.path.join(HERE, "launch.cu"), "-o", out + ".tmp"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
            os.replace(out + ".tmp", out)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return outs


if __name__ == "__main__":
    print(build(*(sys.argv[1:2] or []), force=True))
