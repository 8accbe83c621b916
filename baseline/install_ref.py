"""Install the reference photonfdtd package into baseline/_ref.

    python -m baseline.install_ref [REFERENCE_ROOT]

The offline `pip install --no-index --no-build-isolation --find-links
<wheelhouse> --target baseline/_ref <reference>` cannot build the reference:
its build backend (hatchling) is not in the wheelhouse, and `--no-deps` does
not help because the backend itself is missing. The reference is a pure
Python package whose wheel holds exactly src/photonfdtd/*.py (pyproject.toml
[tool.hatch.build.targets.wheel] packages = ["src/photonfdtd"], compiled
extensions excluded), so this recipe places that same content where pip
would: baseline/_ref/photonfdtd/. baseline/_ref is git-ignored (the reference
is not part of this repository's history) but travels with the working tree,
so the reference's own NumPy and Numba paths can run wherever the benchmark
runs. The sources are copied unmodified; a manifest records where they came
from.
"""
from __future__ import annotations

import json
import os
import shutil
import sys

from baseline.locate import INSTALL_DIR, reference_root


def install(ref_root: str = None, force: bool = False) -> str:
    root = reference_root(ref_root)
    if root is None:
        return ""
    src = os.path.join(root, "src", "photonfdtd")
    dst = os.path.join(INSTALL_DIR, "photonfdtd")
    files = sorted(f for f in os.listdir(src) if f.endswith(".py"))
    if not force and os.path.isdir(dst) and all(
            os.path.exists(os.path.join(dst, f)) and
            os.path.getmtime(os.path.join(dst, f)) >= os.path.getmtime(os.path.join(src, f))
            for f in files):
        return dst
    tmp = dst + ".tmp"
    shutil.rmtree(tmp, ignore_errors=True)
    os.makedirs(tmp)
    for f in files:
        shutil.copy2(os.path.join(src, f), os.path.join(tmp, f))
    shutil.rmtree(dst, ignore_errors=True)
    os.replace(tmp, dst)
    version = None
    with open(os.path.join(root, "pyproject.toml")) as f:
        for line in f:
            if line.startswith("version"):
                version = line.split("=", 1)[1].strip().strip('"')
                break
    with open(os.path.join(INSTALL_DIR, "photonfdtd.manifest.json"), "w") as f:
        json.dump({"package": "photonfdtd", "version": version, "files": files,
                   "how": "wheel content (src/photonfdtd/*.py) copied unmodified"}, f)
    return dst


if __name__ == "__main__":
    print(install(sys.argv[1] if len(sys.argv) > 1 else None, force=True) or
          "reference tree not found (pass it or set PHOTONFDTD_REFERENCE)")
