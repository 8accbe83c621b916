"""Where the reference photonfdtd lives, for the recipes that read it.

The reference source tree is needed only by build recipes (installing the
reference package into baseline/_ref, compiling its CUDA kernels, writing the
golden fixtures). Its location comes from, in order: an explicit argument,
the PHOTONFDTD_REFERENCE environment variable, or a directory named
``reference`` beside this repository's root. Nothing at run time needs it:
the installed copy in baseline/_ref travels with the working tree.
"""
from __future__ import annotations

import os
import sys
from typing import Optional

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INSTALL_DIR = os.path.join(REPO, "baseline", "_ref")


def reference_root(arg: Optional[str] = None) -> Optional[str]:
    """The reference source tree (holding src/photonfdtd), or None."""
    for cand in (arg, os.environ.get("PHOTONFDTD_REFERENCE"),
                 os.path.join(os.path.dirname(REPO), "reference")):
        if cand and os.path.isfile(os.path.join(cand, "src", "photonfdtd", "__init__.py")):
            return os.path.abspath(cand)
    return None


def installed() -> bool:
    """Whether the reference package is installed in baseline/_ref."""
    return os.path.isfile(os.path.join(INSTALL_DIR, "photonfdtd", "__init__.py"))


def import_reference():
    """The reference package: the copy installed in baseline/_ref, else the
    source tree; None when neither is present."""
    paths = []
    if installed():
        paths.append(INSTALL_DIR)
    root = reference_root()
    if root is not None:
        paths.append(os.path.join(root, "src"))
    for p in paths:
        if p not in sys.path:
            sys.path.insert(0, p)
        try:
            import photonfdtd
            return photonfdtd
        except ImportError:
            continue
    return None
