"""Load golden fixtures and compare runs against them."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    return g, json.loads(str(g["meta"]))


def _get(res, kind, mon, comp=None):
    d = getattr(res, kind) if not isinstance(res, dict) else res[kind]
    return d[mon] if comp is None else d[mon][comp]


def compare(res, name):
    """Relative max-abs and relative L2 differences of every golden array.

    Returns {key: (rel_max, rel_l2)} with both scaled by the golden array's
    max |value| / L2 norm. A fixture whose DFT was thinned (meta
    "thin_dft") is compared on the frequencies it kept."""
    g, meta = load(name)
    out = {}
    for k in g.files:
        if k.startswith("f/"):
            _, mon, c = k.split("/")
            a = np.asarray(_get(res, "fields", mon, c))[meta["keep"][mon]]
        elif k.startswith("dft/"):
            _, mon, c = k.split("/")
            a = np.asarray(_get(res, "dft", mon, c))
            thin = meta.get("thin_dft")
            if thin is not None:
                a = a[list(thin["freqs"])]
        elif k.startswith("flux/"):
            a = np.asarray(_get(res, "flux", k.split("/")[1]))
        else:
            continue
        b = g[k]
        assert a.shape == b.shape, (k, a.shape, b.shape)
        diff = np.asarray(a, np.complex128) - np.asarray(b, np.complex128)
        nb = np.abs(b).max() if b.size else 0.0
        l2 = np.linalg.norm(np.asarray(b, np.complex128).ravel())
        out[k] = (np.abs(diff).max() / nb if nb > 0 else np.abs(diff).max(),
                  np.linalg.norm(diff.ravel()) / l2 if l2 > 0 else np.linalg.norm(diff.ravel()))
    return out
