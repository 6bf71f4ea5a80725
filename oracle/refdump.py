"""Reader for the dumps written by the compiled-reference drivers (test infrastructure only).

The drivers in ``oracle/ref_driver`` write raw little-endian arrays named
``<tag>.i32`` / ``<tag>.f64`` and a ``meta.txt`` of ``key=value`` lines; this
module loads such a directory (or the ``.npz`` fixture made from one) into a
plain dict of numpy arrays and scalars.
"""
import os

import numpy as np


def load_dir(path):
    out = {}
    with open(os.path.join(path, "meta.txt")) as f:
        for line in f:
            line = line.strip()
            if not line or "=" not in line:
                continue
            k, v = line.split("=", 1)
            try:
                out[k] = int(v)
            except ValueError:
                out[k] = float(v)
    for fn in os.listdir(path):
        stem, ext = os.path.splitext(fn)
        if ext == ".i32":
            out[stem] = np.fromfile(os.path.join(path, fn), dtype="<i4")
        elif ext == ".f64":
            out[stem] = np.fromfile(os.path.join(path, fn), dtype="<f8")
    return out


def load_npz(path):
    z = np.load(path, allow_pickle=False)
    out = {}
    for k in z.files:
        a = z[k]
        out[k] = a.item() if a.ndim == 0 else a
    return out


def level(d, l):
    """Per-level view with the level prefix stripped."""
    p = f"L{l}_"
    return {k[len(p):]: v for k, v in d.items() if k.startswith(p)}
