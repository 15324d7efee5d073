"""Snapshot files in the reference's OVITO ``.data`` text layout
(io.jl:44-54 ``save_state!`` -> ff_ovito.jl:81-116 ``write_ovito``).

``write_ovito`` writes the particle count, a comment line naming the columns
in sorted order (``# acceleration | damage | id | ...``) and one row per
particle holding every column's values (all components of vector columns).
Numbers are printed the way Julia's ``string`` prints them for the common
cases (shortest round-trip digits, ``1.0e-5`` exponent style).  JLD2 output
is not provided (no HDF5 library in this image).
"""
import os

import numpy as np


def _jl(x):
    if isinstance(x, (int, np.integer)):
        return str(int(x))
    s = repr(float(x))
    if s in ("inf", "-inf"):
        return s.replace("inf", "Inf")
    if s == "nan":
        return "NaN"
    if "e" in s:
        m, e = s.split("e")
        if "." not in m:
            m += ".0"
        return f"{m}e{int(e)}"
    return s


def write_ovito(filename, **cols):
    """ff_ovito.jl:81-116.  Each column is a length-N vector or a K x N
    array (one row per particle, its K components in order)."""
    names = sorted(cols)
    arrs = [np.asarray(cols[k]) for k in names]
    item = arrs[names.index("id")]
    n = item.shape[-1] if item.ndim > 1 else item.size
    with open(filename, "w") as fh:
        fh.write(f"{n} \n# " + " | ".join(names) + "\n")
        for j in range(n):
            vals = []
            for a in arrs:
                if a.ndim == 1:
                    vals.append(_jl(a[j]))
                else:
                    vals.extend(_jl(v) for v in a[:, j])
            fh.write(" ".join(vals) + " \n")


def data_writer(out_dir):
    """A ``writer(filename, data)`` for ``run`` that writes ``.data`` files
    into ``out_dir`` (created if needed)."""
    os.makedirs(out_dir, exist_ok=True)

    def writer(filename, data):
        base = os.path.splitext(filename)[0] + ".data"
        write_ovito(os.path.join(out_dir, base), **data)

    return writer
