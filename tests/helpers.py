"""Shared helpers for the tests: fixture loading, VTI parsing, reference text formats."""
from __future__ import annotations

import json
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def golden_case(name):
    d = os.path.join(GOLDEN, name)
    meta = json.load(open(os.path.join(d, "case.json")))
    fields = dict(np.load(os.path.join(d, "fields.npz")))
    return d, meta, fields


def case_params(meta):
    """Oracle/engine parameters of a golden case (reference defaults + its flags)."""
    args = meta["args"]
    kv = {}
    for i in range(0, len(args), 2):
        kv[args[i].lstrip("-")] = args[i + 1]
    return kv


def read_vti(path, shape=None):
    """Values of a reference VTI file as (L, M, N) float32 plus the header text."""
    data = open(path, "rb").read()
    i = data.index(b"_", data.index(b"<AppendedData"))
    head = data[:i].decode()
    if shape is None:
        import re
        e = [int(v) for v in re.search(r'WholeExtent="([^"]+)"', head).group(1).split()]
        shape = (e[1] - e[0] + 1, e[3] - e[2] + 1, e[5] - e[4] + 1)
    L, M, N = shape
    nbytes = np.frombuffer(data[i + 1:i + 5], np.int32)[0]
    vals = np.frombuffer(data[i + 5:i + 5 + 4 * L * M * N], np.float32)
    return vals.reshape(N, M, L).transpose(2, 1, 0).copy(), head, int(nbytes)


def f4(v):
    return "%.4f" % v


def phimax_misfit_lines(atoms):
    """Phimax_<kd>.txt of the Misfit model (MIS:3515-3535) from atom records."""
    good = [a for a in atoms if np.all(np.isfinite(a)) and a[0] >= 0]
    out = [str(2 * len(good)), "Kommentar"]
    for a in good:
        out.append(" ".join(f4(v) for v in a))
        b = list(a)
        b[2] = a[2] + 20
        out.append(" ".join(f4(v) for v in b))
    return out


def phimax_elastic_lines(atoms):
    out = [str(len(atoms)), "Kommentar"]
    out += [" ".join(f4(v) for v in a) for a in atoms if a[0] >= 0]
    return out


def strain_lines(x, y, z, strain, nb):
    out = [str(len(x)), "Kommentar"]
    out += ["st %s %s %s %s %d" % (f4(x[i]), f4(y[i]), f4(z[i]), f4(strain[i]), nb[i]) for i in range(len(x)) if x[i] >= 0]
    return out


def q4q6_lines(x, y, z, q4, q6):
    out = [str(int((np.asarray(x) >= 0).sum())), "Kommentar"]
    out += ["qc %s %s %s %s %s" % (f4(x[i]), f4(y[i]), f4(z[i]), f4(q4[i]), f4(q6[i])) for i in range(len(x)) if x[i] >= 0]
    return out


def energy_line(kd, e, d):
    """One energy.txt line: ostream default formatting (%g, 6 significant digits)."""
    return "%d %s %s" % (kd, fmt_g(e), fmt_g(d))


def fmt_g(v):
    s = "%g" % v
    return s
