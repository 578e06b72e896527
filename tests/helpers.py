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


# ---------------------------------------------------------------------------
# CVD checkpoint analysis files (CVD:1086-1095, 1205-1250, 1314-1345, 1496-1515).
# All arithmetic in float32 as the reference's float locals.
# ---------------------------------------------------------------------------
F32 = np.float32


def cvd_phimax_txt_lines(kd, phic, phimax):
    """The lines atompositionCFGC2 appends to phimax.txt at one checkpoint (rank 0)."""
    return ["%d , %s , %s , 0" % (kd, fmt_g(phic), fmt_g(phimax)), "phimax is done myid=0", " buf is done ",
            " pc_xyz is initializing ", " pc_xyz is done ", " pc_xyz has been gathered "]


def cvd_frames(L, M, N, dx):
    return F32(L) * F32(dx), F32(M) * F32(dx), F32(N) * F32(dx)


def phiball_lines(rec, L, M, N, dx):
    fx, fy, fz = cvd_frames(L, M, N, dx)
    good = [r for r in rec if r[0] >= 0]
    out = ["Number of particles = %d" % len(good), "A = %s Angstrom (basic length-scale)" % f4(10.0),
           "H0(1,1) = %s A " % f4(fy), "H0(1,2) = 0 A ", "H0(1,3) = 0 A ", "H0(2,1) = 0 A ",
           "H0(2,2) = %s A " % f4(fz), "H0(2,3) = 0 A ", "H0(3,1) = 0 A ", "H0(3,2) = 0 A ",
           "H0(3,3) = %s A " % f4(fx), ".NO_VELOCITY.", "entry_count = 3", "63.546", "Cu"]
    out += ["%s %s %s" % (f4(r[0]), f4(r[1]), f4(r[2])) for r in good]
    return out


def cvd_phimax_lines(rec, L, M, N, dx):
    fx, fy, fz = cvd_frames(L, M, N, dx)
    good = [r for r in rec if r[0] >= 0]
    out = [str(len(good)), "Kommentar"]
    out += ["%s %s %s %s" % (f4(F32(r[2]) * fx), f4(F32(r[0]) * fy), f4(F32(r[1]) * fz), f4(r[3])) for r in good]
    return out


def hist_lines(hist):
    return ["%d %d %d" % (i, h, len(hist)) for i, h in enumerate(hist)]


def grq6_lines(hist, num_t, L, M, N, dx):
    delr = F32(1.0 / 25.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        rho = F32(num_t) / (F32(L * M * N) * F32(dx) * F32(dx) * F32(dx))
        preco = F32(4.0 * 3.1415926 * float(rho) / 3.0)
        out = []
        for jj, h in enumerate(hist):
            rlower = F32(jj) * delr
            rupper = rlower + delr
            nideal = preco * (rupper * rupper * rupper - rlower * rlower * rlower)
            gr = F32(h) / F32(1) / F32(num_t) / nideal
            out.append("%s %s %d %s" % (f4(F32(jj) * delr), f4(gr), h, f4(nideal)))
    return out


def ql_lines(nb, ql, qg):
    return ["%d %d %.6f %.6f" % (i, nb[i], ql[i], qg) for i in range(len(nb))]


def histq_lines(histq):
    return ["%s %d" % (f4(F32(i + 1) * F32(0.05)), h) for i, h in enumerate(histq)]
