"""ctypes wrapper of liboracle.so, the CPU restatement of the reference hot path.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` as the checker.  The product package never
imports it.

Restated reference routines (paths within zhiqing0205/PFC-Exp-GUI):
``src/experiment/misfit_uniform_time_seed_fftw_early.cpp`` (Misfit step, init,
energy, Phimax), ``src/experiment/cvd.cpp`` (CVD step and init) and
``src/experiment/elastic.cpp`` (Elastic peak finder, elastic3D, cryst_order).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

MODEL_MISFIT = 0
MODEL_CVD = 1

_lock = threading.Lock()
_lib = None


class OrcParams(C.Structure):
    _fields_ = [
        ("model", C.c_int),
        ("L", C.c_int),
        ("M", C.c_int),
        ("N", C.c_int),
        ("u0", C.c_float),
        ("con0", C.c_float),
        ("sig", C.c_float),
        ("dt", C.c_float),
        ("dx", C.c_float),
        ("axx", C.c_float),
        ("grainx", C.c_int),
        ("grainy", C.c_int),
        ("grainz", C.c_int),
        ("seed", C.c_uint32),
        ("exact", C.c_int),
    ]


def build() -> str:
    """Compile liboracle.so with the recipe in oracle/Makefile (gcc -O2)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    return LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                build()
            L = C.CDLL(LIB_PATH)
            P = C.POINTER
            dp, fp = P(C.c_double), P(C.c_float)
            L.orc_default_params.argtypes = [C.c_int, P(OrcParams)]
            L.orc_create.argtypes = [P(OrcParams)]
            L.orc_create.restype = C.c_void_p
            L.orc_destroy.argtypes = [C.c_void_p]
            L.orc_init.argtypes = [C.c_void_p]
            L.orc_step.argtypes = [C.c_void_p, C.c_int]
            L.orc_get_fields.argtypes = [C.c_void_p, dp, dp]
            L.orc_set_fields.argtypes = [C.c_void_p, dp, dp]
            L.orc_get_c2.argtypes = [C.c_void_p, fp, fp]
            L.orc_get_kref.argtypes = [C.c_void_p, fp, fp, fp]
            L.orc_energy.argtypes = [C.c_void_p, dp, dp]
            L.orc_phimax_misfit.argtypes = [dp, dp, C.c_int, C.c_int, C.c_float, C.c_float, dp, C.c_int,
                                            P(C.c_int)]
            L.orc_phimax_misfit.restype = C.c_int
            L.orc_phimax_elastic.argtypes = [dp, C.c_int, C.c_int, C.c_int, C.c_float, dp, C.c_int]
            L.orc_phimax_elastic.restype = C.c_int
            L.orc_elastic3d.argtypes = [dp, dp, dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                        dp, P(C.c_uint32)]
            L.orc_cryst_order.argtypes = [dp, dp, dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, dp, dp]
            L.orc_dft3d.argtypes = [C.c_int, C.c_int, C.c_int, dp, dp, C.c_int]
            L.orc_cvd_atoms.argtypes = [fp, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, fp, fp, fp, C.c_int]
            L.orc_cvd_atoms.restype = C.c_int
            L.orc_cvd_gr_hist.argtypes = [fp, fp, fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                          P(C.c_uint32), C.c_int]
            L.orc_cvd_gr_hist.restype = C.c_int
            L.orc_cvd_q6.argtypes = [fp, fp, fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, P(C.c_uint32),
                                     fp, fp, P(C.c_uint32)]
            L.orc_splitmix64_next.argtypes = [P(C.c_uint64)]
            L.orc_splitmix64_next.restype = C.c_uint64
            L.orc_rng_u01.argtypes = [P(C.c_uint64)]
            L.orc_rng_u01.restype = C.c_double
            _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def default_params(model: int = MODEL_MISFIT, **kw) -> OrcParams:
    p = OrcParams()
    lib().orc_default_params(model, C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class Run:
    """One simulation run of the restated reference (Misfit or CVD)."""

    def __init__(self, params: OrcParams):
        self.p = params
        self.L, self.M, self.N = params.L, params.M, params.N
        self.P = self.L * self.M * self.N
        self.h = lib().orc_create(C.byref(params))
        lib().orc_init(self.h)
        self.t = 0

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def step(self, n: int = 1):
        for _ in range(n):
            lib().orc_step(self.h, self.t)
            self.t += 1

    def fields(self):
        phi = np.empty(self.P, np.float64)
        con = np.empty(self.P, np.float64)
        lib().orc_get_fields(self.h, _dp(phi), _dp(con))
        shape = (self.L, self.M, self.N)
        return phi.reshape(shape), con.reshape(shape)

    def set_fields(self, phi, con):
        phi = np.ascontiguousarray(phi, np.float64).ravel()
        con = np.ascontiguousarray(con, np.float64).ravel()
        lib().orc_set_fields(self.h, _dp(phi), _dp(con))

    def c2(self):
        a = np.empty(self.P, np.float32)
        b = np.empty(self.P, np.float32)
        lib().orc_get_c2(self.h, _fp(a), _fp(b))
        shape = (self.L, self.M, self.N)
        return a.reshape(shape), b.reshape(shape)

    def kref(self):
        kl = np.empty(self.L, np.float32)
        km = np.empty(self.M, np.float32)
        kn = np.empty(self.N, np.float32)
        lib().orc_get_kref(self.h, _fp(kl), _fp(km), _fp(kn))
        return kl, km, kn

    def energy(self):
        e = C.c_double()
        d = C.c_double()
        lib().orc_energy(self.h, C.byref(e), C.byref(d))
        return e.value, d.value


def phimax_misfit(phi, con, dx=0.125, con0=0.2):
    """Misfit peak finder; phi/con shaped (L, M) or (L, M, 1).  Returns (atoms[n,5], raw_count)."""
    phi = np.ascontiguousarray(phi, np.float64)
    con = np.ascontiguousarray(con, np.float64)
    L, M = phi.shape[0], phi.shape[1]
    cap = L * M + 1
    out = np.zeros((cap, 5), np.float64)
    raw = C.c_int()
    n = lib().orc_phimax_misfit(_dp(phi), _dp(con), L, M, dx, con0, _dp(out), cap, C.byref(raw))
    return out[:n].copy(), raw.value


def phimax_elastic(phi, dx=0.125):
    """Elastic peak finder; phi shaped (L, M, N).  Returns atoms[n,4] (x, y, z, phimax)."""
    phi = np.ascontiguousarray(phi, np.float64)
    L, M, N = phi.shape
    cap = L * M * N + 1
    out = np.zeros((cap, 4), np.float64)
    n = lib().orc_phimax_elastic(_dp(phi), L, M, N, dx, _dp(out), cap)
    return out[:n].copy()


def elastic3d(x, y, z, L, M, N, dx=0.125, benchel=1.7):
    x, y, z = (np.ascontiguousarray(a, np.float64) for a in (x, y, z))
    n = len(x)
    strain = np.zeros(n, np.float64)
    nb = np.zeros(n, np.uint32)
    lib().orc_elastic3d(_dp(x), _dp(y), _dp(z), n, L, M, N, dx, benchel, _dp(strain),
                        nb.ctypes.data_as(C.POINTER(C.c_uint32)))
    return strain, nb


def cryst_order(x, y, z, L, M, N, dx=0.125):
    x, y, z = (np.ascontiguousarray(a, np.float64) for a in (x, y, z))
    n = len(x)
    q4 = np.zeros(n, np.float64)
    q6 = np.zeros(n, np.float64)
    lib().orc_cryst_order(_dp(x), _dp(y), _dp(z), n, L, M, N, dx, _dp(q4), _dp(q6))
    return q4, q6


def cvd_atoms(phi, u0, dx=0.125):
    """atompositionCFGC2 peak finder (CVD:1076-1165) on a float32 field shaped (L, M, N).
    Returns (phic, phimax, records[n, 4] = (x, y, z, phi) fractional float32)."""
    phi = np.ascontiguousarray(phi, np.float32)
    L, M, N = phi.shape
    cap = L * M * N + 1
    out = np.zeros((cap, 4), np.float32)
    phic, pmax = C.c_float(), C.c_float()
    n = lib().orc_cvd_atoms(_fp(phi), L, M, N, dx, u0, C.byref(phic), C.byref(pmax), _fp(out), cap)
    return np.float32(phic.value), np.float32(pmax.value), out[:n].copy()


def cvd_gr_hist(rec, L, M, N, dx=0.125):
    """GR's pair-distance histogram (CVD:1277-1312) of the records."""
    x, y, z = (np.ascontiguousarray(rec[:, k], np.float32) for k in range(3))
    hist = np.zeros(L * 8 + 16, np.uint32)
    mb = lib().orc_cvd_gr_hist(_fp(x), _fp(y), _fp(z), len(x), L, M, N, dx,
                               hist.ctypes.data_as(C.POINTER(C.c_uint32)), len(hist))
    return hist[:mb].copy()


def cvd_q6(rec, L, M, N, dx=0.125):
    """Q6_GLO (CVD:1349-1520): (neighbour counts, local Q6, global Q6, 30-bin histogram)."""
    x, y, z = (np.ascontiguousarray(rec[:, k], np.float32) for k in range(3))
    n = len(x)
    nb = np.zeros(n, np.uint32)
    ql = np.zeros(n, np.float32)
    qg = C.c_float()
    histq = np.zeros(30, np.uint32)
    lib().orc_cvd_q6(_fp(x), _fp(y), _fp(z), n, L, M, N, dx, nb.ctypes.data_as(C.POINTER(C.c_uint32)), _fp(ql),
                     C.byref(qg), histq.ctypes.data_as(C.POINTER(C.c_uint32)))
    return nb, ql, np.float32(qg.value), histq


def dft3d(a, sign=-1):
    """3-D complex DFT with FFTW conventions (the shim's transform)."""
    a = np.ascontiguousarray(a, np.complex128)
    out = np.empty_like(a)
    n0, n1, n2 = a.shape
    lib().orc_dft3d(n0, n1, n2, a.ctypes.data_as(C.POINTER(C.c_double)),
                    out.ctypes.data_as(C.POINTER(C.c_double)), sign)
    return out


def ref_binary(L, M, N):
    """Path of the reference binary built by ``make -C oracle ref`` for this grid, or None."""
    p = os.path.join(REF_DIR, f"pfc-exp-cli-{L}x{M}x{N}")
    return p if os.path.exists(p) else None
