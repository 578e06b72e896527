"""ctypes binding of libpfc_b200.so (the C ABI declared in include/pfc_b200.h).

This is the Python view of the same entry points a C/C++ caller links against.
Importing it does not need a GPU; creating a run does.  There is no fallback:
if the shared library is missing, :func:`lib` raises, and every call that fails
on the device raises :class:`PfcError` with the library's message.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG_DIR)
LIB_PATH = os.path.join(ROOT, "lib", "libpfc_b200.so")
CLI_PATH = os.path.join(ROOT, "bin", "pfc-exp-cli")
HEADER_PATH = os.path.join(os.path.dirname(ROOT), "include", "pfc_b200.h")

MODEL_MISFIT = 0
MODEL_CVD = 1
FP32 = 0
FP64 = 1
FP64_PURE = 2
MIXED = 3  # FP32 arrays in HBM, FP64 arithmetic (the default precision)

PFC_OK = 0
PFC_E_INVALID, PFC_E_CUDA, PFC_E_NOMEM, PFC_E_IO, PFC_E_STATE, PFC_E_NONFINITE = -1, -2, -3, -4, -5, -6


class PfcError(RuntimeError):
    pass


class RunParams(C.Structure):
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
        ("precision", C.c_int),
        ("device", C.c_int),
    ]


class EngineOpts(C.Structure):
    _fields_ = [
        ("device", C.c_int),
        ("hbm_budget_bytes", C.c_double),
        ("max_active", C.c_int),
        ("quantum_steps", C.c_int),
    ]


class JobSpec(C.Structure):
    _fields_ = [
        ("kind", C.c_int),
        ("params", RunParams),
        ("steps", C.c_int),
        ("mod", C.c_int),
        ("outdir", C.c_char_p),
        ("source_job", C.c_uint64),
        ("input_dir", C.c_char_p),
        ("benchel", C.c_float),
    ]


class Event(C.Structure):
    _fields_ = [
        ("job", C.c_uint64),
        ("type", C.c_int),
        ("status", C.c_int),
        ("step", C.c_int),
        ("atoms", C.c_int),
        ("energy", C.c_double),
        ("mass", C.c_double),
        ("t_submit", C.c_double),
        ("t_admit", C.c_double),
        ("t_event", C.c_double),
        ("t_finish", C.c_double),
    ]


JOB_MISFIT, JOB_CVD, JOB_ELASTIC = 0, 1, 2
EV_ADMITTED, EV_CHECKPOINT, EV_DONE, EV_FAILED, EV_CANCELLED = 1, 2, 3, 4, 5

_lib = None


def build(jobs: int = 8) -> str:
    """Compile the library and the CLI with this package's Makefile (sm_100a)."""
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", ROOT], check=True)
    return LIB_PATH


def lib():
    """Load libpfc_b200.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise PfcError(f"libpfc_b200.so not built ({LIB_PATH}); run `make -C {ROOT}`")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    vp, dp, fp = C.c_void_p, P(C.c_double), P(C.c_float)
    sig = {
        "pfc_last_error": ([], C.c_char_p),
        "pfc_default_params": ([C.c_int, P(RunParams)], C.c_int),
        "pfc_run_create": ([P(RunParams), P(vp)], C.c_int),
        "pfc_run_destroy": ([vp], C.c_int),
        "pfc_run_advance": ([vp, C.c_int, C.c_int], C.c_int),
        "pfc_run_steps": ([vp, P(C.c_int)], C.c_int),
        "pfc_run_advance_timed": ([vp, C.c_int, P(C.c_float)], C.c_int),
        "pfc_run_get_fields": ([vp, dp, dp], C.c_int),
        "pfc_run_get_fields_f32": ([vp, fp, fp], C.c_int),
        "pfc_run_set_fields": ([vp, dp, dp], C.c_int),
        "pfc_run_energy": ([vp, dp, dp], C.c_int),
        "pfc_run_means": ([vp, dp, dp], C.c_int),
        "pfc_run_set_fields_f32": ([vp, fp, fp], C.c_int),
        "pfc_run_nonfinite": ([vp, P(C.c_int)], C.c_int),
        "pfc_batch_create": ([P(vp), C.c_int, P(vp)], C.c_int),
        "pfc_batch_destroy": ([vp], C.c_int),
        "pfc_batch_advance": ([vp, C.c_int], C.c_int),
        "pfc_phimax_misfit": ([fp, fp, C.c_int, C.c_int, C.c_float, C.c_float, dp, C.c_int, P(C.c_int)], C.c_int),
        "pfc_phimax_misfit_noalloc": ([vp, vp, C.c_int, C.c_int, C.c_float, C.c_float, vp, C.c_int, P(C.c_int), vp],
                                      C.c_int),
        "pfc_phimax_elastic": ([fp, C.c_int, C.c_int, C.c_int, C.c_float, dp, C.c_int, P(C.c_int)], C.c_int),
        "pfc_elastic3d": ([dp, dp, dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, dp,
                           P(C.c_uint32)], C.c_int),
        "pfc_cryst_order": ([dp, dp, dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, dp, dp], C.c_int),
        "pfc_dft3d": ([dp, dp, C.c_int, C.c_int, C.c_int, C.c_int], C.c_int),
        "pfc_cvd_atoms": ([fp, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, fp, C.c_int, P(C.c_int), fp, fp],
                          C.c_int),
        "pfc_cvd_gr_hist": ([fp, fp, fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, P(C.c_uint32), C.c_int,
                             P(C.c_int)], C.c_int),
        "pfc_cvd_q6": ([fp, fp, fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, P(C.c_uint32), fp, fp], C.c_int),
        "pfc_batch_advance_timed": ([vp, C.c_int, P(C.c_float)], C.c_int),
        "pfc_batch_kernel_times": ([vp, C.c_int, dp, dp], C.c_int),
        "pfc_run_cli": ([C.c_int, P(C.c_char_p)], C.c_int),
        "pfc_engine_create": ([P(EngineOpts), P(vp)], C.c_int),
        "pfc_engine_destroy": ([vp], C.c_int),
        "pfc_submit": ([vp, P(JobSpec), P(C.c_uint64)], C.c_int),
        "pfc_submit_many": ([vp, P(JobSpec), C.c_int, P(C.c_uint64)], C.c_int),
        "pfc_poll": ([vp, P(Event), C.c_int, P(C.c_int)], C.c_int),
        "pfc_wait": ([vp, P(Event), C.c_int, P(C.c_int), C.c_int], C.c_int),
        "pfc_cancel": ([vp, C.c_uint64], C.c_int),
        "pfc_job_fields": ([vp, C.c_uint64, fp, fp], C.c_int),
        "pfc_release": ([vp, C.c_uint64], C.c_int),
        "pfc_run_bytes": ([P(RunParams), dp], C.c_int),
        "pfc_tile_width": ([C.c_int, C.c_int, C.c_int, C.c_int, P(C.c_int), P(C.c_int), fp, P(C.c_int)], C.c_int),
        "pfc_set_tile_width": ([C.c_int, C.c_int, C.c_int, C.c_int, C.c_int], C.c_int),
        "pfc_col_staging": ([C.c_int, C.c_int, C.c_int, C.c_int, P(C.c_int), fp, fp, P(C.c_int)], C.c_int),
        "pfc_set_col_staging": ([C.c_int, C.c_int, C.c_int, C.c_int, C.c_int], C.c_int),
        "pfc_selftest_tile_stage": ([C.c_int, C.c_int, C.c_int, C.c_double, P(C.c_int), P(C.c_int), dp], C.c_int),
        "pfc_selftest_log": ([C.c_int, dp, dp, C.c_int], C.c_int),
        "pfc_run_advance_energies": ([vp, C.c_int, dp, dp], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _check(rc: int, what: str):
    if rc != PFC_OK:
        msg = lib().pfc_last_error().decode(errors="replace")
        raise PfcError(f"{what} failed ({rc}): {msg}")


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def default_params(model: int = MODEL_MISFIT, **kw) -> RunParams:
    p = RunParams()
    _check(lib().pfc_default_params(model, C.byref(p)), "pfc_default_params")
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class Run:
    """One Misfit or CVD run resident on the GPU."""

    def __init__(self, params: RunParams):
        self.params = params
        self.L, self.M, self.N = params.L, params.M, params.N
        self.P = self.L * self.M * self.N
        self.h = C.c_void_p()
        _check(lib().pfc_run_create(C.byref(params), C.byref(self.h)), "pfc_run_create")

    def close(self):
        if self.h:
            lib().pfc_run_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def advance(self, nsteps: int = 1, analysis: bool = False):
        _check(lib().pfc_run_advance(self.h, nsteps, 1 if analysis else 0), "pfc_run_advance")

    def advance_timed(self, nsteps: int) -> float:
        """Advance and return the device time in ms (CUDA events on the run's stream)."""
        ms = C.c_float()
        _check(lib().pfc_run_advance_timed(self.h, nsteps, C.byref(ms)), "pfc_run_advance_timed")
        return ms.value

    @property
    def steps(self) -> int:
        s = C.c_int()
        _check(lib().pfc_run_steps(self.h, C.byref(s)), "pfc_run_steps")
        return s.value

    def fields(self):
        phi = np.empty(self.P, np.float64)
        con = np.empty(self.P, np.float64)
        _check(lib().pfc_run_get_fields(self.h, _dp(phi), _dp(con)), "pfc_run_get_fields")
        s = (self.L, self.M, self.N)
        return phi.reshape(s), con.reshape(s)

    def fields_f32(self, out=None):
        """FP32 real fields (phi, con) shaped (L, M, N); `out` = (phi, con) float32 arrays of
        P elements (e.g. pinned host buffers) to fill instead of new ones."""
        if out is None:
            phi = np.empty(self.P, np.float32)
            con = np.empty(self.P, np.float32)
        else:
            phi, con = out
        _check(lib().pfc_run_get_fields_f32(self.h, _fp(phi), _fp(con)), "pfc_run_get_fields_f32")
        s = (self.L, self.M, self.N)
        return phi.reshape(s), con.reshape(s)

    def set_fields_f32(self, phi, con):
        """Replace the state with FP32 real fields (copied as they are; pinned arrays make
        the copy asynchronous)."""
        phi = np.ascontiguousarray(phi, np.float32).ravel()
        con = np.ascontiguousarray(con, np.float32).ravel()
        _check(lib().pfc_run_set_fields_f32(self.h, _fp(phi), _fp(con)), "pfc_run_set_fields_f32")

    def set_fields(self, phi, con):
        phi = np.ascontiguousarray(phi, np.float64).ravel()
        con = np.ascontiguousarray(con, np.float64).ravel()
        _check(lib().pfc_run_set_fields(self.h, _dp(phi), _dp(con)), "pfc_run_set_fields")

    def energy(self):
        e, d = C.c_double(), C.c_double()
        _check(lib().pfc_run_energy(self.h, C.byref(e), C.byref(d)), "pfc_run_energy")
        return e.value, d.value

    def advance_energies(self, n):
        """n steps, each followed by the energy analysis; returns (e/P, mass/P) per step as
        float64 arrays of length n (pfc_run_advance_energies)."""
        e, d = np.empty(n, np.float64), np.empty(n, np.float64)
        _check(lib().pfc_run_advance_energies(self.h, n, _dp(e), _dp(d)), "pfc_run_advance_energies")
        return e, d

    def nonfinite(self) -> bool:
        """True when the run met a NaN / Inf nonlinear term since creation or the last call."""
        f = C.c_int()
        _check(lib().pfc_run_nonfinite(self.h, C.byref(f)), "pfc_run_nonfinite")
        return bool(f.value)

    def means(self):
        a, b = C.c_double(), C.c_double()
        _check(lib().pfc_run_means(self.h, C.byref(a), C.byref(b)), "pfc_run_means")
        return a.value, b.value


class Batch:
    """Runs advanced together, one launch per grid size per sweep (CUDA graph)."""

    def __init__(self, runs):
        self.runs = list(runs)
        arr = (C.c_void_p * len(self.runs))(*[r.h.value for r in self.runs])
        self.h = C.c_void_p()
        _check(lib().pfc_batch_create(arr, len(self.runs), C.byref(self.h)), "pfc_batch_create")

    def advance(self, nsteps: int):
        _check(lib().pfc_batch_advance(self.h, nsteps), "pfc_batch_advance")

    def advance_timed(self, nsteps: int) -> float:
        """Advance and return the device time in ms (CUDA events on the batch stream)."""
        ms = C.c_float()
        _check(lib().pfc_batch_advance_timed(self.h, nsteps, C.byref(ms)), "pfc_batch_advance_timed")
        return ms.value

    def kernel_times(self, reps: int):
        """Mean device ms of the row-kernel and column-kernel launches of one step."""
        a, b = C.c_double(), C.c_double()
        _check(lib().pfc_batch_kernel_times(self.h, reps, C.byref(a), C.byref(b)), "pfc_batch_kernel_times")
        return a.value, b.value

    def close(self):
        if self.h:
            lib().pfc_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Engine:
    """Many runs on one GPU: submit jobs, then poll or wait for their events."""

    def __init__(self, device=0, hbm_budget_bytes=0.0, max_active=0, quantum_steps=0):
        o = EngineOpts(device, hbm_budget_bytes, max_active, quantum_steps)
        self.h = C.c_void_p()
        _check(lib().pfc_engine_create(C.byref(o), C.byref(self.h)), "pfc_engine_create")
        self.grids = {}

    def submit(self, kind, params=None, steps=0, mod=0, outdir=None, source_job=0, input_dir=None, benchel=0.0):
        if params is None:
            params = default_params(MODEL_CVD if kind == JOB_CVD else MODEL_MISFIT)
        j = JobSpec(kind, params, steps, mod, outdir.encode() if outdir else None, source_job,
                    input_dir.encode() if input_dir else None, benchel)
        jid = C.c_uint64()
        _check(lib().pfc_submit(self.h, C.byref(j), C.byref(jid)), "pfc_submit")
        self.grids[jid.value] = (params.L, params.M, params.N)
        return jid.value

    def submit_many(self, kind, params_list, steps=0, mod=0):
        """Queue one job per parameter set in a single call (pfc_submit_many); returns their ids."""
        n = len(params_list)
        arr = (JobSpec * n)(*[JobSpec(kind, p, steps, mod, None, 0, None, 0.0) for p in params_list])
        ids = (C.c_uint64 * n)()
        _check(lib().pfc_submit_many(self.h, arr, n, ids), "pfc_submit_many")
        for p, i in zip(params_list, ids):
            self.grids[i] = (p.L, p.M, p.N)
        return list(ids)

    def poll(self, max_events=256):
        ev = (Event * max_events)()
        n = C.c_int()
        _check(lib().pfc_poll(self.h, ev, max_events, C.byref(n)), "pfc_poll")
        return [ev[i] for i in range(n.value)]

    def wait(self, timeout_ms=-1, max_events=256):
        ev = (Event * max_events)()
        n = C.c_int()
        _check(lib().pfc_wait(self.h, ev, max_events, C.byref(n), timeout_ms), "pfc_wait")
        return [ev[i] for i in range(n.value)]

    def cancel(self, jid):
        _check(lib().pfc_cancel(self.h, jid), "pfc_cancel")

    def fields(self, jid):
        L, M, N = self.grids[jid]
        phi = np.empty((L, M, N) if N > 1 else (L, M), np.float32)
        con = np.empty_like(phi)
        _check(lib().pfc_job_fields(self.h, jid, _fp(phi), _fp(con)), "pfc_job_fields")
        return phi, con

    def release(self, jid):
        _check(lib().pfc_release(self.h, jid), "pfc_release")

    def close(self):
        if self.h:
            lib().pfc_engine_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tile_width(L: int, M: int, device: int = 0, precision: int = MIXED):
    """Column tile width fused-path runs (MIXED or FP32) of an L x M grid use (tuned on
    the device on first use) and the autotuner's trials: (width, {candidate: ms per 8
    steps})."""
    w, n = C.c_int(), C.c_int()
    cand = (C.c_int * 4)()
    ms = (C.c_float * 4)()
    _check(lib().pfc_tile_width(device, L, M, precision, C.byref(w), cand, ms, C.byref(n)), "pfc_tile_width")
    return w.value, {cand[i]: ms[i] for i in range(n.value)}


def set_tile_width(L: int, M: int, width: int, device: int = 0, precision: int = MIXED):
    """Fix the column tile width of an L x M grid and precision for the rest of the process."""
    _check(lib().pfc_set_tile_width(device, L, M, precision, width), "pfc_set_tile_width")


STAGE_ASYNC, STAGE_BULK = 0, 1


def col_staging(L: int, M: int, device: int = 0, precision: int = MIXED):
    """Tile staging method of the column kernel for an L x M grid and precision (tuned
    on the device on first use) and the trials: (stage, {candidate width: (ms async,
    ms bulk)})."""
    st, n = C.c_int(), C.c_int()
    a = (C.c_float * 4)()
    b = (C.c_float * 4)()
    _check(lib().pfc_col_staging(device, L, M, precision, C.byref(st), a, b, C.byref(n)), "pfc_col_staging")
    _, trials = tile_width(L, M, device, precision)
    cand = list(trials)
    return st.value, {cand[i]: (a[i], b[i]) for i in range(n.value)}


def set_col_staging(L: int, M: int, stage: int, device: int = 0, precision: int = MIXED):
    """Fix the column kernel's tile staging (STAGE_ASYNC or STAGE_BULK) of an L x M grid."""
    _check(lib().pfc_set_col_staging(device, L, M, precision, stage), "pfc_set_col_staging")


def run_bytes(params) -> float:
    """Device bytes a run with these parameters reserves (pfc_run_bytes)."""
    b = C.c_double()
    _check(lib().pfc_run_bytes(C.byref(params), C.byref(b)), "pfc_run_bytes")
    return b.value


def phimax_misfit(phi, con, dx=0.125, con0=0.2):
    phi = np.ascontiguousarray(phi, np.float32)
    con = np.ascontiguousarray(con, np.float32)
    L, M = phi.shape[0], phi.shape[1]
    cap = L * M + 1
    out = np.empty((cap, 5), np.float64)  # only the first n rows are written and read
    n = C.c_int()
    _check(lib().pfc_phimax_misfit(_fp(phi), _fp(con), L, M, dx, con0, _dp(out), cap, C.byref(n)), "pfc_phimax_misfit")
    return out[: n.value].copy()


def phimax_elastic(phi, dx=0.125):
    phi = np.ascontiguousarray(phi, np.float32)
    L, M, N = phi.shape
    cap = L * M * N + 1
    out = np.empty((cap, 4), np.float64)  # only the first n rows are written and read
    n = C.c_int()
    _check(lib().pfc_phimax_elastic(_fp(phi), L, M, N, dx, _dp(out), cap, C.byref(n)), "pfc_phimax_elastic")
    return out[: n.value].copy()


def elastic3d(x, y, z, L, M, N, dx=0.125, benchel=1.7):
    x, y, z = (np.ascontiguousarray(a, np.float64) for a in (x, y, z))
    n = len(x)
    strain = np.zeros(n, np.float64)
    nb = np.zeros(n, np.uint32)
    _check(lib().pfc_elastic3d(_dp(x), _dp(y), _dp(z), n, L, M, N, dx, benchel, _dp(strain),
                               nb.ctypes.data_as(C.POINTER(C.c_uint32))), "pfc_elastic3d")
    return strain, nb


def cryst_order(x, y, z, L, M, N, dx=0.125):
    x, y, z = (np.ascontiguousarray(a, np.float64) for a in (x, y, z))
    n = len(x)
    q4 = np.zeros(n, np.float64)
    q6 = np.zeros(n, np.float64)
    _check(lib().pfc_cryst_order(_dp(x), _dp(y), _dp(z), n, L, M, N, dx, _dp(q4), _dp(q6)), "pfc_cryst_order")
    return q4, q6


def cvd_atoms(phi, u0, dx=0.125):
    """CVD checkpoint peak finder (atompositionCFGC2) on a float32 field shaped (L, M, N).
    Returns (phic, phimax, records[n, 4]) with records (x, y, z, phi) as the reference's pc_*."""
    phi = np.ascontiguousarray(phi, np.float32)
    L, M, N = phi.shape
    cap = L * M * N + 1
    out = np.empty((cap, 4), np.float32)  # only the first n rows are written and read
    n, phic, pmax = C.c_int(), C.c_float(), C.c_float()
    _check(lib().pfc_cvd_atoms(_fp(phi), L, M, N, dx, u0, _fp(out), cap, C.byref(n), C.byref(phic), C.byref(pmax)),
           "pfc_cvd_atoms")
    return np.float32(phic.value), np.float32(pmax.value), out[: n.value].copy()


def cvd_gr_hist(rec, L, M, N, dx=0.125):
    x, y, z = (np.ascontiguousarray(rec[:, k], np.float32) for k in range(3))
    hist = np.zeros(L * 8 + 16, np.uint32)
    mb = C.c_int()
    _check(lib().pfc_cvd_gr_hist(_fp(x), _fp(y), _fp(z), len(x), L, M, N, dx,
                                 hist.ctypes.data_as(C.POINTER(C.c_uint32)), len(hist), C.byref(mb)), "pfc_cvd_gr_hist")
    return hist[: mb.value].copy()


def cvd_q6(rec, L, M, N, dx=0.125):
    x, y, z = (np.ascontiguousarray(rec[:, k], np.float32) for k in range(3))
    n = len(x)
    nb = np.zeros(n, np.uint32)
    ql = np.zeros(n, np.float32)
    qg = C.c_float()
    _check(lib().pfc_cvd_q6(_fp(x), _fp(y), _fp(z), n, L, M, N, dx, nb.ctypes.data_as(C.POINTER(C.c_uint32)),
                            _fp(ql), C.byref(qg)), "pfc_cvd_q6")
    return nb, ql, np.float32(qg.value)


def dft3d(a, sign=-1):
    """3-D complex-double DFT on the GPU with FFTW's conventions (unnormalised)."""
    a = np.ascontiguousarray(a, np.complex128)
    out = np.empty_like(a)
    n0, n1, n2 = a.shape
    _check(lib().pfc_dft3d(a.ctypes.data_as(C.POINTER(C.c_double)), out.ctypes.data_as(C.POINTER(C.c_double)),
                           n0, n1, n2, sign), "pfc_dft3d")
    return out


def header_functions(path: str = HEADER_PATH):
    """Names of the functions declared in include/pfc_b200.h."""
    import re
    txt = open(path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(pfc_[a-z0-9_]+)\s*\(", txt)))
