"""The allocation-free Misfit peak finder against the allocating one.

pfc_phimax_misfit_noalloc serves callers that cannot allocate device memory: a
serving loop that has committed its whole HBM budget to resident runs, or a host
thread that must not cause the device-wide synchronisation of cudaMalloc and
cudaFree.  It keeps its compaction scratch in a fixed array inside the library,
shared by every call.  Its atoms must equal those of pfc_phimax_misfit on the same
field, bit for bit (the tolerance of the peak-finder tests), on two calls in a row,
so that whatever the first call leaves in the shared array cannot change the second.

This file is collected last on purpose; it needs no state from the other tests.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import pfc_b200 as P

pytestmark = pytest.mark.gpu


def _field(L, M, steps, seed):
    o = O.Run(O.default_params(O.MODEL_MISFIT, L=L, M=M, N=1, seed=seed))
    o.step(steps)
    phi, con = o.fields()
    return np.ascontiguousarray(phi[:, :, 0], np.float32), np.ascontiguousarray(con[:, :, 0], np.float32)


def _noalloc(torch, phi, con, cap):
    L, M = phi.shape
    dphi = torch.from_numpy(phi).cuda()
    dcon = torch.from_numpy(con).cuda()
    dout = torch.full((cap, 5), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    n = C.c_int(-1)
    rc = P.lib().pfc_phimax_misfit_noalloc(C.c_void_p(dphi.data_ptr()), C.c_void_p(dcon.data_ptr()), L, M, 0.125, 0.2,
                                           C.c_void_p(dout.data_ptr()), cap, C.byref(n), None)
    assert rc == P.PFC_OK, P.lib().pfc_last_error()
    return dout[: n.value].cpu().numpy()


def test_noalloc_matches_allocating_entry_point():
    torch = pytest.importorskip("torch")
    cases = [(256, 128, 30, 7), (64, 64, 25, 20200604), (512, 512, 20, 1003)]
    for L, M, steps, seed in cases:
        phi, con = _field(L, M, steps, seed)
        ref = P.phimax_misfit(phi, con)
        assert len(ref) > 1
        cap = L * M + 1
        first = _noalloc(torch, phi, con, cap)
        second = _noalloc(torch, phi, con, cap)
        assert np.array_equal(first, ref)
        assert np.array_equal(second, ref)


def test_noalloc_fallback_and_limit():
    torch = pytest.importorskip("torch")
    flat = np.full((32, 64), 0.25, np.float32)
    con = np.full((32, 64), 0.2, np.float32)
    ref = P.phimax_misfit(flat, con)
    assert np.array_equal(_noalloc(torch, flat, con, 33), ref)
    assert np.array_equal(_noalloc(torch, flat, con, 33), ref)
    # fields beyond the fixed scratch capacity are refused before anything runs
    small = torch.zeros(16, dtype=torch.float32, device="cuda")
    out = torch.zeros(16, dtype=torch.float64, device="cuda")
    n = C.c_int(-1)
    rc = P.lib().pfc_phimax_misfit_noalloc(C.c_void_p(small.data_ptr()), C.c_void_p(small.data_ptr()), 4096, 2048,
                                           0.125, 0.2, C.c_void_p(out.data_ptr()), 1, C.byref(n), None)
    assert rc == -1 and n.value == -1
    assert "4194304" in P.lib().pfc_last_error().decode()
