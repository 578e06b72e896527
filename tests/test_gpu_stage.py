"""Tile staging of the column kernel: one TMA bulk copy per tile, completing on a
shared-memory mbarrier, and a wait on that barrier bounded in time.

pfc_selftest_tile_stage runs the same staging helpers as the column kernel in a
one-CTA kernel.  A staged tile must come back bit for bit.  A wait for a copy that
was never started must run out after its limit, be reported to the host, and leave
the device usable: a run created afterwards steps normally.  No copy is in flight
when that wait gives up, so the kernel exits cleanly.
"""
import ctypes as C

import numpy as np
import pytest

import pfc_b200 as P


def _selftest(issue, n, limit_ms):
    timed_out, match, ms = C.c_int(-1), C.c_int(-1), C.c_double(-1.0)
    rc = P.lib().pfc_selftest_tile_stage(0, issue, n, limit_ms, C.byref(timed_out), C.byref(match), C.byref(ms))
    return rc, timed_out.value, match.value, ms.value


def test_selftest_rejects_bad_sizes_without_a_device():
    for n, limit in [(3, 1.0), (0, 1.0), (8194, 1.0), (512, 0.0), (512, -1.0), (512, 20000.0)]:
        rc, *_ = _selftest(1, n, limit)
        assert rc == P.PFC_E_INVALID


@pytest.mark.gpu
@pytest.mark.parametrize("n", [2, 512, 2048, 4096, 8192])
def test_bulk_copy_round_trip(n):
    rc, timed_out, match, ms = _selftest(1, n, 1000.0)
    assert rc == P.PFC_OK, P.lib().pfc_last_error()
    assert timed_out == 0
    assert match == 1
    assert ms < 1000.0


@pytest.mark.gpu
def test_wait_runs_out_and_device_stays_usable():
    limit_ms = 2.0
    rc, timed_out, match, ms = _selftest(0, 512, limit_ms)
    assert rc == P.PFC_OK, P.lib().pfc_last_error()
    assert timed_out == 1
    assert match == 0  # nothing was written back
    # the wait gave up after its limit (plus the kernel's bounded drain of 100 ms)
    assert limit_ms <= ms < limit_ms + 100.0 + 500.0
    # the device and the library's context still work
    r = P.Run(P.default_params(P.MODEL_MISFIT, L=128, M=128, seed=5))
    try:
        r.advance(5)
        phi, con = r.fields_f32()
        assert np.isfinite(phi).all() and np.isfinite(con).all()
    finally:
        r.close()
