"""GPU tests of the column tile-width autotuner.

The width only regroups the columns that one column-kernel CTA transforms (and the
row-space layout with them); every column goes through the same arithmetic, so runs
with different widths must give bit-identical fields and energies.  The tuner's
choice is therefore free to differ between processes.
"""
import numpy as np
import pytest

import pfc_b200 as P

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("model,L,M", [(P.MODEL_MISFIT, 1024, 1024), (P.MODEL_MISFIT, 256, 256),
                                       (P.MODEL_CVD, 512, 128), (P.MODEL_MISFIT, 128, 512)])
def test_every_tile_width_gives_identical_results(model, L, M):
    tuned, trials = P.tile_width(L, M)
    print(f"{L}x{M}: tuned width {tuned}, trials (ms per 8 steps) {trials}")
    widths = sorted(trials) if trials else [tuned]
    assert tuned in widths
    results = []
    try:
        for w in widths:
            P.set_tile_width(L, M, w)
            r = P.Run(P.default_params(model, L=L, M=M, seed=7))
            r.advance(30, analysis=True)
            phi, con = r.fields_f32()
            results.append((w, phi, con, r.energy()))
            r.close()
    finally:
        P.set_tile_width(L, M, tuned)
    w0, phi0, con0, e0 = results[0]
    for w, phi, con, e in results[1:]:
        assert np.array_equal(phi, phi0), (w0, w)
        assert np.array_equal(con, con0), (w0, w)
        assert e == e0


def test_tuner_reports_its_trials():
    w, trials = P.tile_width(1024, 1024)
    print("1024^2 tile width", w, "trials (ms per 8 steps):", trials)
    if trials:  # PFC_AUTOTUNE=0 leaves no trials
        assert set(trials) == {1, 2, 4, 8}
        assert all(ms > 0 for ms in trials.values())
        assert trials[w] == min(trials.values())
    assert P.tile_width(1024, 1024)[0] == w
    with pytest.raises(P.PfcError):
        P.set_tile_width(1024, 1024, 16)  # the tile would not fit


def test_batch_mixing_tile_widths_equals_single_runs():
    """Runs of one grid created before and after the width is changed keep their own
    layouts; a batch holding both advances each with its own width."""
    L = M = 256
    tuned, trials = P.tile_width(L, M)
    widths = sorted(trials) if len(trials) > 1 else [8, 16]
    try:
        runs = []
        for i, w in enumerate(widths):
            P.set_tile_width(L, M, w)
            runs.append(P.Run(P.default_params(P.MODEL_MISFIT, L=L, M=M, seed=100 + i)))
        batch = P.Batch(runs)
        batch.advance(20)
        singles = []
        for i, w in enumerate(widths):
            P.set_tile_width(L, M, w)
            r = P.Run(P.default_params(P.MODEL_MISFIT, L=L, M=M, seed=100 + i))
            r.advance(20)
            singles.append(r)
        for a, b in zip(runs, singles):
            fa, ca = a.fields_f32()
            fb, cb = b.fields_f32()
            assert np.array_equal(fa, fb) and np.array_equal(ca, cb)
        batch.close()
    finally:
        P.set_tile_width(L, M, tuned)
