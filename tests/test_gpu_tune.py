"""GPU tests of the column tile-width and staging autotuner.

The width only regroups the columns that one column-kernel CTA transforms (and the
row-space layout with them); every column goes through the same arithmetic, so runs
with different widths must give bit-identical fields and energies.  The staging
method (16-byte cp.async copies or one TMA bulk copy per tile) only changes how the
same bytes reach shared memory, so it must not change a bit either.  The tuner's
choice is therefore free to differ between processes.  Both fused precisions (mixed:
FP32 arrays with FP64 arithmetic; FP32) are tuned separately and tested alike.
"""
import numpy as np
import pytest

import pfc_b200 as P

pytestmark = pytest.mark.gpu

PRECS = [P.MIXED, P.FP32]


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("model,L,M", [(P.MODEL_MISFIT, 1024, 1024), (P.MODEL_MISFIT, 256, 256),
                                       (P.MODEL_CVD, 512, 128), (P.MODEL_MISFIT, 128, 512)])
def test_every_tile_width_gives_identical_results(model, L, M, prec):
    tuned, trials = P.tile_width(L, M, precision=prec)
    print(f"{L}x{M}: tuned width {tuned}, trials (ms per 8 steps) {trials}")
    widths = sorted(trials) if trials else [tuned]
    assert tuned in widths
    results = []
    try:
        for w in widths:
            P.set_tile_width(L, M, w, precision=prec)
            r = P.Run(P.default_params(model, L=L, M=M, seed=7, precision=prec))
            r.advance(30, analysis=True)
            phi, con = r.fields_f32()
            results.append((w, phi, con, r.energy()))
            r.close()
    finally:
        P.set_tile_width(L, M, tuned, precision=prec)
    w0, phi0, con0, e0 = results[0]
    for w, phi, con, e in results[1:]:
        assert np.array_equal(phi, phi0), (w0, w)
        assert np.array_equal(con, con0), (w0, w)
        assert e == e0


@pytest.mark.parametrize("prec,widths", [(P.MIXED, {1, 2, 4}), (P.FP32, {1, 2, 4, 8})])
def test_tuner_reports_its_trials(prec, widths):
    w, trials = P.tile_width(1024, 1024, precision=prec)
    print("1024^2 tile width", w, "trials (ms per 8 steps):", trials)
    if trials:  # PFC_AUTOTUNE=0 leaves no trials
        assert set(trials) == widths
        assert all(ms > 0 for ms in trials.values())
        assert trials[w] == min(trials.values())
    assert P.tile_width(1024, 1024, precision=prec)[0] == w
    stage, st_trials = P.col_staging(1024, 1024, precision=prec)
    print("1024^2 staging", stage, "trials (ms per 8 steps, async / bulk):", st_trials)
    assert stage in (P.STAGE_ASYNC, P.STAGE_BULK)
    if trials:
        assert set(st_trials) == set(trials)
        for c, (a, b) in st_trials.items():
            assert a > 0 and b > 0 and trials[c] == min(a, b)
        assert st_trials[w][stage] == trials[w]
    with pytest.raises(P.PfcError):
        P.set_tile_width(1024, 1024, 16, precision=prec)  # the tile would not fit
    with pytest.raises(P.PfcError):
        P.set_col_staging(1024, 1024, 2, precision=prec)  # no such method
    with pytest.raises(P.PfcError):
        P.tile_width(1024, 1024, precision=P.FP64)  # the plain FP64 path has no tiles


@pytest.mark.parametrize("prec", PRECS)
def test_batch_mixing_tile_widths_equals_single_runs(prec):
    """Runs of one grid created before and after the width is changed keep their own
    layouts; a batch holding both advances each with its own width."""
    L = M = 256
    tuned, trials = P.tile_width(L, M, precision=prec)
    widths = sorted(trials) if len(trials) > 1 else [4, 8]
    try:
        runs = []
        for i, w in enumerate(widths):
            P.set_tile_width(L, M, w, precision=prec)
            runs.append(P.Run(P.default_params(P.MODEL_MISFIT, L=L, M=M, seed=100 + i, precision=prec)))
        batch = P.Batch(runs)
        batch.advance(20)
        singles = []
        for i, w in enumerate(widths):
            P.set_tile_width(L, M, w, precision=prec)
            r = P.Run(P.default_params(P.MODEL_MISFIT, L=L, M=M, seed=100 + i, precision=prec))
            r.advance(20)
            singles.append(r)
        for a, b in zip(runs, singles):
            fa, ca = a.fields_f32()
            fb, cb = b.fields_f32()
            assert np.array_equal(fa, fb) and np.array_equal(ca, cb)
        batch.close()
    finally:
        P.set_tile_width(L, M, tuned, precision=prec)


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("model,L,M,width", [(P.MODEL_MISFIT, 1024, 1024, 2), (P.MODEL_MISFIT, 1024, 1024, 4),
                                             (P.MODEL_CVD, 512, 128, None), (P.MODEL_MISFIT, 64, 2048, None)])
def test_both_stagings_give_identical_results(model, L, M, width, prec):
    tuned, _ = P.tile_width(L, M, precision=prec)
    stage0, _ = P.col_staging(L, M, precision=prec)
    results = []
    try:
        if width:
            P.set_tile_width(L, M, width, precision=prec)
        for s in (P.STAGE_ASYNC, P.STAGE_BULK):
            P.set_col_staging(L, M, s, precision=prec)
            r = P.Run(P.default_params(model, L=L, M=M, seed=11, precision=prec))
            r.advance(25, analysis=True)  # the last step writes the checkpoint outputs
            phi, con = r.fields_f32()
            results.append((phi, con, r.energy()))
            r.close()
    finally:
        P.set_tile_width(L, M, tuned, precision=prec)
        P.set_col_staging(L, M, stage0, precision=prec)
    (pa, ca, ea), (pb, cb, eb) = results
    assert np.array_equal(pa, pb)
    assert np.array_equal(ca, cb)
    assert ea == eb


@pytest.mark.parametrize("prec", PRECS)
def test_batch_mixing_stagings_equals_single_runs(prec):
    L = M = 512
    tuned, _ = P.tile_width(L, M, precision=prec)
    stage0, _ = P.col_staging(L, M, precision=prec)
    try:
        runs, singles = [], []
        for i, s in enumerate((P.STAGE_ASYNC, P.STAGE_BULK)):
            P.set_col_staging(L, M, s, precision=prec)
            runs.append(P.Run(P.default_params(P.MODEL_MISFIT, L=L, M=M, seed=300 + i, precision=prec)))
            singles.append(P.Run(P.default_params(P.MODEL_MISFIT, L=L, M=M, seed=300 + i, precision=prec)))
        batch = P.Batch(runs)
        batch.advance(15)
        for r in singles:
            r.advance(15)
        for a, b in zip(runs, singles):
            fa, ca = a.fields_f32()
            fb, cb = b.fields_f32()
            assert np.array_equal(fa, fb) and np.array_equal(ca, cb)
        batch.close()
    finally:
        P.set_col_staging(L, M, stage0, precision=prec)
