"""GPU parity of the checkpoint analysis: peak finders, elastic3D, cryst_order.

Given the same field, the GPU and the oracle must agree bit for bit on atom
indices, positions and Phimax values, on neighbour counts and on strains (all
are IEEE arithmetic without fused multiply-adds).  q4/q6 involve cosf/sinf/acos/
atan, whose last bits may differ between CUDA and the C library: tolerance
1e-6 absolute on q4/q6.
"""
import os

import numpy as np
import pytest

import oracle as O
import pfc_b200 as P
from helpers import golden_case, phimax_elastic_lines, phimax_misfit_lines, strain_lines

pytestmark = pytest.mark.gpu


def field_after(model, L, M, steps, seed=20200604):
    o = O.Run(O.default_params(model, L=L, M=M, N=1, seed=seed))
    o.step(steps)
    phi, con = o.fields()
    return phi.astype(np.float32), con.astype(np.float32)


@pytest.mark.parametrize("L,M,steps", [(64, 64, 25), (128, 128, 40), (256, 256, 30), (128, 256, 10)])
def test_misfit_phimax_bitexact(L, M, steps):
    phi, con = field_after(O.MODEL_MISFIT, L, M, steps)
    got = P.phimax_misfit(phi[:, :, 0], con[:, :, 0])
    ref, raw = O.phimax_misfit(phi[:, :, 0].astype(np.float64), con[:, :, 0].astype(np.float64))
    assert raw > 0
    assert got.shape == ref.shape
    assert np.array_equal(got, ref)
    assert phimax_misfit_lines(got) == phimax_misfit_lines(ref)


def test_misfit_phimax_fallback_and_edges():
    """No local maximum at all -> the global-maximum fallback record; ties and the x edges."""
    L, M = 32, 64
    flat = np.full((L, M), 0.25, np.float32)
    con = np.full((L, M), 0.2, np.float32)
    got = P.phimax_misfit(flat, con)
    ref, raw = O.phimax_misfit(flat.astype(np.float64), con.astype(np.float64))
    assert raw == 0 and np.array_equal(got, ref)
    rng = np.random.default_rng(5)
    f = rng.integers(0, 3, size=(L, M)).astype(np.float32) * 0.5 - 0.2  # many plateaus and ties
    f[0, :] = 1.0  # maxima on the edge-replicated first row
    f[5, 7] = np.nan
    got = P.phimax_misfit(f, con)
    ref, _ = O.phimax_misfit(f.astype(np.float64), con.astype(np.float64))
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("name", ["misfit_64", "misfit_128_s7", "misfit_256_c1"])
def test_elastic_chain_on_reference_fields(name):
    d, meta, fields = golden_case(name)
    L, M, N = meta["grid"]
    for kd in meta["kept"]:
        if kd == 0:
            continue
        phi = fields[f"phi_{kd}"]
        got = P.phimax_elastic(phi)
        ref = O.phimax_elastic(phi.astype(np.float64))
        assert np.array_equal(got, ref)
        sub = f"{d}/elastic0"
        if os.path.exists(f"{sub}/Phimax_{kd}.txt"):
            assert phimax_elastic_lines(got) == open(f"{sub}/Phimax_{kd}.txt").read().splitlines()
        x, y, z = got[:, 0], got[:, 1], got[:, 2]
        for benchel in (1.7, 1.3):
            st, nb = P.elastic3d(x, y, z, L, M, N, benchel=benchel)
            rst, rnb = O.elastic3d(x, y, z, L, M, N, benchel=benchel)
            assert np.array_equal(nb, rnb)
            assert np.array_equal(st, rst)
        if os.path.exists(f"{sub}/strain_{kd}.txt"):
            st, nb = P.elastic3d(x, y, z, L, M, N)
            assert strain_lines(x, y, z, st, nb) == open(f"{sub}/strain_{kd}.txt").read().splitlines()
        q4, q6 = P.cryst_order(x, y, z, L, M, N)
        rq4, rq6 = O.cryst_order(x, y, z, L, M, N)
        assert np.abs(q4 - rq4).max() <= 1e-6
        assert np.abs(q6 - rq6).max() <= 1e-6


def test_elastic_peak_3d_and_wrap_quirks():
    """3-D field: the 27-point test with the reference's y/z wrap rules and x halo."""
    rng = np.random.default_rng(11)
    phi = rng.standard_normal((16, 16, 8)).astype(np.float32)
    phi[0, 0, 0] = 5.0
    phi[-1, -1, -1] = 4.5
    got = P.phimax_elastic(phi)
    ref = O.phimax_elastic(phi.astype(np.float64))
    assert np.array_equal(got, ref)
    x, y, z = ref[:, 0], ref[:, 1], ref[:, 2]
    st, nb = P.elastic3d(x, y, z, 16, 16, 8, benchel=3.0)
    rst, rnb = O.elastic3d(x, y, z, 16, 16, 8, benchel=3.0)
    assert np.array_equal(nb, rnb) and np.array_equal(st, rst)


def test_empty_and_single_atom_inputs():
    st, nb = P.elastic3d([], [], [], 8, 8, 1)
    assert len(st) == 0
    st, nb = P.elastic3d([1.0], [1.0], [0.125], 8, 8, 1)
    assert nb[0] == 0 and st[0] == 0.0
    q4, q6 = P.cryst_order([1.0], [1.0], [0.125], 8, 8, 1)
    assert q4[0] == 0.0 and q6[0] == 0.0


CVD_CASES = ["cvd_64", "cvd_128", "cvd_32x32x8"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", CVD_CASES)
def test_cvd_analysis_matches_oracle(name):
    """atompositionCFGC2 / GR / Q6_GLO (CVD:1067-1520) on the reference's checkpoint
    fields: threshold, atom records and histogram bit-exact; Q6 within 2e-6 (the GPU's
    acosf/atanf/cosf/sinf differ from the C library's in the last bits)."""
    from helpers import case_params
    d, meta, fields = golden_case(name)
    L, M, N = meta["grid"]
    u0 = float(np.float32(case_params(meta).get("u0", 0.01)))
    for kd in meta["checkpoints"]:
        phi = fields[f"phi_{kd}"]
        phic, pmax, rec = P.cvd_atoms(phi, u0)
        ophic, opmax, orec = O.cvd_atoms(phi, u0)
        assert phic == ophic and pmax == opmax
        assert rec.shape == orec.shape and np.array_equal(rec.view(np.uint32), orec.view(np.uint32))
        assert np.array_equal(P.cvd_gr_hist(rec, L, M, N), O.cvd_gr_hist(orec, L, M, N))
        nb, ql, qg = P.cvd_q6(rec, L, M, N)
        onb, oql, oqg, _ = O.cvd_q6(orec, L, M, N)
        assert np.array_equal(nb, onb)
        assert np.abs(ql - oql).max() <= 2e-6
        assert abs(float(qg) - float(oqg)) <= 2e-6


@pytest.mark.gpu
def test_cvd_analysis_without_atoms():
    """A field below the threshold everywhere: the reference's single (-1, -1, -1)
    record, no pairs in the histogram, no neighbours."""
    phi = np.full((32, 32, 1), -2.0, np.float32)
    phic, pmax, rec = P.cvd_atoms(phi, 0.05)
    ophic, opmax, orec = O.cvd_atoms(phi, 0.05)
    assert phic == ophic and pmax == opmax == np.float32(-1.0)
    assert rec.shape == (1, 4) and np.array_equal(rec, orec) and rec[0, 0] == -1.0
    assert not P.cvd_gr_hist(rec, 32, 32, 1).any()
    nb, ql, qg = P.cvd_q6(rec, 32, 32, 1)
    assert nb[0] == 0 and ql[0] == 0.0 and np.isnan(qg)
