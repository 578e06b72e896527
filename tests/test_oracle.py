"""The oracle (CPU restatement) pinned against the reference's own outputs.

The golden fixtures were produced by the unmodified reference program
(tests/golden/make_golden.py).  In reference-exact mode the restatement must
reproduce them bit for bit: the VTI Float32 values, energy.txt, and the Phimax,
strain and q4q6 text files.
"""
import numpy as np
import pytest

import oracle as O
from helpers import (case_params, cvd_phimax_lines, cvd_phimax_txt_lines, energy_line, golden_case, grq6_lines,
                     hist_lines, histq_lines, phimax_elastic_lines, phimax_misfit_lines, phiball_lines, q4q6_lines,
                     ql_lines, strain_lines)

MISFIT_CASES = ["misfit_64", "misfit_128_s7", "misfit_256_c1", "misfit_64_noise"]
CVD_CASES = ["cvd_64", "cvd_32x32x8", "cvd_128"]


def oracle_params(meta, exact=1):
    model = O.MODEL_MISFIT if meta["model"] == "misfit" else O.MODEL_CVD
    L, M, N = meta["grid"]
    p = O.default_params(model, L=L, M=M, N=N, exact=exact)
    kv = case_params(meta)
    for k in ("u0", "con0", "sig", "dt", "dx", "axx"):
        if k in kv:
            setattr(p, k, float(np.float32(kv[k])))
    if "seed" in kv:
        p.seed = int(kv["seed"])
    return p, int(kv["steps"]), int(kv["mod"])


def run_oracle_checkpoints(meta, exact=1):
    """Run the oracle through a golden case; yield (kd, phi, con, energy) at the reference's checkpoints."""
    p, steps, mod = oracle_params(meta, exact)
    r = O.Run(p)
    out = {}
    energies = []
    for t in range(steps):
        r.step()
        if meta["model"] == "misfit":
            if (t + 1) % mod == 0 or t + 1 == steps:
                phi, con = r.fields()
                out[t + 1] = (phi, con, r.energy())
                energies.append(energy_line(t + 1, *r.energy()))
        else:
            if t % mod == 0:
                phi, con = r.fields()
                out[t] = (phi, con, r.energy())
            energies.append(energy_line(t, *r.energy()))
    return out, energies


@pytest.mark.parametrize("name", MISFIT_CASES + CVD_CASES)
def test_oracle_reproduces_reference_run(name):
    d, meta, fields = golden_case(name)
    got, energies = run_oracle_checkpoints(meta)
    for kd in meta["kept"]:
        if kd == 0 and meta["model"] == "misfit":
            continue  # Misfit writes the initial condition as checkpoint 0; CVD writes the state after step 0
        phi, con, _ = got[kd]
        ref_phi, ref_con = fields[f"phi_{kd}"], fields[f"con_{kd}"]
        assert np.array_equal(phi.astype(np.float32).view(np.uint32), ref_phi.view(np.uint32)), f"phi {kd}"
        assert np.array_equal(con.astype(np.float32).view(np.uint32), ref_con.view(np.uint32)), f"con {kd}"
    ref_energy = open(f"{d}/energy.txt").read().splitlines()
    assert energies == ref_energy


@pytest.mark.parametrize("name", MISFIT_CASES)
def test_oracle_initial_condition(name):
    d, meta, fields = golden_case(name)
    if 0 not in meta["kept"]:
        pytest.skip("initial checkpoint not kept for this case")
    p, _, _ = oracle_params(meta)
    r = O.Run(p)
    phi, con = r.fields()
    assert np.array_equal(phi.astype(np.float32), fields["phi_0"])
    assert np.array_equal(con.astype(np.float32), fields["con_0"])


@pytest.mark.parametrize("name", MISFIT_CASES)
def test_oracle_misfit_phimax_text(name):
    d, meta, fields = golden_case(name)
    got, _ = run_oracle_checkpoints(meta)
    for kd in meta["kept"]:
        if kd == 0:
            continue
        phi, con, _ = got[kd]
        atoms, raw = O.phimax_misfit(phi[:, :, 0], con[:, :, 0], dx=0.125, con0=float(np.float32(case_params(meta).get("con0", 0.2))))
        assert raw > 0
        assert phimax_misfit_lines(atoms) == open(f"{d}/Phimax_{kd}.txt").read().splitlines()


@pytest.mark.parametrize("name", ["misfit_64", "misfit_128_s7", "misfit_256_c1"])
def test_oracle_elastic_texts(name):
    """Elastic peak finder, elastic3D and cryst_order on the reference's own VTI fields."""
    d, meta, fields = golden_case(name)
    import glob
    import json
    import os
    for sub in sorted(glob.glob(f"{d}/elastic*")):
        cj = json.load(open(f"{sub}/case.json"))
        benchel = 1.7
        if "--benchel" in cj["args"]:
            benchel = float(np.float32(cj["args"][cj["args"].index("--benchel") + 1]))
        L, M, N = meta["grid"]
        for kd in cj["steps"]:
            if not os.path.exists(f"{sub}/Phimax_{kd}.txt"):
                continue
            phi = fields[f"phi_{kd}"].astype(np.float64)
            atoms = O.phimax_elastic(phi)
            assert phimax_elastic_lines(atoms) == open(f"{sub}/Phimax_{kd}.txt").read().splitlines()
            x, y, z = atoms[:, 0], atoms[:, 1], atoms[:, 2]
            st, nb = O.elastic3d(x, y, z, L, M, N, benchel=benchel)
            assert strain_lines(x, y, z, st, nb) == open(f"{sub}/strain_{kd}.txt").read().splitlines()
            q4, q6 = O.cryst_order(x, y, z, L, M, N)
            assert q4q6_lines(x, y, z, q4, q6) == open(f"{sub}/q4q6_{kd}.txt").read().splitlines()


@pytest.mark.parametrize("shape", [(1, 8, 1), (4, 16, 1), (8, 4, 2), (2, 32, 4), (16, 16, 1), (3, 5, 1)])
def test_shim_dft_matches_numpy(shape):
    rng = np.random.default_rng(1)
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    f = O.dft3d(a, -1)
    b = O.dft3d(a, +1)
    ref_f = np.fft.fftn(a)
    ref_b = np.fft.ifftn(a) * a.size
    scale = np.abs(ref_f).max()
    assert np.abs(f - ref_f).max() <= 1e-13 * scale
    assert np.abs(b - ref_b).max() <= 1e-13 * scale


def test_splitmix64_stream():
    """pfc_common.h:165-181 generator against an independent Python restatement."""
    import ctypes

    def py_next(state):
        state = (state + 0x9E3779B97F4A7C15) & (2**64 - 1)
        z = state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & (2**64 - 1)
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & (2**64 - 1)
        return state, z ^ (z >> 31)

    st = ctypes.c_uint64(20200604)
    pst = 20200604
    for _ in range(100):
        v = O.lib().orc_splitmix64_next(ctypes.byref(st))
        pst, pv = py_next(pst)
        assert v == pv and st.value == pst


def test_pure_fp64_close_to_exact():
    """The pure-FP64 scheme differs from the reference's mixed precision only at float rounding level."""
    d, meta, fields = golden_case("misfit_64")
    pe, _, _ = oracle_params(meta, exact=1)
    pp, _, _ = oracle_params(meta, exact=0)
    a, b = O.Run(pe), O.Run(pp)
    a.step(20)
    b.step(20)
    fa, _ = a.fields()
    fb, _ = b.fields()
    diff = np.abs(fa - fb).max()
    assert 0 < diff < 1e-5


def text(path):
    return open(path).read().split("\n")[:-1]


@pytest.mark.parametrize("name", CVD_CASES)
def test_oracle_cvd_checkpoint_analysis(name):
    """atompositionCFGC2, GR and Q6_GLO (CVD:1067-1520) restated: every analysis file of
    every checkpoint of the reference run, byte for byte."""
    import os
    d, meta, fields = golden_case(name)
    L, M, N = meta["grid"]
    u0 = float(np.float32(case_params(meta).get("u0", 0.01)))
    phimax_txt = []
    for kd in meta["checkpoints"]:
        phic, pmax, rec = O.cvd_atoms(fields[f"phi_{kd}"], u0)
        phimax_txt += cvd_phimax_txt_lines(kd, phic, pmax)
        assert phiball_lines(rec, L, M, N, 0.125) == text(os.path.join(d, f"phiball_{kd}.cfg"))
        assert cvd_phimax_lines(rec, L, M, N, 0.125) == text(os.path.join(d, f"Phimax_{kd}.txt"))
        hist = O.cvd_gr_hist(rec, L, M, N)
        assert hist_lines(hist) == text(os.path.join(d, f"hist_{kd}.txt"))
        num_t = int((rec[:, 0] >= 0).sum())
        assert grq6_lines(hist, num_t, L, M, N, 0.125) == text(os.path.join(d, f"Grq6_{kd}.txt"))
        if kd % 20 == 0:
            nb, ql, qg, histq = O.cvd_q6(rec, L, M, N)
            assert ql_lines(nb, ql, qg) == text(os.path.join(d, f"Ql_{kd}.txt"))
            assert histq_lines(histq) == text(os.path.join(d, f"HistQ_{kd}.txt"))
        else:
            assert not os.path.exists(os.path.join(d, f"Ql_{kd}.txt"))
    assert phimax_txt == text(os.path.join(d, "phimax.txt"))


def test_cvd_3d_state_stays_independent_of_n():
    """The CVD initial condition (INITIAL_C2, cvd.cpp:587-642) does not depend on n, and the
    reference keeps it so exactly: its own 32 x 32 x 8 run's checkpoints, and the oracle in
    both modes over 60 steps, have no spread along n at all.  (A constant row transforms to
    one bin and back without rounding, and equal points give equal terms; the GPU path's
    tests hold it to the same.)"""
    _, _, fields = golden_case("cvd_32x32x8")
    for key, v in fields.items():
        a = v.reshape(32, 32, 8)
        assert (a.max(axis=2) - a.min(axis=2)).max() == 0.0, key
    for exact in (1, 0):
        o = O.Run(O.default_params(O.MODEL_CVD, L=32, M=32, N=8, exact=exact))
        o.step(60)
        for a in o.fields():
            a = a.reshape(32, 32, 8)
            assert (a.max(axis=2) - a.min(axis=2)).max() == 0.0, exact
