"""GPU checks at the C2 scale (Misfit 1024 x 1024, seed 20200604, u0 0.05, con0 0.2).

  * the plain FP64 path in the reference's rounding mode against the CPU oracle (the
    bit-identical restatement of the reference program) over 5 steps at 1024^2: the
    FP64 path is the on-device oracle the fused paths are measured against;
  * the fused paths against the pure-FP64 path at steps 1000 and 10000, on the
    quantities that stay meaningful once the dynamics have amplified every rounding
    (fields decorrelate; the energy, the conserved mass and the number of atoms the
    Misfit peak finder counts do not);
  * Elastic Analysis of a 1024^2 checkpoint (about 10 k atoms): peak finder, elastic3D
    and cryst_order against the oracle, indices and neighbour counts bit for bit.
"""
import numpy as np
import pytest

import oracle as O
import pfc_b200 as P

pytestmark = pytest.mark.gpu

G = 1024
C2 = dict(seed=20200604, u0=0.05, con0=0.2)


def gpu(precision, **kw):
    return P.Run(P.default_params(P.MODEL_MISFIT, L=G, M=G, precision=precision, **{**C2, **kw}))


def test_fp64_path_matches_reference_oracle_at_1024():
    """5 steps of the FP64 path (reference float roundings) against the oracle in its
    reference-exact mode: last-bit FFT differences only, occasionally turned into one
    float ulp by the reference's float roundings (1e-6, the FP64 path's bar at 64^2)."""
    r = gpu(P.FP64)
    o = O.Run(O.default_params(O.MODEL_MISFIT, L=G, M=G, exact=1, **C2))
    r.advance(5)
    o.step(5)
    phi, con = r.fields()
    ophi, ocon = o.fields()
    err = max(np.abs(phi - ophi).max(), np.abs(con - ocon).max())
    print(f"FP64 path vs oracle at {G}^2, 5 steps: {err:.3e}")
    assert err <= 1e-6
    e, d = r.energy()
    oe, od = o.energy()
    assert abs(e - oe) <= 1e-9 * abs(oe) and abs(d - od) <= 1e-12


def atom_count(run):
    phi, con = run.fields_f32()
    return len(P.phimax_misfit(phi[:, :, 0], con[:, :, 0]))


# energy floors (relative to pure FP64) at steps 1000 and 10000, from B200 runs.  By step
# 1000 the dynamics have amplified every last-bit rounding difference into a different
# realisation of the same coarsening, and by step 10000 the fields have decorrelated, so the
# bar is the larger of the floor and twice the distance the reference's own float roundings
# (the FP64 path) put the energy from pure FP64 at that step.  Measured: mixed 1.0e-6 to
# 1.2e-5 and 7.5e-4; FP32 6.4e-5 and 5.6e-3.
ENERGY_FLOOR = {P.MIXED: (2e-5, 2e-3), P.FP32: (3e-4, 1.5e-2)}


@pytest.mark.parametrize("precision", [P.MIXED, P.FP32])
def test_fused_paths_long_run_statistics(precision):
    """Steps 1000 and 10000: the energy within max(floor, 2 x the reference's own rounding
    deviation), the mass within 1e-9 (it is the FP64 k = 0 mode), the Misfit atom count
    within 2 %."""
    a = gpu(precision)
    b = gpu(P.FP64_PURE)
    c = gpu(P.FP64)
    done = 0
    for target, floor in zip((1000, 10000), ENERGY_FLOOR[precision]):
        for x in (a, b, c):
            x.advance(target - done, analysis=x is a)
        done = target
        ea, ma = a.energy()
        eb, mb = b.energy()
        ec, _ = c.energy()
        na, nb = atom_count(a), atom_count(b)
        rel, ref = abs(ea - eb) / abs(eb), abs(ec - eb) / abs(eb)
        print(f"precision {precision} step {target}: e/P {ea:.9e} vs {eb:.9e} (rel {rel:.2e}; the reference's "
              f"roundings {ref:.2e}); mass {ma:.12f} vs {mb:.12f}; atoms {na} vs {nb}")
        assert rel <= max(floor, 2.0 * ref)
        assert abs(ma - mb) <= 1e-9
        assert abs(na - nb) <= 0.02 * nb


def test_elastic_analysis_at_1024_matches_oracle():
    """A 1024^2 checkpoint after 500 steps (about 9.7 k atoms; the crystal keeps growing
    towards the ~17 k of a fully ordered 1024^2 field): the Elastic peak finder's atoms
    (positions, Phimax), elastic3D's strains and neighbour counts, and cryst_order's
    q4/q6 against the oracle on the same Float32 field."""
    r = gpu(P.MIXED)
    r.advance(500, analysis=True)
    phi, _ = r.fields_f32()
    f = phi.reshape(G, G, 1).astype(np.float64)
    atoms = P.phimax_elastic(f)
    oatoms = O.phimax_elastic(f)
    print(f"{G}^2 checkpoint: {len(atoms)} atoms")
    assert len(atoms) > 5000
    assert np.array_equal(atoms, oatoms)
    x, y, z = (np.ascontiguousarray(atoms[:, k]) for k in range(3))
    strain, nb = P.elastic3d(x, y, z, G, G, 1)
    ostrain, onb = O.elastic3d(x, y, z, G, G, 1)
    assert np.array_equal(nb, onb)
    assert np.array_equal(strain, ostrain)
    q4, q6 = P.cryst_order(x, y, z, G, G, 1)
    oq4, oq6 = O.cryst_order(x, y, z, G, G, 1)
    assert np.abs(q4 - oq4).max() <= 1e-6 and np.abs(q6 - oq6).max() <= 1e-6
