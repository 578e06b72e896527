"""GPU parity of the time step, initial conditions, FFT, mass and batching.

Every test calls the CUDA engine through its C ABI (pfc_b200 ctypes binding) and
checks it against the oracle (CPU restatement) and the reference fixtures.

Tolerances:
  * initial conditions: bit-exact (Float32) with the reference;
  * FP32 fused path: max-abs field error <= 1e-5 against the FP64 oracle over the
    first 20-25 steps at every size and 100 steps at 64^2; over 20 steps at most 8x the
    deviation the reference's own float roundings cause (reference-exact vs pure FP64
    on the FP64 GPU paths).  Beyond that the PFC dynamics amplify any rounding-level
    perturbation (the reference's own float roundings put it 3.6e-5 away from pure
    FP64 after 200 steps at 256^2), so the 200-step bound is 40x that amplified
    deviation;
  * stochastic noise: the FP32 path's noise spectrum has the reference generator's
    power in every |k| shell (statistical, 8 seeds);
  * CVD is chaotic at 200 steps (1e-7 -> 1.4e-2): fields are compared over the first
    20 steps, energy and mass after 200;
  * FP64 plain path, pure mode: <= 1e-11 against the pure-FP64 oracle (FFT algorithm
    and libm differences only); reference-exact mode: <= 1e-6, because the
    reference's float roundings turn last-bit double differences into occasional
    float-ulp differences;
  * FFT: <= 1e-12 relative to numpy.
"""
import numpy as np
import pytest

import oracle as O
import pfc_b200 as P
from helpers import golden_case

pytestmark = pytest.mark.gpu


def oracle_run(model, L, M, N=1, exact=1, **kw):
    p = O.default_params(model, L=L, M=M, N=N, exact=exact, **kw)
    return O.Run(p)


def gpu_run(model, L, M, N=1, precision=P.FP32, **kw):
    p = P.default_params(model, L=L, M=M, N=N, precision=precision, **kw)
    return P.Run(p)


@pytest.mark.parametrize("shape", [(8, 16, 1), (64, 64, 1), (32, 32, 8), (256, 128, 1), (2, 4, 2048), (2048, 2, 1)])
def test_dft3d_matches_numpy(shape):
    rng = np.random.default_rng(3)
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    for sign, ref in ((-1, np.fft.fftn(a)), (1, np.fft.ifftn(a) * a.size)):
        got = P.dft3d(a, sign)
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("name", ["misfit_64", "misfit_128_s7"])
def test_misfit_initial_condition_bitexact(name):
    d, meta, fields = golden_case(name)
    L, M, N = meta["grid"]
    kv = dict(zip(meta["args"][::2], meta["args"][1::2]))
    kw = {}
    if "--seed" in kv:
        kw["seed"] = int(kv["--seed"])
    for k in ("u0", "con0"):
        if f"--{k}" in kv:
            kw[k] = float(np.float32(kv[f"--{k}"]))
    r = gpu_run(P.MODEL_MISFIT, L, M, **kw)
    phi, con = r.fields_f32()
    assert np.array_equal(phi.view(np.uint32), fields["phi_0"].view(np.uint32))
    assert np.array_equal(con.view(np.uint32), fields["con_0"].view(np.uint32))


@pytest.mark.parametrize("model,L,M", [(P.MODEL_MISFIT, 256, 256), (P.MODEL_MISFIT, 1024, 512), (P.MODEL_CVD, 128, 64),
                                       (P.MODEL_MISFIT, 64, 2048)])
def test_initial_condition_matches_oracle(model, L, M):
    r = gpu_run(model, L, M)
    o = oracle_run(model, L, M)
    phi, con = r.fields_f32()
    ophi, ocon = o.fields()
    assert np.array_equal(phi, ophi.astype(np.float32))
    assert np.array_equal(con, ocon.astype(np.float32))


@pytest.mark.parametrize("precision,exact,tol", [(P.FP64, 1, 1e-6), (P.FP64_PURE, 0, 1e-11)])
def test_fp64_path_matches_oracle(precision, exact, tol):
    r = gpu_run(P.MODEL_MISFIT, 64, 64, precision=precision)
    o = oracle_run(P.MODEL_MISFIT, 64, 64, exact=exact)
    r.advance(20)
    o.step(20)
    phi, con = r.fields()
    ophi, ocon = o.fields()
    assert np.abs(phi - ophi).max() <= tol
    assert np.abs(con - ocon).max() <= tol
    e, d = r.energy()
    oe, od = o.energy()
    assert abs(e - oe) <= 1e3 * tol * abs(oe) + 1e-12 and abs(d - od) <= 1e-12


def test_fp64_path_cvd_3d_matches_reference():
    d, meta, fields = golden_case("cvd_32x32x8")
    r = gpu_run(P.MODEL_CVD, 32, 32, 8, precision=P.FP64)
    r.advance(1)
    phi, con = r.fields()
    assert np.abs(phi - fields["phi_0"]).max() <= 1e-6
    assert np.abs(con - fields["con_0"]).max() <= 1e-6
    r.advance(10)
    phi, con = r.fields()
    assert np.abs(phi - fields["phi_10"]).max() <= 1e-6


def reference_rounding_noise(model, L, M, steps, **kw):
    """Max-abs difference between the reference's mixed precision and pure FP64 after
    `steps` (both on the FP64 GPU path): the perturbation the reference itself carries."""
    a = gpu_run(model, L, M, precision=P.FP64, **kw)
    b = gpu_run(model, L, M, precision=P.FP64_PURE, **kw)
    a.advance(steps)
    b.advance(steps)
    fa, ca = a.fields()
    fb, cb = b.fields()
    return max(np.abs(fa - fb).max(), np.abs(ca - cb).max()), (fb, cb)


@pytest.mark.parametrize("model,L,M,steps", [(P.MODEL_MISFIT, 64, 64, 100), (P.MODEL_MISFIT, 128, 128, 25),
                                             (P.MODEL_MISFIT, 256, 256, 25), (P.MODEL_CVD, 64, 64, 20),
                                             (P.MODEL_MISFIT, 128, 64, 25), (P.MODEL_MISFIT, 64, 256, 25),
                                             (P.MODEL_MISFIT, 512, 512, 20), (P.MODEL_MISFIT, 256, 32, 25),
                                             (P.MODEL_MISFIT, 32, 256, 25), (P.MODEL_CVD, 32, 32, 20),
                                             (P.MODEL_MISFIT, 2048, 64, 10), (P.MODEL_MISFIT, 64, 2048, 10)])
def test_fp32_path_matches_fp64_oracle(model, L, M, steps):
    """Absolute 1e-5 against the CPU pure-FP64 oracle before chaotic amplification sets in."""
    r = gpu_run(model, L, M)
    o = oracle_run(model, L, M, exact=0)
    r.advance(steps, analysis=True)
    o.step(steps)
    phi, con = r.fields()
    ophi, ocon = o.fields()
    err_phi = np.abs(phi - ophi).max()
    err_con = np.abs(con - ocon).max()
    assert err_phi <= 1e-5, err_phi
    assert err_con <= 1e-5, err_con
    e, d = r.energy()
    oe, od = o.energy()
    assert abs(e - oe) <= 1e-5 * abs(oe) + 1e-7
    # FP32 field-sum rounding scales with the field amplitude, not the (possibly small) mean
    assert abs(d - od) <= 1e-7 * abs(od) + 5e-9


@pytest.mark.parametrize("model,L", [(P.MODEL_MISFIT, 64), (P.MODEL_MISFIT, 128), (P.MODEL_MISFIT, 256),
                                     (P.MODEL_MISFIT, 1024), (P.MODEL_CVD, 64)])
def test_fp32_rounding_injection_vs_reference(model, L):
    """20 steps, before the dynamics amplify perturbations: the FP32 path's deviation from
    pure FP64 is at most 8x the deviation the reference's own float roundings (cmix, Rhat,
    the C2 tables) cause over the same steps (measured 2.4x to 5.4x)."""
    noise, (phi64, con64) = reference_rounding_noise(model, L, L, 20)
    r = gpu_run(model, L, L)
    r.advance(20, analysis=True)
    phi, con = r.fields()
    err = max(np.abs(phi - phi64).max(), np.abs(con - con64).max())
    print(f"model={model} L={L}: FP32 deviation {err:.3e}, reference rounding deviation {noise:.3e}")
    assert err <= 8 * noise


@pytest.mark.parametrize("L", [64, 128, 256, 1024])
def test_fp32_error_after_200_steps(L):
    """200 steps.  The Misfit dynamics amplify any rounding perturbation (the reference's
    own float roundings grow from 4e-8..5e-7 at step 20 to 7e-7..4e-5 at step 200), so
    the FP32 deviation is bounded against that amplified reference deviation; measured
    ratios lie between 2.5x and 17x depending on the grid's unstable modes."""
    noise, (phi64, con64) = reference_rounding_noise(P.MODEL_MISFIT, L, L, 200)
    r = gpu_run(P.MODEL_MISFIT, L, L)
    r.advance(200, analysis=True)
    phi, con = r.fields()
    err = max(np.abs(phi - phi64).max(), np.abs(con - con64).max())
    print(f"L={L}: FP32 deviation {err:.3e}, reference rounding deviation {noise:.3e}")
    assert err <= max(1e-5, 40 * noise)


def test_cvd_long_run_energy_and_mass():
    """CVD after 200 steps: the fields are past the point where rounding perturbations
    have grown to O(0.1) (the reference's own float roundings reach 2e-4 by step 200 and
    keep growing), but the integral quantities stay close to FP64.  The energy e/P is a
    cancellation of O(0.1) densities down to about 1.6e-4, so its bound is absolute."""
    a = gpu_run(P.MODEL_CVD, 64, 64)
    b = gpu_run(P.MODEL_CVD, 64, 64, precision=P.FP64_PURE)
    a.advance(200, analysis=True)
    b.advance(200)
    ea, ma = a.energy()
    eb, mb = b.energy()
    print(f"CVD 64^2 step 200: e/P {ea:.6e} vs FP64 {eb:.6e}")
    assert abs(ea - eb) <= 5e-5
    assert abs(ma - mb) <= 1e-9


def test_fp32_c1_matches_reference_run():
    """C1: Misfit 256^2, 200 steps, against the reference program's own checkpoints."""
    d, meta, fields = golden_case("misfit_256_c1")
    r = gpu_run(P.MODEL_MISFIT, 256, 256, seed=20200604, u0=0.05, con0=0.2)
    r.advance(25, analysis=True)
    phi, con = r.fields_f32()
    assert np.abs(phi - fields["phi_25"]).max() <= 1e-5
    r.advance(175, analysis=True)
    phi, con = r.fields_f32()
    noise, _ = reference_rounding_noise(P.MODEL_MISFIT, 256, 256, 200, seed=20200604, u0=0.05, con0=0.2)
    err = max(np.abs(phi - fields["phi_200"]).max(), np.abs(con - fields["con_200"]).max())
    print(f"C1 step 200: FP32 error vs reference run {err:.3e}; reference rounding noise {noise:.3e}")
    assert err <= max(1e-5, 8 * noise)
    lines = open(f"{d}/energy.txt").read().split()
    e_ref, m_ref = float(lines[-2]), float(lines[-1])
    e, m = r.energy()
    assert abs(e - e_ref) <= 1e-4 * abs(e_ref)
    assert abs(m - m_ref) <= 1e-6


def test_mass_is_conserved():
    """The FP64 k = 0 modes are exact invariants; the FP64 sum over the FP32 real-space
    field carries a rounding deviation of order 1e-8 that does not accumulate: it
    stays below 1e-7 relative over 2000 steps (a drift of the mean would grow with the
    step count and leave that bound)."""
    r = gpu_run(P.MODEL_MISFIT, 256, 256)
    m0 = r.means()
    devs = []
    for n in (10, 90, 400, 1500):
        r.advance(n, analysis=True)
        assert r.means() == m0
        _, mass = r.energy()
        devs.append(abs(mass - m0[0]) / abs(m0[0]))
    print("relative field-sum deviations:", devs)
    assert max(devs) <= 1e-7


def test_batch_results_equal_single_runs():
    shapes = [(128, 128), (256, 256), (128, 128), (512, 512), (256, 128)]
    singles, batched = [], []
    for i, (L, M) in enumerate(shapes):
        kw = dict(seed=1000 + i, u0=0.02 + 0.03 * (i % 4), con0=0.1 + 0.1 * (i % 4))
        singles.append(gpu_run(P.MODEL_MISFIT, L, M, **kw))
        batched.append(gpu_run(P.MODEL_MISFIT, L, M, **kw))
    b = P.Batch(batched)
    b.advance(37)
    for s in singles:
        s.advance(37)
    for s, t in zip(singles, batched):
        a, _ = s.fields_f32()
        c, _ = t.fields_f32()
        assert np.array_equal(a.view(np.uint32), c.view(np.uint32))


def test_set_fields_roundtrip_and_steps():
    o = oracle_run(P.MODEL_MISFIT, 64, 64, exact=0)
    o.step(5)
    phi, con = o.fields()
    r = gpu_run(P.MODEL_MISFIT, 64, 64)
    r.set_fields(phi, con)
    a, b = r.fields()
    assert np.abs(a - phi).max() <= 1e-6 and np.abs(b - con).max() <= 1e-6
    r.advance(50, analysis=True)
    o.step(50)
    a, _ = r.fields()
    assert np.abs(a - o.fields()[0]).max() <= 1e-5
    assert r.steps == 50


def test_invalid_arguments_raise():
    with pytest.raises(P.PfcError):
        gpu_run(P.MODEL_MISFIT, 100, 64)
    with pytest.raises(P.PfcError):
        gpu_run(P.MODEL_MISFIT, 64, 64, 4)
    r = gpu_run(P.MODEL_MISFIT, 64, 64)
    with pytest.raises(P.PfcError):
        r.energy()  # no analysis step yet


def noise_increment_power(make_run, seeds, L, axx, fields):
    """Radially binned |FFT|^2 of the one-step difference between a run with noise and
    the same run without: exactly the noise term of the psi update."""
    kx = np.fft.fftfreq(L) * L
    kr = np.sqrt(kx[:, None] ** 2 + kx[None, :] ** 2)
    shells = [(0.5, 4), (4, 8), (8, 12), (12, 15), (17, 40)]
    power = np.zeros(len(shells))
    for s in seeds:
        a, b = make_run(s, axx), make_run(s, 0.0)
        d = fields(a) - fields(b)
        ps = np.abs(np.fft.fft2(d)) ** 2
        for i, (lo, hi) in enumerate(shells):
            power[i] += ps[(kr >= lo) & (kr < hi)].mean()
    return power / len(seeds)


def test_noise_spectrum_matches_reference_generator():
    """--axx > 0: the FP32 path draws the noise spectrum directly (documented stream,
    not the reference's sequence), the oracle runs the reference's sequential polar
    Box-Muller generator.  One step's noise increment must have the same power in
    every |k| shell (8 seeds; the shells hold 50-350 modes each, so ~5 % sampling
    error), none above the 2 pi lowpass, and none at k = 0 (mass)."""
    L, axx, seeds = 128, 0.005, range(8)

    def gpu(s, a):
        r = gpu_run(P.MODEL_MISFIT, L, L, seed=100 + s, axx=a)
        r.advance(1, analysis=True)
        return r

    def orc(s, a):
        o = oracle_run(P.MODEL_MISFIT, L, L, seed=100 + s, axx=a)
        o.step(1)
        return o

    pg = noise_increment_power(gpu, seeds, L, axx, lambda r: r.fields()[0].reshape(L, L))
    po = noise_increment_power(orc, seeds, L, axx, lambda o: o.fields()[0].reshape(L, L))
    print("shell power GPU / oracle:", pg[:4] / po[:4], "above cutoff:", pg[4], po[4])
    assert np.all(np.abs(pg[:4] / po[:4] - 1.0) < 0.25)
    assert abs(pg[:4].sum() / po[:4].sum() - 1.0) < 0.12
    assert pg[4] < 1e-4 * pg[:4].max()
    # the noise adds nothing to the conserved mean
    r = gpu_run(P.MODEL_MISFIT, L, L, seed=5, axx=axx)
    m0 = r.means()
    r.advance(10, analysis=True)
    assert r.means() == m0


def test_noise_stream_is_deterministic_and_per_step():
    def run(seed, steps):
        r = gpu_run(P.MODEL_MISFIT, 64, 64, seed=seed, axx=0.005)
        r.advance(steps, analysis=True)
        return r.fields_f32()[0]
    a, b = run(3, 5), run(3, 5)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert not np.array_equal(a, run(4, 5))
    # a batch advances each run's own noise stream exactly as alone
    singles = [gpu_run(P.MODEL_MISFIT, 64, 64, seed=9, axx=0.005), gpu_run(P.MODEL_MISFIT, 128, 64, seed=2, axx=0.01)]
    batched = [gpu_run(P.MODEL_MISFIT, 64, 64, seed=9, axx=0.005), gpu_run(P.MODEL_MISFIT, 128, 64, seed=2, axx=0.01)]
    bt = P.Batch(batched)
    bt.advance(20)
    for s in singles:
        s.advance(20)
    for s, t in zip(singles, batched):
        assert np.array_equal(s.fields_f32()[0].view(np.uint32), t.fields_f32()[0].view(np.uint32))


def test_fp64_noise_matches_reference_run():
    """--axx > 0 on the plain FP64 path runs the reference's own sequential generator
    (Gauss, MIS:951-981) on the host, so the reference-exact mode follows the reference
    program's noisy run (golden case: 64^2, --axx 0.005 --seed 11) within the FP64
    path's bar, and the pure mode follows the oracle's pure mode."""
    d, meta, fields = golden_case("misfit_64_noise")
    r = gpu_run(P.MODEL_MISFIT, 64, 64, precision=P.FP64, seed=11, axx=float(np.float32(0.005)))
    for kd in (3, 6):
        r.advance(3)
        phi, con = r.fields_f32()
        err = max(np.abs(phi - fields[f"phi_{kd}"]).max(), np.abs(con - fields[f"con_{kd}"]).max())
        print(f"FP64 path with noise, step {kd}: {err:.3e} from the reference run")
        assert err <= 1e-6
    a = gpu_run(P.MODEL_MISFIT, 64, 64, precision=P.FP64_PURE, seed=11, axx=0.005)
    o = oracle_run(P.MODEL_MISFIT, 64, 64, exact=0, seed=11, axx=0.005)
    a.advance(6)
    o.step(6)
    assert np.abs(a.fields()[0] - o.fields()[0]).max() <= 1e-11
    # the noise moved the fields: the same run without it differs
    q = gpu_run(P.MODEL_MISFIT, 64, 64, precision=P.FP64, seed=11)
    q.advance(6)
    assert np.abs(q.fields_f32()[0] - fields["phi_6"]).max() > 1e-4
