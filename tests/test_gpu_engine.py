"""The engine (pfc_engine_create / pfc_submit / pfc_poll ...): continuous batching of
Misfit / CVD runs and Elastic analyses on one GPU.

Each run's kernels do not depend on the other runs in its launches, so a job's
results must be bit-for-bit the same alone, in any mix, and from pfc-exp-cli; these
tests hold the engine to that, and check admission by memory budget, cancellation and
the Elastic jobs that read a finished run's fields.
"""
import filecmp
import os
import subprocess
import time

import numpy as np
import pytest

import pfc_b200 as P

pytestmark = pytest.mark.gpu


def params(model, L, M, **kw):
    return P.default_params(model, L=L, M=M, **kw)


def drain(eng, ids, timeout_s=180):
    """Wait until every job in ids has finished; returns {id: [events]}."""
    out = {i: [] for i in ids}
    left = set(ids)
    t_end = time.time() + timeout_s
    while left and time.time() < t_end:
        for ev in eng.wait(timeout_ms=1000):
            out.setdefault(ev.job, []).append(ev)
            if ev.type in (P.EV_DONE, P.EV_FAILED, P.EV_CANCELLED):
                left.discard(ev.job)
    assert not left, f"jobs not finished: {left}"
    return out


def single_run(model, L, M, steps, mod, **kw):
    """The same run advanced alone with the CLI's sequence (analysis at checkpoints)."""
    r = P.Run(params(model, L, M, **kw))
    energies = []
    if model == P.MODEL_MISFIT:
        t = 0
        while t < steps:
            nxt = min(steps, (t // mod + 1) * mod)
            r.advance(nxt - t, analysis=True)
            t = nxt
            energies.append(r.energy())
    else:
        for _ in range(steps):
            r.advance(1, analysis=True)
            energies.append(r.energy())
    return r.fields_f32(), energies


def same_bits(a, b):
    a = np.ascontiguousarray(a, np.float32).ravel()
    b = np.ascontiguousarray(b, np.float32).ravel()
    return np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_engine_job_equals_single_run():
    eng = P.Engine()
    jid = eng.submit(P.JOB_MISFIT, params(P.MODEL_MISFIT, 128, 128, seed=11), steps=60, mod=25)
    evs = drain(eng, [jid])[jid]
    phi, con = eng.fields(jid)
    (rphi, rcon), energies = single_run(P.MODEL_MISFIT, 128, 128, 60, 25, seed=11)
    assert same_bits(phi, rphi) and same_bits(con, rcon)
    ck = [e for e in evs if e.type == P.EV_CHECKPOINT]
    assert [e.step for e in ck] == [25, 50, 60]
    assert [(e.energy, e.mass) for e in ck] == energies
    assert evs[0].type == P.EV_ADMITTED and evs[-1].type == P.EV_DONE and evs[-1].step == 60
    eng.close()


def test_engine_cvd_job_equals_single_run():
    eng = P.Engine(quantum_steps=40)
    jid = eng.submit(P.JOB_CVD, params(P.MODEL_CVD, 64, 64, seed=8), steps=45, mod=20)
    evs = drain(eng, [jid])[jid]
    (rphi, rcon), energies = single_run(P.MODEL_CVD, 64, 64, 45, 20, seed=8)
    phi, con = eng.fields(jid)
    assert same_bits(phi, rphi) and same_bits(con, rcon)
    ck = [e for e in evs if e.type == P.EV_CHECKPOINT]
    assert [e.step for e in ck] == [0, 20, 40]  # CVD writes after steps 1, 21, 41 (kd = t)
    assert [(e.energy, e.mass) for e in ck] == [energies[0], energies[20], energies[40]]
    eng.close()


def test_engine_results_same_alone_and_in_mix():
    target = dict(model=P.MODEL_MISFIT, L=128, M=64, seed=5, u0=0.08, con0=0.3)
    cvd = dict(model=P.MODEL_CVD, L=64, M=64, seed=3)

    def submit(eng, spec, steps, mod):
        spec = dict(spec)
        model = spec.pop("model")
        L, M = spec.pop("L"), spec.pop("M")
        kind = P.JOB_CVD if model == P.MODEL_CVD else P.JOB_MISFIT
        return eng.submit(kind, params(model, L, M, **spec), steps=steps, mod=mod)

    alone = P.Engine()
    a = submit(alone, target, 70, 20)
    ev_a = drain(alone, [a])
    fa = alone.fields(a)
    b = submit(alone, cvd, 33, 10)
    ev_b = drain(alone, [b])
    fb = alone.fields(b)
    alone.close()

    mix = P.Engine(quantum_steps=48)
    others = [submit(mix, dict(model=P.MODEL_MISFIT, L=256, M=256, seed=1), 90, 30),
              submit(mix, dict(model=P.MODEL_MISFIT, L=64, M=64, seed=2), 17, 7)]
    a2 = submit(mix, target, 70, 20)
    time.sleep(0.05)  # let the first jobs start so that the next ones join a running batch
    others.append(submit(mix, dict(model=P.MODEL_CVD, L=128, M=128, seed=4), 40, 13))
    b2 = submit(mix, cvd, 33, 10)
    others.append(submit(mix, dict(model=P.MODEL_MISFIT, L=128, M=64, seed=9), 50, 50))
    ev_mix = drain(mix, [a2, b2] + others)
    assert all(v[-1].type == P.EV_DONE for v in ev_mix.values())
    for x, y in zip(fa, mix.fields(a2)):
        assert same_bits(x, y)
    for x, y in zip(fb, mix.fields(b2)):
        assert same_bits(x, y)

    def ckpts(evs):
        return [(e.step, e.energy, e.mass, e.atoms) for e in evs if e.type == P.EV_CHECKPOINT]

    assert ckpts(ev_a[a]) == ckpts(ev_mix[a2])
    assert ckpts(ev_b[b]) == ckpts(ev_mix[b2])
    mix.close()


def test_engine_fails_a_nonfinite_run_alone():
    """A run whose fields go NaN (con0 > 1 puts log((1 - c) / (1 - c0)) out of its domain,
    a host-side way to make one run fail) gets PFC_EV_FAILED with PFC_E_NONFINITE; the
    runs batched with it finish, bit for bit as when they run alone."""
    good = [params(P.MODEL_MISFIT, 128, 128, seed=11), params(P.MODEL_MISFIT, 128, 128, seed=12),
            params(P.MODEL_CVD, 64, 64, seed=3)]
    kinds = [P.JOB_MISFIT, P.JOB_MISFIT, P.JOB_CVD]
    alone = P.Engine()
    ref = []
    for k, p in zip(kinds, good):
        j = alone.submit(k, p, steps=60, mod=30)
        drain(alone, [j])
        ref.append(alone.fields(j))
    alone.close()
    mix = P.Engine(quantum_steps=32)
    bad = mix.submit(P.JOB_MISFIT, params(P.MODEL_MISFIT, 128, 128, seed=13, con0=1.5), steps=60, mod=30)
    ids = [mix.submit(k, p, steps=60, mod=30) for k, p in zip(kinds, good)]
    ev = drain(mix, [bad] + ids)
    last = ev[bad][-1]
    assert last.type == P.EV_FAILED and last.status == P.PFC_E_NONFINITE, (last.type, last.status)
    assert last.step <= 32  # caught at the end of its first quantum
    for j, (rphi, rcon) in zip(ids, ref):
        assert ev[j][-1].type == P.EV_DONE
        phi, con = mix.fields(j)
        assert same_bits(phi, rphi) and same_bits(con, rcon)
    mix.close()


def test_run_reports_nonfinite_fields():
    r = P.Run(params(P.MODEL_MISFIT, 64, 64, con0=1.5))
    r.advance(2)
    assert r.nonfinite()
    assert not r.nonfinite()  # the flag is cleared once reported
    ok = P.Run(params(P.MODEL_MISFIT, 64, 64))
    ok.advance(5)
    assert not ok.nonfinite()


def run_cli(args, outdir):
    subprocess.run([P.CLI_PATH] + args + ["--outdir", outdir], check=True, stdout=subprocess.DEVNULL,
                   stderr=subprocess.DEVNULL)


@pytest.mark.parametrize("model", ["misfit", "cvd"])
def test_engine_files_equal_cli_files(tmp_path, model):
    steps, mod = (50, 20) if model == "misfit" else (25, 10)
    cli_dir, eng_dir = str(tmp_path / "cli"), str(tmp_path / "eng")
    run_cli(["--model", model, "--grid", "64x128x1", "--steps", str(steps), "--mod", str(mod), "--seed", "77"],
            cli_dir)
    eng = P.Engine()
    m = P.MODEL_MISFIT if model == "misfit" else P.MODEL_CVD
    jid = eng.submit(P.JOB_MISFIT if model == "misfit" else P.JOB_CVD, params(m, 64, 128, seed=77), steps=steps,
                     mod=mod, outdir=eng_dir)
    drain(eng, [jid])
    eng.close()
    names = sorted(n for n in os.listdir(cli_dir) if n != "checkpoint_timestamps.txt")
    assert names == sorted(n for n in os.listdir(eng_dir) if n != "checkpoint_timestamps.txt")
    assert any(n.endswith(".vti") for n in names) and "energy.txt" in names
    for n in names:
        assert filecmp.cmp(os.path.join(cli_dir, n), os.path.join(eng_dir, n), shallow=False), n
    cli_ts = open(os.path.join(cli_dir, "checkpoint_timestamps.txt")).read().split("\n")
    eng_ts = open(os.path.join(eng_dir, "checkpoint_timestamps.txt")).read().split("\n")
    assert [l.split(" timestamp_ms")[0] for l in cli_ts] == [l.split(" timestamp_ms")[0] for l in eng_ts]


def test_engine_admission_respects_budget():
    one = P.run_bytes(params(P.MODEL_MISFIT, 256, 256))
    eng = P.Engine(hbm_budget_bytes=2.5 * one)
    ids = [eng.submit(P.JOB_MISFIT, params(P.MODEL_MISFIT, 256, 256, seed=i), steps=40, mod=40) for i in range(6)]
    evs = drain(eng, ids)
    # residency: admission to the moment the run's memory was returned
    timeline = sorted([(e.t_event, 1) for v in evs.values() for e in v if e.type == P.EV_ADMITTED] +
                      [(e.t_finish, -1) for v in evs.values() for e in v if e.type == P.EV_DONE])
    active = peak = 0
    for _, d in timeline:
        active += d
        peak = max(peak, active)
    assert peak == 2
    assert all(v[-1].type == P.EV_DONE for v in evs.values())
    admit_order = sorted(ids, key=lambda i: next(e.t_event for e in evs[i] if e.type == P.EV_ADMITTED))
    assert admit_order == ids  # admission follows submission order
    eng.close()


def test_engine_cancel_and_max_active():
    eng = P.Engine(max_active=1)
    long_job = eng.submit(P.JOB_MISFIT, params(P.MODEL_MISFIT, 512, 512), steps=100000, mod=100000)
    queued = eng.submit(P.JOB_MISFIT, params(P.MODEL_MISFIT, 64, 64), steps=10, mod=10)
    first = eng.wait(timeout_ms=20000)
    assert first and first[0].job == long_job and first[0].type == P.EV_ADMITTED
    assert all(e.job == long_job for e in first)  # the second job waits for the slot
    eng.cancel(long_job)
    evs = drain(eng, [long_job, queued])
    assert evs[long_job][-1].type == P.EV_CANCELLED
    assert evs[queued][-1].type == P.EV_DONE
    with pytest.raises(P.PfcError):
        eng.cancel(long_job)
    eng.close()


def test_engine_elastic_on_finished_run():
    eng = P.Engine()
    src = eng.submit(P.JOB_MISFIT, params(P.MODEL_MISFIT, 128, 128, seed=21), steps=30, mod=30)
    ela = eng.submit(P.JOB_ELASTIC, params(P.MODEL_MISFIT, 128, 128), source_job=src)
    evs = drain(eng, [src, ela])
    assert evs[ela][-1].type == P.EV_DONE
    ck = [e for e in evs[ela] if e.type == P.EV_CHECKPOINT]
    assert len(ck) == 1 and ck[0].step == 30
    phi, _ = eng.fields(src)
    atoms = P.phimax_elastic(phi.reshape(128, 128, 1), dx=0.125)
    assert ck[0].atoms == int((atoms[:, 0] >= 0).sum()) and ck[0].atoms > 0
    eng.release(src)
    with pytest.raises(P.PfcError):
        eng.fields(src)
    eng.close()


def test_engine_elastic_on_input_dir_equals_cli(tmp_path):
    d, cli_out, eng_out = str(tmp_path / "in"), str(tmp_path / "cli"), str(tmp_path / "eng")
    run_cli(["--model", "misfit", "--grid", "128x128x1", "--steps", "20", "--mod", "10", "--seed", "3"], d)
    run_cli(["--model", "elastic", "--input-dir", d], cli_out)
    eng = P.Engine()
    jid = eng.submit(P.JOB_ELASTIC, params(P.MODEL_MISFIT, 128, 128), input_dir=d, outdir=eng_out)
    evs = drain(eng, [jid])[jid]
    eng.close()
    assert [e.step for e in evs if e.type == P.EV_CHECKPOINT] == [10, 20]
    for kd in (10, 20):
        for pre in ("Phimax_", "strain_", "q4q6_"):
            n = f"{pre}{kd}.txt"
            assert filecmp.cmp(os.path.join(cli_out, n), os.path.join(eng_out, n), shallow=False), n


def test_engine_rejects_bad_jobs():
    eng = P.Engine()
    with pytest.raises(P.PfcError):
        eng.submit(P.JOB_MISFIT, params(P.MODEL_MISFIT, 64, 64, precision=P.FP64), steps=10, mod=5)
    with pytest.raises(P.PfcError):
        eng.submit(P.JOB_MISFIT, params(P.MODEL_MISFIT, 64, 64), steps=0, mod=5)
    with pytest.raises(P.PfcError):
        eng.submit(P.JOB_ELASTIC, params(P.MODEL_MISFIT, 64, 64))
    with pytest.raises(P.PfcError):
        eng.submit(P.JOB_ELASTIC, params(P.MODEL_MISFIT, 64, 64), source_job=12345)
    with pytest.raises(P.PfcError):
        eng.submit(7, params(P.MODEL_MISFIT, 64, 64), steps=10, mod=5)
    eng.close()


def test_engine_submit_many():
    """pfc_submit_many queues a whole sweep in one call: all or nothing, ids in order, and
    every job's result equals the same job submitted on its own."""
    eng = P.Engine()
    good = [params(P.MODEL_MISFIT, g, g, seed=40 + i, u0=0.05 + 0.01 * i) for i, g in enumerate((64, 128, 64, 256))]
    bad = good[:2] + [params(P.MODEL_MISFIT, 64, 64, precision=P.FP64)] + good[2:]
    with pytest.raises(P.PfcError, match="job 2"):
        eng.submit_many(P.JOB_MISFIT, bad, steps=30, mod=15)
    assert eng.poll() == []  # nothing was queued
    ids = eng.submit_many(P.JOB_MISFIT, good, steps=30, mod=15)
    assert ids == sorted(ids) and len(set(ids)) == len(good)
    evs = drain(eng, ids)
    assert all(evs[i][-1].type == P.EV_DONE for i in ids)
    fields = [eng.fields(i) for i in ids]
    eng.close()
    one = P.Engine()
    for p, f in zip(good, fields):
        j = one.submit(P.JOB_MISFIT, p, steps=30, mod=15)
        drain(one, [j])
        for x, y in zip(f, one.fields(j)):
            assert same_bits(x, y)
    one.close()
