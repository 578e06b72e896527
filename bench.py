"""Benchmark: PFC Misfit time steps per second at 1024^2, batched fused step.

Workload (one GPU): B Misfit runs of 1024 x 1024 x 1 (the single-run GPU
configuration), seeds 1000+i, u0/con0 = reference defaults, advanced together on the
default mixed-precision path: FP32 complex arrays in HBM, FP64 arithmetic in the
kernels, FP64 k = 0 modes; within 1e-5 of pure FP64 after 200 steps.  One "step"
advances every run of the batch by one time step; `value` is run-steps per second over
all GPUs.  The batch's resident state (B x ~26 MB of row-space arrays) is larger than
the 126 MB L2, so timed steps stream from HBM.  The FP32-arithmetic path, the plain
FP64 path, the 3-D CVD grid, Elastic Analysis at the 1024^2 checkpoint size, the C4
sweep and the C5 serving mix are reported beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B] [--impl ours|reference]

N > 1 runs one process per GPU under torchrun (weak scaling: each rank owns its
own batch, no data-path collective; timing is the max over ranks).
`--impl reference` times the reference program's own CPU implementation of the
step (the unmodified sources compiled by oracle/Makefile) on this host's cores.
"""
from __future__ import annotations

import argparse
import glob
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "pfc-exp-gui_b200"))

GRID = 1024
METRIC = "PFC Misfit steps/s at 1024^2 (batched fused step, FP32 storage / FP64 arithmetic; run-steps/s)"
UNIT = "steps/s"


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--grid", type=int, default=GRID)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-plain", action="store_true")
    ap.add_argument("--no-sweep", action="store_true", help="skip the 64-run mixed-size sweep measurement")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving (Poisson arrivals) measurement")
    ap.add_argument("--serve-requests", type=int, default=48)
    ap.add_argument("--no-cvd3d", action="store_true", help="skip the 3-D CVD (256x256x64) step measurement")
    ap.add_argument("--no-elastic", action="store_true", help="skip the Elastic Analysis measurement")
    ap.add_argument("--no-fp32-path", action="store_true",
                    help="skip the same batch on the FP32-arithmetic fused path")
    ap.add_argument("--tile-width", type=int, default=0,
                    help="fix the column tile width instead of the autotuner's choice (reproducible profiles)")
    ap.add_argument("--staging", choices=["auto", "async", "bulk"], default="auto",
                    help="fix the column kernel's tile staging (cp.async or TMA bulk copies) instead of the autotuner's")
    return ap.parse_args(argv)


# ---------------------------------------------------------------------------
# distributed plumbing (torch.distributed over NCCL: barrier and max-over-ranks)
# ---------------------------------------------------------------------------
class Dist:
    """One process per GPU (torchrun env); NCCL on GPUs, gloo on CPU-only hosts."""

    def __init__(self, n, backend=None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.dev = "cpu"
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                self.dev = f"cuda:{self.local}"
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.pg = dist

    def barrier(self):
        if self.pg:
            import torch
            t = torch.zeros(1, device=self.dev)
            self.pg.all_reduce(t)
            if self.dev != "cpu":
                torch.cuda.synchronize()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64, device=self.dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v: float) -> float:
        if not self.pg:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64, device=self.dev)
        self.pg.all_reduce(t)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        j = json.load(open(p))
        return float(j["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_kernel(kernel):
    """The committed ncu figures of one kernel (profiles/roofline_traffic.json), or None."""
    p = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if not os.path.exists(p):
        return None
    return json.load(open(p)).get("kernels", {}).get(kernel)


def profiled_traffic(grid, batch, kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary (bytes per run of
    the profiled launch, times this batch)."""
    k = profiled_kernel(kernel)
    per_run = None if k is None else k.get("dram_bytes_per_run", {}).get(str(grid))
    return None if per_run is None else per_run * batch


# ---------------------------------------------------------------------------
# CPU baseline: the reference program (or the oracle port) on this host's cores
# ---------------------------------------------------------------------------
def ref_binary(grid):
    p = os.path.join(ROOT, "oracle", "_ref", f"pfc-exp-cli-{grid}x{grid}x1")
    return p if os.path.exists(p) else None


def time_reference_process(exe, steps, outdir):
    t0 = time.perf_counter()
    subprocess.run([exe, "--model", "misfit", "--steps", str(steps), "--mod", str(steps), "--outdir", outdir],
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, check=True)
    return time.perf_counter() - t0


def cpu_steps_per_s(grid, nproc, extra_steps):
    """Per-step throughput of `nproc` concurrent single-threaded reference processes
    (seeds 1000+i, the GPU arm's runs).

    Each process runs once with 1 step and once with 1+extra_steps steps (same init
    and the same single checkpoint), so the difference is exactly extra_steps steps."""
    import tempfile
    exe = ref_binary(grid)
    kind = "reference" if exe is not None else "port"
    with tempfile.TemporaryDirectory() as tmp:
        def phase(steps):
            if exe is not None:
                procs = []
                t0 = time.perf_counter()
                for i in range(nproc):
                    procs.append(subprocess.Popen([exe, "--model", "misfit", "--steps", str(steps), "--mod",
                                                   str(steps), "--seed", str(1000 + i),
                                                   "--outdir", os.path.join(tmp, f"r{i}_{steps}")],
                                                  stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL))
                for p in procs:
                    p.wait()
                return time.perf_counter() - t0
            # oracle port (bit-identical restatement of the reference step), one process per core
            t0 = time.perf_counter()
            procs = []
            for i in range(nproc):
                code = ("import sys; sys.path.insert(0, %r); import oracle as O; "
                        "r = O.Run(O.default_params(0, L=%d, M=%d, seed=%d)); r.step(%d)") % (
                            os.path.join(ROOT, "oracle"), grid, grid, 1000 + i, steps)
                procs.append(subprocess.Popen([sys.executable, "-c", code]))
            for p in procs:
                p.wait()
            return time.perf_counter() - t0
        ta = phase(1)
        tb = phase(1 + extra_steps)
    dt = max(tb - ta, 1e-9)
    return nproc * extra_steps / dt, kind


def workload(grid, runs):
    return f"Misfit {grid}x{grid}x1, {runs} runs (seeds 1000+i, u0 0.05, con0 0.2), run-steps/s"


def cpu_baseline(grid, steps=2):
    v, kind = cpu_steps_per_s(grid, 1, steps)
    what = "reference pfc-exp-cli built from its sources" if kind == "reference" else "oracle port of the reference step"
    return {"value": round(v, 4), "unit": UNIT, "cores": 1, "kind": kind,
            "sample": f"{steps} Misfit {grid}^2 FP64 steps of one run ({what}; FFTW unavailable, "
                      f"project FFTW-API shim FFT), 1 core; time(1+{steps} steps) - time(1 step)"}


def run_reference(args):
    """The reference program's own CPU step on this host's cores: one single-threaded
    process per run, as many runs as the GPU arm's batch (fewer if the host has fewer
    cores), each timed over exactly args.steps steps (capped at 50 so that the arm ends
    within minutes)."""
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    nproc = max(1, min(args.batch, os.cpu_count() or 1))
    steps = max(1, min(args.steps, 50))
    v, kind = cpu_steps_per_s(args.grid, nproc, steps)
    sample = (f"{nproc} concurrent single-threaded processes (one per run, seeds 1000+i), each timed over "
              f"{steps} Misfit {args.grid}^2 FP64 steps as time(1+{steps} steps) - time(1 step) "
              f"({'reference pfc-exp-cli built from its sources' if kind == 'reference' else 'oracle port'}; "
              "FFTW unavailable, project FFTW-API shim FFT)")
    line = {"metric": METRIC, "value": round(v, 4), "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": steps, "warmup": 0, "ms_per_step": round(1000.0 / v, 3) if v else None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload(args.grid, nproc), "grid": [args.grid, args.grid, 1], "runs": nproc},
            "cpu_baseline": {"value": round(v, 4), "unit": UNIT, "cores": nproc, "kind": kind, "sample": sample},
            "e2e": {"value": round(v, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
# ---------------------------------------------------------------------------
# Sweep and serving workloads through the engine (pfc_engine_* in the C ABI)
# ---------------------------------------------------------------------------
MASK64 = (1 << 64) - 1


class SplitMix64:
    """splitmix64 (Steele, Lea, Flood 2014), the generator the reference seeds with."""

    def __init__(self, seed):
        self.x = seed & MASK64

    def next(self):
        self.x = (self.x + 0x9E3779B97F4A7C15) & MASK64
        z = self.x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)


def drain_engine(P, eng, n, timeout_s=900.0):
    """Wait for n jobs to finish; returns {job: final event}."""
    done = {}
    t_end = time.time() + timeout_s
    while len(done) < n and time.time() < t_end:
        for ev in eng.wait(timeout_ms=500):
            if ev.type in (P.EV_DONE, P.EV_FAILED, P.EV_CANCELLED):
                done[ev.job] = ev
    return done


PREC_NAMES = {0: "fp32", 1: "fp64", 2: "fp64-pure", 3: "mixed"}


def cpu_sweep_estimate(grids, steps, extra=3):
    """The sweep as the GUI runs it on the CPU: the reference program once per run, one
    after another (MainWindow.cpp:3453-3522).  Each grid's binary is timed once with 1 and
    once with 1+extra steps; a run costs time(1 step) + (steps - 1) x the per-step time.
    None when a grid's reference binary is missing."""
    import tempfile
    per = {}
    with tempfile.TemporaryDirectory() as tmp:
        for g in grids:
            exe = ref_binary(g)
            if exe is None:
                return None
            t1 = time_reference_process(exe, 1, os.path.join(tmp, f"g{g}_1"))
            tn = time_reference_process(exe, 1 + extra, os.path.join(tmp, f"g{g}_n"))
            per[g] = (t1, (tn - t1) / extra)
    total = sum(n * (per[g][0] + (steps - 1) * per[g][1]) for g, n in grids.items())
    return {"estimate_s": round(total, 1), "runs_per_hour": round(sum(grids.values()) / total * 3600.0, 2),
            "step_s": {f"{g}^2": round(v[1], 5) for g, v in sorted(per.items())},
            "sample": f"each grid's reference pfc-exp-cli (built from its sources; FFTW unavailable, project "
                      f"FFTW-API shim FFT) timed once at 1 and once at {1 + extra} steps on one core"}


def sweep_bench(P, dev, precision, nruns=64, steps=2000, master_seed=4242, reps=3, cpu_reference=False):
    """64 Misfit runs of mixed grids {128, 256, 512}^2, u0 and con0 from the GUI's value
    lists, drawn with splitmix64 from a master seed; 2000 steps, one checkpoint (mod 2000),
    at the given precision.  Timed as one engine sweep (all submitted at once) and as
    sequential GPU runs (the same engine with one run resident at a time, as the GUI's
    one-process queue)."""
    rng = SplitMix64(master_seed)
    jobs = []
    for i in range(nruns):
        g = (128, 256, 512)[rng.next() % 3]
        u0 = (0.02, 0.05, 0.08, 0.11)[rng.next() % 4]
        con0 = (0.1, 0.2, 0.3, 0.4)[rng.next() % 4]
        jobs.append(P.default_params(P.MODEL_MISFIT, L=g, M=g, seed=1000 + i, u0=u0, con0=con0, device=dev,
                                     precision=precision))

    # the autotuner picks each grid's column tile width once per process; it runs here,
    # before either arm is timed, so both arms use the same widths
    t_tune = time.perf_counter()
    widths = {g: P.tile_width(g, g, device=dev, precision=precision)[0] for g in sorted({p.L for p in jobs})}
    tune_s = time.perf_counter() - t_tune

    def run(max_active):
        eng = P.Engine(device=dev, max_active=max_active)
        # warm-up: one short job per grid, with a checkpoint, so that neither arm pays the
        # first use of a grid's kernels (module loading) inside its timed region
        warm = [eng.submit(P.JOB_MISFIT, P.default_params(P.MODEL_MISFIT, L=g, M=g, device=dev, precision=precision),
                           steps=40, mod=20) for g in widths]
        drain_engine(P, eng, len(warm))
        for w in warm:
            eng.release(w)
        t0 = time.perf_counter()
        ids = eng.submit_many(P.JOB_MISFIT, jobs, steps=steps, mod=steps)  # the sweep arrives at once
        done = drain_engine(P, eng, len(ids))
        wall = time.perf_counter() - t0
        ok = sum(1 for j in ids if j in done and done[j].type == P.EV_DONE)
        eng.close()
        return wall, ok

    # three rounds, the arms alternating; each arm reports its median round (the
    # wall-clock arms are host-driven, and single rounds on a shared host show outliers)
    rounds_b, rounds_s = [], []
    for _ in range(reps):
        rounds_b.append(run(0))
        rounds_s.append(run(1))
    wall_b, ok_b = sorted(rounds_b)[len(rounds_b) // 2]
    wall_s, ok_s = sorted(rounds_s)[len(rounds_s) // 2]
    grids = {}
    for p in jobs:
        grids[p.L] = grids.get(p.L, 0) + 1
    cpu = cpu_sweep_estimate(grids, steps) if cpu_reference else None
    return {"runs": nruns, "steps": steps, "precision": PREC_NAMES[precision],
            **({"cpu_reference_sequential": cpu} if cpu else {}),
            "grids": {f"{g}^2": n for g, n in sorted(grids.items())},
            "master_seed": master_seed,
            "batched_s": round(wall_b, 3), "sequential_gpu_s": round(wall_s, 3),
            "batched_s_rounds": [round(w, 3) for w, _ in rounds_b],
            "sequential_gpu_s_rounds": [round(w, 3) for w, _ in rounds_s],
            "runs_per_hour_batched": round(ok_b / wall_b * 3600.0, 1),
            "runs_per_hour_sequential_gpu": round(ok_s / wall_s * 3600.0, 1),
            "batched_over_sequential": round(wall_s / wall_b, 2), "completed": [ok_b, ok_s],
            "column_tile_widths": {f"{g}^2": w for g, w in widths.items()}, "autotune_s": round(tune_s, 3),
            "what": "wall clock from the first submit to the last DONE event (run set-up, 2000 steps, "
                    "final Phimax/energy checkpoint), median of 3 alternating rounds per arm; "
                    "sequential = engine with max_active=1"}


def serve_bench(P, dev, n_req=48, lam=4.0, seed=777, budget=150e9):
    """Poisson arrivals (rate lam/s): 70 % Misfit, 20 % CVD (2-D), 10 % Elastic on a
    finished run's fields; grid 2^U(7,11) rounded to a power of two, steps U[500, 20000],
    u0 U[0.02, 0.12], con0 U[0.1, 0.4], random seeds; HBM admission budget 150 GB.
    Latency = DONE event - submission (files and results ready)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / lam, n_req))
    kinds = rng.choice([P.JOB_MISFIT, P.JOB_CVD, P.JOB_ELASTIC], size=n_req, p=[0.7, 0.2, 0.1])
    # a warm server: the column tile widths of the request grids are tuned before the
    # clock starts (once per process), as the first request of each grid would otherwise do
    t_tune = time.perf_counter()
    for g in (128, 256, 512, 1024, 2048):
        P.tile_width(g, g, device=dev)
    tune_s = time.perf_counter() - t_tune
    eng = P.Engine(device=dev, hbm_budget_bytes=budget)
    warm = eng.submit(P.JOB_MISFIT, P.default_params(P.MODEL_MISFIT, L=128, M=128, device=dev), steps=20, mod=20)
    drain_engine(P, eng, 1)
    eng.release(warm)
    misfit_ids, submitted, done, kind_of = [], [], {}, {}
    t0 = time.perf_counter()
    i = 0
    while len(done) < n_req:
        now = time.perf_counter() - t0
        while i < n_req and arrivals[i] <= now:
            k = int(kinds[i])
            if k == P.JOB_ELASTIC and not misfit_ids:
                k = P.JOB_MISFIT
            if k == P.JOB_ELASTIC:
                src = misfit_ids[int(rng.integers(len(misfit_ids)))]
                jid = eng.submit(P.JOB_ELASTIC, P.default_params(P.MODEL_MISFIT, device=dev), source_job=src)
            else:
                g = 2 ** int(round(rng.uniform(7.0, 11.0)))
                model = P.MODEL_CVD if k == P.JOB_CVD else P.MODEL_MISFIT
                p = P.default_params(model, L=g, M=g, seed=int(rng.integers(1, 2**31)), u0=float(rng.uniform(0.02, 0.12)),
                                     con0=float(rng.uniform(0.1, 0.4)), device=dev)
                steps = int(rng.integers(500, 20001))
                jid = eng.submit(k, p, steps=steps, mod=steps)
                if k == P.JOB_MISFIT:
                    misfit_ids.append(jid)
            kind_of[jid] = k
            submitted.append(jid)
            i += 1
        wait_ms = 200 if i >= n_req else max(1, int((arrivals[i] - (time.perf_counter() - t0)) * 1000))
        for ev in eng.wait(timeout_ms=min(wait_ms, 200)):
            if ev.type in (P.EV_DONE, P.EV_FAILED, P.EV_CANCELLED):
                done[ev.job] = ev
        if time.perf_counter() - t0 > 1200:
            break
    makespan = time.perf_counter() - t0
    eng.close()
    lat = np.array([done[j].t_event - done[j].t_submit for j in submitted if j in done and done[j].type == P.EV_DONE])
    ok = len(lat)
    return {"requests": n_req, "arrival_rate_per_s": lam, "seed": seed, "completed": ok,
            "mix": {"misfit": int(sum(1 for k in kind_of.values() if k == P.JOB_MISFIT)),
                    "cvd": int(sum(1 for k in kind_of.values() if k == P.JOB_CVD)),
                    "elastic": int(sum(1 for k in kind_of.values() if k == P.JOB_ELASTIC))},
            "p50_s": round(float(np.percentile(lat, 50)), 3) if ok else None,
            "p99_s": round(float(np.percentile(lat, 99)), 3) if ok else None,
            "makespan_s": round(makespan, 2), "runs_per_hour": round(ok / makespan * 3600.0, 1),
            "hbm_budget_gb": budget / 1e9,
            "autotune_s": round(tune_s, 3),
            "what": "engine with continuous batching; latency = submission to DONE (results and events ready)"}


def step_roofline(P, batch, G, B, names, reps=20):
    """Event-timed row and column kernel launches of a batch, each against the HBM peak
    with its algorithmic bytes (row: 4 row-space arrays read, 2 written; column: 4 + 4;
    8 bytes per complex half-spectrum element), the DRAM traffic the committed ncu
    capture measured, and (FP64-arithmetic kernels) the FP64 pipe's active fraction there."""
    row_ms, col_ms = batch.kernel_times(reps)
    H1 = G // 2 + 1
    by = {"row": B * G * H1 * 8 * 6, "col": B * G * H1 * 8 * 8}
    peak, _ = measured_peak()
    out = {}
    for name, ms_k in (("row", row_ms), ("col", col_ms)):
        ach = by[name] / (ms_k / 1000.0) / 1e9
        out[name] = {"launch_ms": round(ms_k, 5), "algorithmic_bytes_per_launch": by[name],
                     "achieved": round(ach, 1), "frac": round(ach / peak, 4),
                     "traffic": profiled_traffic(G, B, names[name])}
        prof = profiled_kernel(names[name])
        if prof and prof.get("fp64_pipe_active_pct") is not None:
            out[name]["fp64_pipe_active_pct_profiled"] = prof["fp64_pipe_active_pct"]
        n64 = (prof or {}).get("fp64_warp_insts_per_run", {}).get(str(G))
        if n64:
            # FP64 pipe: 2 warp instructions per cycle per SM (64 lanes); peak at the clock seen
            sms, mhz = sm_info()
            ach64 = n64 * B / (ms_k / 1000.0)
            peak64 = 2.0 * sms * mhz * 1e6
            out[name]["fp64_pipe"] = {"warp_insts_per_launch": n64 * B, "achieved_warp_insts_per_s": round(ach64, 0),
                                      "peak_warp_insts_per_s": round(peak64, 0), "frac": round(ach64 / peak64, 4),
                                      "clock_mhz": mhz}
    return out


def sm_info():
    """SM count and the SM clock (MHz) the FP64 roofline is taken at: the median clock
    sampled during the timed region when known, else the device's maximum."""
    import torch
    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    mhz = _CLOCK_SEEN.get("sm_mhz") or _CLOCK_SEEN.get("sm_max_mhz") or 1965.0
    return props.multi_processor_count, float(mhz)


_CLOCK_SEEN = {}


def elastic_bench(P, dev, G=1024, steps=500):
    """Elastic Analysis on a 1024^2 Misfit checkpoint (C2 checkpoint size): peak finder,
    elastic3D and cryst_order through the C ABI, host arrays in and out."""
    import numpy as np
    r = P.Run(P.default_params(P.MODEL_MISFIT, L=G, M=G, seed=1000, device=dev))
    r.advance(steps, analysis=True)
    phi, _ = r.fields_f32()
    r.close()
    f = phi.reshape(G, G, 1).astype(np.float64)
    atoms = P.phimax_elastic(f)  # first use loads the kernels
    x, y, z = atoms[:, 0].copy(), atoms[:, 1].copy(), atoms[:, 2].copy()
    P.elastic3d(x, y, z, G, G, 1)
    P.cryst_order(x, y, z, G, G, 1)

    def median_s(fn, reps=5):  # host-driven calls: the median of a few is stable on a shared host
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            fn()
            ts.append(time.perf_counter() - t0)
        return sorted(ts)[reps // 2]
    t = {"peak_s": median_s(lambda: P.phimax_elastic(f)),
         "elastic3d_s": median_s(lambda: P.elastic3d(x, y, z, G, G, 1)),
         "cryst_order_s": median_s(lambda: P.cryst_order(x, y, z, G, G, 1))}
    total = sum(t.values())
    n = len(atoms)
    return {"workload": f"Misfit {G}^2 state after {steps} steps (seed 1000), Float32 fields", "atoms": n,
            **{k: round(v, 5) for k, v in t.items()}, "analyses_per_s": round(1.0 / total, 2),
            "elastic3d_pair_tests_per_s": round(n * (n - 1) / t["elastic3d_s"], 1),
            "what": "wall time of pfc_phimax_elastic + pfc_elastic3d + pfc_cryst_order on host arrays "
                    "(each call copies its inputs in and its results out), median of 5 calls each"}


def run_ours(args):
    dist = Dist(args.gpus)
    import numpy as np
    import pfc_b200 as P
    dev = dist.local
    G, B = args.grid, args.batch
    prec = P.MIXED
    for pr in (P.MIXED, P.FP32):  # both fused paths: a pinned width or staging skips their autotuner
        if args.tile_width:
            P.set_tile_width(G, G, args.tile_width, device=dev, precision=pr)
        if args.staging != "auto":
            P.set_col_staging(G, G, P.STAGE_ASYNC if args.staging == "async" else P.STAGE_BULK, device=dev,
                              precision=pr)
    runs = []
    for i in range(B):
        p = P.default_params(P.MODEL_MISFIT, L=G, M=G, N=1, seed=1000 + i + 100000 * dist.rank, device=dev,
                             precision=prec)
        runs.append(P.Run(p))
    batch = P.Batch(runs)
    tile_w, tile_trials = P.tile_width(G, G, device=dev, precision=prec)  # chosen by the autotuner at the first run
    stage, stage_trials = P.col_staging(G, G, device=dev, precision=prec)
    batch.advance(max(3, args.warmup))
    dist.barrier()
    clocks = Clocks(dev)
    clocks.start()
    ms = batch.advance_timed(args.steps)
    clk = clocks.stop()
    if isinstance(clk, dict):
        _CLOCK_SEEN.update({k: clk.get(k) for k in ("sm_mhz", "sm_max_mhz")})
    ms_max = dist.max(ms)
    total_run_steps = dist.sum(B * args.steps)
    value = total_run_steps / (ms_max / 1000.0)

    # per-kernel roofline (dominant kernel), timed with events on the library stream
    names = {"row": "k_mrow_step", "col": "k_mcol_step"}
    kern = step_roofline(P, batch, G, B, names)
    dom = "col" if kern["col"]["launch_ms"] >= kern["row"]["launch_ms"] else "row"
    peak, peak_kind = measured_peak()

    # end to end through the public API: FP32 host fields from pinned memory in, B runs x K
    # steps, FP32 host fields out into pinned memory
    phi0, con0 = runs[0].fields_f32()
    try:
        import torch
        pin = torch.cuda.is_available()
    except Exception:  # noqa: BLE001
        pin = False

    def host_buf():
        if pin:
            return torch.empty(G * G, dtype=torch.float32, pin_memory=True).numpy()
        return np.empty(G * G, np.float32)
    ins = []
    for _ in range(B):
        a, c = host_buf(), host_buf()
        a[:] = phi0.ravel()
        c[:] = con0.ravel()
        ins.append((a, c))
    outs = [(host_buf(), host_buf()) for _ in range(B)]
    dist.barrier()
    t0 = time.perf_counter()
    for r, (a, c) in zip(runs, ins):
        r.set_fields_f32(a, c)
    batch.advance(args.steps)
    for r, o in zip(runs, outs):
        r.fields_f32(out=o)
    e2e_s = time.perf_counter() - t0
    e2e_s = dist.max(e2e_s)
    e2e_value = total_run_steps / e2e_s
    h2d = B * G * G * 8 / args.steps
    d2h = B * G * G * 8 / args.steps

    line = {
        "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": dist.world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": round(ms_max / args.steps, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (reference INITIAL_dis seeded polycrystal, seeds 1000+i)",
        "config": {"workload": workload(G, B), "grid": [G, G, 1], "runs": B,
                   "path": "fused two-sweep step, mixed precision: FP32 complex arrays in HBM, FP64 arithmetic "
                           "(pure-FP64 operator), FP64 k=0 modes; graph-captured row/column sweeps",
                   "parallelism": f"replicas x{dist.world}",
                   "l2": "inputs larger than L2 (resident state ~26 MB/run x batch)",
                   "column_tile_width": tile_w,
                   "column_staging": "async" if stage == P.STAGE_ASYNC else "bulk",
                   "autotuner_trials_ms_per_8_steps": {str(k): {"async": round(a, 4), "bulk": round(b, 4)}
                                                       for k, (a, b) in stage_trials.items()}},
        "roofline": {"bound": "hbm", "kernel": names[dom], "achieved": kern[dom]["achieved"], "peak": peak,
                     "unit": "GB/s", "frac": kern[dom]["frac"], "peak_source": peak_kind,
                     "traffic": kern[dom]["traffic"],
                     "algorithmic_bytes_per_launch": kern[dom]["algorithmic_bytes_per_launch"],
                     "launch_ms": kern[dom]["launch_ms"],
                     "per_kernel": {names[k]: v for k, v in kern.items()}},
        "e2e": {"value": round(e2e_value, 2), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "steps": args.steps, "pinned_host_buffers": pin,
                "what": "pfc_run_set_fields_f32 (FP32 host fields) + pfc_batch_advance(K) + pfc_run_get_fields_f32, "
                        "wall clock"},
        "gpu_launches": 2 * args.steps,
        "clocks": clk,
    }
    if "fp64_pipe" in kern[dom]:
        # the mixed kernels compute in FP64: the bound that holds them is the FP64 pipe's issue
        # rate (and its latency), which this fraction reports beside the HBM one
        line["roofline"]["fp64_pipe"] = kern[dom]["fp64_pipe"]
    batch.close()
    for r in runs:
        r.close()
    if not args.no_fp32_path:
        # the FP32-arithmetic fused path on the same batch (faster, but 7e-5 from pure FP64 after
        # 200 steps at 1024^2, outside the 1e-5 bound)
        runs32 = [P.Run(P.default_params(P.MODEL_MISFIT, L=G, M=G, seed=1000 + i, device=dev, precision=P.FP32))
                  for i in range(B)]
        b32 = P.Batch(runs32)
        b32.advance(5)
        ms32 = b32.advance_timed(min(args.steps, 200))
        k32 = step_roofline(P, b32, G, B, {"row": "k_row_step", "col": "k_col_step"})
        line["fp32_path"] = {"run_steps_per_s": round(B * min(args.steps, 200) / (ms32 / 1000.0), 2),
                             "ms_per_step": round(ms32 / min(args.steps, 200), 5),
                             "column_tile_width": P.tile_width(G, G, device=dev, precision=P.FP32)[0],
                             "per_kernel": {"k_row_step": k32["row"], "k_col_step": k32["col"]},
                             "what": "the same batch on the FP32-arithmetic path (opt-in --precision fp32)"}
        b32.close()
        for r in runs32:
            r.close()
    # the plain FP64 GPU path (one run, the reference's step structure) on the same grid
    if not args.no_fp64_plain:
        r64 = P.Run(P.default_params(P.MODEL_MISFIT, L=G, M=G, N=1, seed=1000, device=dev, precision=P.FP64))
        r64.advance(3)
        n64 = 20
        ms64 = r64.advance_timed(n64)
        r64.close()
        fp64_sps = n64 / (ms64 / 1000.0)
        # 13 complex-double 3-D DFTs per step, each one pass per axis of length > 1 (two on a
        # 2-D grid) reading and writing 16 B per point, plus the pointwise kernels' 14 reads
        # and writes of complex doubles per point
        fp64_bytes = G * G * (13 * 2 * 2 * 16 + 14 * 16)
        ach64 = fp64_bytes / (ms64 / n64 / 1000.0) / 1e9
        line["fp64_plain"] = {"steps_per_s": round(fp64_sps, 2), "ms_per_step": round(ms64 / n64, 4),
                              "what": "one Misfit run, plain FP64 path (13 complex-double 3-D DFTs + pointwise "
                                      "kernels per step, reference roundings), CUDA events",
                              "roofline": {"bound": "hbm", "achieved": round(ach64, 1),
                                           "frac": round(ach64 / peak, 4),
                                           "algorithmic_bytes_per_step": fp64_bytes},
                              "batched_over_fp64_plain": round(value / dist.world / fp64_sps, 2)}
        if "fp32_path" in line:
            line["fp64_plain"]["fp32_path_over_fp64_plain"] = round(line["fp32_path"]["run_steps_per_s"] / fp64_sps, 2)
    # one run alone (the single-run form of the 1024^2 workload): what a single simulation
    # gets, against the batch's per-run share
    if not args.no_fp64_plain:
        r1 = P.Run(P.default_params(P.MODEL_MISFIT, L=G, M=G, N=1, seed=1000, device=dev, precision=P.MIXED))
        r1.advance(5)
        n1 = 200
        ms1 = r1.advance_timed(n1)
        r1.close()
        sps1 = n1 / (ms1 / 1000.0)
        line["single_run"] = {"steps_per_s": round(sps1, 2), "ms_per_step": round(ms1 / n1, 4),
                              "over_fp64_plain": round(sps1 / line["fp64_plain"]["steps_per_s"], 2),
                              "what": "one Misfit 1024^2 run on the mixed path, CUDA events over 200 steps"}
    # the 3-D CVD workload (256 x 256 x 64): the mixed path (four sweeps per step: row
    # kernel along n, m-axis pass, column kernel along l, inverse m-axis pass) and the
    # plain FP64 path
    if not args.no_cvd3d:
        L3, M3, N3 = 256, 256, 64
        out3 = {"workload": f"CVD {L3}x{M3}x{N3} (u0 0.01, con0 0.2, dt 0.05, dx 0.125)"}
        for name, prec in (("mixed", P.MIXED), ("fp64_plain", P.FP64)):
            r3 = P.Run(P.default_params(P.MODEL_CVD, L=L3, M=M3, N=N3, device=dev, precision=prec))
            r3.advance(2)
            n3 = 50 if prec == P.MIXED else 10
            ms3 = r3.advance_timed(n3)
            # the CLI's loop between checkpoints: ENERGYC2 after every step (energy.txt), the
            # energies read back once per call (pfc_run_advance_energies)
            r3.advance_energies(2)
            t0 = time.perf_counter()
            r3.advance_energies(n3)
            cli_ms = (time.perf_counter() - t0) / n3 * 1e3
            r3.close()
            entry = {"ms_per_step": round(ms3 / n3, 4), "steps_per_s": round(n3 / (ms3 / 1000.0), 2),
                     "cli_step_with_energy_ms": round(cli_ms, 3)}
            if prec == P.MIXED:
                # 30 array passes per step (row 4 + 2, m-pass 4 + 4, column 4 + 4, inverse m-pass
                # 4 + 4) over L*M*Hp complex floats, Hp = N/2 + 1 rounded up to the tile width 8
                hp = (N3 // 2 + 1 + 7) // 8 * 8
                by3 = 30 * L3 * M3 * hp * 8
                ach3 = by3 / (ms3 / n3 / 1000.0) / 1e9
                entry["roofline"] = {"bound": "hbm", "achieved": round(ach3, 1), "frac": round(ach3 / peak, 4),
                                     "algorithmic_bytes_per_step": by3}
            out3[name] = entry
        out3["mixed_over_fp64_plain"] = round(out3["fp64_plain"]["ms_per_step"] / out3["mixed"]["ms_per_step"], 2)
        out3["what"] = ("pfc_run_advance_timed (CUDA events) of the steps; cli_step_with_energy_ms is the wall time "
                        "per step of pfc_run_advance_energies (each step with its energy analysis, as pfc-exp-cli's "
                        "CVD loop)")
        line["cvd3d"] = out3
    if not args.no_elastic:
        line["elastic"] = elastic_bench(P, dev, G)
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(G)
        except Exception as e:  # noqa: BLE001
            line["cpu_baseline"] = {"value": None, "error": str(e)}
    # sweep and serving workloads, each rank on its own GPU (rank 0 reports its own)
    if not args.no_sweep:
        # the sweep workload names FP32 arithmetic with FP64 reductions (the FP32 path);
        # the same sweep on the default mixed-precision path beside it
        line["sweep"] = sweep_bench(P, dev, P.FP32,
                                    cpu_reference=dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline)
        line["sweep"]["mixed_precision"] = sweep_bench(P, dev, P.MIXED)
    if not args.no_serve:
        line["serving"] = serve_bench(P, dev, n_req=args.serve_requests, seed=777 + dist.rank)
    if dist.rank == 0:
        print(json.dumps(line), flush=True)
    dist.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
