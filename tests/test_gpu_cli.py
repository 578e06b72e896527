"""The pfc-exp-cli drop-in: same flags, files, progress lines and exit codes.

Runs bin/pfc-exp-cli (a thin main() over pfc_run_cli) and compares its output
directory with the reference program's (golden fixtures): text files byte for
byte where the values are computed identically, and field values within the
FP32 tolerance where they come from the FP32 step.
"""
import os
import re
import subprocess

import numpy as np
import pytest

import oracle as O
import pfc_b200 as P
from helpers import golden_case, read_vti

CLI = P.CLI_PATH


def run_cli(args, **kw):
    return subprocess.run([CLI, *args], capture_output=True, text=True, timeout=600, **kw)


def test_cli_help_and_bad_args():
    """Exit codes and dispatch need no GPU (main_cli.cpp:24-88, MIS:306-308)."""
    r = run_cli(["--help"])
    assert r.returncode == 0 and "Models:" in r.stderr
    r = run_cli(["--model", "misfit", "--help"])
    assert r.returncode == 0 and "--grainx" in r.stderr
    r = run_cli(["--model", "nope"])
    assert r.returncode == 2 and "Unknown model: nope" in r.stderr
    r = run_cli(["--model", "misfit", "--bogus", "1"])
    assert r.returncode == 2 and "Unknown option: --bogus" in r.stderr
    r = run_cli(["--model", "misfit", "--steps", "0"])
    assert r.returncode == 2 and "--steps must be > 0" in r.stderr
    r = run_cli(["--model", "cvd", "--mod", "-1"])
    assert r.returncode == 2 and "Invalid parameter values" in r.stderr
    r = run_cli(["--model"])
    assert r.returncode == 2


@pytest.mark.gpu
def test_cli_misfit_matches_reference(tmp_path):
    d, meta, fields = golden_case("misfit_64")
    out = tmp_path / "run"
    r = run_cli(["--model", "misfit", "--grid", "64x64x1", *meta["args"], "--outdir", str(out)])
    assert r.returncode == 0, r.stderr
    # progress lines as the GUI parses them (MainWindow.cpp:3426)
    prog = [l for l in r.stdout.splitlines() if re.match(r"^PFC_PROGRESS\s+step=(\d+)\s+total=(\d+)\s*$", l)]
    ref_prog = [l for l in open(f"{d}/stdout.txt").read().splitlines() if l.startswith("PFC_PROGRESS")]
    assert prog == ref_prog
    # non-progress stdout lines: identical sequence of tags
    tags = [re.sub(r"\d+", "#", l) for l in r.stdout.splitlines() if not l.startswith("PFC_PROGRESS")]
    ref_tags = [re.sub(r"\d+", "#", l) for l in open(f"{d}/stdout.txt").read().splitlines()
                if not l.startswith("PFC_PROGRESS")]
    assert tags == ref_tags
    assert (out / "run_config.txt").read_text() == open(f"{d}/run_config.txt").read()
    # checkpoint files: byte-identical headers and pvti, values within the FP32 tolerance
    for kd in (0, 25, 50):
        for f in ("phi", "con"):
            vals, head, nbytes = read_vti(out / f"{f}_{kd}_0.vti")
            ref = fields[f"{f}_{kd}"]
            if kd == 0:
                assert np.array_equal(vals, ref)
            else:
                assert np.abs(vals - ref).max() <= 1e-5
            if os.path.exists(f"{d}/{f}_{kd}_0.vti"):
                _, rhead, rbytes = read_vti(f"{d}/{f}_{kd}_0.vti")
                assert head == rhead and nbytes == rbytes
                assert (out / f"{f}_{kd}.pvti").read_text() == open(f"{d}/{f}_{kd}.pvti").read()
                raw = (out / f"{f}_{kd}_0.vti").read_bytes()
                rraw = open(f"{d}/{f}_{kd}_0.vti", "rb").read()
                trailer = b"\n</AppendedData>\n</VTKFile>\n"
                assert len(raw) == len(rraw) and raw.endswith(trailer) and rraw.endswith(trailer)
    # energy.txt: same lines (steps) and values within tolerance
    got = [l.split() for l in (out / "energy.txt").read_text().splitlines()]
    ref = [l.split() for l in open(f"{d}/energy.txt").read().splitlines()]
    assert [g[0] for g in got] == [r_[0] for r_ in ref]
    for g, r_ in zip(got, ref):
        assert abs(float(g[1]) - float(r_[1])) <= 1e-5 * abs(float(r_[1]))
        assert abs(float(g[2]) - float(r_[2])) <= 1e-6
    # Phimax: same atoms (count, ordering) within the FP32 field tolerance
    for kd in (25, 50):
        a = np.loadtxt(out / f"Phimax_{kd}.txt", skiprows=2)
        b = np.loadtxt(f"{d}/Phimax_{kd}.txt", skiprows=2)
        assert a.shape == b.shape
        assert np.abs(a - b).max() <= 2e-3
    ts = (out / "checkpoint_timestamps.txt").read_text().splitlines()
    assert ts[0].startswith("# Checkpoint timestamps") and [l.split()[1] for l in ts[1:]] == ["25", "50"]


@pytest.mark.gpu
def test_cli_elastic_on_reference_checkpoints(tmp_path):
    """Elastic Analysis on the reference's own VTI files: text outputs byte-identical
    (Phimax, strain), q4q6 within the cryst_order tolerance."""
    d, meta, fields = golden_case("misfit_64")
    inp = tmp_path / "in"
    inp.mkdir()
    # write the reference checkpoints back out with the reference's byte layout
    for kd in (25, 50):
        for f in ("phi", "con"):
            arr = fields[f"{f}_{kd}"]
            L, M, N = arr.shape
            raw = open(f"{d}/{f}_25_0.vti", "rb").read()
            i = raw.index(b"_", raw.index(b"<AppendedData"))
            body = arr.transpose(2, 1, 0).astype(np.float32).tobytes()
            (inp / f"{f}_{kd}_0.vti").write_bytes(raw[:i + 5] + body + raw[i + 5 + len(body):])
    for k, extra in enumerate([[], ["--benchel", "1.3"]]):
        out = tmp_path / f"el{k}"
        r = run_cli(["--model", "elastic", "--input-dir", str(inp), "--outdir", str(out), *extra])
        assert r.returncode == 0, r.stderr
        assert "PFC_PROGRESS step=2 total=2" in r.stderr
        for kd in (25, 50):
            for f in ("Phimax", "strain"):
                assert (out / f"{f}_{kd}.txt").read_text() == open(f"{d}/elastic{k}/{f}_{kd}.txt").read()
            a = np.loadtxt(out / f"q4q6_{kd}.txt", skiprows=2, usecols=(1, 2, 3, 4, 5))
            b = np.loadtxt(f"{d}/elastic{k}/q4q6_{kd}.txt", skiprows=2, usecols=(1, 2, 3, 4, 5))
            assert a.shape == b.shape and np.abs(a - b).max() <= 1.01e-4


@pytest.mark.gpu
def test_cli_elastic_missing_input_exits_2(tmp_path):
    r = run_cli(["--model", "elastic", "--input-dir", str(tmp_path / "none"), "--outdir", str(tmp_path / "o"),
                 "--steps", "10", "--mod", "5"])
    assert r.returncode == 2 and "can't open input file" in r.stderr


@pytest.mark.gpu
def test_cli_cvd_matches_reference(tmp_path):
    d, meta, fields = golden_case("cvd_64")
    out = tmp_path / "cvd"
    r = run_cli(["--model", "cvd", "--grid", "64x64x1", *meta["args"], "--outdir", str(out)])
    assert r.returncode == 0, r.stderr
    assert r.stderr.count("PFC_PROGRESS") == 21
    for kd in (0, 10, 20):
        vals, _, _ = read_vti(out / f"phi_{kd}_0.vti")
        assert np.abs(vals - fields[f"phi_{kd}"]).max() <= 1e-5
    got = [l.split() for l in (out / "energy.txt").read_text().splitlines()]
    ref = [l.split() for l in open(f"{d}/energy.txt").read().splitlines()]
    assert [g[0] for g in got] == [r_[0] for r_ in ref]
    for g, r_ in zip(got, ref):
        assert abs(float(g[1]) - float(r_[1])) <= 1e-5 * abs(float(r_[1])) + 1e-9
    check_cvd_analysis_files(out, d, (0, 10, 20), 1e-4)


def numbers(path):
    return [[float(v) if v.replace(".", "", 1).replace("-", "", 1).isdigit() else v for v in l.replace(",", " ").split()]
            for l in open(path).read().splitlines()]


def same_numbers(a, b, tol):
    if len(a) != len(b):
        return False
    for la, lb in zip(a, b):
        if len(la) != len(lb):
            return False
        for x, y in zip(la, lb):
            if isinstance(x, float) and isinstance(y, float):
                if abs(x - y) > tol * max(1.0, abs(y)):
                    return False
            elif x != y:
                return False
    return True


def check_cvd_analysis_files(out, d, kds, tol):
    """The CVD checkpoint analysis files (CVD:1067-1520) against the reference run's:
    the same atoms at the same grid positions (so the same pair histogram); values
    printed from the (FP32-path) fields within tol."""
    for kd in kds:
        for f in (f"phiball_{kd}.cfg", f"hist_{kd}.txt", f"Grq6_{kd}.txt"):
            assert (out / f).read_text() == open(f"{d}/{f}").read(), f
        assert same_numbers(numbers(out / f"Phimax_{kd}.txt"), numbers(f"{d}/Phimax_{kd}.txt"), tol)
        if kd % 20 == 0:
            assert same_numbers(numbers(out / f"Ql_{kd}.txt"), numbers(f"{d}/Ql_{kd}.txt"), 1e-5)
            assert (out / f"HistQ_{kd}.txt").read_text() == open(f"{d}/HistQ_{kd}.txt").read()
    assert same_numbers(numbers(out / "phimax.txt"), numbers(f"{d}/phimax.txt"), tol)


@pytest.mark.gpu
def test_cli_fp64_precision_3d(tmp_path):
    d, meta, fields = golden_case("cvd_32x32x8")
    out = tmp_path / "cvd3"
    r = run_cli(["--model", "cvd", "--grid", "32x32x8", "--precision", "fp64", *meta["args"], "--outdir", str(out)])
    assert r.returncode == 0, r.stderr
    for kd in (0, 5, 10):
        vals, _, _ = read_vti(out / f"phi_{kd}_0.vti")
        assert np.abs(vals - fields[f"phi_{kd}"]).max() <= 1e-6
    check_cvd_analysis_files(out, d, (0, 5, 10), 1e-5)
    # without --precision a 3-D grid with N >= 8 runs on the mixed path (--precision mixed):
    # its fields stay within the reference's own float-rounding distance from this FP64 run
    out2 = tmp_path / "cvd3_default"
    r = run_cli(["--model", "cvd", "--grid", "32x32x8", *meta["args"], "--outdir", str(out2)])
    assert r.returncode == 0, r.stderr
    out3 = tmp_path / "cvd3_mixed"
    r = run_cli(["--model", "cvd", "--grid", "32x32x8", "--precision", "mixed", *meta["args"], "--outdir", str(out3)])
    assert r.returncode == 0, r.stderr
    b, _, _ = read_vti(out2 / "phi_10_0.vti")
    c, _, _ = read_vti(out3 / "phi_10_0.vti")
    assert np.array_equal(b, c)
    assert np.abs(b - fields["phi_10"]).max() <= 1e-5
    check_cvd_analysis_files(out2, d, (0, 5, 10), 1e-4)
    # a 3-D grid the mixed kernels do not take (N < 8) defaults to the FP64 path
    out4 = tmp_path / "cvd3_n4"
    r = run_cli(["--model", "cvd", "--grid", "32x32x4", "--steps", "2", "--mod", "1", "--outdir", str(out4)])
    assert r.returncode == 0, r.stderr
    assert (out4 / "phi_1_0.vti").exists()


def test_cli_batch_file_errors(tmp_path):
    """--batch: a malformed or incomplete sweep file is reported before any GPU work."""
    bad = tmp_path / "bad.json"
    bad.write_text('{"model": "misfit", "params": {"u0": {"range": [0.1, 0.05, 0.01]}}, "out_dir": "x"}')
    r = run_cli(["--batch", str(bad)])
    assert r.returncode == 2 and "End must be >= start." in r.stderr
    bad.write_text('{"model": "misfit", "params": {"u0": 0.1}')
    r = run_cli(["--batch", str(bad)])
    assert r.returncode == 2 and "batch file" in r.stderr
    bad.write_text('{"model": "misfit", "params": {"nope": 1}, "out_dir": "x"}')
    r = run_cli(["--batch", str(bad)])
    assert r.returncode == 2 and "unknown parameter nope" in r.stderr
    r = run_cli(["--batch", str(tmp_path / "missing.json")])
    assert r.returncode == 2 and "can't open batch file" in r.stderr


@pytest.mark.gpu
def test_cli_batch_sweep_equals_single_runs(tmp_path):
    """A 2 x 2 sweep (u0 list x seed range) through the engine: runs in the GUI's
    odometer order (last parameter fastest), each folder with params.json and the same
    files pfc-exp-cli writes for that run alone."""
    import json
    root = tmp_path / "exp"
    spec = {"model": "misfit", "out_dir": str(root), "grid": [64, 64, 1],
            "params": {"u0": {"list": [0.05, 0.08]}, "steps": 20, "mod": 10, "seed": {"range": [3, 4, 1]}}}
    f = tmp_path / "sweep.json"
    f.write_text(json.dumps(spec))
    r = run_cli(["--batch", str(f)])
    assert r.returncode == 0, r.stderr
    assert r.stdout.count("PFC_PROGRESS") == 4 and "step=4 total=4" in r.stdout
    runs = sorted(os.listdir(root))
    assert runs == ["run_0001", "run_0002", "run_0003", "run_0004"]
    order = [(0.05, 3), (0.05, 4), (0.08, 3), (0.08, 4)]
    for name, (u0, seed) in zip(runs, order):
        pj = json.load(open(root / name / "params.json"))
        assert pj["mode"] == "experiment" and pj["run_total"] == 4 and pj["out_dir"] == str(root / name)
        assert pj["params"]["u0"] == u0 and pj["params"]["seed"] == seed and pj["params"]["model"] == "misfit"
    single = tmp_path / "single"
    r = run_cli(["--model", "misfit", "--grid", "64x64x1", "--u0", "0.08", "--seed", "4", "--steps", "20",
                 "--mod", "10", "--outdir", str(single)])
    assert r.returncode == 0
    names = sorted(n for n in os.listdir(single) if n != "checkpoint_timestamps.txt")
    assert names == sorted(n for n in os.listdir(root / "run_0004") if n not in ("checkpoint_timestamps.txt",
                                                                               "params.json"))
    for n in names:
        assert (single / n).read_bytes() == (root / "run_0004" / n).read_bytes(), n


@pytest.mark.gpu
@pytest.mark.parametrize("model", ["misfit", "cvd"])
def test_cli_resume_continues_a_run(tmp_path, model):
    """--resume <kd>: continue from the run's own checkpoint files.  The FP32 state is
    rebuilt from Float32 fields, so the continuation matches the uninterrupted run to
    within rounding (1e-5 after 20 more steps)."""
    full, part = tmp_path / "full", tmp_path / "part"
    kd = 20 if model == "misfit" else 10
    base = ["--model", model, "--grid", "64x64x1", "--mod", "10", "--seed", "5"]
    assert run_cli([*base, "--steps", "40", "--outdir", str(full)]).returncode == 0
    # the first leg ends at checkpoint kd (CVD's checkpoint kd follows step kd + 1)
    first = kd if model == "misfit" else kd + 1
    assert run_cli([*base, "--steps", str(first), "--outdir", str(part)]).returncode == 0
    r = run_cli([*base, "--steps", "40", "--resume", str(kd), "--outdir", str(part)])
    assert r.returncode == 0, r.stderr
    last = 40 if model == "misfit" else 30
    a, _, _ = read_vti(full / f"phi_{last}_0.vti")
    b, _, _ = read_vti(part / f"phi_{last}_0.vti")
    assert np.abs(a - b).max() <= 1e-5
    kds = [int(l.split()[0]) for l in (part / "energy.txt").read_text().splitlines()]
    full_kds = [int(l.split()[0]) for l in (full / "energy.txt").read_text().splitlines()]
    # the first leg's energy lines, then the continuation's: the same steps as one run
    assert kds == full_kds
    r = run_cli([*base, "--steps", "40", "--resume", "7", "--outdir", str(part)])
    assert r.returncode == 2 and "can't open input file" in r.stderr
