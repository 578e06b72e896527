"""Generate the golden fixtures under tests/golden/ from the reference program.

The reference sources (zhiqing0205/PFC-Exp-GUI, src/experiment) are compiled
unmodified by ``make -C oracle ref`` (one binary per grid, FFTW replaced by the
project's FFTW-API shim) into oracle/_ref/.  This script runs those binaries on
the cases below and stores, per case, in tests/golden/<case>/:

  fields.npz        phi_<kd>, con_<kd>: the Float32 values of every kept VTI checkpoint,
                    shaped (L, M, N) in the reference layout n + N*(m + M*l)
  *.txt             the reference's text outputs, verbatim (energy.txt, Phimax_<kd>.txt,
                    run_config.txt; for CVD runs the checkpoint analysis files phimax.txt,
                    phiball_<kd>.cfg, hist_<kd>.txt, Grq6_<kd>.txt, Ql_<kd>.txt, HistQ_<kd>.txt;
                    for the Elastic runs strain_/q4q6_/Phimax_)
  *.vti / *.pvti    a few raw checkpoint files, for byte-level writer tests
  stdout.txt        the reference's stdout (progress and peak-finder lines)
  case.json         the command line and grid

Run from the repository root:  python tests/golden/make_golden.py
It needs the reference sources (only present in the build container); the
fixtures it writes are committed and are all the tests need at run time.
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
ORACLE = os.path.join(ROOT, "oracle")

CASES = [
    # small Misfit run: every checkpoint kept, Elastic on all of them
    dict(name="misfit_64", model="misfit", grid=(64, 64, 1), args=["--steps", "50", "--mod", "25"],
         keep=None, raw=[25], elastic=[[], ["--benchel", "1.3"]]),
    # the plain CPU reference workload: Misfit 256^2, 200 steps, checkpoint every 25; the last
    # checkpoint's fields are kept, Elastic runs on it
    dict(name="misfit_256_c1", model="misfit", grid=(256, 256, 1),
         args=["--steps", "200", "--mod", "25", "--seed", "20200604", "--u0", "0.05", "--con0", "0.2"],
         keep=[25, 200], raw=[], elastic=[[]]),
    # 128^2 with a different seed and composition
    dict(name="misfit_128_s7", model="misfit", grid=(128, 128, 1),
         args=["--steps", "40", "--mod", "20", "--seed", "7", "--u0", "0.08", "--con0", "0.3"],
         keep=None, raw=[], elastic=[[]]),
    # stochastic noise (Gauss + MAINEQUATIONC2_NOI, MIS:490-491, 951-1014)
    dict(name="misfit_64_noise", model="misfit", grid=(64, 64, 1),
         args=["--steps", "6", "--mod", "3", "--axx", "0.005", "--seed", "11"], keep=None, raw=[], elastic=[]),
    # CVD, 2-D and a small 3-D grid
    dict(name="cvd_64", model="cvd", grid=(64, 64, 1), args=["--steps", "21", "--mod", "10"],
         keep=None, raw=[], elastic=[]),
    dict(name="cvd_32x32x8", model="cvd", grid=(32, 32, 8), args=["--steps", "11", "--mod", "5"],
         keep=None, raw=[], elastic=[]),
    # CVD with more atoms: checkpoints 0, 20, 40 (Q6_GLO runs at kd % 20 == 0)
    dict(name="cvd_128", model="cvd", grid=(128, 128, 1), args=["--steps", "41", "--mod", "20", "--u0", "0.05"],
         keep=None, raw=[], elastic=[]),
]

# CVD checkpoint analysis outputs (CVD:1067-1520), kept verbatim
CVD_ANALYSIS = ("phimax.txt", "phiball_", "hist_", "Grq6_", "Ql_", "HistQ_")


def read_vti(path, shape):
    L, M, N = shape
    data = open(path, "rb").read()
    i = data.index(b"_", data.index(b"<AppendedData"))
    vals = np.frombuffer(data[i + 5:i + 5 + 4 * L * M * N], np.float32)
    return vals.reshape(N, M, L).transpose(2, 1, 0).copy()


def ref_binary(grid):
    L, M, N = grid
    path = os.path.join(ORACLE, "_ref", f"pfc-exp-cli-{L}x{M}x{N}")
    if not os.path.exists(path):
        subprocess.run(["make", "-s", "-C", ORACLE, f"_ref/pfc-exp-cli-{L}x{M}x{N}"], check=True)
    return path


def run_case(c):
    out = os.path.join(HERE, c["name"])
    if os.path.isdir(out):
        shutil.rmtree(out)
    os.makedirs(out)
    exe = ref_binary(c["grid"])
    with tempfile.TemporaryDirectory() as tmp:
        run_dir = os.path.join(tmp, "run")
        cmd = [exe, "--model", c["model"], *c["args"], "--outdir", run_dir]
        p = subprocess.run(cmd, capture_output=True, text=True, check=True)
        open(os.path.join(out, "stdout.txt"), "w").write(p.stdout)
        arrays = {}
        steps = sorted(int(f.split("_")[1]) for f in os.listdir(run_dir) if f.startswith("phi_") and f.endswith("_0.vti"))
        keep = steps if c["keep"] is None else [s for s in steps if s in c["keep"]]
        for s in keep:
            arrays[f"phi_{s}"] = read_vti(os.path.join(run_dir, f"phi_{s}_0.vti"), c["grid"])
            arrays[f"con_{s}"] = read_vti(os.path.join(run_dir, f"con_{s}_0.vti"), c["grid"])
        np.savez_compressed(os.path.join(out, "fields.npz"), **arrays)
        for f in sorted(os.listdir(run_dir)):
            if f == "energy.txt" or f == "run_config.txt" or (f.startswith("Phimax_") and int(f[7:-4]) in keep):
                shutil.copy(os.path.join(run_dir, f), out)
            elif c["model"] == "cvd" and f.startswith(CVD_ANALYSIS):
                shutil.copy(os.path.join(run_dir, f), out)
        for s in c["raw"]:
            for f in (f"phi_{s}_0.vti", f"con_{s}_0.vti", f"phi_{s}.pvti", f"con_{s}.pvti"):
                shutil.copy(os.path.join(run_dir, f), out)
        for k, extra in enumerate(c["elastic"]):
            el_in = os.path.join(tmp, "el_in")
            os.makedirs(el_in, exist_ok=True)
            for s in keep:
                for pre in ("phi", "con"):
                    shutil.copy(os.path.join(run_dir, f"{pre}_{s}_0.vti"), el_in)
            el_out = os.path.join(tmp, f"el_out{k}")
            cmd_e = [exe, "--model", "elastic", "--input-dir", el_in, "--outdir", el_out, *extra]
            pe = subprocess.run(cmd_e, capture_output=True, text=True, check=True)
            dst = os.path.join(out, f"elastic{k}")
            os.makedirs(dst)
            open(os.path.join(dst, "stderr.txt"), "w").write(
                "\n".join(l for l in pe.stderr.splitlines() if l.startswith("q4q6_")) + "\n")
            for f in sorted(os.listdir(el_out)):
                if f.split("_")[0] in ("Phimax", "strain", "q4q6"):
                    shutil.copy(os.path.join(el_out, f), dst)
            json.dump({"args": extra, "steps": keep}, open(os.path.join(dst, "case.json"), "w"))
    json.dump({"model": c["model"], "grid": list(c["grid"]), "args": c["args"], "checkpoints": steps, "kept": keep},
              open(os.path.join(out, "case.json"), "w"), indent=1)
    print("wrote", out, "checkpoints", keep)


def main(argv):
    names = set(argv[1:])
    for c in CASES:
        if not names or c["name"] in names:
            run_case(c)


if __name__ == "__main__":
    main(sys.argv)
