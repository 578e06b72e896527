"""CPU checks of the product library: it loads, and exports every symbol its header declares."""
import ctypes
import os
import subprocess

import pytest

import pfc_b200 as P


def test_header_declares_the_abi():
    names = P.header_functions()
    for n in ("pfc_run_cli", "pfc_run_create", "pfc_run_advance", "pfc_batch_advance", "pfc_phimax_misfit",
              "pfc_phimax_elastic", "pfc_elastic3d", "pfc_cryst_order", "pfc_dft3d", "pfc_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(P.LIB_PATH)
    missing = [n for n in P.header_functions() if not hasattr(lib, n)]
    assert missing == []


def test_nm_shows_c_linkage():
    out = subprocess.run(["nm", "-D", "--defined-only", P.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    for n in P.header_functions():
        assert n in exported


def test_errors_without_device_are_reported_not_fatal():
    """Without a GPU (this container) run creation fails with a message, never a crash."""
    import numpy as np
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("device present")
    with pytest.raises(P.PfcError, match="CUDA|device"):
        P.Run(P.default_params(P.MODEL_MISFIT, L=64, M=64))
    assert P.lib().pfc_last_error()


def test_default_params_follow_reference_cli():
    p = P.default_params(P.MODEL_MISFIT)
    assert (p.L, p.M, p.N) == (256, 256, 1)
    assert abs(p.u0 - 0.05) < 1e-7 and abs(p.sig - 0.05) < 1e-7 and p.grainx == 16 and p.seed == 20200604
    c = P.default_params(P.MODEL_CVD)
    assert abs(c.u0 - 0.01) < 1e-7 and abs(c.sig - 0.03) < 1e-7


def test_cli_binary_links_library():
    assert os.path.exists(P.CLI_PATH)
    out = subprocess.run(["ldd", P.CLI_PATH], capture_output=True, text=True).stdout
    assert "libpfc_b200.so" in out and "not found" not in out.split("libpfc_b200.so")[1].splitlines()[0]
