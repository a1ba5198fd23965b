"""Hand-written adjoints of the per-face and per-cell physics against the
Dual tangent of the same forward code (dot-product tests, host build).

tests/adjoint_local/check_local.cu is compiled by nvcc as host code: the
templated forward functions run on Dual numbers, the *_rev functions on
doubles, and <l, J v> is compared with <J^T l, v> over random inputs that
reach every HLLC state, limiter branch and floor/cap clamp."""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
NVCC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    if not os.path.exists(NVCC):
        pytest.skip("nvcc not available")
    exe = str(tmp_path_factory.mktemp("adj") / "check_local")
    subprocess.run([NVCC, "-std=c++17", "-O2", "-Wno-deprecated-gpu-targets", "-Xcompiler", "-ffp-contract=off",
                    "-o", exe, os.path.join(HERE, "adjoint_local", "check_local.cu")], check=True)
    return exe


def test_local_adjoints_match_tangent(checker):
    out = subprocess.run([checker], capture_output=True, text=True)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr
    lines = {ln.split()[0]: ln for ln in out.stdout.splitlines() if "max_rel=" in ln}
    for name in ("riemann_flux", "visc_flux", "source_cell", "update_chain", "plm_p_slope"):
        assert name in lines
        rel = float(lines[name].split("max_rel=")[1].split()[0])
        assert rel < 1e-10, lines[name]
    # every Riemann state and every limiter branch was exercised
    assert "left 0" not in lines["riemann_flux"] and "right 0" not in lines["riemann_flux"]
    assert "centred 0" not in lines["plm_p_slope"]
