"""The diagnostics fixtures are the reference's own output: rebuilt from the
reference build (where its sources are), they come out bit for bit."""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

import oracle
from disco2_b200 import configs

HERE = os.path.dirname(os.path.abspath(__file__))


def test_fixture_shapes():
    for name, nr in (("cbd32", 32), ("kepler24", 24)):
        d = np.load(os.path.join(HERE, "golden", f"diag_{name}.npz"))
        assert d["vector"].shape == (nr, 17) and d["scalar"].shape == (16,)
        assert d["equat"].shape[1] == 18 and d["mdot_line"].shape == (13,)


@pytest.mark.skipif(not oracle.have_ref(), reason="reference build not present")
def test_reference_reproduces_fixture():
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_diag_golden import read_diag
    ref = np.load(os.path.join(HERE, "golden", "diag_cbd32.npz"))
    with tempfile.TemporaryDirectory() as td:
        par = configs.write_parfile(configs.circumbinary(num_r=32), os.path.join(td, "w.par"))
        out = os.path.join(td, "d.bin")
        subprocess.run([oracle.REF_BIN, "diag", par, str(int(ref["nsteps"])), out], check=True, cwd=td,
                       stdout=subprocess.DEVNULL)
        d = read_diag(out)
    assert d["t"] == ref["t"]
    for k in ("vector", "scalar"):
        v, r = d[k].copy(), ref[k].copy()
        if k == "vector":  # the passive-scalar column reads past prim[]
            v[:, 8] = r[:, 8] = 0.0
        assert np.array_equal(v, r), k
