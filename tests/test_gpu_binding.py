"""The Disco2-side binding, compiled: the reference's own set-up and main loop
with timestep_rk2 replaced by timestep_rk2_gpu, a function of the same
signature over the library (oracle/binding, linked against the reference's
objects and libdisco_gpu.so), against the reference build running
timestep_rk2 on the same parfile.

The C caller packs the reference's cells into the library's row layout,
steps on the GPU and unpacks the result into the reference's own structures
after every step (or, lazy, only at the end), which it dumps.  Bars as in test_gpu_parity: bit-exact where no device
transcendental reaches the result (Gresho), max relative 1e-12 otherwise.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle
from conftest import golden, max_rel

pytestmark = pytest.mark.gpu

EXACT = {"gresho16"}


@pytest.mark.parametrize("name", ["gresho16", "kepler24", "cbd32"])
@pytest.mark.parametrize("fused,lazy", [(False, False), (True, False), (False, True)])
def test_c_main_loop_through_the_library_matches_the_reference(name, fused, lazy):
    if not (os.path.exists(oracle.BINDING_BIN) and oracle.have_ref()):
        pytest.skip("binding or reference build absent (built where the reference sources are mounted)")
    g = golden(name)
    with tempfile.TemporaryDirectory() as td:
        par = os.path.join(td, "case.par")
        with open(par, "w") as f:
            f.write(str(g["parfile"]))
        out = os.path.join(td, "gpu.bin")
        cmd = [oracle.BINDING_BIN, par, "5", out] + (["--fused"] if fused else []) + (["--lazy"] if lazy else [])
        r = subprocess.run(cmd, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        got = oracle.read_state(out)
        want, _, _ = oracle.run(par, 5)
    assert (got.NR, got.N) == (want.NR, want.N)
    for k in ("prim", "cons", "tiph", "dphi"):
        a, b = getattr(got, k), getattr(want, k)
        if name in EXACT:
            assert np.array_equal(a, b), k
        elif k in ("tiph", "dphi"):
            assert np.abs(a - b).max() <= 1e-12 * 2 * np.pi, k
        else:
            assert max_rel(a, b) <= 1e-12, k
    assert abs(got.t - want.t) <= 1e-12 * abs(want.t)
    assert max_rel(got.gm[:, :4], want.gm[:, :4]) <= 1e-12
