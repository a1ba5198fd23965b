"""Golden outputs of the reference's diagnostics_set for the diagnostics test
(run here, where the reference sources are).

For the circumbinary disk at 32 annuli and the Keplerian ring at 24 annuli:
the reference build (oracle/_ref/disco_ref, "diag" mode) creates its
Diagnostics at t = 0, runs 5 RK2 steps and calls diagnostics_set once.  Saved
per workload: t, VectorDiag, ScalarDiag, EquatDiag and the DiagMdot.dat line.

    python tests/golden/make_diag_golden.py      -> tests/golden/diag_*.npz
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from disco2_b200 import configs  # noqa: E402
try:  # run as a script (repo root on the path) or imported by a test (oracle/ on the path)
    from oracle import oracle  # noqa: E402
except ImportError:
    import oracle  # noqa: E402

NSTEPS = 5
WORKLOADS = {"cbd32": lambda: configs.circumbinary(num_r=32), "kepler24": lambda: configs.kepler_ring(num_r=24)}


def read_diag(path: str) -> dict:
    buf = open(path, "rb").read()
    assert buf[:8] == b"DDIAG1\0\0"
    nr, neq = np.frombuffer(buf, np.int32, 2, 8)
    o = 16
    t = np.frombuffer(buf, np.float64, 1, o)[0]
    o += 8
    vec = np.frombuffer(buf, np.float64, nr * 17, o).reshape(nr, 17)
    o += nr * 17 * 8
    scal = np.frombuffer(buf, np.float64, 16, o)
    o += 16 * 8
    eq = np.frombuffer(buf, np.float64, neq * 18, o).reshape(neq, 18)
    return {"t": t, "vector": vec.copy(), "scalar": scal.copy(), "equat": eq.copy()}


def main() -> None:
    oracle.build(ref=True, port=False)
    for name, mk in WORKLOADS.items():
        with tempfile.TemporaryDirectory() as td:
            par = configs.write_parfile(mk(), os.path.join(td, "w.par"))
            out = os.path.join(td, "diag.bin")
            subprocess.run([oracle.REF_BIN, "diag", par, str(NSTEPS), out], check=True, cwd=td,
                           stdout=subprocess.DEVNULL)
            d = read_diag(out)
            line = open(os.path.join(td, "DiagMdot.dat")).read().split()
            d["mdot_line"] = np.array([float(x) for x in line])
        np.savez_compressed(os.path.join(HERE, f"diag_{name}.npz"), nsteps=NSTEPS, **d)
        print(name, "t", d["t"], "rows", d["vector"].shape, "equat", d["equat"].shape)


if __name__ == "__main__":
    main()
