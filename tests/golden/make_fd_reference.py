"""Central finite differences of the reference C code for the gradient check
(run here, where the reference sources are; the GPU test reads the output).

Workload: the circumbinary disk reduced to 192 annuli, 500 RK2 steps, the
objectives averaged (dt-weighted) over steps 251-500: the binary torque and
the accretion rate through the innermost non-ghost annulus, computed after
each step by oracle/_ref/disco_ref in its "objective" mode.  The dt schedule
is frozen at the unperturbed run's CFL values (--dtfile), which is how the
derivatives are defined.  Parameters: the mass ratio q, alpha and 16 seeded
directions of the initial surface density (d rho = rho u, d P = P u with
u ~ N(0, 1) per cell from numpy's default_rng(1000 + k)); relative steps
1e-6 and 1e-8.

    python tests/golden/make_fd_reference.py [--jobs 8]
writes tests/golden/cbd192_fd.json.

    python tests/golden/make_fd_reference.py --short
writes tests/golden/cbd192_fd_short.json: the same disk without its initial
1e-4 noise (IC_Noise 0) over 20 steps, the objectives averaged over steps
11-20, relative steps 1e-6, 1e-7 and 1e-8.  With the noise the phi slopes
are noise-dominated and a perturbation of 1e-6 reorders the limiter's
candidates in many cells, so no step converges; without it the base phi
slopes are smooth.  The spread of the three steps measures how far the
differences themselves have converged.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
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

NUM_R, NSTEPS, WINDOW = 192, 500, 250
Q0, ALPHA0 = 1.0, 0.1
EXTRA = {}  # parameters over the circumbinary defaults (the converged case: IC_Noise 0)
STEPS = (1e-6, 1e-8)
N_DIRS = 16
OUT = os.path.join(HERE, "cbd192_fd.json")


def direction(prim0: np.ndarray, k: int) -> np.ndarray:
    u = np.random.default_rng(1000 + k).standard_normal(prim0.shape[0])
    d = np.zeros_like(prim0)
    d[:, 0] = prim0[:, 0] * u
    d[:, 1] = prim0[:, 1] * u
    return d


def _set_extra(extra: dict) -> None:
    EXTRA.update(extra)


def _objective(args) -> list[float]:
    """J = (torque, accretion) means over the window for one perturbed run."""
    work, tag, q, alpha, prim_file, dtfile, NSTEPS, WINDOW = args
    par = os.path.join(work, f"{tag}.par")
    configs.write_parfile(configs.circumbinary(num_r=NUM_R, q=q, alpha=alpha, **EXTRA), par)
    out = os.path.join(work, f"{tag}.txt")
    cmd = [oracle.REF_BIN, "objective", par, str(NSTEPS), out, "--load", prim_file]
    if dtfile:
        cmd += ["--dtfile", dtfile]
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
    a = np.loadtxt(out)
    w = a[WINDOW:, 2]
    return [float(np.sum(w * a[WINDOW:, 3]) / np.sum(w)), float(np.sum(w * a[WINDOW:, 4]) / np.sum(w))]


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 4)
    ap.add_argument("--short", action="store_true")
    args = ap.parse_args()
    if args.short:
        NSTEPS, WINDOW, STEPS_ = 20, 10, (1e-6, 1e-7, 1e-8)
        EXTRA.update({"IC_Noise": 0.0})
        out_path = OUT.replace(".json", "_short.json")
    else:
        NSTEPS, WINDOW, STEPS_ = globals()["NSTEPS"], globals()["WINDOW"], STEPS
        out_path = OUT
    oracle.build(ref=True, port=False)
    work = tempfile.mkdtemp(prefix="fdref_")
    par0 = os.path.join(work, "base.par")
    configs.write_parfile(configs.circumbinary(num_r=NUM_R, q=Q0, alpha=ALPHA0, **EXTRA), par0)
    init = oracle.run(par0, 0)[0]  # the reference's initial state
    base_state = os.path.join(work, "init.bin")
    oracle.write_state(base_state, init)
    # unperturbed run with the CFL dt: the schedule every other run replays
    out0 = os.path.join(work, "base.txt")
    subprocess.run([oracle.REF_BIN, "objective", par0, str(NSTEPS), out0, "--load", base_state], check=True,
                   stdout=subprocess.DEVNULL)
    a0 = np.loadtxt(out0)
    dtfile = os.path.join(work, "dt.txt")
    np.savetxt(dtfile, a0[:, 2], fmt="%.17g")
    w0 = a0[WINDOW:, 2]
    J0 = [float(np.sum(w0 * a0[WINDOW:, 3]) / np.sum(w0)), float(np.sum(w0 * a0[WINDOW:, 4]) / np.sum(w0))]

    jobs, keys = [], []
    for h in STEPS_:
        for sgn in (+1, -1):
            jobs.append((work, f"q_{h}_{sgn}", Q0 * (1 + sgn * h), ALPHA0, base_state, dtfile, NSTEPS, WINDOW))
            keys.append(("q", h, sgn))
            jobs.append((work, f"a_{h}_{sgn}", Q0, ALPHA0 * (1 + sgn * h), base_state, dtfile, NSTEPS, WINDOW))
            keys.append(("alpha", h, sgn))
            for k in range(N_DIRS):
                st = oracle.read_state(base_state)
                st.prim = init.prim + sgn * h * direction(init.prim, k)
                f = os.path.join(work, f"s{k}_{h}_{sgn}.bin")
                oracle.write_state(f, st)
                jobs.append((work, f"s{k}_{h}_{sgn}", Q0, ALPHA0, f, dtfile, NSTEPS, WINDOW))
                keys.append((f"sigma{k}", h, sgn))
    with mp.get_context("spawn").Pool(args.jobs, initializer=_set_extra, initargs=(dict(EXTRA),)) as pool:
        res = pool.map(_objective, jobs)
    J = {key: np.array(r) for key, r in zip(keys, res)}
    fd = {}
    for h in STEPS_:
        d = {}
        d["q"] = ((J[("q", h, 1)] - J[("q", h, -1)]) / (2 * h * Q0)).tolist()
        d["alpha"] = ((J[("alpha", h, 1)] - J[("alpha", h, -1)]) / (2 * h * ALPHA0)).tolist()
        d["sigma"] = [((J[(f"sigma{k}", h, 1)] - J[(f"sigma{k}", h, -1)]) / (2 * h)).tolist()
                      for k in range(N_DIRS)]
        fd[f"{h:g}"] = d
    out = {"workload": f"circumbinary disk, {NUM_R} annuli, q={Q0}, alpha={ALPHA0}",
           "params": dict(EXTRA),
           "num_r": NUM_R, "nsteps": NSTEPS, "window_start": WINDOW, "cells": int(init.N),
           "J": J0, "dt_sum_window": float(np.sum(w0)), "fd": fd,
           "direction": "d rho = rho0 u, d P = P0 u, u = numpy default_rng(1000 + k).standard_normal(N)",
           "generator": "tests/golden/make_fd_reference.py (reference objective mode, frozen dt)"}
    with open(out_path, "w") as fh:
        json.dump(out, fh, indent=1)
    print("wrote", out_path, "J", J0)


if __name__ == "__main__":
    main()
