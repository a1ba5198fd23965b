"""Generate the golden fixtures of tests/golden/ from the reference build.

Run where the reference sources are mounted (oracle/_ref/disco_ref is built
from them by oracle/Makefile):

    python tests/golden/make_golden.py               # <case>.npz
    python tests/golden/make_golden.py --substep2    # <case>_sub2.npz
    python tests/golden/make_golden.py --three-d     # the 3-D cases' <case>.npz
    python tests/golden/make_golden.py --checkpoint  # ckpt_<case>.npz

Every fixture is the reference's own output (timestep_rk2 / face_create /
the substep phases of timestep_substep) on a small disk, stored as a
compressed .npz.  The reference has no tests or golden data of its own, so
these are the pins of the oracle and of the GPU path.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402
from disco2_b200 import configs  # noqa: E402

# name -> parameter dict of a small disk of each workload
CASES = {
    "gresho16": configs.gresho(num_r=16),
    "kepler24": configs.kepler_ring(num_r=24),
    "cbd32": configs.circumbinary(num_r=32),
    # outflow radial boundary (cell_boundary_outflow_r): one ghost annulus a
    # side, so the boundary also overwrites the last non-ghost annulus NR-2
    "kepler24out": configs.kepler_ring(num_r=24, BoundTypeR=1),
    # two ghost annuli a side, outer damping zone applied after the boundary
    "cbd32out": configs.circumbinary(num_r=32, BoundTypeR=1, ng=2),
    # no inner boundary (annulus 0 reaches the origin): outer boundary only
    "kepler12noin": configs.kepler_ring(num_r=12, BoundTypeR=1, NoInnerBC=1),
    # three annuli: annulus 0 is written by the inner boundary and then read
    # by the outer one, annulus 1 is read by the inner one and then written
    "kepler1out": configs.kepler_ring(num_r=1, R_Min=1.0, R_Max=1.2, BoundTypeR=1),
    # the reference's test problems (parfiles/code_tests) and the other
    # initial-data families (src/Cell/initial_data), reduced in size
    "shear12": configs.shear_test(num_r=12),
    "sstest32": configs.sstest(num_r=32),
    "vortex16": configs.vortex_test(num_r=16, R_Min=0.1),
    "torus16": configs.torus_2d(num_r=16),
    "milos16": configs.milos_macfadyen(num_r=16),
    "raddom16": configs.rad_dom(num_r=16),
    "middle16": configs.middle(num_r=16),
    # a passive scalar (NUM_N = 1): the vortex's dye, HLLC with the fixed
    # boundary that resets it by phi, and HLL with the outflow boundary
    "vortex16dye": configs.vortex_test(num_r=16, R_Min=0.1, NUM_N=1),
    "vortex16dyeout": configs.vortex_test(num_r=16, R_Min=0.1, NUM_N=1, BoundTypeR=1, RiemannSolver=1),
}
STEPS = (1, 5, 100)
PHASES = (0, 1, 2, 3, 4, 5, 6, 7)
# per phase, the arrays that phase of timestep_substep changes
PHASE_KEYS = {0: ("cons", "wiph", "RKcons"), 1: ("grad", "gradp"), 2: ("cons",), 3: ("cons",),
              4: ("cons",), 5: ("prim", "tiph", "dphi", "RKtiph"), 6: ("prim",),
              7: ("prim", "cons")}


def _state_dict(st: oracle.State, prefix: str, ext: bool = False) -> dict:
    d = {f"{prefix}prim": st.prim, f"{prefix}cons": st.cons, f"{prefix}tiph": st.tiph,
         f"{prefix}dphi": st.dphi, f"{prefix}gm": st.gm, f"{prefix}t": np.float64(st.t),
         f"{prefix}dt": np.float64(st.dt)}
    if ext:
        for k, v in st.ext.items():
            d[f"{prefix}{k}"] = v
    return d


def _faces_dict(fc: oracle.Faces, prefix: str, full: bool = True) -> dict:
    keys = ("nri", "L", "R", "r", "dphi", "dA", "deltaL", "deltaR", "cm") if full else \
        ("nri", "L", "R", "dphi", "dA", "cm")
    return {f"{prefix}{k}": getattr(fc, k) for k in keys}


def face_cases(par: str, st0: oracle.State, rng: np.random.Generator) -> dict:
    """Face lists of perturbed phi-edge layouts: random rotations, exactly aligned
    edges, edges given far outside [0, 2pi] (the wrap loops), jittered cells."""
    out = {}
    off = st0.cell_off
    layouts = {}
    # 1. a random rotation per annulus
    t = st0.tiph.copy()
    d = st0.dphi.copy()
    for i in range(st0.NR):
        a, b = off[i], off[i + 1]
        n = b - a
        dp = 2 * np.pi / n
        t[a:b] = rng.uniform(0, 2 * np.pi) + np.arange(n) * dp
        d[a:b] = dp
    layouts["rot"] = (t.copy(), d.copy())
    # 2. all annuli start at phi = 0: inner and outer edges coincide exactly where
    #    j/N_i == k/N_o
    t2 = t.copy()
    for i in range(st0.NR):
        a, b = off[i], off[i + 1]
        n = b - a
        t2[a:b] = np.arange(1, n + 1) * (2 * np.pi / n)
    layouts["aligned"] = (t2, d.copy())
    # 3. the rotated layout shifted by whole turns (the reference wraps on the fly)
    t3 = t + 2 * np.pi * rng.integers(-3, 4, size=t.size)
    layouts["turns"] = (t3, d.copy())
    # 4. jittered cell widths (sliding mesh after many steps): edges perturbed, dphi
    #    recomputed as cell_update_dphi does
    t4 = t.copy()
    d4 = d.copy()
    for i in range(st0.NR):
        a, b = off[i], off[i + 1]
        n = b - a
        dp = 2 * np.pi / n
        t4[a:b] += rng.uniform(-0.3, 0.3, size=n) * dp
        for j in range(n):
            jm = j - 1 if j > 0 else n - 1
            x = t4[a + j] - t4[a + jm]
            while x > 2 * np.pi:
                x -= 2 * np.pi
            while x < 0.0:
                x += 2 * np.pi
            d4[a + j] = x
    # with fewer than 3 cells in an annulus a jittered layout can leave an inner
    # cell ahead of every outer edge, where build_jloop's advance loop never ends
    if st0.N_p.min() >= 3:
        layouts["jitter"] = (t4, d4)
    for name, (tt, dd) in layouts.items():
        st = oracle.State(st0.NR, st0.NZ, st0.NQ, st0.N, 0.0, 0.0, st0.gm, st0.N_p, st0.r_faces,
                          st0.prim, st0.cons, tt, dd)
        _, fc, _ = oracle.run(par, 0, load=st, faces=True)
        out[f"layout_{name}_tiph"] = tt
        out[f"layout_{name}_dphi"] = dd
        out.update(_faces_dict(fc, f"layout_{name}_face_", full=False))
    return out


# the second substep's phases (dgpu_stage / the driver's stage mode 8-15):
# the whole first substep, gravMass_move, then the second substep stopped
# after phase - 8.  Its RKtiph is left out: the reference re-adjusts RKtiph by
# whole turns in the second cell_update_phi, a copy that nothing reads after
# the substep and that the GPU does not store.
PHASES2 = tuple(range(8, 16))
PHASE2_KEYS = {ph: tuple(k for k in PHASE_KEYS[ph - 8] if k != "RKtiph") for ph in PHASES2}


def substep2(names: list[str]) -> None:
    """Writes <name>_sub2.npz: the second substep's phases of each case, from
    the same 5-step state as the first substep's phases."""
    if not oracle.have_ref():
        oracle.build(ref=True, port=False)
    with tempfile.TemporaryDirectory() as td:
        for name, p in CASES.items():
            if names and name not in names:
                continue
            par = configs.write_parfile(p, os.path.join(td, name + ".par"))
            data = {"parfile": np.array(configs.parfile_text(p))}
            st5 = oracle.run(par, 5)[0]
            for ph in PHASES2:
                st = oracle.stage(par, ph, load=st5)
                full = _state_dict(st, "", ext=True)
                for k in PHASE2_KEYS[ph]:
                    data[f"stage{ph}_{k}"] = full[k]
                data[f"stage{ph}_dt"] = np.float64(st.dt)
                data[f"stage{ph}_gm"] = st.gm
            path = os.path.join(HERE, name + "_sub2.npz")
            np.savez_compressed(path, **data)
            print(name, "second substep", os.path.getsize(path), "bytes")


# 3-D disks (NumZ > 1): the reference's own torus.par reduced in size.  The C
# restatement of the oracle is 2-D only, so these pin the GPU path alone.
CASES3D = {
    "torus3d16": configs.torus_3d(num_r=16, num_z=8),
}


def three_d(names: list[str]) -> None:
    """Writes <name>.npz for the 3-D cases: the initial state, its r- and
    z-face lists, and the states after 1, 5 and 100 RK2 steps."""
    if not oracle.have_ref():
        oracle.build(ref=True, port=False)
    with tempfile.TemporaryDirectory() as td:
        for name, p in CASES3D.items():
            if names and name not in names:
                continue
            par = configs.write_parfile(p, os.path.join(td, name + ".par"))
            data = {"parfile": np.array(configs.parfile_text(p))}
            st0, fr, _ = oracle.run(par, 0, faces=True)
            _, fz, _ = oracle.run(par, 0, faces=True, zfaces=True)
            data.update(_state_dict(st0, "init_"))
            data["N_p"] = st0.N_p
            data.update(_faces_dict(fr, "init_face_"))
            data.update(_faces_dict(fz, "init_zface_"))
            for n in STEPS:
                st, _, log = oracle.run(par, n, dtlog=True)
                data.update(_state_dict(st, f"step{n}_"))
                data[f"step{n}_dtlog"] = log
            path = os.path.join(HERE, name + ".npz")
            np.savez_compressed(path, **data)
            print(name, st0.N, "cells", os.path.getsize(path), "bytes")


CKPT_CASES = ("gresho16", "kepler24", "cbd32", "torus3d16", "vortex16dye")


def checkpoint(names: list[str]) -> None:
    """Writes ckpt_<name>.npz: the reference's checkpoint buffer (io_setbuf)
    of the initial state (ck0_) and after 5 RK2 steps (ck5_), the state
    after the reference's restart set-up from the 5-step buffer (rs_), and
    after 5 more steps from there (rs5_)."""
    if not oracle.have_ref():
        oracle.build(ref=True, port=False)
    cases = {**CASES, **CASES3D}
    with tempfile.TemporaryDirectory() as td:
        for name in CKPT_CASES:
            if names and name not in names:
                continue
            p = cases[name]
            par = configs.write_parfile(p, os.path.join(td, name + ".par"))
            data = {"parfile": np.array(configs.parfile_text(p))}
            for n in (0, 5):
                ck = oracle.checkpoint(par, n)
                data[f"ck{n}_t"] = np.float64(ck["t"])
                data[f"ck{n}_gm"] = ck["gravmass"]
                data[f"ck{n}_data"] = ck["data"]
            ck5 = oracle.checkpoint(par, 5)
            for n in (0, 5):
                st = oracle.run(par, n, restart=ck5)[0]
                data.update(_state_dict(st, "rs_" if n == 0 else f"rs{n}_"))
            path = os.path.join(HERE, f"ckpt_{name}.npz")
            np.savez_compressed(path, **data)
            print(name, os.path.getsize(path), "bytes")


def main(names: list[str]) -> None:
    """Writes the fixtures of the named cases (all cases when none is named);
    each case draws its face layouts from its own seeded generator."""
    if not oracle.have_ref():
        oracle.build(ref=True, port=False)
    with tempfile.TemporaryDirectory() as td:
        for k, (name, p) in enumerate(CASES.items()):
            if names and name not in names:
                continue
            rng = np.random.default_rng(20251203 + k)
            par = configs.write_parfile(p, os.path.join(td, name + ".par"))
            data = {"parfile": np.array(configs.parfile_text(p))}
            st0, fc0, _ = oracle.run(par, 0, faces=True)
            data.update(_state_dict(st0, "init_"))
            data["N_p"] = st0.N_p
            data["r_faces"] = st0.r_faces
            data.update(_faces_dict(fc0, "init_face_"))
            for n in STEPS:
                st, _, log = oracle.run(par, n, dtlog=True)
                data.update(_state_dict(st, f"step{n}_"))
                data[f"step{n}_dtlog"] = log
            # stage phases of one substep from the 5-step state (loaded: prim, tiph,
            # dphi; t = 0 and the initial GravMass)
            st5 = oracle.run(par, 5)[0]
            for ph in PHASES:
                st = oracle.stage(par, ph, load=st5)
                full = _state_dict(st, "", ext=True)
                for k in PHASE_KEYS[ph]:
                    data[f"stage{ph}_{k}"] = full[k]
                data[f"stage{ph}_dt"] = np.float64(st.dt)
                data[f"stage{ph}_gm"] = st.gm
            data.update(face_cases(par, st0, rng))
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **data)
            print(name, st0.N, "cells", os.path.getsize(os.path.join(HERE, name + ".npz")), "bytes")


if __name__ == "__main__":
    if sys.argv[1:2] == ["--substep2"]:
        substep2(sys.argv[2:])
    elif sys.argv[1:2] == ["--three-d"]:
        three_d(sys.argv[2:])
    elif sys.argv[1:2] == ["--checkpoint"]:
        checkpoint(sys.argv[2:])
    else:
        main(sys.argv[1:])
