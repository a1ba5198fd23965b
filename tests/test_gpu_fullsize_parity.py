"""Parity at the benchmark sizes: the device step against the oracle (the
reference build where it was compiled, else the C restatement) on the same
full-size disks, three RK2 steps from the same initial state.

Bars as in test_gpu_parity.py: bit-exact where no device transcendental
reaches the result (Gresho vortex, shear layer, isentropic vortex), max
relative 1e-12 per array otherwise; the Shakura-Sunyaev test problem carries last-ulp
differences further (its bar is CASE_TOL's).
"""
import os
import tempfile

import numpy as np
import pytest

import oracle
from conftest import CASE_TOL, l1_rel, max_rel
from disco2_b200 import configs, lib

pytestmark = pytest.mark.gpu

STEPS = 3
# name -> (parameters, bit-exact, per-step bar)
DISKS = {
    "gresho_96": (configs.gresho(), True, 0.0),
    "kepler_ring_256": (configs.kepler_ring(), False, 1e-12),
    "circumbinary_400": (configs.circumbinary(), False, 1e-12),
    "shear_128": (configs.shear_test(), True, 0.0),
    "sstest_128": (configs.sstest(), False, CASE_TOL["sstest32"][0]),
    # the reference's other initial-data families at their parfiles' sizes
    "vortex_67": (configs.vortex_test(), True, 0.0),
    # its passive scalar (the dye), with the fixed and the outflow boundary
    "vortex_67_dye": (configs.vortex_test(NUM_N=1), True, 0.0),
    "vortex_67_dye_outflow": (configs.vortex_test(NUM_N=1, BoundTypeR=1, RiemannSolver=1), True, 0.0),
    "torus_83": (configs.torus_2d(), False, 1e-12),
    "milos_131": (configs.milos_macfadyen(), False, 1e-12),
    "raddom_131": (configs.rad_dom(), False, 1e-12),
    "middle_131": (configs.middle(), False, 1e-12),
}


@pytest.fixture(scope="module")
def impl():
    if not (oracle.have_ref() or oracle.have_port()):
        oracle.build()
    return "ref" if oracle.have_ref() else "port"


@pytest.mark.parametrize("name", sorted(DISKS))
def test_full_size_steps_match_the_oracle(name, impl):
    p, exact, tol = DISKS[name]
    with tempfile.TemporaryDirectory() as td:
        par = configs.write_parfile(p, os.path.join(td, name + ".par"))
        want, _, _ = oracle.run(par, STEPS, impl=impl)
    sim = lib.Sim(p)
    ctx = lib.Context(sim)
    ctx.init_state(0)
    ctx.step(STEPS)
    got = ctx.get_state(0)
    t, dt = ctx.time(0)
    ctx.close()
    for k in ("prim", "cons"):
        a, b = got[k], getattr(want, k)
        if exact:
            assert np.array_equal(a, b), (k, float(np.abs(a - b).max()))
        else:
            assert max_rel(a, b) <= tol, (k, max_rel(a, b))
    for k in ("tiph", "dphi"):
        d = float(np.abs(got[k] - getattr(want, k)).max())
        assert (d == 0.0) if exact else (d <= max(tol, 1e-12) * 2 * np.pi), (k, d)
    assert abs(t - want.t) <= (0.0 if exact else max(tol, 1e-12) * abs(want.t))


def test_wide_annuli_merge_from_global_memory(impl):
    """Annuli of about 1,500 cells: the pair's phi edges and runs no longer
    fit the merge's 48 KB of shared memory, so it reads them from global
    memory. The face lists of the initial state and of the state three steps
    later, and that state, must be the reference's bit for bit (a Gresho
    vortex, no device transcendental). The reference dumps the face list of
    the state it starts from, so the later list comes from loading the later
    state into it."""
    p = configs.gresho(num_r=8, R_Min=0.3, R_Max=0.31)
    sim = lib.Sim(p)
    N_p, _ = sim.grid()
    need = max(16 * (int(N_p[i]) + int(N_p[i + 1])) + 4 * (int(N_p[i + 1]) + 8) for i in range(len(N_p) - 1))
    assert need > 48 * 1024
    with tempfile.TemporaryDirectory() as td:
        par = configs.write_parfile(p, os.path.join(td, "wide.par"))
        _, f0, _ = oracle.run(par, 0, impl=impl, faces=True)
        want, _, _ = oracle.run(par, STEPS, impl=impl)
        _, f3, _ = oracle.run(par, 0, impl=impl, load=want, faces=True)
    ctx = lib.Context(sim)
    ctx.init_state(0)
    got0 = ctx.face_list(0)
    ctx.step(STEPS)
    got = ctx.get_state(0)
    got3 = ctx.face_list(0)
    ctx.close()
    for f, wf in ((got0, f0), (got3, f3)):
        for k in ("nri", "L", "R", "r", "dphi", "dA", "deltaL", "deltaR", "cm"):
            assert np.array_equal(f[k], getattr(wf, k)), k
    for k in ("prim", "cons", "tiph", "dphi"):
        assert np.array_equal(got[k], getattr(want, k)), k


def test_sweep_disks_in_one_context_match_the_oracle(impl):
    """The two smallest disks of the 48-disk circumbinary sweep (unequal-mass
    binaries, q = 0.62 and 0.017, with their own alpha, h/r, N_r and outer
    radius), advanced together in one context, against the reference run on
    each disk alone: three RK2 steps, max relative 1e-12 per array."""
    sweep = configs.circumbinary_sweep(48, seed=3)
    sims_all = [lib.Sim(p) for p in sweep]
    pick = sorted(range(len(sweep)), key=lambda k: sims_all[k].num_cells)[:2]
    assert all(sweep[k]["MassRatio"] < 0.99 for k in pick)
    sims = [sims_all[k] for k in pick]
    ctx = lib.Context(sims)
    for i in range(len(sims)):
        ctx.init_state(i)
    ctx.step(STEPS)
    tol = 1e-12
    with tempfile.TemporaryDirectory() as td:
        for i, k in enumerate(pick):
            par = configs.write_parfile(sweep[k], os.path.join(td, f"sweep{k}.par"))
            want, _, _ = oracle.run(par, STEPS, impl=impl)
            got = ctx.get_state(i)
            t, _ = ctx.time(i)
            for key in ("prim", "cons"):
                assert max_rel(got[key], getattr(want, key)) <= tol, (k, key, max_rel(got[key], getattr(want, key)))
            for key in ("tiph", "dphi"):
                d = float(np.abs(got[key] - getattr(want, key)).max())
                assert d <= tol * 2 * np.pi, (k, key, d)
            assert abs(t - want.t) <= tol * abs(want.t), (k, t, want.t)
    ctx.close()


@pytest.mark.parametrize("name,make,exact", [("gresho_96", configs.gresho, True),
                                              ("kepler_ring_256", configs.kepler_ring, False),
                                              ("circumbinary_400", configs.circumbinary, False)])
def test_full_size_100_steps_l1(name, make, exact, impl):
    """The headline correctness bar on the three benchmark disks at their full
    sizes: the Gresho vortex (96 annuli, 36k cells), the viscous Keplerian ring
    (256 annuli, 199k cells) and the circumbinary disk (400 annuli, 258k cells)
    after 100 RK2 steps, against the reference run on the host from the same
    initial state. rho (D), momenta (S_r, L) and energy (tau) agree to
    L1-relative 1e-10 and t to 1e-12 relative; the Gresho vortex (no device
    transcendental on its path) bit for bit."""
    p = make()
    with tempfile.TemporaryDirectory() as td:
        par = configs.write_parfile(p, os.path.join(td, name + ".par"))
        want, _, _ = oracle.run(par, 100, impl=impl)
    sim = lib.Sim(p)
    ctx = lib.Context(sim)
    ctx.init_state(0)
    ctx.step(100)
    got = ctx.get_state(0)
    t, _ = ctx.time(0)
    ctx.close()
    if exact:
        for k in ("prim", "cons", "tiph", "dphi"):
            assert np.array_equal(got[k], getattr(want, k)), (k, float(np.abs(got[k] - getattr(want, k)).max()))
        assert t == want.t
    for q in (0, 2, 3, 1):
        assert l1_rel(got["cons"][:, q], want.cons[:, q]) <= 1e-10, (q, l1_rel(got["cons"][:, q], want.cons[:, q]))
    assert abs(t - want.t) <= 1e-12 * abs(want.t)
