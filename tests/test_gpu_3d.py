"""The 3-D path (NumZ > 1) against the reference build: the torus of the
reference's parfiles/torus.par (a torus about a point mass, at most 20 cells
per ring, two ghost annuli and layers, outflow in r, periodic in z).

- tests/golden/torus3d16.npz (16 annuli x 8 layers, 4,200 cells, made by
  tests/golden/make_golden.py --three-d): the r- and z-face lists bit for bit,
  the state after 1 and 5 steps within max relative 1e-12 and after 100 steps
  within L1-relative 1e-10 (rho, S_r, L, tau; the device pow, sin and cos
  differ from the host's in the last ulp);
- torus.par at its own size (80 x 80, 139,440 cells): three steps against the
  reference run on the host, max relative 1e-12.
"""
import os
import tempfile

import numpy as np
import pytest

import oracle
from conftest import golden, l1_rel, max_rel
from disco2_b200 import configs, lib

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-12


def _ctx(g):
    sim = lib.Sim(str(g["parfile"]))
    ctx = lib.Context(sim)
    ctx.init_state(0)
    return ctx


def _compare(st, g, prefix, tol):
    for k in ("prim", "cons"):
        assert max_rel(st[k], g[prefix + k]) <= tol, (k, max_rel(st[k], g[prefix + k]))
    for k in ("tiph", "dphi"):
        d = float(np.abs(st[k] - g[prefix + k]).max())
        assert d <= tol * 2 * np.pi, (k, d)


def test_initial_state_and_face_lists_bitexact():
    g = golden("torus3d16")
    ctx = _ctx(g)
    st = ctx.get_state(0)
    for k in ("prim", "cons", "tiph", "dphi"):
        assert np.array_equal(st[k], g["init_" + k]), k
    fr = ctx.face_list(0)
    fz = ctx.face_list(0, z=True)
    ctx.close()
    for k in ("nri", "L", "R", "r", "dphi", "dA", "deltaL", "deltaR", "cm"):
        assert np.array_equal(fr[k], g["init_face_" + k]), ("r", k)
        assert np.array_equal(fz[k], g["init_zface_" + k]), ("z", k)


@pytest.mark.parametrize("nsteps", [1, 5])
def test_steps(nsteps):
    g = golden("torus3d16")
    ctx = _ctx(g)
    ctx.step(nsteps)
    st = ctx.get_state(0)
    t, dt = ctx.time(0)
    ctx.close()
    _compare(st, g, f"step{nsteps}_", STEP_TOL)
    assert abs(t - float(g[f"step{nsteps}_t"])) <= STEP_TOL * abs(float(g[f"step{nsteps}_t"]))


def test_100_steps_l1():
    g = golden("torus3d16")
    ctx = _ctx(g)
    ctx.step(100)
    st = ctx.get_state(0)
    t, _ = ctx.time(0)
    ctx.close()
    want = g["step100_cons"]
    for q in (0, 2, 3, 1):
        assert l1_rel(st["cons"][:, q], want[:, q]) <= 1e-10, (q, l1_rel(st["cons"][:, q], want[:, q]))
    assert abs(t - float(g["step100_t"])) <= 1e-10 * abs(float(g["step100_t"]))


def test_torus_par_full_size_three_steps():
    if not oracle.have_ref():
        pytest.skip("the reference build is needed for the full-size run")
    p = configs.torus_3d()
    with tempfile.TemporaryDirectory() as td:
        par = configs.write_parfile(p, os.path.join(td, "torus.par"))
        want, _, _ = oracle.run(par, 3)
    sim = lib.Sim(p)
    assert sim.num_cells == want.N == 139440
    ctx = lib.Context(sim)
    ctx.init_state(0)
    ctx.step(3)
    got = ctx.get_state(0)
    t, _ = ctx.time(0)
    ctx.close()
    for k in ("prim", "cons"):
        assert max_rel(got[k], getattr(want, k)) <= STEP_TOL, (k, max_rel(got[k], getattr(want, k)))
    for k in ("tiph", "dphi"):
        assert float(np.abs(got[k] - getattr(want, k)).max()) <= STEP_TOL * 2 * np.pi, k
    assert abs(t - want.t) <= STEP_TOL * abs(want.t)


def test_three_d_refusals():
    g = golden("torus3d16")
    ctx = _ctx(g)
    with pytest.raises(lib.DiscoError):
        ctx.set_fused(True)
    with pytest.raises(lib.DiscoError):
        ctx.stage(0)
    ctx.close()
    with pytest.raises(lib.DiscoError):
        lib.Context(lib.Sim(configs.torus_3d(num_r=16, num_z=8, BoundTypeZ=1)))


def test_torus_par_full_size_100_steps_l1():
    """torus.par at its own size after 100 RK2 steps against the reference on
    the host: L1-relative 1e-10 in rho, S_r, L and tau."""
    if not oracle.have_ref():
        pytest.skip("the reference build is needed for the full-size run")
    p = configs.torus_3d()
    with tempfile.TemporaryDirectory() as td:
        par = configs.write_parfile(p, os.path.join(td, "torus.par"))
        want, _, _ = oracle.run(par, 100)
    ctx = lib.Context(lib.Sim(p))
    ctx.init_state(0)
    ctx.step(100)
    got = ctx.get_state(0)
    t, _ = ctx.time(0)
    ctx.close()
    for q in (0, 2, 3, 1):
        assert l1_rel(got["cons"][:, q], want.cons[:, q]) <= 1e-10, (q, l1_rel(got["cons"][:, q], want.cons[:, q]))
    assert abs(t - want.t) <= 1e-12 * abs(want.t)
