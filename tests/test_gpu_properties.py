"""Size-independent properties of the GPU step at the full workload sizes, the
batched (multi-disk) context, the torque objective and the error paths.
"""
import math

import numpy as np
import pytest

from conftest import CASES, golden
from disco2_b200 import configs, lib

pytestmark = pytest.mark.gpu


def test_full_size_determinism_circumbinary():
    """Two runs of the full 258k-cell circumbinary disk are bitwise identical
    (the face merge and every reduction are deterministic, no atomics on data)."""
    sim = lib.Sim(configs.circumbinary())
    out = []
    for _ in range(2):
        ctx = lib.Context(sim)
        ctx.init_state(0)
        ctx.step(3)
        out.append(ctx.get_state(0))
        ctx.close()
    for k in ("prim", "cons", "tiph", "dphi"):
        assert np.array_equal(out[0][k], out[1][k]), k


@pytest.mark.parametrize("make", [configs.circumbinary, configs.kepler_ring, configs.gresho])
def test_full_size_flux_conservation(make):
    """Every face adds -dt*dA*F to its left cell and +dt*dA*F to its right cell, so
    after the phi and r flux phases the sum over all cells of D, tau and L
    (inviscid and viscous parts alike) is unchanged to round-off."""
    sim = lib.Sim(make())
    ctx = lib.Context(sim)
    ctx.init_state(0)
    ctx.step(2)
    st = ctx.get_state(0)
    ctx.stage(0)
    c0 = ctx.get_state(0)["cons"]
    ctx.set_state(0, st["prim"], st["tiph"], st["dphi"])
    ctx.stage(3)
    c3 = ctx.get_state(0)["cons"]
    for q in (0, 1, 3):  # D, tau, L
        d = c3[:, q] - c0[:, q]
        net = math.fsum(d)
        assert abs(net) <= 1e-11 * math.fsum(np.abs(d)), (q, net)
        # and the change is not trivially zero
        assert math.fsum(np.abs(d)) > 0


def test_face_list_full_size_invariants():
    """Per annulus pair the face widths tile the circle, each inner cell's faces
    tile that cell, and every face joins adjacent annuli."""
    sim = lib.Sim(configs.circumbinary())
    ctx = lib.Context(sim)
    ctx.init_state(0)
    ctx.step(5)
    f = ctx.face_list(0)
    N_p, _ = sim.grid()
    off = np.concatenate([[0], np.cumsum(N_p)])
    ann = np.searchsorted(off, f["L"], side="right") - 1
    annR = np.searchsorted(off, f["R"], side="right") - 1
    assert np.all(annR == ann + 1)
    assert np.all(f["dphi"] > 0)
    for i in range(len(N_p) - 1):
        a, b = f["nri"][i], (f["nri"][i + 1] if i + 1 < len(N_p) else len(f["L"]))
        assert abs(f["dphi"][a:b].sum() - 2 * np.pi) < 1e-9
    assert len(f["L"]) == f["nri"][-1]


def test_batched_context_equals_single_disks():
    """One context holding three different disks advances each exactly as a
    context holding that disk alone (per-disk dt, GravMass and boundaries)."""
    gs = [golden(n) for n in CASES]
    sims = [lib.Sim(str(g["parfile"])) for g in gs]
    batch = lib.Context(sims)
    for k in range(len(sims)):
        batch.init_state(k)
    batch.step(5)
    for k, (g, s) in enumerate(zip(gs, sims)):
        single = lib.Context(s)
        single.init_state(0)
        single.step(5)
        a = batch.get_state(k)
        b = single.get_state(0)
        for key in ("prim", "cons", "tiph", "dphi"):
            assert np.array_equal(a[key], b[key]), (k, key)
        assert batch.time(k) == single.time(0)
        single.close()


def _z_span(sim) -> float:
    """dz of the single z layer as sim_set_rz computes it (sim_set.c:130-141)."""
    zs = sim.param("ZLogScale")
    zmin, zmax = sim.param("Z_Min"), sim.param("Z_Max")
    sgn = lambda x: (x > 0) - (x < 0)  # noqa: E731
    z1max = sgn(zmax) * zs * math.log(1.0 + abs(zmax) / zs)
    z1min = sgn(zmin) * zs * math.log(1.0 + abs(zmin) / zs)
    zf = [sgn(z1) * zs * (math.exp(abs(z1) / zs) - 1.0)
          for z1 in (z1min, z1min + (z1max - z1min) / 1.0)]
    return zf[1] - zf[0]


def test_outflow_boundary_full_size():
    """The outflow radial boundary on the full 256-annulus ring: from the prims
    after cons2prim (phase 5), the annuli 0, NR-2 and NR-1 after phase 6 are,
    bit for bit, the dA-weighted sums over the substep's face list divided by
    dz * FacePos(i) * dphi, computed here in face order; every other annulus
    is unchanged (no damping zone)."""
    sim = lib.Sim(configs.kepler_ring(BoundTypeR=1))
    ctx = lib.Context(sim)
    ctx.init_state(0)
    ctx.step(3)
    st = ctx.get_state(0)
    f = ctx.face_list(0)
    ctx.set_state(0, st["prim"], st["tiph"], st["dphi"])
    ctx.stage(5)
    p5 = ctx.get_state(0)
    ctx.set_state(0, st["prim"], st["tiph"], st["dphi"])
    ctx.stage(6)
    p6 = ctx.get_state(0)["prim"]
    N_p, rf = sim.grid()
    NR = len(N_p)
    off = np.concatenate([[0], np.cumsum(N_p)])
    dz = _z_span(sim)
    want = p5["prim"].copy()
    nri = list(f["nri"]) + [len(f["L"])]

    def pair(i, outer):
        dst = i + outer
        acc = {}
        for n in range(nri[i], nri[i + 1]):
            to, frm = (f["R"][n], f["L"][n]) if outer else (f["L"][n], f["R"][n])
            acc.setdefault(to, [0.0] * 5)
            for q in range(5):
                acc[to][q] += float(want[frm, q]) * float(f["dA"][n])
        for g in range(off[dst], off[dst + 1]):
            dA = dz * float(rf[i + 1]) * float(p5["dphi"][g])
            src = acc.get(g, [float(v) for v in want[g]])
            want[g] = [v / dA for v in src]

    pair(0, 0)
    pair(NR - 3, 1)
    pair(NR - 2, 1)
    assert np.array_equal(p6, want)
    inner = slice(off[1], off[NR - 2])
    assert np.array_equal(p6[inner], p5["prim"][inner])
    ctx.close()


def test_batched_sweep_runs():
    """A reduced circumbinary sweep (uneven N_r and N_phi, different q, alpha,
    h/r, outer radius) steps in one context; every disk keeps finite state and
    its own dt."""
    ps = configs.circumbinary_sweep(6, seed=3)
    for p in ps:
        p["NumR"] = min(p["NumR"], 96)
    sims = [lib.Sim(p) for p in ps]
    ctx = lib.Context(sims)
    for k in range(len(sims)):
        ctx.init_state(k)
    ctx.step(4)
    dts = []
    for k in range(len(sims)):
        st = ctx.get_state(k)
        assert np.all(np.isfinite(st["cons"]))
        dts.append(ctx.time(k)[1])
    assert len(set(dts)) > 1


def test_torque_matches_host_formula():
    """dgpu_torque = -sum over non-ghost cells of r*rho*dV*F_phi with the
    point-mass force of gravMassForce (src/Cell/cell_source.c:49-71)."""
    p = configs.circumbinary(num_r=32)
    sim = lib.Sim(p)
    ctx = lib.Context(sim)
    ctx.init_state(0)
    ctx.step(3)
    st = ctx.get_state(0)
    gm = ctx.gravmass(0)
    N_p, rf = sim.grid()
    off = np.concatenate([[0], np.cumsum(N_p)])
    eps = p["G_EPS"]
    tot = 0.0
    for i in range(1, len(N_p) - 1):
        rm, rp = rf[i], rf[i + 1]
        r = 0.5 * (rp + rm)
        sl = slice(off[i], off[i + 1])
        dphi = st["dphi"][sl]
        phi = st["tiph"][sl] - 0.5 * dphi
        rho = st["prim"][sl, 0]
        dV = dphi * 0.5 * (rp * rp - rm * rm) * 2.0  # dz of the single layer is ~2
        Fp = np.zeros_like(phi)
        for q in range(2):
            dx = r * np.cos(phi) - gm[q, 0] * np.cos(gm[q, 1])
            dy = r * np.sin(phi) - gm[q, 0] * np.sin(gm[q, 1])
            sr = np.sqrt(dx * dx + dy * dy)
            f = gm[q, 2] * sr / (sr * sr + eps * eps) ** 1.5
            Fp += (dy / sr * np.cos(phi) - dx / sr * np.sin(phi)) * -f
        tot += -(r * rho * dV * Fp).sum()
    got = ctx.torque(0)
    assert got == pytest.approx(tot, rel=1e-6)


def test_nan_state_is_reported():
    """A NaN in one interior cell spreads through its fluxes; the reference's
    CFL minimum skips such cells and runs on, here the step also reports it."""
    g = golden("kepler24")
    sim = lib.Sim(str(g["parfile"]))
    ctx = lib.Context(sim)
    ctx.init_state(0)
    st = ctx.get_state(0)
    prim = st["prim"].copy()
    prim[500, 0] = np.nan
    ctx.set_state(0, prim, st["tiph"], st["dphi"])
    with pytest.raises(lib.DiscoError, match="non-finite"):
        ctx.step(2)
    ctx.close()


def test_nonfinite_phi_edge_is_reported_not_hung():
    """A non-finite phi edge makes the reference loop forever in its wrap loops;
    here the bounded loops set an error flag that surfaces as NUMERIC."""
    g = golden("gresho16")
    sim = lib.Sim(str(g["parfile"]))
    ctx = lib.Context(sim)
    ctx.init_state(0)
    st = ctx.get_state(0)
    tiph = st["tiph"].copy()
    tiph[100] = np.inf
    ctx.set_state(0, st["prim"], tiph, st["dphi"])
    with pytest.raises(lib.DiscoError) as e:
        ctx.step(1)
    assert e.value.code in (-5, -6)
    # the context stays usable after the error is reported
    ctx2 = lib.Context(sim)
    ctx2.init_state(0)
    ctx2.step(1)
