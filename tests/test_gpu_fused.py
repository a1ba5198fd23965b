"""The fused substep (k_prep + k_sweep) against the eight-kernel substep.

Both forms evaluate the same per-face and per-cell functions in the same
order, so the fused step must equal the eight-kernel step bit for bit: state,
time, dt and the GravMass orbit.  The eight-kernel form, the default, is
itself pinned to the reference build (test_gpu_parity.py,
test_gpu_fullsize_parity.py).
"""
import numpy as np
import pytest

from conftest import CASES, golden
from disco2_b200 import configs, lib

pytestmark = pytest.mark.gpu

KEYS = ("prim", "cons", "tiph", "dphi")


def _advance(sims, fused: bool, nsteps: int, loads=None):
    ctx = lib.Context(sims)
    ctx.set_fused(fused)
    for k in range(len(ctx.sims)):
        ctx.init_state(k)
        if loads is not None and loads[k] is not None:
            ctx.set_state(k, *loads[k])
    ctx.step(nsteps)
    out = []
    for k in range(len(ctx.sims)):
        st = ctx.get_state(k)
        st["time"] = np.array(ctx.time(k))
        st["gm"] = ctx.gravmass(k)
        out.append(st)
    ctx.close()
    return out


def _same(a, b, what):
    for k in KEYS + ("time", "gm"):
        assert np.array_equal(a[k], b[k]), (what, k, np.abs(a[k] - b[k]).max())


def _eligible(sim) -> bool:
    ctx = lib.Context(sim)
    try:
        ctx.set_fused(True)
        return True
    except lib.DiscoError:
        return False
    finally:
        ctx.close()


@pytest.mark.parametrize("name", CASES)
def test_fused_equals_eight_kernels_on_the_golden_disks(name):
    g = golden(name)
    sim = lib.Sim(str(g["parfile"]))
    if not _eligible(sim):
        pytest.skip("passive scalars, outflow boundary or sink: eight-kernel substep only")
    load = [(g["step5_prim"], g["step5_tiph"], g["step5_dphi"])]
    for n in (1, 7):
        f = _advance([sim], True, n, load)[0]
        e = _advance([sim], False, n, load)[0]
        _same(f, e, (name, n))


@pytest.mark.parametrize("make", [configs.gresho, configs.kepler_ring, configs.circumbinary])
def test_fused_equals_eight_kernels_at_full_size(make):
    sim = lib.Sim(make())
    f = _advance([sim], True, 3)[0]
    e = _advance([sim], False, 3)[0]
    _same(f, e, make.__name__)


def test_fused_equals_eight_kernels_with_many_disks():
    """Four disks of the sweep (unequal q, alpha, h/r, N_r, R_out) in one
    context: the wavefront crosses disk boundaries without waiting on another
    disk."""
    sweep = configs.circumbinary_sweep(48, seed=3)
    sims = [lib.Sim(p) for p in sweep[:4]]
    f = _advance(sims, True, 3)
    e = _advance(sims, False, 3)
    for k in range(len(sims)):
        _same(f[k], e[k], k)


def test_fused_is_opt_in_and_refused_where_not_covered():
    ctx = lib.Context(lib.Sim(configs.gresho(num_r=16)))
    assert not ctx.fused and len(ctx.kernels) == 8
    ctx.set_fused(True)
    assert ctx.fused and ctx.kernels == ("prep", "sweep")
    ctx.close()
    g = golden("vortex16dye")  # passive scalar
    ctx = lib.Context(lib.Sim(str(g["parfile"])))
    assert not ctx.fused
    with pytest.raises(lib.DiscoError):
        ctx.set_fused(True)
    ctx.close()


def test_fused_timed_step_equals_graph_step():
    """The kernel-by-kernel timed step runs the same two kernels."""
    sim = lib.Sim(configs.circumbinary(num_r=64))
    a = _advance([sim], True, 2)[0]
    ctx = lib.Context(sim)
    ctx.set_fused(True)
    ctx.init_state(0)
    ms = ctx.step_timed(2)
    assert set(ms) == {"prep", "sweep"} and all(v[0] > 0 and v[1] > 0 for v in ms.values())
    st = ctx.get_state(0)
    ctx.close()
    for k in KEYS:
        assert np.array_equal(st[k], a[k]), k
