"""The launch-shape autotuner: every choice gives bitwise the same step, and
tuning leaves the state where it found it."""
from __future__ import annotations

import numpy as np
import pytest

from disco2_b200 import configs, lib

pytestmark = pytest.mark.gpu


def _run(choice=None, tune_steps=0, nsteps=4, fused=False):
    s = lib.Sim(configs.circumbinary(num_r=64))
    ctx = lib.Context(s)
    ctx.set_fused(fused)
    ctx.init_state(0)
    chosen = None
    if choice is not None:
        chosen = ctx.autotune(0, choice)
    if tune_steps:
        before = ctx.get_state(0)
        t0 = ctx.time(0)
        chosen = ctx.autotune(tune_steps)
        after = ctx.get_state(0)
        assert ctx.time(0) == t0
        for k in ("prim", "cons", "tiph", "dphi"):
            assert np.array_equal(before[k], after[k]), k
    ctx.step(nsteps)
    st = ctx.get_state(0)
    ctx.close()
    return st, chosen


def test_every_launch_shape_gives_the_same_step():
    ref, _ = _run()
    for choice in ([2, 2, 2, 2, 2, 0], [5, 5, 5, 5, 5, 0], [3, 4, 5, 2, 3, 0]):
        st, got = _run(choice=choice)
        assert list(got.values()) == choice
        for k in ("prim", "cons", "tiph", "dphi"):
            assert np.array_equal(st[k], ref[k]), (choice, k)


def test_every_sweep_shape_gives_the_same_step():
    """The fused substep under each register budget of k_sweep equals the
    eight-kernel step bit for bit."""
    ref, _ = _run()
    for sw in (2, 3, 4):
        st, got = _run(choice=[0, 0, 0, 0, 0, sw], fused=True)
        assert got["sweep"] == sw
        for k in ("prim", "cons", "tiph", "dphi"):
            assert np.array_equal(st[k], ref[k]), (sw, k)


@pytest.mark.parametrize("fused", [False, True])
def test_autotune_restores_state_and_picks_valid_shapes(fused):
    ref, _ = _run()
    st, chosen = _run(tune_steps=2, fused=fused)
    assert all(v in (0, 2, 3, 4, 5) for v in chosen.values()), chosen
    if fused:
        assert chosen["sweep"] in (2, 3, 4), chosen
    for k in ("prim", "cons", "tiph", "dphi"):
        assert np.array_equal(st[k], ref[k]), k


def test_autotune_rejects_bad_choice():
    s = lib.Sim(configs.circumbinary(num_r=64))
    ctx = lib.Context(s)
    with pytest.raises(lib.DiscoError):
        ctx.autotune(0, [1, 0, 0, 0, 0, 0])
    ctx.close()
