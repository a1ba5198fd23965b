"""Checkpoint and restart through the C ABI on the GPU, against the
reference's own checkpoint buffer and restart branch (tests/golden/ckpt_*.npz).

  - dgpu_checkpoint_out of the initial state equals io_setbuf's buffer bit
    for bit; after 5 steps it carries the step's parity bars (bit-exact on the
    Gresho vortex, max relative 1e-12 elsewhere, phi edges against 2 pi);
  - dgpu_checkpoint_in from the reference's 5-step buffer gives the state of
    the reference's restart (cons included), and 5 further steps match the
    reference's 5 steps after its restart;
  - checkpoint_in then checkpoint_out returns the file's rows unchanged;
  - the compiled Disco2-side binding writes checkpoints on the reference's
    cadence through dgpu_hdf5_out and restarts from input.h5 through
    dgpu_hdf5_in.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, max_rel
from disco2_b200 import lib

pytestmark = pytest.mark.gpu

CASES = ("gresho16", "kepler24", "cbd32", "torus3d16", "vortex16dye")
EXACT = {"gresho16", "vortex16dye"}  # no device transcendental reaches them
STEP_TOL = 1e-12


def ckpt(name):
    with np.load(os.path.join(GOLDEN, f"ckpt_{name}.npz")) as z:
        return {k: z[k] for k in z.files}


def close(name, got, want, key, tol=STEP_TOL):
    got, want = np.asarray(got), np.asarray(want)
    if name in EXACT:
        assert np.array_equal(got, want), key
    elif key in ("tiph", "dphi"):
        assert np.abs(got - want).max() <= tol * 2 * np.pi, key
    else:
        assert max_rel(got, want) <= tol, key


def check_rows(name, got, want, t_got, t_want, gm_got, gm_want):
    # the r and z centre columns are grid constants
    assert np.array_equal(got[:, 1:3], want[:, 1:3])
    close(name, got[:, 0], want[:, 0], "tiph")
    close(name, got[:, 3:], want[:, 3:], "prim")
    close(name, [t_got], [t_want], "t")
    close(name, gm_got, gm_want, "gm")


@pytest.mark.parametrize("name", CASES)
def test_checkpoint_out_matches_io_setbuf(name, tmp_path):
    g = ckpt(name)
    ctx = lib.Context(lib.Sim(str(g["parfile"])))
    ctx.init_state(0)
    p0 = str(tmp_path / "ck0.h5")
    ctx.checkpoint_out(p0)
    r = lib.hdf5_in(p0)
    assert r["t"] == g["ck0_t"]
    assert np.array_equal(r["gravmass"], g["ck0_gm"])
    assert np.array_equal(r["data"], g["ck0_data"])
    ctx.step(5)
    p5 = str(tmp_path / "ck5.h5")
    ctx.checkpoint_out(p5)
    r = lib.hdf5_in(p5)
    check_rows(name, r["data"], g["ck5_data"], r["t"], g["ck5_t"], r["gravmass"], g["ck5_gm"])


@pytest.mark.parametrize("name", CASES)
def test_restart_matches_the_reference_restart(name, tmp_path):
    g = ckpt(name)
    path = str(tmp_path / "input.h5")
    lib.hdf5_out(path, float(g["ck5_t"]), g["ck5_gm"], g["ck5_data"])
    ctx = lib.Context(lib.Sim(str(g["parfile"])))
    ctx.checkpoint_in(path)
    st = ctx.get_state(0)
    for k in ("prim", "tiph", "dphi"):
        assert np.array_equal(st[k], g["rs_" + k]), k
    close(name, st["cons"], g["rs_cons"], "cons")
    t, _ = ctx.time(0)
    assert t == g["rs_t"]
    assert np.array_equal(ctx.gravmass(0)[:, :4], g["rs_gm"][:, :4])
    # the identity: what was read is what is written back
    back = str(tmp_path / "back.h5")
    ctx.checkpoint_out(back)
    r = lib.hdf5_in(back)
    want = g["ck5_data"].copy()
    if lib.Sim(str(g["parfile"])).param("NumZ") == 1:
        want[:, 3 + 4] = 0.0  # io_readbuf zeroes UZZ on a 2-D disk
    assert np.array_equal(r["data"], want)
    assert r["t"] == g["ck5_t"]
    ctx.step(5)
    st = ctx.get_state(0)
    for k in ("prim", "cons", "tiph", "dphi"):
        close(name, st[k], g["rs5_" + k], k)
    t, _ = ctx.time(0)
    close(name, [t], [g["rs5_t"]], "t")
    close(name, ctx.gravmass(0)[:, :4], g["rs5_gm"][:, :4], "gm")


def test_checkpoint_in_refuses_another_grid(tmp_path):
    g = ckpt("kepler24")
    h = ckpt("cbd32")
    path = str(tmp_path / "input.h5")
    lib.hdf5_out(path, 0.0, h["ck5_gm"], h["ck5_data"])
    ctx = lib.Context(lib.Sim(str(g["parfile"])))
    ctx.init_state(0)
    before = ctx.get_state(0)["prim"]
    with pytest.raises(lib.DiscoError, match="IO"):
        ctx.checkpoint_in(path)
    assert np.array_equal(ctx.get_state(0)["prim"], before)


BINDING = os.path.join(ROOT, "oracle", "_ref", "disco_gpu_main")


@pytest.mark.skipif(not os.path.exists(BINDING), reason="binding not built (make -C oracle binding)")
def test_binding_checkpoints_and_restart(tmp_path):
    """The reference's main loop with the library: checkpoints written when t
    passes each T_MAX/Num_Checkpoints, each equal to the library's own
    checkpoint after the same number of steps; then a Restart 1 run from one
    of them continues as a library restart from the same file does."""
    import oracle
    from disco2_b200 import configs

    g = ckpt("kepler24")
    t_max = 1.6 * float(g["ck5_t"])  # about 8 steps, a checkpoint every quarter
    run_dir = tmp_path / "run"
    run_dir.mkdir()
    par = configs.write_parfile(configs.kepler_ring(num_r=24, Time_Max=t_max, Num_Checkpoints=4),
                                str(run_dir / "kepler.par"))
    res = subprocess.run([BINDING, par, "1000", str(run_dir / "final.bin")], cwd=run_dir, capture_output=True,
                         text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    written = [ln.split() for ln in res.stderr.splitlines() if ln.startswith("checkpoint ")]
    assert len(written) >= 3, res.stderr
    sim = lib.Sim(par)
    for _, fname, _, step in written:
        ctx = lib.Context(sim)
        ctx.init_state(0)
        ctx.step(int(step))
        mine = str(tmp_path / "mine.h5")
        ctx.checkpoint_out(mine)
        a, b = lib.hdf5_in(str(run_dir / fname)), lib.hdf5_in(mine)
        assert np.array_equal(a["data"], b["data"]), fname
        assert a["t"] == b["t"] and np.array_equal(a["gravmass"], b["gravmass"]), fname
    # Restart 1 from the second checkpoint, run to T_MAX
    rs_dir = tmp_path / "restart"
    rs_dir.mkdir()
    os.link(run_dir / written[1][1], rs_dir / "input.h5")
    par_rs = configs.write_parfile(configs.kepler_ring(num_r=24, Time_Max=t_max, Num_Checkpoints=4, Restart=1),
                                   str(rs_dir / "kepler.par"))
    res = subprocess.run([BINDING, par_rs, "1000", str(rs_dir / "final.bin")], cwd=rs_dir, capture_output=True,
                         text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    got = oracle.read_state(str(rs_dir / "final.bin"))
    ctx = lib.Context(lib.Sim(par_rs))
    ctx.checkpoint_in(str(rs_dir / "input.h5"))
    n = 0
    while ctx.time(0)[0] < t_max:
        ctx.step(1)
        n += 1
    assert n >= 1
    st = ctx.get_state(0)
    for k in ("prim", "tiph", "dphi"):
        assert np.array_equal(getattr(got, k), st[k]), k
    assert got.t == ctx.time(0)[0]


def test_checkpoints_of_one_disk_in_a_batch(tmp_path):
    """In a context of several disks, checkpoint_out / checkpoint_in act on the
    named disk alone: its file equals that of a context holding it alone, and
    a restart of disk 1 leaves disk 0 as it was."""
    ga, gb = ckpt("kepler24"), ckpt("cbd32")
    sa, sb = lib.Sim(str(ga["parfile"])), lib.Sim(str(gb["parfile"]))
    both = lib.Context([sa, sb])
    both.init_state(0)
    both.init_state(1)
    both.step(3)
    alone = lib.Context(sb)
    alone.init_state(0)
    alone.step(3)
    p1, p2 = str(tmp_path / "b1.h5"), str(tmp_path / "alone.h5")
    both.checkpoint_out(p1, inst=1)
    alone.checkpoint_out(p2)
    a, b = lib.hdf5_in(p1), lib.hdf5_in(p2)
    assert np.array_equal(a["data"], b["data"]) and a["t"] == b["t"]
    assert np.array_equal(a["gravmass"], b["gravmass"])
    before = both.get_state(0)
    path = str(tmp_path / "input.h5")
    lib.hdf5_out(path, float(gb["ck5_t"]), gb["ck5_gm"], gb["ck5_data"])
    both.checkpoint_in(path, inst=1)
    after = both.get_state(0)
    for k in ("prim", "cons", "tiph", "dphi"):
        assert np.array_equal(before[k], after[k]), k
    st = both.get_state(1)
    for k in ("prim", "tiph", "dphi"):
        assert np.array_equal(st[k], gb["rs_" + k]), k
