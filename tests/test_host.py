"""CPU tests of the host C layer: parfile reader, grid, initial state, guards.

The grid and the initial state must equal the reference's bit for bit
(sim_set_rz / sim_set_N_p, src/Sim/sim_set.c:10-143; cell_create's phi offsets
and the initial data, src/main.c:74-119); the fixtures hold the reference's
own values.
"""
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

from conftest import CASES, golden
from disco2_b200 import configs, lib


@pytest.mark.parametrize("name", CASES)
def test_grid_matches_reference(name):
    g = golden(name)
    sim = lib.Sim(str(g["parfile"]))
    N_p, rf = sim.grid()
    assert np.array_equal(N_p, g["N_p"])
    assert np.array_equal(rf, g["r_faces"])  # bit-exact, including the bisection remap
    assert sim.num_cells == int(g["N_p"].sum())


@pytest.mark.parametrize("name", CASES)
def test_initial_state_matches_reference(name):
    g = golden(name)
    h = lib.Sim(str(g["parfile"])).initial_state()
    for k in ("prim", "tiph", "dphi"):
        assert np.array_equal(h[k], g["init_" + k]), k
    assert np.array_equal(h["gm"][:, :4], g["init_gm"][:, :4])


def test_full_size_cell_counts():
    # the reference's N_p rule (sim_set.c:25) on the three full workloads
    assert lib.Sim(configs.gresho()).num_cells == 36075
    assert lib.Sim(configs.kepler_ring()).num_cells == 199428
    assert lib.Sim(configs.circumbinary()).num_cells == 258078


def test_parfile_reader_semantics():
    base = configs.parfile_text(configs.gresho(num_r=16))
    # first matching line wins; separators "\t :=>_" after the key are skipped
    txt = base.replace("CFL 0.4", "CFL := 0.25\nCFL 0.9")
    assert lib.Sim(txt).param("CFL") == 0.25
    # ints are truncated from the parsed double, like readvar's (int)temp
    txt = base.replace("NumR 16", "NumR 17.7")
    assert lib.Sim(txt).param("NumR") == 17
    # a key must be the first token of its line
    txt = base.replace("PLM 1.5", "//PLM 1.5\nPLM 1.25")
    assert lib.Sim(txt).param("PLM") == 1.25


def test_missing_key_is_an_error():
    base = configs.parfile_text(configs.gresho(num_r=16))
    txt = "\n".join(l for l in base.splitlines() if not l.startswith("Vel_Cap"))
    with pytest.raises(lib.DiscoError, match="Vel_Cap"):
        lib.Sim(txt)


def test_optional_initial_data_keys_default():
    p = configs.gresho(num_r=16)
    txt = "\n".join(l for l in configs.parfile_text(p).splitlines() if not l.startswith("IC_"))
    s = lib.Sim(txt)
    assert s.param("IC_HoR") == 0.05 and s.param("IC_Noise") == 0.0


@pytest.mark.parametrize("over,msg", [
    ({"NumZ": 4}, "NumZ"),
    ({"NUM_N": 4}, "NUM_N"),
    ({"NUM_N": 1, "DAMP_TIME": 1.0}, "passive scalars in a damping zone"),
    ({"w_numeric_type": 1}, "w_numeric_type"),
    ({"RiemannSolver": 7}, "RiemannSolver"),
    ({"InitialDataType": 0}, "single-cell"),
])
def test_unsupported_options_refused_before_any_device_work(over, msg):
    # dgpu_create validates the disk before touching the GPU, so this runs on CPU
    p = configs.gresho(num_r=16)
    p.update(over)
    sim = lib.Sim(p)
    with pytest.raises(lib.DiscoError, match=msg):
        lib.Context(sim)


def test_sweep_generator_is_deterministic():
    a = configs.circumbinary_sweep(48, seed=3)
    b = configs.circumbinary_sweep(48, seed=3)
    assert a == b and len(a) == 48
    qs = [d["MassRatio"] for d in a]
    assert 0.01 <= min(qs) and max(qs) <= 1.0
    assert all(128 <= d["NumR"] <= 512 for d in a)
    cells = sum(lib.Sim(d).num_cells for d in a)
    assert 3e6 < cells < 2e7


def test_missing_library_fails_loudly(tmp_path):
    # a fresh process, so no library is cached yet
    code = ("import sys; sys.path.insert(0, %r)\n"
            "from disco2_b200 import lib\n"
            "try:\n"
            "    lib.load(%r)\n"
            "except ImportError as e:\n"
            "    print('refused:', e)\n" % (os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                          str(tmp_path / "libdisco_gpu.so")))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert "refused:" in r.stdout and "missing" in r.stdout


@pytest.mark.skipif(torch.cuda.is_available(), reason="needs a host without a CUDA device")
def test_no_device_is_an_error_not_a_host_fallback():
    # a supported disk: creation reaches the device and fails there
    sim = lib.Sim(configs.gresho(num_r=16))
    with pytest.raises(lib.DiscoError, match="CUDA"):
        lib.Context(sim)


def test_three_d_initial_state_matches_the_reference():
    """A 3-D torus (torus.par reduced to 16 annuli x 8 layers): the grid, the
    phi offsets drawn ring after ring, the initial data over the layers and
    the set-up's periodic z copy into the ghost layers reproduce the
    reference's initial state bit for bit (host code, no GPU)."""
    from conftest import golden
    g = golden("torus3d16")
    sim = lib.Sim(str(g["parfile"]))
    assert sim.num_cells == g["init_prim"].shape[0]
    h = sim.initial_state()
    for k in ("prim", "tiph", "dphi"):
        assert np.array_equal(h[k], g["init_" + k]), k


@pytest.mark.parametrize("over,code", [
    ({"NumR": 0}, "PARFILE"),
    ({"NumR": -5}, "PARFILE"),
    ({"NumR": 2147483647}, "ARG"),
    ({"NumZ": 2147483647}, "ARG"),
    ({"NumR": 400000, "NumZ": 400000}, "ARG"),
    ({"ng": 100000}, "ARG"),
])
def test_impossible_grids_are_refused_quickly(over, code):
    """Grids the int cell numbering cannot hold (or nonsense sizes) are
    refused before the grid is laid out, not by an allocation failure or an
    overflow."""
    import time

    p = configs.kepler_ring(num_r=24)
    p.update(over)
    t0 = time.perf_counter()
    with pytest.raises(lib.DiscoError, match=code):
        lib.Sim(configs.parfile_text(p))
    assert time.perf_counter() - t0 < 5.0
