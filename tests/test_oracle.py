"""The oracle is pinned to the reference's own outputs (tests/golden).

Both halves must reproduce the golden fixtures bit for bit on the host:
  - the reference build (oracle/_ref, compiled from the unmodified reference
    sources), where it exists -- a check that the fixtures are current;
  - the C restatement (oracle/port), everywhere -- the portable oracle.
"""
import os
import tempfile

import numpy as np
import pytest

from conftest import CASE_TOL, CASES, SUB2_SLOPE_L1, SUB2_STATE, golden, golden_sub2, l1_rel, max_rel
import oracle

IMPLS = ["port"] + (["ref"] if oracle.have_ref() else [])


@pytest.fixture(scope="module", autouse=True)
def built():
    if not oracle.have_port():
        oracle.build(ref=False, port=True)
    assert oracle.have_port()


def _par(g, td):
    path = os.path.join(td, "case.par")
    with open(path, "w") as f:
        f.write(str(g["parfile"]))
    return path


@pytest.mark.parametrize("impl", IMPLS)
@pytest.mark.parametrize("name", CASES)
def test_oracle_steps_and_faces_match_reference(impl, name):
    g = golden(name)
    with tempfile.TemporaryDirectory() as td:
        par = _par(g, td)
        st0, fc, _ = oracle.run(par, 0, impl=impl, faces=True)
        for k in ("prim", "cons", "tiph", "dphi"):
            assert np.array_equal(getattr(st0, k), g["init_" + k]), k
        for k in ("nri", "L", "R", "r", "dphi", "dA", "deltaL", "deltaR", "cm"):
            assert np.array_equal(getattr(fc, k), g["init_face_" + k]), k
        for n in (5, 100):
            st, _, log = oracle.run(par, n, impl=impl, dtlog=True)
            for k in ("prim", "cons", "tiph", "dphi"):
                assert np.array_equal(getattr(st, k), g[f"step{n}_" + k]), (n, k)
            assert np.array_equal(st.gm, g[f"step{n}_gm"])
            assert np.array_equal(log, g[f"step{n}_dtlog"])


@pytest.mark.parametrize("impl", IMPLS)
@pytest.mark.parametrize("name", CASES)
def test_oracle_phases_and_layouts_match_reference(impl, name):
    g = golden(name)
    keys = {0: ("cons", "wiph", "RKcons"), 1: ("grad", "gradp"), 2: ("cons",), 3: ("cons",),
            4: ("cons",), 5: ("prim", "tiph", "dphi", "RKtiph"), 6: ("prim",), 7: ("prim", "cons")}
    with tempfile.TemporaryDirectory() as td:
        par = _par(g, td)
        st5 = oracle.run(par, 5, impl=impl)[0]
        for ph, ks in keys.items():
            st = oracle.stage(par, ph, impl=impl, load=st5)
            full = {"prim": st.prim, "cons": st.cons, "tiph": st.tiph, "dphi": st.dphi, **st.ext}
            for k in ks:
                assert np.array_equal(full[k], g[f"stage{ph}_{k}"]), (ph, k)
        st0 = oracle.run(par, 0, impl=impl)[0]
        for lay in ("rot", "aligned", "turns", "jitter"):
            if f"layout_{lay}_tiph" not in g:
                continue  # no jittered layout for annuli of fewer than 3 cells
            st0.tiph = g[f"layout_{lay}_tiph"]
            st0.dphi = g[f"layout_{lay}_dphi"]
            _, fc, _ = oracle.run(par, 0, impl=impl, load=st0, faces=True)
            for k in ("nri", "L", "R", "dphi", "dA", "cm"):
                assert np.array_equal(getattr(fc, k), g[f"layout_{lay}_face_{k}"]), (lay, k)


@pytest.mark.parametrize("name", sorted(CASE_TOL))
def test_case_tolerances_cover_last_ulp_sensitivity(name):
    """The looser bars of CASE_TOL are what last-ulp differences of libm cost
    on that case: the oracle built with one-ulp noise on every libm result of
    the step stays within them, and leaves the default bars (1e-12 per step,
    1e-10 L1 after 100 steps)."""
    oracle.build_port_ulp()
    step_tol, l1_tol = CASE_TOL[name]
    g = golden(name)
    with tempfile.TemporaryDirectory() as td:
        par = _par(g, td)
        worst = 0.0
        for n in (1, 5):
            st = oracle.run(par, n, impl="port_ulp")[0]
            worst = max(worst, max_rel(st.prim, g[f"step{n}_prim"]), max_rel(st.cons, g[f"step{n}_cons"]))
        st = oracle.run(par, 100, impl="port_ulp")[0]
        l1 = max(l1_rel(st.cons[:, q], g["step100_cons"][:, q]) for q in (0, 1, 2, 3))
    assert 1e-12 < worst <= step_tol
    assert 1e-10 < l1 <= l1_tol


@pytest.mark.parametrize("impl", IMPLS)
@pytest.mark.parametrize("name", CASES)
def test_oracle_second_substep_phases_match_reference(impl, name):
    """Phases 8-15: the whole first substep and gravMass_move, then the second
    substep stopped after each phase."""
    g = golden_sub2(name)
    with tempfile.TemporaryDirectory() as td:
        par = _par(g, td)
        st5 = oracle.run(par, 5, impl=impl)[0]
        for ph in range(8, 16):
            st = oracle.stage(par, ph, impl=impl, load=st5)
            full = {"prim": st.prim, "cons": st.cons, "tiph": st.tiph, "dphi": st.dphi, **st.ext}
            for k in [k for k in g if k.startswith(f"stage{ph}_")]:
                key = k.split("_", 1)[1]
                if key in ("dt", "gm"):
                    want = g[k]
                    got = np.float64(st.dt) if key == "dt" else st.gm
                    assert np.array_equal(got, want), (ph, key)
                else:
                    assert np.array_equal(full[key], g[k]), (ph, key)


@pytest.mark.parametrize("name", sorted(set(SUB2_SLOPE_L1) | set(SUB2_STATE)))
def test_second_substep_bars_cover_last_ulp_sensitivity(name):
    """The looser second-substep bars are inside what last-ulp differences of
    libm cost the reference's own arithmetic: the one-ulp-noise build moves
    the case's slopes (L1) or state (max relative) beyond the bar used for
    the GPU."""
    oracle.build_port_ulp()
    g, g2 = golden(name), golden_sub2(name)
    with tempfile.TemporaryDirectory() as td:
        par = _par(g, td)
        st5 = oracle.run(par, 5, impl=IMPLS[0])[0]
        if name in SUB2_SLOPE_L1:
            st = oracle.stage(par, 9, impl="port_ulp", load=st5)
            l1 = max(l1_rel(st.ext[k].ravel(), g2[f"stage9_{k}"].ravel()) for k in ("grad", "gradp"))
            assert l1 > SUB2_SLOPE_L1[name], l1
        if name in SUB2_STATE:
            st = oracle.stage(par, 13, impl="port_ulp", load=st5)
            assert max_rel(st.prim, g2["stage13_prim"]) > 0.5 * SUB2_STATE[name]
