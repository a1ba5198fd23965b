"""Differentiation of the step on the GPU: objective, tangent and adjoint.

The tangent (Dual instances of the forward kernels) must reproduce the
forward trajectory bit for bit and agree with central finite differences of
the GPU forward; the adjoint must be the transpose of the tangent (the
dot-product test <grad J, v> = dJ/de along v, to round-off) for q, alpha and
random directions in the initial prims, whatever the checkpoint spacing.
The derivatives hold the dt schedule fixed, so the finite differences replay
the unperturbed run's dt schedule (dgpu_objective with dt_in)."""
from __future__ import annotations

import numpy as np
import pytest

from disco2_b200 import configs, lib

pytestmark = pytest.mark.gpu

NSTEPS, W0 = 40, 20
Q0, ALPHA0 = 0.5, 0.1  # q = 1 is the symmetric point, where dJ/dq is round-off small


def _cbd(q=Q0, alpha=ALPHA0):
    return configs.circumbinary(num_r=64, q=q, alpha=alpha)


@pytest.fixture(scope="module")
def base():
    s = lib.Sim(_cbd())
    ctx = lib.Context(s)
    ctx.init_state(0)
    st = ctx.get_state(0)
    J, dt = ctx.objective(NSTEPS, W0, return_dt=True)
    ctx.close()
    return {"prim": st["prim"], "tiph": st["tiph"], "dphi": st["dphi"], "N": s.num_cells, "dt": dt, "J": J}


def _ctx(base, q=Q0, alpha=ALPHA0, prim=None):
    ctx = lib.Context(lib.Sim(_cbd(q, alpha)))
    ctx.init_state(0)  # binary of this q
    ctx.set_state(0, base["prim"] if prim is None else prim, base["tiph"], base["dphi"])
    return ctx


def _J(base, **kw):
    """J with the unperturbed run's dt schedule."""
    ctx = _ctx(base, **kw)
    J = ctx.objective(NSTEPS, W0, dt=base["dt"])
    ctx.close()
    return J


def _direction(base, seed):
    """A relative perturbation of the surface density with the pressure
    following it (P/rho fixed): d rho = rho u, d P = P u, u ~ N(0, 1)."""
    u = np.random.default_rng(seed).standard_normal(base["N"])
    d = np.zeros((base["N"], 5))
    d[:, 0] = base["prim"][:, 0] * u
    d[:, 1] = base["prim"][:, 1] * u
    return d


def test_tangent_reproduces_forward(base):
    ctx = _ctx(base)
    J, dJ = ctx.tangent(NSTEPS, W0, dq=1.0)
    st_t = ctx.get_state(0)
    ctx.close()
    ctx = _ctx(base)
    J0 = ctx.objective(NSTEPS, W0)
    st_f = ctx.get_state(0)
    ctx.close()
    assert np.array_equal(J, J0)
    assert np.array_equal(st_t["prim"], st_f["prim"])
    # the frozen-dt forward with the run's own schedule is the same run
    assert np.array_equal(_J(base), J0)
    assert np.all(np.isfinite(dJ)) and np.any(dJ != 0.0)


@pytest.mark.parametrize("which", ["q", "alpha", "sigma"])
def test_tangent_matches_finite_differences(base, which):
    """Central differences of the frozen-dt GPU forward.  The accretion rate
    uses a relative step of 1e-8: small enough that no limiter or Riemann-state
    branch flips between the two runs (at 1e-6 some do, and its differences
    then move by up to ~1e-2), large enough that round-off stays below ~1e-7 of
    the derivative.  The torque is a sum with strong cancellation whose
    round-off grows as 1/h, so it takes the best of the steps 1e-5..1e-7."""
    v = _direction(base, 3)

    def fd(h):
        if which == "q":
            return (_J(base, q=Q0 * (1 + h)) - _J(base, q=Q0 * (1 - h))) / (2 * Q0 * h)
        if which == "alpha":
            return (_J(base, alpha=ALPHA0 * (1 + h)) - _J(base, alpha=ALPHA0 * (1 - h))) / (2 * ALPHA0 * h)
        return (_J(base, prim=base["prim"] + h * v) - _J(base, prim=base["prim"] - h * v)) / (2 * h)

    ctx = _ctx(base)
    if which == "q":
        _, dJ = ctx.tangent(NSTEPS, W0, dq=1.0)
    elif which == "alpha":
        _, dJ = ctx.tangent(NSTEPS, W0, dalpha=1.0)
    else:
        _, dJ = ctx.tangent(NSTEPS, W0, dprim=v)
    ctx.close()
    f8 = fd(1e-8)
    rel_m = abs(dJ[1] - f8[1]) / abs(f8[1])
    rel_t = min(abs(dJ[0] - f[0]) / abs(f[0]) for f in (fd(1e-5), fd(1e-6), fd(1e-7)))
    print(which, dJ, f8, rel_m, rel_t)
    assert rel_m < 1e-6, (which, dJ, f8, rel_m)   # accretion rate
    assert rel_t < 1e-4, (which, dJ, rel_t)       # torque


@pytest.mark.parametrize("weights", [(1.0, 0.0), (0.0, 1.0)])
def test_adjoint_is_transpose_of_tangent(base, weights):
    w = np.array(weights)
    ctx = _ctx(base)
    g = ctx.adjoint(NSTEPS, W0, ckpt_every=7, weights=weights)
    ctx.close()
    checks = []
    ctx = _ctx(base)
    _, dJ = ctx.tangent(NSTEPS, W0, dq=1.0)
    ctx.close()
    checks.append((g["dq"], w @ dJ))
    ctx = _ctx(base)
    _, dJ = ctx.tangent(NSTEPS, W0, dalpha=1.0)
    ctx.close()
    checks.append((g["dalpha"], w @ dJ))
    for seed in (1, 2):
        v = _direction(base, seed)
        ctx = _ctx(base)
        _, dJ = ctx.tangent(NSTEPS, W0, dprim=v)
        ctx.close()
        checks.append((float(np.sum(g["dprim"] * v)), w @ dJ))
    # a direction in every prim, ghost annuli included
    v = np.random.default_rng(5).standard_normal((base["N"], 5)) * 1e-2
    ctx = _ctx(base)
    _, dJ = ctx.tangent(NSTEPS, W0, dprim=v)
    ctx.close()
    checks.append((float(np.sum(g["dprim"] * v)), w @ dJ))
    for a, t in checks:
        assert abs(a - t) <= 1e-9 * max(abs(t), 1e-300), checks


def test_adjoint_independent_of_checkpoint_spacing(base):
    out = []
    for K in (1, 6, NSTEPS):
        ctx = _ctx(base)
        g = ctx.adjoint(NSTEPS, W0, ckpt_every=K)
        st = ctx.get_state(0)
        ctx.close()
        out.append((g, st))
    for g, st in out[1:]:
        assert g["dq"] == out[0][0]["dq"] and g["dalpha"] == out[0][0]["dalpha"]
        assert np.array_equal(g["dprim"], out[0][0]["dprim"])
        assert np.array_equal(st["prim"], out[0][1]["prim"])


@pytest.mark.parametrize("par,msg", [
    (configs.gresho(num_r=16), "C_RIGID"),
    (configs.kepler_ring(num_r=16, BoundTypeR=1), "outflow"),
    (configs.kepler_ring(num_r=16, NUM_N=1), "passive"),
])
def test_differentiation_refuses_unsupported(par, msg):
    s = lib.Sim(par)
    ctx = lib.Context(s)
    ctx.init_state(0)
    with pytest.raises(lib.DiscoError, match=msg):
        ctx.objective(4, 2)
    ctx.close()


def test_gradient_matches_reference_finite_differences():
    """The adjoint gradient of the circumbinary disk at 192 annuli over 500
    steps (objectives averaged over steps 251-500, checkpoints every 25 steps)
    against central finite differences of the reference C code with the same
    frozen dt schedule (tests/golden/cbd192_fd.json, made by
    tests/golden/make_fd_reference.py): q, alpha and 16 seeded directions of
    the initial surface density."""
    import json
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "cbd192_fd.json")
    ref = json.load(open(path))
    s = lib.Sim(configs.circumbinary(num_r=ref["num_r"]))
    assert s.num_cells == ref["cells"]
    grads = []
    for w in ((1.0, 0.0), (0.0, 1.0)):
        ctx = lib.Context(s)
        ctx.init_state(0)
        prim0 = ctx.get_state(0)["prim"]
        grads.append(ctx.adjoint(ref["nsteps"], ref["window_start"], ckpt_every=25, weights=w))
        ctx.close()
    assert np.allclose([grads[0]["J"][0], grads[1]["J"][1]], ref["J"], rtol=1e-8, atol=0)
    rows = []
    for k in range(2):
        g = grads[k]
        vals = [("q", g["dq"]), ("alpha", g["dalpha"])]
        for d in range(len(ref["fd"]["1e-08"]["sigma"])):
            u = np.random.default_rng(1000 + d).standard_normal(prim0.shape[0])
            dirv = np.zeros_like(prim0)
            dirv[:, 0] = prim0[:, 0] * u
            dirv[:, 1] = prim0[:, 1] * u
            vals.append((f"sigma{d}", float(np.sum(g["dprim"] * dirv))))
        for name, a in vals:
            f8 = ref["fd"]["1e-08"][name][k] if not name.startswith("sigma") else \
                ref["fd"]["1e-08"]["sigma"][int(name[5:])][k]
            f6 = ref["fd"]["1e-06"][name][k] if not name.startswith("sigma") else \
                ref["fd"]["1e-06"]["sigma"][int(name[5:])][k]
            rows.append((name, k, a, f8, abs(a - f8) / abs(f8), abs(a - f6) / abs(f6)))
    for name, k, a, f8, r8, r6 in rows:
        print(f"{name:8s} {'torque' if k == 0 else 'mdot':6s} adjoint={a:+.9e} reference_fd(1e-8)={f8:+.9e} "
              f"rel={r8:.2e}   rel vs step 1e-6: {r6:.2e}")
    r8 = np.array([r[4] for r in rows])
    # 500 steps of limiter and Riemann-state switching: the central differences
    # carry kink and round-off errors of up to a few 1e-4 (see the 1e-6 column)
    assert np.median(r8) < 5e-5, np.median(r8)
    assert np.max(r8) < 1e-3, np.max(r8)


def test_gradient_against_reference_differences_over_step_sizes():
    """The adjoint against the reference's central differences at three step
    sizes (tests/golden/cbd192_fd_short.json: the gradient-check disk without
    its 1e-4 initial noise, 20 steps, objectives averaged over steps 11-20,
    relative steps 1e-6, 1e-7, 1e-8, frozen dt).

    - alpha, accretion rate: the differences converge (they agree to 1e-7),
      and the adjoint agrees with them to 1e-6 relative.
    - the mass ratio q (both objectives) and every torque entry: the torque
      is a cancelling sum whose differences move by 1e-4 to 1e-1 between the
      step sizes (limiter and Riemann-state branches flip inside the step);
      the adjoint lies within twice that spread of the differences.
    - the Sigma_0 directions of the accretion rate are printed, not asserted:
      without noise the initial disk is exactly axisymmetric, so every phi
      limiter of the first substep is evaluated at its kink (all slopes 0).
      The differences converge there to the directional derivative, which the
      branch-replaying adjoint does not give at a kink (it differentiates the
      branch that the forward took)."""
    import json
    import os
    ref = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "cbd192_fd_short.json")))
    s = lib.Sim(configs.circumbinary(num_r=ref["num_r"], **ref["params"]))
    assert s.num_cells == ref["cells"]
    grads = []
    for w in ((1.0, 0.0), (0.0, 1.0)):
        ctx = lib.Context(s)
        ctx.init_state(0)
        prim0 = ctx.get_state(0)["prim"]
        grads.append(ctx.adjoint(ref["nsteps"], ref["window_start"], ckpt_every=5, weights=w))
        ctx.close()
    assert np.allclose([grads[0]["J"][0], grads[1]["J"][1]], ref["J"], rtol=1e-8, atol=0)
    fd = ref["fd"]
    steps = ("1e-06", "1e-07", "1e-08")
    for k in range(2):
        g = grads[k]
        vals = [("q", g["dq"]), ("alpha", g["dalpha"])]
        for d in range(len(fd["1e-07"]["sigma"])):
            u = np.random.default_rng(1000 + d).standard_normal(prim0.shape[0])
            dirv = np.zeros_like(prim0)
            dirv[:, 0] = prim0[:, 0] * u
            dirv[:, 1] = prim0[:, 1] * u
            vals.append((f"sigma{d}", float(np.sum(g["dprim"] * dirv))))
        for name, a in vals:
            f = np.array([fd[h]["sigma"][int(name[5:])][k] if name.startswith("sigma") else fd[h][name][k]
                          for h in steps])
            spread = (f.max() - f.min()) / abs(f[-1])
            rel = np.abs(a - f) / np.abs(f)
            print(f"{name:8s} {'torque' if k == 0 else 'mdot':6s} adjoint={a:+.10e} "
                  f"reference_fd={' '.join(f'{x:+.10e}' for x in f)} rel={' '.join(f'{x:.1e}' for x in rel)} "
                  f"fd spread={spread:.1e}")
            if name == "alpha" and k == 1:
                assert spread <= 1e-6 and rel.max() <= 1e-6, (rel, spread)
            elif k == 0 or name == "q":
                assert np.abs(a - f).max() <= 2.0 * (f.max() - f.min()) + 1e-6 * abs(f[-1]), (name, k, rel, spread)


def test_autograd_wrapper_matches_adjoint(base):
    """The torch.autograd.Function of the check harness: backward of a scalar
    function of J is one dgpu_adjoint call with the incoming weights."""
    import torch
    from disco2_b200.autograd import DiskRun
    prim0 = torch.tensor(base["prim"], requires_grad=True)
    q = torch.tensor(Q0, dtype=torch.float64, requires_grad=True)
    a = torch.tensor(ALPHA0, dtype=torch.float64, requires_grad=True)
    J = DiskRun.apply(prim0, q, a, _cbd(), NSTEPS, W0)
    assert np.array_equal(J.detach().numpy(), base["J"])
    (J[0] + 2.0 * J[1]).backward()
    ctx = _ctx(base)
    g = ctx.adjoint(NSTEPS, W0, ckpt_every=25, weights=(1.0, 2.0))
    ctx.close()
    assert q.grad.item() == g["dq"] and a.grad.item() == g["dalpha"]
    assert np.array_equal(prim0.grad.numpy(), g["dprim"])
