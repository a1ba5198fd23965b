"""torch.autograd wrapper of the differentiated run (for the gradient checks).

    J = DiskRun.apply(prim0, q, alpha, params, nsteps, window_start)

prim0 is a float64 tensor [N, 5] (the initial prims in the disk's (k, i, j)
order), q and alpha are float64 scalar tensors, params the workload dict of
disco2_b200.configs (its MassRatio and Explicit_Viscosity are replaced by q
and alpha).  J = (mean torque, mean accretion rate) over steps
window_start+1 .. nsteps.  The forward runs dgpu_objective; the backward runs
dgpu_adjoint with the incoming gradient as the objective weights, so the
gradient of any scalar function of J comes from one reverse sweep.  All the
arithmetic is in the library's CUDA kernels; torch only carries the tensors.
"""
from __future__ import annotations

import numpy as np
import torch

from . import lib

CKPT_EVERY = 25


def _context(params: dict, q: float, alpha: float, prim0: np.ndarray):
    p = dict(params)
    p["MassRatio"] = q
    p["Explicit_Viscosity"] = alpha
    sim = lib.Sim(p)
    ctx = lib.Context(sim)
    ctx.init_state(0)  # mesh, phi edges and the binary of this q
    st = ctx.get_state(0)
    ctx.set_state(0, prim0, st["tiph"], st["dphi"])
    return ctx


class DiskRun(torch.autograd.Function):
    @staticmethod
    def forward(fctx, prim0, q, alpha, params, nsteps, window_start):
        p0 = prim0.detach().cpu().numpy().astype(np.float64)
        qv, av = float(q), float(alpha)
        ctx = _context(params, qv, av, p0)
        J = ctx.objective(nsteps, window_start)
        ctx.close()
        fctx.save_for_backward(prim0)
        fctx.args = (params, qv, av, nsteps, window_start)
        fctx.devs = (getattr(q, "device", torch.device("cpu")), getattr(alpha, "device", torch.device("cpu")))
        return torch.as_tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(fctx, gJ):
        (prim0,) = fctx.saved_tensors
        params, qv, av, nsteps, window_start = fctx.args
        ctx = _context(params, qv, av, prim0.detach().cpu().numpy().astype(np.float64))
        g = ctx.adjoint(nsteps, window_start, ckpt_every=CKPT_EVERY,
                        weights=gJ.detach().cpu().numpy().astype(np.float64))
        ctx.close()
        dev_q, dev_a = fctx.devs
        return (torch.as_tensor(g["dprim"], dtype=torch.float64).to(prim0.device),
                torch.tensor(g["dq"], dtype=torch.float64, device=dev_q),
                torch.tensor(g["dalpha"], dtype=torch.float64, device=dev_a),
                None, None, None)
