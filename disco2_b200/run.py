"""Run a named workload for a few RK2 steps on cuda:0.

    python -m disco2_b200.run --workload circumbinary --steps 3 [--timed] [--batch N] [--fused]
    python -m disco2_b200.run --workload circumbinary --num-r 192 --steps 0 --adjoint 10 --ckpt 5
    python -m disco2_b200.run --workload kepler_ring --steps 10 --checkpoint-out ck.h5
    python -m disco2_b200.run --workload kepler_ring --restart ck.h5 --steps 10

Used for profiling (ncu attaches to this process) and as a minimal example of
the C ABI from Python.  --timed adds one step launched kernel by kernel
with CUDA events and prints the per-kernel device times.  --batch N steps N
copies of the disk in one context.  --adjoint N then runs the gradient of an
N-step run (objectives over its second half, checkpoints every --ckpt steps).
--fused steps with the fused substep (k_prep + k_sweep) instead of the eight kernels.
--restart FILE starts disk 0 from a checkpoint file (the reference's restart
set-up) instead of the initial data; --checkpoint-out FILE writes disk 0 as a
checkpoint file after the steps.
"""
from __future__ import annotations

import argparse

from . import configs, lib

WORKLOADS = configs.WORKLOADS


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="circumbinary", choices=sorted(WORKLOADS))
    ap.add_argument("--num-r", type=int, default=None)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--timed", action="store_true")
    ap.add_argument("--batch", type=int, default=1)
    ap.add_argument("--adjoint", type=int, default=0)
    ap.add_argument("--ckpt", type=int, default=25)
    ap.add_argument("--fused", action="store_true")
    ap.add_argument("--restart", default=None)
    ap.add_argument("--checkpoint-out", default=None)
    args = ap.parse_args()
    p = WORKLOADS[args.workload]() if args.num_r is None else WORKLOADS[args.workload](num_r=args.num_r)
    sims = [lib.Sim(p) for _ in range(args.batch)]
    ctx = lib.Context(sims)
    if args.fused:
        ctx.set_fused(True)
    for k in range(args.batch):
        ctx.init_state(k)
    if args.restart:
        ctx.checkpoint_in(args.restart, 0)
    if args.steps:
        ctx.step(args.steps)
    if args.adjoint:
        g = ctx.adjoint(args.adjoint, args.adjoint // 2, ckpt_every=args.ckpt)
        print(f"adjoint: J={g['J']} dJ/dq={g['dq']:.9e} dJ/dalpha={g['dalpha']:.9e}")
    if args.timed:
        ms = ctx.step_timed(1)
        print(" ".join(f"{n}{s + 1}={v[s]:.4f}ms" for s in (0, 1) for n, v in ms.items()))
    if args.checkpoint_out:
        ctx.checkpoint_out(args.checkpoint_out, 0)
    t, dt = ctx.time(0)
    print(f"{args.workload}: {sims[0].num_cells} cells x {args.batch}, t={t:.6g} dt={dt:.6g}")
    ctx.close()


if __name__ == "__main__":
    main()
