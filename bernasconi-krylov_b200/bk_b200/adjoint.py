"""Differentiable Trotter objective: torch.autograd.Function over ``bk_adjoint``.

The field schedule g(t) is piecewise constant over segments; the objective is
O(T) = <psi_T| W |psi_T> with W the P_< projector [E(s) < E0] (the reference's
P_<, src/sampling/sampler.cuh:149-195) or the Hamming weight popcount(s ^ s0)
(its <d_H>). The forward call runs the engine's adjoint entry point, which
returns O(T) and dO/dg_j from one forward run and one reverse sweep on the GPU;
backward only scales the stored gradient. When no gradient is needed the
forward is a plain ``bk_evolve`` with one measurement at T.

``python -m bk_b200.adjoint`` runs a schedule optimisation: N = 22, one trap
from the lowest 5% of 1000 seeded descents, 64 segments with g_j ~ U[0.25, 0.45],
dt = 0.02, 1280 steps, checkpoints every 128 steps, 20 Adam steps maximising P_<.
"""
import argparse
import json
import time

import numpy as np
import torch

from ._lib import BK_C64, BK_C128, BK_OBJ_P_LESS, Engine, select_trap


class TrotterObjective(torch.autograd.Function):
    """O(T) as a function of the per-segment field g (1-D float64 tensor)."""

    @staticmethod
    def forward(ctx, g, engine, n, s0, dt, n_steps, precision, objective, checkpoint_every, e0):
        gs = g.detach().to("cpu", torch.float64).numpy()
        if ctx.needs_input_grad[0]:
            value, grad, stats = engine.adjoint(n, s0, gs, dt, n_steps, e0=e0, precision=precision,
                                                objective=objective, checkpoint_every=checkpoint_every)
            ctx.save_for_backward(torch.from_numpy(grad).to(g.device, g.dtype))
            ctx.stats = stats
        else:
            g_steps = np.repeat(gs, n_steps // len(gs))
            p, d, _ = engine.evolve(n, s0, g_steps, dt, n_steps, measure=[n_steps], e0=e0, precision=precision)
            value = float(p[0] if objective == BK_OBJ_P_LESS else d[0])
        return torch.tensor(value, dtype=g.dtype, device=g.device)

    @staticmethod
    def backward(ctx, grad_out):
        (grad,) = ctx.saved_tensors
        return (grad_out * grad,) + (None,) * 9


class TrotterSchedule(torch.nn.Module):
    """A trainable piecewise-constant field schedule for one trap."""

    def __init__(self, engine, n, s0, g_init, dt, n_steps, precision=BK_C64, objective=BK_OBJ_P_LESS,
                 checkpoint_every=128, e0=-1):
        super().__init__()
        if n_steps % len(g_init):
            raise ValueError("n_steps must be a multiple of the number of segments")
        self.g = torch.nn.Parameter(torch.as_tensor(np.asarray(g_init, dtype=np.float64)))
        self.engine, self.n, self.s0, self.dt, self.n_steps = engine, n, s0, dt, n_steps
        self.precision, self.objective, self.checkpoint_every, self.e0 = precision, objective, checkpoint_every, e0

    def forward(self):
        return TrotterObjective.apply(self.g, self.engine, self.n, self.s0, self.dt, self.n_steps, self.precision,
                                      self.objective, self.checkpoint_every, self.e0)


def optimize(schedule, steps=20, lr=0.01, maximize=True):
    """Adam on the schedule; returns the objective before each step and after the last."""
    opt = torch.optim.Adam(schedule.parameters(), lr=lr, maximize=maximize)
    history = []
    for _ in range(steps):
        opt.zero_grad()
        value = schedule()
        value.backward()
        history.append(float(value))
        opt.step()
    with torch.no_grad():
        history.append(float(schedule()))
    return history


def main(argv=None):
    ap = argparse.ArgumentParser(description="Adam on a piecewise-constant field schedule through the adjoint")
    ap.add_argument("--n", type=int, default=22)
    ap.add_argument("--segments", type=int, default=64)
    ap.add_argument("--steps", type=int, default=1280)
    ap.add_argument("--dt", type=float, default=0.02)
    ap.add_argument("--checkpoint-every", type=int, default=128)
    ap.add_argument("--adam-steps", type=int, default=20)
    ap.add_argument("--lr", type=float, default=0.01)
    ap.add_argument("--precision", choices=["c64", "c128"], default="c64")
    ap.add_argument("--seed", type=int, default=42)
    args = ap.parse_args(argv)
    bits, e0 = select_trap(args.n, seed=args.seed, n_descents=1000, quantile=0.05)
    g0 = np.random.default_rng(args.seed).uniform(0.25, 0.45, args.segments)
    eng = Engine(0)
    sched = TrotterSchedule(eng, args.n, bits, g0, args.dt, args.steps,
                            precision=BK_C64 if args.precision == "c64" else BK_C128,
                            checkpoint_every=args.checkpoint_every, e0=e0)
    t0 = time.perf_counter()
    hist = optimize(sched, steps=args.adam_steps, lr=args.lr)
    print(json.dumps({"n": args.n, "trap": hex(bits), "e0": int(e0), "segments": args.segments,
                      "steps": args.steps, "p_less": hist, "seconds": time.perf_counter() - t0}))
    eng.close()


if __name__ == "__main__":
    main()
