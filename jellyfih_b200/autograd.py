"""torch.autograd front end of the differentiable rollout.

`rollout_displacement(engine, actuation, contraction, freq, positions, ...)`
loads every instance from `positions`, runs `steps` substeps with checkpoints
(jf_grad_forward) and returns the (M,) payload CoM displacement as a tensor;
its backward calls the hand-written adjoint kernels (jf_grad_backward,
jf_grad_positions).  The engine keeps the checkpoints of its latest rollout
only, so a rollout's backward runs before the next rollout on the same engine
(grad_forward, grad_step or another forward here); a later backward raises
RuntimeError instead of differentiating the wrong rollout.
`refine_timing_genes` takes gradient steps on the two
actuation-timing genes (contraction fraction, frequency multiplier) beside
CMA-ES, as an optional refinement, each step's forward and backward replayed
as one CUDA graph (jf_grad_step).
"""
from __future__ import annotations

import numpy as np
import torch

from .tank import GENOME_LOWER, GENOME_UPPER


class RolloutDisplacement(torch.autograd.Function):
    @staticmethod
    def forward(ctx, actuation, contraction, freq, positions, engine, materials, fibers, steps,
                checkpoint_every, t0):
        M = engine.M
        engine.set_params(actuation=actuation.detach().cpu().numpy(),
                          contraction=contraction.detach().cpu().numpy(),
                          freq=freq.detach().cpu().numpy())
        pos = positions.detach().to("cpu", torch.float32).numpy()
        for m in range(M):
            engine.load(m, pos[m], materials[m], fibers[m])
        engine.time = t0
        loss = engine.grad_forward(int(steps), int(checkpoint_every))
        ctx.engine = engine
        ctx.rollout = engine.rollouts
        ctx.shape = positions.shape
        ctx.device = positions.device
        return torch.from_numpy(loss).to(actuation.device)

    @staticmethod
    def backward(ctx, gout):
        e = ctx.engine
        if e.rollouts != ctx.rollout:
            # the engine keeps the checkpoints of its latest rollout only
            raise RuntimeError("the engine ran another differentiable rollout after this one's forward; "
                               "run the backward of a rollout before the next forward on the same engine")
        g = e.grad_backward()
        go = gout.detach().to("cpu", torch.float64).numpy()
        gx = np.stack([e.grad_positions(m) for m in range(e.M)]).astype(np.float64)
        gx *= go[:, None, None]
        dev = gout.device

        def t(a):
            return torch.from_numpy(np.asarray(a) * go).to(dev)

        return (t(g["actuation"]), t(g["contraction"]), t(g["freq"]),
                torch.from_numpy(gx).to(ctx.device, torch.float32).reshape(ctx.shape),
                None, None, None, None, None, None)


def rollout_displacement(engine, actuation, contraction, freq, positions, materials, fibers, steps,
                         checkpoint_every=100, t0=0.0):
    """Differentiable (M,) payload displacement after `steps` substeps."""
    return RolloutDisplacement.apply(actuation, contraction, freq, positions, engine, materials, fibers,
                                     steps, checkpoint_every, t0)


def refine_timing_genes(engine, genomes, positions, materials, fibers, steps, iterations=3,
                        step_frac=0.05, actuation=500.0, checkpoint_every=100):
    """Gradient steps on genes 9 (contraction) and 10 (frequency multiplier).

    Each iteration loads every instance's initial particles, runs the
    checkpointed forward and the backward of all instances as one CUDA graph
    (Engine.grad_step; the graph is captured on the first iteration and
    replayed after), and moves each gene by step_frac of its range in the
    direction that raises the payload's displacement, clipped to the gene
    bounds (evolve.py:55-62).  An instance whose rollout or adjoint went
    non-finite (the engine's error flags) keeps its genes for that iteration.
    Returns the refined genomes and the displacement before every step.
    """
    g = np.array(genomes, dtype=np.float64, copy=True)
    M = len(g)
    history = []
    for _ in range(iterations):
        engine.clear_error_flags()
        c = np.clip(g[:, 9], 0.05, 0.60)
        f = np.clip(g[:, 10], 0.5, 2.0)
        engine.set_params(actuation=np.full(M, actuation, np.float32), contraction=c.astype(np.float32),
                          freq=f.astype(np.float32))
        for m in range(M):
            engine.load(m, positions[m], materials[m], fibers[m])
        engine.time = 0.0
        disp, grads = engine.grad_step(int(steps), int(checkpoint_every))
        history.append(disp.copy())
        ok = engine.error_flags() == 0
        for k, name in ((9, "contraction"), (10, "freq")):
            span = GENOME_UPPER[k] - GENOME_LOWER[k]
            step = np.where(ok, step_frac * span * np.sign(np.nan_to_num(grads[name])), 0.0)
            g[:, k] = np.clip(g[:, k] + step, GENOME_LOWER[k], GENOME_UPPER[k])
    return g, history
