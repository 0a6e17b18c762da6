"""Instance sharding across GPUs: one rank per GPU, no data-path collective.

Instances never interact (mpm_sim.py:168,274,312 index only their own
instance), so a batch is split into contiguous instance ranges balanced by
live-particle count, each rank steps its range on its own engine, and the
only exchange is one gather of the (M, 5) result rows at episode end.
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np


def contiguous_partition(weights: Sequence[float], parts: int) -> list[tuple[int, int]]:
    """Split 0..M-1 into `parts` contiguous [lo, hi) ranges of near-equal weight.

    Cut k sits at the first index whose prefix weight reaches k/parts of the
    total, kept so that every range is non-empty when M >= parts; with fewer
    instances than parts, rank k takes instance k.
    """
    w = np.asarray(weights, dtype=np.float64)
    M = len(w)
    if parts <= 0:
        raise ValueError("parts must be positive")
    if M <= parts:  # one instance per rank, the remaining ranks idle
        return [(k, k + 1) if k < M else (M, M) for k in range(parts)]
    prefix = np.concatenate([[0.0], np.cumsum(w)])
    cuts = [0]
    for k in range(1, parts):
        c = int(np.searchsorted(prefix, prefix[-1] * k / parts, side="left"))
        cuts.append(min(max(c, cuts[-1] + 1), M - (parts - k)))
    cuts.append(M)
    return [(cuts[k], cuts[k + 1]) for k in range(parts)]


def gather_rows(rows: np.ndarray, group=None) -> np.ndarray:
    """All ranks receive the concatenation of every rank's rows, in rank order.

    Ranks may hold different row counts; rows are padded to the largest count
    for the collective (NCCL needs equal shapes) and trimmed afterwards.
    """
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    backend = dist.get_backend(group)
    device = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    rows = np.ascontiguousarray(rows, dtype=np.float64)
    n = torch.tensor([rows.shape[0]], dtype=torch.int64, device=device)
    counts = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(counts, n, group=group)
    counts = [int(c.item()) for c in counts]
    width = rows.shape[1] if rows.ndim == 2 else 1
    pad = torch.zeros((max(counts), width), dtype=torch.float64, device=device)
    if rows.shape[0]:
        pad[: rows.shape[0]] = torch.from_numpy(rows.reshape(rows.shape[0], width)).to(device)
    out = [torch.zeros_like(pad) for _ in range(world)]
    dist.all_gather(out, pad, group=group)
    return np.concatenate([o[:c].cpu().numpy() for o, c in zip(out, counts)], axis=0)


def run_headless_sharded(make_engine: Callable[[int], object], inputs: Sequence, steps: int,
                         group=None) -> np.ndarray:
    """run_batch_headless over all instances, sharded across the ranks of `group`.

    `inputs[m]` = (pos, material, fiber, contraction, freq); `make_engine(n)`
    builds this rank's engine for n instances.  Returns the (M, 5) rows of the
    whole batch on every rank.
    """
    import torch.distributed as dist

    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    live = [int((np.asarray(i[1]) >= 0).sum()) for i in inputs]
    lo, hi = contiguous_partition(live, world)[rank]
    local = np.zeros((0, 5))
    if hi > lo:
        eng = make_engine(hi - lo)
        for k, m in enumerate(range(lo, hi)):
            pos, mat, fib = inputs[m][:3]
            eng.load(k, pos, mat, fib)
        eng.set_params(contraction=[inputs[m][3] for m in range(lo, hi)],
                       freq=[inputs[m][4] for m in range(lo, hi)])
        local = eng.run_headless(steps)
    return gather_rows(local, group)
