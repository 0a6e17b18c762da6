"""Autotuner of the batched path: picks the threads per CTA, the cell cap, the
cluster size and the re-sort interval by timing short trials on the caller's
own batch.

Candidates are the kernel layouts (threads per CTA: fewer warps per SM leave
more registers and L1 per warp but hide less latency; the cell cap chosen by
the sort's cost model at every re-sort, or fixed), the cluster sizes whose
shared-memory window fits (CTAs per instance: more CTAs give each instance
more SMs but more halo rows) and the re-sort intervals (longer intervals
amortise the counting sort; particles that drift out of their cell's register
block fall back to per-particle atomics).  Each trial loads the same particle
sets, runs a warm-up chunk, then times `trial_steps` substeps with CUDA events
around every chunk and re-sort launch.
"""
from __future__ import annotations

import itertools

from .engine import Engine
from ._lib import JfError

# (block_threads, cell_cap); cell_cap 0 = chosen by the cost model at every re-sort.
# 768 threads keep the cell lanes' node blocks in TMEM (24 warps per SM), 512
# in registers (16 warps per SM)
LAYOUTS = ((768, 0), (512, 0), (768, 4))


def autotune(specs, inputs, clusters=(0, 4, 8, 16), resorts=(16, 32, 64, 128), trial_steps=256,
             device=0, params=None, layouts=LAYOUTS):
    """Returns (best config dict, list of trial results).

    `inputs[m]` = (pos, material, fiber); `params` = kwargs of Engine.set_params.
    The best config holds the Engine keyword arguments cluster_size,
    resort_interval, block_threads and cell_cap.  Each trial
    result: that config plus ms_per_substep and atomic_scatter_fraction, or an
    "error" entry for configurations the device cannot run (shared memory,
    cluster scheduling).
    """
    results = []
    for (threads, cap), cs, ri in itertools.product(layouts, clusters, resorts):
        cfg = {"cluster_size": cs, "resort_interval": ri, "block_threads": threads, "cell_cap": cap}
        try:
            e = Engine(list(specs), path="batched", device=device, **cfg)
        except JfError as err:
            results.append(dict(cfg, error=str(err)))
            continue
        try:
            for m, (pos, mat, fib) in enumerate(inputs):
                e.load(m, pos, mat, fib)
            if params:
                e.set_params(**params)
            e.step(ri)
            e.sync()
            e.set_kernel_timing(True)
            e.path_counts(reset=True)
            steps = max(ri, (trial_steps // ri) * ri)
            e.step(steps)
            kt = e.kernel_timing()
            pc = e.path_counts()
            total = pc["register_scatters"] + pc["atomic_scatters"]
            results.append(dict(cfg, ms_per_substep=(kt["step_ms"] + kt["sort_ms"]) / steps,
                                atomic_scatter_fraction=pc["atomic_scatters"] / max(total, 1)))
        except JfError as err:
            results.append(dict(cfg, error=str(err)))
        finally:
            e.close()
    ok = [r for r in results if "ms_per_substep" in r]
    if not ok:
        raise RuntimeError("no batched configuration could run on this device")
    best = min(ok, key=lambda r: r["ms_per_substep"])
    return {k: best[k] for k in ("cluster_size", "resort_interval", "block_threads", "cell_cap")}, results
