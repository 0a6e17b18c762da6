"""The batched path's autotuner (jellyfih_b200/autotune.py) on the CPU with a
stand-in engine: every (layout, cluster size, re-sort interval) candidate is
tried once on the caller's particles, configurations the device rejects are
recorded as errors and skipped, the fastest trial (step and re-sort time per
substep) wins, and no runnable configuration at all is an error.
"""
import pytest

from jellyfih_b200 import autotune
from jellyfih_b200._lib import JfError


class StandInEngine:
    """Times a trial from its configuration; rejects cluster size 16."""
    made = []

    def __init__(self, specs, path, device, cluster_size, resort_interval, block_threads, cell_cap):
        if cluster_size == 16:
            raise JfError(4, "cluster of 16 does not fit")
        self.cfg = dict(cluster_size=cluster_size, resort_interval=resort_interval,
                        block_threads=block_threads, cell_cap=cell_cap)
        self.loaded, self.params, self.substeps, self.closed = 0, None, 0, False
        StandInEngine.made.append(self)

    def load(self, m, pos, mat, fib):
        self.loaded += 1

    def set_params(self, **kw):
        self.params = kw

    def step(self, n):
        self.substeps += n

    def sync(self):
        pass

    def set_kernel_timing(self, on):
        self.timed_from = self.substeps

    def path_counts(self, reset=False):
        return {"register_scatters": 90, "atomic_scatters": 10, "remote_gathers": 0, "overflow_scatters": 0}

    def kernel_timing(self):
        c = self.cfg
        per = 1.0 + (0.1 if c["block_threads"] == 512 else 0.0) + abs(c["resort_interval"] - 32) / 1000
        per += 0.05 * (c["cluster_size"] != 4) + 0.02 * (c["cell_cap"] != 0)
        n = self.substeps - self.timed_from
        return {"step_ms": 0.9 * per * n, "sort_ms": 0.1 * per * n, "step_launches": 1, "sort_launches": 1}

    def close(self):
        self.closed = True


def test_fastest_configuration_wins_and_rejected_ones_are_recorded(monkeypatch):
    monkeypatch.setattr(autotune, "Engine", StandInEngine)
    StandInEngine.made = []
    inputs = [("pos", "mat", "fib")] * 3
    best, trials = autotune.autotune(["spec"] * 3, inputs, clusters=(4, 8, 16), resorts=(16, 32, 64),
                                     trial_steps=64, params={"actuation": [500.0] * 3})
    assert best == {"cluster_size": 4, "resort_interval": 32, "block_threads": 768, "cell_cap": 0}
    assert len(trials) == len(autotune.LAYOUTS) * 3 * 3
    errors = [t for t in trials if "error" in t]
    assert len(errors) == len(autotune.LAYOUTS) * 3 and all(t["cluster_size"] == 16 for t in errors)
    timed = [t for t in trials if "ms_per_substep" in t]
    assert all(t["atomic_scatter_fraction"] == pytest.approx(0.1) for t in timed)
    # every engine that was made got every instance, the parameters, and was closed
    assert all(e.loaded == 3 and e.params == {"actuation": [500.0] * 3} and e.closed for e in StandInEngine.made)
    # each trial: a warm-up of one re-sort interval, then whole intervals of at least trial_steps
    for e in StandInEngine.made:
        ri = e.cfg["resort_interval"]
        assert e.timed_from == ri and (e.substeps - ri) % ri == 0 and e.substeps - ri >= min(64, ri)


def test_no_runnable_configuration_is_an_error(monkeypatch):
    monkeypatch.setattr(autotune, "Engine", StandInEngine)
    with pytest.raises(RuntimeError, match="no batched configuration"):
        autotune.autotune(["spec"], [("p", "m", "f")], clusters=(16,), resorts=(16,))
