"""The drop-in mpm_sim module's host side (jellyfih_b200/mpm_sim.py) on the CPU,
with a stand-in engine: its import reads the reference's JELLY_* variables
(mpm_sim.py:11-17) and sizes the engine from them, the fields read and write
single elements and whole arrays in the reference's shapes, load_particles
defaults the fibre to (0, 1), the fitness buffer accumulates the engine's FP64
sums as compute_payload_stats / compute_body_stats do (mpm_sim.py:740-762),
and fields that only load_particles may set refuse a direct write.
"""
import importlib
import sys

import numpy as np
import pytest


class StandInEngine:
    def __init__(self, instances, path="batched", dt=2e-5, glow=False, axisym=False, **kw):
        self.instances, self.path, self.dt, self.glow, self.axisym = list(instances), path, dt, glow, axisym
        self.M = len(self.instances)
        self.params = {k: np.zeros(self.M, np.float32) for k in ("actuation", "contraction", "freq",
                                                                   "payload_density")}
        self.time = np.float32(0.0)
        self.loads, self.steps = [], 0
        n = self.instances[0].n_slots
        self.state = [{"x": np.zeros((n, 2), np.float32), "v": np.zeros((n, 2), np.float32),
                       "C": np.zeros((n, 2, 2), np.float32), "F": np.zeros((n, 2, 2), np.float32),
                       "material": np.zeros(n, np.int32), "Jp": np.ones(n, np.float32),
                       "glow": np.zeros(n, np.float32), "fiber": np.zeros((n, 2), np.float32)}
                      for _ in range(self.M)]

    def get_params(self):
        return {k: v.copy() for k, v in self.params.items()}

    def set_params(self, **kw):
        for k, v in kw.items():
            if v is not None:
                self.params[k][...] = v

    def load(self, m, pos, mat, fib):
        self.loads.append((m, np.array(pos), np.array(mat), np.array(fib)))

    def step(self, n):
        self.steps += n

    def read(self, m):
        return {k: v.copy() for k, v in self.state[m].items()}

    def write(self, m, **kw):
        for k, v in kw.items():
            self.state[m][k][...] = v

    def stats_raw(self):
        return np.tile(np.arange(6, dtype=np.float64), (self.M, 1)) + 1.0


@pytest.fixture
def sim(monkeypatch):
    from jellyfih_b200 import engine as engine_mod
    monkeypatch.setenv("JELLY_INSTANCES", "3")
    monkeypatch.setenv("JELLY_PARTICLES", "5")
    monkeypatch.setenv("JELLY_GRID_Y", "256")
    monkeypatch.setenv("JELLY_DOMAIN_H", "2.0")
    monkeypatch.setenv("JELLY_B200_PATH", "plain")
    monkeypatch.setattr(engine_mod, "Engine", StandInEngine)
    sys.modules.pop("jellyfih_b200.mpm_sim", None)
    mod = importlib.import_module("jellyfih_b200.mpm_sim")
    yield mod
    sys.modules.pop("jellyfih_b200.mpm_sim", None)


def test_import_sizes_the_engine_from_the_environment(sim):
    e = sim.engine()
    assert (sim.n_instances, sim.n_particles, sim.n_grid, sim.n_grid_y, sim.domain_height) == (3, 5, 128, 256, 2.0)
    assert e.M == 3 and e.path == "plain" and e.dt == pytest.approx(2e-5)
    assert {(s.n_slots, s.n_grid, s.n_grid_y, s.domain_height) for s in e.instances} == {(5, 128, 256, 2.0)}
    assert sim.grid_side == 2 and sim.res_sub == 512


def test_parameter_and_time_fields(sim):
    sim.instance_freq.fill(1.0)
    sim.instance_freq[1] = 1.7
    assert sim.instance_freq.to_numpy().tolist() == pytest.approx([1.0, 1.7, 1.0])
    assert sim.instance_freq[1] == pytest.approx(1.7)
    sim.instance_act_contraction.from_numpy([0.1, 0.2, 0.3])
    assert sim.engine().params["contraction"].tolist() == pytest.approx([0.1, 0.2, 0.3])
    sim.sim_time[None] = 0.25
    assert sim.sim_time[None] == 0.25 and sim.sim_time.to_numpy().dtype == np.float32


def test_load_particles_defaults_the_fibre(sim):
    pos = np.full((5, 2), 0.5, np.float32)
    mat = np.array([0, 1, 2, 3, -1], np.int32)
    sim.load_particles(2, pos, mat)
    m, _, _, fib = sim.engine().loads[-1]
    assert m == 2 and fib.shape == (5, 2)
    assert np.all(fib[:, 0] == 0) and np.all(fib[:, 1] == 1)
    sim.substep()
    assert sim.engine().steps == 1


def test_particle_fields_and_fitness_buffer(sim):
    sim.v[1, 3] = [0.5, -0.5]
    assert sim.v[1, 3].tolist() == [0.5, -0.5]
    assert sim.v.to_numpy().shape == (3, 5, 2)
    sim.F.fill(2.0)
    assert np.all(sim.F.to_numpy() == 2.0)
    with pytest.raises(NotImplementedError):
        sim.material[0, 0] = 3
    with pytest.raises(NotImplementedError):
        sim.fiber_dir.from_numpy(np.zeros((3, 5, 2)))
    sim.clear_fitness_buffer()
    sim.compute_payload_stats()
    sim.compute_body_stats()
    assert sim.fitness_buffer.to_numpy()[0].tolist() == [1.0 + 4.0, 2.0 + 5.0, 3.0 + 6.0]
    sim.clear_fitness_buffer()
    assert not sim.fitness_buffer.to_numpy().any()
