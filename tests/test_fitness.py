"""Fitness restatement (evolve.py:90-124), host side; the GPU kernel is
compared with it in test_gpu_parity."""
import numpy as np

from jellyfih_b200.fitness import compute_fitness


def test_fitness_modes_penalty_and_cap():
    rows = np.array([[0.40, 0.5, 0.42, 0.5, 1.0],     # rises 0.02
                     [0.40, 0.5, 0.38, 0.5, 1.0],     # sinks 0.02
                     [0.40, 0.5, 0.99, 0.5, 1.0],     # capped at 1 - 0.07
                     [0.40, 0.5, 0.45, 0.5, 0.0],     # invalid (floor)
                     [0.40, 0.5, 0.45, 0.5, 1.0]])    # invalid (muscle floor)
    muscle = [500, 500, 500, 500, 150]
    genomes = [np.r_[np.zeros(9), 0.2, 1.0]] * 5
    f = compute_fitness(rows, muscle, genomes)
    cost = (500 * 0.2 / 500) ** 0.5
    np.testing.assert_allclose(f[:3], [-0.02 / cost, 0.02 / cost, -(0.93 - 0.40) / cost])
    assert f[3] == f[4] == max(f[:3]) + 1.0
    d = compute_fitness(rows, muscle, mode="displacement")
    np.testing.assert_allclose(d[:3], [-0.02, 0.02, -(0.93 - 0.40)])
    assert compute_fitness(rows[3:4], [500]) == [100.0]
