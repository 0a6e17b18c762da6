"""Small differentiable-rollout cases shared by the CPU and GPU gradient tests."""
from jellyfih_b200 import tank


def small_tank(seed=3, grid=32, slots=6000):
    """A 32^2 tank: jellyfish from a seeded genome plus the water lattice."""
    g = tank.uniform_genomes(1, seed)[0]
    g[9] = 0.35  # contraction window longer than the rollouts here: no 1 -> 0 drop inside
    pos, mat, fib, st = tank.fill_tank(g, slots, grid_res=grid, jitter=0.25, seed=seed)
    return pos, mat, fib, dict(actuation=900.0, contraction=float(g[9]), freq=1.3, payload_density=2.5)
