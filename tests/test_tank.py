"""Input generator (make_jelly.py restatement) sanity checks, CPU only."""
import numpy as np

from jellyfih_b200 import tank


def test_fill_tank_layout():
    g = np.concatenate([tank.AURELIA_GENOME, [0.2, 1.0]])
    pos, mat, fib, st = tank.fill_tank(g, 80000)
    n = st["n_total"]
    assert pos.dtype == np.float32 and mat.dtype == np.int32 and fib.dtype == np.float32
    assert 55000 < n < 70000                       # ~62K live of 80K slots
    assert np.all(mat[:n] >= 0) and np.all(mat[n:] == -1)
    assert np.all(pos[n:] == -1.0)
    assert np.all(fib[n:, 1] == 1.0)
    assert (mat == 2).sum() == 240                 # 20 x 12 payload lattice
    assert st["muscle_count"] == (mat == 3).sum()
    muscle = mat == 3
    np.testing.assert_allclose(np.linalg.norm(fib[muscle], axis=1), 1.0, atol=1e-5)
    # mirror symmetry of the soft body about the spawn axis
    body = (mat == 1) | (mat == 3)
    xs = np.sort(np.round(pos[body, 0] - 0.5, 6))
    np.testing.assert_allclose(xs, -xs[::-1], atol=1e-6)


def test_water_lattice_spacing_and_margin():
    pos, mat, _, _ = tank.fill_tank(np.concatenate([tank.AURELIA_GENOME, [0.2, 1.0]]), 80000)
    w = pos[mat == 0]
    assert w[:, 0].min() >= 3 / 256 - 1e-6 and w[:, 1].min() >= 3 / 256 - 1e-6
    assert w[:, 0].max() < 1 - 3 / 256 and w[:, 1].max() < 1 - 3 / 256
    u = np.unique(np.round(w[:, 0] * 256, 3))
    np.testing.assert_allclose(np.diff(u), 1.0, atol=1e-3)


def test_jitter_is_seeded_and_bounded():
    g = tank.uniform_genomes(1, 3)[0]
    a = tank.fill_tank(g, 80000, jitter=0.25, seed=5)[0]
    b = tank.fill_tank(g, 80000, jitter=0.25, seed=5)[0]
    c = tank.fill_tank(g, 80000)[0]
    assert np.array_equal(a, b)
    live = c[:, 0] >= 0
    d = np.abs(a[live] - c[live])
    assert d.max() <= 0.25 / 128 + 1e-6 and d.max() > 0.1 / 128


def test_points_in_polygon_matches_brute_force():
    rng = np.random.default_rng(0)
    square = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], float)
    pts = rng.uniform(-0.5, 1.5, (2000, 2))
    inside = tank.points_in_polygon(pts, square)
    truth = (pts[:, 0] > 0) & (pts[:, 0] < 1) & (pts[:, 1] > 0) & (pts[:, 1] < 1)
    assert np.array_equal(inside, truth)
    th = np.linspace(0, 2 * np.pi, 200, endpoint=False)
    circle = np.stack([np.cos(th), np.sin(th)], 1)
    pts = rng.uniform(-1.2, 1.2, (4000, 2))
    r = np.linalg.norm(pts, axis=1)
    got = tank.points_in_polygon(pts, circle)
    sure = (r < 0.99) | (r > 1.01)
    assert np.array_equal(got[sure], (r < 1)[sure])


def test_genome_samplers_respect_bounds():
    for g in (tank.uniform_genomes(64, 1), tank.gaussian_genomes(64, 2)):
        assert np.all(g >= tank.GENOME_LOWER) and np.all(g <= tank.GENOME_UPPER)
    c, f = tank.timing_params(np.array([0] * 9 + [0.9, 3.0]))
    assert (c, f) == (0.60, 2.0)


def test_tall_tank_and_coarse_grid():
    g = np.concatenate([tank.AURELIA_GENOME, [0.2, 1.0]])
    pos, mat, _, st = tank.fill_tank(g, 160000, domain_height=2.0, spawn_offset=tank.TALL_SPAWN)
    assert 115000 < st["n_total"] <= 160000 and pos[mat >= 0, 1].max() > 1.9
    pos, mat, _, st = tank.fill_tank(g, 24000, grid_res=64)
    assert 14000 < st["n_total"] < 24000


def _self_intersects_loop(polygon):
    """The reference's pair loop (make_jelly.py:46-58) over _segments_intersect."""
    n = len(polygon)
    for i in range(n):
        a, b = polygon[i], polygon[(i + 1) % n]
        for j in range(i + 2, n):
            if j == n - 1 and i == 0:
                continue
            if tank._segments_intersect(a, b, polygon[j], polygon[(j + 1) % n]):
                return True
    return False


def test_vectorised_self_intersection_matches_the_pair_loop():
    rng = np.random.default_rng(11)
    verdicts = []
    for k in range(60):
        n = int(rng.integers(4, 40))
        if k % 2:
            # star-shaped polygon ordered by angle: simple (no crossing)
            th = np.sort(rng.uniform(0, 2 * np.pi, n))
            poly = np.stack([np.cos(th), np.sin(th)], 1) * rng.uniform(0.5, 1.0, (n, 1))
        else:
            poly = rng.uniform(0, 1, (n, 2))
        got = tank.polygon_self_intersects(poly)
        assert got == _self_intersects_loop(poly), k
        verdicts.append(got)
    assert any(verdicts) and not all(verdicts)
    for g in tank.uniform_genomes(8, 5):
        pos, mat, fib, st = tank.fill_tank(g, 80000)
        assert isinstance(st["self_intersecting"], bool)


def test_phenotypes_over_a_process_pool_match_serial():
    """generate_phenotype spread over spawned workers returns the serial
    results bit for bit, in genome order."""
    from jellyfih_b200 import tank
    genomes = tank.gaussian_genomes(6, 21)
    serial = tank.phenotypes(genomes, grid_res=[128, 64, 128, 64, 128, 128])
    pool = tank.make_pool(2)
    try:
        pooled = tank.phenotypes(genomes, grid_res=[128, 64, 128, 64, 128, 128], executor=pool)
    finally:
        pool.shutdown()
    assert len(pooled) == len(serial)
    for a, b in zip(serial, pooled):
        for x, y in zip(a[:3], b[:3]):
            np.testing.assert_array_equal(x, y)
        assert a[3] == b[3]
