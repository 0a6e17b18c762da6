"""GPU tank fill (jf_load_robot through the C ABI) against the host
restatement of make_jelly.py:336-402 (jellyfih_b200.tank.fill_tank, whose
generator is pinned to the reference's in tests/test_tank.py): slot contents
must be identical bit for bit — positions, materials, fibres, the load reset,
and the robot / water counts — over seeded genomes, grid shapes, lattice
spacings and slot limits that cut the water or the robot."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

PATHS = ("plain", "batched")


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from jellyfih_b200 import build
    build.build()


# (slots, n_grid, n_grid_y, domain_height, spawn, spacing_div, with_payload, axisym)
CASES = [
    (80000, 128, 128, 1.0, None, 2.0, True, False),      # the bench tank
    (20000, 128, 128, 1.0, None, 2.0, True, False),      # water cut at the slot limit
    (1000, 128, 128, 1.0, None, 2.0, True, False),       # robot cut, no water
    (20000, 64, 64, 1.0, None, 2.0, True, False),        # 64^2 population tanks
    (160000, 128, 256, 2.0, (0.5, 0.60), 2.0, True, False),  # tall tank
    (120000, 128, 128, 1.0, None, 2.7, True, False),     # denser lattice (live counts up to 120K)
    (60000, 128, 128, 1.0, None, 1.6, False, False),     # sparser lattice, no payload
    (80000, 128, 256, 2.0, "axisym", 2.0, True, True),  # axisymmetric half profile
]


def _compare(e, m, fx, stats_ref, counts):
    got = e.read(m)
    pos, mat, fib, _st = fx
    np.testing.assert_array_equal(got["material"], mat)
    np.testing.assert_array_equal(got["x"], pos)
    np.testing.assert_array_equal(got["fiber"], fib)
    assert not got["v"].any() and not got["C"].any()
    np.testing.assert_array_equal(got["F"], np.broadcast_to(np.eye(2, dtype=np.float32), got["F"].shape))
    np.testing.assert_array_equal(got["Jp"], np.ones_like(got["Jp"]))
    assert counts["n_robot"] == stats_ref["n_robot"] and counts["n_water"] == stats_ref["n_water"]
    assert counts["muscle_count"] == stats_ref["muscle_count"]


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("case", range(len(CASES)))
def test_gpu_tank_matches_host_fill(case, path):
    from jellyfih_b200 import Engine, InstanceSpec, tank
    slots, nx, ny, dh, spawn, sd, payload, axisym = CASES[case]
    genomes = tank.gaussian_genomes(3, 100 + case)
    spawn = tank.AXISYM_SPAWN if spawn == "axisym" else (None if spawn is None else np.array(spawn))
    e = Engine([InstanceSpec(slots, nx, ny, dh)] * len(genomes), path=path, axisym=axisym)
    try:
        for m, g in enumerate(genomes):
            fx = tank.fill_tank(g, slots, grid_res=nx, spawn_offset=spawn, with_payload=payload,
                                domain_height=dh, spacing_div=sd, axisym=axisym)
            st = tank.load_tank(e, m, g, spawn_offset=spawn, with_payload=payload, spacing_div=sd, axisym=axisym)
            _compare(e, m, fx, fx[3], st)
    finally:
        e.close()


def test_gpu_tank_without_robot_is_the_whole_lattice():
    from jellyfih_b200 import Engine, InstanceSpec
    e = Engine([InstanceSpec(70000)], path="plain")
    try:
        nr, nw = e.load_robot(0, np.zeros((0, 2)), np.zeros(0, np.int32))
        sp = 1.0 / 256
        mg = 3.0 / 256
        wx = np.arange(mg, 1.0 - mg, sp)
        wy = np.arange(mg, 1.0 - mg, sp)
        gx, gy = np.meshgrid(wx, wy)
        lat = np.vstack([gx.ravel(), gy.ravel()]).T.astype(np.float32)
        assert nr == 0 and nw == len(lat)
        got = e.read(0)
        np.testing.assert_array_equal(got["x"][:nw], lat)
        assert (got["material"][:nw] == 0).all() and (got["material"][nw:] == -1).all()
    finally:
        e.close()


def test_gpu_tank_then_step_runs():
    """A tank loaded on the GPU steps like one loaded from host arrays."""
    from jellyfih_b200 import Engine, InstanceSpec, tank
    g = tank.gaussian_genomes(2, 7)
    a = Engine([InstanceSpec(80000)] * 2, path="batched")
    b = Engine([InstanceSpec(80000)] * 2, path="batched")
    try:
        for m in range(2):
            tank.load_tank(a, m, g[m])
            pos, mat, fib, _ = tank.fill_tank(g[m], 80000)
            b.load(m, pos, mat, fib)
        for m in range(2):
            np.testing.assert_array_equal(a.read(m)["x"], b.read(m)["x"])
        a.step(64)
        b.step(64)
        # the same start; float atomics make the two runs differ by rounding only
        for m in range(2):
            np.testing.assert_allclose(a.read(m)["x"], b.read(m)["x"], atol=1e-5)
    finally:
        a.close()
        b.close()


def test_gpu_tanks_over_a_pool_match_host_fill():
    """load_tanks with the robots generated over spawned workers: every
    instance's slots equal fill_tank's."""
    from jellyfih_b200 import Engine, InstanceSpec, tank
    genomes = tank.gaussian_genomes(4, 55)
    e = Engine([InstanceSpec(80000)] * 4, path="batched")
    pool = tank.make_pool(2)
    try:
        stats = tank.load_tanks(e, genomes, executor=pool)
        for m, g in enumerate(genomes):
            fx = tank.fill_tank(g, 80000)
            _compare(e, m, fx, fx[3], stats[m])
    finally:
        pool.shutdown()
        e.close()
