"""Instance sharding host logic, world_size 2 over gloo on CPU.

The engine is replaced by a deterministic stand-in (a CPU function of the
instance's inputs), so these tests exercise the partition and the result
gather of the multi-GPU path without a GPU.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from jellyfih_b200 import shard


class FakeEngine:
    def __init__(self, n):
        self.n = n
        self.rows = np.zeros((n, 5))
        self.params = {}

    def load(self, k, pos, mat, fib):
        live = mat >= 0
        self.rows[k] = [pos[live, 1].mean(), pos[live, 0].mean(), live.sum(), mat.sum(), 1.0]

    def set_params(self, **kw):
        self.params = kw

    def run_headless(self, steps):
        out = self.rows.copy()
        out[:, 2] += steps * np.asarray(self.params["freq"])
        return out


def _inputs(M, seed):
    rng = np.random.default_rng(seed)
    out = []
    for m in range(M):
        n = int(rng.integers(50, 400))
        pos = rng.uniform(0, 1, (n, 2)).astype(np.float32)
        mat = rng.integers(-1, 4, n).astype(np.int32)
        out.append((pos, mat, None, 0.2 + 0.01 * m, 1.0 + 0.1 * m))
    return out


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, M, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = shard.run_headless_sharded(FakeEngine, _inputs(M, 3), 7)
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("M", [5, 2, 1])
def test_sharded_headless_matches_single_rank(M):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, M, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ref_engine = FakeEngine(M)
    inp = _inputs(M, 3)
    for m, (pos, mat, fib, c, f) in enumerate(inp):
        ref_engine.load(m, pos, mat, fib)
    ref_engine.set_params(contraction=[i[3] for i in inp], freq=[i[4] for i in inp])
    ref = ref_engine.run_headless(7)
    for r in (0, 1):
        np.testing.assert_array_equal(results[r], ref)


def test_contiguous_partition_balances_and_covers():
    w = [62000, 61000, 63000, 120000, 40000, 41000, 160000, 60000]
    for parts in (1, 2, 3, 4, 8):
        b = shard.contiguous_partition(w, parts)
        assert b[0][0] == 0 and b[-1][1] == len(w)
        assert all(b[k][1] == b[k + 1][0] for k in range(parts - 1))
        assert all(hi > lo for lo, hi in b)
        loads = [sum(w[lo:hi]) for lo, hi in b]
        assert max(loads) <= sum(w) / parts + max(w)
    assert shard.contiguous_partition([1, 1], 4) == [(0, 1), (1, 2), (2, 2), (2, 2)]
    assert shard.contiguous_partition([], 2) == [(0, 0), (0, 0)]


def _nccl_worker(port, q):
    """One NCCL rank on cuda:0: the sharded headless run on real engines, the
    row gather through NCCL (device tensors), and the scalar all-reduce the
    benchmark uses for its max-over-ranks time."""
    import torch
    from jellyfih_b200 import Engine, InstanceSpec
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=torch.device("cuda", 0))
    try:
        inputs = _tank_inputs()
        got = shard.run_headless_sharded(
            lambda n: Engine([InstanceSpec(8000, 64, 64, 1.0)] * n, path="batched"), inputs, 20)
        t = torch.tensor([3.5], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        q.put((dist.get_backend(), got, float(t.item())))
    finally:
        dist.destroy_process_group()


def _tank_inputs():
    from jellyfih_b200 import tank
    out = []
    for g in tank.uniform_genomes(3, 11):
        pos, mat, fib, _ = tank.fill_tank(g, 8000, grid_res=64)
        c, f = tank.timing_params(g)
        out.append((pos, mat, fib, c, f))
    return out


@pytest.mark.gpu
def test_sharded_headless_over_nccl_matches_one_engine():
    """The NCCL branch of the result gather (rows staged on the GPU), run as a
    one-rank NCCL group in a spawned process, against run_headless of one
    engine holding every instance (the same substeps; rows agree to the
    summation-order noise of 20 substeps)."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from jellyfih_b200 import Engine, InstanceSpec
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_nccl_worker, args=(_free_port(), q))
    p.start()
    backend, got, tmax = q.get(timeout=300)
    p.join(timeout=60)
    assert p.exitcode == 0 and backend == "nccl" and tmax == 3.5
    inputs = _tank_inputs()
    e = Engine([InstanceSpec(8000, 64, 64, 1.0)] * len(inputs), path="batched")
    try:
        for m, (pos, mat, fib, c, f) in enumerate(inputs):
            e.load(m, pos, mat, fib)
        e.set_params(contraction=[i[3] for i in inputs], freq=[i[4] for i in inputs])
        ref = e.run_headless(20)
    finally:
        e.close()
    assert got.shape == (len(inputs), 5)
    np.testing.assert_array_equal(got[:, [0, 1, 4]], ref[:, [0, 1, 4]])
    np.testing.assert_allclose(got[:, 2:4], ref[:, 2:4], rtol=0, atol=1e-6)
