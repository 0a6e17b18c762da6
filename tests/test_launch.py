"""bench.py --gpus N without torchrun: one process per rank (CPU, gloo).

jellyfih_b200.launch.spawn_ranks is what bench.py calls when --gpus N > 1 and
no WORLD_SIZE is set.  Here it drives a stand-in benchmark
(tests/launch_stub.py) at N = 2: exactly one JSON line comes back, from rank
0, with n_gpus == 2 and the rows of both ranks gathered in rank order; a rank
that exits non-zero makes the launcher return its code.
"""
import json
import os
import tempfile

from jellyfih_b200 import launch

STUB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "launch_stub.py")


def _run(argv, n=2):
    with tempfile.TemporaryFile(mode="w+") as out:
        rc = launch.spawn_ranks(n, STUB, argv, timeout_s=120, stdout=out)
        out.seek(0)
        lines = [ln for ln in out.read().splitlines() if ln.strip()]
    return rc, lines


def test_two_ranks_one_line_all_rows():
    M = 3
    rc, lines = _run(["--instances", str(M)])
    assert rc == 0
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["n_gpus"] == 2
    assert d["gathered_results"] == 2 * M
    assert d["ranks_seen"] == [0, 1]
    assert d["first_column"] == list(range(2 * M))


def test_failing_rank_is_reported():
    rc, _ = _run(["--instances", "2", "--fail-on-rank", "1"])
    assert rc == 3


def test_rank_environment():
    env = launch.rank_env(1, 4, 12345, base={})
    assert env == {"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "4", "LOCAL_WORLD_SIZE": "4",
                   "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": "12345"}


def test_reference_arm_uses_every_core_under_torchrun_and_only_on_rank_0():
    """bench.py --impl reference at N = 2 under torchrun's environment
    (OMP_NUM_THREADS=1 for every rank): rank 0 prints the one line and times the
    oracle on all of its cores; rank 1 exits 0 without output."""
    import subprocess
    import sys
    bench = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "bench.py")
    argv = [sys.executable, bench, "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0",
            "--instances", "1", "--substeps", "2"]
    cores = len(os.sched_getaffinity(0))
    outs = []
    for rank in (0, 1):
        env = launch.rank_env(rank, 2, 29500)
        env["OMP_NUM_THREADS"] = "1"
        p = subprocess.run(argv, env=env, capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, p.stderr[-2000:]
        outs.append([ln for ln in p.stdout.splitlines() if ln.strip()])
    assert outs[1] == []
    assert len(outs[0]) == 1
    d = json.loads(outs[0][0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2
    assert d["cpu_baseline"]["cores"] == cores
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
