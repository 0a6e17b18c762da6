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
