"""A rank of a stand-in benchmark for tests/test_launch.py (CPU, gloo).

Run by jellyfih_b200.launch.spawn_ranks as bench.py is: it reads RANK /
WORLD_SIZE / MASTER_* from the environment, steps a stand-in engine for its
share of the instances (rows that are a function of the instance index), and
gathers the (M, 5) rows of every rank the way bench.py's e2e leg does
(jellyfih_b200.shard.gather_rows); rank 0 prints one JSON line.
"""
import json
import os
import sys
from datetime import timedelta

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def main():
    import torch.distributed as dist
    from jellyfih_b200.shard import gather_rows

    M = int(sys.argv[sys.argv.index("--instances") + 1]) if "--instances" in sys.argv else 4
    rank = int(os.environ["RANK"])
    world = int(os.environ["WORLD_SIZE"])
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    try:
        rows = np.array([[rank * M + m, rank, m, 0.5, 1.0] for m in range(M)], np.float64)
        allrows = gather_rows(rows)
        if rank == 0:
            print(json.dumps({"n_gpus": world, "gathered_results": int(allrows.shape[0]),
                              "ranks_seen": sorted({int(r) for r in allrows[:, 1]}),
                              "first_column": allrows[:, 0].tolist()}), flush=True)
        dist.barrier()
    finally:
        dist.destroy_process_group()
    if "--fail-on-rank" in sys.argv and rank == int(sys.argv[sys.argv.index("--fail-on-rank") + 1]):
        return 3
    return 0


if __name__ == "__main__":
    sys.exit(main())
