"""One process per GPU on one node, without torchrun.

`spawn_ranks(n, script, argv)` starts `python script argv` n times with the
environment a torch.distributed env:// rendezvous reads (RANK, LOCAL_RANK,
WORLD_SIZE, LOCAL_WORLD_SIZE, MASTER_ADDR = 127.0.0.1, MASTER_PORT = a free
port), so rank r drives GPU r, as the reference runs one independent process
per GPU.  Rank 0's standard output passes through (the other ranks' is
dropped, so a benchmark prints one line); standard error of every rank passes
through.  When a rank exits non-zero the others are terminated, so that none
waits for good in a collective its peer will never join.
"""
from __future__ import annotations

import os
import socket
import subprocess
import sys
import time


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_env(rank: int, world: int, port: int, base=None) -> dict:
    env = dict(os.environ if base is None else base)
    env.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), LOCAL_WORLD_SIZE=str(world),
               MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    return env


def spawn_ranks(n: int, script: str, argv, timeout_s: float | None = None, stdout=None) -> int:
    """Runs n ranks of `script` and returns the first non-zero exit code (0 if
    every rank succeeded).  `stdout` receives rank 0's output (default: this
    process's standard output).  After `timeout_s` seconds every rank still
    running is terminated and 124 is returned."""
    if n < 1:
        raise ValueError("n must be >= 1")
    port = free_port()
    procs = []
    for r in range(n):
        out = stdout if r == 0 else subprocess.DEVNULL
        procs.append(subprocess.Popen([sys.executable, script, *argv], env=rank_env(r, n, port), stdout=out))
    rc = 0
    t0 = time.monotonic()
    kill_at = None  # ranks still running 10 s after being terminated are killed
    alive = set(range(n))

    def stop_all(now):
        nonlocal kill_at
        for q in alive:
            procs[q].terminate()
        kill_at = now + 10.0 if kill_at is None else kill_at

    try:
        while alive:
            now = time.monotonic()
            for r in sorted(alive):
                code = procs[r].poll()
                if code is None:
                    continue
                alive.discard(r)
                if code != 0 and rc == 0:
                    rc = code
                    stop_all(now)
            if timeout_s is not None and alive and now - t0 > timeout_s and kill_at is None:
                rc = rc or 124
                stop_all(now)
            if kill_at is not None and now > kill_at:
                for q in alive:
                    procs[q].kill()
            if alive:
                time.sleep(0.1)
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
                p.wait()
    return rc
