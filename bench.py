#!/usr/bin/env python
"""Throughput benchmark of the batched MLS-MPM substep (particle-steps/s).

Workload (one bench step): 32 jellyfish instances per GPU, 80,000 particle
slots each (about 62K live: water lattice + robot from a seeded genome), 128^2
grid, FP32, advanced by ``--substeps`` (default 1,000) substeps through the
batched path.  Genomes are drawn from an isotropic Gaussian (sigma = 0.3 of
each gene's range) around the bound midpoint and clipped, per rank seed.
Inputs are synthetic (no reference datasets exist for this path).

``value`` is live particles x substeps / device time of the timed steps
(CUDA events on the engine's stream, max over ranks), inputs resident in HBM.
``e2e`` repeats the workload through the public API with host buffers: every
step loads each instance from pinned host memory, runs the episode with
``run_headless`` and reads the (M, 5) result back.  ``roofline`` rates the
dominant kernel (the batched chunk kernel) at 100 algorithmic bytes per live
particle-substep (x, v, C, F read and written, material read) against the
measured HBM copy bandwidth.  ``cpu_baseline`` times the CPU oracle (a
restatement of the reference's substep) on the host cores.  ``plain`` times
the plain per-instance launch path on the same inputs.  ``render`` times the
headless renderer (a 1024^2 viewer frame of every particle) on the final
state, beside the CPU oracle rendering the same frame.  ``tank`` times one
generation's tank loading: host-built slot arrays against the GPU water fill.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

ALGO_BYTES = 100  # bytes per live particle-substep: (x,v,C,F) 48 read + 48 write, material 4
METRIC = "particle-steps/s @32x80K, 128^2 (batched)"
UNIT = "particle-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--substeps", type=int, default=1000, help="substeps per bench step")
    ap.add_argument("--instances", type=int, default=32, help="instances per GPU")
    ap.add_argument("--slots", type=int, default=80000)
    ap.add_argument("--resort", type=int, default=64)
    ap.add_argument("--block", type=int, default=0,
                    help="threads per CTA of the chunk kernel (above 512: node blocks in TMEM); "
                         "0 = the engine's choice")
    ap.add_argument("--no-extras", action="store_true", help="skip plain / e2e / CPU legs")
    ap.add_argument("--no-uneven", action="store_true", help="skip the uneven-batch leg")
    ap.add_argument("--no-refine", action="store_true", help="skip the 256 x 64^2 gradient-refinement leg")
    ap.add_argument("--no-render", action="store_true", help="skip the headless-renderer leg")
    ap.add_argument("--render-only", action="store_true",
                    help="run only the renderer leg on the workload after --substeps substeps and print it")
    ap.add_argument("--grad-substeps", type=int, default=2000,
                    help="substeps of the differentiable rollout leg (checkpoint every 100)")
    ap.add_argument("--grad-only", action="store_true",
                    help="run only the differentiable leg (8 of the workload's instances) and print it")
    ap.add_argument("--tank-only", action="store_true",
                    help="run only the tank-loading leg (host fill vs the GPU water fill) and print it")
    ap.add_argument("--plain-only", action="store_true",
                    help="run only the plain per-instance path (50 substeps from the loaded inputs) and print it")
    ap.add_argument("--grad-checkpoint", type=int, default=100,
                    help="checkpoint interval of the differentiable rollout leg")
    ap.add_argument("--episode-only", action="store_true",
                    help="run only the end-to-end episode leg (jf_run_episode, --steps episodes of --substeps)")
    ap.add_argument("--noalloc-only", action="store_true",
                    help="run only the allocation-free substep (jf_substep_noalloc) on one instance, --substeps calls")
    return ap.parse_args()


def host_cores():
    """Host cores this process may run on (its CPU affinity where the platform
    reports it, else the machine's count)."""
    try:
        return len(os.sched_getaffinity(0)) or 1
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def make_inputs(M, slots, seed):
    from jellyfih_b200 import tank
    genomes = tank.gaussian_genomes(M, seed)
    out = []
    for g in genomes:
        pos, mat, fib, st = tank.fill_tank(g, slots)
        c, f = tank.timing_params(g)
        out.append((pos, mat, fib, c, f, st))
    return out


def load_all(engine, inputs):
    for m, (pos, mat, fib, c, f, st) in enumerate(inputs):
        engine.load(m, pos, mat, fib)
    engine.set_params(contraction=[i[3] for i in inputs], freq=[i[4] for i in inputs])


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except ValueError:
                continue
            for name, val in zip(self.NAMES, f[3:7]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_per_particle_step():
    """DRAM bytes per live particle-substep of the chunk kernel from the
    committed ncu measurement, and the measurement's record.  The figure is
    None when the kernel's sources changed since that measurement (the file
    records a hash of them); the record still names the figure and the sources
    it was measured on."""
    import hashlib
    p = os.path.join(HERE, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None, None
    with open(p) as f:
        d = json.load(f)
    h = hashlib.sha256()
    for src in d.get("kernel_sources", []):
        with open(os.path.join(HERE, src), "rb") as f:
            h.update(f.read())
    if h.hexdigest()[:16] != d.get("kernel_sources_sha256_16"):
        return None, d
    return d.get("chunk_kernel_dram_bytes_per_live_particle_substep"), d


def cpu_baseline(inputs, target_s=12.0):
    """The CPU oracle on all host cores (OpenMP over instances), a bounded sample."""
    cores = host_cores()
    os.environ["OMP_NUM_THREADS"] = str(cores)
    from oracle import oracle as O
    insts, states = [], []
    for pos, mat, fib, c, f, st in inputs:
        insts.append(O.Instance(contraction=c, freq=f))
        states.append(O.new_state(pos, mat, fib))
    live = sum(int((i[1] >= 0).sum()) for i in inputs)
    # two untimed substeps first (page faults on the fresh states, the OpenMP
    # pool's start); then a short probe and one of about a tenth of the sample
    # (every call also pays a fixed cost, which a short probe overstates) size
    # the timed sample, one call of ~target_s
    t = O.run_batch(insts, states, np.float32(0), 2)
    n = 2
    for _ in range(2):
        t0 = time.perf_counter()
        t = O.run_batch(insts, states, t, n)
        per = (time.perf_counter() - t0) / n
        n = int(max(2, min(200, 0.1 * target_s / max(per, 1e-6))))
    n = int(max(2, min(2000, target_s / max(per, 1e-6))))
    t0 = time.perf_counter()
    O.run_batch(insts, states, t, n)
    el = time.perf_counter() - t0
    return {"value": live * n / el, "unit": UNIT, "cores": int(os.environ["OMP_NUM_THREADS"]),
            "kind": "port",
            "sample": f"{len(inputs)} instances x {n} substeps of the same workload on the CPU oracle "
                      f"({el:.1f} s)"}


def uneven_inputs(seed=3000):
    """48 instances on 128^2 with 40K-120K live particles (lattice spacing
    dx/k, k seeded in [1.6, 2.7]) and 16 tall tanks 128x256 (domain height 2,
    spawn (0.5, 0.6), ~126K live of 160K slots); genomes uniform in bounds."""
    from jellyfih_b200 import InstanceSpec, tank
    rng = np.random.default_rng(seed)
    genomes = tank.uniform_genomes(64, seed)
    specs, data = [], []
    for m, g in enumerate(genomes):
        c, f = tank.timing_params(g)
        if m < 48:
            k = float(rng.uniform(1.6, 2.7))
            pos, mat, fib, st = tank.fill_tank(g, 120000, spacing_div=k)
            specs.append(InstanceSpec(120000, 128, 128, 1.0))
        else:
            pos, mat, fib, st = tank.fill_tank(g, 160000, domain_height=2.0, spawn_offset=tank.TALL_SPAWN)
            specs.append(InstanceSpec(160000, 128, 256, 2.0))
        data.append((pos, mat, fib, c, f, st))
    return specs, data


def uneven_leg(device, stream, substeps=5000):
    """Particle-steps/s of the uneven batch in one batched launch per chunk,
    CUDA-graph replay on, over the configuration's 5,000 substeps, for
    re-sort intervals 1, 4, 16 and the autotuned configuration (kernel layout,
    cluster size, re-sort interval; the autotuner's trials are short)."""
    import torch
    from jellyfih_b200 import Engine
    from jellyfih_b200.autotune import autotune
    specs, data = uneven_inputs()
    live = sum(int((d[1] >= 0).sum()) for d in data)
    out = {"instances": len(specs), "live_particles": live, "substeps": substeps, "resort": {}}

    def timed(**cfg):
        e = Engine(specs, path="batched", device=device, **cfg)
        e.set_stream(stream)
        load_all(e, data)
        e.time = 0.0
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        e.step(substeps)
        ev1.record(stream)
        ev1.synchronize()
        assert not e.error_flags().any()
        e.close()
        return live * substeps / (ev0.elapsed_time(ev1) / 1e3)

    for ri in (1, 4, 16):
        out["resort"][str(ri)] = timed(resort_interval=ri)
    best, table = autotune(specs, [d[:3] for d in data], clusters=(0, 8), resorts=(16, 32, 64),
                           trial_steps=64, device=device)
    out["autotuned"] = dict(best, value=timed(**best))
    out["autotune_trials"] = len(table)
    out["unit"] = UNIT
    return out


def refine_leg(device, stream, M=256, steps=4000, iterations=3, checkpoint_every=50):
    """The gradient-refined search step of the 256 x 64^2 configuration (dx = 1/64,
    20,000 slots, ~14.9K live) over its 4,000-substep horizon: genomes from a
    seeded Gaussian (CMA-ES style) sample, `iterations` gradient steps of 0.05
    of the range on the two timing genes (each the checkpointed forward and
    the backward of all instances replayed as one CUDA graph), then the
    initial and refined genomes re-evaluated by the plain forward path and the
    GPU fitness kernel.  The first iteration of an untimed warm-up run
    captures the graph."""
    import torch
    from jellyfih_b200 import Engine, InstanceSpec, tank
    from jellyfih_b200.autograd import refine_timing_genes
    genomes = tank.gaussian_genomes(M, 5000)
    data = [tank.fill_tank(g, 20000, grid_res=64) for g in genomes]
    pos = [d[0] for d in data]
    mats = [d[1] for d in data]
    fibs = [d[2] for d in data]
    muscle = np.array([d[3]["muscle_count"] for d in data], np.int32)
    spec = InstanceSpec(20000, 64, 64, 1.0)
    e = Engine([spec] * M, path="plain", device=device)
    e.set_stream(stream)
    refine_timing_genes(e, genomes, pos, mats, fibs, steps, 1, checkpoint_every=checkpoint_every)  # warm-up, capture
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    refined, hist = refine_timing_genes(e, genomes, pos, mats, fibs, steps, iterations,
                                        checkpoint_every=checkpoint_every)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    e.close()

    evaluator = Engine([spec] * M, path="plain", device=device)
    evaluator.set_stream(stream)
    fits = {}
    for name, g in (("initial", genomes), ("refined", refined)):
        for m in range(M):
            evaluator.load(m, pos[m], mats[m], fibs[m])
        c = np.clip(g[:, 9], 0.05, 0.60)
        evaluator.set_params(contraction=c, freq=np.clip(g[:, 10], 0.5, 2.0))
        rows = evaluator.run_headless(steps)
        fits[name] = {"mean_displacement": float(np.mean(rows[:, 2] - rows[:, 0])),
                      "fitness": evaluator.fitness(rows, muscle, c, mode="displacement")}
    evaluator.close()
    better = float(np.mean(fits["refined"]["fitness"] < fits["initial"]["fitness"]))
    return {"instances": M, "grid": "64x64", "slots": 20000, "live_per_instance": float(np.mean([(m >= 0).sum() for m in mats])),
            "substeps": steps, "checkpoint_every": checkpoint_every, "gradient_steps": iterations,
            "s_per_gradient_step": wall / iterations,
            "mean_displacement_per_step": [float(np.mean(h)) for h in hist],
            "plain_evaluation": {"initial_mean_displacement": fits["initial"]["mean_displacement"],
                            "refined_mean_displacement": fits["refined"]["mean_displacement"],
                            "fraction_with_better_fitness": better}}


def grad_leg(inputs, device, stream, steps=2000, checkpoint_every=100):
    """fwd+bwd / fwd of the differentiable rollout: 8 instances x 80,000 slots,
    2,000 substeps with a checkpoint every 100 (the gradient workload), device
    time of the checkpointed forward and of the backward (recompute + adjoint)."""
    import torch
    from jellyfih_b200 import Engine, InstanceSpec
    M = len(inputs)
    e = Engine([InstanceSpec(len(inputs[0][1]))] * M, path="plain", device=device)
    e.set_stream(stream)
    load_all(e, inputs)
    e.time = 0.0
    e.grad_forward(steps, checkpoint_every)  # warm-up: module load, checkpoint and segment buffers
    e.grad_backward()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    load_all(e, inputs)
    e.time = 0.0
    ev[0].record(stream)
    e.grad_forward(steps, checkpoint_every)
    ev[1].record(stream)
    e.grad_backward()
    ev[2].record(stream)
    ev[2].synchronize()
    fwd = ev[0].elapsed_time(ev[1])
    bwd = ev[1].elapsed_time(ev[2])
    # the batched product forward on the same instances and substeps
    b = Engine([InstanceSpec(len(inputs[0][1]))] * M, path="batched", device=device)
    b.set_stream(stream)
    load_all(b, inputs)
    b.step(64)
    ev[0].record(stream)
    b.step(steps)
    ev[1].record(stream)
    ev[1].synchronize()
    fast = ev[0].elapsed_time(ev[1])
    b.close()
    e.close()
    # the FP64 build of the same kernels on the same rollout
    d = Engine([InstanceSpec(len(inputs[0][1]))] * M, path="plain", device=device, grad_fp64=True)
    d.set_stream(stream)
    times = []
    for _ in range(2):  # the first pass loads the FP64 kernels and allocates their buffers
        load_all(d, inputs)
        d.time = 0.0
        ev[0].record(stream)
        d.grad_forward(steps, checkpoint_every)
        ev[1].record(stream)
        d.grad_backward()
        ev[2].record(stream)
        ev[2].synchronize()
        times.append((ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])))
    d.close()
    fwd64, bwd64 = times[-1]
    return {"instances": M, "substeps": steps, "checkpoint_every": checkpoint_every,
            "fwd_ms": fwd, "bwd_ms": bwd, "fwd_bwd_over_fwd": (fwd + bwd) / fwd,
            "batched_fwd_ms": fast, "fwd_bwd_over_batched_fwd": (fwd + bwd) / fast,
            "fp64": {"fwd_ms": fwd64, "bwd_ms": bwd64, "fwd_bwd_over_fwd": (fwd64 + bwd64) / fwd64}}


def plain_leg(inputs, spec, device, stream, S, W, K, batched_value, live, points=4, P=50):
    """The plain per-instance launch path on the batched run's own trajectory.

    The batched value averages substeps W*S .. (W+K)*S of the trajectory from
    the loaded inputs.  A second batched engine replays that trajectory and
    stops at the middle of each of `points` equal parts of the window; each
    state is copied into a plain-path engine, which is timed for P substeps
    (after 5 untimed ones).  The plain rate is live particles x substeps over
    the summed time of all points, so batched_over_plain compares the two
    paths on the same stretch of the trajectory."""
    import torch
    from jellyfih_b200 import Engine
    M = len(inputs)
    replay = Engine([spec] * M, path="batched", device=device)
    replay.set_stream(stream)
    load_all(replay, inputs)
    replay.time = 0.0
    targets = [int(W * S + (i + 0.5) * K * S / points) for i in range(points)]
    done = 0
    rows = []
    total_ms = 0.0
    for target in targets:
        replay.step(target - done)
        done = target
        states = [replay.read(m) for m in range(M)]
        params, t_now = replay.get_params(), float(replay.time)
        plain = Engine([spec] * M, path="plain", device=device)
        plain.set_stream(stream)
        for m, st in enumerate(states):
            plain.load(m, st["x"], st["material"], st["fiber"])
            plain.write(m, v=st["v"], C=st["C"], F=st["F"], Jp=st["Jp"], glow=st["glow"])
        plain.set_params(**params)
        plain.time = t_now
        plain.step(5)
        plain.sync()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        plain.step(P)
        p1.record(stream)
        p1.synchronize()
        ms = p0.elapsed_time(p1)
        plain.close()
        total_ms += ms
        rows.append({"substep": target, "ms_per_substep": ms / P, "value": live * P / (ms / 1e3)})
    replay.close()
    value = live * P * points / (total_ms / 1e3)
    return {"value": value, "unit": UNIT, "batched_over_plain": batched_value / value,
            "substeps_per_point": P, "points": rows,
            "window": f"substeps {W * S}..{(W + K) * S} of the trajectory from the loaded inputs "
                      "(the batched value's window)"}


def tank_leg(engine, M, seed=1000, workers=None):
    """One generation's tanks into the engine: host fill_tank + load (slot
    arrays built on the host and copied) against load_tank (robot on the
    host, water lattice, exclusion and slot layout on the GPU)."""
    from jellyfih_b200 import tank
    genomes = tank.gaussian_genomes(M, seed)
    t0 = time.perf_counter()
    for m, g in enumerate(genomes):
        pos, mat, fib, _ = tank.fill_tank(g, engine.instances[m].n_slots)
        engine.load(m, pos, mat, fib)
    engine.sync()
    host_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    for m, g in enumerate(genomes):
        tank.load_tank(engine, m, g)
    engine.sync()
    gpu_s = time.perf_counter() - t0
    workers = workers or os.cpu_count() or 1
    pool = tank.make_pool(workers)
    try:
        tank.load_tanks(engine, genomes, executor=pool)  # starts the workers
        t0 = time.perf_counter()
        tank.load_tanks(engine, genomes, executor=pool)
        engine.sync()
        pool_s = time.perf_counter() - t0
    finally:
        pool.shutdown()
    return {"instances": M, "host_fill_and_load_s": host_s, "gpu_fill_s": gpu_s,
            "gpu_fill_pooled_robots_s": pool_s, "workers": workers, "speedup": host_s / pool_s,
            "note": "per generation; load_tank generates the robot on the host, the water on the GPU; "
                    "the pooled run spreads the robots over spawned worker processes"}


def render_leg(engine, stream, M, cpu, frames=20, res=1024):
    """One headless frame per step of the reference's viewer pipeline
    (run_population.py:60-65 plus the vorticity views): clear, abyss splats of
    every particle (rainbow water, radius 1.5), vorticity overlay, tone map,
    vorticity grid, RdBu blend, on the engine's current state; device time
    with CUDA events.  ``cpu`` adds the CPU oracle rendering the same frame
    (one thread) and the frame read-back."""
    import torch
    from oracle import oracle as O
    gs = int(np.ceil(np.sqrt(M)))
    rs = res // gs
    hue = np.full(M, 0.55, np.float32)
    mhue = np.full(M, 0.70, np.float32)
    engine.frame_create(res)

    def frame():
        engine.frame_clear(0.0)
        engine.render_abyss(rs, gs, 1.5, hue, mhue, 2)
        engine.render_vorticity_overlay(rs, gs, 0.001)
        engine.tone_map()
        engine.compute_vorticity(0.003)
        engine.render_vorticity(rs, gs, 0.6, 0)

    for _ in range(3):
        frame()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    l0 = engine.kernel_launches
    ev[0].record(stream)
    for _ in range(frames):
        frame()
    ev[1].record(stream)
    launches = engine.kernel_launches - l0
    for _ in range(frames):
        engine.render_abyss(rs, gs, 1.5, hue, mhue, 2)
    ev[2].record(stream)
    ev[2].synchronize()
    ms = ev[0].elapsed_time(ev[1]) / frames
    abyss_ms = ev[1].elapsed_time(ev[2]) / frames
    live = sum(int((engine.read(m)["material"] >= 0).sum()) for m in range(M))
    # the web viewers' flat frame (payload_sink.py, view_*.py): white clear and
    # one single-colour splat pass per palette entry (mpm_sim.py WEB_PALETTE)
    palette = ((0, 0.933, 0.949, 0.957), (1, 0.678, 0.882, 0.875), (3, 0.976, 0.757, 0.765),
               (2, 0.961, 0.824, 0.576))
    flat_radius = max(1.0, rs / 128 * 0.6)

    def flat_frame():
        engine.frame_clear(1.0)
        for mat_id, r, g, b in palette:
            engine.render_flat(rs, gs, flat_radius, mat_id, r, g, b)

    for _ in range(3):
        flat_frame()
    ev[2].record(stream)
    for _ in range(frames):
        flat_frame()
    ev[3].record(stream)
    ev[3].synchronize()
    flat_ms = ev[2].elapsed_time(ev[3]) / frames
    out = {"ms_per_frame": ms, "frames_per_s": 1e3 / ms, "abyss_ms": abyss_ms, "flat_ms_per_frame": flat_ms,
           "splat_particles_per_s": live / (abyss_ms / 1e3), "video_res": res, "grid_side": gs,
           "res_sub": rs, "particles": live, "kernels_per_frame": launches / frames,
           "pipeline": "clear, abyss (rainbow water, radius 1.5), vorticity overlay, tone map, vorticity grid, rdbu"}
    frame()  # one clean frame (the abyss-only passes above accumulated)
    engine.sync()
    t0 = time.perf_counter()
    img = engine.read_frame()
    out["read_frame_ms"] = (time.perf_counter() - t0) * 1e3
    if cpu:
        st = [engine.read(m) for m in range(M)]
        grids = [engine.read_grid(m) for m in range(M)]
        prm = engine.get_params()
        sc = O.RenderScene([s["x"] for s in st], [s["v"] for s in st], [s["material"] for s in st],
                           [s["Jp"] for s in st], [g[0] for g in grids], [g[1] for g in grids], [1.0] * M,
                           prm["freq"], prm["contraction"], hue, mhue, engine.time)
        fb = O.new_frame(res)
        t0 = time.perf_counter()
        O.render_clear(fb, 0.0)
        O.render_abyss(fb, sc, rs, gs, 1.5, 2)
        O.render_vorticity_overlay(fb, sc, rs, gs, 0.001)
        O.render_tone_map(fb)
        vort = O.vorticity_grid(sc, 0.003)
        O.render_vorticity(fb, sc, vort, rs, gs, 0.6, 0)
        cpu_s = time.perf_counter() - t0
        out["cpu_baseline"] = {"ms_per_frame": cpu_s * 1e3, "cores": 1, "kind": "port",
                               "sample": "one frame of the same pipeline on the same state"}
        out["gpu_over_cpu"] = cpu_s * 1e3 / ms
        out["max_abs_diff_vs_oracle"] = float(np.max(np.abs(img - fb)))
    return out


def run_reference(args):
    """--impl reference: the CPU oracle (the reference's substep restated; Taichi
    is not installed) on the host cores, rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    # rank 0 runs alone, on every core this process may use: torchrun's default
    # OMP_NUM_THREADS=1 for its ranks is overridden (the oracle's OpenMP runtime
    # reads the variable when the library is loaded, below)
    cores = host_cores()
    os.environ["OMP_NUM_THREADS"] = str(cores)
    from oracle import oracle as O
    inputs = make_inputs(args.instances, args.slots, 1000)
    insts = [O.Instance(contraction=i[3], freq=i[4]) for i in inputs]
    states = [O.new_state(i[0], i[1], i[2]) for i in inputs]
    live = sum(int((i[1] >= 0).sum()) for i in inputs)
    # one untimed call first (page faults on the fresh states, the OpenMP
    # pool's start), then a probe of 8 substeps
    t = O.run_batch(insts, states, np.float32(0), 2)
    t0 = time.perf_counter()
    t = O.run_batch(insts, states, t, 8)
    probe = (time.perf_counter() - t0) / 8
    budget = 120.0  # seconds for warmup + timed steps
    per_step = max(1, int(budget / max(args.steps + args.warmup, 1) / max(probe, 1e-6)))
    per_step = min(per_step, args.substeps)
    for _ in range(args.warmup):
        t = O.run_batch(insts, states, t, per_step)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        t = O.run_batch(insts, states, t, per_step)
    el = time.perf_counter() - t0
    value = live * per_step * args.steps / el
    sample = (f"{args.instances} instances x {per_step} substeps per step (bounded sample of the "
              f"{args.substeps}-substep step)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": f"{args.instances} instances x {args.slots} slots, 128^2 grid, "
                                   "CPU oracle of the reference substep", "instances": args.instances,
                       "slots": args.slots, "live_particles": live, "substeps_per_step": per_step},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": int(os.environ["OMP_NUM_THREADS"]),
                             "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    import torch.distributed as dist

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    def allreduce(x, op):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=op)
        return float(t.item())

    from jellyfih_b200 import Engine, InstanceSpec
    M, S, K, W = args.instances, args.substeps, args.steps, args.warmup
    inputs = make_inputs(M, args.slots, 1000 + rank)
    live = sum(int((i[1] >= 0).sum()) for i in inputs)
    spec = InstanceSpec(args.slots)
    engine = Engine([spec] * M, path="batched", device=local, resort_interval=args.resort,
                    block_threads=args.block)
    stream = torch.cuda.Stream()
    engine.set_stream(stream)
    layout = engine.layout()
    load_all(engine, inputs)
    engine.time = 0.0

    for _ in range(W):
        engine.step(S)
    engine.sync()
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    engine.set_kernel_timing(True)
    engine.path_counts(reset=True)
    launches0 = engine.kernel_launches
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        for _ in range(K):
            engine.step(S)
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    kt = engine.kernel_timing()
    engine.set_kernel_timing(False)
    gpu_launches = engine.kernel_launches - launches0
    paths = engine.path_counts()
    flags = engine.error_flags()
    ms_max = allreduce(ms, dist.ReduceOp.MAX if world > 1 else None)
    live_total = allreduce(float(live), dist.ReduceOp.SUM if world > 1 else None)
    value = live_total * S * K / (ms_max / 1e3)

    # dominant kernel roofline: algorithmic bytes per chunk launch / mean launch time
    peak, peak_kind = peaks()
    chunk_substeps = S * K / max(kt["step_launches"], 1)
    bytes_per_launch = live * chunk_substeps * ALGO_BYTES
    mean_launch_s = kt["step_ms"] / max(kt["step_launches"], 1) / 1e3
    achieved = bytes_per_launch / mean_launch_s / 1e9
    tpps, trec = traffic_per_particle_step()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": (tpps * live * chunk_substeps) if tpps else None,
                "kernel": "chunk_kernel", "algorithmic_bytes_per_launch": bytes_per_launch,
                "mean_launch_ms": mean_launch_s * 1e3, "launches": kt["step_launches"],
                "step_kernel_share": kt["step_ms"] / ms if ms > 0 else None,
                "scatter_paths": paths,
                "sort_ms": kt["sort_ms"], "sort_launches": kt["sort_launches"]}
    if tpps is None and trec is not None:
        # the kernel changed since the ncu measurement: no traffic figure for this
        # source, but the last measured one, scaled to this launch, and the sources
        # it belongs to
        last = trec.get("chunk_kernel_dram_bytes_per_live_particle_substep")
        roofline["traffic_last_measured"] = {
            "bytes_per_launch": last * live * chunk_substeps if last else None,
            "kernel_sources_sha256_16": trec.get("kernel_sources_sha256_16"),
            "note": "ncu figure of an earlier revision of the chunk kernel's sources"}

    extras = {}
    if world > 1 and args.gpus != world:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE {world}")
    if not args.no_extras:
        # the same engine and state, (sort, chunk) pairs replayed from CUDA graphs
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(2):
            engine.step(S)
        e1.record(stream)
        e1.synchronize()
        gms = allreduce(e0.elapsed_time(e1), dist.ReduceOp.MAX if world > 1 else None)
        extras["graphs"] = {"value": live_total * 2 * S / (gms / 1e3), "unit": UNIT,
                            "steps": 2, "note": "two more bench steps, graphs replayed, kernel timing off"}

        # e2e through the public API: one evaluation episode per step (jf_run_episode:
        # every instance loaded from pinned host arrays, run_headless, GPU fitness,
        # (M, 5) rows and (M,) fitness read back)
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
        pos_all = pin(np.concatenate([i[0] for i in inputs]))
        mat_all = pin(np.concatenate([i[1] for i in inputs]))
        fib_all = pin(np.concatenate([i[2] for i in inputs]))
        con = np.array([i[3] for i in inputs], np.float32)
        frq = np.array([i[4] for i in inputs], np.float32)
        mus = np.array([i[5]["muscle_count"] for i in inputs], np.int32)
        h2d = pos_all.nbytes + mat_all.nbytes + fib_all.nbytes + con.nbytes + frq.nbytes + mus.nbytes
        e2e_steps = max(2, K // 4)
        # one untimed episode first: the call allocates its staging buffers once
        engine.run_episode(pos_all, mat_all, con, S, fibers=fib_all, freq=frq, muscle_counts=mus)
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            res, fit = engine.run_episode(pos_all, mat_all, con, S, fibers=fib_all, freq=frq, muscle_counts=mus)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        barrier()
        el = allreduce(el, dist.ReduceOp.MAX if world > 1 else None)
        extras["e2e"] = {"value": live_total * S * e2e_steps / el, "unit": UNIT,
                         "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": res.nbytes + fit.nbytes,
                         "steps": e2e_steps,
                         "api": "Engine.run_episode (jf_run_episode: loads, headless run, GPU fitness)"}
        if world > 1:
            from jellyfih_b200.shard import gather_rows
            extras["e2e"]["gathered_results"] = int(gather_rows(res).shape[0])

    if not args.no_extras and world == 1:
        # plain per-instance launch path (the batched / plain ratio), timed at
        # points inside the window of substeps the batched value averages over
        extras["plain"] = plain_leg(inputs, spec, local, stream, S, W, K, value, live)

        extras["differentiable"] = grad_leg(inputs[:8], local, stream, steps=args.grad_substeps,
                                            checkpoint_every=args.grad_checkpoint)
        if not args.no_refine:
            extras["refine"] = refine_leg(local, stream)

        if not args.no_uneven:
            extras["uneven"] = uneven_leg(local, stream)

        if not args.no_render:
            extras["render"] = render_leg(engine, stream, M, cpu=(rank == 0 and world == 1))

        # the host's cores are shared by the ranks of this node
        extras["tank"] = tank_leg(engine, M, workers=max(1, (os.cpu_count() or 1) // world))

        if rank == 0 and world == 1:
            extras["cpu_baseline"] = cpu_baseline(inputs)

    engine.close()
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
                "warmup": W, "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"batched {M} instances x {args.slots} slots per GPU, 128^2 grid, "
                                       f"FP32, {S} substeps per step",
                           "instances_per_gpu": M, "slots": args.slots, "live_particles": int(live_total),
                           "substeps_per_step": S, "resort_interval": args.resort,
                           "block_threads": layout["block_threads"], "cluster_size": layout["cluster_size"],
                           "l2": "inputs larger than L2: particle state plus sort buffers ~260 MB per GPU",
                           "path": "batched"},
                "roofline": roofline, "clocks": clocks.summary(), "gpu_launches": gpu_launches,
                "nonfinite_instances": int(np.count_nonzero(flags)),
                # allocated slots (live and dead) x substeps / time: the count the
                # reference's published per-generation rates use
                "value_slots": M * args.slots * world * S * K / (ms_max / 1e3),
                "fwd_bwd_over_fwd": extras.get("differentiable", {}).get("fwd_bwd_over_fwd")}
        line.update(extras)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_grad_only(args):
    import torch
    torch.cuda.set_device(0)
    inputs = make_inputs(args.instances, args.slots, 1000)
    stream = torch.cuda.Stream()
    out = {"differentiable": grad_leg(inputs[:8], 0, stream, steps=args.grad_substeps,
                                      checkpoint_every=args.grad_checkpoint)}
    if not args.no_refine:
        out["refine"] = refine_leg(0, stream)
    print(json.dumps(out), flush=True)
    return 0


def run_render_only(args):
    import torch
    torch.cuda.set_device(0)
    from jellyfih_b200 import Engine, InstanceSpec
    inputs = make_inputs(args.instances, args.slots, 1000)
    # the viewers step with the render-only glow on (JELLY_B200_GLOW=1)
    engine = Engine([InstanceSpec(args.slots)] * args.instances, path="batched", device=0, glow=True)
    stream = torch.cuda.Stream()
    engine.set_stream(stream)
    load_all(engine, inputs)
    engine.step(args.substeps)
    engine.sync()
    out = {"render": render_leg(engine, stream, args.instances, cpu=True), "substeps_before": args.substeps,
           "glow": True}
    engine.close()
    print(json.dumps(out), flush=True)
    return 0


def run_tank_only(args):
    import torch
    torch.cuda.set_device(0)
    from jellyfih_b200 import Engine, InstanceSpec
    engine = Engine([InstanceSpec(args.slots)] * args.instances, path="batched", device=0)
    out = {"tank": tank_leg(engine, args.instances)}
    engine.close()
    print(json.dumps(out), flush=True)
    return 0


def run_plain_only(args, P=50):
    import torch
    torch.cuda.set_device(0)
    from jellyfih_b200 import Engine, InstanceSpec
    inputs = make_inputs(args.instances, args.slots, 1000)
    live = sum(int((i[1] >= 0).sum()) for i in inputs)
    stream = torch.cuda.Stream()
    plain = Engine([InstanceSpec(args.slots)] * args.instances, path="plain", device=0)
    plain.set_stream(stream)
    load_all(plain, inputs)
    plain.step(5)
    plain.sync()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    plain.step(P)
    ev1.record(stream)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    plain.close()
    print(json.dumps({"plain": {"value": live * P / (ms / 1e3), "unit": UNIT, "substeps": P,
                                "ms_per_substep": ms / P, "state": "from the loaded inputs"}}), flush=True)
    return 0


def run_episode_only(args):
    """jf_run_episode alone: every instance loaded from pinned host arrays, a
    headless run of --substeps, GPU fitness, rows and fitness read back."""
    import torch
    torch.cuda.set_device(0)
    from jellyfih_b200 import Engine, InstanceSpec
    inputs = make_inputs(args.instances, args.slots, 1000)
    live = sum(int((i[1] >= 0).sum()) for i in inputs)
    engine = Engine([InstanceSpec(args.slots)] * args.instances, path="batched", device=0)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    pos_all = pin(np.concatenate([i[0] for i in inputs]))
    mat_all = pin(np.concatenate([i[1] for i in inputs]))
    fib_all = pin(np.concatenate([i[2] for i in inputs]))
    con = np.array([i[3] for i in inputs], np.float32)
    frq = np.array([i[4] for i in inputs], np.float32)
    mus = np.array([i[5]["muscle_count"] for i in inputs], np.int32)
    run = lambda: engine.run_episode(pos_all, mat_all, con, args.substeps, fibers=fib_all, freq=frq,  # noqa: E731
                                     muscle_counts=mus)
    run()  # allocates the call's staging buffers
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        res, fit = run()
    el = time.perf_counter() - t0
    engine.close()
    print(json.dumps({"episode": {"value": live * args.substeps * args.steps / el, "unit": UNIT,
                                  "episodes": args.steps, "substeps": args.substeps,
                                  "valid": int(res[:, 4].sum())}}), flush=True)
    return 0


def run_noalloc_only(args):
    """jf_substep_noalloc alone: one instance of the workload on caller-owned
    device arrays (the engine's state after 300 substeps), --substeps calls,
    CUDA events around them."""
    import torch
    torch.cuda.set_device(0)
    from jellyfih_b200 import Engine, InstanceSpec, _lib
    pos, mat, fib, c, f, st = make_inputs(1, args.slots, 1000)[0]
    live = int((mat >= 0).sum())
    eng = Engine([InstanceSpec(args.slots)], path="plain", device=0)
    eng.load(0, pos, mat, fib)
    eng.set_params(contraction=[c], freq=[f])
    eng.time = 0.0
    eng.step(300)
    s0 = eng.read(0)
    t = eng.time
    eng.close()
    dev = torch.device("cuda", 0)
    fields = ("x", "v", "C", "F", "material", "Jp", "glow", "fiber")
    bufs = {k: torch.from_numpy(np.ascontiguousarray(s0[k])).to(dev) for k in fields}
    ptrs = [bufs[k].data_ptr() for k in fields]
    lib = _lib.load()
    stream = torch.cuda.current_stream(dev)
    dt = np.float32(2e-5)

    def call(t):
        rc = lib.jf_substep_noalloc(args.slots, 128, 128, 1.0, float(dt), float(t), 500.0, float(c), float(f),
                                    2.5, *ptrs, stream.cuda_stream)
        if rc != 0:
            raise RuntimeError(lib.jf_last_error(None).decode())
        return np.float32(t + dt)

    for _ in range(5):
        t = call(t)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.substeps):
        t = call(t)
    ev1.record(stream)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    print(json.dumps({"noalloc": {"value": live * args.substeps / (ms / 1e3), "unit": UNIT,
                                  "substeps": args.substeps, "us_per_substep": ms / args.substeps * 1e3,
                                  "live_particles": live}}), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU (RANK / LOCAL_RANK / WORLD_SIZE / MASTER_* set per
        # rank); under torchrun the ranks already exist
        from jellyfih_b200.launch import spawn_ranks
        return spawn_ranks(args.gpus, os.path.abspath(__file__), sys.argv[1:])
    if args.grad_only:
        return run_grad_only(args)
    if args.render_only:
        return run_render_only(args)
    if args.tank_only:
        return run_tank_only(args)
    if args.plain_only:
        return run_plain_only(args)
    if args.episode_only:
        return run_episode_only(args)
    if args.noalloc_only:
        return run_noalloc_only(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
