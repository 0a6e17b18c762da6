"""Generate renderer golden fixtures by executing the reference's own renderer.

Usage (needs the reference checkout, so it runs only where that exists):

    python tests/golden/make_render_golden.py --reference <path of a reference checkout>

The reference's render kernels (mpm_sim.py:343-712: clear_frame_buffer,
render_frame_abyss, tone_map_and_encode, clear_frame_buffer_white,
render_flat_pass, render_vorticity_overlay, compute_vorticity_grid,
render_vorticity_rdbu / _hueshift / _white) run unmodified under the numpy
stand-in of the Taichi runtime (tests/golden/taichi_standin), in a fresh
subprocess per case because mpm_sim.py reads JELLY_* at import.  Two module
attributes are replaced before rendering, the kernels' code is not:
``video_res`` and ``frame_buffer`` (a smaller frame, so that the fixtures
stay small; the kernels read both as module globals at call time).

Each fixture (``render_<case>.npz``) holds the state written into the
reference's fields (x, v, material, Jp, grid_v, grid_m, the per-instance
waveform parameters and hues, sim_time) and every frame / vorticity grid read
back after the listed call sequences.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))

CASES = {
    # name: (env, video_res, splat radius of the abyss pass, radius of the flat passes)
    "render_2inst": ({"JELLY_INSTANCES": "2", "JELLY_PARTICLES": "2048"}, 100, 1.5, 1.0),
    "render_3inst": ({"JELLY_INSTANCES": "3", "JELLY_PARTICLES": "768"}, 90, 1.0, 1.0),
    "render_tall": ({"JELLY_INSTANCES": "1", "JELLY_PARTICLES": "1536", "JELLY_GRID_Y": "256",
                     "JELLY_DOMAIN_H": "2.0"}, 64, 3.0, 3.0),
}


def _particles(sim, m, rng):
    """A subsampled robot (jelly, muscle, payload) in water, then the
    render-relevant perturbations: fast and near-still water (around the
    vel > 0.02 threshold), a Jp spread, an unknown material id, dead slots
    and live slots parked at x < 0."""
    sys.path.insert(0, REPO)
    from jellyfih_b200 import tank
    n = sim.n_particles
    dh = float(sim.domain_height)
    genome = np.concatenate([tank.AURELIA_GENOME, [0.3, 1.2]])
    rpos, rmat, rfib, _ = tank.generate_phenotype(genome, np.array([0.45 + 0.05 * m, 0.4 * dh]), 128, True)
    keep = rng.random(len(rpos)) < (0.4 * n) / len(rpos)
    rpos, rmat, rfib = rpos[keep], rmat[keep], rfib[keep]
    nw = int(0.95 * n) - len(rpos)
    wpos = np.stack([rng.uniform(0.02, 0.98, nw), rng.uniform(0.02, 0.98 * dh, nw)], -1)
    pos = np.full((n, 2), -1.0, np.float32)
    mat = np.full(n, -1, np.int32)
    fib = np.zeros((n, 2), np.float32)
    fib[:, 1] = 1
    order = rng.permutation(len(rpos) + nw)
    allpos = np.concatenate([rpos, wpos]).astype(np.float32)
    allmat = np.concatenate([rmat, np.zeros(nw, np.int32)]).astype(np.int32)
    allfib = np.concatenate([rfib, np.tile([0.0, 1.0], (nw, 1))]).astype(np.float32)
    pos[:len(order)] = allpos[order]
    mat[:len(order)] = allmat[order]
    fib[:len(order)] = allfib[order]
    live = np.flatnonzero(mat >= 0)
    v = np.round(rng.normal(0, 0.8, (n, 2)) * 1024) / 1024
    still = rng.random(n) < 0.2
    v[still] = np.round(rng.normal(0, 0.008, (still.sum(), 2)) * 4096) / 4096
    v = v.astype(np.float32)
    Jp = (np.round(rng.uniform(0.8, 1.2, n) * 1024) / 1024).astype(np.float32)
    unknown = rng.choice(live, size=max(1, len(live) // 100), replace=False)
    mat[unknown] = 4
    parked = rng.choice(np.flatnonzero(mat >= 0), size=max(1, len(live) // 100), replace=False)
    pos[parked] = (-0.25, 0.5)
    return pos, mat, fib, v, Jp


def _grid(sim, rng):
    """A smooth field of a few Gaussian vortices (curl up to ~1e3, so that the
    overlay and tanh mappings cover below-threshold, graded and saturated
    cells) on a mass mask with empty nodes."""
    nx, ny = sim.n_grid, sim.n_grid_y
    dh = float(sim.domain_height)
    xi = (np.arange(nx) + 0.0) / nx
    yj = (np.arange(ny) + 0.0) / nx
    X, Y = np.meshgrid(xi, yj, indexing="ij")
    vx = np.zeros((nx, ny))
    vy = np.zeros((nx, ny))
    for _ in range(3):
        cx, cy = rng.uniform(0.2, 0.8), rng.uniform(0.2, 0.8) * dh
        gam = rng.uniform(-600, 600)
        sig = rng.uniform(0.06, 0.12)
        dxp, dyp = X - cx, Y - cy
        e = np.exp(-(dxp * dxp + dyp * dyp) / (sig * sig))
        vx += -gam * dyp * e
        vy += gam * dxp * e
    vx += rng.normal(0, 0.05, vx.shape)
    vy += rng.normal(0, 0.05, vy.shape)
    # values on coarse lattices (velocity in 1/64 steps, three mass levels)
    # keep the fixtures compressible
    gm = rng.choice([0.5e-5, 1e-5, 2e-5], (nx, ny))
    gm[rng.random((nx, ny)) < 0.15] = 0.0
    gm[:, int(0.9 * ny):] = 0.0
    gv = (np.round(np.stack([vx, vy], -1) * 64) / 64).astype(np.float32)
    gv[gm == 0] = 0.0
    return gv, gm.astype(np.float32)


def _run_case(case, reference):
    env, video_res, radius, flat_radius = CASES[case]
    sys.path.insert(0, os.path.join(HERE, "taichi_standin"))
    sys.path.insert(0, reference)
    import mpm_sim as sim  # the reference module, under the stand-in runtime
    import taichi as ti
    rng = np.random.default_rng(sum(map(ord, case)))
    M = sim.n_instances
    sim.video_res = video_res
    sim.frame_buffer = ti.field(dtype=float, shape=(video_res, video_res, 3))
    grid_side = int(np.ceil(np.sqrt(M)))
    res_sub = video_res // grid_side
    out = {"video_res": np.int32(video_res), "grid_side": np.int32(grid_side), "res_sub": np.int32(res_sub),
           "radius": np.float32(radius), "flat_radius": np.float32(flat_radius),
           "n_grid": np.int32(sim.n_grid), "n_grid_y": np.int32(sim.n_grid_y),
           "domain_height": np.float64(sim.domain_height)}
    freq = rng.uniform(0.8, 1.6, M).astype(np.float32)
    contraction = rng.uniform(0.2, 0.4, M).astype(np.float32)
    hue = rng.uniform(0.0, 1.0, M).astype(np.float32)
    mhue = ((hue + 0.15) % 1.0).astype(np.float32)
    if M == 3:
        # hues outside [0, 1) reach hsv2rgb's int() truncation and Python-style %
        hue = np.array([-0.3, 1.25, 0.5], np.float32)
        mhue = np.array([0.4, -1.1, 2.7], np.float32)
    t = np.float32(0.05)
    for m in range(M):
        pos, mat, fib, v, Jp = _particles(sim, m, rng)
        sim.load_particles(m, pos, mat, fib)
        sim.v.data[m] = v
        sim.Jp.data[m] = Jp
        gv, gm = _grid(sim, rng)
        sim.grid_v.data[m] = gv
        sim.grid_m.data[m] = gm
        sim.instance_freq[m] = freq[m]
        sim.instance_act_contraction[m] = contraction[m]
        sim.instance_hue[m] = hue[m]
        sim.instance_muscle_hue[m] = mhue[m]
        out[f"in{m}_x"] = sim.x.to_numpy()[m]
        out[f"in{m}_material"] = sim.material.to_numpy()[m]
        out[f"in{m}_fiber"] = fib
        out[f"in{m}_v"] = sim.v.to_numpy()[m]
        out[f"in{m}_Jp"] = sim.Jp.to_numpy()[m]
        out[f"in{m}_grid_v"] = sim.grid_v.to_numpy()[m]
        out[f"in{m}_grid_m"] = sim.grid_m.to_numpy()[m]
    sim.sim_time[None] = t
    out.update(time=t, param_freq=freq, param_contraction=contraction, hue=hue, muscle_hue=mhue)

    r32 = np.float32(radius)
    frame = lambda: sim.frame_buffer.to_numpy()  # noqa: E731
    for mode in (0, 1, 2):
        sim.clear_frame_buffer()
        sim.water_angle_color[None] = mode
        sim.render_frame_abyss(res_sub, grid_side, r32)
        out[f"abyss_w{mode}"] = frame()
    sim.tone_map_and_encode()
    out["abyss_w2_tm"] = frame()

    sim.clear_frame_buffer()
    sim.render_frame_abyss(res_sub, grid_side, r32)
    sim.render_vorticity_overlay(res_sub, grid_side, np.float32(0.001))
    out["overlay_hdr"] = frame()
    sim.tone_map_and_encode()
    out["overlay_tm"] = frame()

    sim.compute_vorticity_grid(np.float32(0.003))
    out["vort"] = sim.vort_grid.to_numpy()

    sim.clear_frame_buffer()
    sim.water_angle_color[None] = 0
    sim.render_frame_abyss(res_sub, grid_side, r32)
    sim.tone_map_and_encode()
    sim.render_vorticity_rdbu(res_sub, grid_side, np.float32(0.6))
    out["rdbu"] = frame()

    sim.clear_frame_buffer()
    sim.water_angle_color[None] = 1
    sim.render_frame_abyss(res_sub, grid_side, r32)
    sim.tone_map_and_encode()
    sim.render_vorticity_hueshift(res_sub, grid_side, np.float32(0.5))
    out["hueshift"] = frame()

    sim.render_vorticity_white(res_sub, grid_side, np.float32(0.65))
    out["white"] = frame()

    sim.clear_frame_buffer_white()
    for mat_id, r, g, b in sim.WEB_PALETTE:
        sim.render_flat_pass(res_sub, grid_side, np.float32(flat_radius), mat_id,
                             np.float32(r), np.float32(g), np.float32(b))
    out["web"] = frame()
    np.savez_compressed(os.path.join(HERE, f"{case}.npz"), **out)
    print(f"{case}: wrote {len(out)} arrays")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("JELLYFIH_REFERENCE"),
                    required="JELLYFIH_REFERENCE" not in os.environ,
                    help="checkout of the reference (or set JELLYFIH_REFERENCE)")
    ap.add_argument("--case", default=None)
    args = ap.parse_args()
    if args.case:
        _run_case(args.case, args.reference)
        return
    for case, (env, *_rest) in CASES.items():
        e = dict(os.environ)
        e.update(env)
        subprocess.run([sys.executable, os.path.abspath(__file__), "--reference", args.reference,
                        "--case", case], check=True, env=e)


if __name__ == "__main__":
    main()
