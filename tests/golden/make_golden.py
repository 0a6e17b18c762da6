"""Generate golden fixtures by executing the reference's own mpm_sim.py.

Usage (needs the reference checkout, so it runs only where that exists):

    python tests/golden/make_golden.py --reference <path of a reference checkout>

Each case runs in a fresh subprocess because mpm_sim.py reads its JELLY_* env
vars and allocates its fields at import (mpm_sim.py:11-17,86-142).  The
reference imports ``taichi``, which is absent here; tests/golden/taichi_standin
supplies a numpy stand-in of the Taichi runtime (see its docstring), so the
reference kernels substep(), compute_payload_stats(), get_payload_stats(),
_get_stats_any() and run_batch_headless() execute unmodified as Python.

Fixtures (``<case>.npz``) hold the inputs written into the reference's fields
and the fields read back after the listed step counts.  Grids are stored
sparsely (flat indices of nodes with nonzero mass).
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
    # name: (env, builder)
    "perturbed_1inst": {"JELLY_INSTANCES": "1", "JELLY_PARTICLES": "4608"},
    "walls_2inst": {"JELLY_INSTANCES": "2", "JELLY_PARTICLES": "1024"},
    "tall_1inst": {"JELLY_INSTANCES": "1", "JELLY_PARTICLES": "1536", "JELLY_GRID_Y": "256",
                   "JELLY_DOMAIN_H": "2.0"},
    "headless_3inst": {"JELLY_INSTANCES": "3", "JELLY_PARTICLES": "2560"},
    # axisymmetric (r, z) substep, JELLY_AXISYM=1 (mpm_sim.py:17,163-165,235-268,292-303)
    "axisym_1inst": {"JELLY_INSTANCES": "1", "JELLY_PARTICLES": "3072", "JELLY_AXISYM": "1"},
    "axisym_tall_2inst": {"JELLY_INSTANCES": "2", "JELLY_PARTICLES": "1536", "JELLY_GRID_Y": "256",
                          "JELLY_DOMAIN_H": "2.0", "JELLY_AXISYM": "1"},
}


def _robot_window(genome, n_slots, window, rng, with_payload=True, spawn=None):
    """Robot particles plus the water lattice inside ``window``, padded to n_slots."""
    sys.path.insert(0, REPO)
    from scipy.spatial import cKDTree
    from jellyfih_b200 import tank
    rpos, rmat, rfib, _ = tank.generate_phenotype(genome, spawn, 128, with_payload)
    sp = 1.0 / 256
    wx = np.arange(window[0], window[1], sp)
    wy = np.arange(window[2], window[3], sp)
    g = np.stack(np.meshgrid(wx, wy), -1).reshape(-1, 2)
    if len(rpos):
        d, _ = cKDTree(rpos).query(g)
        g = g[d > 0.005]
    pos = np.full((n_slots, 2), -1.0, np.float32)
    mat = np.full(n_slots, -1, np.int32)
    fib = np.zeros((n_slots, 2), np.float32)
    fib[:, 1] = 1
    nr = min(len(rpos), n_slots)
    pos[:nr] = rpos[:nr]
    mat[:nr] = rmat[:nr]
    fib[:nr] = rfib[:nr]
    nw = min(len(g), n_slots - nr)
    pos[nr:nr + nw] = g[:nw]
    mat[nr:nr + nw] = 0
    # interleave some dead slots inside the live range
    live = nr + nw
    dead = rng.choice(live, size=max(1, live // 50), replace=False)
    mat[dead] = -1
    pos[dead] = -1.0
    return pos, mat, fib


def _perturb(pos, mat, rng, inverted_frac=0.02, vel=0.05):
    n = len(mat)
    v = rng.normal(0, vel, (n, 2)).astype(np.float32)
    C = rng.normal(0, 2.0, (n, 2, 2)).astype(np.float32)
    F = (np.eye(2) + rng.normal(0, 0.02, (n, 2, 2))).astype(np.float32)
    # a few inverted deformation gradients (det F < 0) pin the SVD convention
    inv = rng.random(n) < inverted_frac
    F[inv, 1, :] *= -1
    # a few rotations with shear
    rot = rng.random(n) < 0.05
    th = rng.uniform(-0.5, 0.5, rot.sum())
    R = np.stack([np.stack([np.cos(th), -np.sin(th)], -1), np.stack([np.sin(th), np.cos(th)], -1)], -2)
    F[rot] = (R @ F[rot].astype(np.float64)).astype(np.float32)
    Jp = rng.uniform(0.9, 1.1, n).astype(np.float32)
    glow = rng.uniform(0.0, 0.2, n).astype(np.float32)
    dead = mat < 0
    v[dead] = 0
    C[dead] = 0
    F[dead] = np.eye(2, dtype=np.float32)
    return v, C, F, Jp, glow


def _axisym_instance(n, rng, y_hi):
    """Particles crowded near the axis (0.01 < r < 0.06) plus a uniform spread;
    the load positions set r_ref (mpm_sim.py:727) and the positions written
    after the load differ radially, so the hoop stretch r / r_ref is not 1.
    The reference's axisymmetric P2G divides the unweighted stress force by
    the r-weighted mass, which scales stress near the axis by ~1/r (a 1e-3
    deformation of payload at r = 0.01 already gives |v| ~ 100 after one
    substep), so particles at r < 0.2 start stress-free (F = I, C = 0, no
    muscle) and the deformation, inverted and rotated F, muscle and radial
    moves (hoop stretch) stay at r > 0.2.  A few stress-free water particles
    have load radii below the dx/10 floor or positions below dx/20."""
    pos = np.empty((n, 2), np.float32)
    near = rng.random(n) < 0.4
    pos[:, 0] = np.where(near, rng.uniform(0.01, 0.06, n), rng.uniform(0.001, 0.999, n))
    pos[:, 1] = rng.uniform(0.001, y_hi, n)
    strip = rng.random(n) < 0.03
    pos[strip, 0] = rng.uniform(126.0 / 128, 0.999, strip.sum())
    mat = rng.choice([0, 0, 0, 1, 2, 3, 4], n).astype(np.int32)
    far = pos[:, 0] > 0.2
    mat[~far & (mat == 3)] = 1
    x_now = pos.copy()
    x_now[far, 0] = np.clip(pos[far, 0] * rng.uniform(0.95, 1.05, far.sum()), 0.001, 0.999)
    v = rng.normal(0, 0.05, (n, 2)).astype(np.float32)
    C = rng.normal(0, 0.05, (n, 2, 2)).astype(np.float32)
    F = (np.eye(2) + rng.normal(0, 0.001, (n, 2, 2))).astype(np.float32)
    F[(mat == 0) | ~far] = np.eye(2, dtype=np.float32)
    C[~far] = 0
    inv = far & (rng.random(n) < 0.03)
    F[inv, 1, :] *= -1
    rot = far & (rng.random(n) < 0.05)
    th = rng.uniform(-0.5, 0.5, rot.sum())
    R = np.stack([np.stack([np.cos(th), -np.sin(th)], -1), np.stack([np.sin(th), np.cos(th)], -1)], -2)
    F[rot] = (R @ F[rot].astype(np.float64)).astype(np.float32)
    edge = rng.random(n) < 0.04
    tiny_ref = edge & (rng.random(n) < 0.5)
    tiny_x = edge & ~tiny_ref
    pos[tiny_ref, 0] = rng.uniform(0.0001, 0.0007, tiny_ref.sum())
    x_now[tiny_ref, 0] = rng.uniform(0.003, 0.01, tiny_ref.sum())
    x_now[tiny_x, 0] = rng.uniform(0.0001, 0.0003, tiny_x.sum())
    mat[edge] = 0
    F[edge] = np.eye(2, dtype=np.float32)
    C[edge] = 0
    dead = rng.random(n) < 0.03
    mat[dead] = -1
    pos[dead] = -1
    x_now[dead] = -1
    v[dead] = 0
    C[dead] = 0
    F[dead] = np.eye(2, dtype=np.float32)
    Jp = rng.uniform(0.9, 1.1, n).astype(np.float32)
    glow = rng.uniform(0.0, 0.2, n).astype(np.float32)
    fib = rng.normal(size=(n, 2)).astype(np.float32)
    fib /= np.linalg.norm(fib, axis=1, keepdims=True)
    return dict(pos=pos, x_now=x_now.astype(np.float32), mat=mat, fib=fib, v=v, C=C, F=F, Jp=Jp, glow=glow)


def _inputs(case, rng):
    sys.path.insert(0, REPO)
    from jellyfih_b200 import tank
    if case == "axisym_1inst":
        params = dict(actuation=[900.0], contraction=[0.4], freq=[1.3], payload_density=[2.5])
        # one substep: near the axis these states grow several-fold per substep, which
        # amplifies summation-order noise in later ones
        return [_axisym_instance(3072, rng, 0.999)], params, 0.21, [1]
    if case == "axisym_tall_2inst":
        params = dict(actuation=[500.0, 1100.0], contraction=[0.25, 0.5], freq=[1.0, 0.7],
                      payload_density=[2.5, 3.5])
        return [_axisym_instance(1536, rng, 1.999) for _ in range(2)], params, 0.03, [1]
    if case == "perturbed_1inst":
        genome = np.concatenate([tank.AURELIA_GENOME, [0.2, 1.0]])
        pos, mat, fib = _robot_window(genome, 4608, (0.40, 0.60, 0.33, 0.47), rng)
        v, C, F, Jp, glow = _perturb(pos, mat, rng)
        params = dict(actuation=[500.0], contraction=[0.2], freq=[1.0], payload_density=[2.5])
        return [dict(pos=pos, mat=mat, fib=fib, v=v, C=C, F=F, Jp=Jp, glow=glow)], params, 0.1, [1, 5]
    if case == "walls_2inst":
        insts = []
        for k in range(2):
            n = 1024
            pos = np.empty((n, 2), np.float32)
            # bands along each wall, corners, the x >= 126.5/128 skip strip, interior
            b = rng.integers(0, 6, n)
            u = rng.uniform(0.001, 0.999, n)
            e = rng.uniform(0.001, 0.035, n)
            pos[:, 0] = np.where(b == 0, e, np.where(b == 1, 1 - e, u))
            pos[:, 1] = np.where(b == 2, e, np.where(b == 3, 1 - e, u))
            corner = b == 4
            pos[corner, 0] = np.where(rng.random(corner.sum()) < 0.5, e[corner], 1 - e[corner])
            pos[corner, 1] = np.where(rng.random(corner.sum()) < 0.5, e[corner][::-1], 1 - e[corner][::-1])
            strip = b == 5
            pos[strip, 0] = rng.uniform(126.0 / 128, 0.999, strip.sum())
            pos = np.clip(pos, 0.001, 0.999).astype(np.float32)
            mat = rng.choice([0, 0, 0, 1, 2, 3, 4], n).astype(np.int32)
            dead = rng.random(n) < 0.05
            mat[dead] = -1
            pos[dead] = -1
            fib = rng.normal(size=(n, 2)).astype(np.float32)
            fib /= np.linalg.norm(fib, axis=1, keepdims=True)
            v, C, F, Jp, glow = _perturb(pos, mat, rng, vel=0.5)
            # velocities pointing into the nearest wall exercise the wall clamps
            v[:, 0] += np.where(pos[:, 0] < 0.5, -1.0, 1.0).astype(np.float32)
            v[:, 1] += np.where(pos[:, 1] < 0.5, -1.0, 1.0).astype(np.float32)
            v[dead] = 0
            insts.append(dict(pos=pos, mat=mat, fib=fib, v=v, C=C, F=F, Jp=Jp, glow=glow))
        params = dict(actuation=[500.0, 1200.0], contraction=[0.45, 0.1], freq=[1.0, 1.7],
                      payload_density=[2.5, 4.0])
        return insts, params, 0.37, [1, 3]
    if case == "tall_1inst":
        n = 1536
        pos = np.empty((n, 2), np.float32)
        pos[:, 0] = rng.uniform(0.001, 0.999, n)
        pos[:, 1] = np.concatenate([rng.uniform(0.001, 0.12, n // 4), rng.uniform(1.88, 1.999, n // 4),
                                    rng.uniform(0.001, 1.999, n - 2 * (n // 4))])
        mat = rng.choice([0, 0, 1, 2, 3], n).astype(np.int32)
        mat[rng.random(n) < 0.03] = -1
        pos[mat < 0] = -1
        fib = rng.normal(size=(n, 2)).astype(np.float32)
        fib /= np.linalg.norm(fib, axis=1, keepdims=True)
        v, C, F, Jp, glow = _perturb(pos, mat, rng, vel=0.3)
        params = dict(actuation=[800.0], contraction=[0.3], freq=[0.8], payload_density=[3.0])
        return [dict(pos=pos, mat=mat, fib=fib, v=v, C=C, F=F, Jp=Jp, glow=glow)], params, 0.05, [1, 2]
    if case == "headless_3inst":
        genome = np.concatenate([tank.AURELIA_GENOME, [0.3, 1.2]])
        insts = []
        for k in range(3):
            if k == 1:
                pos, mat, fib = _robot_window(genome, 2560, (0.42, 0.58, 0.38, 0.45), rng,
                                              with_payload=False)
            elif k == 2:
                pos, mat, fib = _robot_window(genome, 2560, (0.42, 0.58, 0.38, 0.45), rng,
                                              spawn=np.array([0.5, 0.31]))
                pay = mat == 2
                # payload squashed onto the floor: CoM y < 0.01 marks the run invalid
                pos[pay, 1] = (0.002 + (pos[pay, 1] - 0.31) * 0.1).astype(np.float32)
            else:
                pos, mat, fib = _robot_window(genome, 2560, (0.42, 0.58, 0.38, 0.45), rng)
            insts.append(dict(pos=pos, mat=mat, fib=fib))
        params = dict(actuation=[500.0, 700.0, 500.0], contraction=[0.3, 0.3, 0.3],
                      freq=[1.2, 1.2, 1.2], payload_density=[2.5, 2.5, 2.5])
        return insts, params, 0.0, [3]
    raise KeyError(case)


def _run_case(case, reference):
    sys.path.insert(0, os.path.join(HERE, "taichi_standin"))
    sys.path.insert(0, reference)
    import mpm_sim as sim  # the reference module, under the stand-in runtime
    rng = np.random.default_rng(sum(map(ord, case)))
    insts, params, t0, checkpoints = _inputs(case, rng)
    out = {"t0": np.float32(t0), "checkpoints": np.array(checkpoints, np.int32),
           "n_grid": np.int32(sim.n_grid), "n_grid_y": np.int32(sim.n_grid_y),
           "domain_height": np.float64(sim.domain_height), "dt": np.float64(sim.dt),
           "axisym": np.int32(1 if sim.axisym else 0)}
    for k, vals in params.items():
        out[f"param_{k}"] = np.array(vals, np.float32)
    for m, d in enumerate(insts):
        sim.load_particles(m, d["pos"], d["mat"], d["fib"])
        out[f"in{m}_x"] = d["pos"]
        if "x_now" in d:
            # positions moved after the load: r_ref keeps the load radius
            sim.x.data[m] = d["x_now"]
            out[f"in{m}_x_load"] = d["pos"]
            out[f"in{m}_x"] = d["x_now"]
        out[f"in{m}_material"] = d["mat"]
        out[f"in{m}_fiber"] = d["fib"]
        if "v" in d:
            sim.v.data[m] = d["v"]
            sim.C.data[m] = d["C"]
            sim.F.data[m] = d["F"]
            sim.Jp.data[m] = d["Jp"]
            sim.visual_glow.data[m] = d["glow"]
        for key, field in (("v", sim.v), ("C", sim.C), ("F", sim.F), ("Jp", sim.Jp),
                           ("glow", sim.visual_glow)):
            out[f"in{m}_{key}"] = field.to_numpy()[m]
    for m in range(len(insts)):
        sim.instance_actuation[m] = params["actuation"][m]
        sim.instance_act_contraction[m] = params["contraction"][m]
        sim.instance_freq[m] = params["freq"][m]
        sim.instance_payload_density[m] = params["payload_density"][m]

    if case == "headless_3inst":
        out["payload_stats_before"] = sim.get_payload_stats()
        out["stats_any_before"] = sim._get_stats_any()
        out["headless"] = sim.run_batch_headless(int(checkpoints[-1]))
        out["payload_stats_after"] = sim.get_payload_stats()
        out["time_after"] = np.float32(sim.sim_time[None])
        for m in range(len(insts)):
            out[f"s{checkpoints[-1]}_{m}_x"] = sim.x.to_numpy()[m]
    else:
        sim.sim_time[None] = t0
        done = 0
        for cp in checkpoints:
            while done < cp:
                sim.substep()
                done += 1
            out[f"time_{cp}"] = np.float32(sim.sim_time[None])
            for m in range(len(insts)):
                for key, field in (("x", sim.x), ("v", sim.v), ("C", sim.C), ("F", sim.F),
                                   ("Jp", sim.Jp), ("glow", sim.visual_glow)):
                    out[f"s{cp}_{m}_{key}"] = field.to_numpy()[m]
                gm = sim.grid_m.to_numpy()[m]
                gv = sim.grid_v.to_numpy()[m]
                nz = np.flatnonzero(gm.reshape(-1) != 0).astype(np.int32)
                out[f"s{cp}_{m}_grid_idx"] = nz
                out[f"s{cp}_{m}_grid_m"] = gm.reshape(-1)[nz]
                out[f"s{cp}_{m}_grid_v"] = gv.reshape(-1, 2)[nz]
                out[f"s{cp}_{m}_grid_v_nonzero_outside"] = np.int32(
                    np.count_nonzero(np.delete(gv.reshape(-1, 2), nz, axis=0)))
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
    for case, env in CASES.items():
        e = dict(os.environ)
        e.update(env)
        subprocess.run([sys.executable, os.path.abspath(__file__), "--reference", args.reference,
                        "--case", case], check=True, env=e)


if __name__ == "__main__":
    main()
