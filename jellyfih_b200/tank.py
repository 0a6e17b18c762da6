"""Particle-set generator: genome -> jellyfish phenotype -> filled tank.

This is the caller-side input generator that feeds the engine.  It restates
make_jelly.py of the reference (generate_phenotype :74-334, fill_tank
:336-402, random_genome :404-420) with numpy and scipy only:

* matplotlib's ``Path.contains_points`` (make_jelly.py:151-156,209-215) is
  replaced by :func:`points_in_polygon`, a vectorised crossings test (even-odd
  rule, Haines' "crossings multiply" form) over the implicitly closed polygon.
* ``scipy.spatial.cKDTree`` is used exactly as the reference uses it.

Extensions that the reference does not have (all off by default, so the
default output matches fill_tank):

* ``spacing_div``: lattice spacing dx / spacing_div (the reference uses 2).
* ``jitter``: seeded uniform jitter of every live particle by +-jitter*dx.

The axisymmetric mode (make_jelly.py:13-14,275-307: the right half-profile is
the whole cross-section, payload over r in [0, W/2]) follows the reference's
JELLY_AXISYM environment variable unless ``axisym`` is passed explicitly.

Gene bounds follow evolve.py:55-62.
"""
from __future__ import annotations

import os

import numpy as np
from scipy.spatial import cKDTree

PAYLOAD_WIDTH = 0.08                       # make_jelly.py:8
PAYLOAD_HEIGHT = 0.05                      # make_jelly.py:9
DEFAULT_SPAWN = np.array([0.5, 0.40])      # make_jelly.py:10
TALL_SPAWN = np.array([0.5, 0.60])         # evolve.py:136
AXISYM_SPAWN = np.array([0.0, 0.40])       # make_jelly.py:11


def _axisym_default(axisym):
    """make_jelly.py:14 reads JELLY_AXISYM once at import; here per call."""
    return os.environ.get("JELLY_AXISYM", "0") == "1" if axisym is None else bool(axisym)

# evolve.py:60-61: [cp1_x, cp1_y, cp2_x, cp2_y, end_x, end_y, t_base, t_mid,
# t_tip, contraction_frac, freq_mult]
GENOME_LOWER = np.array([0.0, -0.15, 0.0, -0.2, 0.05, -0.30, 0.025, 0.025, 0.01, 0.05, 0.5])
GENOME_UPPER = np.array([0.25, 0.15, 0.3, 0.15, 0.35, +0.10, 0.08, 0.1, 0.04, 0.60, 2.0])

AURELIA_GENOME = np.array([0.05, 0.04, 0.18, -0.03, 0.22, -0.12, 0.04, 0.05, 0.015])  # make_jelly.py:19-29


def points_in_polygon(points: np.ndarray, polygon: np.ndarray) -> np.ndarray:
    """Even-odd containment of ``points`` (K,2) in the closed ``polygon`` (V,2).

    For each edge v0->v1 that straddles the test row (y flags taken with >=),
    the point is toggled when it lies on the inner side of the edge, decided
    by the sign of a cross product rather than an explicit intersection.
    """
    px = points[:, 0]
    py = points[:, 1]
    inside = np.zeros(len(points), dtype=bool)
    n = len(polygon)
    if n < 3:
        return inside
    v0 = polygon[-1]
    yflag0 = v0[1] >= py
    for k in range(n):
        v1 = polygon[k]
        yflag1 = v1[1] >= py
        straddle = yflag0 != yflag1
        if np.any(straddle):
            lhs = (v1[1] - py) * (v0[0] - v1[0]) >= (v1[0] - px) * (v0[1] - v1[1])
            inside ^= straddle & (lhs == yflag1)
        v0 = v1
        yflag0 = yflag1
    return inside


def _segments_intersect(a, b, c, d):
    """make_jelly.py:31-43."""
    def cross2d(u, v):
        return u[0] * v[1] - u[1] * v[0]
    r = b - a
    s = d - c
    rxs = cross2d(r, s)
    if abs(rxs) < 1e-12:
        return False
    qp = c - a
    t = cross2d(qp, s) / rxs
    u = cross2d(qp, r) / rxs
    return 0 < t < 1 and 0 < u < 1


def polygon_self_intersects(polygon) -> bool:
    """make_jelly.py:46-58: any non-adjacent edge pair crossing.

    The pair loop of the reference, evaluated for all pairs at once with the
    same float64 operations as _segments_intersect (same decisions)."""
    P = np.asarray(polygon, dtype=np.float64)
    n = len(P)
    if n < 4:
        return False
    i, j = np.triu_indices(n, k=2)
    keep = ~((i == 0) & (j == n - 1))
    i, j = i[keep], j[keep]
    a, b = P[i], P[(i + 1) % n]
    c, d = P[j], P[(j + 1) % n]
    r = b - a
    s = d - c
    rxs = r[:, 0] * s[:, 1] - r[:, 1] * s[:, 0]
    ok = np.abs(rxs) >= 1e-12
    qp = c - a
    with np.errstate(divide="ignore", invalid="ignore"):
        t = (qp[:, 0] * s[:, 1] - qp[:, 1] * s[:, 0]) / rxs
        u = (qp[:, 0] * r[:, 1] - qp[:, 1] * r[:, 0]) / rxs
    return bool(np.any(ok & (t > 0) & (t < 1) & (u > 0) & (u < 1)))


def cubic_bezier(p0, p1, p2, p3, t):
    """make_jelly.py:61-63."""
    return (1 - t) ** 3 * p0 + 3 * (1 - t) ** 2 * t * p1 + 3 * (1 - t) * t ** 2 * p2 + t ** 3 * p3


def _normals_2d(points):
    """make_jelly.py:65-73."""
    tangents = np.gradient(points, axis=0)
    normals = np.zeros_like(tangents)
    normals[:, 0] = -tangents[:, 1]
    normals[:, 1] = tangents[:, 0]
    norm = np.linalg.norm(normals, axis=1, keepdims=True)
    norm[norm == 0] = 1
    return normals / norm


def generate_phenotype(genome, spawn_offset=None, grid_res=128, with_payload=True, axisym=None):
    """Genome -> (pos (K,2) f64, mat (K,) int, fiber (K,2) f32, self_intersecting).

    Follows make_jelly.py:74-334 step by step: Bezier spine from genes 0-5,
    thickness envelope from genes 6-8, subumbrellar muscle layer, collar and
    transverse bridge masks, right half mirrored to the left, 20x12 payload
    lattice, spawn offset.
    """
    if spawn_offset is None:
        spawn_offset = DEFAULT_SPAWN
    start_p = np.array([PAYLOAD_WIDTH / 2.0, 0.0])
    cp1 = start_p + np.array([abs(genome[0]), genome[1]])
    cp2 = start_p + np.array([abs(genome[2]), genome[3]])
    end_p = start_p + np.array([abs(genome[4]), genome[5]])
    t_base = abs(genome[6])
    t_mid = abs(genome[7])
    t_tip = abs(genome[8])

    t_steps = np.linspace(0, 1, 50)
    spine_points = np.array([cubic_bezier(start_p, cp1, cp2, end_p, t) for t in t_steps])
    spine_tangent_raw = np.gradient(spine_points, axis=0)
    spine_tangent_norms = np.linalg.norm(spine_tangent_raw, axis=1, keepdims=True)
    spine_tangent_norms[spine_tangent_norms < 1e-10] = 1.0
    spine_tangents = spine_tangent_raw / spine_tangent_norms

    normals = _normals_2d(spine_points)
    t_profile = np.interp(t_steps, [0, 0.5, 1], [t_base, t_mid, t_tip])
    semi_thickness = t_profile[:, None] / 2.0
    outer_curve = spine_points + normals * semi_thickness
    inner_curve = spine_points - normals * semi_thickness

    spacing = 1.0 / (grid_res * 2.0)
    min_base_muscle = spacing * 1.2
    muscle_ratio = 0.2
    effective_muscle_thick = min_base_muscle + (semi_thickness * muscle_ratio)
    effective_muscle_thick = np.minimum(effective_muscle_thick, semi_thickness * 0.9)
    muscle_interface = spine_points - normals * (semi_thickness - effective_muscle_thick)

    body_polygon = np.vstack([outer_curve, inner_curve[::-1]])
    muscle_polygon = np.vstack([muscle_interface, inner_curve[::-1]])
    self_intersecting = (polygon_self_intersects(body_polygon) or
                         polygon_self_intersects(muscle_polygon))

    raster_res = grid_res * 2
    min_x = min(np.min(body_polygon[:, 0]), -PAYLOAD_WIDTH)
    max_x = max(np.max(body_polygon[:, 0]), PAYLOAD_WIDTH)
    min_y = min(np.min(body_polygon[:, 1]), -0.05)
    max_y = max(np.max(body_polygon[:, 1]), PAYLOAD_HEIGHT)
    PAD = 0.05
    x_range = np.linspace(min_x - PAD, max_x + PAD, int((max_x - min_x + 2 * PAD) * raster_res))
    y_range = np.linspace(min_y - PAD, max_y + PAD, int((max_y - min_y + 2 * PAD) * raster_res))
    grid_x, grid_y = np.meshgrid(x_range, y_range)
    candidate_points = np.vstack([grid_x.ravel(), grid_y.ravel()]).T

    mask_bell = points_in_polygon(candidate_points, body_polygon)
    mask_muscle = points_in_polygon(candidate_points, muscle_polygon)
    mask_payload_space_positive = ((candidate_points[:, 0] <= PAYLOAD_WIDTH / 2.0) &
                                   (candidate_points[:, 1] <= PAYLOAD_HEIGHT))

    collar_top_y = PAYLOAD_HEIGHT * 0.50
    collar_thickness_top = t_base * 0.35
    collar_t_vals = np.linspace(0, 1, 20)
    ci_P0 = np.array([PAYLOAD_WIDTH / 2.0, collar_top_y])
    ci_P3 = inner_curve[0]
    ci_P1 = np.array([PAYLOAD_WIDTH / 2.0, collar_top_y - collar_top_y * 0.4])
    ci_P2 = ci_P3 + np.array([0.0, min(collar_top_y * 0.3, abs(ci_P3[1] - ci_P0[1]) * 0.4)])
    collar_inner_edge = np.array([cubic_bezier(ci_P0, ci_P1, ci_P2, ci_P3, t) for t in collar_t_vals])
    bell_outer_start = outer_curve[0]

    if bell_outer_start[0] > PAYLOAD_WIDTH / 2.0:
        P0 = np.array([PAYLOAD_WIDTH / 2.0 + collar_thickness_top, collar_top_y])
        P3 = bell_outer_start
        P1 = np.array([P0[0], P0[1] - collar_top_y * 0.5])
        bell_tangent = outer_curve[min(2, len(outer_curve) - 1)] - outer_curve[0]
        bt_len = np.linalg.norm(bell_tangent)
        if bt_len > 1e-10:
            P2 = P3 - (bell_tangent / bt_len) * (collar_top_y * 0.6)
        else:
            P2 = P3 + np.array([0, 0.01])
        collar_outer_edge = np.array([cubic_bezier(P0, P1, P2, P3, t) for t in collar_t_vals])
        collar_polygon = np.vstack([collar_outer_edge, collar_inner_edge[::-1]])
        collar_muscle_edge = collar_inner_edge + muscle_ratio * (collar_outer_edge - collar_inner_edge)
        collar_muscle_polygon = np.vstack([collar_muscle_edge, collar_inner_edge[::-1]])
        mask_collar = points_in_polygon(candidate_points, collar_polygon) & ~mask_payload_space_positive
        mask_collar_muscle = (points_in_polygon(candidate_points, collar_muscle_polygon)
                              & ~mask_payload_space_positive)
        bridge_half_w = max(bell_outer_start[0], PAYLOAD_WIDTH / 2.0 + collar_thickness_top)
    else:
        mask_collar = np.zeros(len(candidate_points), dtype=bool)
        mask_collar_muscle = np.zeros(len(candidate_points), dtype=bool)
        bridge_half_w = PAYLOAD_WIDTH / 2.0 + 0.015

    if not with_payload:
        bridge_half_w = max(bridge_half_w, PAYLOAD_WIDTH / 2.0 + 0.02)
    bridge_thick = 0.03
    bridge_top = PAYLOAD_HEIGHT if not with_payload else 0.0
    mask_bridge = ((candidate_points[:, 0] >= -bridge_half_w) &
                   (candidate_points[:, 0] <= bridge_half_w) &
                   (candidate_points[:, 1] >= -bridge_thick) &
                   (candidate_points[:, 1] <= bridge_top))

    final_mats = np.zeros(len(candidate_points), dtype=int)
    final_mats[mask_bridge] = 1
    final_mats[mask_collar] = 1
    final_mats[mask_collar_muscle] = 3
    final_mats[mask_bell] = 1
    final_mats[mask_bell & mask_muscle] = 3

    mask_right_side = (candidate_points[:, 0] >= 0) & (final_mats > 0)
    right_points = candidate_points[mask_right_side]
    right_mats = final_mats[mask_right_side]
    right_fiber = np.zeros((len(right_points), 2), dtype=np.float32)
    right_fiber[:, 1] = 1.0
    if len(right_points) > 0 and np.any(right_mats == 3):
        spine_tree = cKDTree(spine_points)
        muscle_mask_r = right_mats == 3
        _, sp_idx = spine_tree.query(right_points[muscle_mask_r])
        right_fiber[muscle_mask_r] = spine_tangents[sp_idx]

    axisym = _axisym_default(axisym)
    if axisym:
        # make_jelly.py:276-280: the right half-profile is the whole (r >= 0) section
        all_soft_pos = right_points
        all_soft_mats = right_mats
        all_soft_fiber = right_fiber
    elif len(right_points) > 0:
        left_pos = right_points.copy()
        left_pos[:, 0] *= -1
        left_fiber = right_fiber.copy()
        left_fiber[:, 0] *= -1
        all_soft_pos = np.vstack([right_points, left_pos])
        all_soft_mats = np.concatenate([right_mats, right_mats.copy()])
        all_soft_fiber = np.vstack([right_fiber, left_fiber])
    else:
        all_soft_pos = np.zeros((0, 2))
        all_soft_mats = np.zeros(0, dtype=int)
        all_soft_fiber = np.zeros((0, 2), dtype=np.float32)

    payload_particles = None
    if with_payload:
        if axisym:  # make_jelly.py:300-301
            px = np.linspace(0, PAYLOAD_WIDTH / 2, int(PAYLOAD_WIDTH / 2 * raster_res))
        else:
            px = np.linspace(-PAYLOAD_WIDTH / 2, PAYLOAD_WIDTH / 2, int(PAYLOAD_WIDTH * raster_res))
        py = np.linspace(0, PAYLOAD_HEIGHT, int(PAYLOAD_HEIGHT * raster_res))
        pgx, pgy = np.meshgrid(px, py)
        payload_particles = np.vstack([pgx.ravel(), pgy.ravel()]).T

    offset = np.array(spawn_offset)
    final_pos, final_mat, final_fiber = [], [], []
    if len(all_soft_pos) > 0:
        final_pos.append(all_soft_pos + offset)
        final_mat.append(all_soft_mats)
        final_fiber.append(all_soft_fiber)
    if payload_particles is not None and len(payload_particles) > 0:
        final_pos.append(payload_particles + offset)
        final_mat.append(np.ones(len(payload_particles), dtype=int) * 2)
        pf = np.zeros((len(payload_particles), 2), dtype=np.float32)
        pf[:, 1] = 1.0
        final_fiber.append(pf)
    if final_pos:
        return (np.vstack(final_pos), np.concatenate(final_mat).astype(int),
                np.vstack(final_fiber).astype(np.float32), self_intersecting)
    return np.zeros((0, 2)), np.zeros(0, dtype=int), np.zeros((0, 2), dtype=np.float32), True


def fill_tank(genome, max_particles, grid_res=128, spawn_offset=None, water_margin=0.005,
              with_payload=True, domain_height=1.0, spacing_div=2.0, jitter=0.0, seed=None,
              axisym=None):
    """Robot + water lattice padded to ``max_particles`` slots (make_jelly.py:336-402).

    Returns (positions f32 (N,2), materials i32 (N,), fibers f32 (N,2), stats).
    Dead slots hold position -1, material -1 and fiber (0, 1).  Water that does
    not fit is truncated, as the reference does (make_jelly.py:371-374).
    """
    if spawn_offset is None:
        spawn_offset = DEFAULT_SPAWN
    robot_pos, robot_mat, robot_fiber, self_intersecting = generate_phenotype(
        genome, spawn_offset, grid_res=grid_res, with_payload=with_payload, axisym=axisym)
    n_robot = len(robot_pos)

    spacing = 1.0 / (grid_res * spacing_div)
    margin = (1.0 / (grid_res * 2.0)) * 3
    wx = np.arange(margin, 1.0 - margin, spacing)
    wy = np.arange(margin, domain_height - margin, spacing)
    wgx, wgy = np.meshgrid(wx, wy)
    water_candidates = np.vstack([wgx.ravel(), wgy.ravel()]).T
    if n_robot > 0:
        # make_jelly.py:361-364.  The search is bounded just above the margin:
        # candidates with no robot point that close come back at distance inf,
        # the others with their exact distance, so the kept set is the same.
        tree = cKDTree(robot_pos)
        distances, _ = tree.query(water_candidates, k=1, distance_upper_bound=water_margin * (1 + 1e-9))
        water_pos = water_candidates[distances > water_margin]
    else:
        water_pos = water_candidates
    n_water = len(water_pos)
    if n_robot + n_water > max_particles:
        n_water = max(0, max_particles - n_robot)
        n_robot = min(n_robot, max_particles)

    positions = np.full((max_particles, 2), -1.0, dtype=np.float32)
    materials = np.full(max_particles, -1, dtype=np.int32)
    fibers = np.zeros((max_particles, 2), dtype=np.float32)
    fibers[:, 1] = 1.0
    if n_robot > 0:
        positions[:n_robot] = robot_pos[:n_robot]
        materials[:n_robot] = robot_mat[:n_robot]
        fibers[:n_robot] = robot_fiber[:n_robot]
    if n_water > 0:
        positions[n_robot:n_robot + n_water] = water_pos[:n_water]
        materials[n_robot:n_robot + n_water] = 0
    n_live = n_robot + n_water
    if jitter > 0.0 and n_live > 0:
        rng = np.random.default_rng(seed)
        dx = 1.0 / grid_res
        noise = rng.uniform(-jitter * dx, jitter * dx, size=(n_live, 2))
        positions[:n_live] = (positions[:n_live] + noise).astype(np.float32)
        lo, hi = 0.001, (1.0 - 0.001, domain_height - 0.001)
        positions[:n_live, 0] = np.clip(positions[:n_live, 0], lo, hi[0])
        positions[:n_live, 1] = np.clip(positions[:n_live, 1], lo, hi[1])
    muscle_count = int(np.sum(materials[:n_robot] == 3))
    return positions, materials, fibers, {
        'n_robot': n_robot,
        'n_water': n_water,
        'n_total': n_live,
        'n_dead': max_particles - n_live,
        'muscle_count': muscle_count,
        'n_jelly': int(np.sum(materials[:n_robot] == 1)),
        'self_intersecting': self_intersecting,
    }


def _phenotype_job(args):
    genome, spawn_offset, grid_res, with_payload, axisym = args
    return generate_phenotype(genome, spawn_offset, grid_res=grid_res, with_payload=with_payload, axisym=axisym)


def make_pool(workers=None):
    """A process pool for phenotypes(): spawned workers (they inherit no CUDA
    state and import only numpy and scipy).  Reuse it across generations;
    close it with .shutdown().  Spawned workers import the caller's main
    module, so a script that uses the pool keeps its top-level work under
    ``if __name__ == "__main__":``."""
    import concurrent.futures
    import multiprocessing
    return concurrent.futures.ProcessPoolExecutor(max_workers=workers or os.cpu_count(),
                                                  mp_context=multiprocessing.get_context("spawn"))


def phenotypes(genomes, spawn_offset=None, grid_res=128, with_payload=True, axisym=None, executor=None):
    """generate_phenotype of every genome, in order; with an ``executor``
    (make_pool()) the genomes are spread over its worker processes.  The
    results are those of the serial calls (same float64 operations)."""
    if spawn_offset is None:
        spawn_offset = DEFAULT_SPAWN
    axisym = _axisym_default(axisym)  # resolved here, not from the workers' environment
    res = grid_res if np.ndim(grid_res) else [grid_res] * len(genomes)
    jobs = [(g, spawn_offset, int(r), with_payload, axisym) for g, r in zip(genomes, res)]
    if executor is None:
        return [_phenotype_job(j) for j in jobs]
    workers = getattr(executor, "_max_workers", None) or os.cpu_count() or 1
    return list(executor.map(_phenotype_job, jobs, chunksize=max(1, len(jobs) // (4 * workers))))


def _tank_stats(engine, m, robot_mat, n_robot, n_water, self_intersecting):
    mats = np.asarray(robot_mat[:n_robot])
    return {
        'n_robot': n_robot,
        'n_water': n_water,
        'n_total': n_robot + n_water,
        'n_dead': engine.instances[m].n_slots - n_robot - n_water,
        'muscle_count': int(np.sum(mats == 3)),
        'n_jelly': int(np.sum(mats == 1)),
        'self_intersecting': self_intersecting,
    }


def load_tanks(engine, genomes, spawn_offset=None, water_margin=0.005, with_payload=True, spacing_div=2.0,
               axisym=None, executor=None):
    """load_tank for instances 0 .. len(genomes) - 1, the robots generated
    first (over ``executor``'s workers when given); returns the stats dicts."""
    robots = phenotypes(genomes, spawn_offset, [engine.instances[m].n_grid for m in range(len(genomes))],
                        with_payload, axisym, executor)
    out = []
    for m, (rp, rm, rf, si) in enumerate(robots):
        n_robot, n_water = engine.load_robot(m, rp, rm, rf, water_margin, spacing_div)
        out.append(_tank_stats(engine, m, rm, n_robot, n_water, si))
    return out


def load_tank(engine, m, genome, spawn_offset=None, water_margin=0.005, with_payload=True, spacing_div=2.0,
              axisym=None):
    """fill_tank straight into instance m of ``engine``: the robot is generated
    here (generate_phenotype), the water lattice, its exclusion around the
    robot and the slot layout run on the GPU (Engine.load_robot).  The slots
    hold exactly what fill_tank(genome, n_slots, grid_res=n_grid,
    domain_height=..., jitter=0) returns; the stats dict is fill_tank's."""
    spec = engine.instances[m]
    if spawn_offset is None:
        spawn_offset = DEFAULT_SPAWN
    robot_pos, robot_mat, robot_fiber, self_intersecting = generate_phenotype(
        genome, spawn_offset, grid_res=spec.n_grid, with_payload=with_payload, axisym=axisym)
    n_robot, n_water = engine.load_robot(m, robot_pos, robot_mat, robot_fiber, water_margin, spacing_div)
    return _tank_stats(engine, m, robot_mat, n_robot, n_water, self_intersecting)


def uniform_genomes(n, seed):
    """n genomes drawn uniformly within the gene bounds (evolve.py:60-61)."""
    rng = np.random.default_rng(seed)
    return rng.uniform(GENOME_LOWER, GENOME_UPPER, size=(n, len(GENOME_LOWER)))


def gaussian_genomes(n, seed, sigma_frac=0.3):
    """n genomes ~ N(bound midpoint, (sigma_frac * range)^2), clipped to bounds."""
    rng = np.random.default_rng(seed)
    mid = (GENOME_LOWER + GENOME_UPPER) / 2
    rng_w = GENOME_UPPER - GENOME_LOWER
    g = rng.normal(mid, sigma_frac * rng_w, size=(n, len(mid)))
    return np.clip(g, GENOME_LOWER, GENOME_UPPER)


def timing_params(genome):
    """Per-instance waveform parameters from genes 9-10, clipped as evolve.py:149-152 does."""
    contraction = float(np.clip(genome[9], 0.05, 0.60)) if len(genome) > 9 else 0.20
    freq = float(np.clip(genome[10], 0.5, 2.0)) if len(genome) > 10 else 1.0
    return contraction, freq
