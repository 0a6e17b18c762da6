"""Renderer fixtures (tests/golden/render_*.npz, recorded from the reference's
own render kernels by tests/golden/make_render_golden.py) and the call
sequences that produced them, replayed against any backend with the
reference's kernel names (the CPU oracle, or the engine through the C ABI)."""
from __future__ import annotations

import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RENDER_CASES = ["render_2inst", "render_3inst", "render_tall"]

# Frame tolerances against the fixtures.  Additive splats are summed in
# another order on the GPU (float atomics), and the stand-in that recorded the
# fixtures evaluates some f32 expressions of the reference in double
# (hsv2rgb's saturation, Python-float constants); per-pixel deviations from
# both stay below 1e-5 relative on HDR sums of up to ~80.
RTOL = 2e-5
ATOL = 2e-6


def load(case):
    return dict(np.load(os.path.join(HERE, "golden", f"{case}.npz")))


def n_instances(fx):
    return len(fx["param_freq"])


def scene_arrays(fx):
    """Per-instance arrays in slot order / reference grid layout."""
    M = n_instances(fx)
    return {
        "x": [fx[f"in{m}_x"] for m in range(M)],
        "v": [fx[f"in{m}_v"] for m in range(M)],
        "material": [fx[f"in{m}_material"] for m in range(M)],
        "fiber": [fx[f"in{m}_fiber"] for m in range(M)],
        "Jp": [fx[f"in{m}_Jp"] for m in range(M)],
        "grid_v": [fx[f"in{m}_grid_v"] for m in range(M)],
        "grid_m": [fx[f"in{m}_grid_m"] for m in range(M)],
    }


def run_sequences(ops, fx):
    """Replays make_render_golden.py's call sequences; ``ops`` provides
    clear(value), abyss(res_sub, grid_side, radius, water_mode), tone_map(),
    overlay(res_sub, grid_side, scale), vort_grid(scale) -> [(nx, ny)],
    vort(res_sub, grid_side, alpha, style), flat(res_sub, grid_side, radius,
    material, r, g, b) and frame() -> (res, res, 3) float32."""
    rs, gs = int(fx["res_sub"]), int(fx["grid_side"])
    r = float(fx["radius"])
    out = {}
    for mode in (0, 1, 2):
        ops.clear(0.0)
        ops.abyss(rs, gs, r, mode)
        out[f"abyss_w{mode}"] = ops.frame()
    ops.tone_map()
    out["abyss_w2_tm"] = ops.frame()
    ops.clear(0.0)
    ops.abyss(rs, gs, r, 2)
    ops.overlay(rs, gs, 0.001)
    out["overlay_hdr"] = ops.frame()
    ops.tone_map()
    out["overlay_tm"] = ops.frame()
    out["vort"] = np.stack(ops.vort_grid(0.003))
    ops.clear(0.0)
    ops.abyss(rs, gs, r, 0)
    ops.tone_map()
    ops.vort(rs, gs, 0.6, 0)
    out["rdbu"] = ops.frame()
    ops.clear(0.0)
    ops.abyss(rs, gs, r, 1)
    ops.tone_map()
    ops.vort(rs, gs, 0.5, 1)
    out["hueshift"] = ops.frame()
    ops.vort(rs, gs, 0.65, 2)
    out["white"] = ops.frame()
    ops.clear(0.98)
    for mat_id, cr, cg, cb in WEB_PALETTE:
        ops.flat(rs, gs, float(fx["flat_radius"]), mat_id, cr, cg, cb)
    out["web"] = ops.frame()
    return out


# mpm_sim.py:70-75
WEB_PALETTE = [
    (0, 0.933, 0.949, 0.957),
    (1, 0.678, 0.882, 0.875),
    (3, 0.976, 0.757, 0.765),
    (2, 0.961, 0.824, 0.576),
]

FRAME_KEYS = ["abyss_w0", "abyss_w1", "abyss_w2", "abyss_w2_tm", "overlay_hdr", "overlay_tm", "vort",
              "rdbu", "hueshift", "white", "web"]
