"""The renderer oracle (oracle/render_oracle.c) against frames recorded from
the reference's own render kernels (mpm_sim.py:343-712)."""
from __future__ import annotations

import numpy as np
import pytest

import render_cases as rc
from oracle import oracle


class OracleOps:
    """The reference's render calls, on the CPU oracle."""

    def __init__(self, fx):
        s = rc.scene_arrays(fx)
        M = rc.n_instances(fx)
        self.sc = oracle.RenderScene(s["x"], s["v"], s["material"], s["Jp"], s["grid_v"], s["grid_m"],
                                     [float(fx["domain_height"])] * M, fx["param_freq"],
                                     fx["param_contraction"], fx["hue"], fx["muscle_hue"], fx["time"])
        self.fb = oracle.new_frame(int(fx["video_res"]))
        self.vgrid = None

    def clear(self, value):
        oracle.render_clear(self.fb, value)

    def abyss(self, rs, gs, r, mode):
        oracle.render_abyss(self.fb, self.sc, rs, gs, r, mode)

    def tone_map(self):
        oracle.render_tone_map(self.fb)

    def overlay(self, rs, gs, scale):
        oracle.render_vorticity_overlay(self.fb, self.sc, rs, gs, scale)

    def vort_grid(self, scale):
        self.vgrid = oracle.vorticity_grid(self.sc, scale)
        return self.vgrid

    def vort(self, rs, gs, alpha, style):
        oracle.render_vorticity(self.fb, self.sc, self.vgrid, rs, gs, alpha, style)

    def flat(self, rs, gs, r, mat, cr, cg, cb):
        oracle.render_flat(self.fb, self.sc, rs, gs, r, mat, cr, cg, cb)

    def frame(self):
        return self.fb.copy()


@pytest.mark.parametrize("case", rc.RENDER_CASES)
def test_render_oracle_matches_reference_frames(case):
    fx = rc.load(case)
    got = rc.run_sequences(OracleOps(fx), fx)
    for k in rc.FRAME_KEYS:
        np.testing.assert_allclose(got[k], fx[k], rtol=rc.RTOL, atol=rc.ATOL, err_msg=f"{case} {k}")


def test_render_oracle_coverage_is_exact():
    """Which pixels a splat touches depends only on exactly rounded f32 ops
    (centre, footprint, distance test): the oracle's coverage of every frame
    equals the reference's pixel for pixel."""
    for case in rc.RENDER_CASES:
        fx = rc.load(case)
        got = rc.run_sequences(OracleOps(fx), fx)
        for k in ("abyss_w0", "abyss_w1", "abyss_w2", "overlay_hdr", "web"):
            base = 0.98 if k == "web" else 0.0
            np.testing.assert_array_equal(got[k] != base, fx[k] != base, err_msg=f"{case} {k}")
