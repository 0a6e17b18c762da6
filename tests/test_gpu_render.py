"""GPU parity of the headless renderer (jf_render.cu through the C ABI).

* Fixtures recorded from the reference's own render kernels
  (tests/golden/render_*.npz, mpm_sim.py:343-712) are replayed call for call
  on the engine: every frame and vorticity grid agrees within the tolerance in
  tests/render_cases.py (additive splats summed in another order), and which
  pixels each splat or vorticity cell touches agrees exactly.
* At full size (1024^2 frame, 8 instances of about 62K live particles from a
  stepped simulation, particles in the batched path's sorted order) the GPU
  frames are compared with the CPU oracle rendering the same state read back
  in slot order.
"""
import numpy as np
import pytest

import render_cases as rc

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

PATHS = ("plain", "batched")


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from jellyfih_b200 import build
    build.build()


class EngineOps:
    """The reference's render calls, on the engine (C ABI)."""

    def __init__(self, e, fx):
        self.e = e
        self.hue = fx["hue"]
        self.mhue = fx["muscle_hue"]
        e.frame_create(int(fx["video_res"]))

    def clear(self, value):
        self.e.frame_clear(value)

    def abyss(self, rs, gs, r, mode):
        self.e.render_abyss(rs, gs, r, self.hue, self.mhue, mode)

    def tone_map(self):
        self.e.tone_map()

    def overlay(self, rs, gs, scale):
        self.e.render_vorticity_overlay(rs, gs, scale)

    def vort_grid(self, scale):
        self.e.compute_vorticity(scale)
        return [self.e.read_vorticity(m) for m in range(self.e.M)]

    def vort(self, rs, gs, alpha, style):
        self.e.render_vorticity(rs, gs, alpha, style)

    def flat(self, rs, gs, r, mat, cr, cg, cb):
        self.e.render_flat(rs, gs, r, mat, cr, cg, cb)

    def frame(self):
        return self.e.read_frame()


def _engine_for(fx, path):
    from jellyfih_b200 import Engine, InstanceSpec
    M = rc.n_instances(fx)
    s = rc.scene_arrays(fx)
    spec = InstanceSpec(len(s["material"][0]), int(fx["n_grid"]), int(fx["n_grid_y"]), float(fx["domain_height"]))
    e = Engine([spec] * M, path=path)
    for m in range(M):
        e.load(m, s["x"][m], s["material"][m], s["fiber"][m])
        e.write(m, v=s["v"][m], Jp=s["Jp"][m])
        e.write_grid(m, s["grid_v"][m], s["grid_m"][m])
    e.set_params(freq=fx["param_freq"], contraction=fx["param_contraction"])
    e.time = float(fx["time"])
    return e


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("case", rc.RENDER_CASES)
def test_render_matches_reference_frames(case, path):
    fx = rc.load(case)
    e = _engine_for(fx, path)
    try:
        got = rc.run_sequences(EngineOps(e, fx), fx)
    finally:
        e.close()
    for k in rc.FRAME_KEYS:
        np.testing.assert_allclose(got[k], fx[k], rtol=rc.RTOL, atol=rc.ATOL, err_msg=f"{case} {path} {k}")
    for k in ("abyss_w0", "abyss_w1", "abyss_w2", "overlay_hdr", "web"):
        base = 0.98 if k == "web" else 0.0
        np.testing.assert_array_equal(got[k] != base, fx[k] != base, err_msg=f"{case} {path} {k} coverage")


def test_render_errors():
    from jellyfih_b200 import Engine, InstanceSpec, JfError
    e = Engine([InstanceSpec(64)], path="plain")
    try:
        with pytest.raises(JfError):
            e.tone_map()  # no frame yet
        with pytest.raises(JfError):
            e.read_frame()
        e.frame_create(32)
        with pytest.raises(JfError):
            e.render_vorticity(32, 1, 0.5, 7)  # unknown style
        with pytest.raises(JfError):
            e.render_flat(0, 1, 1.0, 0, 1.0, 1.0, 1.0)  # res_sub 0
        with pytest.raises(JfError):
            e.frame_create(0)
        # the vorticity grid exists (zero) before the first compute
        assert not e.read_vorticity(0).any()
        assert not e.read_frame().any()
    finally:
        e.close()


def test_render_full_frame_matches_oracle(oracle):
    """1024^2, 8 instances x 80K slots after 200 substeps (batched, sorted
    particles): abyss (rainbow water), vorticity overlay, tone map, vorticity
    grid and rdbu against the oracle rendering the read-back state."""
    import bench
    from jellyfih_b200 import Engine, InstanceSpec
    M, res = 8, 1024
    inputs = bench.make_inputs(M, 80000, 77)
    e = Engine([InstanceSpec(80000)] * M, path="batched")
    try:
        bench.load_all(e, inputs)
        e.step(200)
        gs = int(np.ceil(np.sqrt(M)))
        rs = res // gs
        radius = max(1.0, rs / 128 * 0.6)
        hue = np.linspace(0.05, 0.95, M).astype(np.float32)
        mhue = ((hue + 0.15) % 1.0).astype(np.float32)
        st = [e.read(m) for m in range(M)]
        grids = [e.read_grid(m) for m in range(M)]
        params = e.get_params()
        sc = oracle.RenderScene([s["x"] for s in st], [s["v"] for s in st], [s["material"] for s in st],
                                [s["Jp"] for s in st], [g[0] for g in grids], [g[1] for g in grids], [1.0] * M,
                                params["freq"], params["contraction"], hue, mhue, e.time)
        fb = oracle.new_frame(res)
        e.frame_create(res)
        e.render_abyss(rs, gs, 1.5, hue, mhue, 2)
        oracle.render_abyss(fb, sc, rs, gs, 1.5, 2)
        got = e.read_frame()
        np.testing.assert_allclose(got, fb, rtol=1e-4, atol=1e-6)
        np.testing.assert_array_equal(got != 0, fb != 0)
        e.render_vorticity_overlay(rs, gs, 0.001)
        oracle.render_vorticity_overlay(fb, sc, rs, gs, 0.001)
        e.tone_map()
        oracle.render_tone_map(fb)
        np.testing.assert_allclose(e.read_frame(), fb, rtol=1e-4, atol=1e-6)
        e.compute_vorticity(0.003)
        vort = oracle.vorticity_grid(sc, 0.003)
        for m in range(M):
            np.testing.assert_allclose(e.read_vorticity(m), vort[m], rtol=1e-6, atol=1e-7)
        e.render_vorticity(rs, gs, 0.6, 0)
        oracle.render_vorticity(fb, sc, vort, rs, gs, 0.6, 0)
        np.testing.assert_allclose(e.read_frame(), fb, rtol=1e-4, atol=1e-6)
        e.frame_clear(0.98)
        oracle.render_clear(fb, 0.98)
        for mat_id, cr, cg, cb in rc.WEB_PALETTE:
            e.render_flat(rs, gs, radius, mat_id, cr, cg, cb)
            oracle.render_flat(fb, sc, rs, gs, radius, mat_id, cr, cg, cb)
        np.testing.assert_array_equal(e.read_frame(), fb)
    finally:
        e.close()
