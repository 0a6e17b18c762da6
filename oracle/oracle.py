"""ctypes front end of the CPU oracle (oracle/mpm_oracle.c: the substep;
oracle/render_oracle.c: the headless renderer).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the checker or the timed CPU baseline,
never by the product path.

State dictionaries use the reference's field layouts (mpm_sim.py:86-93):
``x, v, fiber`` (N,2), ``C, F`` (N,2,2), ``material`` (N,) int32, ``Jp``,
``glow`` (N,), ``r_ref`` (N,) (the load radius, mpm_sim.py:727; read only by the
axisymmetric variant), ``grid_v`` (nx,ny,2), ``grid_m`` (nx,ny).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_mpm.so")
_lib = None

DT = 2e-5  # mpm_sim.py:19


class OracleInst(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("domain_h", ctypes.c_double),
                ("dt", ctypes.c_double), ("actuation", ctypes.c_double),
                ("contraction", ctypes.c_double), ("freq", ctypes.c_double),
                ("payload_density", ctypes.c_double), ("axisym", ctypes.c_int32),
                ("fixed_p2g", ctypes.c_int32)]


@dataclass
class Instance:
    """Static grid description plus the per-instance waveform parameters."""
    nx: int = 128
    ny: int = 128
    domain_h: float = 1.0
    dt: float = DT
    actuation: float = 500.0        # mpm_sim.py:53,146
    contraction: float = 0.20       # mpm_sim.py:56,148
    freq: float = 1.0               # mpm_sim.py:149
    payload_density: float = 2.5    # mpm_sim.py:147
    axisym: bool = False            # JELLY_AXISYM, mpm_sim.py:17
    # not in the reference: P2G sums in 2^-44 fixed point (order-free), as the
    # GPU engine's deterministic forward sums them; see mpm_oracle.c
    fixed_p2g: bool = False

    def c(self) -> OracleInst:
        return OracleInst(self.nx, self.ny, self.domain_h, self.dt, self.actuation,
                          self.contraction, self.freq, self.payload_density, 1 if self.axisym else 0,
                          1 if self.fixed_p2g else 0)


def build(force: bool = False) -> str:
    """Compile liboracle_mpm.so with the committed Makefile."""
    if force or not os.path.exists(_LIB_PATH) or any(
            os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, f))
            for f in ("mpm_oracle.c", "render_oracle.c")):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        for sfx in ("f32", "f64"):
            getattr(L, f"oracle_substep_{sfx}").argtypes = [
                ctypes.POINTER(OracleInst), ctypes.c_int64] + [P] * 11 + [
                ctypes.c_float if sfx == "f32" else ctypes.c_double]
            getattr(L, f"oracle_run_{sfx}").argtypes = [
                ctypes.POINTER(OracleInst), ctypes.c_int64] + [P] * 11 + [P, ctypes.c_int64]
            getattr(L, f"oracle_run_batch_{sfx}").argtypes = [
                ctypes.c_int32, P, P, P, P] + [P] * 11 + [P, ctypes.c_int64]
            getattr(L, f"oracle_stats_{sfx}").argtypes = [ctypes.c_int64, P, P, ctypes.c_int32, P]
            getattr(L, f"oracle_svd2_{sfx}").argtypes = [P, P, P, P]
            getattr(L, f"oracle_activation_{sfx}").argtypes = [
                ctypes.POINTER(OracleInst), ctypes.c_float if sfx == "f32" else ctypes.c_double]
            getattr(L, f"oracle_activation_{sfx}").restype = (
                ctypes.c_float if sfx == "f32" else ctypes.c_double)
        I32, F32, RI = ctypes.c_int32, ctypes.c_float, ctypes.POINTER(RoInst)
        L.ro_clear.argtypes = [P, I32, F32]
        L.ro_tone_map.argtypes = [P, I32]
        L.ro_abyss.argtypes = [P, I32, I32, RI, P, P, P, P, F32, I32, I32, F32, I32]
        L.ro_flat.argtypes = [P, I32, I32, RI, P, P, I32, I32, F32, I32, F32, F32, F32]
        L.ro_vort_overlay.argtypes = [P, I32, I32, RI, P, P, I32, I32, F32]
        L.ro_vort_grid.argtypes = [P, I32, RI, P, P, F32]
        L.ro_vort_blend.argtypes = [P, I32, I32, RI, P, I32, I32, F32, I32]
        _lib = L
    return _lib


def _dtype(precision):
    return np.float32 if precision == "f32" else np.float64


def new_state(pos, mat, fiber=None, precision="f32", nx=128, ny=128):
    """State after load_particles (mpm_sim.py:715-736): v=0, F=I, C=0, Jp=1."""
    dt = _dtype(precision)
    n = len(mat)
    if fiber is None:
        fiber = np.zeros((n, 2), np.float32)
        fiber[:, 1] = 1.0
    F = np.zeros((n, 2, 2), dt)
    F[:, 0, 0] = 1
    F[:, 1, 1] = 1
    return {
        "x": np.ascontiguousarray(pos, dtype=dt).copy(),
        "v": np.zeros((n, 2), dt),
        "C": np.zeros((n, 2, 2), dt),
        "F": F,
        "material": np.ascontiguousarray(mat, dtype=np.int32).copy(),
        "Jp": np.ones(n, dt),
        "glow": np.zeros(n, dt),
        "fiber": np.ascontiguousarray(fiber, dtype=dt).copy(),
        "r_ref": np.ascontiguousarray(np.asarray(pos)[:, 0], dtype=dt).copy(),
        "grid_v": np.zeros((nx, ny, 2), dt),
        "grid_m": np.zeros((nx, ny), dt),
    }


def cast_state(state, precision):
    dt = _dtype(precision)
    out = {}
    for k, a in state.items():
        out[k] = np.ascontiguousarray(a, dtype=np.int32 if k == "material" else dt).copy()
    return out


def _ptrs(s):
    return [s[k].ctypes.data for k in ("x", "v", "C", "F", "material", "Jp", "glow", "fiber",
                                        "r_ref", "grid_v", "grid_m")]


def _check(inst: Instance, s):
    dt = s["x"].dtype
    for k in ("x", "v", "C", "F", "Jp", "glow", "fiber", "r_ref", "grid_v", "grid_m"):
        assert s[k].dtype == dt and s[k].flags.c_contiguous, k
    assert s["material"].dtype == np.int32 and s["material"].flags.c_contiguous
    assert s["grid_m"].shape == (inst.nx, inst.ny)
    return "f32" if dt == np.float32 else "f64"


def substep(inst: Instance, state, t):
    """One substep in place (mpm_sim.py:153-339); returns the advanced time."""
    sfx = _check(inst, state)
    ci = inst.c()
    n = len(state["material"])
    getattr(lib(), f"oracle_substep_{sfx}")(ctypes.byref(ci), n, *_ptrs(state), t)
    dt = _dtype(sfx)
    return dt(dt(t) + dt(inst.dt))


def run(inst: Instance, state, t, steps):
    """``steps`` substeps in place; returns the advanced time (REAL running sum)."""
    sfx = _check(inst, state)
    ci = inst.c()
    n = len(state["material"])
    tt = np.array([t], dtype=_dtype(sfx))
    getattr(lib(), f"oracle_run_{sfx}")(ctypes.byref(ci), n, *_ptrs(state), tt.ctypes.data, steps)
    return tt[0]


def run_batch(insts, states, t, steps, precision="f32"):
    """Advance many instances together, OpenMP-parallel over instances.

    ``states`` is a list of per-instance state dicts; they are packed into
    contiguous buffers, advanced, and unpacked in place.
    """
    dt = _dtype(precision)
    M = len(insts)
    counts = np.array([len(s["material"]) for s in states], np.int64)
    offs = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.int64)
    nodes = np.array([i.nx * i.ny for i in insts], np.int64)
    goffs = np.concatenate([[0], np.cumsum(nodes)[:-1]]).astype(np.int64)
    packed = {}
    for k in ("x", "v", "C", "F", "material", "Jp", "glow", "fiber", "r_ref"):
        packed[k] = np.ascontiguousarray(np.concatenate([s[k] for s in states], axis=0))
    for k in ("grid_v", "grid_m"):
        packed[k] = np.ascontiguousarray(np.concatenate([s[k].reshape(-1) for s in states]))
    cis = (OracleInst * M)(*[i.c() for i in insts])
    tt = np.array([t], dtype=dt)
    getattr(lib(), f"oracle_run_batch_{precision}")(
        M, ctypes.addressof(cis), counts.ctypes.data, offs.ctypes.data, goffs.ctypes.data,
        *_ptrs(packed), tt.ctypes.data, steps)
    for m, s in enumerate(states):
        o, c = offs[m], counts[m]
        for k in ("x", "v", "C", "F", "Jp", "glow"):
            s[k][...] = packed[k][o:o + c]
        g0, ng = goffs[m], nodes[m]
        s["grid_m"][...] = packed["grid_m"][g0:g0 + ng].reshape(s["grid_m"].shape)
        s["grid_v"][...] = packed["grid_v"][2 * g0:2 * (g0 + ng)].reshape(s["grid_v"].shape)
    return tt[0]


def stats_sums(x, mat, mode=0):
    """[sum_y, count, sum_x] of payload (mode 0) or body (mode 1), mpm_sim.py:746-762."""
    x = np.ascontiguousarray(x)
    mat = np.ascontiguousarray(mat, dtype=np.int32)
    sfx = "f32" if x.dtype == np.float32 else "f64"
    out = np.zeros(3, np.float64)
    getattr(lib(), f"oracle_stats_{sfx}")(len(mat), x.ctypes.data, mat.ctypes.data, mode,
                                          out.ctypes.data)
    return out


def stats_any(xs, mats):
    """_get_stats_any (mpm_sim.py:779-800): (M,3) [com_y, com_x, count], payload
    CoM where present, else the jelly+muscle body CoM."""
    M = len(xs)
    out = np.zeros((M, 3))
    for m in range(M):
        raw = stats_sums(xs[m], mats[m], 0)
        if raw[1] == 0:
            raw = stats_sums(xs[m], mats[m], 1)
        if raw[1] > 0:
            out[m] = [raw[0] / raw[1], raw[2] / raw[1], raw[1]]
    return out


def payload_stats(xs, mats):
    """get_payload_stats (mpm_sim.py:764-777)."""
    M = len(xs)
    out = np.zeros((M, 3))
    for m in range(M):
        raw = stats_sums(xs[m], mats[m], 0)
        if raw[1] > 0:
            out[m] = [raw[0] / raw[1], raw[2] / raw[1], raw[1]]
    return out


def headless_rows(initial, final):
    """run_batch_headless result assembly (mpm_sim.py:821-834)."""
    M = len(initial)
    res = np.zeros((M, 5))
    for i in range(M):
        if initial[i, 2] > 0 and final[i, 2] > 0:
            res[i, 0] = initial[i, 0]
            res[i, 1] = initial[i, 1]
            res[i, 2] = final[i, 0]
            res[i, 3] = final[i, 1]
            res[i, 4] = 0.0 if final[i, 0] < 0.01 else 1.0
    return res


def svd2(A):
    A = np.ascontiguousarray(A)
    sfx = "f32" if A.dtype == np.float32 else "f64"
    U = np.zeros((2, 2), A.dtype)
    sig = np.zeros(2, A.dtype)
    V = np.zeros((2, 2), A.dtype)
    getattr(lib(), f"oracle_svd2_{sfx}")(A.ctypes.data, U.ctypes.data, sig.ctypes.data,
                                         V.ctypes.data)
    return U, sig, V


def activation(inst: Instance, t, precision="f32"):
    ci = inst.c()
    return getattr(lib(), f"oracle_activation_{precision}")(ctypes.byref(ci), t)


# --- renderer (render_oracle.c, mpm_sim.py:343-712) ----------------------------
class RoInst(ctypes.Structure):
    _fields_ = [("n_slots", ctypes.c_int32), ("nx", ctypes.c_int32), ("ny", ctypes.c_int32),
                ("domain_h", ctypes.c_float), ("freq", ctypes.c_float), ("contraction", ctypes.c_float),
                ("hue", ctypes.c_float), ("muscle_hue", ctypes.c_float)]


class RenderScene:
    """What the renderer reads, for every instance: particle x, v, material,
    Jp (slot order), grid_v (nx, ny, 2) and grid_m (nx, ny) of the last
    substep, grid shape, domain height, waveform parameters, hues, sim_time."""

    def __init__(self, x, v, material, Jp, grid_v, grid_m, domain_h, freq, contraction, hue,
                 muscle_hue, t):
        M = len(x)
        self.M = M
        self.x = np.ascontiguousarray(np.concatenate(x), np.float32)
        self.v = np.ascontiguousarray(np.concatenate(v), np.float32)
        self.mat = np.ascontiguousarray(np.concatenate(material), np.int32)
        self.Jp = np.ascontiguousarray(np.concatenate(Jp), np.float32)
        self.gv = np.ascontiguousarray(np.concatenate([g.reshape(-1) for g in grid_v]), np.float32)
        self.gm = np.ascontiguousarray(np.concatenate([g.reshape(-1) for g in grid_m]), np.float32)
        self.shapes = [g.shape for g in grid_m]
        self.t = float(np.float32(t))
        arr = (RoInst * M)()
        for m in range(M):
            arr[m] = RoInst(len(material[m]), grid_m[m].shape[0], grid_m[m].shape[1], float(domain_h[m]),
                            float(freq[m]), float(contraction[m]), float(hue[m]), float(muscle_hue[m]))
        self.inst = arr


def new_frame(res, value=0.0):
    return np.full((res, res, 3), value, np.float32)


def _fp(a):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data


def render_clear(fb, value):
    lib().ro_clear(_fp(fb), fb.shape[0], float(value))


def render_tone_map(fb):
    lib().ro_tone_map(_fp(fb), fb.shape[0])


def render_abyss(fb, sc: RenderScene, res_sub, grid_side, radius, water_mode):
    lib().ro_abyss(_fp(fb), fb.shape[0], sc.M, sc.inst, sc.x.ctypes.data, sc.v.ctypes.data,
                   sc.mat.ctypes.data, sc.Jp.ctypes.data, sc.t, int(res_sub), int(grid_side),
                   float(radius), int(water_mode))


def render_flat(fb, sc: RenderScene, res_sub, grid_side, radius, target, r, g, b):
    lib().ro_flat(_fp(fb), fb.shape[0], sc.M, sc.inst, sc.x.ctypes.data, sc.mat.ctypes.data,
                  int(res_sub), int(grid_side), float(radius), int(target), float(r), float(g), float(b))


def render_vorticity_overlay(fb, sc: RenderScene, res_sub, grid_side, scale):
    lib().ro_vort_overlay(_fp(fb), fb.shape[0], sc.M, sc.inst, sc.gv.ctypes.data, sc.gm.ctypes.data,
                          int(res_sub), int(grid_side), float(scale))


def vorticity_grid(sc: RenderScene, scale):
    """tanh-mapped curl per node, one (nx, ny) array per instance."""
    out = np.zeros(sc.gm.shape, np.float32)
    lib().ro_vort_grid(_fp(out), sc.M, sc.inst, sc.gv.ctypes.data, sc.gm.ctypes.data, float(scale))
    res, o = [], 0
    for shp in sc.shapes:
        n = shp[0] * shp[1]
        res.append(out[o:o + n].reshape(shp))
        o += n
    return res


def render_vorticity(fb, sc: RenderScene, vort, res_sub, grid_side, alpha, style):
    """style 0 rdbu, 1 hueshift, 2 white (over a cleared white frame)."""
    flat = np.ascontiguousarray(np.concatenate([a.reshape(-1) for a in vort]), np.float32)
    lib().ro_vort_blend(_fp(fb), fb.shape[0], sc.M, sc.inst, flat.ctypes.data, int(res_sub),
                        int(grid_side), float(alpha), int(style))
