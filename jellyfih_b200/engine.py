"""Python host of the engine: one :class:`Engine` owns one libjellyfih handle.

Arrays passed in and returned use the reference's field layouts
(mpm_sim.py:86-93): positions / velocities / fibres (n, 2), C and F (n, 2, 2)
row-major, material (n,) int32, grids (nx, ny, 2) and (nx, ny).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _lib as L

DT = 2e-5  # mpm_sim.py:19


@dataclass(frozen=True)
class InstanceSpec:
    """Slots and grid of one instance (mpm_sim.py:11-16)."""
    n_slots: int = 80000
    n_grid: int = 128
    n_grid_y: int = 128
    domain_height: float = 1.0


def _f32(a, shape=None):
    arr = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None and arr.shape != shape:
        raise ValueError(f"expected shape {shape}, got {arr.shape}")
    return arr


def _ptr(a):
    return None if a is None else a.ctypes.data


_PATHS = {"plain": L.JF_PATH_PLAIN, "batched": L.JF_PATH_BATCHED}
_FITNESS_MODES = {"efficiency": 0, "displacement": 1}


def _choice(table, value, what):
    try:
        return table[value]
    except (KeyError, TypeError):
        raise ValueError(f"unknown {what} {value!r}; expected one of {sorted(table)}") from None


class Engine:
    """A batch of independent MLS-MPM instances on one GPU.

    ``path='batched'`` advances every instance in one persistent cluster launch
    per chunk; ``path='plain'`` launches clear / P2G / grid update / G2P per
    instance and substep, as the reference's substep() offloads do.
    ``axisym=True`` runs the axisymmetric (r, z) substep of JELLY_AXISYM=1
    (every instance; the load positions' x becomes each particle's r_ref).
    ``grad_fp64=True`` runs the differentiable rollout (grad_forward /
    grad_backward / grad_step) in FP64, the same kernels built for double.
    """

    def __init__(self, instances: Sequence[InstanceSpec], path: str = "batched", dt: float = DT,
                 glow: bool = False, device: int = 0, resort_interval: int = 64,
                 block_threads: int = 0, cluster_size: int = 0, graphs: bool = True,
                 cell_cap: int = 0, axisym: bool = False, grad_fp64: bool = False):
        self._lib = L.load()
        self.instances = list(instances)
        self.M = len(self.instances)
        self.path = path
        descs = (L.JfInstanceDesc * self.M)(*[
            L.JfInstanceDesc(s.n_slots, s.n_grid, s.n_grid_y, s.domain_height) for s in self.instances])
        flags = ((L.JF_FLAG_GLOW if glow else 0) | (0 if graphs else L.JF_FLAG_NO_GRAPHS)
                 | (L.JF_FLAG_AXISYM if axisym else 0) | (L.JF_FLAG_GRAD_FP64 if grad_fp64 else 0))
        cfg = L.JfConfig(self.M, descs, dt, _choice(_PATHS, path, "path"),
                         flags, device, resort_interval, block_threads, cluster_size, cell_cap)
        h = L._E()
        rc = self._lib.jf_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != L.JF_OK:
            raise L.JfError(rc, self._lib.jf_last_error(None).decode())
        self._h = h
        self.dt = dt
        self.nonfinite_message = ""  # set when a run reported a non-finite particle state
        self.rollouts = 0  # differentiable rollouts run (grad_forward / grad_step); a backward
        # differentiates the latest one
        self.config = dict(path=path, resort_interval=resort_interval, block_threads=block_threads,
                           cluster_size=cluster_size, graphs=graphs, cell_cap=cell_cap, axisym=axisym)

    # -- plumbing --------------------------------------------------------
    def _check(self, rc):
        if rc != L.JF_OK:
            raise L.JfError(rc, self._lib.jf_last_error(self._h).decode())

    def _check_run(self, rc):
        """As _check, but a non-finite particle state is recorded, not raised:
        results are still written and, as in the reference, an exploded
        instance simply scores as invalid.  error_flags() tells which."""
        if rc == L.JF_ERR_NONFINITE:
            self.nonfinite_message = self._lib.jf_last_error(self._h).decode()
            return
        self._check(rc)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.jf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def kernel_launches(self) -> int:
        return int(self._lib.jf_kernel_launches(self._h))

    def set_kernel_timing(self, enable: bool) -> None:
        """Bracket step / sort kernels with CUDA events (resets the totals)."""
        self._check(self._lib.jf_set_kernel_timing(self._h, 1 if enable else 0))

    def kernel_timing(self) -> dict:
        """Summed device time (ms) and launches of step and re-sort kernels."""
        sm, sl, om, ol = ctypes.c_double(), ctypes.c_int64(), ctypes.c_double(), ctypes.c_int64()
        self._check(self._lib.jf_kernel_timing(self._h, ctypes.byref(sm), ctypes.byref(sl),
                                               ctypes.byref(om), ctypes.byref(ol)))
        return {"step_ms": sm.value, "step_launches": sl.value, "sort_ms": om.value,
                "sort_launches": ol.value}

    def path_counts(self, reset: bool = False) -> dict:
        """Batched path counters: register-block scatters, per-particle scatters
        of drifted particles, gathers outside the CTA window, and particles
        beyond their cell lane's cap (scattered in the CTA's overflow pass)."""
        out = np.zeros(4, np.int64)
        self._check(self._lib.jf_path_counts(self._h, _ptr(out), 1 if reset else 0))
        return {"register_scatters": int(out[0]), "atomic_scatters": int(out[1]),
                "remote_gathers": int(out[2]), "overflow_scatters": int(out[3])}

    def layout(self) -> dict:
        """The batched launch layout the engine chose: CTAs per instance and
        threads per CTA (above 512 the cell lanes' node blocks live in TMEM)."""
        cs, bt = np.zeros(1, np.int32), np.zeros(1, np.int32)
        self._check(self._lib.jf_get_layout(self._h, _ptr(cs), _ptr(bt)))
        return {"cluster_size": int(cs[0]), "block_threads": int(bt[0])}

    def set_stream(self, stream) -> None:
        """Queue work on ``stream`` (a cudaStream_t as int, or a torch.cuda.Stream)."""
        handle = getattr(stream, "cuda_stream", stream)
        self._check(self._lib.jf_set_stream(self._h, handle))

    # -- state -------------------------------------------------------------
    def load(self, m: int, pos, material, fiber=None) -> None:
        """load_particles (mpm_sim.py:730-736) for instance ``m``."""
        n = len(material)
        pos = _f32(pos, (n, 2))
        mat = np.ascontiguousarray(material, dtype=np.int32)
        fib = None if fiber is None else _f32(fiber, (n, 2))
        self._check(self._lib.jf_load_instance(self._h, m, _ptr(pos), _ptr(mat), _ptr(fib), n))

    def set_params(self, actuation=None, contraction=None, freq=None, payload_density=None) -> None:
        arrs = [None if a is None else _f32(np.broadcast_to(np.asarray(a, np.float32), (self.M,)))
                for a in (actuation, contraction, freq, payload_density)]
        self._check(self._lib.jf_set_params(self._h, *[_ptr(a) for a in arrs]))

    def get_params(self) -> dict:
        out = {k: np.zeros(self.M, np.float32) for k in ("actuation", "contraction", "freq",
                                                          "payload_density")}
        self._check(self._lib.jf_get_params(self._h, *[_ptr(out[k]) for k in (
            "actuation", "contraction", "freq", "payload_density")]))
        return out

    @property
    def time(self) -> np.float32:
        t = ctypes.c_float()
        self._check(self._lib.jf_get_time(self._h, ctypes.byref(t)))
        return np.float32(t.value)

    @time.setter
    def time(self, t) -> None:
        self._check(self._lib.jf_set_time(self._h, float(np.float32(t))))

    def step(self, n: int = 1) -> None:
        self._check(self._lib.jf_step(self._h, int(n)))

    def sync(self, timeout: float | None = None) -> bool:
        """Waits for the queued work (ti.sync()).  With a timeout in seconds,
        waits at most that long and returns False if the work is still
        running (it is not cancelled; a later sync waits for it)."""
        if timeout is None:
            self._check_run(self._lib.jf_sync(self._h))
            return True
        rc = self._lib.jf_sync_timeout(self._h, int(max(timeout, 0.0) * 1000))
        if rc == L.JF_ERR_TIMEOUT:
            return False
        self._check_run(rc)
        return True

    # -- readback ------------------------------------------------------------
    def payload_stats(self) -> np.ndarray:
        out = np.zeros((self.M, 3), np.float64)
        self._check(self._lib.jf_payload_stats(self._h, _ptr(out)))
        return out

    def stats_any(self) -> np.ndarray:
        out = np.zeros((self.M, 3), np.float64)
        self._check(self._lib.jf_stats_any(self._h, _ptr(out)))
        return out

    def stats_raw(self) -> np.ndarray:
        """(M, 6) FP64 sums: payload [sum_y, count, sum_x], body [sum_y, count, sum_x]."""
        out = np.zeros((self.M, 6), np.float64)
        self._check(self._lib.jf_stats_raw(self._h, _ptr(out)))
        return out

    def run_headless(self, steps: int) -> np.ndarray:
        out = np.zeros((self.M, 5), np.float64)
        self._check_run(self._lib.jf_run_headless(self._h, int(steps), _ptr(out)))
        return out

    def fitness(self, results, muscle_counts, contraction=None, mode: str = "efficiency") -> np.ndarray:
        """Per-instance fitness of run_headless rows, computed on the GPU in FP64
        (evolve.py:90-124); lower is better, as CMA-ES minimises."""
        rows = np.ascontiguousarray(results, dtype=np.float64).reshape(self.M, 5)
        mus = np.ascontiguousarray(muscle_counts, dtype=np.int32).reshape(self.M)
        con = None if contraction is None else np.ascontiguousarray(contraction, dtype=np.float64).reshape(self.M)
        out = np.zeros(self.M, np.float64)
        self._check(self._lib.jf_fitness(self._h, _ptr(rows), _ptr(mus), _ptr(con),
                                         _choice(_FITNESS_MODES, mode, "fitness mode"), _ptr(out)))
        return out

    def run_episode(self, positions, materials, contraction, steps: int, fibers=None, freq=None,
                    muscle_counts=None, mode: str = "efficiency"):
        """One evaluation episode of every instance with one host round trip:
        load every instance, set the timing genes, run_headless(steps), and
        (with muscle_counts) the GPU fitness.  positions / materials / fibers:
        per-instance slot arrays (lists) or the instances' arrays back to back.
        Returns (rows (M, 5), fitness (M,) or None)."""
        S = sum(s.n_slots for s in self.instances)
        cat = lambda a, dt, w: np.ascontiguousarray(  # noqa: E731
            np.concatenate([np.asarray(x, dt).reshape(-1, w) for x in a]) if isinstance(a, (list, tuple))
            else np.asarray(a, dt).reshape(-1, w), dtype=dt)
        pos = cat(positions, np.float32, 2)
        mat = cat(materials, np.int32, 1).reshape(-1)
        if pos.shape[0] != S or mat.shape[0] != S:
            raise ValueError(f"positions and materials must cover all {S} slots")
        fib = None if fibers is None else cat(fibers, np.float32, 2)
        con = np.ascontiguousarray(contraction, dtype=np.float32).reshape(self.M)
        frq = None if freq is None else np.ascontiguousarray(freq, dtype=np.float32).reshape(self.M)
        mus = None if muscle_counts is None else np.ascontiguousarray(muscle_counts, dtype=np.int32).reshape(self.M)
        rows = np.zeros((self.M, 5), np.float64)
        fit = None if mus is None else np.zeros(self.M, np.float64)
        self._check_run(self._lib.jf_run_episode(self._h, _ptr(pos), _ptr(mat), _ptr(fib), _ptr(con), _ptr(frq),
                                                 int(steps), _ptr(mus), _choice(_FITNESS_MODES, mode, "fitness mode"),
                                                 _ptr(rows), _ptr(fit)))
        return rows, fit

    # -- differentiable rollout -----------------------------------------------
    def grad_forward(self, steps: int, checkpoint_every: int = 100) -> np.ndarray:
        """Rollout with checkpoints; returns the (M,) CoM displacement (the loss).
        An instance whose state turned non-finite (or too large for the
        fixed-point P2G) is recorded as for run_headless: error_flags() names
        it, and its loss and gradients are not to be used."""
        loss = np.zeros(self.M, np.float64)
        self.rollouts += 1
        self._check_run(self._lib.jf_grad_forward(self._h, int(steps), int(checkpoint_every), _ptr(loss)))
        return loss

    def grad_backward(self) -> dict:
        """d loss / d (actuation, contraction, freq), each (M,).  Non-finite
        adjoint states are recorded as in grad_forward."""
        g = {k: np.zeros(self.M, np.float64) for k in ("actuation", "contraction", "freq")}
        self._check_run(self._lib.jf_grad_backward(self._h, _ptr(g["actuation"]), _ptr(g["contraction"]),
                                                   _ptr(g["freq"])))
        return g

    def grad_step(self, steps: int, checkpoint_every: int = 100):
        """grad_forward + grad_backward as one CUDA graph (replayed on later
        calls with the same sizes and start time); returns (loss, gradients)."""
        loss = np.zeros(self.M, np.float64)
        g = {k: np.zeros(self.M, np.float64) for k in ("actuation", "contraction", "freq")}
        self.rollouts += 1
        self._check_run(self._lib.jf_grad_step(self._h, int(steps), int(checkpoint_every), _ptr(loss),
                                               _ptr(g["actuation"]), _ptr(g["contraction"]), _ptr(g["freq"])))
        return loss, g

    def grad_positions(self, m: int) -> np.ndarray:
        """d loss / d initial positions of instance m, (n_slots, 2) in slot order."""
        out = np.zeros((self.instances[m].n_slots, 2), np.float32)
        self._check(self._lib.jf_grad_positions(self._h, m, _ptr(out)))
        return out

    def read(self, m: int) -> dict:
        n = self.instances[m].n_slots
        d = {"x": np.zeros((n, 2), np.float32), "v": np.zeros((n, 2), np.float32),
             "C": np.zeros((n, 2, 2), np.float32), "F": np.zeros((n, 2, 2), np.float32),
             "material": np.zeros(n, np.int32), "Jp": np.zeros(n, np.float32),
             "glow": np.zeros(n, np.float32), "fiber": np.zeros((n, 2), np.float32)}
        self._check(self._lib.jf_read_particles(self._h, m, *[_ptr(d[k]) for k in (
            "x", "v", "C", "F", "material", "Jp", "glow", "fiber")]))
        return d

    def write(self, m: int, x=None, v=None, C=None, F=None, Jp=None, glow=None) -> None:
        n = self.instances[m].n_slots
        args = [None if x is None else _f32(x, (n, 2)), None if v is None else _f32(v, (n, 2)),
                None if C is None else _f32(C, (n, 2, 2)), None if F is None else _f32(F, (n, 2, 2)),
                None if Jp is None else _f32(Jp, (n,)), None if glow is None else _f32(glow, (n,))]
        self._check(self._lib.jf_write_particles(self._h, m, *[_ptr(a) for a in args]))

    def read_grid(self, m: int):
        s = self.instances[m]
        gv = np.zeros((s.n_grid, s.n_grid_y, 2), np.float32)
        gm = np.zeros((s.n_grid, s.n_grid_y), np.float32)
        self._check(self._lib.jf_read_grid(self._h, m, _ptr(gv), _ptr(gm)))
        return gv, gm

    def load_robot(self, m: int, robot_pos, robot_mat, robot_fiber=None, water_margin=0.005,
                   spacing_div=2.0):
        """Load instance m from its robot particles with the water filled on
        the GPU (make_jelly.py:336-402; jf_load_robot): the slot contents of
        tank.fill_tank without jitter.  Returns (robot particles, water
        particles) placed."""
        rp = np.ascontiguousarray(robot_pos, np.float64).reshape(-1, 2)
        n = len(rp)
        rm = np.ascontiguousarray(robot_mat, np.int32).reshape(n)
        rf = None if robot_fiber is None else _f32(robot_fiber, (n, 2))
        out = np.zeros(2, np.int32)
        self._check(self._lib.jf_load_robot(self._h, int(m), _ptr(rp) if n else None, _ptr(rm) if n else None,
                                            _ptr(rf) if n else None, n, float(water_margin), float(spacing_div),
                                            _ptr(out)))
        return int(out[0]), int(out[1])

    def write_grid(self, m: int, grid_v, grid_m) -> None:
        """grid_v (nx, ny, 2) / grid_m (nx, ny) of instance m (from_numpy)."""
        s = self.instances[m]
        gv = _f32(grid_v, (s.n_grid, s.n_grid_y, 2))
        gm = _f32(grid_m, (s.n_grid, s.n_grid_y))
        self._check(self._lib.jf_write_grid(self._h, m, _ptr(gv), _ptr(gm)))

    # --- headless renderer (mpm_sim.py:343-712) --------------------------------
    def frame_create(self, video_res: int) -> None:
        """Allocate (or resize) the device frame buffer and clear it to 0."""
        self._check(self._lib.jf_frame_create(self._h, int(video_res)))
        self.frame_res = int(video_res)

    def frame_clear(self, value: float = 0.0) -> None:
        self._check(self._lib.jf_frame_clear(self._h, float(value)))

    def render_abyss(self, res_sub, grid_side, radius, hue, muscle_hue, water_mode=0) -> None:
        h = _f32(hue, (self.M,))
        mh = _f32(muscle_hue, (self.M,))
        self._check(self._lib.jf_render_abyss(self._h, int(res_sub), int(grid_side), float(radius), _ptr(h),
                                              _ptr(mh), int(water_mode)))

    def render_flat(self, res_sub, grid_side, radius, material, r, g, b) -> None:
        self._check(self._lib.jf_render_flat(self._h, int(res_sub), int(grid_side), float(radius), int(material),
                                             float(r), float(g), float(b)))

    def render_vorticity_overlay(self, res_sub, grid_side, vort_scale) -> None:
        self._check(self._lib.jf_render_vorticity_overlay(self._h, int(res_sub), int(grid_side),
                                                          float(vort_scale)))

    def compute_vorticity(self, vort_scale) -> None:
        self._check(self._lib.jf_compute_vorticity(self._h, float(vort_scale)))

    def render_vorticity(self, res_sub, grid_side, alpha, style) -> None:
        """style: L.JF_VORT_RDBU, JF_VORT_HUESHIFT or JF_VORT_WHITE."""
        self._check(self._lib.jf_render_vorticity(self._h, int(res_sub), int(grid_side), float(alpha),
                                                  int(style)))

    def tone_map(self) -> None:
        self._check(self._lib.jf_tone_map(self._h))

    def read_frame(self) -> np.ndarray:
        """(video_res, video_res, 3) float32, frame_buffer.to_numpy() layout."""
        res = getattr(self, "frame_res", 0)
        out = np.zeros((max(res, 1), max(res, 1), 3), np.float32)
        self._check(self._lib.jf_read_frame(self._h, _ptr(out)))
        return out

    def read_vorticity(self, m: int) -> np.ndarray:
        s = self.instances[m]
        out = np.zeros((s.n_grid, s.n_grid_y), np.float32)
        self._check(self._lib.jf_read_vorticity(self._h, m, _ptr(out)))
        return out

    def error_flags(self) -> np.ndarray:
        out = np.zeros(self.M, np.int32)
        self._check(self._lib.jf_error_flags(self._h, _ptr(out)))
        return out

    def clear_error_flags(self) -> None:
        self._check(self._lib.jf_clear_error_flags(self._h))
