"""Drop-in replacement of jellyfih's mpm_sim module, backed by libjellyfih.so.

Importing it does what importing the reference module does (mpm_sim.py:6-149):
it reads JELLY_INSTANCES, JELLY_PARTICLES, JELLY_GRID_Y and JELLY_DOMAIN_H,
allocates every instance on the GPU, and sets the per-instance defaults.  The
module-level names callers use are all here: the constants, the fields
(``x``, ``v``, ``C``, ``F``, ``material``, ``Jp``, ``grid_v``, ``grid_m``,
``sim_time``, ``fitness_buffer``, ``instance_*``, ``visual_glow``) with
``[i]`` / ``[None]`` access, ``to_numpy()``, ``from_numpy()`` and ``fill()``,
and the functions ``substep``, ``load_particles``, ``get_payload_stats``,
``_get_stats_any``, ``run_batch_headless``, ``clear_fitness_buffer``,
``compute_payload_stats`` and ``compute_body_stats``.  ``ti.sync()`` is
available as ``mpm_sim.ti.sync()``.

Engine selection (not in the reference): JELLY_B200_PATH = batched (default)
or plain; JELLY_B200_GLOW = 1 keeps the render-only visual_glow updated.
JELLY_AXISYM=1 selects the axisymmetric (r, z) substep, as in the reference;
its r_ref (the load radius) lives inside the engine and is not exposed as a
field.  The renderer (mpm_sim.py:343-712) runs as CUDA kernels into a device
frame buffer: ``clear_frame_buffer``, ``clear_frame_buffer_white``,
``render_frame_abyss``, ``render_flat_pass``, ``render_vorticity_overlay``,
``compute_vorticity_grid``, ``render_vorticity_rdbu`` / ``_hueshift`` /
``_white``, ``tone_map_and_encode``; ``frame_buffer`` and ``vort_grid`` read
back with ``to_numpy()``.
"""
from __future__ import annotations

import math
import os

import numpy as np

from .engine import Engine, InstanceSpec

# --- configuration (mpm_sim.py:11-22) ---
n_instances = int(os.environ.get("JELLY_INSTANCES", "16"))
quality = 1
n_particles = int(os.environ.get("JELLY_PARTICLES", "80000"))
n_grid = 128 * quality
n_grid_y = int(os.environ.get("JELLY_GRID_Y", str(n_grid)))
domain_height = float(os.environ.get("JELLY_DOMAIN_H", "1.0"))
axisym = os.environ.get("JELLY_AXISYM", "0") == "1"  # axisymmetric (r, z) MPM, mpm_sim.py:17
dx, inv_dx = 1 / n_grid, float(n_grid)
dt = 2e-5 / quality
p_vol = (dx * 0.5) ** 2
p_rho = 1
p_mass = p_vol * p_rho

# --- material constants (mpm_sim.py:24-49) ---
E_base = 0.1e4
nu_base = 0.2
mu_0_base = E_base / (2 * (1 + nu_base))
lambda_0_base = E_base * nu_base / ((1 + nu_base) * (1 - 2 * nu_base))
E_jelly = 0.7e3
nu_jelly = 0.3
mu_jelly = E_jelly / (2 * (1 + nu_jelly))
lambda_jelly = E_jelly * nu_jelly / ((1 + nu_jelly) * (1 - 2 * nu_jelly))
E_payload = 2.0e5
nu_payload = 0.2
mu_payload = E_payload / (2 * (1 + nu_payload))
lambda_payload = E_payload * nu_payload / ((1 + nu_payload) * (1 - 2 * nu_payload))
water_lambda = 100000.0
gravity = 10.0
actuation_freq = 1
actuation_strength = 500.0
ACT_CONTRACTION_END = 0.2
ACT_RELAXATION_END = 0.6

WEB_PALETTE = [
    (0, 0.933, 0.949, 0.957),
    (1, 0.678, 0.882, 0.875),
    (3, 0.976, 0.757, 0.765),
    (2, 0.961, 0.824, 0.576),
]
video_res = 1024
grid_side = int(math.ceil(math.sqrt(n_instances)))
res_sub = video_res // grid_side

print(f"Allocating {n_instances} instances with {n_particles} particles each..."
      + (" [AXISYM mode: JELLY_AXISYM=1]" if axisym else ""))
_engine = Engine([InstanceSpec(n_particles, n_grid, n_grid_y, domain_height)] * n_instances,
                 path=os.environ.get("JELLY_B200_PATH", "batched"), dt=dt,
                 glow=os.environ.get("JELLY_B200_GLOW", "0") == "1", axisym=axisym)


def engine() -> Engine:
    """The process-wide engine behind this module."""
    return _engine


class _Ti:
    """The part of the taichi namespace that callers reach through mpm_sim.ti."""

    @staticmethod
    def sync():
        _engine.sync()


ti = _Ti()


# --- fields -----------------------------------------------------------------
class _ParamField:
    """A per-instance parameter (mpm_sim.py:116-149), mirrored on the host."""

    def __init__(self, name):
        self.name = name
        self.shape = (n_instances,)

    def to_numpy(self):
        return _engine.get_params()[self.name].copy()

    def from_numpy(self, arr):
        _engine.set_params(**{self.name: np.asarray(arr, np.float32).reshape(n_instances)})

    def fill(self, value):
        _engine.set_params(**{self.name: np.full(n_instances, value, np.float32)})

    def __getitem__(self, i):
        return float(self.to_numpy()[int(i)])

    def __setitem__(self, i, value):
        arr = self.to_numpy()
        arr[int(i)] = value
        self.from_numpy(arr)


class _HostField:
    """Render-only per-instance values kept on the host (hues, colour mode)."""

    def __init__(self, shape, value, dtype=np.float32):
        self.shape = shape
        self._a = np.full(shape, value, dtype)

    def to_numpy(self):
        return self._a.copy()

    def from_numpy(self, arr):
        self._a[...] = arr

    def fill(self, value):
        self._a[...] = value

    def __getitem__(self, i):
        return self._a[() if i is None else i]

    def __setitem__(self, i, value):
        self._a[() if i is None else i] = value


class _TimeField:
    """sim_time (mpm_sim.py:95): FP32 scalar, sim_time[None]."""
    shape = ()

    def __getitem__(self, key):
        return float(_engine.time)

    def __setitem__(self, key, value):
        _engine.time = value

    def to_numpy(self):
        return np.array(_engine.time, np.float32)

    def from_numpy(self, arr):
        _engine.time = float(np.asarray(arr))

    def fill(self, value):
        _engine.time = value


_PARTICLE_SHAPES = {"x": (2,), "v": (2,), "C": (2, 2), "F": (2, 2), "material": (), "Jp": (),
                    "glow": (), "fiber": (2,)}


class _ParticleField:
    """A per-particle field (n_instances, n_particles, ...) read and written
    through the engine in slot order."""

    def __init__(self, key):
        self.key = key
        self.shape = (n_instances, n_particles)

    def to_numpy(self):
        return np.stack([_engine.read(m)[self.key] for m in range(n_instances)])

    def from_numpy(self, arr):
        if self.key in ("material", "fiber"):
            raise NotImplementedError(f"{self.key}: set it through load_particles()")
        arr = np.asarray(arr, np.float32)
        for m in range(n_instances):
            _engine.write(m, **{self.key: arr[m]})

    def fill(self, value):
        self.from_numpy(np.full(self.shape + _PARTICLE_SHAPES[self.key], value, np.float32))

    def __getitem__(self, key):
        m, p = key
        return _engine.read(int(m))[self.key][int(p)]

    def __setitem__(self, key, value):
        m, p = int(key[0]), int(key[1])
        if self.key in ("material", "fiber"):
            raise NotImplementedError(f"{self.key}: set it through load_particles()")
        cur = _engine.read(m)[self.key]
        cur[p] = value
        _engine.write(m, **{self.key: cur})


class _GridField:
    """grid_v / grid_m (mpm_sim.py:92-93) of the last substep, (M, nx, ny[, 2])."""

    def __init__(self, idx):
        self.idx = idx
        self.shape = (n_instances, n_grid, n_grid_y)

    def to_numpy(self):
        return np.stack([_engine.read_grid(m)[self.idx] for m in range(n_instances)])

    def __getitem__(self, key):
        m = int(key[0])
        return _engine.read_grid(m)[self.idx][tuple(int(k) for k in key[1:])]


class _FitnessBuffer(_HostField):
    """fitness_buffer (mpm_sim.py:109): [sum_y, count, sum_x] per instance."""

    def __init__(self):
        super().__init__((n_instances, 3), 0.0)


x = _ParticleField("x")
v = _ParticleField("v")
C = _ParticleField("C")
F = _ParticleField("F")
material = _ParticleField("material")
Jp = _ParticleField("Jp")
visual_glow = _ParticleField("glow")
fiber_dir = _ParticleField("fiber")
r_ref = None  # axisymmetric load radius (mpm_sim.py:131): kept inside the engine
grid_v = _GridField(0)
grid_m = _GridField(1)
sim_time = _TimeField()
fitness_buffer = _FitnessBuffer()
instance_actuation = _ParamField("actuation")
instance_act_contraction = _ParamField("contraction")
instance_freq = _ParamField("freq")
instance_payload_density = _ParamField("payload_density")
instance_hue = _HostField((n_instances,), 0.55)
instance_muscle_hue = _HostField((n_instances,), (0.55 + 0.15) % 1.0)
water_angle_color = _HostField((), 0, np.int32)


# --- kernels ------------------------------------------------------------------
def substep():
    """One MLS-MPM substep of every instance (mpm_sim.py:153-340)."""
    _engine.step(1)


def load_particles(instance, pos_np, mat_np, fiber_np=None):
    """Reset one instance (mpm_sim.py:730-736)."""
    if fiber_np is None:
        fiber_np = np.zeros((n_particles, 2), dtype=np.float32)
        fiber_np[:, 1] = 1.0
    _engine.load(int(instance), pos_np, mat_np, fiber_np)


def clear_fitness_buffer():
    """mpm_sim.py:740-744."""
    fitness_buffer.fill(0.0)


def compute_payload_stats():
    """Adds payload [sum_y, count, sum_x] to fitness_buffer (mpm_sim.py:746-753)."""
    fitness_buffer.from_numpy(fitness_buffer.to_numpy() + _engine.stats_raw()[:, 0:3])


def compute_body_stats():
    """Adds jelly + muscle [sum_y, count, sum_x] to fitness_buffer (mpm_sim.py:755-762)."""
    fitness_buffer.from_numpy(fitness_buffer.to_numpy() + _engine.stats_raw()[:, 3:6])


def get_payload_stats():
    """(n_instances, 3) [com_y, com_x, count] of the payload (mpm_sim.py:764-777)."""
    return _engine.payload_stats()


def _get_stats_any():
    """Payload CoM, or jelly + muscle CoM without payload (mpm_sim.py:779-800)."""
    return _engine.stats_any()


def run_batch_headless(steps):
    """(n_instances, 5) [init_y, init_x, final_y, final_x, valid] (mpm_sim.py:802-834)."""
    return _engine.run_headless(int(steps))


# --- headless renderer (mpm_sim.py:343-712) ----------------------------------
# The frame lives on the GPU (allocated at the first render call, video_res x
# video_res); frame_buffer.to_numpy() reads it back.  hsv2rgb is a device
# function of the kernels, not a Python-scope call, in the reference too.
def _frame():
    if getattr(_engine, "frame_res", 0) != video_res:
        _engine.frame_create(video_res)


class _FrameBuffer:
    """frame_buffer (mpm_sim.py:96): (video_res, video_res, 3) float32."""

    @property
    def shape(self):
        return (video_res, video_res, 3)

    def to_numpy(self):
        _frame()
        return _engine.read_frame()


class _VortGrid:
    """vort_grid (mpm_sim.py:106): (n_instances, n_grid, n_grid_y) float32."""
    shape = (n_instances, n_grid, n_grid_y)

    def to_numpy(self):
        return np.stack([_engine.read_vorticity(m) for m in range(n_instances)])


frame_buffer = _FrameBuffer()
vort_grid = _VortGrid()


def clear_frame_buffer():
    """mpm_sim.py:361-364."""
    _frame()
    _engine.frame_clear(0.0)


def clear_frame_buffer_white():
    """mpm_sim.py:483-486."""
    _frame()
    _engine.frame_clear(0.98)


def tone_map_and_encode():
    """mpm_sim.py:366-383."""
    _frame()
    _engine.tone_map()


def render_frame_abyss(p_res_sub, p_grid_side, radius):
    """mpm_sim.py:385-481."""
    _frame()
    _engine.render_abyss(p_res_sub, p_grid_side, radius, instance_hue.to_numpy(),
                         instance_muscle_hue.to_numpy(), int(water_angle_color[None]))


def render_flat_pass(p_res_sub, p_grid_side, radius, target_mat, cr, cg, cb):
    """mpm_sim.py:489-517."""
    _frame()
    _engine.render_flat(p_res_sub, p_grid_side, radius, target_mat, cr, cg, cb)


def render_vorticity_overlay(p_res_sub, p_grid_side, vort_scale):
    """mpm_sim.py:520-558."""
    _frame()
    _engine.render_vorticity_overlay(p_res_sub, p_grid_side, vort_scale)


def compute_vorticity_grid(vort_scale):
    """mpm_sim.py:561-579."""
    _engine.compute_vorticity(vort_scale)


def render_vorticity_rdbu(p_res_sub, p_grid_side, alpha_max):
    """mpm_sim.py:582-625."""
    _frame()
    _engine.render_vorticity(p_res_sub, p_grid_side, alpha_max, 0)


def render_vorticity_hueshift(p_res_sub, p_grid_side, strength):
    """mpm_sim.py:628-670."""
    _frame()
    _engine.render_vorticity(p_res_sub, p_grid_side, strength, 1)


def render_vorticity_white(p_res_sub, p_grid_side, alpha_max):
    """mpm_sim.py:673-711."""
    _frame()
    _engine.render_vorticity(p_res_sub, p_grid_side, alpha_max, 2)
