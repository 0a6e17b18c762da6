"""ctypes binding of libjellyfih.so (include/jellyfih.h).

The library is the only compute path: there is no CPU fallback, and loading
fails loudly when the shared object has not been built.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libjellyfih.so")

JF_OK = 0
JF_ERR_INVALID = 1
JF_ERR_CUDA = 2
JF_ERR_NONFINITE = 3
JF_ERR_UNSUPPORTED = 4
JF_ERR_TIMEOUT = 5
JF_PATH_PLAIN = 0
JF_PATH_BATCHED = 1
JF_FLAG_GLOW = 1
JF_FLAG_NO_GRAPHS = 2
JF_FLAG_AXISYM = 4
JF_FLAG_GRAD_FP64 = 8
JF_VORT_RDBU = 0
JF_VORT_HUESHIFT = 1
JF_VORT_WHITE = 2
JF_NOALLOC_MAX_NODES = 32768


class JfInstanceDesc(ctypes.Structure):
    _fields_ = [("n_slots", ctypes.c_int32), ("n_grid", ctypes.c_int32),
                ("n_grid_y", ctypes.c_int32), ("domain_height", ctypes.c_float)]


class JfConfig(ctypes.Structure):
    _fields_ = [("n_instances", ctypes.c_int32), ("instances", ctypes.POINTER(JfInstanceDesc)),
                ("dt", ctypes.c_double), ("path", ctypes.c_int32), ("flags", ctypes.c_uint32),
                ("device", ctypes.c_int32), ("resort_interval", ctypes.c_int32),
                ("block_threads", ctypes.c_int32), ("cluster_size", ctypes.c_int32),
                ("cell_cap", ctypes.c_int32)]


_P = ctypes.c_void_p
_E = ctypes.c_void_p  # jf_engine*
# name -> (restype, argtypes); every symbol include/jellyfih.h declares
EXPORTS = {
    "jf_create": (ctypes.c_int, [ctypes.POINTER(JfConfig), ctypes.POINTER(_E)]),
    "jf_destroy": (ctypes.c_int, [_E]),
    "jf_last_error": (ctypes.c_char_p, [_E]),
    "jf_version": (ctypes.c_char_p, []),
    "jf_set_stream": (ctypes.c_int, [_E, _P]),
    "jf_load_instance": (ctypes.c_int, [_E, ctypes.c_int32, _P, _P, _P, ctypes.c_int32]),
    "jf_set_params": (ctypes.c_int, [_E, _P, _P, _P, _P]),
    "jf_get_params": (ctypes.c_int, [_E, _P, _P, _P, _P]),
    "jf_set_time": (ctypes.c_int, [_E, ctypes.c_float]),
    "jf_get_time": (ctypes.c_int, [_E, ctypes.POINTER(ctypes.c_float)]),
    "jf_step": (ctypes.c_int, [_E, ctypes.c_int64]),
    "jf_sync": (ctypes.c_int, [_E]),
    "jf_sync_timeout": (ctypes.c_int, [_E, ctypes.c_int64]),
    "jf_payload_stats": (ctypes.c_int, [_E, _P]),
    "jf_stats_any": (ctypes.c_int, [_E, _P]),
    "jf_stats_raw": (ctypes.c_int, [_E, _P]),
    "jf_run_headless": (ctypes.c_int, [_E, ctypes.c_int64, _P]),
    "jf_fitness": (ctypes.c_int, [_E, _P, _P, _P, ctypes.c_int32, _P]),
    "jf_run_episode": (ctypes.c_int, [_E, _P, _P, _P, _P, _P, ctypes.c_int64, _P, ctypes.c_int32, _P, _P]),
    "jf_grad_forward": (ctypes.c_int, [_E, ctypes.c_int64, ctypes.c_int32, _P]),
    "jf_grad_backward": (ctypes.c_int, [_E, _P, _P, _P]),
    "jf_grad_positions": (ctypes.c_int, [_E, ctypes.c_int32, _P]),
    "jf_grad_step": (ctypes.c_int, [_E, ctypes.c_int64, ctypes.c_int32, _P, _P, _P, _P]),
    "jf_read_particles": (ctypes.c_int, [_E, ctypes.c_int32, _P, _P, _P, _P, _P, _P, _P, _P]),
    "jf_write_particles": (ctypes.c_int, [_E, ctypes.c_int32, _P, _P, _P, _P, _P, _P]),
    "jf_read_grid": (ctypes.c_int, [_E, ctypes.c_int32, _P, _P]),
    "jf_write_grid": (ctypes.c_int, [_E, ctypes.c_int32, _P, _P]),
    "jf_load_robot": (ctypes.c_int, [_E, ctypes.c_int32, _P, _P, _P, ctypes.c_int32, ctypes.c_double,
                                     ctypes.c_double, _P]),
    "jf_frame_create": (ctypes.c_int, [_E, ctypes.c_int32]),
    "jf_frame_clear": (ctypes.c_int, [_E, ctypes.c_float]),
    "jf_render_abyss": (ctypes.c_int, [_E, ctypes.c_int32, ctypes.c_int32, ctypes.c_float, _P, _P,
                                       ctypes.c_int32]),
    "jf_render_flat": (ctypes.c_int, [_E, ctypes.c_int32, ctypes.c_int32, ctypes.c_float, ctypes.c_int32,
                                      ctypes.c_float, ctypes.c_float, ctypes.c_float]),
    "jf_render_vorticity_overlay": (ctypes.c_int, [_E, ctypes.c_int32, ctypes.c_int32, ctypes.c_float]),
    "jf_compute_vorticity": (ctypes.c_int, [_E, ctypes.c_float]),
    "jf_render_vorticity": (ctypes.c_int, [_E, ctypes.c_int32, ctypes.c_int32, ctypes.c_float, ctypes.c_int32]),
    "jf_tone_map": (ctypes.c_int, [_E]),
    "jf_read_frame": (ctypes.c_int, [_E, _P]),
    "jf_read_vorticity": (ctypes.c_int, [_E, ctypes.c_int32, _P]),
    "jf_error_flags": (ctypes.c_int, [_E, _P]),
    "jf_clear_error_flags": (ctypes.c_int, [_E]),
    "jf_kernel_launches": (ctypes.c_int64, [_E]),
    "jf_substep_noalloc": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                          ctypes.c_float, ctypes.c_double, ctypes.c_float,
                                          ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                          ctypes.c_float] + [_P] * 9),
    "jf_path_counts": (ctypes.c_int, [_E, _P, ctypes.c_int32]),
    "jf_get_layout": (ctypes.c_int, [_E, _P, _P]),
    "jf_set_kernel_timing": (ctypes.c_int, [_E, ctypes.c_int32]),
    "jf_kernel_timing": (ctypes.c_int, [_E, ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ctypes.c_int64),
                                        ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ctypes.c_int64)]),
}

_lib = None


class JfError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"jellyfih error {code}: {msg}")
        self.code = code


def load(build_if_missing: bool = False):
    """Load libjellyfih.so; raises if it is missing (no fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if build_if_missing:
            from . import build
            build.build()
        else:
            raise RuntimeError(
                f"{LIB_PATH} is not built; run `python -m jellyfih_b200.build` (nvcc, sm_100a)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
