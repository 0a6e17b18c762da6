"""The C-ABI library loads and exports every symbol include/jellyfih.h declares.

CPU only: nothing here calls into CUDA; jf_create is only driven down the
argument checks that return before any device call.
"""
import ctypes
import os
import re

import pytest

from jellyfih_b200 import _lib as L

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "jellyfih.h")


def _declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|const char\*)\s+(jf_\w+)\s*\(", text, re.M)))


@pytest.fixture(scope="module")
def lib():
    from jellyfih_b200 import build
    build.build()
    return L.load()


def test_every_declared_symbol_is_exported(lib):
    names = _declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
        assert n in L.EXPORTS, f"{n} missing from the ctypes table"


def test_ctypes_table_matches_header():
    assert sorted(L.EXPORTS) == _declared()


def test_version(lib):
    assert lib.jf_version().startswith(b"jellyfih-b200")


def test_create_rejects_bad_config_before_touching_the_device(lib):
    h = L._E()
    cfg = L.JfConfig(0, None, 2e-5, 0, 0, 0, 0, 0, 0)
    assert lib.jf_create(ctypes.byref(cfg), ctypes.byref(h)) == L.JF_ERR_INVALID
    assert b"n_instances" in lib.jf_last_error(None)
    descs = (L.JfInstanceDesc * 1)(L.JfInstanceDesc(10, 128, 128, 1.0))
    cfg = L.JfConfig(1, descs, 2e-5, 7, 0, 0, 0, 0, 0)
    assert lib.jf_create(ctypes.byref(cfg), ctypes.byref(h)) == L.JF_ERR_INVALID
    assert lib.jf_create(None, ctypes.byref(h)) == L.JF_ERR_INVALID


def test_null_handle_calls_fail_cleanly(lib):
    assert lib.jf_step(None, 1) == L.JF_ERR_INVALID
    assert lib.jf_last_error(None) == b"NULL engine handle"
    assert lib.jf_sync(None) == L.JF_ERR_INVALID
    assert lib.jf_sync_timeout(None, 10) == L.JF_ERR_INVALID
    assert lib.jf_payload_stats(None, None) == L.JF_ERR_INVALID
    assert lib.jf_destroy(None) == L.JF_ERR_INVALID
    assert lib.jf_kernel_launches(None) == -1


def test_null_handle_render_calls_fail_cleanly(lib):
    bad = L.JF_ERR_INVALID
    assert lib.jf_frame_create(None, 64) == bad
    assert lib.jf_frame_clear(None, 0.0) == bad
    assert lib.jf_render_abyss(None, 64, 1, 1.5, None, None, 2) == bad
    assert lib.jf_render_flat(None, 64, 1, 1.0, 0, 1.0, 1.0, 1.0) == bad
    assert lib.jf_render_vorticity_overlay(None, 64, 1, 0.001) == bad
    assert lib.jf_compute_vorticity(None, 0.003) == bad
    assert lib.jf_render_vorticity(None, 64, 1, 0.6, L.JF_VORT_RDBU) == bad
    assert lib.jf_tone_map(None) == bad
    assert lib.jf_read_frame(None, None) == bad
    assert lib.jf_read_vorticity(None, 0, None) == bad
    assert lib.jf_write_grid(None, 0, None, None) == bad
    assert lib.jf_load_robot(None, 0, None, None, None, 0, 0.005, 2.0, None) == bad


def test_struct_layout():
    assert ctypes.sizeof(L.JfInstanceDesc) == 16
    assert L.JfConfig.instances.offset == 8 and L.JfConfig.dt.offset == 16
    assert ctypes.sizeof(L.JfConfig) == 56


def test_engine_rejects_unknown_path_before_touching_the_device(lib):
    from jellyfih_b200 import Engine, InstanceSpec
    with pytest.raises(ValueError, match="unknown path 'gpu'"):
        Engine([InstanceSpec(16)], path="gpu")
