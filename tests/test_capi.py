"""The C ABI library loads and exports every entry point include/raygpu.h
declares (CPU only: nothing here launches a kernel)."""
import ctypes as C

import pytest

from raydemo_b200 import capi


def test_header_declares_entry_points():
    syms = capi.declared_symbols()
    assert "ray_scene_trace_closest" in syms and "ray_render" in syms and len(syms) >= 40


def test_library_exports_all_declared_symbols():
    L = capi.lib()
    missing = [s for s in capi.declared_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(capi.declared_symbols()) <= set(capi._SIGS)


def test_struct_sizes():
    assert C.sizeof(capi.Pixel) == 16
    assert C.sizeof(capi.TraceInfo) == 24


def test_null_arguments_are_rejected():
    L = capi.lib()
    assert L.ray_create_renderer(None, None) == capi.RAY_ERR_INVALID_ARG
    assert b"null" in L.ray_last_error()
    assert L.ray_scene_trace_closest(None, None, 0, None, None, 0, None) == capi.RAY_ERR_INVALID_ARG
