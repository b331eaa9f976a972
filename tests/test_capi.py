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


def test_no_device_fails_loudly():
    """Without a usable CUDA device every path fails with an error, through the
    C ABI, the Python API and the C++ adapter alike: there is no CPU fallback."""
    import os
    import subprocess

    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from raydemo_b200 import api

    with pytest.raises(RuntimeError):
        api.Renderer(8, 8)
    check = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "adapter_check")
    if os.path.exists(check):
        out = subprocess.run([check, "8", "8", "1", "0"], capture_output=True, text=True, timeout=300)
        assert out.returncode == 2 and '"error"' in out.stdout


def test_unknown_handles_are_rejected():
    """A pointer that ray_create_* did not return is refused before anything
    dereferences it (no device needed)."""
    L = capi.lib()
    bogus = C.c_void_p(0x1234560)
    assert L.ray_scene_commit(bogus) == capi.RAY_ERR_INVALID_ARG
    assert b"handle" in L.ray_last_error()
    assert L.ray_destroy_scene(bogus) == capi.RAY_ERR_INVALID_ARG
    assert L.ray_resize(bogus, 8, 8) == capi.RAY_ERR_INVALID_ARG
    assert L.ray_destroy_scene(None) == capi.RAY_OK
