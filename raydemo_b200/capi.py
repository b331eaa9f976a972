"""ctypes binding of libraygpu.so (the C ABI declared in include/raygpu.h).

There is no CPU fallback: if the CUDA library cannot be loaded, `lib()`
raises. Struct layouts mirror include/raygpu.h field for field.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libraygpu.so")
HEADER = os.path.join(HERE, "..", "include", "raygpu.h")

RAY_OK = 0
RAY_ERR_INVALID_ARG = -1
RAY_ERR_CUDA = -2
RAY_ERR_OUT_OF_MEMORY = -3
RAY_ERR_NOT_FOUND = -4
RAY_ERR_STACK_OVERFLOW = -5
RAY_ERR_TIMEOUT = -6
RAY_ERR_UNSUPPORTED = -7
RAY_INVALID_INDEX = 0xFFFFFFFF
RAY_MEM_HOST = 0
RAY_MEM_DEVICE = 1
RAY_MAT_PRINCIPLED = 6
RAY_LIGHT_QUAD = 3
RAY_LIGHT_SUN = 4

f3 = C.c_float * 3


class Settings(C.Structure):
    _fields_ = [("w", C.c_int), ("h", C.c_int), ("use_wide_bvh", C.c_int), ("device", C.c_int)]


class Rect(C.Structure):
    _fields_ = [("x", C.c_int), ("y", C.c_int), ("w", C.c_int), ("h", C.c_int)]


class Region(C.Structure):
    _fields_ = [("rect", Rect), ("iteration", C.c_int)]


class Pixel(C.Structure):
    _fields_ = [("r", C.c_float), ("g", C.c_float), ("b", C.c_float), ("a", C.c_float)]


class Stats(C.Structure):
    _fields_ = [(n, C.c_ulonglong) for n in ("time_primary_ray_gen_us", "time_primary_trace_us", "time_primary_shade_us",
                                              "time_secondary_sort_us", "time_secondary_trace_us", "time_secondary_shade_us")]


class MatDesc(C.Structure):
    _fields_ = [("type", C.c_int), ("main_color", f3), ("main_texture", C.c_uint32), ("normal_map", C.c_uint32),
                ("mix_materials", C.c_uint32 * 2), ("roughness", C.c_float), ("strength", C.c_float), ("fresnel", C.c_float),
                ("int_ior", C.c_float), ("ext_ior", C.c_float), ("metallic", C.c_float)]


class ShapeDesc(C.Structure):
    _fields_ = [("mat_index", C.c_uint32), ("back_mat_index", C.c_uint32), ("vtx_start", C.c_uint64), ("vtx_count", C.c_uint64)]


class MeshDesc(C.Structure):
    _fields_ = [("prim_type", C.c_int), ("layout", C.c_int), ("vtx_attrs", C.c_void_p), ("vtx_attrs_count", C.c_uint64),
                ("vtx_indices", C.c_void_p), ("vtx_indices_count", C.c_uint64), ("base_vertex", C.c_int),
                ("shapes", C.POINTER(ShapeDesc)), ("shapes_count", C.c_uint64), ("allow_spatial_splits", C.c_int),
                ("use_fast_bvh_build", C.c_int)]


class TexDesc(C.Structure):
    _fields_ = [("data", C.c_void_p), ("w", C.c_int), ("h", C.c_int), ("is_srgb", C.c_int), ("generate_mipmaps", C.c_int)]


class LightDesc(C.Structure):
    _fields_ = [("type", C.c_int), ("position", f3), ("radius", C.c_float), ("color", f3), ("direction", f3), ("angle", C.c_float),
                ("edge_u", f3), ("edge_v", f3)]


class CameraDesc(C.Structure):
    _fields_ = [("type", C.c_int), ("filter", C.c_int), ("dtype", C.c_int), ("origin", f3), ("fwd", f3), ("up", f3),
                ("fov", C.c_float), ("gamma", C.c_float), ("focus_distance", C.c_float), ("focus_factor", C.c_float),
                ("mi_index", C.c_uint32), ("uv_index", C.c_uint32)] + [
                   (n, C.c_int) for n in ("lighting_only", "skip_direct_lighting", "skip_indirect_lighting", "no_background", "clamp",
                                          "output_sh", "use_coherent_sampling", "max_diff_depth", "max_glossy_depth",
                                          "max_refr_depth", "max_transp_depth", "max_total_depth", "termination_start_depth")]


class EnvDesc(C.Structure):
    _fields_ = [("env_col", f3), ("env_clamp", C.c_float), ("env_map", C.c_uint32)]


class TraceInfo(C.Structure):
    _fields_ = [("error_flags", C.c_uint32), ("node_visits", C.c_uint64), ("tri_tests", C.c_uint64)]


class FrameInfo(C.Structure):
    _fields_ = [("error_flags", C.c_uint32), ("kernel", C.c_int32), ("rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("sort_mask", C.c_uint32), ("trace_one_tri", C.c_uint32), ("trace_variant", C.c_int32), ("trace_refill", C.c_int32),
                ("trace_block", C.c_int32), ("trace_stack", C.c_int32)]


class DiffParams(C.Structure):
    _fields_ = [("albedo", C.c_void_p), ("albedo_w", C.c_int), ("albedo_h", C.c_int), ("roughness", C.c_void_p), ("n_roughness", C.c_int),
                ("material_slot", C.POINTER(C.c_int32)), ("n_materials", C.c_int), ("roughness_sampling", C.c_void_p),
                ("color", C.c_void_p)]


class TraceTuning(C.Structure):
    _fields_ = [("kernel", C.c_int), ("refill_min", C.c_int), ("deep_stack", C.c_int), ("reorder", C.c_int), ("reorder_bits", C.c_int),
                ("block", C.c_int), ("smem_stack", C.c_int), ("stream_hint", C.c_int), ("l2_persist", C.c_int),
                ("instance_tree", C.c_int)]


class InstanceTreeInfo(C.Structure):
    _fields_ = [("instances", C.c_uint32), ("refit", C.c_int), ("ms", C.c_double)]


class BvhInfo(C.Structure):
    _fields_ = [("nodes", C.c_uint32), ("tris", C.c_uint32), ("depth", C.c_uint32), ("root", C.c_uint32), ("bbox_min", f3),
                ("bbox_max", f3)]


class RayError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"raygpu error {code}: {msg}")
        self.code = code


_lib = None
_lock = threading.Lock()

_P = C.c_void_p
_U32P = C.POINTER(C.c_uint32)
_SIGS = {
    "ray_last_error": ([], C.c_char_p),
    "ray_version": ([], C.c_int),
    "ray_create_renderer": ([C.POINTER(Settings), C.POINTER(_P)], C.c_int),
    "ray_destroy_renderer": ([_P], C.c_int),
    "ray_renderer_type": ([_P, C.POINTER(C.c_int)], C.c_int),
    "ray_renderer_size": ([_P, C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
    "ray_resize": ([_P, C.c_int, C.c_int], C.c_int),
    "ray_clear": ([_P, C.POINTER(Pixel)], C.c_int),
    "ray_create_scene": ([_P, C.POINTER(_P)], C.c_int),
    "ray_destroy_scene": ([_P], C.c_int),
    "ray_render": ([_P, _P, C.POINTER(Region)], C.c_int),
    "ray_get_pixels": ([_P, C.POINTER(_P), C.c_int], C.c_int),
    "ray_get_sh_data": ([_P, C.POINTER(_P)], C.c_int),
    "ray_get_stats": ([_P, C.POINTER(Stats)], C.c_int),
    "ray_reset_stats": ([_P], C.c_int),
    "ray_scene_get_environment": ([_P, C.POINTER(EnvDesc)], C.c_int),
    "ray_scene_set_environment": ([_P, C.POINTER(EnvDesc)], C.c_int),
    "ray_scene_add_texture": ([_P, C.POINTER(TexDesc), _U32P], C.c_int),
    "ray_scene_remove_texture": ([_P, C.c_uint32], C.c_int),
    "ray_scene_add_material": ([_P, C.POINTER(MatDesc), _U32P], C.c_int),
    "ray_scene_remove_material": ([_P, C.c_uint32], C.c_int),
    "ray_scene_add_mesh": ([_P, C.POINTER(MeshDesc), _U32P], C.c_int),
    "ray_scene_remove_mesh": ([_P, C.c_uint32], C.c_int),
    "ray_scene_add_light": ([_P, C.POINTER(LightDesc), _U32P], C.c_int),
    "ray_scene_remove_light": ([_P, C.c_uint32], C.c_int),
    "ray_scene_add_mesh_instance": ([_P, C.c_uint32, C.POINTER(C.c_float), _U32P], C.c_int),
    "ray_scene_set_mesh_instance_transform": ([_P, C.c_uint32, C.POINTER(C.c_float)], C.c_int),
    "ray_scene_remove_mesh_instance": ([_P, C.c_uint32], C.c_int),
    "ray_scene_add_camera": ([_P, C.POINTER(CameraDesc), _U32P], C.c_int),
    "ray_scene_get_camera": ([_P, C.c_uint32, C.POINTER(CameraDesc)], C.c_int),
    "ray_scene_set_camera": ([_P, C.c_uint32, C.POINTER(CameraDesc)], C.c_int),
    "ray_scene_remove_camera": ([_P, C.c_uint32], C.c_int),
    "ray_scene_current_cam": ([_P, _U32P], C.c_int),
    "ray_scene_set_current_cam": ([_P, C.c_uint32], C.c_int),
    "ray_scene_triangle_count": ([_P, _U32P], C.c_int),
    "ray_scene_node_count": ([_P, _U32P], C.c_int),
    "ray_scene_commit": ([_P], C.c_int),
    "ray_scene_trace_closest": ([_P, _P, C.c_uint64, _P, _P, C.c_int, _P], C.c_int),
    "ray_scene_set_counting": ([_P, C.c_int], C.c_int),
    "ray_scene_last_trace_info": ([_P, C.POINTER(TraceInfo)], C.c_int),
    "ray_scene_mesh_bvh_info": ([_P, C.c_uint32, C.POINTER(BvhInfo)], C.c_int),
    "ray_scene_debug_read": ([_P, C.c_int, _P, C.c_uint64, C.POINTER(C.c_uint64)], C.c_int),
    "ray_renderer_debug_read": ([_P, C.c_int, _P, C.c_uint64, C.POINTER(C.c_uint64)], C.c_int),
    "ray_renderer_frame_info": ([_P, C.POINTER(FrameInfo)], C.c_int),
    "ray_renderer_set_stream": ([_P, _P], C.c_int),
    "ray_renderer_set_kernel": ([_P, C.c_int], C.c_int),
    "ray_renderer_set_trace_variant": ([_P, C.c_int], C.c_int),
    "ray_renderer_set_ray_sort": ([_P, C.c_int], C.c_int),
    "ray_scene_set_diff_params": ([_P, C.POINTER(DiffParams)], C.c_int),
    "ray_render_diff": ([_P, _P, C.c_int, C.c_int, _P, _P], C.c_int),
    "ray_render_adjoint": ([_P, _P, C.c_int, C.c_int, _P, _P, _P, _P], C.c_int),
    "ray_render_adjoint_color": ([_P, _P, C.c_int, C.c_int, _P, _P, _P, _P, _P], C.c_int),
    "ray_render_batch": ([C.POINTER(_P), C.POINTER(_P), C.POINTER(C.POINTER(Region)), C.c_int, C.c_int], C.c_int),
    "ray_sort_rays": ([_P, _P, C.c_uint64, C.POINTER(C.c_float), C.POINTER(C.c_float), _P, _P, _P, _P], C.c_int),
    "ray_sort_rays_noalloc": ([_P, C.c_uint64, C.POINTER(C.c_float), C.POINTER(C.c_float), _P, _P, _P, _P], C.c_int),
    "ray_scene_set_camera_axes": ([_P, C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_float)], C.c_int),
    "ray_scene_set_trace_tuning": ([_P, C.POINTER(TraceTuning)], C.c_int),
    "ray_scene_get_trace_tuning": ([_P, C.POINTER(TraceTuning)], C.c_int),
    "ray_scene_debug_write": ([_P, C.c_int, C.c_uint64, _P, C.c_uint64], C.c_int),
    "ray_scene_instance_tree_info": ([_P, C.POINTER(InstanceTreeInfo)], C.c_int),
    "ray_debug_fail_device_alloc": ([C.c_int64], C.c_int),
    "ray_set_wait_timeout_ms": ([C.c_int64], C.c_int),
    "ray_scene_tune_trace": ([_P, _P, C.c_uint64, _P, C.c_int, _P, C.POINTER(TraceTuning), C.c_char_p, C.c_uint64], C.c_int),
}


def lib() -> C.CDLL:
    """Loads libraygpu.so (building it first when only the sources exist)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                from . import build as _build

                _build.build()
            L = C.CDLL(LIB_PATH)
            for name, (args, res) in _SIGS.items():
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = res
            _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != RAY_OK:
        raise RayError(rc, lib().ray_last_error().decode(errors="replace"))


def declared_symbols() -> list[str]:
    """Entry points include/raygpu.h declares."""
    import re

    src = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:const char \*|int )(ray_\w+)\(", src, flags=re.M)))
