"""ctypes front end of the CPU oracle (test infrastructure only).

`Oracle` wraps the C restatement (``_build/libray_oracle.so``, built from
``ray_oracle.c``); `RefLib` wraps the reference Ray library compiled from its
own sources plus ``ref_bridge.cpp`` (``_ref/libray_ref.so``). Only the tests,
``__graft_entry__.smoke()`` and the benchmark's CPU-baseline leg use them, and
only as checkers or as the timed reference.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libray_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libray_ref.so")

TRI_DTYPE = np.dtype([("nu", "<f4"), ("nv", "<f4"), ("np", "<f4"), ("pu", "<f4"), ("pv", "<f4"), ("ci", "<i4"),
                      ("e0u", "<f4"), ("e0v", "<f4"), ("e1u", "<f4"), ("e1v", "<f4"), ("mi", "<u4"), ("back_mi", "<u4")])
HIT_DTYPE = np.dtype([("prim", "<i4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4")])
# Ref::ray_packet_t (96 bytes), src/Ray/internal/CoreRef.h:34-45
PACKET_DTYPE = np.dtype([("o", "<f4", 3), ("d", "<f4", 3), ("c", "<f4", 3), ("ior", "<f4"), ("do_dx", "<f4", 3),
                         ("dd_dx", "<f4", 3), ("do_dy", "<f4", 3), ("dd_dy", "<f4", 3), ("xy", "<i4"), ("ray_depth", "<i4")])
assert TRI_DTYPE.itemsize == 48 and HIT_DTYPE.itemsize == 16 and PACKET_DTYPE.itemsize == 96


class OrcCamera(C.Structure):
    _fields_ = [("filter", C.c_int), ("fov", C.c_float), ("gamma", C.c_float), ("focus_distance", C.c_float),
                ("focus_factor", C.c_float), ("origin", C.c_float * 3), ("fwd", C.c_float * 3), ("side", C.c_float * 3),
                ("up", C.c_float * 3)]


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def build(quiet: bool = True) -> None:
    """Build the oracle (and the reference bridge when the sources exist)."""
    out = subprocess.run(["make", "-C", HERE, "-j8"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout[-4000:] + out.stderr[-4000:])
    if not quiet:
        print(out.stdout)


class Oracle:
    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build()
        self.lib = L = C.CDLL(path)
        vp, i64, i32 = C.c_void_p, C.c_int64, C.c_int
        L.orc_preprocess_tris.argtypes = [vp, i64, vp, i64, vp]
        L.orc_preprocess_tris.restype = i64
        L.orc_closest_hit_brute.argtypes = [vp, i64, vp, i64, vp, i32, vp]
        L.orc_bvh_build.argtypes = [vp, i64]
        L.orc_bvh_build.restype = vp
        L.orc_bvh_free.argtypes = [vp]
        L.orc_closest_hit_bvh.argtypes = [vp, vp, vp, i64, vp, i32, vp]
        L.orc_ray_hash.argtypes = [vp, i64, vp, vp, vp]
        L.orc_sort_perm.argtypes = [vp, i64, vp]
        L.orc_construct_camera.argtypes = [i32, vp, vp, vp, C.c_float, C.c_float, C.c_float, C.c_float, C.POINTER(OrcCamera)]
        L.orc_generate_primary_rays.argtypes = [C.POINTER(OrcCamera), i32, i32, i32, i32, i32, i32, i32, vp, vp]
        L.orc_halton_perms.argtypes = [vp]
        L.orc_halton_table.argtypes = [i32, vp, vp]
        L.orc_hash.argtypes = [C.c_int32]
        L.orc_hash.restype = C.c_int32
        L.orc_construct_float.argtypes = [C.c_uint32]
        L.orc_construct_float.restype = C.c_float

    # -- triangles / hits
    def preprocess_tris(self, pos: np.ndarray, idx: np.ndarray, stride: int = 3) -> np.ndarray:
        pos = np.ascontiguousarray(pos, np.float32)
        idx = np.ascontiguousarray(idx, np.uint32)
        n = idx.size // 3
        out = np.zeros(n, TRI_DTYPE)
        self.lib.orc_preprocess_tris(_p(pos), stride, _p(idx), n, _p(out))
        return out

    @staticmethod
    def _box(world_box):
        return None if world_box is None else np.ascontiguousarray(world_box, np.float32).reshape(6)

    def closest_hit_brute(self, tris: np.ndarray, rays: np.ndarray, nthreads: int = 8, world_box=None) -> np.ndarray:
        """world_box: the single instance's box (min xyz, max xyz), tested as
        the reference's macro traversal does; None skips that test."""
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        hits = np.zeros(len(rays), HIT_DTYPE)
        box = self._box(world_box)
        self.lib.orc_closest_hit_brute(_p(tris), len(tris), _p(rays), len(rays), _p(hits), nthreads, _p(box))
        return hits

    def closest_hit_bvh(self, tris: np.ndarray, aabbs: np.ndarray, rays: np.ndarray, nthreads: int = 8, world_box=None) -> np.ndarray:
        aabbs = np.ascontiguousarray(aabbs, np.float32).reshape(-1, 6)
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        hits = np.zeros(len(rays), HIT_DTYPE)
        box = self._box(world_box)
        b = self.lib.orc_bvh_build(_p(aabbs), len(aabbs))
        try:
            self.lib.orc_closest_hit_bvh(b, _p(tris), _p(rays), len(rays), _p(hits), nthreads, _p(box))
        finally:
            self.lib.orc_bvh_free(b)
        return hits

    # -- sorting
    def ray_hash(self, rays: np.ndarray, root_min, cell_size) -> np.ndarray:
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        rm = np.asarray(root_min, np.float32)
        cs = np.asarray(cell_size, np.float32)
        keys = np.zeros(len(rays), np.uint32)
        self.lib.orc_ray_hash(_p(rays), len(rays), _p(rm), _p(cs), _p(keys))
        return keys

    def sort_perm(self, keys: np.ndarray) -> np.ndarray:
        keys = np.ascontiguousarray(keys, np.uint32)
        perm = np.zeros(len(keys), np.uint32)
        self.lib.orc_sort_perm(_p(keys), len(keys), _p(perm))
        return perm

    # -- camera / rays
    def construct_camera(self, origin, fwd, up, fov, filter=0, gamma=1.0, focus_distance=1.0, focus_factor=0.0) -> OrcCamera:
        cam = OrcCamera()
        o, f, u = (np.asarray(v, np.float32) for v in (origin, fwd, up))
        self.lib.orc_construct_camera(filter, _p(o), _p(f), _p(u), fov, gamma, focus_distance, focus_factor, C.byref(cam))
        return cam

    def generate_primary_rays(self, cam: OrcCamera, iteration: int, rect, w: int, h: int, halton: np.ndarray) -> np.ndarray:
        x, y, rw, rh = rect
        halton = np.ascontiguousarray(halton, np.float32)
        out = np.zeros(rw * rh, PACKET_DTYPE)
        self.lib.orc_generate_primary_rays(C.byref(cam), iteration, x, y, rw, rh, w, h, _p(halton), _p(out))
        return out

    def halton_perms(self) -> np.ndarray:
        p = np.zeros(1002, np.uint16)
        self.lib.orc_halton_perms(_p(p))
        return p

    def halton_table(self, iteration: int) -> np.ndarray:
        perms = self.halton_perms()
        out = np.zeros(24 * 256, np.float32)
        self.lib.orc_halton_table(iteration, _p(perms), _p(out))
        return out


# ----------------------------------------------------------------- reference


class RbMatDesc(C.Structure):
    _fields_ = [("type", C.c_int), ("main_color", C.c_float * 3), ("main_texture", C.c_uint32), ("normal_map", C.c_uint32),
                ("mix_materials", C.c_uint32 * 2), ("roughness", C.c_float), ("strength", C.c_float), ("fresnel", C.c_float),
                ("int_ior", C.c_float), ("ext_ior", C.c_float)]


class RbLightDesc(C.Structure):
    _fields_ = [("type", C.c_int), ("position", C.c_float * 3), ("radius", C.c_float), ("color", C.c_float * 3),
                ("direction", C.c_float * 3), ("angle", C.c_float)]


class RbCameraDesc(C.Structure):
    _fields_ = [("type", C.c_int), ("filter", C.c_int), ("dtype", C.c_int), ("origin", C.c_float * 3), ("fwd", C.c_float * 3),
                ("up", C.c_float * 3), ("fov", C.c_float), ("gamma", C.c_float), ("focus_distance", C.c_float),
                ("focus_factor", C.c_float), ("mi_index", C.c_uint32), ("uv_index", C.c_uint32)] + [
                   (n, C.c_int) for n in ("lighting_only", "skip_direct_lighting", "skip_indirect_lighting", "no_background",
                                          "clamp", "output_sh", "use_coherent_sampling", "max_diff_depth", "max_glossy_depth",
                                          "max_refr_depth", "max_transp_depth", "max_total_depth", "termination_start_depth")]


def ref_available() -> bool:
    return os.path.exists(REF_SO)


class RefLib:
    """The reference library (oracle/_ref). Raises if it was not built."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = L = C.CDLL(path)
        vp, i64, i32, u32, sz = C.c_void_p, C.c_int64, C.c_int, C.c_uint32, C.c_size_t
        L.rb_scene_new.argtypes = [i32]
        L.rb_scene_new.restype = vp
        L.rb_scene_free.argtypes = [vp]
        L.rb_add_texture.argtypes = [vp, vp, i32, i32, i32, i32]
        L.rb_add_texture.restype = u32
        L.rb_add_material.argtypes = [vp, C.POINTER(RbMatDesc)]
        L.rb_add_material.restype = u32
        L.rb_add_mesh.argtypes = [vp, i32, vp, sz, vp, sz, i32, vp, i32, i32]
        L.rb_add_mesh.restype = u32
        L.rb_add_instance.argtypes = [vp, u32, vp]
        L.rb_add_instance.restype = u32
        L.rb_add_light.argtypes = [vp, C.POINTER(RbLightDesc)]
        L.rb_add_light.restype = u32
        L.rb_set_environment.argtypes = [vp, vp, C.c_float, u32]
        L.rb_add_camera.argtypes = [vp, C.POINTER(RbCameraDesc)]
        L.rb_add_camera.restype = u32
        L.rb_triangle_count.argtypes = [vp]
        L.rb_triangle_count.restype = u32
        L.rb_trace_closest.argtypes = [vp, vp, i64, vp, vp, vp, i32, i32]
        L.rb_trace_closest.restype = i32
        L.rb_sort_rays.argtypes = [vp, i64, vp, vp, vp, vp]
        L.rb_construct_camera.argtypes = [C.POINTER(RbCameraDesc), vp]
        L.rb_generate_primary_rays.argtypes = [C.POINTER(RbCameraDesc), i32, i32, i32, i32, i32, i32, i32, vp, vp]
        L.rb_halton_table.argtypes = [i32, vp]
        L.rb_halton_perms.argtypes = [vp]
        L.rb_renderer_new.argtypes = [i32, i32, i32, i32]
        L.rb_renderer_new.restype = vp
        L.rb_renderer_free.argtypes = [vp]
        L.rb_renderer_type.argtypes = [vp]
        L.rb_renderer_type.restype = i32
        L.rb_render.argtypes = [vp, vp, i32, i32, i32, i32, i32, i32, i32]
        L.rb_get_pixels.argtypes = [vp, vp]
        L.rb_get_stats.argtypes = [vp, vp]
        L.rb_clear.argtypes = [vp]

    def halton_table(self, iteration: int) -> np.ndarray:
        out = np.zeros(24 * 256, np.float32)
        self.lib.rb_halton_table(iteration, _p(out))
        return out

    def halton_perms(self) -> np.ndarray:
        out = np.zeros(1002, np.uint16)
        self.lib.rb_halton_perms(_p(out))
        return out

    def sort_rays(self, rays: np.ndarray, root_min, cell_size):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        rm = np.asarray(root_min, np.float32)
        cs = np.asarray(cell_size, np.float32)
        keys = np.zeros(len(rays), np.uint32)
        perm = np.zeros(len(rays), np.uint32)
        self.lib.rb_sort_rays(_p(rays), len(rays), _p(rm), _p(cs), _p(keys), _p(perm))
        return keys, perm

    def generate_primary_rays(self, cam: RbCameraDesc, iteration: int, rect, w: int, h: int, halton: np.ndarray) -> np.ndarray:
        x, y, rw, rh = rect
        halton = np.ascontiguousarray(halton, np.float32)
        out = np.zeros(rw * rh, PACKET_DTYPE)
        self.lib.rb_generate_primary_rays(C.byref(cam), iteration, x, y, rw, rh, w, h, _p(halton), _p(out))
        return out


class RefScene:
    """A reference Ref::Scene built through SceneBase (wide BVH by default)."""

    def __init__(self, ref: RefLib, use_wide: bool = True):
        self.ref = ref
        self.h = ref.lib.rb_scene_new(int(use_wide))
        self._keep = []

    def __del__(self):
        if getattr(self, "h", None):
            self.ref.lib.rb_scene_free(self.h)
            self.h = None

    def add_texture(self, rgba: np.ndarray, is_srgb=True, gen_mips=False) -> int:
        rgba = np.ascontiguousarray(rgba, np.uint8)
        return self.ref.lib.rb_add_texture(self.h, _p(rgba), rgba.shape[1], rgba.shape[0], int(is_srgb), int(gen_mips))

    def add_material(self, type, main_color=(1, 1, 1), main_texture=0, normal_map=0xFFFFFFFF, mix_materials=(0xFFFFFFFF, 0xFFFFFFFF),
                     roughness=0.0, strength=1.0, fresnel=1.0, int_ior=1.0, ext_ior=1.0) -> int:
        d = RbMatDesc(type, (C.c_float * 3)(*main_color), main_texture, normal_map, (C.c_uint32 * 2)(*mix_materials), roughness,
                      strength, fresnel, int_ior, ext_ior)
        return self.ref.lib.rb_add_material(self.h, C.byref(d))

    def add_mesh(self, attrs: np.ndarray, indices: np.ndarray, shapes, layout=0, base_vertex=0, fast_bvh=False) -> int:
        attrs = np.ascontiguousarray(attrs, np.float32)
        indices = np.ascontiguousarray(indices, np.uint32)
        sh = np.ascontiguousarray(np.asarray(shapes, np.uint32).reshape(-1, 4))
        stride = (8, 10, 11, 13)[layout]
        self._keep += [attrs, indices, sh]
        return self.ref.lib.rb_add_mesh(self.h, layout, _p(attrs), attrs.size // stride, _p(indices), indices.size, base_vertex,
                                        _p(sh), len(sh), int(fast_bvh))

    def add_instance(self, mesh: int, xform=None) -> int:
        x = np.eye(4, dtype=np.float32).reshape(-1) if xform is None else np.ascontiguousarray(xform, np.float32).reshape(-1)
        return self.ref.lib.rb_add_instance(self.h, mesh, _p(x))

    def add_light(self, type, position=(0, 0, 0), radius=1.0, color=(1, 1, 1), direction=(0, -1, 0), angle=0.0) -> int:
        d = RbLightDesc(type, (C.c_float * 3)(*position), radius, (C.c_float * 3)(*color), (C.c_float * 3)(*direction), angle)
        return self.ref.lib.rb_add_light(self.h, C.byref(d))

    def set_environment(self, env_col=(0, 0, 0), env_clamp=0.0, env_map=0xFFFFFFFF):
        c = np.asarray(env_col, np.float32)
        self.ref.lib.rb_set_environment(self.h, _p(c), env_clamp, env_map)

    def add_camera(self, desc: RbCameraDesc) -> int:
        return self.ref.lib.rb_add_camera(self.h, C.byref(desc))

    def triangle_count(self) -> int:
        return self.ref.lib.rb_triangle_count(self.h)

    def trace_closest(self, rays: np.ndarray, nthreads: int = 8, backend: int = 0):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = len(rays)
        prim = np.zeros(n, np.int32)
        obj = np.zeros(n, np.int32)
        tuv = np.zeros((n, 3), np.float32)
        rc = self.ref.lib.rb_trace_closest(self.h, _p(rays), n, _p(prim), _p(obj), _p(tuv), nthreads, backend)
        if rc != 0:
            raise RuntimeError("reference trace failed (empty scene?)")
        hits = np.zeros(n, HIT_DTYPE)
        hits["prim"], hits["t"], hits["u"], hits["v"] = prim, tuv[:, 0], tuv[:, 1], tuv[:, 2]
        return hits, obj


class RefRenderer:
    REF, SSE2, AVX, AVX2 = 1, 2, 4, 8

    def __init__(self, ref: RefLib, w: int, h: int, type: int = 1, use_wide: bool = True):
        self.ref, self.w, self.h = ref, w, h
        self.r = ref.lib.rb_renderer_new(type, w, h, int(use_wide))

    def __del__(self):
        if getattr(self, "r", None):
            self.ref.lib.rb_renderer_free(self.r)
            self.r = None

    def type(self) -> int:
        return self.ref.lib.rb_renderer_type(self.r)

    def render(self, scene: RefScene, iterations: int, rect=(0, 0, 0, 0), reset=True, nthreads=1):
        self.ref.lib.rb_render(self.r, scene.h, iterations, *rect, int(reset), nthreads)

    def pixels(self) -> np.ndarray:
        out = np.zeros((self.h, self.w, 4), np.float32)
        self.ref.lib.rb_get_pixels(self.r, _p(out))
        return out

    def stats(self) -> np.ndarray:
        out = np.zeros(6, np.uint64)
        self.ref.lib.rb_get_stats(self.r, _p(out))
        return out
