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


def reference_src() -> str | None:
    """The reference's `src` directory: $RAY_REFERENCE_SRC, else the one the
    oracle Makefile built oracle/_ref from (oracle/_ref/refsrc.txt); None
    when neither names an existing directory."""
    d = os.environ.get("RAY_REFERENCE_SRC")
    if d:
        d = os.path.join(d, "src") if os.path.isdir(os.path.join(d, "src", "Ray")) else d
    else:
        f = os.path.join(HERE, "_ref", "refsrc.txt")
        d = open(f).read().strip() if os.path.exists(f) else None
    return d if d and os.path.isdir(d) else None


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
        L.orc_render_principled.argtypes = [C.POINTER(OrcPrincipledScene), C.POINTER(OrcCamera), i32, i32, i32, i32, i32, i32, vp, i32, i32]
        L.orc_area_light.argtypes = [i32, vp, vp, vp, C.c_float, vp, vp, vp]
        L.orc_area_light.restype = i32

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

    # -- metallic-roughness scenes
    def area_light(self, type: int, position=(0.0, 0.0, 0.0), color=(1.0, 1.0, 1.0), direction=(0.0, -1.0, 0.0), angle=0.0,
                   edge_u=(0.0, 0.0, 0.0), edge_v=(0.0, 0.0, 0.0), **_) -> np.ndarray:
        out = np.zeros(20, np.float32)
        args = [np.asarray(v, np.float32) for v in (position, color, direction)]
        eu, ev = np.asarray(edge_u, np.float32), np.asarray(edge_v, np.float32)
        if self.lib.orc_area_light(type, _p(args[0]), _p(args[1]), _p(args[2]), C.c_float(angle), _p(eu), _p(ev), _p(out)) != 0:
            raise ValueError("invalid quad or sun light")
        return out

    def principled_scene(self, spec: dict, albedo=None, roughness=None, material_slot=None,
                         roughness_sampling=None) -> "PrincipledScene":
        """Flattens a scene spec (the format of raydemo_b200.scenes) whose
        materials are all RAY_MAT_PRINCIPLED and whose lights are quad or sun
        lights into the arrays orc_render_principled reads; albedo (h, w, 3),
        roughness (n,), material_slot: the differentiable parameters;
        roughness_sampling: frozen roughness for sampling and pdfs."""
        return PrincipledScene(self, spec, albedo, roughness, material_slot, roughness_sampling)

    def render_principled(self, spec: dict, spp: int, nthreads: int = 8, scene: "PrincipledScene" = None,
                          plain_mean: bool = False) -> np.ndarray:
        """The mean of iterations 1..spp, (h, w, 4): the renderer's clean buffer,
        or with plain_mean the differentiable forward pass's sum / spp."""
        ps = scene if scene is not None else self.principled_scene(spec)
        w, h = spec["size"]
        cam = spec["camera"]
        c = self.construct_camera(cam["origin"], cam["fwd"], cam["up"], cam.get("fov", 45.0), filter=cam.get("filter", 1),
                                  gamma=cam.get("gamma", 1.0), focus_distance=cam.get("focus_distance", 1.0),
                                  focus_factor=cam.get("focus_factor", 0.0))
        out = np.zeros((h, w, 4), np.float32)
        self.lib.orc_render_principled(C.byref(ps.c), C.byref(c), w, h, spp, cam.get("max_diff_depth", 4), cam.get("max_total_depth", 4),
                                       cam.get("termination_start_depth", 3), _p(out), nthreads, int(plain_mean))
        return out


class OrcPrincipledScene(C.Structure):
    _fields_ = [("tris", C.c_void_p), ("aabbs", C.c_void_p), ("normals", C.c_void_p), ("uvs", C.c_void_p), ("mat", C.c_void_p),
                ("mesh_tris", C.c_void_p), ("inst_mesh", C.c_void_p), ("inst_xform", C.c_void_p), ("mats", C.c_void_p),
                ("texels", C.c_void_p), ("tex_info", C.c_void_p), ("lights", C.c_void_p), ("diff_albedo", C.c_void_p),
                ("diff_rough", C.c_void_p), ("diff_rough_sampling", C.c_void_p), ("ntris", C.c_int64), ("nmeshes", C.c_int), ("ninst", C.c_int), ("nmats", C.c_int),
                ("ntex", C.c_int), ("nlights", C.c_int), ("diff_aw", C.c_int), ("diff_ah", C.c_int), ("n_diff_rough", C.c_int),
                ("env_col", C.c_float * 3)]


class PrincipledScene:
    """The arrays of one scene spec for orc_render_principled (kept alive with
    the structure that points at them)."""

    INVALID = 0xFFFFFFFF
    FIRST_TEXTURE = 2  # a scene's textures 0 and 1 are its default environment and normal map

    def __init__(self, orc: Oracle, spec: dict, albedo=None, roughness=None, material_slot=None, roughness_sampling=None):
        texels, tex_info, off = [], [], 0
        for rgba, srgb, _mips in spec.get("textures", []):
            a = np.ascontiguousarray(rgba, np.uint8)
            th, tw = a.shape[:2]
            texels.append(a.view(np.uint32).reshape(-1))
            tex_info += [off, tw, th, int(bool(srgb))]
            off += tw * th
        ntex = len(tex_info) // 4
        mats = []
        slots = list(material_slot) if material_slot is not None else []
        for mi, m in enumerate(spec.get("materials", [])):
            if m.get("type") != 6:
                raise ValueError("only metallic-roughness materials")
            t = m.get("main_texture", self.INVALID)
            if t == self.INVALID:
                ti = -1
            elif self.FIRST_TEXTURE <= t < self.FIRST_TEXTURE + ntex:
                ti = t - self.FIRST_TEXTURE
            else:
                raise ValueError("main texture must be one of the spec's textures")
            slot = slots[mi] if mi < len(slots) else -1
            mats += [*map(float, m.get("main_color", (1.0, 1.0, 1.0))), float(m.get("roughness", 0.0)), float(m.get("metallic", 0.0)),
                     float(ti), float(slot), 0.0]
        tris, aabbs, normals, uvs, mat, mesh_tris = [], [], [], [], [], []
        first = 0
        for attrs, idx, shapes, layout in spec.get("meshes", []):
            stride = (8, 10, 11, 13)[layout]
            A = np.ascontiguousarray(attrs, np.float32).reshape(-1, stride)
            I = np.ascontiguousarray(idx, np.uint32).reshape(-1, 3)
            n = len(I)
            uv_off = 6 if layout in (0, 1) else 9
            V = A[I.astype(np.int64)]  # (n, 3, stride)
            tris.append(orc.preprocess_tris(np.ascontiguousarray(A[:, :3]), I))
            aabbs.append(np.concatenate([V[:, :, :3].min(axis=1), V[:, :, :3].max(axis=1)], axis=1))
            normals.append(V[:, :, 3:6].reshape(n, 9))
            uvs.append(V[:, :, uv_off:uv_off + 2].reshape(n, 6))
            mt = np.zeros((n, 2), np.int32)  # triangles no shape covers: material 0 on both sides
            for s in shapes:
                if len(s) == 3:
                    s = (s[0], self.INVALID, s[1], s[2])
                mi, back, start, count = (int(x) for x in s)
                for i in range(start, start + count, 3):
                    if i // 3 < n:
                        mt[i // 3] = (mi, -1 if back == self.INVALID else back)
            mat.append(mt)
            mesh_tris += [first, n]
            first += n
        inst_mesh, inst_xform = [], []
        for mesh, xf in spec.get("instances", []):
            inst_mesh.append(int(mesh))
            inst_xform.append(np.eye(4, dtype=np.float32).reshape(-1) if xf is None else np.asarray(xf, np.float32).reshape(-1))
        lights = [orc.area_light(**l) for l in spec.get("lights", [])]
        env = spec.get("env", {})
        if env.get("env_map", self.INVALID) != self.INVALID:
            raise ValueError("only the default environment map")
        self.arrays = {
            "tris": np.concatenate(tris) if tris else np.zeros(0, TRI_DTYPE),
            "aabbs": np.ascontiguousarray(np.concatenate(aabbs) if aabbs else np.zeros((0, 6)), np.float32),
            "normals": np.ascontiguousarray(np.concatenate(normals) if normals else np.zeros((0, 9)), np.float32),
            "uvs": np.ascontiguousarray(np.concatenate(uvs) if uvs else np.zeros((0, 6)), np.float32),
            "mat": np.ascontiguousarray(np.concatenate(mat) if mat else np.zeros((0, 2)), np.int32),
            "mesh_tris": np.asarray(mesh_tris, np.int64),
            "inst_mesh": np.asarray(inst_mesh, np.int32),
            "inst_xform": np.ascontiguousarray(np.concatenate(inst_xform) if inst_xform else np.zeros(0), np.float32),
            "mats": np.asarray(mats, np.float32),
            "texels": np.concatenate(texels) if texels else np.zeros(1, np.uint32),
            "tex_info": np.asarray(tex_info, np.int32),
            "lights": np.ascontiguousarray(np.concatenate(lights) if lights else np.zeros(0), np.float32),
            "diff_albedo": np.ascontiguousarray(albedo, np.float32) if albedo is not None else np.zeros(0, np.float32),
            "diff_rough": np.ascontiguousarray(roughness, np.float32).reshape(-1) if roughness is not None else np.zeros(0, np.float32),
            "diff_rough_sampling": (np.ascontiguousarray(roughness_sampling, np.float32).reshape(-1) if roughness_sampling is not None
                                    else np.zeros(0, np.float32)),
        }
        a = self.arrays
        c = OrcPrincipledScene()
        for k in ("tris", "aabbs", "normals", "uvs", "mat", "mesh_tris", "inst_mesh", "inst_xform", "mats", "texels", "tex_info", "lights",
                  "diff_albedo", "diff_rough", "diff_rough_sampling"):
            setattr(c, k, a[k].ctypes.data if a[k].size else None)
        if albedo is not None:
            c.diff_ah, c.diff_aw = a["diff_albedo"].shape[:2]
            c.n_diff_rough = a["diff_rough"].size
        c.ntris = len(a["tris"])
        c.nmeshes = len(mesh_tris) // 2
        c.ninst = len(inst_mesh)
        c.nmats = len(mats) // 8
        c.ntex = ntex
        c.nlights = len(lights)
        for k, v in enumerate(env.get("env_col", (0.0, 0.0, 0.0))):
            c.env_col[k] = float(v)
        self.c = c


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
        L.rb_remove_instance.argtypes = [vp, u32]
        L.rb_set_instance_xform.argtypes = [vp, u32, vp]
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
        L.rb_get_sh.argtypes = [vp, vp]
        L.rb_get_sh.restype = C.c_int
        L.rb_get_stats.argtypes = [vp, vp]
        L.rb_clear.argtypes = [vp]
        self.has_loader = hasattr(L, "rb_load_scene")
        if self.has_loader:  # the demo's scene loader (src/DemoLib/load/Load.cpp), when built
            L.rb_load_scene.argtypes = [vp, C.c_char_p]
            L.rb_load_scene.restype = vp
            L.rb_loaded_free.argtypes = [vp]
            L.rb_render_loaded.argtypes = [vp, vp, i32, i32]
            L.rb_loaded_camera.argtypes = [vp, C.POINTER(RbCameraDesc)]
            L.rb_loaded_environment.argtypes = [vp, vp, vp, vp]
            L.rb_loaded_triangles.argtypes = [vp]
            L.rb_loaded_triangles.restype = u32
            L.rb_loaded_instance_xform.argtypes = [vp, u32, vp]
            L.rb_loaded_instance_xform.restype = i32
            L.rb_load_image.argtypes = [C.c_char_p, i32, C.POINTER(i32), C.POINTER(i32), vp, sz]
            L.rb_load_image.restype = C.c_longlong
            L.rb_load_mesh.argtypes = [C.c_char_p, i32, vp, sz, vp, sz, vp, sz, vp]
            L.rb_load_mesh.restype = i32

    def load_image(self, path: str, hdr: bool = False):
        """Load_stb_image / LoadHDR of the reference: (h, w, 4) uint8, or None on error."""
        w, h = C.c_int32(), C.c_int32()
        n = self.lib.rb_load_image(path.encode(), int(hdr), C.byref(w), C.byref(h), None, 0)
        if n < 0:
            return None
        out = np.zeros((h.value, w.value, 4), np.uint8)
        self.lib.rb_load_image(path.encode(), int(hdr), C.byref(w), C.byref(h), _p(out), out.nbytes)
        return out

    def load_mesh(self, path: str, bin: bool = False):
        """LoadOBJ / LoadBIN of the reference: (attrs (n, 8) float32, indices, groups), or None."""
        sizes = np.zeros(3, np.uint64)
        if self.lib.rb_load_mesh(path.encode(), int(bin), None, 0, None, 0, None, 0, _p(sizes)) != 0:
            return None
        a = np.zeros(int(sizes[0]), np.float32)
        i = np.zeros(int(sizes[1]), np.uint32)
        g = np.zeros(int(sizes[2]), np.uint32)
        self.lib.rb_load_mesh(path.encode(), int(bin), _p(a), a.size, _p(i), i.size, _p(g), g.size, _p(sizes))
        return a.reshape(-1, 8), i, g

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


class RefLoadedScene:
    """A scene made by the reference's LoadScene (Load.cpp:22) on a Ref renderer
    from JSON text (paths relative to the working directory); .ok is False
    where LoadScene returned null."""

    def __init__(self, renderer: "RefRenderer", json_text: str):
        self.ref = renderer.ref
        self.h = self.ref.lib.rb_load_scene(renderer.r, json_text.encode())
        self.ok = bool(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.ref.lib.rb_loaded_free(self.h)
            self.h = None

    def camera(self) -> "RbCameraDesc":
        d = RbCameraDesc()
        self.ref.lib.rb_loaded_camera(self.h, C.byref(d))
        return d

    def environment(self):
        col = np.zeros(3, np.float32)
        clamp = np.zeros(1, np.float32)
        env_map = np.zeros(1, np.uint32)
        self.ref.lib.rb_loaded_environment(self.h, _p(col), _p(clamp), _p(env_map))
        return col, float(clamp[0]), int(env_map[0])

    def triangle_count(self) -> int:
        return self.ref.lib.rb_loaded_triangles(self.h)

    def instance_xforms(self) -> list:
        out, i = [], 0
        while True:
            x = np.zeros(16, np.float32)
            if not self.ref.lib.rb_loaded_instance_xform(self.h, i, _p(x)):
                return out
            out.append(x)
            i += 1


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

    def remove_instance(self, i: int) -> None:
        self.ref.lib.rb_remove_instance(self.h, i)

    def set_instance_xform(self, i: int, xform) -> None:
        x = np.ascontiguousarray(xform, np.float32).reshape(-1)
        self.ref.lib.rb_set_instance_xform(self.h, i, _p(x))

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

    def render_loaded(self, scene: RefLoadedScene, iterations: int, nthreads: int = 1):
        self.ref.lib.rb_render_loaded(self.r, scene.h, iterations, nthreads)

    def sh_data(self):
        """get_sh_data_ref: (h, w, 12) float32, or None."""
        out = np.zeros((self.h, self.w, 12), np.float32)
        return out if self.ref.lib.rb_get_sh(self.r, _p(out)) else None

    def stats(self) -> np.ndarray:
        out = np.zeros(6, np.uint64)
        self.ref.lib.rb_get_stats(self.r, _p(out))
        return out
