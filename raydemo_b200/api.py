"""Python mirror of Ray::RendererBase / Ray::SceneBase over the C ABI.

Method names follow the reference (src/Ray/RendererBase.h, src/Ray/SceneBase.h)
so that code written against it reads the same. Errors raise RayError where
the reference returns silently, except where the reference documents a
sentinel (0xffffffff) for a failed add, which is kept.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import capi
from .capi import check, lib

# eMaterialType (SceneBase.h:45-52)
DiffuseMaterial, GlossyMaterial, RefractiveMaterial, EmissiveMaterial, MixMaterial, TransparentMaterial = range(6)
# eLightType (SceneBase.h:108-112), then this library's quad and sun lights
PointLight, SpotLight, DirectionalLight, QuadLight, SunLight = range(5)
# this library's metallic-roughness material (include/raygpu.h RAY_MAT_PRINCIPLED)
PrincipledMaterial = 6
# eCamType / eFilterType / eDeviceType (Types.h:33-37)
Persp, Ortho, Geo = range(3)
Box, Tent = range(2)
NoDevice, SRGB = range(2)

HIT_DTYPE = np.dtype([("prim", "<i4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4")])


@dataclass
class CameraDesc:
    """camera_desc_t (SceneBase.h:122-145) with the reference defaults."""
    type: int = Persp
    filter: int = Tent
    dtype: int = SRGB
    origin: tuple = (0.0, 0.0, 0.0)
    fwd: tuple = (0.0, 0.0, 0.0)
    up: tuple = (0.0, 0.0, 0.0)
    fov: float = 45.0
    gamma: float = 1.0
    focus_distance: float = 1.0
    focus_factor: float = 0.0
    mi_index: int = 0
    uv_index: int = 0
    lighting_only: bool = False
    skip_direct_lighting: bool = False
    skip_indirect_lighting: bool = False
    no_background: bool = False
    clamp: bool = False
    output_sh: bool = False
    use_coherent_sampling: bool = False
    max_diff_depth: int = 4
    max_glossy_depth: int = 4
    max_refr_depth: int = 4
    max_transp_depth: int = 4
    max_total_depth: int = 4
    termination_start_depth: int = 3

    def to_c(self) -> capi.CameraDesc:
        c = capi.CameraDesc()
        for f in ("type", "filter", "dtype", "fov", "gamma", "focus_distance", "focus_factor", "mi_index", "uv_index",
                  "max_diff_depth", "max_glossy_depth", "max_refr_depth", "max_transp_depth", "max_total_depth",
                  "termination_start_depth"):
            setattr(c, f, getattr(self, f))
        for f in ("lighting_only", "skip_direct_lighting", "skip_indirect_lighting", "no_background", "clamp", "output_sh",
                  "use_coherent_sampling"):
            setattr(c, f, int(bool(getattr(self, f))))
        c.origin = capi.f3(*self.origin)
        c.fwd = capi.f3(*self.fwd)
        c.up = capi.f3(*self.up)
        return c

    @staticmethod
    def from_c(c: capi.CameraDesc) -> "CameraDesc":
        d = CameraDesc()
        for f in d.__dataclass_fields__:
            v = getattr(c, f)
            if f in ("origin", "fwd", "up"):
                v = tuple(v)
            elif f in ("lighting_only", "skip_direct_lighting", "skip_indirect_lighting", "no_background", "clamp", "output_sh",
                       "use_coherent_sampling"):
                v = bool(v)
            setattr(d, f, v)
        return d


class Scene:
    """SceneBase over ray_scene (created by Renderer.CreateScene)."""

    def __init__(self, handle: int, renderer: "Renderer"):
        self._h = C.c_void_p(handle)
        self._renderer = renderer  # keeps the device context's owner alive

    def __del__(self):
        try:
            if getattr(self, "_h", None) and self._h.value:
                lib().ray_destroy_scene(self._h)
                self._h = C.c_void_p()
        except Exception:  # interpreter shutdown: the module state may be gone
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # environment
    def SetEnvironment(self, env_col=(0.0, 0.0, 0.0), env_clamp=0.0, env_map=capi.RAY_INVALID_INDEX) -> None:
        e = capi.EnvDesc(capi.f3(*env_col), env_clamp, env_map)
        check(lib().ray_scene_set_environment(self._h, C.byref(e)))

    def GetEnvironment(self) -> dict:
        e = capi.EnvDesc()
        check(lib().ray_scene_get_environment(self._h, C.byref(e)))
        return {"env_col": tuple(e.env_col), "env_clamp": e.env_clamp, "env_map": e.env_map}

    # resources
    def AddTexture(self, rgba: np.ndarray, is_srgb: bool = True, generate_mipmaps: bool = False) -> int:
        rgba = np.ascontiguousarray(rgba, np.uint8)
        if rgba.ndim != 3 or rgba.shape[2] != 4:
            raise ValueError("texture must be (h, w, 4) RGBA8")
        d = capi.TexDesc(rgba.ctypes.data, rgba.shape[1], rgba.shape[0], int(is_srgb), int(generate_mipmaps))
        out = C.c_uint32()
        check(lib().ray_scene_add_texture(self._h, C.byref(d), C.byref(out)))
        return out.value

    def AddMaterial(self, type=DiffuseMaterial, main_color=(1.0, 1.0, 1.0), main_texture=0, normal_map=capi.RAY_INVALID_INDEX,
                    mix_materials=(capi.RAY_INVALID_INDEX, capi.RAY_INVALID_INDEX), roughness=0.0, strength=1.0, fresnel=1.0,
                    int_ior=1.0, ext_ior=1.0, metallic=0.0) -> int:
        d = capi.MatDesc(type, capi.f3(*main_color), main_texture, normal_map, (C.c_uint32 * 2)(*mix_materials), roughness, strength,
                         fresnel, int_ior, ext_ior, metallic)
        out = C.c_uint32()
        check(lib().ray_scene_add_material(self._h, C.byref(d), C.byref(out)))
        return out.value

    def AddMesh(self, vtx_attrs: np.ndarray, vtx_indices: np.ndarray, shapes, layout: int = 0, base_vertex: int = 0,
                use_fast_bvh_build: bool = False) -> int:
        """shapes: iterable of (mat_index, back_mat_index, vtx_start, vtx_count) or (mat_index, vtx_start, vtx_count)."""
        attrs = np.ascontiguousarray(vtx_attrs, np.float32).reshape(-1)
        idx = np.ascontiguousarray(vtx_indices, np.uint32).reshape(-1)
        stride = (8, 10, 11, 13)[layout]
        sh = []
        for s in shapes:
            if len(s) == 3:
                s = (s[0], capi.RAY_INVALID_INDEX, s[1], s[2])
            sh.append(capi.ShapeDesc(*[int(x) for x in s]))
        arr = (capi.ShapeDesc * max(1, len(sh)))(*sh)
        d = capi.MeshDesc(0, layout, attrs.ctypes.data, attrs.size // stride, idx.ctypes.data, idx.size, base_vertex, arr, len(sh), 0,
                          int(use_fast_bvh_build))
        out = C.c_uint32()
        check(lib().ray_scene_add_mesh(self._h, C.byref(d), C.byref(out)))
        return out.value

    def RemoveMesh(self, i: int) -> None:
        check(lib().ray_scene_remove_mesh(self._h, i))

    def AddLight(self, type=PointLight, position=(0.0, 0.0, 0.0), radius=1.0, color=(1.0, 1.0, 1.0), direction=(0.0, -1.0, 0.0),
                 angle=0.0, edge_u=(0.0, 0.0, 0.0), edge_v=(0.0, 0.0, 0.0)) -> int:
        d = capi.LightDesc(type, capi.f3(*position), radius, capi.f3(*color), capi.f3(*direction), angle, capi.f3(*edge_u),
                           capi.f3(*edge_v))
        out = C.c_uint32()
        check(lib().ray_scene_add_light(self._h, C.byref(d), C.byref(out)))
        return out.value

    def AddMeshInstance(self, mesh: int, xform=None) -> int:
        x = np.eye(4, dtype=np.float32).reshape(-1) if xform is None else np.ascontiguousarray(xform, np.float32).reshape(-1)
        out = C.c_uint32()
        check(lib().ray_scene_add_mesh_instance(self._h, mesh, x.ctypes.data_as(C.POINTER(C.c_float)), C.byref(out)))
        return out.value

    def SetMeshInstanceTransform(self, mi: int, xform) -> None:
        x = np.ascontiguousarray(xform, np.float32).reshape(-1)
        check(lib().ray_scene_set_mesh_instance_transform(self._h, mi, x.ctypes.data_as(C.POINTER(C.c_float))))

    def RemoveMeshInstance(self, mi: int) -> None:
        check(lib().ray_scene_remove_mesh_instance(self._h, mi))

    # cameras (SceneBase.cpp:8-89)
    def AddCamera(self, desc: CameraDesc) -> int:
        c = desc.to_c()
        out = C.c_uint32()
        check(lib().ray_scene_add_camera(self._h, C.byref(c), C.byref(out)))
        return out.value

    def GetCamera(self, i: int) -> CameraDesc:
        c = capi.CameraDesc()
        check(lib().ray_scene_get_camera(self._h, i, C.byref(c)))
        return CameraDesc.from_c(c)

    def SetCamera(self, i: int, desc: CameraDesc) -> None:
        c = desc.to_c()
        check(lib().ray_scene_set_camera(self._h, i, C.byref(c)))

    def RemoveCamera(self, i: int) -> None:
        check(lib().ray_scene_remove_camera(self._h, i))

    def current_cam(self) -> int:
        out = C.c_uint32()
        check(lib().ray_scene_current_cam(self._h, C.byref(out)))
        return out.value

    def set_current_cam(self, i: int) -> None:
        check(lib().ray_scene_set_current_cam(self._h, i))

    def set_diff_params(self, albedo_ptr: int, albedo_w: int, albedo_h: int, roughness_ptr: int, n_roughness: int,
                        material_slot=None, roughness_sampling_ptr: int = 0, color_ptr: int = 0) -> None:
        """Differentiable parameters (ray_scene_set_diff_params): device pointers
        to a float RGB albedo texture (albedo_h x albedo_w x 3; 0 for none when
        no RAY_MAT_PRINCIPLED material has a slot) and n_roughness slots;
        material_slot: per material its slot or -1 (None: no slots);
        roughness_sampling_ptr: frozen roughness for sampling (0: none);
        color_ptr: the RAY_MAT_DIFFUSE slots' main colours (n_roughness x 3; 0: none)."""
        if albedo_ptr is None:
            check(lib().ray_scene_set_diff_params(self._h, None))
            return
        slots = None
        n = 0
        if material_slot is not None:
            n = len(material_slot)
            slots = (C.c_int32 * max(n, 1))(*[int(k) for k in material_slot])
        p = capi.DiffParams(albedo_ptr or None, albedo_w, albedo_h, roughness_ptr, n_roughness,
                            C.cast(slots, C.POINTER(C.c_int32)) if slots is not None else None, n, roughness_sampling_ptr or None,
                            color_ptr or None)
        check(lib().ray_scene_set_diff_params(self._h, C.byref(p)))

    def triangle_count(self) -> int:
        out = C.c_uint32()
        check(lib().ray_scene_triangle_count(self._h, C.byref(out)))
        return out.value

    def node_count(self) -> int:
        out = C.c_uint32()
        check(lib().ray_scene_node_count(self._h, C.byref(out)))
        return out.value

    def Commit(self) -> None:
        check(lib().ray_scene_commit(self._h))

    def mesh_bvh_info(self, mesh: int) -> capi.BvhInfo:
        out = capi.BvhInfo()
        check(lib().ray_scene_mesh_bvh_info(self._h, mesh, C.byref(out)))
        return out

    # batch closest hit (Traverse_MacroTree_WithStack_ClosestHit over a batch)
    def trace_closest(self, rays: np.ndarray, with_obj: bool = False):
        """rays: (n, 8) float32 host array. Returns hits (HIT_DTYPE) [, obj]."""
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = len(rays)
        hits = np.zeros(n, HIT_DTYPE)
        obj = np.zeros(n, np.int32) if with_obj else None
        check(lib().ray_scene_trace_closest(self._h, rays.ctypes.data, n, hits.ctypes.data, obj.ctypes.data if with_obj else None,
                                            capi.RAY_MEM_HOST, None))
        return (hits, obj) if with_obj else hits

    def trace_closest_device(self, rays_ptr: int, n: int, hits_ptr: int, obj_ptr: int = 0, stream: int = 0) -> None:
        """Device-pointer form (stream-ordered, asynchronous)."""
        check(lib().ray_scene_trace_closest(self._h, rays_ptr, n, hits_ptr, obj_ptr or None, capi.RAY_MEM_DEVICE, stream or None))

    def set_trace_tuning(self, kernel: int = 0, refill_min: int = 0, deep_stack: int = 0, reorder: int = 0, reorder_bits: int = 0,
                         block: int = 0, smem_stack: int = 0, stream_hint: int = 0, l2_persist: int = 0,
                         instance_tree: int = 0) -> None:
        """ray_scene_set_trace_tuning: kernel (1 per ray, 2 persistent, 3
        persistent with one triangle test per step; 0 keeps), refill threshold (0 keeps), deep stack, trace order (0 input,
        1 ray hash, 2 origin cell first), the key bits it sorts on, threads
        per block and shared stack entries (0: 64 and 16), streaming cache
        hint on rays and hits, L2 residency (1 nodes, 2 leaf triangles),
        instance tree (0 from 32 instances, 1 always, -1 never)."""
        t = capi.TraceTuning(kernel, refill_min, deep_stack, reorder, reorder_bits, block, smem_stack, stream_hint, l2_persist,
                             instance_tree)
        check(lib().ray_scene_set_trace_tuning(self._h, C.byref(t)))

    def tune_trace_device(self, rays_ptr: int, n: int, hits_ptr: int, stream: int = 0, force: bool = False) -> tuple:
        """ray_scene_tune_trace on n device rays (hits_ptr: an n-entry device
        buffer): keeps the fastest traversal settings for this scene; returns
        (settings tuple as get_trace_tuning, report string)."""
        t = capi.TraceTuning()
        buf = C.create_string_buffer(4096)
        check(lib().ray_scene_tune_trace(self._h, rays_ptr, n, hits_ptr, 1 if force else 0, stream or None, C.byref(t), buf, 4096))
        return self.get_trace_tuning(), buf.value.decode()

    def debug_write(self, what: int, offset: int, data: bytes) -> None:
        """ray_scene_debug_write: overwrite bytes of the committed wide nodes
        (0) or leaf triangles (1), for failure-detection tests."""
        b = C.create_string_buffer(bytes(data), len(data))
        check(lib().ray_scene_debug_write(self._h, what, offset, b, len(data)))

    def get_trace_tuning(self) -> tuple:
        """(kernel, refill_min, deep_stack, reorder, reorder_bits, block, smem_stack, stream_hint, l2_persist, instance_tree)"""
        t = capi.TraceTuning()
        check(lib().ray_scene_get_trace_tuning(self._h, C.byref(t)))
        return (t.kernel, t.refill_min, t.deep_stack, t.reorder, t.reorder_bits, t.block, t.smem_stack, t.stream_hint,
                t.l2_persist, t.instance_tree)

    def instance_tree_info(self) -> capi.InstanceTreeInfo:
        """ray_scene_instance_tree_info: instances the tree covers (0: none),
        whether the last commit refitted it, and its host time in ms."""
        i = capi.InstanceTreeInfo()
        check(lib().ray_scene_instance_tree_info(self._h, C.byref(i)))
        return i

    def set_counting(self, enable: bool) -> None:
        check(lib().ray_scene_set_counting(self._h, int(enable)))

    def last_trace_info(self) -> capi.TraceInfo:
        out = capi.TraceInfo()
        check(lib().ray_scene_last_trace_info(self._h, C.byref(out)))
        return out


class Renderer:
    """RendererBase over ray_renderer."""

    def __init__(self, w: int, h: int, device: int = 0, use_wide_bvh: bool = True):
        s = capi.Settings(w, h, int(use_wide_bvh), device)
        out = C.c_void_p()
        check(lib().ray_create_renderer(C.byref(s), C.byref(out)))
        self._h = out

    def __del__(self):
        try:
            if getattr(self, "_h", None) and self._h.value:
                lib().ray_destroy_renderer(self._h)
                self._h = C.c_void_p()
        except Exception:  # interpreter shutdown: the module state may be gone
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def type(self) -> int:
        out = C.c_int()
        check(lib().ray_renderer_type(self._h, C.byref(out)))
        return out.value

    def size(self) -> tuple:
        w, h = C.c_int(), C.c_int()
        check(lib().ray_renderer_size(self._h, C.byref(w), C.byref(h)))
        return w.value, h.value

    def Resize(self, w: int, h: int) -> None:
        check(lib().ray_resize(self._h, w, h))

    def Clear(self, c=(0.0, 0.0, 0.0, 0.0)) -> None:
        px = capi.Pixel(*c)
        check(lib().ray_clear(self._h, C.byref(px)))

    def CreateScene(self) -> Scene:
        out = C.c_void_p()
        check(lib().ray_create_scene(self._h, C.byref(out)))
        return Scene(out.value, self)

    def render_diff(self, scene: Scene, first_iteration: int, samples: int, image_ptr: int, sample_ptr: int) -> None:
        """Differentiable forward pass (ray_render_diff): device pointers to the
        mean image (h x w x 3) and the per-sample radiance (samples x h x w x 3)."""
        check(lib().ray_render_diff(self._h, scene.handle, first_iteration, samples, image_ptr, sample_ptr))

    def render_adjoint(self, scene: Scene, first_iteration: int, samples: int, sample_ptr: int, d_image_ptr: int, grad_albedo_ptr: int,
                       grad_rough_ptr: int, grad_color_ptr: int = 0) -> None:
        """Path-replay adjoint (ray_render_adjoint_color): accumulates the
        gradients (albedo texture, roughness slots, diffuse slots' colours)."""
        check(lib().ray_render_adjoint_color(self._h, scene.handle, first_iteration, samples, sample_ptr, d_image_ptr,
                                             grad_albedo_ptr or None, grad_rough_ptr, grad_color_ptr or None))

    def RenderScene(self, scene: Scene, region: capi.Region) -> None:
        check(lib().ray_render(self._h, scene.handle, C.byref(region)))

    def get_pixels_ref(self) -> np.ndarray:
        w, h = self.size()
        out = C.c_void_p()
        check(lib().ray_get_pixels(self._h, C.byref(out), 0))
        return np.ctypeslib.as_array(C.cast(out, C.POINTER(C.c_float)), shape=(h, w, 4)).copy()

    def sort_rays_device(self, rays_ptr: int, n: int, root_min, cell_size, perm_ptr: int, keys_ptr: int = 0, rays_out_ptr: int = 0,
                         stream: int = 0) -> None:
        """SortRays_CPU (CoreRef.cpp:615-657) on device buffers: keys (optional),
        the stable-sort permutation and (optional) the reordered rays."""
        rm = (C.c_float * 3)(*root_min)
        cs = (C.c_float * 3)(*cell_size)
        check(lib().ray_sort_rays(self._h, rays_ptr, n, rm, cs, keys_ptr or None, perm_ptr, rays_out_ptr or None, stream or None))

    def get_sh_data_ref(self):
        """get_sh_data_ref: (h, w, 12) float32 (coeff_r[4], coeff_g[4], coeff_b[4]) or None."""
        w, h = self.size()
        out = C.c_void_p()
        check(lib().ray_get_sh_data(self._h, C.byref(out)))
        if not out.value:
            return None
        return np.ctypeslib.as_array(C.cast(out, C.POINTER(C.c_float)), shape=(h, w, 12)).copy()

    def debug_read(self, what: int) -> np.ndarray:
        """Renderer device arrays (ray_renderer_debug_read): 0 first ray buffer
        (n, 8) float32, 1 payloads (n, 20) float32, 2 sample table (6144,),
        3 sample buffer (h, w, 4)."""
        size = C.c_uint64()
        check(lib().ray_renderer_debug_read(self._h, what, None, 0, C.byref(size)))
        buf = np.zeros(size.value // 4, np.float32)
        check(lib().ray_renderer_debug_read(self._h, what, buf.ctypes.data, size.value, C.byref(size)))
        if what == 0:
            return buf.reshape(-1, 8)
        if what == 1:
            return buf.reshape(-1, 20)
        if what == 3:
            w, h = self.size()
            return buf.reshape(h, w, 4)
        return buf

    def set_kernel(self, kernel: int = 0) -> None:
        """1 wavefront, 2 path kernel, 0 chosen by timing (ray_renderer_set_kernel)."""
        check(lib().ray_renderer_set_kernel(self._h, kernel))

    def set_trace_variant(self, variant: int = -1) -> None:
        """ray_renderer_set_trace_variant: -1 timed by the frame tuner, else
        an index of its trace settings (0: the scene's own)."""
        check(lib().ray_renderer_set_trace_variant(self._h, variant))

    def set_ray_sort(self, policy: int = -1) -> None:
        """Ray sorting before the wavefront's bounces (ray_renderer_set_ray_sort):
        -1 chosen per bounce by timing, 0 never, else a mask of bounces (0x3FF all)."""
        check(lib().ray_renderer_set_ray_sort(self._h, policy))

    def set_stream(self, stream: int = 0) -> None:
        """Enqueue the renderer's work on this cudaStream_t (0: its own stream)."""
        check(lib().ray_renderer_set_stream(self._h, stream or None))

    def frame_info(self) -> capi.FrameInfo:
        """Ray counts and error flags of the last RenderScene (waits for it)."""
        out = capi.FrameInfo()
        check(lib().ray_renderer_frame_info(self._h, C.byref(out)))
        return out

    def GetStats(self) -> dict:
        st = capi.Stats()
        check(lib().ray_get_stats(self._h, C.byref(st)))
        return {f: getattr(st, f) for f, _ in capi.Stats._fields_}

    def ResetStats(self) -> None:
        check(lib().ray_reset_stats(self._h))


def RegionContext(x: int = 0, y: int = 0, w: int = 0, h: int = 0) -> capi.Region:
    """RegionContext (RendererBase.h:35-51): a rect plus the iteration counter."""
    return capi.Region(capi.Rect(x, y, w, h), 0)


def render_batch(renderers, scenes, regions, samples: int = 1) -> None:
    """`samples` samples of every (renderer, scene, region) in one launch (ray_render_batch)."""
    n = len(renderers)
    if not (len(scenes) == n == len(regions)):
        raise ValueError("renderers, scenes and regions must have the same length")
    rs = (C.c_void_p * max(n, 1))(*[r.handle.value for r in renderers])
    ss = (C.c_void_p * max(n, 1))(*[s.handle.value for s in scenes])
    gs = (C.POINTER(capi.Region) * max(n, 1))(*[C.pointer(g) for g in regions])
    check(lib().ray_render_batch(rs, ss, gs, n, samples))


def create_renderer(w: int, h: int, device: int = 0) -> Renderer:
    """Ray::CreateRenderer (RendererFactory.h:19): always the CUDA renderer."""
    return Renderer(w, h, device)
