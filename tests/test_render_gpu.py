"""Render-loop parity: the GPU renderer against the reference renderer.

* the sample table and the primary rays, bit for bit, against the reference's
  UpdateHaltonSequence and GeneratePrimaryRays (RendererRef.cpp:327-358,
  CoreRef.cpp:427-505);
* the reference's own image tests: test_mesh_lights (64x64, 2048 samples, mean
  absolute 8-bit error <= 1.0 against its golden image, test_mesh_lights.cpp:
  216-240) and test_texture (256x256, 256 samples, mean |p - 0.5| <= 0.0015,
  test_texture.cpp:144-168);
* whole images against the reference's Ref renderer run on the same scene with
  the same sample sequence: per-pixel RMSE over RGB. The shading arithmetic is
  the reference's; the two differ where libm's float cos/sin/acos/pow return
  other than the correctly rounded value, which the GPU computes.
"""
import numpy as np
import pytest

from raydemo_b200 import api, scenes

from render_scenes import build_gpu, image_diff, render_gpu, render_ref

pytestmark = pytest.mark.gpu


def _mesh_lights_spec(ref_tests, w=64, h=64):
    attrs = ref_tests["scene1_attrs"].reshape(-1, 8)
    idx = ref_tests["scene1_indices"]
    g = ref_tests["scene1_groups"]
    white = np.full((1, 1, 4), 255, np.uint8)
    mats = [{"type": api.EmissiveMaterial, "strength": 10.0, "main_color": (1.0, 0.0, 0.0), "main_texture": 2},
            {"type": api.EmissiveMaterial, "strength": 10.0, "main_color": (0.0, 1.0, 0.0), "main_texture": 2},
            {"type": api.EmissiveMaterial, "strength": 10.0, "main_color": (0.0, 0.0, 1.0), "main_texture": 2},
            {"type": api.DiffuseMaterial, "main_color": (1.0, 1.0, 1.0), "main_texture": 2}]
    shapes = [(k, 0xFFFFFFFF, int(g[2 * k]), int(g[2 * k + 1])) for k in range(4)]
    cam = {"type": api.Persp, "filter": api.Box, "dtype": api.NoDevice, "origin": (2.0, 2.0, 0.0), "fwd": (-1.0, 0.0, 0.0),
           "fov": 45.0, "gamma": 1.0, "focus_distance": 1.0, "focus_factor": 0.0}
    return {"textures": [(white, True, True)], "materials": mats, "meshes": [(attrs, idx, shapes, 0)],
            "instances": [(0, np.eye(4, dtype=np.float32).reshape(-1))], "env": {"env_col": (0.0, 0.0, 0.0)}, "camera": cam,
            "size": (w, h)}


def _texture_spec(ref_tests):
    attrs = ref_tests["scene2_attrs"].reshape(-1, 8)
    idx = ref_tests["scene2_indices"]
    i, j = np.meshgrid(np.arange(512), np.arange(512))
    chk = np.where((i + j) % 2 == 1, 255, 0).astype(np.uint8)
    tex = np.stack([chk, chk, chk, np.full_like(chk, 255)], axis=-1)
    cam = {"type": api.Persp, "filter": api.Box, "dtype": api.NoDevice, "origin": (0.0, 10.0, 0.0), "fwd": (0.0, -1.0, 0.0),
           "up": (0.0, 0.0, -1.0), "fov": 90.0, "gamma": 1.0, "focus_distance": 1.0, "focus_factor": 0.0}
    return {"textures": [(tex, False, True)], "materials": [{"type": api.EmissiveMaterial, "main_texture": 2}],
            "meshes": [(attrs, idx, [(0, 0xFFFFFFFF, 0, len(idx))], 0)], "instances": [(0, np.eye(4, dtype=np.float32).reshape(-1))],
            "env": {"env_col": (0.5, 0.5, 0.5)}, "camera": cam, "size": (256, 256)}


def _camera_rb(spec):
    from oracle.oracle import RbCameraDesc

    c = api.CameraDesc(**spec["camera"]).to_c()
    d = RbCameraDesc()
    for f, _ in RbCameraDesc._fields_:
        setattr(d, f, getattr(c, f))
    return d


def test_sample_table_and_primary_rays_bit_exact(reflib, cuda_device, ref_tests):
    from oracle.oracle import PACKET_DTYPE

    spec = _mesh_lights_spec(ref_tests, 48, 40)
    spec["camera"].update(filter=api.Tent, focus_factor=0.3, focus_distance=1.7, skip_indirect_lighting=True)
    r = api.Renderer(48, 40)
    r.set_kernel(1)  # the wavefront keeps the primary rays in its first buffer
    sc = build_gpu(r, spec)
    rect = (5, 3, 30, 29)
    reg = api.RegionContext(*rect)
    for it in range(1, 4):
        r.RenderScene(sc, reg)
        table = r.debug_read(2)
        ref_table = reflib.halton_table(1)
        np.testing.assert_array_equal(table.view(np.uint32), ref_table.view(np.uint32))
        rays = r.debug_read(0)[: rect[2] * rect[3]]
        pay = r.debug_read(1)[: rect[2] * rect[3]]
        want = reflib.generate_primary_rays(_camera_rb(spec), it, rect, 48, 40, ref_table)
        o = np.stack([want["o"][:, k] for k in range(3)], 1)
        assert want.dtype == PACKET_DTYPE
        np.testing.assert_array_equal(rays[:, 0:3].view(np.uint32), o.astype(np.float32).view(np.uint32))
        np.testing.assert_array_equal(rays[:, 4:7].view(np.uint32), want["d"].astype(np.float32).view(np.uint32))
        np.testing.assert_array_equal(rays[:, 7].view(np.uint32), want["xy"].astype(np.int32).view(np.uint32))
        for name, cols in (("c", slice(0, 3)), ("do_dx", slice(4, 7)), ("dd_dx", slice(7, 10)), ("do_dy", slice(10, 13)),
                           ("dd_dy", slice(13, 16))):
            np.testing.assert_array_equal(pay[:, cols].view(np.uint32), want[name].astype(np.float32).view(np.uint32), err_msg=name)


def test_sample_table_past_256_iterations(reflib, cuda_device, ref_tests):
    spec = _mesh_lights_spec(ref_tests, 8, 8)
    spec["camera"]["skip_indirect_lighting"] = True
    r = api.Renderer(8, 8)
    sc = build_gpu(r, spec)
    reg = api.RegionContext()
    for _ in range(300):
        r.RenderScene(sc, reg)
    np.testing.assert_array_equal(r.debug_read(2).view(np.uint32), reflib.halton_table(256).view(np.uint32))


def test_mesh_lights_golden(ref_tests, cuda_device):
    """test_mesh_lights (mode 0): 2048 samples against the reference's golden
    image, with the reference's own tolerance."""
    img, r, _ = render_gpu(_mesh_lights_spec(ref_tests), 2048)
    golden = ref_tests["img1"]
    h, w = golden.shape[:2]
    p = np.minimum(img[..., :3], 1.0)
    u8 = (p * 255).astype(np.uint8)
    diff = np.abs(u8[::-1].astype(int) - golden[..., :3].astype(int)).mean()  # the test flips rows (test_mesh_lights.cpp:221-233)
    assert diff <= 1.0, diff


@pytest.mark.parametrize("kernel", [1, 2], ids=["wavefront", "path"])
def test_mesh_lights_matches_ref_renderer(reflib, ref_tests, cuda_device, kernel):
    spec = _mesh_lights_spec(ref_tests)
    gpu, _, _ = render_gpu(spec, 16, kernel=kernel)
    cpu = render_ref(reflib, spec, 16)
    d = image_diff(gpu, cpu)
    assert d["rmse"] <= 1e-3, d
    assert d["identical_px"] >= 0.95, d


def test_texture_scene(ref_tests, cuda_device):
    """test_texture: an emissive plane with a mipmapped checkerboard must
    average to grey (mean |p - 0.5| <= 0.0015 after 256 samples)."""
    img, _, _ = render_gpu(_texture_spec(ref_tests), 256)
    d = np.abs(img[..., :3] - 0.5).mean()
    assert d <= 0.0015, d


@pytest.mark.parametrize("kernel", [1, 2], ids=["wavefront", "path"])
def test_texture_matches_ref_renderer(reflib, ref_tests, cuda_device, kernel):
    spec = _texture_spec(ref_tests)
    gpu, _, _ = render_gpu(spec, 4, kernel=kernel)
    cpu = render_ref(reflib, spec, 4)
    d = image_diff(gpu, cpu)
    assert d["rmse"] <= 1e-3, d


@pytest.mark.parametrize("kernel", [1, 2], ids=["wavefront", "path"])
def test_cornell_matches_ref_renderer(reflib, cuda_device, kernel):
    """The small render configuration (Cornell box, 256x256, 1 sample, 4
    bounces) against the reference's Ref renderer."""
    spec = scenes.cornell_box(0)
    gpu, _, _ = render_gpu(spec, 1, kernel=kernel)
    cpu = render_ref(reflib, spec, 1)
    d = image_diff(gpu, cpu)
    print("cornell 1 spp", d)
    assert d["identical_px"] >= 0.95, d
    gpu8, _, _ = render_gpu(spec, 8, kernel=kernel)
    cpu8 = render_ref(reflib, spec, 8)
    d8 = image_diff(gpu8, cpu8)
    print("cornell 8 spp", d8)
    assert d8["rmse"] <= 1e-3, d8


def _lights_spec():
    """Punctual lights (point, spot, directional) with every Ref material:
    diffuse with roughness, glossy, refractive, transparent, mix; a sRGB
    texture with mips and the default normal map; a sRGB camera with gamma."""
    spec = scenes.cornell_box(3, 96, 80, max_bounces=6)
    rng = np.random.default_rng(7)
    tex = rng.integers(0, 256, (32, 32, 4)).astype(np.uint8)
    spec["textures"].append((tex, True, True))
    m = spec["materials"]
    m[0].update(main_texture=3, roughness=0.6)                       # floor: textured Oren-Nayar
    m[1] = {"type": api.GlossyMaterial, "main_color": (0.9, 0.8, 0.7), "main_texture": 2, "roughness": 0.3}
    m[5] = {"type": api.RefractiveMaterial, "main_color": (1, 1, 1), "main_texture": 2, "roughness": 0.05, "int_ior": 1.5,
            "ext_ior": 1.0}
    m.append({"type": api.TransparentMaterial, "main_color": (1, 1, 1), "main_texture": 2})
    transp = len(m) - 1
    m.append({"type": api.MixMaterial, "main_texture": 2, "strength": 0.5, "mix_materials": (1, transp), "int_ior": 1.3,
              "ext_ior": 1.0})
    mix = len(m) - 1
    # the short box: mix of glossy and transparent (non-solid triangles in shadow rays)
    attrs, idx, shapes, layout = spec["meshes"][0]
    shapes = list(shapes)
    shapes[6] = (mix, mix, shapes[6][2], shapes[6][3])
    spec["meshes"][0] = (attrs, idx, shapes, layout)
    spec["lights"] = [{"type": api.PointLight, "position": (0.5, 0.9, 0.5), "radius": 0.05, "color": (2.0, 2.0, 2.0)},
                      {"type": api.SpotLight, "position": (0.2, 0.8, 0.2), "radius": 0.02, "color": (3.0, 1.0, 1.0),
                       "direction": (0.3, -1.0, 0.4), "angle": 30.0},
                      {"type": api.DirectionalLight, "position": (0, 0, 0), "radius": 0.0, "color": (0.5, 0.5, 0.6),
                       "direction": (-0.2, -1.0, 0.3), "angle": 2.0}]
    spec["env"] = {"env_col": (0.2, 0.3, 0.4)}
    spec["camera"].update(dtype=api.SRGB, gamma=2.2, clamp=True)
    return spec


@pytest.mark.parametrize("kernel", [1, 2], ids=["wavefront", "path"])
def test_lights_and_materials_match_ref_renderer(reflib, cuda_device, kernel):
    spec = _lights_spec()
    gpu, _, _ = render_gpu(spec, 4, kernel=kernel)
    cpu = render_ref(reflib, spec, 4)
    d = image_diff(gpu, cpu)
    print("lights/materials 4 spp", d)
    assert d["identical_px"] >= 0.9, d
    assert d["rmse"] <= 1e-3, d


@pytest.mark.parametrize("kernel", [1, 2], ids=["wavefront", "path"])
def test_region_and_sh_match_ref_renderer(reflib, ref_tests, cuda_device, kernel):
    """A sub-rectangle region, coherent sampling and spherical-harmonics output
    (test_mesh_lights mode 1)."""
    spec = _mesh_lights_spec(ref_tests)
    spec["camera"].update(output_sh=True, use_coherent_sampling=True)
    rect = (8, 4, 40, 52)
    gpu, r, _ = render_gpu(spec, 8, rect=rect, kernel=kernel)
    cpu = render_ref(reflib, spec, 8, rect=rect)
    d = image_diff(gpu, cpu)
    assert d["identical_px"] >= 0.95, d
    assert d["rmse"] <= 1e-3, d
    sh = r.get_sh_data_ref()
    assert sh is not None and np.isfinite(sh).all()


def test_clear_resize_stats(ref_tests, cuda_device):
    spec = _mesh_lights_spec(ref_tests, 32, 32)
    r = api.Renderer(32, 32)
    sc = build_gpu(r, spec)
    r.Clear((0.25, 0.5, 0.75, 1.0))
    reg = api.RegionContext()
    r.RenderScene(sc, reg)
    assert reg.iteration == 1
    st = r.GetStats()
    assert st["time_primary_trace_us"] >= 0 and st["time_secondary_shade_us"] >= 0
    r.ResetStats()
    assert all(v == 0 for v in r.GetStats().values())
    r.Resize(40, 24)
    assert r.size() == (40, 24)
    reg = api.RegionContext()
    r.RenderScene(sc, reg)
    assert r.get_pixels_ref().shape == (24, 40, 4)
    with pytest.raises(api.capi.RayError):
        r.RenderScene(sc, api.RegionContext(30, 0, 20, 10))  # outside the framebuffer


@pytest.mark.parametrize("kernel", [1, 2], ids=["wavefront", "path"])
def test_batch_matches_single_renders(reflib, ref_tests, cuda_device, kernel):
    """The batched form: four scenes of different sizes (the mesh-lights
    scene, the texture scene, the Cornell box and the lights/materials scene,
    one of them as two regions of one framebuffer) rendered together, 3
    samples in two calls: the images equal each scene rendered alone, and the
    Cornell box equals the Ref renderer's."""
    specs = [_mesh_lights_spec(ref_tests), _texture_spec(ref_tests), scenes.cornell_box(0), _lights_spec()]
    rs, scs = [], []
    for sp in specs:
        w, h = sp["size"]
        r = api.Renderer(w, h)
        rs.append(r)
        scs.append(build_gpu(r, sp))
        r.Clear()
    rs[0].set_kernel(kernel)
    w3, h3 = specs[3]["size"]
    regions = [api.RegionContext(), api.RegionContext(), api.RegionContext(), api.RegionContext(0, 0, w3, h3 // 2),
               api.RegionContext(0, h3 // 2, w3, h3 - h3 // 2)]
    rr = rs + [rs[3]]
    ss = scs + [scs[3]]
    api.render_batch(rr, ss, regions)       # one sample
    api.render_batch(rr, ss, regions, 2)    # two more in one call
    info = rs[0].frame_info()
    assert info.kernel == kernel and info.error_flags == 0
    for sp, r in zip(specs, rs):
        alone, _, _ = render_gpu(sp, 3, kernel=1)
        batch = r.get_pixels_ref()
        np.testing.assert_array_equal(batch.view(np.uint32), alone.view(np.uint32))
    cpu = render_ref(reflib, specs[2], 3)
    d = image_diff(rs[2].get_pixels_ref(), cpu)
    assert d["rmse"] <= 1e-3 and d["identical_px"] >= 0.95, d


def test_kernel_choice_by_timing(ref_tests, cuda_device):
    """Default kernel choice: both kernels are timed on the first frames of a
    configuration, then one is kept; the image is the same either way."""
    spec = _mesh_lights_spec(ref_tests, 32, 32)
    img_auto, r, _ = render_gpu(spec, 12)
    kinds = {r.frame_info().kernel}
    img_wave, _, _ = render_gpu(spec, 12, kernel=1)
    np.testing.assert_array_equal(img_auto.view(np.uint32), img_wave.view(np.uint32))
    assert kinds <= {1, 2}
