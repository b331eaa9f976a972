"""Geo (lightmap) cameras against the reference's Ref renderer: a camera with
type Geo renders the UV layer uv_index of instance mi_index's mesh, each
texel's jittered sample point rasterised to the first covering triangle
(SampleMeshInTextureSpace, src/Ray/internal/CoreRef.cpp:507-603) and shaded
as a camera-ray hit, texels no triangle covers showing the background
(RendererRef.cpp:142-149). The parity bars are those of the perspective
renders: the same pixels as the Ref renderer save for the rare path that
rounding sends elsewhere, and spherical-harmonics output likewise."""
import numpy as np
import pytest

from raydemo_b200 import api, scenes

from render_scenes import build_gpu, build_ref, image_diff, render_gpu, render_ref

pytestmark = pytest.mark.gpu


def _ref_render(reflib, spec, iterations, rect=(0, 0, 0, 0)):
    from oracle.oracle import RefRenderer

    w, h = spec["size"]
    rr = RefRenderer(reflib, w, h, RefRenderer.REF, True)
    sc = build_ref(reflib, spec)
    rr.render(sc, iterations, rect=rect, reset=True, nthreads=1)
    return rr.pixels(), rr.sh_data()


@pytest.mark.parametrize("overlap", [False, True], ids=["atlas", "overlapping"])
def test_lightmap_matches_ref_renderer(reflib, cuda_device, overlap):
    spec = scenes.lightmap_box(0, 96, overlap=overlap)
    gpu, r, _ = render_gpu(spec, 4)
    cpu = render_ref(reflib, spec, 4)
    d = image_diff(gpu, cpu)
    print("lightmap 4 spp", d)
    assert d["identical_px"] >= 0.95, d
    assert d["rmse"] <= 1e-3, d
    assert r.frame_info().kernel == 1 and r.frame_info().error_flags == 0
    # texels between the cells: the environment colour (0.1) with alpha 1, as in the reference
    bg = np.all(cpu == np.float32([0.1, 0.1, 0.1, 1.0]), axis=-1)
    assert bg.mean() > 0.05
    np.testing.assert_array_equal(gpu[bg], cpu[bg])
    # texels inside the cells that the paths of 4 samples found the light from
    assert (gpu[~bg][:, :3].sum(-1) > 0).mean() > 0.2


def test_lightmap_sh_region_and_path_kernel_setting(reflib, cuda_device):
    """Spherical-harmonics output (the lightmap baker's form) over a region,
    with the path kernel asked for: Geo cameras run on the wavefront."""
    spec = scenes.lightmap_box(1, 80)
    spec["camera"].update(output_sh=True)
    rect = (8, 4, 60, 52)
    gpu, r, _ = render_gpu(spec, 6, rect=rect, kernel=2)
    cpu, cpu_sh = _ref_render(reflib, spec, 6, rect=rect)
    d = image_diff(gpu, cpu)
    print("lightmap sh", d)
    assert d["identical_px"] >= 0.95, d
    assert d["rmse"] <= 1e-3, d
    sh = r.get_sh_data_ref()
    assert sh is not None and cpu_sh is not None
    x, y, w, h = rect
    a, b = sh[y:y + h, x:x + w], cpu_sh[y:y + h, x:x + w]
    same = np.all(a == b, axis=-1).mean()
    assert same >= 0.95, same
    assert np.sqrt(np.mean((a.astype(np.float64) - b) ** 2)) <= 1e-3


def test_lightmap_of_transformed_instance(reflib, cuda_device):
    """The icosphere instance (a translated transform) in its first UV layer:
    spherical UVs whose seam triangles wind backwards in texel space and
    sample nothing, as in the reference."""
    spec = scenes.cornell_box(2, 64, 64)
    spec["camera"] = {"type": api.Geo, "mi_index": 1, "uv_index": 0, "gamma": 1.0, "max_total_depth": 3, "max_diff_depth": 3,
                      "termination_start_depth": 3}
    spec["env"] = {"env_col": (0.3, 0.2, 0.1)}
    gpu, _, _ = render_gpu(spec, 3)
    cpu = render_ref(reflib, spec, 3)
    d = image_diff(gpu, cpu)
    print("sphere lightmap", d)
    assert d["identical_px"] >= 0.95, d
    assert d["rmse"] <= 1e-3, d


def test_geo_and_perspective_jobs_in_one_batch(reflib, cuda_device):
    """A batch of a lightmap and a perspective view: each equals its render alone."""
    specs = [scenes.lightmap_box(0, 64), scenes.cornell_box(0, 48, 40)]
    rs, scs = [], []
    for sp in specs:
        r = api.Renderer(*sp["size"])
        rs.append(r)
        scs.append(build_gpu(r, sp))
        r.Clear()
    regions = [api.RegionContext(), api.RegionContext()]
    api.render_batch(rs, scs, regions, 3)
    for sp, r in zip(specs, rs):
        alone, _, _ = render_gpu(sp, 3, kernel=1)
        np.testing.assert_array_equal(r.get_pixels_ref().view(np.uint32), alone.view(np.uint32))
    cpu = render_ref(reflib, specs[0], 3)
    d = image_diff(rs[0].get_pixels_ref(), cpu)
    assert d["identical_px"] >= 0.95 and d["rmse"] <= 1e-3, d


def test_geo_camera_api(cuda_device):
    """SceneBase::SetCamera / GetCamera for Geo cameras (SceneBase.cpp:22-84):
    a Geo camera keeps the slot's perspective fields and reports only its own;
    a bad instance or UV layer is an argument error at render time."""
    spec = scenes.lightmap_box(0, 32)
    r = api.Renderer(32, 32)
    sc = build_gpu(r, spec)
    persp = api.CameraDesc(type=api.Persp, dtype=api.SRGB, origin=(0.5, 0.5, -1.0), fwd=(0.0, 0.0, 1.0), fov=60.0)
    i = sc.AddCamera(persp)
    sc.SetCamera(i, api.CameraDesc(type=api.Geo, dtype=api.NoDevice, mi_index=0, uv_index=1, gamma=2.2))
    got = sc.GetCamera(i)
    assert got.type == api.Geo and got.mi_index == 0 and got.uv_index == 1
    assert got.dtype == api.SRGB  # the slot's, as SetCamera leaves it
    assert abs(got.gamma - 2.2) < 1e-6
    sc.SetCamera(i, api.CameraDesc(type=api.Geo, mi_index=7, uv_index=0))
    sc.set_current_cam(i)
    with pytest.raises(RuntimeError):
        r.RenderScene(sc, api.RegionContext())
    sc.SetCamera(i, api.CameraDesc(type=api.Geo, mi_index=0, uv_index=2))
    with pytest.raises(RuntimeError):
        r.RenderScene(sc, api.RegionContext())
    sc.SetCamera(i, api.CameraDesc(type=api.Ortho))
    with pytest.raises(RuntimeError):
        r.RenderScene(sc, api.RegionContext())
