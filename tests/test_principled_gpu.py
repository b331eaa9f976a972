"""The metallic-roughness material (RAY_MAT_PRINCIPLED) with next-event
estimation from quad and sun lights, against the oracle's CPU restatement
(orc_render_principled) on the same scenes and the same scrambled Sobol
sequence.

The oracle intersects instanced meshes the way the renderer does (instance box
test, ray taken to object space, the reference's triangle arithmetic), so hits
agree bit for bit and paths take the same directions; cos, sin, acos and pow
are computed in double and rounded once on both sides. The bar: per-pixel RMSE
over RGB of the clean buffer <= 1e-3, with at least 99% of pixels identical.
"""
import numpy as np
import pytest

from raydemo_b200 import api, scenes

from render_scenes import build_gpu, image_diff, render_gpu

pytestmark = pytest.mark.gpu

RMSE_MAX = 1e-3
IDENTICAL_MIN = 0.99


def _small_atrium(seed=0, w=64, h=48, bounces=4):
    return scenes.atrium(seed, w, h, bounces, level=2, n_spheres=4, tex_res=64)


@pytest.mark.parametrize("kernel", [1, 2], ids=["wavefront", "path"])
def test_atrium_matches_oracle(cuda_device, oracle, kernel):
    spec = _small_atrium()
    spp = 4
    gpu, r, sc = render_gpu(spec, spp, kernel=kernel)
    info = r.frame_info()
    assert info.error_flags == 0
    ref = oracle.render_principled(spec, spp)
    d = image_diff(gpu, ref)
    assert d["rmse"] <= RMSE_MAX, d
    assert d["identical_px"] >= IDENTICAL_MIN, d
    assert float(ref[..., :3].mean()) > 0.01  # the scene is lit


def test_atrium_deeper_paths(cuda_device, oracle):
    """8 bounces, 2 samples, a wider frame: the Russian-roulette and MIS
    branches of every bounce depth."""
    spec = _small_atrium(seed=3, w=96, h=54, bounces=8)
    gpu, r, _ = render_gpu(spec, 2, kernel=1)
    ref = oracle.render_principled(spec, 2)
    d = image_diff(gpu, ref)
    assert d["rmse"] <= RMSE_MAX, d
    assert d["identical_px"] >= IDENTICAL_MIN, d


def test_sun_reaches_open_scene(cuda_device, oracle):
    """No room: a ground quad and spheres lit by the sun alone (its shadow
    rays unblocked) and a sky colour."""
    spec = _small_atrium(seed=5)
    # keep only the floor of the room (its first two triangles)
    attrs, idx, shapes, layout = spec["meshes"][0]
    spec["meshes"][0] = (attrs, idx[:6], [(shapes[0][0], shapes[0][1], 0, 6)], layout)
    spec["lights"] = [spec["lights"][0]]
    spec["env"] = {"env_col": (0.3, 0.35, 0.45)}
    spec["camera"] = dict(spec["camera"], origin=(0.0, 6.0, -22.0), fwd=(0.0, -0.3, 1.0))
    gpu, r, _ = render_gpu(spec, 2, kernel=1)
    ref = oracle.render_principled(spec, 2)
    d = image_diff(gpu, ref)
    assert d["rmse"] <= RMSE_MAX, d
    assert d["identical_px"] >= IDENTICAL_MIN, d
    assert r.frame_info().shadow_rays > 0


def test_batch_of_principled_scenes(cuda_device):
    """render_batch over metallic-roughness scenes equals one render per scene."""
    specs = [_small_atrium(seed=s, w=48 + 16 * s, h=32 + 8 * s, bounces=4) for s in range(3)]
    single = [render_gpu(sp, 2, kernel=1)[0] for sp in specs]
    rs, scs = [], []
    for sp in specs:
        w, h = sp["size"]
        r = api.Renderer(w, h)
        rs.append(r)
        scs.append(build_gpu(r, sp))
    for r in rs:
        r.Clear()
    for kernel in (1, 2):
        for r in rs:
            r.Clear()
            r.set_kernel(kernel)
        api.render_batch(rs, scs, [api.RegionContext(0, 0, 0, 0) for _ in rs], samples=2)
        for r, ref in zip(rs, single):
            assert np.array_equal(r.get_pixels_ref(), ref), kernel


def test_principled_argument_checks(cuda_device):
    r = api.Renderer(8, 8)
    sc = r.CreateScene()
    with pytest.raises(RuntimeError):
        sc.AddMaterial(type=api.PrincipledMaterial, roughness=1.5)
    with pytest.raises(RuntimeError):
        sc.AddMaterial(type=api.PrincipledMaterial, metallic=-0.1)
    with pytest.raises(RuntimeError):
        sc.AddMaterial(type=api.PrincipledMaterial, main_texture=7)
    sc.AddMaterial(type=api.PrincipledMaterial, main_texture=0xFFFFFFFF, roughness=0.5, metallic=1.0)
    with pytest.raises(RuntimeError):  # parallel edges
        sc.AddLight(type=api.QuadLight, edge_u=(1.0, 0.0, 0.0), edge_v=(2.0, 0.0, 0.0))
    with pytest.raises(RuntimeError):  # no cone
        sc.AddLight(type=api.SunLight, direction=(0.0, -1.0, 0.0), angle=0.0)
