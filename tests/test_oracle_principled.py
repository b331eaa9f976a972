"""The oracle's metallic-roughness path tracer on its own (CPU): light
records, determinism, and physical sanity checks of the restated formulas."""
import numpy as np

from raydemo_b200 import scenes


def _sphere_in_furnace(metallic, roughness, env=1.0, w=32, h=32):
    a, i = scenes.displaced_sphere(2, 0, amplitude=0.0)
    mats = [{"type": 6, "main_color": (1.0, 1.0, 1.0), "main_texture": 0xFFFFFFFF, "roughness": roughness, "metallic": metallic}]
    cam = {"type": 0, "filter": 1, "dtype": 0, "origin": (0.0, 0.0, -3.0), "fwd": (0.0, 0.0, 1.0), "up": (0.0, 1.0, 0.0), "fov": 30.0,
           "gamma": 1.0, "max_total_depth": 8, "max_diff_depth": 8, "termination_start_depth": 8}
    return {"textures": [], "materials": mats, "meshes": [(a, i, [(0, 0, 0, len(i))], 0)],
            "instances": [(0, np.eye(4, dtype=np.float32).reshape(-1))], "lights": [], "env": {"env_col": (env, env, env)},
            "camera": cam, "size": (w, h)}


def test_area_light_records(oracle):
    q = oracle.area_light(3, position=(1.0, 2.0, 3.0), color=(4.0, 5.0, 6.0), edge_u=(2.0, 0.0, 0.0), edge_v=(0.0, 0.0, 3.0))
    assert q[3].view(np.uint32) == 3
    np.testing.assert_array_equal(q[0:3], [1.0, 2.0, 3.0])
    assert q[7] == 6.0  # area
    np.testing.assert_array_equal(q[12:15], [0.0, -1.0, 0.0])  # u x v / |u x v|
    np.testing.assert_array_equal(q[16:19], [4.0, 5.0, 6.0])
    s = oracle.area_light(4, color=(5.0, 5.0, 5.0), direction=(0.0, -2.0, 0.0), angle=1.0)
    np.testing.assert_array_equal(s[12:15], [0.0, 1.0, 0.0])
    assert abs(float(s[11]) - np.cos(np.radians(0.5))) < 1e-7
    for bad in [dict(type=3, edge_u=(1.0, 0.0, 0.0), edge_v=(2.0, 0.0, 0.0)), dict(type=4, direction=(0.0, -1.0, 0.0), angle=0.0)]:
        try:
            oracle.area_light(**bad)
        except ValueError:
            continue
        raise AssertionError(bad)


def test_render_is_deterministic(oracle):
    spec = scenes.atrium(1, 40, 24, 4, level=1, n_spheres=3, tex_res=32)
    a = oracle.render_principled(spec, 2, nthreads=3)
    b = oracle.render_principled(spec, 2, nthreads=5)
    assert np.array_equal(a, b)
    assert np.isfinite(a).all() and a[..., :3].mean() > 0.0


def _ggx_albedo(mu, alpha, n=1 << 21, seed=0):
    """Directional albedo of the F = 1 GGX lobe with height-correlated Smith
    shadowing, by uniform hemisphere sampling (another estimator than the
    renderer's visible-normal sampling)."""
    rng = np.random.default_rng(seed)
    z, phi = rng.random(n), 2 * np.pi * rng.random(n)
    r = np.sqrt(1 - z * z)
    wi = np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)
    wo = np.array([np.sqrt(1 - mu * mu), 0.0, mu])
    hv = wi + wo
    hv /= np.linalg.norm(hv, axis=1, keepdims=True)
    a2 = alpha * alpha
    k = hv[:, 2] ** 2 * (a2 - 1) + 1
    d = a2 / (np.pi * k * k)
    lam = lambda c: 0.5 * (np.sqrt(1 + a2 * (1 - c * c) / (c * c)) - 1)
    g2 = 1 / (1 + lam(mu) + lam(wi[:, 2]))
    return float(np.mean(d * g2 / (4 * mu)) * 2 * np.pi)


def test_furnace_metal_matches_albedo(oracle):
    """A white metal sphere (F = 1) in a uniform white environment, seen head
    on: each pixel's value is the lobe's directional albedo (single
    scattering: below 1 at high roughness), which the renderer estimates by
    visible-normal sampling with weight G2 / G1."""
    for rough in (0.1, 0.6, 0.9):
        spec = _sphere_in_furnace(1.0, rough)
        img = oracle.render_principled(spec, 64)
        on = float(img[14:18, 14:18, :3].mean())
        assert on <= 1.005, (rough, on)
        if rough < 0.3:  # a near-mirror: uniform sampling cannot resolve the lobe
            assert on >= 0.98, (rough, on)
            continue
        want = _ggx_albedo(0.995, rough * rough)
        assert abs(on - want) <= 0.02 * want, (rough, on, want)


def test_furnace_background_is_environment(oracle):
    spec = _sphere_in_furnace(1.0, 0.3, env=0.5)
    img = oracle.render_principled(spec, 1)
    np.testing.assert_allclose(img[0, 0, :3], 0.5, rtol=1e-6)
    assert img[0, 0, 3] == 1.0
