"""The adjoint for the reference's own diffuse material: gradients of an image
loss with respect to RAY_MAT_DIFFUSE main colours and Oren-Nayar roughness
(BRDF_OrenNayar, CoreRef.cpp:1579-1603; the diffuse branch of ShadeSurface,
CoreRef.cpp:2194-2256) in a Cornell box lit by its emissive quad and a point
light (whose shadow rays the adjoint traces again), checked against central
differences of the compiled reference renderer (the Ref backend through
oracle/_ref: the same scene with the material perturbed, rendered with the
same sample sequence) and of this renderer's forward pass.

Russian roulette is off (termination at the bounce limit), so the rendered
estimator is a smooth function of the parameters away from the Oren-Nayar
clamp, and its derivative is what the adjoint computes."""
import numpy as np
import pytest

from raydemo_b200 import api, scenes

from render_scenes import build_gpu, build_ref

pytestmark = pytest.mark.gpu

SPP = 4
H_FD = 1e-3
SLOTTED = (5, 8)  # the tall box and the icosphere
ROUGH = (0.45, 0.7)


def _spec(colors=None, rough=ROUGH):
    spec = scenes.cornell_box(0, 40, 32, max_bounces=3)
    spec["lights"] = [{"type": api.PointLight, "position": (0.5, 0.6, 0.0), "radius": 0.05, "color": (2.0, 1.8, 1.6)}]
    for k, m in enumerate(SLOTTED):
        spec["materials"][m] = dict(spec["materials"][m], roughness=float(rough[k]))
        if colors is not None:
            spec["materials"][m]["main_color"] = tuple(float(c) for c in colors[k])
    return spec


def _ref_image(reflib, spec):
    from oracle.oracle import RefRenderer

    w, h = spec["size"]
    rr = RefRenderer(reflib, w, h, RefRenderer.REF, True)
    rr.render(build_ref(reflib, spec), SPP, reset=True, nthreads=1)
    return rr.pixels()[..., :3].astype(np.float64)


def test_diffuse_adjoint_matches_reference_differences(reflib, cuda_device):
    import torch

    from raydemo_b200 import diff

    spec = _spec()
    colors0 = np.array([spec["materials"][m]["main_color"] for m in SLOTTED], np.float32)
    w, h = spec["size"]
    r = api.Renderer(w, h)
    sc = build_gpu(r, spec)
    slots = [-1] * len(spec["materials"])
    for k, m in enumerate(SLOTTED):
        slots[m] = k
    color = torch.tensor(colors0, device="cuda", requires_grad=True)
    rough = torch.tensor(ROUGH, dtype=torch.float32, device="cuda", requires_grad=True)
    # the forward pass with the parameters at the materials' values is the reference's image
    img = diff.render(None, rough, r, sc, slots, 1, SPP, color=color)
    ref0 = _ref_image(reflib, spec)
    assert np.abs(img.detach().cpu().numpy() - ref0).max() < 1e-4
    target = torch.tensor(_ref_image(reflib, _spec(colors0 * 0.8, (0.3, 0.5))), dtype=torch.float32, device="cuda")
    loss = ((img - target) ** 2).sum()
    loss.backward()
    g_col = color.grad.cpu().numpy()
    g_rough = rough.grad.cpu().numpy()
    tnp = target.cpu().numpy().astype(np.float64)

    def ref_loss(colors, rgh):
        return float(((_ref_image(reflib, _spec(colors, rgh)) - tnp) ** 2).sum())

    def our_loss(colors, rgh):
        with torch.no_grad():
            im = diff.render(None, torch.tensor(rgh, dtype=torch.float32, device="cuda"), r, sc, slots, 1, SPP,
                             color=torch.tensor(colors, dtype=torch.float32, device="cuda"))
        return float(((im.double() - target.double()) ** 2).sum())

    checks = []
    for k in range(len(SLOTTED)):
        for c in range(3):
            cp, cm = colors0.copy(), colors0.copy()
            cp[k, c] += H_FD
            cm[k, c] -= H_FD
            fd_ref = (ref_loss(cp, ROUGH) - ref_loss(cm, ROUGH)) / (2 * H_FD)
            fd_our = (our_loss(cp, ROUGH) - our_loss(cm, ROUGH)) / (2 * H_FD)
            checks.append(("color", k, c, float(g_col[k, c]), fd_ref, fd_our))
        rp, rm = list(ROUGH), list(ROUGH)
        rp[k] += H_FD
        rm[k] -= H_FD
        fd_ref = (ref_loss(colors0, rp) - ref_loss(colors0, rm)) / (2 * H_FD)
        fd_our = (our_loss(colors0, rp) - our_loss(colors0, rm)) / (2 * H_FD)
        checks.append(("roughness", k, 0, float(g_rough[k]), fd_ref, fd_our))
    for name, k, c, g, fr, fo in checks:
        print(f"{name} slot {k} ch {c}: adjoint {g:.6g}  reference FD {fr:.6g}  this renderer's FD {fo:.6g}")
    for name, k, c, g, fr, fo in checks:
        assert abs(fr) > 1e-3, (name, k, c, fr)
        assert abs(g - fr) <= 0.02 * abs(fr), (name, k, c, g, fr)
        assert abs(g - fo) <= 0.02 * abs(fo), (name, k, c, g, fo)


def test_diffuse_parameters_default_to_the_materials(cuda_device):
    """With the slot parameters equal to the materials' own values, the
    forward pass renders what the plain renderer renders (same samples)."""
    import torch

    from raydemo_b200 import diff

    spec = _spec()
    w, h = spec["size"]
    r = api.Renderer(w, h)
    sc = build_gpu(r, spec)
    slots = [-1] * len(spec["materials"])
    for k, m in enumerate(SLOTTED):
        slots[m] = k
    colors = torch.tensor([spec["materials"][m]["main_color"] for m in SLOTTED], dtype=torch.float32, device="cuda")
    with torch.no_grad():
        a = diff.render(None, torch.tensor(ROUGH, dtype=torch.float32, device="cuda"), r, sc, slots, 1, SPP, color=colors)
        sc.set_diff_params(None, 0, 0, 0, 0)
        b = diff.render(None, torch.tensor(ROUGH, dtype=torch.float32, device="cuda"), r, sc, [-1] * len(slots), 1, SPP)
    assert np.array_equal(a.cpu().numpy().view(np.uint32), b.cpu().numpy().view(np.uint32))
