"""The differentiable form: the forward pass with float albedo and roughness
parameters against the oracle, and the path-replay adjoint's gradients
against central finite differences (h = 1e-3) of this renderer and of the
oracle, with the loss sum((image - target)^2) over a small view of the atrium.

Albedo enters the estimator without changing any sampled direction (Russian
roulette is off in this configuration), so the adjoint equals the derivative
of the very estimator the finite differences difference: they agree to the
differences' own precision. Roughness also moves the sampled directions; the
adjoint holds sampling fixed (detached sampling: unbiased for the gradient
of the expected image), while differences of the same random numbers see the
paths jump across visibility edges as directions turn -- an estimator of the
same expectation, but one whose variance at these sample counts dwarfs the
gradient. The roughness differences are therefore taken with the sampling
roughness frozen at the evaluation point (ray_diff_params::
roughness_sampling), where the estimator is a smooth function of the
roughness and its derivative is exactly what the adjoint computes.
"""
import numpy as np
import pytest

from raydemo_b200 import api, scenes

from render_scenes import build_gpu

pytestmark = pytest.mark.gpu

H = 1e-3
REL_TOL = 0.02


def _setup(w=64, h=64, spp=4, level=2, n_spheres=6):
    import torch

    spec = scenes.diff_atrium(0, w, h, 4, level=level, n_spheres=n_spheres, tex_res=128)
    r = api.Renderer(w, h)
    sc = build_gpu(r, spec)
    dev = torch.device("cuda", 0)
    tgt_a = torch.tensor(spec["albedo_target"], device=dev)
    tgt_r = torch.tensor(spec["rough_target"], device=dev)
    return spec, r, sc, dev, tgt_a, tgt_r


def _render(r, sc, spec, albedo, rough, spp, rough_sampling=None):
    from raydemo_b200 import diff

    return diff.render(albedo, rough, r, sc, spec["material_slot"], 1, spp, rough_sampling)


def _loss(img, target):
    return float(((img.double() - target.double()) ** 2).sum())


def test_forward_matches_oracle(cuda_device, oracle):
    import torch

    spec, r, sc, dev, tgt_a, tgt_r = _setup()
    img = _render(r, sc, spec, tgt_a, tgt_r, 4).cpu().numpy()
    ps = oracle.principled_scene(spec, spec["albedo_target"], spec["rough_target"], spec["material_slot"])
    ref = oracle.render_principled(spec, 4, scene=ps, plain_mean=True)[..., :3]
    d = img.astype(np.float64) - ref
    assert np.sqrt(np.mean(d ** 2)) <= 1e-3
    assert np.mean(np.all(img == ref, axis=-1)) >= 0.99
    assert img.mean() > 0.01
    # the parameters matter: a constant albedo renders another image
    flat = _render(r, sc, spec, torch.full_like(tgt_a, 0.5), tgt_r, 4).cpu().numpy()
    assert np.abs(flat - img).max() > 1e-3


def _gradients(spec, r, sc, dev, tgt_a, tgt_r, spp):
    import torch

    target = _render(r, sc, spec, tgt_a, tgt_r, spp).detach()
    albedo = torch.full_like(tgt_a, 0.5).requires_grad_(True)
    rough = torch.full_like(tgt_r, 0.5).requires_grad_(True)
    img = _render(r, sc, spec, albedo, rough, spp)
    loss = ((img - target) ** 2).sum()
    loss.backward()
    return target, albedo, rough


def _fd(r, sc, spec, albedo, rough, target, spp, which, idx):
    import torch

    vals = []
    for s in (+1, -1):
        a = albedo.detach().clone()
        g = rough.detach().clone()
        if which == "albedo":
            a.view(-1)[idx] += s * H
        else:
            g[idx] += s * H
        with torch.no_grad():
            frozen = rough.detach() if which == "rough" else None
            vals.append(_loss(_render(r, sc, spec, a, g, spp, frozen), target))
    return (vals[0] - vals[1]) / (2 * H)


def test_adjoint_albedo_matches_finite_differences(cuda_device):
    spec, r, sc, dev, tgt_a, tgt_r = _setup()
    spp = 4
    target, albedo, rough = _gradients(spec, r, sc, dev, tgt_a, tgt_r, spp)
    g = albedo.grad.detach().cpu().numpy().reshape(-1)
    assert np.isfinite(g).all()
    order = np.argsort(-np.abs(g))
    cand = order[: max(1, int(np.count_nonzero(g) * 0.2))]  # texels the view sees well
    rng = np.random.default_rng(0)
    pick = rng.choice(cand, size=min(16, len(cand)), replace=False)
    for i in pick:
        fd = _fd(r, sc, spec, albedo, rough, target, spp, "albedo", int(i))
        assert abs(g[i] - fd) <= REL_TOL * abs(fd) + 1e-6, (int(i), float(g[i]), fd)


def test_adjoint_roughness_matches_finite_differences(cuda_device):
    spec, r, sc, dev, tgt_a, tgt_r = _setup(spp=8)
    spp = 8
    target, albedo, rough = _gradients(spec, r, sc, dev, tgt_a, tgt_r, spp)
    g = rough.grad.detach().cpu().numpy()
    assert np.isfinite(g).all()
    scale = np.abs(g).max()
    for k in range(len(g)):
        fd = _fd(r, sc, spec, albedo, rough, target, spp, "rough", k)
        assert abs(g[k] - fd) <= REL_TOL * max(abs(fd), 0.05 * scale), (k, float(g[k]), fd)


def test_adjoint_against_oracle_differences(cuda_device, oracle):
    """Central differences of the CPU restatement (the forward passes being
    identical) for the roughness slots and a few texels."""
    import torch

    spec, r, sc, dev, tgt_a, tgt_r = _setup(w=48, h=48, n_spheres=4)
    spp = 4
    target, albedo, rough = _gradients(spec, r, sc, dev, tgt_a, tgt_r, spp)
    ga = albedo.grad.detach().cpu().numpy().reshape(-1)
    gr = rough.grad.detach().cpu().numpy()
    tnp = target.cpu().numpy().astype(np.float64)
    a0 = albedo.detach().cpu().numpy()
    r0 = rough.detach().cpu().numpy()

    def oloss(a, g):
        ps = oracle.principled_scene(spec, a, g, spec["material_slot"], roughness_sampling=r0)
        img = oracle.render_principled(spec, spp, scene=ps, plain_mean=True)[..., :3].astype(np.float64)
        return float(((img - tnp) ** 2).sum())

    scale = np.abs(gr).max()
    for k in range(len(gr)):
        gp, gm = r0.copy(), r0.copy()
        gp[k] += H
        gm[k] -= H
        fd = (oloss(a0, gp) - oloss(a0, gm)) / (2 * H)
        assert abs(gr[k] - fd) <= REL_TOL * max(abs(fd), 0.05 * scale), (k, float(gr[k]), fd)
    for i in np.argsort(-np.abs(ga))[:4]:
        ap, am = a0.copy().reshape(-1), a0.copy().reshape(-1)
        ap[i] += H
        am[i] -= H
        fd = (oloss(ap.reshape(a0.shape), r0) - oloss(am.reshape(a0.shape), r0)) / (2 * H)
        assert abs(ga[i] - fd) <= REL_TOL * abs(fd) + 1e-6, (int(i), float(ga[i]), fd)
    del torch


def test_inverse_rendering_reduces_loss(cuda_device):
    import torch

    spec, r, sc, dev, tgt_a, tgt_r = _setup()
    spp = 4
    target = _render(r, sc, spec, tgt_a, tgt_r, spp).detach()
    albedo = torch.full_like(tgt_a, 0.5).requires_grad_(True)
    rough = torch.full_like(tgt_r, 0.5).requires_grad_(True)
    opt = torch.optim.Adam([albedo, rough], lr=0.02)
    losses = []
    for _ in range(30):
        opt.zero_grad()
        img = _render(r, sc, spec, albedo, rough, spp)
        loss = ((img - target) ** 2).sum()
        loss.backward()
        opt.step()
        with torch.no_grad():
            albedo.clamp_(0.0, 1.0)
            rough.clamp_(0.05, 1.0)
        losses.append(float(loss.detach()))
    assert losses[-1] < 0.5 * losses[0], losses[::5]


def test_inverse_rendering_recovers_parameters(cuda_device):
    """Parameter recovery: Adam towards a 1,024-sample target (16 calls of 64
    samples, each inside one 256-iteration block of the sample tables), the
    residual and the adjoint from independent renders, cosine-decayed rates.
    Both the roughness error and the albedo error of the texels the view sees
    well (the top fifth by gradient magnitude) fall."""
    import torch

    from raydemo_b200 import diff

    spec, r, sc, dev, tgt_a, tgt_r = _setup()
    slots = spec["material_slot"]

    def render(a, g, first, n):
        return diff.render(a, g, r, sc, slots, first, n)

    with torch.no_grad():
        firsts = [1, 65, 129] + [256 * b + 64 * k for b in (1, 2, 3) for k in range(4)] + [1024]
        target = sum(render(tgt_a, tgt_r, f, 64) for f in firsts) / len(firsts)
    a = torch.full_like(tgt_a, 0.5).requires_grad_(True)
    g = torch.full_like(tgt_r, 0.5).requires_grad_(True)
    ((render(a, g, 1536, 64) - target) ** 2).sum().backward()
    ga = a.grad.detach().abs().reshape(-1)
    well = ga >= torch.quantile(ga[ga > 0], 0.8)
    spp, steps = 16, 150
    opt = torch.optim.Adam([{"params": [a], "lr": 4e-3}, {"params": [g], "lr": 4e-3}])
    sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, steps)
    for step in range(steps):
        opt.zero_grad()
        first = 1280 + (2 * spp * step) % (256 - 2 * spp)
        with torch.no_grad():
            resid = render(a, g, first, spp) - target
        (2.0 * resid * render(a, g, first + spp, spp)).sum().backward()
        opt.step()
        sched.step()
        with torch.no_grad():
            a.clamp_(0.0, 1.0)
            g.clamp_(0.05, 1.0)

    def errs(av, gv):
        d = (av.detach().reshape(-1) - tgt_a.reshape(-1))[well]
        return float((gv.detach() - tgt_r).abs().mean()), float((d ** 2).mean().sqrt())

    r0, a0 = errs(torch.full_like(tgt_a, 0.5), torch.full_like(tgt_r, 0.5))
    r1, a1 = errs(a, g)
    print(f"roughness MAE {r0:.4f} -> {r1:.4f}; well-seen albedo RMSE {a0:.4f} -> {a1:.4f} ({int(well.sum())} texels)")
    assert r1 < 0.95 * r0, (r0, r1)
    assert a1 < 0.9 * a0, (a0, a1)


def test_adjoint_argument_checks(cuda_device):
    import torch

    spec, r, sc, dev, tgt_a, tgt_r = _setup(w=16, h=16)
    buf = torch.zeros(16 * 16 * 3 * 4, device=dev)
    with pytest.raises(RuntimeError):  # iterations must lie in one block of 256
        r.render_diff(sc, 250, 10, buf.data_ptr(), buf.data_ptr())
    sc2 = r.CreateScene()
    with pytest.raises(RuntimeError):  # no differentiable parameters
        r.render_adjoint(sc2, 1, 1, buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), buf.data_ptr())
    with pytest.raises(RuntimeError):  # slot out of range
        sc.set_diff_params(tgt_a.data_ptr(), 128, 128, tgt_r.data_ptr(), 8, [9] * len(spec["materials"]))
