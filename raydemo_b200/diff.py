"""Differentiable rendering of RAY_MAT_PRINCIPLED scenes from PyTorch.

`render` is a thin torch.autograd.Function over the C ABI: its forward is
`ray_render_diff` (the render loop with the parameters read from the given
tensors), its backward is the path-replay adjoint `ray_render_adjoint`. Both
run on the renderer's device, ordered on torch's current stream. torch is the
harness only (tensors, the optimiser); every pixel and gradient comes from
the library's kernels.
"""
from __future__ import annotations

import torch

from . import api

_SIDE = {}


def _enter(dev):
    """The stream the library's work goes on, ordered after torch's current
    stream: that stream itself, or (torch's legacy default stream does not
    order the library's non-blocking streams) a side stream made to wait for
    it. Returns (stream, the stream that must wait for it afterwards)."""
    cur = torch.cuda.current_stream(dev)
    if cur.cuda_stream != 0:
        return cur, None
    side = _SIDE.get(dev.index)
    if side is None:
        side = _SIDE[dev.index] = torch.cuda.Stream(dev)
    side.wait_stream(cur)
    return side, cur


def _leave(side, cur):
    if cur is not None:
        cur.wait_stream(side)


class _DiffRender(torch.autograd.Function):
    @staticmethod
    def forward(ctx, albedo, roughness, renderer, scene, material_slot, first_iteration, samples, roughness_sampling):
        if not (albedo.is_cuda and roughness.is_cuda):
            raise ValueError("parameters must be CUDA tensors")
        albedo = albedo.detach().contiguous().float()
        roughness = roughness.detach().contiguous().float()
        ah, aw, three = albedo.shape
        if three != 3:
            raise ValueError("albedo must be (h, w, 3)")
        rs = roughness_sampling.detach().contiguous().float() if roughness_sampling is not None else None
        scene.set_diff_params(albedo.data_ptr(), aw, ah, roughness.data_ptr(), roughness.numel(), material_slot,
                              rs.data_ptr() if rs is not None else 0)
        w, h = renderer.size()
        image = torch.empty((h, w, 3), dtype=torch.float32, device=albedo.device)
        per_sample = torch.empty((samples, h, w, 3), dtype=torch.float32, device=albedo.device)
        side, cur = _enter(albedo.device)
        renderer.set_stream(side.cuda_stream)
        renderer.render_diff(scene, first_iteration, samples, image.data_ptr(), per_sample.data_ptr())
        _leave(side, cur)
        ctx.save_for_backward(albedo, roughness, per_sample)
        ctx.rough_sampling = rs
        ctx.renderer, ctx.scene, ctx.slots = renderer, scene, material_slot
        ctx.first_iteration, ctx.samples = first_iteration, samples
        return image

    @staticmethod
    def backward(ctx, d_image):
        albedo, roughness, per_sample = ctx.saved_tensors
        r, sc = ctx.renderer, ctx.scene
        ah, aw, _ = albedo.shape
        # the parameters the forward pass read (the caller may have rebound them since)
        rs = ctx.rough_sampling
        sc.set_diff_params(albedo.data_ptr(), aw, ah, roughness.data_ptr(), roughness.numel(), ctx.slots,
                           rs.data_ptr() if rs is not None else 0)
        d = d_image.detach().contiguous().float()
        g_albedo = torch.zeros_like(albedo)
        g_rough = torch.zeros_like(roughness)
        side, cur = _enter(albedo.device)
        r.set_stream(side.cuda_stream)
        r.render_adjoint(sc, ctx.first_iteration, ctx.samples, per_sample.data_ptr(), d.data_ptr(), g_albedo.data_ptr(), g_rough.data_ptr())
        _leave(side, cur)
        return g_albedo, g_rough, None, None, None, None, None, None


def render(albedo: torch.Tensor, roughness: torch.Tensor, renderer: api.Renderer, scene: api.Scene, material_slot,
           first_iteration: int = 1, samples: int = 8, roughness_sampling: torch.Tensor | None = None) -> torch.Tensor:
    """The (h, w, 3) mean of `samples` samples (iterations first_iteration ..)
    of scene's current camera with the differentiable parameters albedo
    (ah, aw, 3) and roughness (n,); differentiable with respect to both.
    roughness_sampling: frozen roughness for direction sampling and pdfs."""
    return _DiffRender.apply(albedo, roughness, renderer, scene, material_slot, first_iteration, samples, roughness_sampling)
