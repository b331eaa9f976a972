// Render-loop entry points of the C ABI (RendererBase::RenderScene and the
// framebuffer accessors).
#include "../../include/raygpu.h"
#include "scene.hpp"
#include "sort.cuh"

using namespace rg;

extern "C" {

int ray_sort_rays(ray_renderer *r, const float *rays, uint64_t n, const float root_min[3], const float cell_size[3], uint32_t *keys_out,
                  uint32_t *perm_out, float *rays_out, void *stream) {
    if (!r || !root_min || !cell_size || (n && (!rays || !perm_out))) {
        set_error("ray_sort_rays: null argument");
        return RAY_ERR_INVALID_ARG;
    }
    if (n > 0xffffffffull) {
        set_error("ray_sort_rays: at most 2^32 - 1 rays per call");
        return RAY_ERR_INVALID_ARG;
    }
    if (n == 0) return RAY_OK;
    RG_CUDA_TRY(cudaSetDevice(r->device));
    RG_CUDA_TRY(r->d_sort_scratch.ensure(sort_rays_scratch_bytes(n)));
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : r->stream;
    RG_CUDA_TRY(sort_rays(reinterpret_cast<const float4 *>(rays), n, root_min, cell_size, keys_out, perm_out,
                          reinterpret_cast<float4 *>(rays_out), r->d_sort_scratch.p, st));
    return RAY_OK;
}

int ray_clear(ray_renderer *r, const ray_pixel *c) {
    if (!r) {
        set_error("null renderer");
        return RAY_ERR_INVALID_ARG;
    }
    (void)c;
    set_error("ray_clear: the render loop is not built yet");
    return RAY_ERR_UNSUPPORTED;
}

int ray_render(ray_renderer *r, ray_scene *s, ray_region *region) {
    (void)r;
    (void)s;
    (void)region;
    set_error("ray_render: the render loop is not built yet");
    return RAY_ERR_UNSUPPORTED;
}

int ray_get_pixels(ray_renderer *r, const ray_pixel **out, int on_device) {
    (void)r;
    (void)out;
    (void)on_device;
    set_error("ray_get_pixels: the render loop is not built yet");
    return RAY_ERR_UNSUPPORTED;
}

int ray_get_sh_data(ray_renderer *r, const ray_shl1 **out) {
    (void)r;
    (void)out;
    set_error("ray_get_sh_data: the render loop is not built yet");
    return RAY_ERR_UNSUPPORTED;
}
}
