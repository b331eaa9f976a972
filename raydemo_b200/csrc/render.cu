// Render-loop entry points of the C ABI (RendererBase::RenderScene and the
// framebuffer accessors).
#include "../../include/raygpu.h"
#include "scene.hpp"

using namespace rg;

extern "C" {

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
