/* Ray::CreateRenderer (src/Ray/RendererFactory.h:19) for builds that use this
 * library as the Ray library's backend: compile this file in place of
 * src/Ray/RendererFactory.cpp, with the Ray library's headers and this
 * directory on the include path, and link libraygpu.so. Code written against
 * the reference's interface -- its own tests, the demo's states -- then gets
 * the GPU renderer (raygpu_ray.hpp) for every backend flag: the reference's
 * factory picks OpenCL, AVX2, AVX, SSE2 or Ref by flag and CPU support
 * (RendererFactory.cpp:23-75), and falls back to a CPU backend when OpenCL
 * creation fails; this one has no CPU fallback, and without a usable CUDA
 * device it throws std::runtime_error with ray_last_error()'s message. The GPU
 * is settings_t::device_index where the build has that field (OpenCL
 * enabled) and it is set, else device 0. */
#include "Ray/RendererFactory.h"
#include "raygpu_ray.hpp"

std::shared_ptr<Ray::RendererBase> Ray::CreateRenderer(const settings_t &s, uint32_t flags, std::ostream &log_stream) {
    (void)flags;
    int device = 0;
#if !defined(DISABLE_OCL)
    if (s.device_index >= 0) device = s.device_index;
#endif
    log_stream << "Ray: Creating CUDA sm_100a renderer " << s.w << "x" << s.h << std::endl;
    return Gpu::CreateRenderer(s, device);
}
