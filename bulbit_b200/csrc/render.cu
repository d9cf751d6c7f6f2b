// Placeholder while the wavefront path tracer is written.
#include "accel.cuh"

using namespace bbg;

extern "C" {
bbg_status bbg_integrator_create(bbg_accel*, const int32_t*, const bbg_material*, int32_t, const bbg_light*, int32_t,
                                 int32_t, int32_t, int32_t, bbg_integrator** out)
{
    if (out) *out = nullptr;
    return Fail(BBG_ERR_UNSUPPORTED, "integrator not built yet");
}
bbg_status bbg_integrator_destroy(bbg_integrator*) { return BBG_OK; }
bbg_status bbg_integrator_light_pmf(const bbg_integrator*, float*) { return BBG_ERR_UNSUPPORTED; }
bbg_status bbg_render(bbg_integrator*, const bbg_camera*, const bbg_render_params*, bbg_film*, bbg_memory,
                      bbg_render_stats*)
{
    return BBG_ERR_UNSUPPORTED;
}
bbg_status bbg_sampler_draws(int32_t, int32_t, int32_t, int32_t, int32_t, float*) { return BBG_ERR_UNSUPPORTED; }
}
