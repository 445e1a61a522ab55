/*
 * oracle/refglsl/refglsl_probes.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * The reference's light-probe field update, compiled from its shaders as the
 * reference dispatches it (src/Renderer/lightProbFieldPass.cpp:90-140):
 *   - genLightProbField.comp with TRACING_STEP (one closest-hit ray per probe and
 *     direction, plus the leaf-light shadow mask),
 *   - genLightProbField.comp with USE_LPF (the lit value of each ray; the shader
 *     itself defines NO_LPF), and
 *   - updateLightProbField.comp (SH9 projection, blend with the previous field,
 *     FP16 image store).
 * Each shader copy is compiled in its own file (refglsl_probe_*.cpp include this
 * one with REFGLSL_PROBE_PART set), since their include guards allow one copy per
 * translation unit.
 */
#include "glsl_shim.h"

#if REFGLSL_PROBE_PART == 0
namespace glsl { namespace probe_trace {
#define TRACING_STEP 1
#include "genLightProbField.comp"
uint tlas_collide(uint, Ray, ClosestHit&) { g_refglsl_error |= 4u; return 0; }
bool tlas_collide_fast(uint, Ray, float) { g_refglsl_error |= 4u; return false; }
}}
namespace P = glsl::probe_trace;
#elif REFGLSL_PROBE_PART == 1
namespace glsl { namespace probe_light {
#define USE_LPF 1
#include "genLightProbField.comp"
uint tlas_collide(uint, Ray, ClosestHit&) { g_refglsl_error |= 4u; return 0; }
bool tlas_collide_fast(uint, Ray, float) { g_refglsl_error |= 4u; return false; }
}}
namespace P = glsl::probe_light;
#else
namespace glsl { namespace probe_update {
#include "updateLightProbField.comp"
}}
namespace P = glsl::probe_update;
#endif

#include "refglsl_common.h"

static_assert(sizeof(P::GenLightProbFieldConstants) == 80 + 16 * NUM_RAYS_PER_PROB, "constants layout");

/* GenLightProbFieldConstants from the oracle's probe description and the 64 ray
 * directions (four floats each, as the reference's constant buffer holds them). */
static void fill_constants(const orc_probe_desc* d, const float* dirs) {
    using namespace glsl;
    P::GenLightProbFieldConstants& c = P::g_lpfCst;
    c.lpfMin = vec4(d->aabbMin[0], d->aabbMin[1], d->aabbMin[2], d->aabbMin[3]);
    c.lpfMax = vec4(d->aabbMax[0], d->aabbMax[1], d->aabbMax[2], d->aabbMax[3]);
    c.lpfResolution = uvec4(d->resolution[0], d->resolution[1], d->resolution[2], d->resolution[3]);
    c.sunDir = vec4(d->sunDir[0], d->sunDir[1], d->sunDir[2], d->sunDir[3]);
    c.sunColor = vec4(d->sunColor[0], d->sunColor[1], d->sunColor[2], d->sunColor[3]);
    for (int i = 0; i < NUM_RAYS_PER_PROB; ++i)
        c.rays[i] = dirs ? vec4(dirs[4 * i], dirs[4 * i + 1], dirs[4 * i + 2], dirs[4 * i + 3]) : vec4(0.0f);
}

static uint32_t num_probes(const orc_probe_desc* d) { return d->resolution[0] * d->resolution[1] * d->resolution[2]; }

extern "C" {

#if REFGLSL_PROBE_PART == 0
/* Trace step over the whole field: trace_out = probes*64*2 uvec4 (g_tracingData),
 * zeroed first; sample = probe * 64 + direction. */
int refglsl_probe_trace(const orc_scene* s, const orc_probe_desc* d, const float* dirs, uint32_t* trace_out) {
    using namespace glsl;
    g_refglsl_error = 0;
    REFGLSL_BIND_SCENE(P, s);
    fill_constants(d, dirs);
    const uint64_t np = num_probes(d), bytes = 32ull * np * NUM_RAYS_PER_PROB;
    std::memset(trace_out, 0, bytes);
    P::g_tracingData.bind(trace_out, bytes);
    const uint32_t groups = (uint32_t)((np + UPDATE_LPF_NUM_PROBS_PER_GROUP - 1) / UPDATE_LPF_NUM_PROBS_PER_GROUP);
    refglsl_dispatch(groups, NUM_RAYS_PER_PROB, 1, UPDATE_LPF_NUM_PROBS_PER_GROUP, 1,
                     [] { for (auto& h : P::g_hitData) h = uvec4(0u, 0u, 0u, 0xFFFFFFFFu); },
                     [] { P::glsl_main(); });
    P::g_tracingData.bind(nullptr, 0);
    return (int)g_refglsl_error;
}
#elif REFGLSL_PROBE_PART == 1
/* Lighting step: reads the trace records, writes irradiance = probes*64*3 floats. */
int refglsl_probe_light(const orc_scene* s, const orc_probe_desc* d, const float* dirs, const uint32_t* trace_in,
                        float* irradiance) {
    using namespace glsl;
    g_refglsl_error = 0;
    REFGLSL_BIND_SCENE(P, s);
    fill_constants(d, dirs);
    const uint64_t np = num_probes(d);
    P::g_tracingData.bind(trace_in, 32ull * np * NUM_RAYS_PER_PROB);
    P::g_irradiance.bind(irradiance, 12ull * np * NUM_RAYS_PER_PROB);
    const uint32_t groups = (uint32_t)((np + UPDATE_LPF_NUM_PROBS_PER_GROUP - 1) / UPDATE_LPF_NUM_PROBS_PER_GROUP);
    refglsl_dispatch(groups, NUM_RAYS_PER_PROB, 1, UPDATE_LPF_NUM_PROBS_PER_GROUP, 1, [] {}, [] { P::glsl_main(); });
    P::g_tracingData.bind(nullptr, 0);
    P::g_irradiance.bind(nullptr, 0);
    return (int)g_refglsl_error;
}
#else
/* SH9 update: sh_basis = 64*9 floats (g_shCoef), irradiance = probes*64*3 floats,
 * images = the 7 rgba16f images (x fastest, 4 halves per texel), updated in place. */
int refglsl_probe_update(const orc_probe_desc* d, const float* sh_basis, const float* irradiance, uint16_t* images) {
    using namespace glsl;
    g_refglsl_error = 0;
    fill_constants(d, nullptr);
    const uint64_t np = num_probes(d);
    P::g_shCoef.bind(sh_basis, 4ull * 9 * NUM_RAYS_PER_PROB);
    P::g_irradiance.bind(irradiance, 12ull * np * NUM_RAYS_PER_PROB);
    for (int k = 0; k < 7; ++k) {
        image3D& im = P::g_lpfTextures[k];
        im.w = (int)d->resolution[0]; im.h = (int)d->resolution[1]; im.d = (int)d->resolution[2];
        im.data = images + 4ull * np * k;
    }
    const uint32_t groups = (uint32_t)((np + UPDATE_LPF_LOCALSIZE - 1) / UPDATE_LPF_LOCALSIZE);
    refglsl_dispatch(groups, 1, 1, UPDATE_LPF_LOCALSIZE, 1, [] {}, [] { P::glsl_main(); });
    P::g_shCoef.bind(nullptr, 0);
    P::g_irradiance.bind(nullptr, 0);
    return (int)g_refglsl_error;
}
#endif

}  // extern "C"
