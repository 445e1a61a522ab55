/*
 * oracle/refglsl/refglsl_tlas.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * The reference's camera shader compiled with USE_TRAVERSE_TLAS (the two-level
 * variant the reference's Scene::build enables with useTlasBlas,
 * src/Renderer/raytracingPass.cpp:100-135 and src/main.cpp:233-244), for its
 * any-hit entry point traverseForShadow -> traverseTlasFast -> tlas_collide_fast
 * (src/Shaders/bvh/bvhLighting.glsl:100-108, bvhTraversal_inline.glsl:83-151,
 * bvhCollision.glsl:321-348). The variant's closest-hit half (tlas_collide,
 * bvhCollision.glsl:286-319) does not compile in the reference (it names Hit,
 * HitBox and ClosestHit::nid, none of which exist); make_refglsl.py replaces its
 * body with a call to refglsl_unreachable, defined here to flag an error. The
 * any-hit path never reaches it.
 */
#include "glsl_shim.h"

namespace glsl { namespace tlas_pass {
inline void refglsl_unreachable() { g_refglsl_error |= 8u; }
#define TRACING_STEP 1
#define USE_TRAVERSE_TLAS 1
#include "cameraPass.comp"
}}  // namespace glsl::tlas_pass

#include "refglsl_common.h"

namespace T = glsl::tlas_pass;

extern "C" {

/* Any-hit rays of a two-level scene through the shader's traverseForShadow:
 * hit[4i] = (occluded, 0, 0, bits(tmax)), as orc_trace reports any-hit rays. */
int refglsl_trace_tlas(const orc_scene* s, const orc_ray* rays, uint64_t n, uint32_t* hit) {
    using namespace glsl;
    g_refglsl_error = 0;
    REFGLSL_BIND_SCENE(T, s);
    gl_LocalInvocationIndex = 0;
    for (uint64_t i = 0; i < n; ++i) {
        const orc_ray& rr = rays[i];
        T::Ray r = T::createRay(vec3(rr.o[0], rr.o[1], rr.o[2]), vec3(rr.d[0], rr.d[1], rr.d[2]));
        const bool occ = T::traverseForShadow(r, rr.tmax);
        hit[4 * i + 0] = occ ? 1u : 0u;
        hit[4 * i + 1] = 0;
        hit[4 * i + 2] = 0;
        hit[4 * i + 3] = floatBitsToUint(rr.tmax);
    }
    return (int)g_refglsl_error;
}

}  // extern "C"
