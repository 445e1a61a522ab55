/*
 * oracle/refglsl/refglsl_camera.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * The reference's cameraPass.comp, compiled with the flags its tracing pass sets
 * (src/Renderer/raytracingPass.cpp:100-101: TRACING_STEP, USE_LPF_MASK), and its
 * traversal entry points (baseRaytracingPass.glsl rayTrace, bvhTraversal_inline.glsl
 * traverseBvh, bvhLighting.glsl traverseForShadow), exported for the tests.
 */
#include "glsl_shim.h"

namespace glsl { namespace camera_pass {
#define TRACING_STEP 1
#define USE_LPF_MASK 1
#include "cameraPass.comp"

/* Declared by bvhTraversal.glsl for its TLAS variant but only defined under
 * USE_TRAVERSE_TLAS, which the reference leaves off; never reached here. */
uint tlas_collide(uint, Ray, ClosestHit&) { g_refglsl_error |= 4u; return 0; }
bool tlas_collide_fast(uint, Ray, float) { g_refglsl_error |= 4u; return false; }
}}  // namespace glsl::camera_pass

#include "refglsl_common.h"

namespace C = glsl::camera_pass;
static_assert(sizeof(C::PassData) == sizeof(orc_pass_data), "PassData layout");
static_assert(sizeof(C::PackedBVHNode) == 64 && sizeof(C::BlasHeader) == 32 && sizeof(C::PackedLight) == 56,
              "std430 record sizes");

extern "C" {

int refglsl_version(void) { return 1; }

/* Same contract as orc_trace (oracle/reftrace.h): hit[4i] = the ClosestHit_getHitData
 * record (vertexOffset, index01, index2_matId, bits(t)) and nid[i] = ClosestHit_getNid
 * for closest-hit rays; (occluded, 0, 0, bits(tmax)) and 0xFFFFFFFF for any-hit rays.
 * The reference leaves a miss's triangle words and nid undefined (shared memory that
 * no hit wrote); they read (0, 0, 0) and 0xFFFFFFFF here, as in the oracle. */
int refglsl_trace(const orc_scene* s, const orc_ray* rays, uint64_t n, uint32_t mode, uint32_t* hit, uint32_t* nid) {
    using namespace glsl;
    g_refglsl_error = 0;
    REFGLSL_BIND_SCENE(C, s);
    gl_LocalInvocationIndex = 0;
    for (uint64_t i = 0; i < n; ++i) {
        const orc_ray& rr = rays[i];
        C::Ray r = C::createRay(vec3(rr.o[0], rr.o[1], rr.o[2]), vec3(rr.d[0], rr.d[1], rr.d[2]));
        bool any = mode == ORC_MODE_ANY || (mode == ORC_MODE_PER_RAY && (rr.flags & 1u));
        if (any) {
            bool occ = C::traverseForShadow(r, rr.tmax);
            hit[4 * i + 0] = occ ? 1u : 0u; hit[4 * i + 1] = 0; hit[4 * i + 2] = 0; hit[4 * i + 3] = floatBitsToUint(rr.tmax);
            if (nid) nid[i] = 0xFFFFFFFFu;
            continue;
        }
        C::g_hitData[0] = uvec4(0u, 0u, 0u, 0xFFFFFFFFu);
        C::ClosestHit h;
        if (rr.tmax == float(TMAX)) {
            C::rayTrace(r, h);                                    /* starts at t = TMAX */
        } else {
            h.t = rr.tmax;                                        /* rayTrace with the ray's own tmax */
            C::traverseBvh(r, C::g_Constants.numNodes == 1 ? NID_LEAF_BIT : 0, h);
        }
        uvec4 rec = C::ClosestHit_getHitData(h);
        for (int k = 0; k < 4; ++k) hit[4 * i + k] = rec.v[k];
        if (nid) nid[i] = C::ClosestHit_getNid(h);
    }
    return (int)g_refglsl_error;
}

/* cameraPass.comp TRACING_STEP over a whole frame: out = W*H*2 uvec4 (g_tracingData),
 * zeroed first. LPF images are not read by the tracing step. */
int refglsl_camera(const orc_scene* s, const orc_pass_data* pd, uint32_t* out) {
    using namespace glsl;
    g_refglsl_error = 0;
    REFGLSL_BIND_SCENE(C, s);
    std::memcpy((void*)&C::g_passData, pd, sizeof(orc_pass_data));
    const uint64_t W = pd->frameSize[0], H = pd->frameSize[1];
    std::memset(out, 0, 32ull * W * H);
    C::g_tracingData.bind(out, 32ull * W * H);
    const uint32_t L = LOCAL_SIZE;
    refglsl_dispatch((uint32_t)((W + L - 1) / L), (uint32_t)((H + L - 1) / L), 1, L, L,
                     [] { for (auto& d : C::g_hitData) d = uvec4(0u, 0u, 0u, 0xFFFFFFFFu); },
                     [] { C::glsl_main(); });
    C::g_tracingData.bind(nullptr, 0);
    return (int)g_refglsl_error;
}

}  // extern "C"
