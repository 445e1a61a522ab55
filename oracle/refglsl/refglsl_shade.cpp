/*
 * oracle/refglsl/refglsl_shade.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * The lighting step of the reference's cameraPass.comp, compiled with the flags
 * RayTracingPass::lightingPass sets (src/Renderer/raytracingPass.cpp:113-135:
 * FIRST_RECURSION_STEP, USE_LPF, USE_LPF_MASK): per pixel, the tracing step's
 * record and masks -> computeLighting -> the RGBA16F output image.
 */
#include "glsl_shim.h"

namespace glsl { namespace shade_pass {
#define FIRST_RECURSION_STEP 1
#define USE_LPF 1
#define USE_LPF_MASK 1
#include "cameraPass.comp"
uint tlas_collide(uint, Ray, ClosestHit&) { g_refglsl_error |= 4u; return 0; }
bool tlas_collide_fast(uint, Ray, float) { g_refglsl_error |= 4u; return false; }
}}  // namespace glsl::shade_pass

#include "refglsl_common.h"

namespace S = glsl::shade_pass;

extern "C" {

/* tracing: W*H*8 u32 (the tracing step's g_tracingData); sh16: the 7 rgba16f
 * light-probe images of resolution pd->lpfResolution; out: W*H*4 halves, zeroed
 * first (pixels the dispatch does not reach stay 0). */
int refglsl_shade(const orc_scene* s, const orc_pass_data* pd, const uint32_t* tracing, const uint16_t* sh16,
                  uint16_t* out) {
    using namespace glsl;
    g_refglsl_error = 0;
    REFGLSL_BIND_SCENE(S, s);
    std::memcpy((void*)&S::g_passData, pd, sizeof(orc_pass_data));
    const uint64_t W = pd->frameSize[0], H = pd->frameSize[1];
    S::g_tracingData.bind(tracing, 32ull * W * H);
    std::memset(out, 0, 8ull * W * H);
    S::g_outputImage.data = out;
    S::g_outputImage.w = (int)W;
    S::g_outputImage.h = (int)H;
    const uint64_t texels = (uint64_t)pd->lpfResolution[0] * pd->lpfResolution[1] * pd->lpfResolution[2];
    for (int k = 0; k < 7; ++k) {
        image3D& im = S::g_lpfTextures[k];
        im.w = (int)pd->lpfResolution[0];
        im.h = (int)pd->lpfResolution[1];
        im.d = (int)pd->lpfResolution[2];
        im.data = const_cast<uint16_t*>(sh16) + 4ull * texels * k;
    }
    const uint32_t L = LOCAL_SIZE;
    refglsl_dispatch((uint32_t)((W + L - 1) / L), (uint32_t)((H + L - 1) / L), 1, L, L, [] {}, [] { S::glsl_main(); });
    S::g_tracingData.bind(nullptr, 0);
    S::g_outputImage = image2D{};
    return (int)g_refglsl_error;
}

}  // extern "C"
