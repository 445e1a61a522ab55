/*
 * oracle/refglsl/refglsl_common.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Binds an orc_scene (the reference's fillGpuBuffer bytes and geometry arrays,
 * oracle/reftrace.h) to the buffer views that a compiled shader copy declares,
 * and dispatches compute invocations one at a time. Included by each driver
 * after its shader copy.
 */
#pragma once
#include "../reftrace.h"

#include <cstdint>
#include <cstring>

/* Binds the scene buffers of bvhBindings.glsl and the push constants of a shader
 * copy living in namespace NS. numTriangles / numBlas / numPrimitives come from
 * the buffer sizes (12, 32 and 28 bytes per record). */
#define REFGLSL_BIND_SCENE(NS, s)                                                                          \
    do {                                                                                                   \
        const orc_scene* s_ = (s);                                                                         \
        auto rng = [&](int k) { return (const void*)(s_->blob + s_->ranges[k][0]); };                      \
        NS::g_blasHeader.bind(rng(ORC_RANGE_BLAS), s_->ranges[ORC_RANGE_BLAS][1]);                          \
        NS::g_BvhTriangleData.bind(rng(ORC_RANGE_TRI), s_->ranges[ORC_RANGE_TRI][1]);                       \
        NS::g_BvhPrimitiveData.bind(rng(ORC_RANGE_PRIM), s_->ranges[ORC_RANGE_PRIM][1]);                    \
        NS::g_BvhMaterialData.bind(rng(ORC_RANGE_MAT), s_->ranges[ORC_RANGE_MAT][1]);                       \
        NS::g_BvhLightData.bind(rng(ORC_RANGE_LIGHT), s_->ranges[ORC_RANGE_LIGHT][1]);                      \
        NS::g_BvhNodeData.bind(rng(ORC_RANGE_NODE), s_->ranges[ORC_RANGE_NODE][1]);                         \
        NS::g_BvhLeafData.bind(rng(ORC_RANGE_LEAF), s_->ranges[ORC_RANGE_LEAF][1]);                         \
        NS::g_positionData.bind(s_->pos, 12ull * s_->num_vertex);                                          \
        NS::g_normalData.bind(s_->nrm, 12ull * s_->num_vertex);                                            \
        NS::g_texCoordData.bind(nullptr, 0);                                                               \
        NS::g_Constants.numTriangles = s_->ranges[ORC_RANGE_TRI][1] / 12u;                                 \
        NS::g_Constants.numBlas = s_->ranges[ORC_RANGE_BLAS][1] / 32u;                                     \
        NS::g_Constants.numPrimitives = s_->ranges[ORC_RANGE_PRIM][1] / 28u;                               \
        NS::g_Constants.numLights = s_->num_lights;                                                        \
        NS::g_Constants.numNodes = s_->num_nodes;                                                          \
    } while (0)

/* Runs `body` once per invocation of a dispatch of (gx, gy, gz) work groups of
 * (lx, ly, 1) invocations, with the gl_* built-ins set; `group_begin` runs before
 * each work group's first invocation (shared memory starts cleared). */
template <class G, class B>
inline void refglsl_dispatch(uint32_t gx, uint32_t gy, uint32_t gz, uint32_t lx, uint32_t ly, G&& group_begin, B&& body) {
    using namespace glsl;
    gl_NumWorkGroups = uvec3(gx, gy, gz);
    for (uint32_t z = 0; z < gz; ++z)
        for (uint32_t y = 0; y < gy; ++y)
            for (uint32_t x = 0; x < gx; ++x) {
                gl_WorkGroupID = uvec3(x, y, z);
                group_begin();
                for (uint32_t j = 0; j < ly; ++j)
                    for (uint32_t i = 0; i < lx; ++i) {
                        gl_LocalInvocationID = uvec3(i, j, 0u);
                        gl_LocalInvocationIndex = j * lx + i;
                        gl_GlobalInvocationID = uvec3(x * lx + i, y * ly + j, z);
                        body();
                    }
            }
}
