/*
 * oracle/refbuild/refbuild_capi.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * A C entry point around the reference's own CPU BVH builder
 * (src/Renderer/BVHBuilder.cpp, src/Renderer/BVHGeometry.cpp, compiled from
 * the reference sources by oracle/Makefile). It mirrors what the reference's
 * Scene::build and BVHData::build do for a triangle-only scene:
 *   BVHGeometry::addTriangleList      (src/Renderer/Scene.cpp:185-227)
 *   BVHBuilder::addTriangleList       (src/Renderer/BVHBuilder.cpp:265-280)
 *   BVHBuilder::addSphereLight        (src/Renderer/BVHBuilder.cpp:282-285)
 *   BVHBuilder::build / getBvhGpuSize / fillGpuBuffer
 *                                     (src/Renderer/BVHData.cpp:28-49)
 * and returns the packed buffer with its seven ranges in memory order
 * (blas, tri, prim, mat, light, node, leaf).
 */
#include "Renderer/BVHBuilder.h"
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace
{
    class NullRenderer final : public tim::IRenderer
    {
    public:
        tim::BufferHandle CreateBuffer(u32, tim::MemoryType, tim::BufferUsage) override { return {}; }
        void DestroyBuffer(tim::BufferHandle&) override {}
        void UploadBuffer(tim::BufferHandle, void*, u32) override {}
        void UploadBuffer(tim::BufferHandle, u32, void*, u32) override {}
    };
}

extern "C" {

struct timref_params {
    uint32_t maxDepth;
    uint32_t minObjPerNode;
    uint32_t minObjGain;
    float expandNodeVolumeThreshold;
    float expandNodeDimensionFactor;
};

struct timref_result {
    uint8_t* blob;
    uint64_t blob_size;
    uint32_t ranges[7][2];
    uint32_t num_triangles, num_blas, num_primitives, num_lights, num_nodes;
    float aabb_min[3], aabb_max[3];
    uint32_t vertex_offsets_count;
    uint32_t* vertex_offsets;   /* vertexOffset returned per chunk */
};

void timref_default_params(timref_params* p)
{
    tim::BVHBuildParameters d;
    p->maxDepth = d.maxDepth;
    p->minObjPerNode = d.minObjPerNode;
    p->minObjGain = d.minObjGain;
    p->expandNodeVolumeThreshold = d.expandNodeVolumeThreshold;
    p->expandNodeDimensionFactor = d.expandNodeDimensionFactor;
}

/*
 * Chunk c covers vertices [chunk[4c+0], chunk[4c+0]+chunk[4c+1]) of pos/nrm and
 * triangles [chunk[4c+2], chunk[4c+2]+chunk[4c+3]) of `local_idx` (3 u32 per
 * triangle, local to the chunk, < 65536). Chunk c's Lambert colour is
 * colors[3c..3c+2]. Light l: lights[8l..8l+7] = pos.xyz, radius, color.xyz,
 * sphereRadius (SphereLight, src/Shaders/core/primitive_cpp.glsl:96-102).
 */
int timref_build(const float* pos, const float* nrm, uint32_t num_vertex,
                 const uint32_t* chunk, uint32_t num_chunks, const uint32_t* local_idx,
                 const float* colors, const float* lights, uint32_t num_lights,
                 const timref_params* params, int multithread, timref_result* out)
{
    std::memset(out, 0, sizeof(*out));
    NullRenderer renderer;
    tim::BVHGeometry geometry(&renderer, num_vertex + 4);
    tim::BVHBuilder builder("oracle", geometry, false);

    out->vertex_offsets = (uint32_t*)std::malloc(sizeof(uint32_t) * (num_chunks ? num_chunks : 1));
    out->vertex_offsets_count = num_chunks;
    for (uint32_t c = 0; c < num_chunks; ++c) {
        const uint32_t v0 = chunk[4 * c + 0], nv = chunk[4 * c + 1];
        const uint32_t t0 = chunk[4 * c + 2], nt = chunk[4 * c + 3];
        if (nv > 65536u) return 1;
        u32 voff = geometry.addTriangleList(nv, reinterpret_cast<const vec3*>(pos + 3ull * v0),
                                            reinterpret_cast<const vec3*>(nrm + 3ull * v0), nullptr);
        out->vertex_offsets[c] = voff;
        builder.addTriangleList(voff, nt, local_idx + 3ull * t0,
                                tim::BVHBuilder::createLambertianMaterial({ colors[3 * c], colors[3 * c + 1], colors[3 * c + 2] }));
    }
    for (uint32_t l = 0; l < num_lights; ++l) {
        SphereLight sl;
        sl.pos = { lights[8 * l + 0], lights[8 * l + 1], lights[8 * l + 2] };
        sl.radius = lights[8 * l + 3];
        sl.color = { lights[8 * l + 4], lights[8 * l + 5], lights[8 * l + 6] };
        sl.sphereRadius = lights[8 * l + 7];
        builder.addSphereLight(sl);
    }

    tim::BVHBuildParameters bp;
    if (params) {
        bp.maxDepth = params->maxDepth;
        bp.minObjPerNode = params->minObjPerNode;
        bp.minObjGain = params->minObjGain;
        bp.expandNodeVolumeThreshold = params->expandNodeVolumeThreshold;
        bp.expandNodeDimensionFactor = params->expandNodeDimensionFactor;
    }
    builder.setParameters(bp);
    builder.build(multithread != 0);

    const u32 size = builder.getBvhGpuSize();
    out->blob = (uint8_t*)std::calloc(size ? size : 1, 1);
    out->blob_size = size;
    uvec2 tri, prim, mat, light, node, leaf, blas;
    builder.fillGpuBuffer(out->blob, tri, prim, mat, light, node, leaf, blas);
    const uvec2 r[7] = { blas, tri, prim, mat, light, node, leaf };
    for (int i = 0; i < 7; ++i) { out->ranges[i][0] = r[i].x; out->ranges[i][1] = r[i].y; }
    out->num_triangles = builder.getTrianglesCount();
    out->num_blas = builder.getBlasInstancesCount();
    out->num_primitives = builder.getPrimitivesCount();
    out->num_lights = builder.getLightsCount();
    out->num_nodes = builder.getNodesCount();
    Box bb = builder.getAABB();
    out->aabb_min[0] = bb.minExtent.x; out->aabb_min[1] = bb.minExtent.y; out->aabb_min[2] = bb.minExtent.z;
    out->aabb_max[0] = bb.maxExtent.x; out->aabb_max[1] = bb.maxExtent.y; out->aabb_max[2] = bb.maxExtent.z;
    return 0;
}

void timref_free(timref_result* r)
{
    std::free(r->blob);
    std::free(r->vertex_offsets);
    std::memset(r, 0, sizeof(*r));
}

}
