/*
 * oracle/reftrace.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of TIM_Raytracing's GLSL traversal path, used as the
 * parity checker for the CUDA kernels and as the timed CPU baseline.
 * Nothing in the shipped library links or calls this code.
 *
 * Inputs are exactly the byte layouts the reference produces:
 *   - `blob` + `ranges`: the buffer written by BVHBuilder::fillGpuBuffer
 *     (src/Renderer/BVHBuilder.cpp:1319-1534) and its seven sub-ranges,
 *     indexed here in memory order (blas, tri, prim, mat, light, node, leaf).
 *   - `pos`: the position array of BVHGeometry (src/Renderer/BVHGeometry.cpp:69-78),
 *     three floats per vertex.
 */
#ifndef TIM_RT_ORACLE_REFTRACE_H
#define TIM_RT_ORACLE_REFTRACE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ORC_RANGE_BLAS = 0, ORC_RANGE_TRI = 1, ORC_RANGE_PRIM = 2, ORC_RANGE_MAT = 3,
    ORC_RANGE_LIGHT = 4, ORC_RANGE_NODE = 5, ORC_RANGE_LEAF = 6
};

typedef struct {
    const uint8_t *blob;
    uint64_t blob_size;
    uint32_t ranges[7][2];      /* {offset bytes, size bytes} */
    const float *pos;           /* xyz per vertex */
    const float *nrm;           /* xyz per vertex (lighting only) */
    uint32_t num_vertex;
    uint32_t num_nodes;         /* PushConstants.numNodes */
    uint32_t num_lights;        /* PushConstants.numLights */
} orc_scene;

/* One ray: {origin.xyz, tmax, dir.xyz, flags}; flags bit0 = any-hit. 32 bytes. */
typedef struct { float o[3]; float tmax; float d[3]; uint32_t flags; } orc_ray;

/* Per-ray memory-traffic counters of the reference's binary traversal. */
typedef struct { uint32_t node_fetch, backtrack_reload, leaf_visit, tri_test; } orc_stats;

#define ORC_MODE_CLOSEST 0u
#define ORC_MODE_ANY 1u
#define ORC_MODE_PER_RAY 2u
/* or'ed into the mode: any-hit rays take the two-level walk of USE_TRAVERSE_TLAS
 * scenes (traverseTlasFast); closest-hit rays keep the one-level walk */
#define ORC_MODE_TLAS 4u

int orc_version(void);

/* Batched trace. hit[4*i] = (vertexOffset, index01, index2_matId, bits(t)) for
 * closest hits (t = tmax, xyz = 0 on a miss); (occluded, 0, 0, bits(tmax)) for
 * any-hit rays. nid / bary / stats may be NULL. */
void orc_trace(const orc_scene *s, const orc_ray *rays, uint64_t n, uint32_t mode,
               uint32_t *hit, uint32_t *nid, float *bary, orc_stats *stats, int threads);

/* PassData of src/Shaders/struct_cpp.glsl:10-28, C layout (240 bytes). */
typedef struct {
    uint32_t frameSize[2]; float invFrameSize[2];
    float cameraPos[4]; float cameraDir[4];
    float frustumCorner00[4]; float frustumCorner10[4]; float frustumCorner01[4];
    float invProjView[16];
    float sunDir[4]; float sunColor[4];
    float sceneMinExtent[4]; float sceneMaxExtent[4];
    uint32_t lpfResolution[4];
} orc_pass_data;

#define ORC_CAM_PROB_MASK   1u  /* USE_LPF_MASK: 8 probe-visibility segments */
#define ORC_CAM_TILE_LIGHTS 2u  /* shadow rays to tile-culled lights instead of the leaf list */
#define ORC_CAM_BOUNCE      4u  /* one cosine-weighted diffuse bounce per hit */

/* cameraPass.comp TRACING_STEP. out: W*H*8 u32 = tracingData[2*pix], [2*pix+1].
 * tile_counts / tile_lists: output of orc_cull_lights (needed with TILE_LIGHTS).
 * bounce_out: W*H*4 u32 hit records of the bounce rays (BOUNCE). ray_counts[4]
 * accumulates (primary, shadow, probe, bounce) rays traced. */
void orc_camera(const orc_scene *s, const orc_pass_data *pd, uint32_t flags, uint32_t seed,
                const uint32_t *tile_counts, const uint32_t *tile_lists,
                uint32_t *out, uint32_t *bounce_out, uint64_t *ray_counts,
                uint64_t pix_begin, uint64_t pix_end, int threads);

/* Tile light-frustum culling (cullFrustum.glsl:9-13,63-100,136-151). Lists are
 * in ascending light order, at most 16 per tile. */
void orc_cull_lights(const orc_scene *s, const orc_pass_data *pd, uint32_t tiles_x, uint32_t tiles_y,
                     uint32_t *counts, uint32_t *lists, int threads);

/* Light-probe field. */
typedef struct {
    float aabbMin[4]; float aabbMax[4]; uint32_t resolution[4];
    float sunDir[4]; float sunColor[4];
    float hysteresis;           /* 0.03 in the reference */
    uint32_t num_dirs;
    uint32_t flags;
    uint32_t pad;
} orc_probe_desc;

void orc_probe_coord(uint32_t index, const uint32_t res[3], uint32_t coord[3]);
void orc_probe_trace(const orc_scene *s, const orc_probe_desc *pd, const float *dirs,
                     uint32_t probe_begin, uint32_t probe_end,
                     uint32_t *trace_out, float *irradiance, uint64_t *ray_counts, int threads);
void orc_probe_sh9(const orc_probe_desc *pd, const float *sh_basis, const float *irradiance,
                   uint32_t probe_begin, uint32_t probe_end, const float *prev, float *out_sh);
void orc_probe_octa(const orc_probe_desc *pd, const float *irradiance,
                    uint32_t probe_begin, uint32_t probe_end, float *out_texels);

/* cameraPass.comp lighting step (USE_LPF, USE_LPF_MASK): per pixel, from the
 * tracing step's records (tracing: W*H*8 u32) and the light-probe field's 7 RGBA16F
 * images (sh16, resolution pd->lpfResolution, the layout of orc_probe_sh9's images),
 * the lit colour as RGBA16F (out_rgba16, W*H*4) and optionally FP32 rgb (W*H*3).
 * Output row 0 is never reached by the reference's dispatch and is written as 0. */
#define ORC_SHADE_NO_LPF 1u   /* leave out the light-probe term */
void orc_shade_camera(const orc_scene *s, const orc_pass_data *pd, uint32_t flags, const uint32_t *tracing,
                      const uint16_t *sh16, uint16_t *out_rgba16, float *out_rgb32, int threads);
/* Bounce direction and basis helpers exposed for tests. */
void orc_bounce_dir(const float n[3], uint32_t pixel, uint32_t seed, float out[3]);
uint32_t orc_hash32(uint32_t x);

#ifdef __cplusplus
}
#endif
#endif
