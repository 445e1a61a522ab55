/* Compiled as C99 against include/tim_rt.h and linked with libtim_rt.so by
 * tests/test_abi.py: the boundary header is plain C (what a cgo, JNI or other FFI
 * binding parses), and its host-only entry points work when called from C. Needs
 * no GPU: it builds a BVH on the host, validates it, checks its 8-wide form and
 * has a malformed image refused. Exit status 0 on success, else the failing step. */
#include <stdio.h>
#include <string.h>

#include "tim_rt.h"

int main(void) {
    if (sizeof(tim_rt_pass_data) != 240 || sizeof(tim_rt_push_constants) != 20 || sizeof(tim_rt_ray) != 32) {
        fprintf(stderr, "struct sizes differ from the reference layouts\n");
        return 1;
    }
    const char *version = tim_rt_version();
    if (!version || !strstr(version, "sm_100a")) return 2;

    /* a 3 x 3 vertex grid in the z = 0 plane, two triangles per cell: 8 triangles */
    float pos[9 * 3];
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
            float *p = pos + 3 * (3 * j + i);
            p[0] = (float)i;
            p[1] = (float)j;
            p[2] = 0.25f * (float)(i * j);
        }
    uint32_t tri[8 * 3];
    int t = 0;
    for (uint32_t j = 0; j < 2; ++j)
        for (uint32_t i = 0; i < 2; ++i) {
            const uint32_t a = 3 * j + i, b = a + 1, c = a + 3, d = a + 4;
            const uint32_t quad[2][3] = {{a, b, d}, {a, d, c}};
            for (int k = 0; k < 2; ++k, ++t) {   /* Triangle record: vertexOffset, i0 | i1 << 16, i2 | matId << 16 */
                tri[3 * t + 0] = 0u;
                tri[3 * t + 1] = quad[k][0] | (quad[k][1] << 16);
                tri[3 * t + 2] = quad[k][2];
            }
        }
    unsigned char material[48];
    memset(material, 0, sizeof(material));

    tim_rt_build_params bp;
    tim_rt_build_params_default(&bp);
    bp.max_leaf_size = 2;
    tim_rt_bvh_blob *blob = NULL;
    if (tim_rt_build_bvh(pos, 9, tri, 8, material, 1, NULL, 0, &bp, &blob) != TIM_RT_OK || !blob) {
        fprintf(stderr, "build: %s\n", tim_rt_last_error());
        return 3;
    }
    const uint8_t *bytes = NULL;
    uint64_t size = 0;
    uint32_t ranges[7][2];
    tim_rt_push_constants pc;
    float aabb[6];
    if (tim_rt_bvh_blob_info(blob, &bytes, &size, ranges, &pc, aabb) != TIM_RT_OK || !bytes || !size) return 4;
    if (pc.numTriangles != 8u || !(aabb[0] <= 0.0f && aabb[3] >= 2.0f && aabb[3] < 2.001f)) {
        fprintf(stderr, "image: %u triangles, box x [%g, %g]\n", pc.numTriangles, aabb[0], aabb[3]);
        return 5;
    }
    uint32_t depth = 0;
    if (tim_rt_validate_bvh(bytes, size, (const uint32_t(*)[2])ranges, &pc, 9, &depth) != TIM_RT_OK || depth == 0) {
        fprintf(stderr, "validate: %s\n", tim_rt_last_error());
        return 6;
    }
    tim_rt_wide_report rep;
    if (tim_rt_wide_check(bytes, size, (const uint32_t(*)[2])ranges, &pc, pos, 9, &rep) != TIM_RT_OK ||
        rep.triangles != 8u || rep.nodes == 0u) {
        fprintf(stderr, "wide check: %s\n", tim_rt_last_error());
        return 7;
    }
    ranges[TIM_RT_RANGE_NODE][0] += 4u;   /* a misaligned node range is refused, with a message */
    if (tim_rt_validate_bvh(bytes, size, (const uint32_t(*)[2])ranges, &pc, 9, &depth) != TIM_RT_EINVAL) return 8;
    const char *msg = tim_rt_last_error();
    if (!msg || !msg[0]) return 9;
    tim_rt_bvh_blob_free(blob);
    printf("ok %u nodes, depth %u, %u wide nodes\n", pc.numNodes, depth, rep.nodes);
    return 0;
}
