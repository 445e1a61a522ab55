/*
 * oracle/reftrace.c -- TEST INFRASTRUCTURE ONLY (parity checker and CPU baseline).
 *
 * Scalar C restatement of TIM_Raytracing's GLSL compute path. Each function
 * names the reference lines it follows. Floating-point policy (pinned, the
 * same in the CUDA kernels): no FMA contraction (-ffp-contract=off), IEEE
 * division and square root, C99 fminf/fmaxf for GLSL min/max, dot products
 * summed left to right, GLSL cross() component order.
 *
 * Built by oracle/Makefile with -O2 -ffp-contract=off -fno-fast-math -fopenmp.
 */
#include "reftrace.h"
#include <math.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define TMAX 100.0f                    /* struct_cpp.glsl:5 */
#define EPSILON_TRI 1e-7f              /* collision.glsl:62, 10e-8 */
#define OFFSET_RAY_COLLISION 1e-5f     /* system.glsl:45, 10e-6 */
#define NID_LEAF_BIT 0x80000000u       /* struct_cpp.glsl:52-55 */
#define NID_MASK 0x3FFFFFFFu
#define NID_LEFT_LEAF_BIT 0x80000000u
#define NID_RIGHT_LEAF_BIT 0x40000000u
#define TRIANGLE_BITS 12u              /* primitive_cpp.glsl:18-21 */
#define BLAS_BITS 8u
#define PRIM_BITS 8u
#define LIGHT_BITS 4u
#define LIGHT_SPHERE 1u                /* primitive_cpp.glsl:8 */
#define MAT_EMISSIVE 1u
#define MAT_LAMBERT 2u
#define MAT_TRANSPARENT 4u
#define MAT_PBR 5u

int orc_version(void) { return 3; }

typedef struct { float x, y, z; } v3;

static inline v3 mk(float x, float y, float z) { v3 r; r.x = x; r.y = y; r.z = z; return r; }
static inline v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 mul(v3 a, v3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3 muls(v3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline v3 divs(v3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
static inline v3 neg(v3 a) { return mk(-a.x, -a.y, -a.z); }
static inline float dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross3(v3 a, v3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
static inline float length3(v3 a) { return sqrtf(dot3(a, a)); }
static inline v3 normalize3(v3 a) { return divs(a, sqrtf(dot3(a, a))); }
static inline uint32_t fbits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline v3 ld3(const float *p) { return mk(p[0], p[1], p[2]); }

/* ---------------------------------------------------------------- scene access */
typedef struct { uint32_t nid[4]; float n0xy[4]; float n1xy[4]; float nz[4]; } packed_node; /* primitive_cpp.glsl:80-86 */
typedef struct { float mn[3]; uint32_t matId; float mx[3]; uint32_t rootIndex; } blas_header; /* primitive_cpp.glsl:88-94 */
typedef struct { uint32_t iparam; float fparam[13]; } packed_light;                         /* primitive_cpp.glsl:113-117 */
typedef struct { uint32_t type_ids[4]; float color[4]; float params[4]; } material;        /* primitive_cpp.glsl:67-72 */

static inline const packed_node *node_at(const orc_scene *s, uint32_t i) {
    return (const packed_node *)(s->blob + s->ranges[ORC_RANGE_NODE][0]) + i;
}
static inline const uint32_t *leaf_data(const orc_scene *s) {
    return (const uint32_t *)(s->blob + s->ranges[ORC_RANGE_LEAF][0]);
}
static inline uint32_t leaf_words(const orc_scene *s) { return s->ranges[ORC_RANGE_LEAF][1] / 4u; }
static inline const blas_header *blas_at(const orc_scene *s, uint32_t i) {
    return (const blas_header *)(s->blob + s->ranges[ORC_RANGE_BLAS][0]) + i;
}
static inline const packed_light *light_at(const orc_scene *s, uint32_t i) {
    return (const packed_light *)(s->blob + s->ranges[ORC_RANGE_LIGHT][0]) + i;
}
static inline const material *material_at(const orc_scene *s, uint32_t i) {
    return (const material *)(s->blob + s->ranges[ORC_RANGE_MAT][0]) + i;
}

/* Leaf header read. The reference reads g_BvhLeafData[0xFFFFFFFF] for nodes whose
 * packed count was 0 (BVHBuilder.cpp:1515); with robust buffer access that read
 * yields 0, which this restatement (and the CUDA path) define as "no objects". */
static inline uint32_t leaf_header(const orc_scene *s, uint32_t off) {
    return (off == 0xFFFFFFFFu || off >= leaf_words(s)) ? 0u : leaf_data(s)[off];
}

typedef struct { v3 from, dir; } ray_t;
typedef struct { v3 mn, mx; } box_t;

/* collision.glsl:23-40 CollideBox (STORE_RAY_INVDIR = 0: true division). */
static inline float collide_box(const ray_t *r, box_t b, float tmax) {
    float t0x = (b.mn.x - r->from.x) / r->dir.x;
    float t0y = (b.mn.y - r->from.y) / r->dir.y;
    float t0z = (b.mn.z - r->from.z) / r->dir.z;
    float t1x = (b.mx.x - r->from.x) / r->dir.x;
    float t1y = (b.mx.y - r->from.y) / r->dir.y;
    float t1z = (b.mx.z - r->from.z) / r->dir.z;
    float sx = fminf(t0x, t1x), sy = fminf(t0y, t1y), sz = fminf(t0z, t1z);
    float bx = fmaxf(t0x, t1x), by = fmaxf(t0y, t1y), bz = fmaxf(t0z, t1z);
    float tmin = fmaxf(0.0f, fmaxf(sx, fmaxf(sy, sz)));
    float tm = fminf(tmax, fminf(bx, fminf(by, bz)));
    return (tmin < tm) ? tmin : -1.0f;
}

/* collision.glsl:58-95 CollideTriangle (Moller-Trumbore, IGNORE_BACKFACE off).
 * Also returns the barycentrics u, v of an accepted hit. */
static inline float collide_triangle(const ray_t *r, v3 p0, v3 p1, v3 p2, float tmax, float *uo, float *vo) {
    v3 edge1 = sub(p1, p0);
    v3 edge2 = sub(p2, p0);
    v3 h = cross3(r->dir, edge2);
    float a = dot3(edge1, h);
    if (fabsf(a) < EPSILON_TRI) return -1.0f;
    float f = 1.0f / a;
    v3 s = sub(r->from, p0);
    float u = f * dot3(s, h);
    if (clampf(u, 0.0f, 1.0f) != u) return -1.0f;
    v3 q = cross3(s, edge1);
    float v = f * dot3(r->dir, q);
    if (v < 0.0f || u + v > 1.0f) return -1.0f;
    float t = f * dot3(edge2, q);
    if (t > EPSILON_TRI && t < tmax) { *uo = u; *vo = v; return t; }
    return -1.0f;
}

/* bvhBindings.glsl:57-62 loadTriangleVertices + primitive_cpp.glsl:121-134 getIndex*. */
static inline void tri_vertices(const orc_scene *s, const uint32_t *rec, v3 *p0, v3 *p1, v3 *p2) {
    uint32_t i0 = rec[0] + (rec[1] & 0xFFFFu);
    uint32_t i1 = rec[0] + ((rec[1] & 0xFFFF0000u) >> 16);
    uint32_t i2 = rec[0] + (rec[2] & 0xFFFFu);
    *p0 = ld3(s->pos + 3u * i0);
    *p1 = ld3(s->pos + 3u * i1);
    *p2 = ld3(s->pos + 3u * i2);
}

/* bvhGetter.glsl:27-42 bvh_getNodeBoxes. */
static inline void node_boxes(const packed_node *n, box_t *b0, box_t *b1) {
    b0->mn = mk(n->n0xy[0], n->n0xy[1], n->nz[0]);
    b0->mx = mk(n->n0xy[2], n->n0xy[3], n->nz[1]);
    b1->mn = mk(n->n1xy[0], n->n1xy[1], n->nz[2]);
    b1->mx = mk(n->n1xy[2], n->n1xy[3], n->nz[3]);
}

typedef struct {
    float t;
    uint32_t tri[3];
    uint32_t nid;
    float u, v;
    int hit;
} closest_t;

/* bvhCollision.glsl:177-239 bvh_collide (INLINE_TRIANGLE). */
static inline void bvh_collide(const orc_scene *s, uint32_t nid, const ray_t *r, closest_t *c, orc_stats *st) {
    nid &= NID_MASK;
    uint32_t off = node_at(s, nid)->nid[3];
    uint32_t hdr = leaf_header(s, off);
    uint32_t ntri = hdr & ((1u << TRIANGLE_BITS) - 1u);
    st->leaf_visit++;
    const uint32_t *ld = leaf_data(s);
    for (uint32_t i = 0; i < ntri; ++i) {
        const uint32_t *rec = ld + 1u + off + i * 3u;
        v3 p0, p1, p2;
        tri_vertices(s, rec, &p0, &p1, &p2);
        float u = 0.f, v = 0.f;
        st->tri_test++;
        float t = collide_triangle(r, p0, p1, p2, c->t, &u, &v);
        if (t > 0.0f) {
            c->t = t - OFFSET_RAY_COLLISION;
            c->tri[0] = rec[0]; c->tri[1] = rec[1]; c->tri[2] = rec[2];
            c->nid = nid;
            c->u = u; c->v = v;
            c->hit = 1;
        }
    }
}

static inline int point_in_box(box_t b, v3 p) { /* collision.glsl:17-21 */
    return p.x > b.mn.x && p.y > b.mn.y && p.z > b.mn.z && p.x < b.mx.x && p.y < b.mx.y && p.z < b.mx.z;
}

/* bvhCollision.glsl:241-284 bvh_collide_fast. */
static inline int bvh_collide_fast(const orc_scene *s, uint32_t nid, const ray_t *r, float tmax, orc_stats *st) {
    nid &= NID_MASK;
    uint32_t off = node_at(s, nid)->nid[3];
    uint32_t hdr = leaf_header(s, off);
    uint32_t ntri = hdr & ((1u << TRIANGLE_BITS) - 1u);
    uint32_t nblas = (hdr >> TRIANGLE_BITS) & ((1u << BLAS_BITS) - 1u);
    st->leaf_visit++;
    const uint32_t *ld = leaf_data(s);
    for (uint32_t i = 0; i < ntri; ++i) {
        const uint32_t *rec = ld + 1u + off + i * 3u;
        v3 p0, p1, p2;
        tri_vertices(s, rec, &p0, &p1, &p2);
        float u, v;
        st->tri_test++;
        if (collide_triangle(r, p0, p1, p2, tmax, &u, &v) > 0.0f) return 1;
    }
    for (uint32_t i = 0; i < nblas; ++i) {
        uint32_t bi = ld[1u + off + ntri * 3u + i];
        const blas_header *bh = blas_at(s, bi);
        box_t b; b.mn = ld3(bh->mn); b.mx = ld3(bh->mx);
        if (!point_in_box(b, r->from)) {
            if (collide_box(r, b, tmax) > 0.0f) return 1;
        }
    }
    return 0;
}

static inline uint32_t root_id(const orc_scene *s) {   /* baseRaytracingPass.glsl:20 */
    return s->num_nodes == 1u ? NID_LEAF_BIT : 0u;
}

/* bvhTraversal_inline.glsl:5-78 traverseBvh (closest hit, bitstack + parent/sibling links). */
static void traverse_closest(const orc_scene *s, const ray_t *r, closest_t *c, orc_stats *st) {
    uint32_t nodeId = root_id(s);
    uint32_t bitstack = 0, parentId = 0, siblingId = 0;
    for (;;) {
        while (!(nodeId & NID_LEAF_BIT)) {
            const packed_node *n = node_at(s, nodeId);
            st->node_fetch++;
            uint32_t packed = n->nid[2];
            uint32_t c0 = packed & NID_MASK, c1 = c0 + 1u;
            c0 |= (packed & NID_LEFT_LEAF_BIT) ? NID_LEAF_BIT : 0u;
            c1 |= (packed & NID_RIGHT_LEAF_BIT) ? NID_LEAF_BIT : 0u;
            box_t b0, b1;
            node_boxes(n, &b0, &b1);
            float d0 = collide_box(r, b0, c->t);
            float d1 = collide_box(r, b1, c->t);
            if (d0 < 0.0f && d1 < 0.0f) break;
            bitstack <<= 1;
            if (d0 >= 0.0f && d1 >= 0.0f) {
                nodeId = (d1 < d0) ? c1 : c0;
                bitstack |= 1u;
            } else {
                nodeId = (d0 >= 0.0f) ? c0 : c1;
            }
        }
        if (nodeId & NID_LEAF_BIT) bvh_collide(s, nodeId, r, c, st);
        {
            const packed_node *n = node_at(s, nodeId & NID_MASK);
            st->backtrack_reload++;
            parentId = n->nid[0]; siblingId = n->nid[1];
        }
        while ((bitstack & 1u) == 0u) {
            if (bitstack == 0u) return;
            nodeId = parentId;
            const packed_node *n = node_at(s, nodeId & NID_MASK);
            st->backtrack_reload++;
            parentId = n->nid[0]; siblingId = n->nid[1];
            bitstack >>= 1;
        }
        nodeId = siblingId;
        bitstack ^= 1u;
    }
}

/* bvhTraversal_inline.glsl:83-151 traverseBvhFast (any hit). */
static int traverse_any(const orc_scene *s, const ray_t *r, float tmax, orc_stats *st) {
    uint32_t nodeId = root_id(s);
    uint32_t bitstack = 0, parentId = 0, siblingId = 0;
    for (;;) {
        while (!(nodeId & NID_LEAF_BIT)) {
            const packed_node *n = node_at(s, nodeId);
            st->node_fetch++;
            uint32_t packed = n->nid[2];
            uint32_t c0 = packed & NID_MASK, c1 = c0 + 1u;
            c0 |= (packed & NID_LEFT_LEAF_BIT) ? NID_LEAF_BIT : 0u;
            c1 |= (packed & NID_RIGHT_LEAF_BIT) ? NID_LEAF_BIT : 0u;
            box_t b0, b1;
            node_boxes(n, &b0, &b1);
            float d0 = collide_box(r, b0, tmax);
            float d1 = collide_box(r, b1, tmax);
            if (d0 < 0.0f && d1 < 0.0f) break;
            bitstack <<= 1;
            if (d0 >= 0.0f && d1 >= 0.0f) {
                nodeId = (d1 < d0) ? c1 : c0;
                bitstack |= 1u;
            } else {
                nodeId = (d0 >= 0.0f) ? c0 : c1;
            }
        }
        if (nodeId & NID_LEAF_BIT) {
            if (bvh_collide_fast(s, nodeId, r, tmax, st)) return 1;
        }
        {
            const packed_node *n = node_at(s, nodeId & NID_MASK);
            st->backtrack_reload++;
            parentId = n->nid[0]; siblingId = n->nid[1];
        }
        while ((bitstack & 1u) == 0u) {
            if (bitstack == 0u) return 0;
            nodeId = parentId;
            const packed_node *n = node_at(s, nodeId & NID_MASK);
            st->backtrack_reload++;
            parentId = n->nid[0]; siblingId = n->nid[1];
            bitstack >>= 1;
        }
        nodeId = siblingId;
        bitstack ^= 1u;
    }
}

/* The two-level any-hit walk of USE_TRAVERSE_TLAS scenes:
 * bvhTraversal_inline.glsl:83-151 compiled as traverseTlasFast (the same walk over
 * the top-level nodes from the scene root) whose leaves call tlas_collide_fast
 * (bvhCollision.glsl:321-348): only the leaf's BLAS instances are tested (its
 * triangle records are skipped, and instances the builder lifted into inner
 * nodes' lists are never looked at), each with CollideBox(..., tmax) > 0 -- so an
 * origin inside the instance box (tmin = 0) skips it -- and on a pass the
 * one-level any-hit walk traverseBvhFast from the instance's rootIndex (a node
 * id without the leaf bit). */
static int walk_any_from(const orc_scene *s, uint32_t root, const ray_t *r, float tmax, int tlas, orc_stats *st);

static int tlas_collide_fast(const orc_scene *s, uint32_t nid, const ray_t *r, float tmax, orc_stats *st) {
    nid &= NID_MASK;
    uint32_t off = node_at(s, nid)->nid[3];
    if (off == 0xFFFFFFFFu) return 0;
    uint32_t hdr = leaf_header(s, off);
    uint32_t ntri = hdr & ((1u << TRIANGLE_BITS) - 1u);
    uint32_t nblas = (hdr >> TRIANGLE_BITS) & ((1u << BLAS_BITS) - 1u);
    st->leaf_visit++;
    const uint32_t *ld = leaf_data(s);
    for (uint32_t i = 0; i < nblas; ++i) {
        uint32_t bi = ld[1u + off + ntri * 3u + i];
        const blas_header *bh = blas_at(s, bi);
        box_t b; b.mn = ld3(bh->mn); b.mx = ld3(bh->mx);
        if (collide_box(r, b, tmax) > 0.0f) {
            if (bh->rootIndex >= s->num_nodes) continue;   /* not produced by the reference builder */
            if (walk_any_from(s, bh->rootIndex, r, tmax, 0, st)) return 1;
        }
    }
    return 0;
}

/* traverseBvhFast / traverseTlasFast from `root` (bvhTraversal_inline.glsl:83-151). */
static int walk_any_from(const orc_scene *s, uint32_t root, const ray_t *r, float tmax, int tlas, orc_stats *st) {
    uint32_t nodeId = root;
    uint32_t bitstack = 0, parentId = 0, siblingId = 0;
    for (;;) {
        while (!(nodeId & NID_LEAF_BIT)) {
            const packed_node *n = node_at(s, nodeId);
            st->node_fetch++;
            uint32_t packed = n->nid[2];
            uint32_t c0 = packed & NID_MASK, c1 = c0 + 1u;
            c0 |= (packed & NID_LEFT_LEAF_BIT) ? NID_LEAF_BIT : 0u;
            c1 |= (packed & NID_RIGHT_LEAF_BIT) ? NID_LEAF_BIT : 0u;
            box_t b0, b1;
            node_boxes(n, &b0, &b1);
            float d0 = collide_box(r, b0, tmax);
            float d1 = collide_box(r, b1, tmax);
            if (d0 < 0.0f && d1 < 0.0f) break;
            bitstack <<= 1;
            if (d0 >= 0.0f && d1 >= 0.0f) {
                nodeId = (d1 < d0) ? c1 : c0;
                bitstack |= 1u;
            } else {
                nodeId = (d0 >= 0.0f) ? c0 : c1;
            }
        }
        if (nodeId & NID_LEAF_BIT) {
            if (tlas ? tlas_collide_fast(s, nodeId, r, tmax, st) : bvh_collide_fast(s, nodeId, r, tmax, st)) return 1;
        }
        {
            const packed_node *n = node_at(s, nodeId & NID_MASK);
            st->backtrack_reload++;
            parentId = n->nid[0]; siblingId = n->nid[1];
        }
        while ((bitstack & 1u) == 0u) {
            if (bitstack == 0u) return 0;
            nodeId = parentId;
            const packed_node *n = node_at(s, nodeId & NID_MASK);
            st->backtrack_reload++;
            parentId = n->nid[0]; siblingId = n->nid[1];
            bitstack >>= 1;
        }
        nodeId = siblingId;
        bitstack ^= 1u;
    }
}

/* baseRaytracingPass.glsl:16-27 rayTrace, with the ray's own tmax as the start t
 * (the reference always starts at TMAX = 100). */
static inline void ray_trace(const orc_scene *s, const ray_t *r, float tmax, closest_t *c, orc_stats *st) {
    c->t = tmax; c->tri[0] = c->tri[1] = c->tri[2] = 0; c->nid = 0xFFFFFFFFu; c->u = c->v = 0.f; c->hit = 0;
    traverse_closest(s, r, c, st);
}

static int nthreads(int threads) {
#ifdef _OPENMP
    return threads > 0 ? threads : omp_get_max_threads();
#else
    (void)threads; return 1;
#endif
}

void orc_trace(const orc_scene *s, const orc_ray *rays, uint64_t n, uint32_t mode,
               uint32_t *hit, uint32_t *nid, float *bary, orc_stats *stats, int threads) {
    int nt = nthreads(threads);
    (void)nt;
    int64_t nn = (int64_t)n;
    const int tlas = (mode & ORC_MODE_TLAS) != 0u;
    const uint32_t m = mode & ~ORC_MODE_TLAS;
#pragma omp parallel for schedule(dynamic, 256) num_threads(nt)
    for (int64_t i = 0; i < nn; ++i) {
        const orc_ray *rr = rays + i;
        ray_t r; r.from = ld3(rr->o); r.dir = ld3(rr->d);
        orc_stats st = {0, 0, 0, 0};
        int any = (m == ORC_MODE_ANY) || (m == ORC_MODE_PER_RAY && (rr->flags & 1u));
        if (any) {
            int occ = tlas ? walk_any_from(s, root_id(s), &r, rr->tmax, 1, &st) : traverse_any(s, &r, rr->tmax, &st);
            hit[4 * i + 0] = (uint32_t)occ; hit[4 * i + 1] = 0; hit[4 * i + 2] = 0; hit[4 * i + 3] = fbits(rr->tmax);
            if (nid) nid[i] = 0xFFFFFFFFu;
            if (bary) { bary[2 * i] = 0.f; bary[2 * i + 1] = 0.f; }
        } else {
            closest_t c;
            ray_trace(s, &r, rr->tmax, &c, &st);
            hit[4 * i + 0] = c.tri[0]; hit[4 * i + 1] = c.tri[1]; hit[4 * i + 2] = c.tri[2]; hit[4 * i + 3] = fbits(c.t);
            if (nid) nid[i] = c.nid;
            if (bary) { bary[2 * i] = c.u; bary[2 * i + 1] = c.v; }
        }
        if (stats) stats[i] = st;
    }
}

/* ------------------------------------------------------------ light-probe helpers */
/* lightprobHelpers.glsl:10-14 computeLpfStep */
static inline v3 lpf_step(const float mn[3], const float mx[3], const uint32_t res[3]) {
    v3 dim = sub(ld3(mx), ld3(mn));
    return mk(dim.x / (float)res[0], dim.y / (float)res[1], dim.z / (float)res[2]);
}
/* lightprobHelpers.glsl:63-69 getLightProbPosition */
static inline v3 lpf_position(const uint32_t c[3], const uint32_t res[3], const float mn[3], const float mx[3]) {
    v3 step = lpf_step(mn, mx, res);
    v3 k = mk((float)c[0] + 0.5f, (float)c[1] + 0.5f, (float)c[2] + 0.5f);
    return add(ld3(mn), mul(step, k));
}
/* lightprobHelpers.glsl:33-61 getLightProbCoord (LP_TILE_RES = 4) */
void orc_probe_coord(uint32_t index, const uint32_t res[3], uint32_t coord[3]) {
    uint32_t trx = res[0] / 4u, try_ = res[1] / 4u;
    uint32_t tile = index / 64u, in = index % 64u;
    uint32_t z = tile / (trx * try_);
    tile = tile % (trx * try_);
    uint32_t y = tile / trx, x = tile % trx;
    coord[0] = x * 4u + in % 4u;
    coord[1] = y * 4u + (in / 4u) % 4u;
    coord[2] = z * 4u + (in / 16u) % 4u;
}

/* ------------------------------------------------------------ shadows and masks */
/* bvhLighting.glsl:100-108 traverseForShadow */
static inline int trace_shadow(const orc_scene *s, v3 pos, v3 dir, float len, orc_stats *st) {
    ray_t r; r.from = pos; r.dir = dir;
    return traverse_any(s, &r, len, st);
}

/* bvhLighting.glsl:110-131 evalShadow. *traced is set when a ray was cast. */
static inline int eval_shadow(const orc_scene *s, uint32_t li, v3 pos, orc_stats *st, uint64_t *traced) {
    if (li >= s->num_lights && s->num_lights != 0xFFFFFFFFu) {
        /* out-of-range light ids are not produced by the builders; treat as "no shadow info" */
    }
    const packed_light *L = light_at(s, li);
    if (L->iparam != LIGHT_SPHERE) return 0;
    v3 lp = mk(L->fparam[0], L->fparam[1], L->fparam[2]);
    float radius = L->fparam[3];
    v3 dir = sub(lp, pos);
    float len = length3(dir);
    if (len < radius) {
        (*traced)++;
        return trace_shadow(s, pos, divs(dir, len), len, st);
    }
    return 1;
}

static inline uint32_t light_bit(uint32_t li) { return (li + 1u) < 32u ? (1u << (li + 1u)) : 0u; }

/* bvhLighting.glsl:143-163 computeShadowMask (leaf light list of the hit node). */
static uint32_t shadow_mask_leaf(const orc_scene *s, v3 pos, uint32_t hit_nid, v3 sunDir, orc_stats *st, uint64_t *traced) {
    uint32_t mask = 0;
    (*traced)++;
    mask |= trace_shadow(s, pos, neg(sunDir), TMAX, st) ? 1u : 0u;
    uint32_t off = node_at(s, hit_nid)->nid[3];
    uint32_t hdr = leaf_header(s, off);
    /* bvhLighting.glsl:133-141 unpackLightCountAndOffset (NodeTriangleStride = 3) */
    uint32_t skip = 3u * (hdr & ((1u << TRIANGLE_BITS) - 1u));
    skip += (hdr >> TRIANGLE_BITS) & ((1u << BLAS_BITS) - 1u);
    skip += (hdr >> (TRIANGLE_BITS + BLAS_BITS)) & ((1u << PRIM_BITS) - 1u);
    uint32_t nl = (hdr >> (TRIANGLE_BITS + BLAS_BITS + PRIM_BITS)) & ((1u << LIGHT_BITS) - 1u);
    uint32_t base = skip + 1u + off;
    const uint32_t *ld = leaf_data(s);
    for (uint32_t i = 0; i < nl; ++i) {
        uint32_t li = ld[base + i];
        if (li + 1u >= 32u) continue;   /* the 32-bit mask has no bit for this light */
        mask |= eval_shadow(s, li, pos, st, traced) ? light_bit(li) : 0u;
    }
    return mask;
}

/* Same shadow semantics, with the light list taken from the tile culling output. */
static uint32_t shadow_mask_tile(const orc_scene *s, v3 pos, const uint32_t *list, uint32_t count, v3 sunDir,
                                 orc_stats *st, uint64_t *traced) {
    uint32_t mask = 0;
    (*traced)++;
    mask |= trace_shadow(s, pos, neg(sunDir), TMAX, st) ? 1u : 0u;
    for (uint32_t i = 0; i < count; ++i) {
        uint32_t li = list[i];
        if (li + 1u >= 32u) continue;   /* the 32-bit mask has no bit for this light */
        mask |= eval_shadow(s, li, pos, st, traced) ? light_bit(li) : 0u;
    }
    return mask;
}

/* bvhLighting.glsl:165-184 computeProbMask (USE_LPF_MASK) with lightprobHelpers.glsl:71-77. */
static uint32_t prob_mask(const orc_scene *s, v3 pos, const orc_pass_data *pd, orc_stats *st, uint64_t *traced) {
    const uint32_t *res = pd->lpfResolution;
    v3 step = lpf_step(pd->sceneMinExtent, pd->sceneMaxExtent, res);
    v3 uvw = sub(mk((pos.x - pd->sceneMinExtent[0]) / step.x, (pos.y - pd->sceneMinExtent[1]) / step.y,
                    (pos.z - pd->sceneMinExtent[2]) / step.z), mk(0.5f, 0.5f, 0.5f));
    uvw = mk(fminf(fmaxf(uvw.x, 0.0f), (float)res[0] - 1.0f), fminf(fmaxf(uvw.y, 0.0f), (float)res[1] - 1.0f),
             fminf(fmaxf(uvw.z, 0.0f), (float)res[2] - 1.0f));
    uint32_t c[3];
    uint32_t ix = (uint32_t)(int32_t)uvw.x, iy = (uint32_t)(int32_t)uvw.y, iz = (uint32_t)(int32_t)uvw.z;
    c[0] = ix < res[0] - 2u ? ix : res[0] - 2u;
    c[1] = iy < res[1] - 2u ? iy : res[1] - 2u;
    c[2] = iz < res[2] - 2u ? iz : res[2] - 2u;
    uint32_t mask = 0;
    for (uint32_t i = 0; i < 8u; ++i) {
        uint32_t cc[3] = {c[0] + (i & 1u), c[1] + ((i >> 1) & 1u), c[2] + ((i >> 2) & 1u)};
        v3 pp = lpf_position(cc, res, pd->sceneMinExtent, pd->sceneMaxExtent);
        (*traced)++;
        mask |= (trace_shadow(s, pos, sub(pp, pos), 1.0f, st) ? 1u : 0u) << i;
    }
    return mask;
}

/* ------------------------------------------------------------ diffuse bounce */
/* Integer hash (Wellons' "lowbias32" finaliser). */
uint32_t orc_hash32(uint32_t x) {
    x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
    return x;
}
static inline float u01(uint32_t h) { return (float)(h >> 8) * (1.0f / 16777216.0f); }

/* Cosine-weighted hemisphere direction around unit normal n: a point drawn
 * uniformly in the unit disk by rejection (Malley's method) lifted to the
 * hemisphere, in the orthonormal basis of Duff et al., "Building an Orthonormal
 * Basis, Revisited" (JCGT 2017). Only + - * / sqrt, so CUDA and C agree bitwise. */
void orc_bounce_dir(const float nn[3], uint32_t pixel, uint32_t seed, float out[3]) {
    v3 n = ld3(nn);
    float x = 0.f, y = 0.f;
    for (uint32_t k = 0; k < 16u; ++k) {
        uint32_t h0 = orc_hash32(pixel * 2u + 0x9E3779B9u * (seed + 1u) + k * 0x85EBCA6Bu);
        uint32_t h1 = orc_hash32(h0 ^ 0x27D4EB2Fu);
        float a = u01(h0) * 2.0f - 1.0f, b = u01(h1) * 2.0f - 1.0f;
        if (a * a + b * b < 1.0f) { x = a; y = b; break; }
    }
    float z = sqrtf(fmaxf(0.0f, 1.0f - x * x - y * y));
    float sign = copysignf(1.0f, n.z);
    float a = -1.0f / (sign + n.z);
    float b = n.x * n.y * a;
    v3 b1 = mk(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
    v3 b2 = mk(b, sign + n.y * n.y * a, -n.y);
    v3 d = add(add(muls(b1, x), muls(b2, y)), muls(n, z));
    out[0] = d.x; out[1] = d.y; out[2] = d.z;
}

/* Geometric normal of the hit triangle, facing the incoming ray. */
static inline v3 face_normal(const orc_scene *s, const uint32_t *rec, v3 dir) {
    v3 p0, p1, p2;
    tri_vertices(s, rec, &p0, &p1, &p2);
    v3 n = normalize3(cross3(sub(p1, p0), sub(p2, p0)));
    if (dot3(n, dir) > 0.0f) n = neg(n);
    return n;
}

/* ------------------------------------------------------------ camera pass */
/* cameraPass.comp:44-76 (TRACING_STEP). The output is iterated per output pixel:
 * pixel (px, py) is produced by invocation (gx = px, gy = 16*ceil(H/16) - py)
 * (cameraPass.comp:46), so row py = 0 is never traced and is written as zeros. */
void orc_camera(const orc_scene *s, const orc_pass_data *pd, uint32_t flags, uint32_t seed,
                const uint32_t *tile_counts, const uint32_t *tile_lists,
                uint32_t *out, uint32_t *bounce_out, uint64_t *ray_counts,
                uint64_t pix_begin, uint64_t pix_end, int threads) {
    const uint32_t W = pd->frameSize[0], H = pd->frameSize[1];
    const uint32_t ngy = (H + 15u) / 16u, tiles_x = (W + 15u) / 16u;
    v3 c00 = ld3(pd->frustumCorner00), c10 = ld3(pd->frustumCorner10), c01 = ld3(pd->frustumCorner01);
    v3 cam = ld3(pd->cameraPos), sun = ld3(pd->sunDir);
    v3 stepW = muls(sub(c10, c00), pd->invFrameSize[0]);
    v3 stepH = muls(sub(c01, c00), pd->invFrameSize[1]);
    if (pix_end > (uint64_t)W * H) pix_end = (uint64_t)W * H;
    uint64_t cnt_primary = 0, cnt_shadow = 0, cnt_probe = 0, cnt_bounce = 0;
    int nt = nthreads(threads);
    (void)nt;
    int64_t b = (int64_t)pix_begin, e = (int64_t)pix_end;
#pragma omp parallel for schedule(dynamic, 256) num_threads(nt) reduction(+ : cnt_primary, cnt_shadow, cnt_probe, cnt_bounce)
    for (int64_t pix = b; pix < e; ++pix) {
        uint32_t px = (uint32_t)(pix % W), py = (uint32_t)(pix / W);
        uint32_t *o = out + 8u * (uint64_t)pix;
        uint32_t *bo = bounce_out ? bounce_out + 4u * (uint64_t)pix : 0;
        memset(o, 0, 32);
        if (bo) memset(bo, 0, 16);
        if (py == 0u) continue;
        uint32_t gx = px, gy = ngy * 16u - py;
        v3 target = add(add(c00, muls(stepW, (float)gx)), muls(stepH, (float)gy));
        ray_t r; r.from = cam; r.dir = normalize3(sub(target, cam));
        orc_stats st = {0, 0, 0, 0};
        closest_t c;
        ray_trace(s, &r, TMAX, &c, &st);
        cnt_primary++;
        o[0] = c.tri[0]; o[1] = c.tri[1]; o[2] = c.tri[2]; o[3] = fbits(c.t);
        /* baseRaytracingPass.glsl:85-97 computeAdditionalHitData */
        if (c.t < TMAX) {
            v3 hp = add(r.from, muls(r.dir, c.t));
            uint64_t sh = 0, pr = 0;
            if (flags & ORC_CAM_TILE_LIGHTS) {
                uint32_t tile = (gy / 16u) * tiles_x + gx / 16u;
                o[4] = shadow_mask_tile(s, hp, tile_lists + 16u * tile, tile_counts[tile], sun, &st, &sh);
            } else {
                o[4] = shadow_mask_leaf(s, hp, c.nid, sun, &st, &sh);
            }
            if (flags & ORC_CAM_PROB_MASK) o[5] = prob_mask(s, hp, pd, &st, &pr);
            cnt_shadow += sh; cnt_probe += pr;
            if ((flags & ORC_CAM_BOUNCE) && bo) {
                v3 n = face_normal(s, c.tri, r.dir);
                float nn[3] = {n.x, n.y, n.z}, d[3];
                orc_bounce_dir(nn, (uint32_t)pix, seed, d);
                ray_t br; br.from = hp; br.dir = ld3(d);
                closest_t bc;
                ray_trace(s, &br, TMAX, &bc, &st);
                cnt_bounce++;
                bo[0] = bc.tri[0]; bo[1] = bc.tri[1]; bo[2] = bc.tri[2]; bo[3] = fbits(bc.t);
            }
        }
    }
    if (ray_counts) {
        ray_counts[0] += cnt_primary; ray_counts[1] += cnt_shadow;
        ray_counts[2] += cnt_probe; ray_counts[3] += cnt_bounce;
    }
}

/* ------------------------------------------------------------ tile light culling */
/* cullFrustum.glsl:9-13 computePlan */
static inline void compute_plan(v3 p1, v3 p2, v3 p3, float out[4]) {
    v3 n = normalize3(cross3(sub(p1, p2), sub(p3, p2)));
    out[0] = n.x; out[1] = n.y; out[2] = n.z; out[3] = -dot3(n, p2);
}

/* cullFrustum.glsl:63-100 (tile corners and planes) and 136-151 (light loop),
 * collision.glsl:219-227 sphereFrustum4Collision. */
void orc_cull_lights(const orc_scene *s, const orc_pass_data *pd, uint32_t tiles_x, uint32_t tiles_y,
                     uint32_t *counts, uint32_t *lists, int threads) {
    v3 c00 = ld3(pd->frustumCorner00), c10 = ld3(pd->frustumCorner10), c01 = ld3(pd->frustumCorner01);
    v3 cam = ld3(pd->cameraPos);
    v3 step_x = divs(sub(c10, c00), (float)tiles_x);
    v3 step_y = divs(sub(c01, c00), (float)tiles_y);
    int nt = nthreads(threads);
    (void)nt;
    int64_t ntiles = (int64_t)tiles_x * tiles_y;
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int64_t t = 0; t < ntiles; ++t) {
        uint32_t wx = (uint32_t)(t % tiles_x), wy = (uint32_t)(t / tiles_x);
        v3 bl = add(add(c00, muls(step_x, (float)wx)), muls(step_y, (float)wy));
        v3 br = add(add(c00, muls(step_x, (float)(wx + 1u))), muls(step_y, (float)wy));
        v3 tl = add(add(c00, muls(step_x, (float)wx)), muls(step_y, (float)(wy + 1u)));
        v3 tr = add(add(c00, muls(step_x, (float)(wx + 1u))), muls(step_y, (float)(wy + 1u)));
        v3 dx = muls(step_x, 0.25f), dy = muls(step_y, 0.25f);
        bl = sub(sub(bl, dx), dy);
        br = sub(add(br, dx), dy);
        tl = add(sub(tl, dx), dy);
        tr = add(add(tr, dx), dy);
        float pl[4][4];
        compute_plan(cam, tl, bl, pl[0]);
        compute_plan(cam, br, tr, pl[1]);
        compute_plan(cam, tr, tl, pl[2]);
        compute_plan(cam, bl, br, pl[3]);
        uint32_t cnt = 0;
        uint32_t *lst = lists + 16u * (uint64_t)t;
        for (uint32_t i = 0; i < s->num_lights && cnt < 16u; ++i) {
            const packed_light *L = light_at(s, i);
            v3 c = mk(L->fparam[0], L->fparam[1], L->fparam[2]);
            float r = L->fparam[3];
            int inside = 1;
            for (int k = 0; k < 4; ++k) {
                if (dot3(mk(pl[k][0], pl[k][1], pl[k][2]), c) + pl[k][3] < -r) { inside = 0; break; }
            }
            if (inside) lst[cnt++] = i;
        }
        for (uint32_t k = cnt; k < 16u; ++k) lst[k] = 0xFFFFFFFFu;
        counts[t] = cnt;
    }
}

/* ------------------------------------------------------------ probe field */
/* core/lighting.glsl:16-20 computeAttenuation */
static inline float attenuation(float dist, float radius) {
    float att = (radius * radius + 1.0f) / (255.0f * dist * dist);
    return clampf(att - (1.0f / 255.0f), 0.0f, 1.0f);
}

/* core/lighting.glsl:22-57 computeLighting (texColor = 1; COMPUTE_SHADOW_ON_THE_FLY = 0). */
static v3 compute_lighting(const material *m, v3 lightColor, v3 P, v3 L, v3 N, v3 E, float att) {
    if (m->type_ids[0] == MAT_EMISSIVE) return ld3(m->color);
    if (m->type_ids[0] == MAT_TRANSPARENT) return mk(0, 0, 0);
    v3 lit = mk(0, 0, 0);
    float dotL = clampf(dot3(N, L), 0.0f, 1.0f);
    if (m->type_ids[0] == MAT_PBR) {
        /* core/lighting.glsl:137-182 computePbrLighting */
        v3 albedo = ld3(m->color);
        float metal = m->params[0];
        v3 v = normalize3(sub(E, P));
        v3 h = normalize3(add(v, L));
        float NoV = fabsf(dot3(N, v)) + 1e-5f;
        float NoL = clampf(dot3(N, L), 0.0f, 1.0f);
        float NoH = clampf(dot3(N, h), 0.0f, 1.0f);
        float LoH = clampf(dot3(L, h), 0.0f, 1.0f);
        float rough = 0.02f * 0.02f;
        float a2 = rough * rough;
        float f = (NoH * a2 - NoH) * NoH + 1.0f;
        float D = a2 / (3.141592f * f * f);
        v3 f0 = add(muls(mk(0.04f, 0.04f, 0.04f), 1.0f - metal), muls(albedo, metal));
        float p5 = powf(1.0f - LoH, 5.0f);
        v3 F = add(f0, muls(sub(mk(1, 1, 1), f0), p5));
        float GGXL = NoV * sqrtf((-NoL * a2 + NoL) * NoL + a2);
        float GGXV = NoL * sqrtf((-NoV * a2 + NoV) * NoV + a2);
        float V = 0.5f / (GGXV + GGXL);
        v3 Fr = muls(F, D * V);
        v3 Fd = divs(muls(albedo, 1.0f - metal), 3.141592f);
        lit = muls(mul(add(Fd, Fr), lightColor), NoL);
    } else if (m->type_ids[0] == MAT_LAMBERT) {
        lit = mul(muls(lightColor, dotL), ld3(m->color));
    }
    return muls(lit, att);
}

/* baseRaytracingPass.glsl:38-64 fillUvNormal (normal only). */
static v3 interp_normal(const orc_scene *s, const uint32_t *rec, v3 pos) {
    uint32_t i0 = rec[0] + (rec[1] & 0xFFFFu);
    uint32_t i1 = rec[0] + ((rec[1] & 0xFFFF0000u) >> 16);
    uint32_t i2 = rec[0] + (rec[2] & 0xFFFFu);
    v3 p0 = ld3(s->pos + 3u * i0), p1 = ld3(s->pos + 3u * i1), p2 = ld3(s->pos + 3u * i2);
    v3 v0 = sub(p1, p0), v1 = sub(p2, p0), v2 = sub(pos, p0);
    float d00 = dot3(v0, v0), d01 = dot3(v0, v1), d11 = dot3(v1, v1);
    float d20 = dot3(v2, v0), d21 = dot3(v2, v1);
    float denom = d00 * d11 - d01 * d01;
    float v = (d11 * d20 - d01 * d21) / denom;
    float w = (d00 * d21 - d01 * d20) / denom;
    float u = 1.0f - v - w;
    v3 n0 = ld3(s->nrm + 3u * i0), n1 = ld3(s->nrm + 3u * i1), n2 = ld3(s->nrm + 3u * i2);
    return add(add(muls(n0, u), muls(n1, v)), muls(n2, w));
}

/* bvhLighting.glsl:42-85 computeLighting, direct part: texColor 1 (untextured
 * materials), the lights whose mask bit is clear (evalLighting -> evalSphereLight;
 * a light out of range contributes 0, where lighting.glsl:92-101 falls off the end
 * of a non-void function), then the sun (evalSunLight), summed in that order. */
static v3 direct_lit(const orc_scene *s, const material *m, v3 pos, v3 N, v3 eye, uint32_t mask, v3 sunDir,
                     v3 sunColor) {
    v3 lit = mk(0, 0, 0);
    for (uint32_t i = 0; i < s->num_lights && i < 31u; ++i) {
        if ((mask & (1u << (i + 1u))) != 0u) continue;
        const packed_light *L = light_at(s, i);
        if (L->iparam != LIGHT_SPHERE) continue;
        v3 lp = mk(L->fparam[0], L->fparam[1], L->fparam[2]);
        float d = length3(sub(lp, pos));
        if (d < L->fparam[3]) {
            v3 Ld = divs(sub(lp, pos), d);
            d = fmaxf(0.01f, d - L->fparam[7]);
            lit = add(lit, compute_lighting(m, mk(L->fparam[4], L->fparam[5], L->fparam[6]), pos, Ld, N, eye,
                                            attenuation(d, L->fparam[3])));
        }
    }
    if ((mask & 1u) == 0u) lit = add(lit, compute_lighting(m, sunColor, pos, neg(sunDir), N, eye, 1.0f));
    return lit;
}

static inline v3 sky_colour(void) {   /* baseRaytracingPass.glsl:81: 0.3 * vec3(200,220,255) / 255 */
    return divs(muls(mk(200.0f, 220.0f, 255.0f), 0.3f), 255.0f);
}

/* bvhLighting.glsl:42-85 computeLighting with NO_LPF (genLightProbField.comp:5), and
 * baseRaytracingPass.glsl:67-82 for the miss colour. */
static v3 probe_lit(const orc_scene *s, const orc_probe_desc *pd, const ray_t *r, float t, const uint32_t *rec, uint32_t mask) {
    if (!(t < TMAX)) return sky_colour();
    v3 pos = add(r->from, muls(r->dir, t));
    v3 N = interp_normal(s, rec, pos);
    const material *m = material_at(s, (rec[2] & 0xFFFF0000u) >> 16);
    return direct_lit(s, m, pos, N, r->from, mask, ld3(pd->sunDir), ld3(pd->sunColor));
}

/* genLightProbField.comp:41-81: trace step (closest hit + leaf-light shadow mask;
 * USE_LPF_MASK is not set there, so the probe mask is 0) followed by the lit value. */
void orc_probe_trace(const orc_scene *s, const orc_probe_desc *pd, const float *dirs,
                     uint32_t probe_begin, uint32_t probe_end,
                     uint32_t *trace_out, float *irradiance, uint64_t *ray_counts, int threads) {
    const uint32_t nd = pd->num_dirs;
    uint64_t cnt_primary = 0, cnt_shadow = 0;
    int nt = nthreads(threads);
    (void)nt;
    int64_t total = (int64_t)(probe_end - probe_begin) * nd;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nt) reduction(+ : cnt_primary, cnt_shadow)
    for (int64_t k = 0; k < total; ++k) {
        uint32_t p = probe_begin + (uint32_t)(k / nd), ri = (uint32_t)(k % nd);
        uint64_t sample = (uint64_t)(p - probe_begin) * nd + ri;
        uint32_t coord[3];
        orc_probe_coord(p, pd->resolution, coord);
        ray_t r;
        r.from = lpf_position(coord, pd->resolution, pd->aabbMin, pd->aabbMax);
        r.dir = ld3(dirs + 4u * ri);
        orc_stats st = {0, 0, 0, 0};
        closest_t c;
        ray_trace(s, &r, TMAX, &c, &st);
        cnt_primary++;
        uint32_t mask = 0;
        if (c.t < TMAX) {
            v3 hp = add(r.from, muls(r.dir, c.t));
            uint64_t sh = 0;
            mask = shadow_mask_leaf(s, hp, c.nid, ld3(pd->sunDir), &st, &sh);
            cnt_shadow += sh;
        }
        if (trace_out) {
            uint32_t *o = trace_out + 8u * sample;
            o[0] = c.tri[0]; o[1] = c.tri[1]; o[2] = c.tri[2]; o[3] = fbits(c.t);
            o[4] = mask; o[5] = 0; o[6] = 0; o[7] = 0;
        }
        if (irradiance) {
            v3 L = probe_lit(s, pd, &r, c.t, c.tri, mask);
            irradiance[3u * sample + 0] = L.x; irradiance[3u * sample + 1] = L.y; irradiance[3u * sample + 2] = L.z;
        }
    }
    if (ray_counts) { ray_counts[0] += cnt_primary; ray_counts[1] += cnt_shadow; }
}

/* updateLightProbField.comp:33-64: SH9 projection, normalisation by 4*pi/N and
 * GLSL mix(prev, new, hysteresis). out_sh / prev: 27 floats per probe (coef j, rgb). */
void orc_probe_sh9(const orc_probe_desc *pd, const float *sh_basis, const float *irradiance,
                   uint32_t probe_begin, uint32_t probe_end, const float *prev, float *out_sh) {
    const uint32_t nd = pd->num_dirs;
    const float norm = (4.0f * 3.14159265358979323846f) / (float)nd;
    const float a = pd->hysteresis;
    for (uint32_t p = probe_begin; p < probe_end; ++p) {
        uint64_t lp = p - probe_begin;
        float acc[9][3];
        memset(acc, 0, sizeof(acc));
        for (uint32_t i = 0; i < nd; ++i) {
            const float *L = irradiance + 3u * (lp * nd + i);
            for (uint32_t j = 0; j < 9u; ++j) {
                float w = sh_basis[i * 9u + j];
                acc[j][0] += L[0] * w; acc[j][1] += L[1] * w; acc[j][2] += L[2] * w;
            }
        }
        for (uint32_t j = 0; j < 9u; ++j)
            for (uint32_t c = 0; c < 3u; ++c) {
                float sh = acc[j][c] * norm;
                float pv = prev ? prev[27u * lp + 3u * j + c] : 0.0f;
                out_sh[27u * lp + 3u * j + c] = pv * (1.0f - a) + sh * a;
            }
    }
}

/* Octahedral 8x8 texels per probe: direction k of a side x side octahedral grid
 * (side = sqrt(num_dirs), k = j*side + i) is binned into texel (i*8/side, j*8/side);
 * each texel holds the mean radiance of its rays (FP32). */
void orc_probe_octa(const orc_probe_desc *pd, const float *irradiance,
                    uint32_t probe_begin, uint32_t probe_end, float *out_texels) {
    const uint32_t nd = pd->num_dirs;
    uint32_t side = 1;
    while (side * side < nd) side++;
    const uint32_t per = nd / 64u;
    for (uint32_t p = probe_begin; p < probe_end; ++p) {
        uint64_t lp = p - probe_begin;
        float *o = out_texels + 192u * lp;
        memset(o, 0, 192 * sizeof(float));
        for (uint32_t k = 0; k < nd; ++k) {
            uint32_t i = k % side, j = k / side;
            uint32_t tx = i * 8u / side, ty = j * 8u / side;
            const float *L = irradiance + 3u * (lp * nd + k);
            float *t = o + 3u * (ty * 8u + tx);
            t[0] += L[0]; t[1] += L[1]; t[2] += L[2];
        }
        float inv = 1.0f / (float)(per ? per : 1u);
        for (uint32_t q = 0; q < 192u; ++q) o[q] *= inv;
    }
}

/* ------------------------------------------------------------ camera lighting step */
static inline float half_to_float(uint16_t h) { _Float16 f; memcpy(&f, &h, 2); return (float)f; }
static inline uint16_t float_to_half(float x) { _Float16 f = (_Float16)x; uint16_t h; memcpy(&h, &f, 2); return h; }
static inline float mixf(float a, float b, float x) { return a * (1.0f - x) + b * x; }   /* GLSL mix */

/* fetchSH_inline.glsl:82-118 sampleSH9 with the probe mask, per image channel:
 * v[x + 2y + 4z] are the eight corner values, bit (x + 2y + 4z) of mask set =
 * corner masked. The same lerp tree as the shader, so the same rounding. */
static float masked_trilinear(const float v[8], v3 f, uint32_t mask) {
#define M(i) (((mask >> (i)) & 1u) == 0u)
    float shx0 = M(0) && M(1) ? mixf(v[0], v[1], f.x) : (M(0) ? v[0] : v[1]);
    float shx1 = M(2) && M(3) ? mixf(v[2], v[3], f.x) : (M(2) ? v[2] : v[3]);
    int b00 = M(0) || M(1), b10 = M(2) || M(3);
    float z0 = b00 && b10 ? mixf(shx0, shx1, f.y) : (b00 ? shx0 : shx1);
    shx0 = M(4) && M(5) ? mixf(v[4], v[5], f.x) : (M(4) ? v[4] : v[5]);
    shx1 = M(6) && M(7) ? mixf(v[6], v[7], f.x) : (M(6) ? v[6] : v[7]);
    int b01 = M(4) || M(5), b11 = M(6) || M(7);
    float z1 = b01 && b11 ? mixf(shx0, shx1, f.y) : (b01 ? shx0 : shx1);
    int bxy0 = b00 || b10, bxy1 = b01 || b11;
#undef M
    return bxy0 && bxy1 ? mixf(z0, z1, f.z) : (bxy0 ? z0 : z1);
}

/* bvhLighting.glsl:24-40 computeLPFLighting with USE_LPF_MASK: probe-grid uvw
 * (lightprobHelpers.glsl:71-77), masked SH9 sample from the 7 FP16 images
 * (fetchSH_inline.glsl:6-31 channel layout), evalSH (lightprobHelpers.glsl:90-101)
 * and computeIndirectLighting (core/lighting.glsl:59-74, texColor 1). */
static v3 lpf_lit(const orc_pass_data *pd, const uint16_t *sh16, const material *m, v3 pos, v3 N, uint32_t mask) {
    const uint32_t *res = pd->lpfResolution;
    v3 step = lpf_step(pd->sceneMinExtent, pd->sceneMaxExtent, res);
    v3 uvw = sub(mk((pos.x - pd->sceneMinExtent[0]) / step.x, (pos.y - pd->sceneMinExtent[1]) / step.y,
                    (pos.z - pd->sceneMinExtent[2]) / step.z), mk(0.5f, 0.5f, 0.5f));
    uvw = mk(fminf(fmaxf(uvw.x, 0.0f), (float)res[0] - 1.0f), fminf(fmaxf(uvw.y, 0.0f), (float)res[1] - 1.0f),
             fminf(fmaxf(uvw.z, 0.0f), (float)res[2] - 1.0f));
    /* min(int(uvw), res - 2) in GLSL's int -> uint conversion */
    uint32_t ix = (uint32_t)(int32_t)uvw.x, iy = (uint32_t)(int32_t)uvw.y, iz = (uint32_t)(int32_t)uvw.z;
    ix = ix < res[0] - 2u ? ix : res[0] - 2u;
    iy = iy < res[1] - 2u ? iy : res[1] - 2u;
    iz = iz < res[2] - 2u ? iz : res[2] - 2u;
    v3 f = sub(uvw, mk((float)(int32_t)ix, (float)(int32_t)iy, (float)(int32_t)iz));
    const uint64_t img = (uint64_t)res[0] * res[1] * res[2];
    float ch[7][4];
    for (int k = 0; k < 7; ++k)
        for (int c = 0; c < 4; ++c) {
            float v[8];
            for (int q = 0; q < 8; ++q) {
                uint64_t x = ix + (q & 1), y = iy + ((q >> 1) & 1), z = iz + ((q >> 2) & 1);
                v[q] = half_to_float(sh16[4u * (k * img + (z * res[1] + y) * res[0] + x) + c]);
            }
            ch[k][c] = masked_trilinear(v, f, mask);
        }
    float w[9][3];   /* SH9Color.w[j].rgb from the storeSH9 layout */
    for (int c = 0; c < 3; ++c) w[0][c] = ch[0][c];
    for (int j = 1; j <= 8; ++j)
        for (int c = 0; c < 3; ++c) w[j][c] = j <= 4 ? ch[1 + 2 * c][j - 1] : ch[2 + 2 * c][j - 5];
    const float c1 = 0.429043f, c2 = 0.511664f, c3 = 0.743125f, c4 = 0.886227f, c5 = 0.247708f;
    /* SH_Y00 0, Y11 1, Y10 2, Y1_1 3, Y21 4, Y2_1 5, Y2_2 6, Y20 7, Y22 8 (lightprob.glsl) */
    float L[3];
    for (int c = 0; c < 3; ++c) {
        float t1 = (c1 * (N.x * N.x - N.y * N.y)) * w[8][c];
        float t2 = ((c3 * w[7][c]) * N.z) * N.z;
        float t3 = c4 * w[0][c];
        float t4 = c5 * w[7][c];
        float t5 = (2.0f * c1) * (((w[6][c] * N.x) * N.y + (w[4][c] * N.x) * N.z) + (w[5][c] * N.y) * N.z);
        float t6 = (2.0f * c2) * ((w[1][c] * N.x + w[3][c] * N.y) + w[2][c] * N.z);
        L[c] = ((((t1 + t2) + t3) - t4) + t5) + t6;
    }
    const float pi = 3.14159265359f;   /* TIM_PI, core/math.glsl:4 */
    if (m->type_ids[0] == MAT_PBR) {
        float k = 1.0f - m->params[0];
        return mk(((k * m->color[0]) * L[0]) / pi, ((k * m->color[1]) * L[1]) / pi, ((k * m->color[2]) * L[2]) / pi);
    }
    if (m->type_ids[0] == MAT_LAMBERT)
        return mk((L[0] * m->color[0]) / pi, (L[1] * m->color[1]) / pi, (L[2] * m->color[2]) / pi);
    return mk(0, 0, 0);
}

/* cameraPass.comp:78-88, the lighting step (RayTracingPass::lightingPass,
 * raytracingPass.cpp:113-135: USE_LPF, USE_LPF_MASK): per pixel the tracing
 * record and masks -> computeLighting (baseRaytracingPass.glsl:67-82) -> RGBA16F. */
void orc_shade_camera(const orc_scene *s, const orc_pass_data *pd, uint32_t flags, const uint32_t *tracing,
                      const uint16_t *sh16, uint16_t *out_rgba16, float *out_rgb32, int threads) {
    const uint32_t W = pd->frameSize[0], H = pd->frameSize[1];
    const uint32_t ngy = (H + 15u) / 16u;
    v3 c00 = ld3(pd->frustumCorner00), c10 = ld3(pd->frustumCorner10), c01 = ld3(pd->frustumCorner01);
    v3 cam = ld3(pd->cameraPos);
    v3 stepW = muls(sub(c10, c00), pd->invFrameSize[0]);
    v3 stepH = muls(sub(c01, c00), pd->invFrameSize[1]);
    int nt = nthreads(threads);
    (void)nt;
    int64_t npix = (int64_t)W * H;
#pragma omp parallel for schedule(dynamic, 256) num_threads(nt)
    for (int64_t pix = 0; pix < npix; ++pix) {
        uint32_t px = (uint32_t)(pix % W), py = (uint32_t)(pix / W);
        uint16_t *o = out_rgba16 + 4u * (uint64_t)pix;
        float *of = out_rgb32 ? out_rgb32 + 3u * (uint64_t)pix : 0;
        memset(o, 0, 8);
        if (of) memset(of, 0, 12);
        if (py == 0u) continue;   /* the dispatch never reaches output row 0 */
        uint32_t gx = px, gy = ngy * 16u - py;
        v3 target = add(add(c00, muls(stepW, (float)gx)), muls(stepH, (float)gy));
        ray_t r; r.from = cam; r.dir = normalize3(sub(target, cam));
        const uint32_t *rec = tracing + 8u * (uint64_t)pix;
        float t;
        memcpy(&t, rec + 3, 4);
        v3 lit;
        if (!(t < TMAX)) {
            lit = sky_colour();
        } else {
            v3 pos = add(r.from, muls(r.dir, t));
            v3 N = interp_normal(s, rec, pos);
            const material *m = material_at(s, (rec[2] & 0xFFFF0000u) >> 16);
            lit = direct_lit(s, m, pos, N, r.from, rec[4], ld3(pd->sunDir), ld3(pd->sunColor));
            if (!(flags & ORC_SHADE_NO_LPF)) lit = add(lit, lpf_lit(pd, sh16, m, pos, N, rec[5]));
        }
        o[0] = float_to_half(lit.x); o[1] = float_to_half(lit.y); o[2] = float_to_half(lit.z);
        o[3] = float_to_half(1.0f);
        if (of) { of[0] = lit.x; of[1] = lit.y; of[2] = lit.z; }
    }
}
