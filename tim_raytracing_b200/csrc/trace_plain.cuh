// trace_plain.cuh -- traversal of the reference's binary BVH layout.
//
// The reference walks its binary BVH stacklessly: a 32-bit bitstack records,
// per level, whether the far child is still pending, and parent/sibling links
// bring it back up (bvhTraversal_inline.glsl:5-151). The node sequence it
// visits is a depth-first order in which, at an inner node whose two child
// boxes are both hit, child1 is entered first iff d1 < d0 and the other child
// is visited later without re-testing its box. A depth-first walk with an
// explicit stack that pushes that far child produces the same sequence, so it
// reproduces the reference's leaf order, box-test t values and hence its
// order-dependent closest-hit tie rule exactly, without the parent/sibling
// reloads. The stack lives in shared memory (one 32-entry column per thread,
// bank-conflict-free stride).
#pragma once
#include "common.cuh"

namespace timrt {

struct TravState {
    Ray r;
    float t;          // closest: current closest t (box tmax); any: fixed tmax
    uint32_t node;    // current node id (leaf bit set for leaves)
    int sp;
    bool any;
    bool done;
    bool hit;         // closest: a triangle was accepted; any: occluded
    uint32_t rec0, rec1, rec2, nid;
    float u, v;
    // work counters (dead code unless a counting kernel reads them)
    uint32_t c_node, c_leaf, c_tri, c_reload;
    uint32_t slot;      // policy scratch (pixel or queue slot of the ray)
    uint32_t slot2;     // policy scratch (secondary rays: the pixel)
    float ix, iy, iz;   // 1 / direction (8-wide form: zero components replaced, see wide_inv)
    float boxabs;       // binary walk: absolute margin of the filtered box test (+inf: exact test only)
    // 8-wide form only
    uint32_t order;     // rank mask of the current wide node's hit slots still to visit
    uint32_t oct;       // ray octant: bit a set when the direction's component a is negative
    uint32_t first;     // rank of the nearest hit slot still to visit first (8 = none)
    WideHdr h;          // header of the current wide node
    float t0;           // the ray's tmax
    float t1;           // closest: the smallest hit t; any: t of the hit
    bool near2;         // closest: another hit t2 has RN(t2 - 1e-5) <= t1
    bool dup_ok;        // closest: the hit leaf's id is not an output (see wide_leaf)
    uint32_t leaf;      // pending leaf slot of the current wide node (8 = none)
    uint32_t* err;      // two-level walk: the device error word (a nested walk's stack guard)
};

// Direction components for which the binary walk's filtered box test is exact
// (see box_filter): 0, or a magnitude within [2^-100, 2^100].
__device__ __forceinline__ bool box_dir_ok(float d) {
    const float a = fabsf(d);
    return a == 0.0f || (a >= 7.888609052210118e-31f && a <= 1.2676506002282294e30f);   // 0 or [2^-100, 2^100]
}

__device__ __forceinline__ void trav_init(TravState& st, uint32_t root) {
    st.ix = 1.0f / st.r.dx;
    st.iy = 1.0f / st.r.dy;
    st.iz = 1.0f / st.r.dz;
    st.boxabs = (box_dir_ok(st.r.dx) && box_dir_ok(st.r.dy) && box_dir_ok(st.r.dz) && st.t <= 1.2676506002282294e30f)
                    ? 7.888609052210118e-31f   // 2^-100
                    : __int_as_float(0x7F800000);
    st.node = root;
    st.c_node = st.c_leaf = st.c_tri = st.c_reload = 0u;
    st.sp = 0;
    st.done = false;
    st.hit = false;
    st.rec0 = st.rec1 = st.rec2 = 0u;
    st.nid = 0xFFFFFFFFu;
    st.u = st.v = 0.0f;
}

// The two child boxes of an inner node, with CollideBox's outcome: which children
// are hit and whether child 1 is entered first (d1 < d0).
//
// Filtered test. CollideBox divides, t = RN(RN(p - o) / d); the filter multiplies
// by inv = RN(1/d) instead, t' = RN(RN(p - o) * inv). For a ray whose direction
// components are 0 or within [2^-100, 2^100] (box_dir_ok) and whose tmax is at
// most 2^100 each slab value obeys
// |t - t'| <= 3.05u |t'| + 2^-148 (u = 2^-24), or both are at least 2^126 in
// magnitude with the same sign (overflow), and for d = 0 the two are identical
// (x / +-0 and x * +-inf give the same infinities, 0 / 0 and 0 * inf both NaN).
// min and max carry such bounds through to the aggregates M (largest slab entry)
// and T = min(tmax, smallest slab exit), so with m = 2^-20 (|M| + |T|) + 2^-100
// (four times the error plus the rounding of the tests themselves):
//   tmin + m < T - m   -> CollideBox hits, with its tmin in [lo, hi];
//   tmin - m >= T + m  -> CollideBox misses.
// Anything else (a box grazed within the margin, a ray outside the safe range:
// boxabs = +inf makes m infinite, every infinity or NaN in M or T does too), and
// an order that the tmin intervals cannot settle, takes the reference's
// divisions. The outcome is CollideBox's in every case; only the work differs.
// The slab values t = RN(RN(p - o) * inv) arrive computed (box_slabs); this
// decides from them.
__device__ __forceinline__ bool box_filter(const TravState& st, float t0x, float t0y, float t0z, float t1x, float t1y,
                                           float t1z, bool& hit, float& lo, float& hi) {
    const float M = fmaxf(fminf(t0x, t1x), fmaxf(fminf(t0y, t1y), fminf(t0z, t1z)));
    const float T = fminf(st.t, fminf(fmaxf(t0x, t1x), fminf(fmaxf(t0y, t1y), fmaxf(t0z, t1z))));
    const float m = __fmaf_rn(fabsf(M) + fabsf(T), 9.5367431640625e-07f, st.boxabs);   // 2^-20
    const float tmin = fmaxf(0.0f, M);
    if (tmin + m < T - m) {
        hit = true;
        const bool zero = M + m <= 0.0f;   // the entry lies behind the origin: tmin is exactly 0
        lo = zero ? 0.0f : fmaxf(0.0f, M - m);
        hi = zero ? 0.0f : tmin + m;
        return true;
    }
    hit = false;
    lo = hi = 0.0f;
    return tmin - m >= T + m;
}

// CollideBox of both children with the reference's divisions. Not inlined: the
// filter settles nearly every node, and the division code stays out of the loop.
static __device__ __noinline__ float2 exact_children(Ray r, float4 a, float4 b, float4 c, float tmax) {
    return make_float2(collide_box(r, a.x, a.y, c.x, a.z, a.w, c.y, tmax), collide_box(r, b.x, b.y, c.z, b.z, b.w, c.w, tmax));
}

// The six slab values of one child box, (p - o) * inv per plane, two planes per
// packed f32x2 subtract and multiply: the node record holds (min.x, min.y) and
// (max.x, max.y) of a child in adjacent words, its (min.z, max.z) likewise, so
// the pairs need no moves. Each element is rounded as the scalar operation
// rounds it, so the values are the scalar form's.
__device__ __forceinline__ void box_slabs(uint64_t oxy, uint64_t ixy, uint64_t ozz, uint64_t izz, float mnx, float mny,
                                          float mxx, float mxy, float mnz, float mxz, float& t0x, float& t0y, float& t0z,
                                          float& t1x, float& t1y, float& t1z) {
    unpack2f(mul2(sub2(pack2f(mnx, mny), oxy), ixy), t0x, t0y);
    unpack2f(mul2(sub2(pack2f(mxx, mxy), oxy), ixy), t1x, t1y);
    unpack2f(mul2(sub2(pack2f(mnz, mxz), ozz), izz), t0z, t1z);
}

__device__ __forceinline__ void plain_children(const TravState& st, const float4& a, const float4& b, const float4& c,
                                               bool& h0, bool& h1, bool& first1) {
    float lo0, hi0, lo1, hi1;
    const uint64_t oxy = pack2f(st.r.ox, st.r.oy), ixy = pack2f(st.ix, st.iy);
    const uint64_t ozz = pack2f(st.r.oz, st.r.oz), izz = pack2f(st.iz, st.iz);
    float t0x, t0y, t0z, t1x, t1y, t1z;
    box_slabs(oxy, ixy, ozz, izz, a.x, a.y, a.z, a.w, c.x, c.y, t0x, t0y, t0z, t1x, t1y, t1z);
    bool ok = box_filter(st, t0x, t0y, t0z, t1x, t1y, t1z, h0, lo0, hi0);
    box_slabs(oxy, ixy, ozz, izz, b.x, b.y, b.z, b.w, c.z, c.w, t0x, t0y, t0z, t1x, t1y, t1z);
    ok = box_filter(st, t0x, t0y, t0z, t1x, t1y, t1z, h1, lo1, hi1) && ok;
    first1 = hi1 < lo0;
    if (ok && h0 && h1 && !first1 && !(lo1 >= hi0)) ok = false;
    if (!ok) {
        const float2 d = exact_children(st.r, a, b, c, st.t);
        h0 = d.x >= 0.0f;
        h1 = d.y >= 0.0f;
        first1 = d.y < d.x;
    }
}

// What a leaf visit tests. kLeafOne: the one-level scene walk (bvh_collide /
// bvh_collide_fast: triangles, then for any-hit rays the leaf's BLAS boxes).
// kLeafTlasTop: the top level of a two-level walk (USE_TRAVERSE_TLAS, any-hit
// only): the leaf's BLAS instances (tlas_collide_fast). kLeafInBlas: a leaf of a
// BLAS entered from the top level (bvh_collide_fast compiled with
// USE_TRAVERSE_TLAS: triangles only).
constexpr int kLeafOne = 0, kLeafTlasTop = 1, kLeafInBlas = 2;

template <int LEAF>
__device__ __forceinline__ void plain_leaf(const SceneView& s, TravState& st, uint32_t node);

// Acceptance of one triangle hit (bvh_collide / bvh_collide_fast): any-hit rays
// end, closest-hit rays keep it and shrink their t by 1e-5. Returns true when
// the ray ends.
__device__ __forceinline__ bool plain_accept(TravState& st, float t, float u, float v, uint32_t r0, uint32_t r1,
                                             uint32_t r2, uint32_t nidm) {
    if (st.any) {
        st.hit = true;
        st.done = true;
        return true;
    }
    st.t = t - kOffsetRayCollision;
    st.rec0 = r0; st.rec1 = r1; st.rec2 = r2;
    st.nid = nidm;
    st.u = u; st.v = v;
    st.hit = true;
    return false;
}

// Leaf visit: bvh_collide (bvhCollision.glsl:177-239) for closest-hit rays,
// bvh_collide_fast (bvhCollision.glsl:241-284) for any-hit rays. With the
// scene's leaf-triangle copy the leaf's record is one 16-byte load and each
// triangle three 16-byte loads of (p0, e1, e2) with the reference's record words
// in .w; without it (the allocation-free entry point and the 8-wide kernels'
// fallback walk) the record words and the vertex positions are gathered from the
// reference's own buffers. Same triangles, same order, same arithmetic.
// The top-level leaf of a two-level any-hit walk; defined below.
static __device__ __noinline__ bool tlas_leaf_any(SceneView s, uint32_t nidm, Ray r, float tmax, uint32_t* err);

template <int LEAF>
__device__ __forceinline__ void plain_leaf(const SceneView& s, TravState& st, uint32_t node) {
    const uint32_t nidm = node & kNidMask;
    uint32_t hdr, off;
    st.c_leaf++;
    if (LEAF == kLeafTlasTop) {
        if (tlas_leaf_any(s, nidm, st.r, st.t, st.err)) {
            st.hit = true;
            st.done = true;
        }
        return;
    }
    if (s.ptris) {
        const uint4 li = __ldg(s.pleaf + nidm);
        hdr = li.y;
        off = li.z;
        const uint32_t ntri = hdr & ((1u << kTriBits) - 1u);
        const float4* tp = s.ptris + 3u * li.x;
        for (uint32_t i = 0; i < ntri; ++i, tp += 3) {
            st.c_tri++;
            const float4 A = __ldg(tp), B = __ldg(tp + 1), C = __ldg(tp + 2);
            float u, v;
            const float t = collide_triangle_e(st.r, A.x, A.y, A.z, B.x, B.y, B.z, C.x, C.y, C.z, st.t, u, v);
            if (t > 0.0f && plain_accept(st, t, u, v, __float_as_uint(A.w), __float_as_uint(B.w), __float_as_uint(C.w),
                                         nidm))
                return;
        }
    } else {
        off = __ldg(reinterpret_cast<const uint32_t*>(s.nodes + 4u * nidm) + 3);
        hdr = leaf_header(s, off);
        const uint32_t ntri = hdr & ((1u << kTriBits) - 1u);
        const uint32_t* rec = s.leaf + off + 1u;
        for (uint32_t i = 0; i < ntri; ++i, rec += 3) {
            st.c_tri++;
            const uint32_t r0 = __ldg(rec), r1 = __ldg(rec + 1), r2 = __ldg(rec + 2);
            const uint32_t i0 = r0 + (r1 & 0xFFFFu), i1 = r0 + (r1 >> 16), i2 = r0 + (r2 & 0xFFFFu);
            const float* P0 = s.pos + 3u * i0;
            const float* P1 = s.pos + 3u * i1;
            const float* P2 = s.pos + 3u * i2;
            const float p0x = __ldg(P0), p0y = __ldg(P0 + 1), p0z = __ldg(P0 + 2);
            const float e1x = __ldg(P1) - p0x, e1y = __ldg(P1 + 1) - p0y, e1z = __ldg(P1 + 2) - p0z;
            const float e2x = __ldg(P2) - p0x, e2y = __ldg(P2 + 1) - p0y, e2z = __ldg(P2 + 2) - p0z;
            float u, v;
            const float t = collide_triangle_e(st.r, p0x, p0y, p0z, e1x, e1y, e1z, e2x, e2y, e2z, st.t, u, v);
            if (t > 0.0f && plain_accept(st, t, u, v, r0, r1, r2, nidm)) return;
        }
    }
    if (LEAF == kLeafOne && st.any) {
        const uint32_t ntri = hdr & ((1u << kTriBits) - 1u);
        const uint32_t nblas = (hdr >> kTriBits) & ((1u << kBlasBits) - 1u);
        for (uint32_t i = 0; i < nblas; ++i) {
            const uint32_t bi = __ldg(s.leaf + off + 1u + 3u * ntri + i);
            const float* bh = s.blas + 8u * bi;
            const float mnx = __ldg(bh), mny = __ldg(bh + 1), mnz = __ldg(bh + 2);
            const float mxx = __ldg(bh + 4), mxy = __ldg(bh + 5), mxz = __ldg(bh + 6);
            const bool inside = st.r.ox > mnx && st.r.oy > mny && st.r.oz > mnz && st.r.ox < mxx &&
                                st.r.oy < mxy && st.r.oz < mxz;
            if (!inside && collide_box(st.r, mnx, mny, mnz, mxx, mxy, mxz, st.t) > 0.0f) {
                st.hit = true;
                st.done = true;
                return;
            }
        }
    }
}

// One traversal step: descend to the next leaf (or exhaust the stack), test it,
// and pop the next pending subtree. Returns with st.done set when the ray ends.
template <int BLOCK, int LEAF = kLeafOne>
__device__ __forceinline__ void plain_step(const SceneView& s, TravState& st, uint32_t* stk, uint32_t* err,
                                           int sdepth) {
    uint32_t node = st.node;
    while (!(node & kNidLeafBit)) {
        const float4* np = s.nodes + 4u * node;
        st.c_node++;
        const uint4 nid = __ldg(reinterpret_cast<const uint4*>(np));
        const float4 a = __ldg(np + 1);   // n0xy = (c0.min.x, c0.min.y, c0.max.x, c0.max.y)
        const float4 b = __ldg(np + 2);   // n1xy
        const float4 c = __ldg(np + 3);   // nz = (c0.min.z, c0.max.z, c1.min.z, c1.max.z)
        // the reference's divisions: this walk only retraces the rare rays the 8-wide
        // walk cannot settle, and the filter's code would only add registers there
        const float d0 = collide_box(st.r, a.x, a.y, c.x, a.z, a.w, c.y, st.t);
        const float d1 = collide_box(st.r, b.x, b.y, c.z, b.z, b.w, c.w, st.t);
        const bool h0 = d0 >= 0.0f, h1 = d1 >= 0.0f, first1 = d1 < d0;
        const uint32_t packed = nid.z;
        uint32_t c0 = packed & kNidMask;
        uint32_t c1 = c0 + 1u;
        c0 |= (packed & kNidLeftLeafBit) ? kNidLeafBit : 0u;
        c1 |= (packed & kNidRightLeafBit) ? kNidLeafBit : 0u;
        if (!h0 && !h1) {
            if (st.sp == 0) {
                st.done = true;
                return;
            }
            node = stk[(--st.sp) * BLOCK];
            continue;
        }
        if (h0 && h1) {
            if (st.sp >= sdepth) {   // unreachable: the stack holds the tree depth
                atomicOr(err, 1u);
                st.done = true;
                return;
            }
            stk[(st.sp++) * BLOCK] = first1 ? c0 : c1;
            node = first1 ? c1 : c0;
        } else {
            node = h0 ? c0 : c1;
        }
    }
    plain_leaf<LEAF>(s, st, node);
    if (st.done) return;
    if (st.sp == 0) {
        st.done = true;
        return;
    }
    st.node = stk[(--st.sp) * BLOCK];
}

// One advance of one lane from the inner node st.node: test its two child boxes
// and move to the child the reference enters first (pushing the other when both
// are hit), or pop the next pending subtree when neither is hit. At most one node
// per call, so that lanes calling it together test their nodes together.
template <int BLOCK>
__device__ __forceinline__ void plain_advance(const SceneView& s, TravState& st, uint32_t* stk, uint32_t* err,
                                              int sdepth) {
    const uint32_t node = st.node;
    const float4* np = s.nodes + 4u * node;
    st.c_node++;
    const uint4 nid = __ldg(reinterpret_cast<const uint4*>(np));
    const float4 a = __ldg(np + 1);
    const float4 b = __ldg(np + 2);
    const float4 c = __ldg(np + 3);
    bool h0, h1, first1;
    plain_children(st, a, b, c, h0, h1, first1);
    const uint32_t packed = nid.z;
    uint32_t c0 = packed & kNidMask;
    uint32_t c1 = c0 + 1u;
    c0 |= (packed & kNidLeftLeafBit) ? kNidLeafBit : 0u;
    c1 |= (packed & kNidRightLeafBit) ? kNidLeafBit : 0u;
    if (!h0 && !h1) {
        if (st.sp == 0) {
            st.done = true;
            return;
        }
        st.node = stk[(--st.sp) * BLOCK];
        return;
    }
    if (h0 && h1) {
        if (st.sp >= sdepth) {   // unreachable: the stack holds the tree depth
            atomicOr(err, 1u);
            st.done = true;
            return;
        }
        stk[(st.sp++) * BLOCK] = first1 ? c0 : c1;
        st.node = first1 ? c1 : c0;
    } else {
        st.node = h0 ? c0 : c1;
    }
}

// One traversal step of the whole warp, called by all 32 lanes (`active`: the
// lane has a ray): node rounds in lockstep until every lane stands on a leaf or
// has finished, or until only `sw` lanes still need nodes while some lane stands
// on a leaf; then the leaves are tested together and each lane pops its next
// pending subtree. Same per-ray visit order as plain_step.
template <int BLOCK, int LEAF = kLeafOne>
__device__ __forceinline__ void plain_step_warp(const SceneView& s, TravState& st, bool active, uint32_t* stk,
                                                uint32_t* err, int sdepth, uint32_t sw) {
    for (;;) {
        const bool need = active && !st.done && !(st.node & kNidLeafBit);
        const uint32_t nm = __ballot_sync(0xFFFFFFFFu, need);
        if (nm == 0u) break;
        if ((uint32_t)__popc(nm) <= sw &&
            __any_sync(0xFFFFFFFFu, active && !st.done && (st.node & kNidLeafBit))) break;
        if (need) plain_advance<BLOCK>(s, st, stk, err, sdepth);
    }
    if (active && !st.done && (st.node & kNidLeafBit)) {
        plain_leaf<LEAF>(s, st, st.node);
        if (!st.done) {
            if (st.sp == 0) st.done = true;
            else st.node = stk[(--st.sp) * BLOCK];
        }
    }
}

// tlas_collide_fast (bvhCollision.glsl:321-348) at top-level leaf nidm: for
// each BLAS instance of the leaf, in order, CollideBox(ray, instance box, tmax)
// > 0 -- an origin inside the box gives tmin = 0 and skips the instance -- then
// traverseBvhFast from the instance's rootIndex, entered as an inner node
// (bvhTraversal_inline.glsl:83-151; the image check makes every rootIndex an
// inner node). The leaf's triangle records are not tested. Not inlined, with its
// own stack in local memory: the nested walk runs while the top-level walk's
// shared-memory stack is in use.
static __device__ __noinline__ bool tlas_leaf_any(SceneView s, uint32_t nidm, Ray r, float tmax, uint32_t* err) {
    uint32_t hdr, off;
    if (s.ptris) {
        const uint4 li = __ldg(s.pleaf + nidm);
        hdr = li.y;
        off = li.z;
    } else {
        off = __ldg(reinterpret_cast<const uint32_t*>(s.nodes + 4u * nidm) + 3);
        hdr = leaf_header(s, off);
    }
    if (off == 0xFFFFFFFFu) return false;
    const uint32_t ntri = hdr & ((1u << kTriBits) - 1u);
    const uint32_t nblas = (hdr >> kTriBits) & ((1u << kBlasBits) - 1u);
    uint32_t stk[kStackSize];
    for (uint32_t i = 0; i < nblas; ++i) {
        const uint32_t bi = __ldg(s.leaf + off + 1u + 3u * ntri + i);
        const float* bh = s.blas + 8u * bi;
        const float mnx = __ldg(bh), mny = __ldg(bh + 1), mnz = __ldg(bh + 2);
        const float mxx = __ldg(bh + 4), mxy = __ldg(bh + 5), mxz = __ldg(bh + 6);
        if (!(collide_box(r, mnx, mny, mnz, mxx, mxy, mxz, tmax) > 0.0f)) continue;
        TravState st;
        st.r = r;
        st.t = tmax;
        st.any = true;
        st.err = err;
        trav_init(st, __float_as_uint(__ldg(bh + 7)));   // rootIndex, an inner node id
        do {
            plain_step<1, kLeafInBlas>(s, st, stk, err, kStackSize);
        } while (!st.done);
        if (st.hit) return true;
    }
    return false;
}

}  // namespace timrt
