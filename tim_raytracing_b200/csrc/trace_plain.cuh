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
    // 8-wide form only
    float ix, iy, iz;   // 1 / direction
    uint32_t order;     // rank mask of the current wide node's hit slots still to visit
    uint32_t oct;       // ray octant: bit a set when the direction's component a is negative
    uint32_t first;     // rank of the nearest hit slot still to visit first (8 = none)
    WideHdr h;          // header of the current wide node
    float t0;           // the ray's tmax
    float t1;           // closest: the smallest hit t; any: t of the hit
    bool near2;         // closest: another hit t2 has RN(t2 - 1e-5) <= t1
    uint32_t leaf;      // pending leaf slot of the current wide node (8 = none)
};

__device__ __forceinline__ void trav_init(TravState& st, uint32_t root) {
    st.node = root;
    st.c_node = st.c_leaf = st.c_tri = st.c_reload = 0u;
    st.sp = 0;
    st.done = false;
    st.hit = false;
    st.rec0 = st.rec1 = st.rec2 = 0u;
    st.nid = 0xFFFFFFFFu;
    st.u = st.v = 0.0f;
}

// Leaf visit: bvh_collide (bvhCollision.glsl:177-239) for closest-hit rays,
// bvh_collide_fast (bvhCollision.glsl:241-284) for any-hit rays.
__device__ __forceinline__ void plain_leaf(const SceneView& s, TravState& st, uint32_t node) {
    const uint32_t nidm = node & kNidMask;
    const uint32_t off = __ldg(reinterpret_cast<const uint32_t*>(s.nodes + 4u * nidm) + 3);
    const uint32_t hdr = leaf_header(s, off);
    const uint32_t ntri = hdr & ((1u << kTriBits) - 1u);
    const uint32_t* rec = s.leaf + off + 1u;
    st.c_leaf++;
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
        if (t > 0.0f) {
            if (st.any) {
                st.hit = true;
                st.done = true;
                return;
            }
            st.t = t - kOffsetRayCollision;
            st.rec0 = r0; st.rec1 = r1; st.rec2 = r2;
            st.nid = nidm;
            st.u = u; st.v = v;
            st.hit = true;
        }
    }
    if (st.any) {
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
template <int BLOCK>
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
        const float d0 = collide_box(st.r, a.x, a.y, c.x, a.z, a.w, c.y, st.t);
        const float d1 = collide_box(st.r, b.x, b.y, c.z, b.z, b.w, c.w, st.t);
        const uint32_t packed = nid.z;
        uint32_t c0 = packed & kNidMask;
        uint32_t c1 = c0 + 1u;
        c0 |= (packed & kNidLeftLeafBit) ? kNidLeafBit : 0u;
        c1 |= (packed & kNidRightLeafBit) ? kNidLeafBit : 0u;
        if (d0 < 0.0f && d1 < 0.0f) {
            if (st.sp == 0) {
                st.done = true;
                return;
            }
            node = stk[(--st.sp) * BLOCK];
            continue;
        }
        if (d0 >= 0.0f && d1 >= 0.0f) {
            const bool first1 = d1 < d0;
            if (st.sp >= sdepth) {   // unreachable: the stack holds the tree depth
                atomicOr(err, 1u);
                st.done = true;
                return;
            }
            stk[(st.sp++) * BLOCK] = first1 ? c0 : c1;
            node = first1 ? c1 : c0;
        } else {
            node = (d0 >= 0.0f) ? c0 : c1;
        }
    }
    plain_leaf(s, st, node);
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
    const float d0 = collide_box(st.r, a.x, a.y, c.x, a.z, a.w, c.y, st.t);
    const float d1 = collide_box(st.r, b.x, b.y, c.z, b.z, b.w, c.w, st.t);
    const uint32_t packed = nid.z;
    uint32_t c0 = packed & kNidMask;
    uint32_t c1 = c0 + 1u;
    c0 |= (packed & kNidLeftLeafBit) ? kNidLeafBit : 0u;
    c1 |= (packed & kNidRightLeafBit) ? kNidLeafBit : 0u;
    if (d0 < 0.0f && d1 < 0.0f) {
        if (st.sp == 0) {
            st.done = true;
            return;
        }
        st.node = stk[(--st.sp) * BLOCK];
        return;
    }
    if (d0 >= 0.0f && d1 >= 0.0f) {
        const bool first1 = d1 < d0;
        if (st.sp >= sdepth) {   // unreachable: the stack holds the tree depth
            atomicOr(err, 1u);
            st.done = true;
            return;
        }
        stk[(st.sp++) * BLOCK] = first1 ? c0 : c1;
        st.node = first1 ? c1 : c0;
    } else {
        st.node = (d0 >= 0.0f) ? c0 : c1;
    }
}

// One traversal step of the whole warp, called by all 32 lanes (`active`: the
// lane has a ray): node rounds in lockstep until every lane stands on a leaf or
// has finished, or until only `sw` lanes still need nodes while some lane stands
// on a leaf; then the leaves are tested together and each lane pops its next
// pending subtree. Same per-ray visit order as plain_step.
template <int BLOCK>
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
        plain_leaf(s, st, st.node);
        if (!st.done) {
            if (st.sp == 0) st.done = true;
            else st.node = stk[(--st.sp) * BLOCK];
        }
    }
}

}  // namespace timrt
