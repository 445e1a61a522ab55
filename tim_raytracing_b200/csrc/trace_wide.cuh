// trace_wide.cuh -- traversal of the 8-wide BVH with 8-bit quantised child bounds.
//
// Node layout (80 B = 5 x 16 B, built by wide_build.cpp from the reference's
// binary tree):
//   w0..w2  origin (float) of the quantisation grid
//   w3      ex | ey << 8 | ez << 16 | imask << 24   (scale per axis = 2^(e-127);
//           imask bit k: slot k is an internal wide node)
//   w4      index of the first internal child node (internal children are contiguous)
//   w5      first triangle (in the leaf-triangle array) of this node's leaf slots
//   w6,w7   meta byte per slot: triangle count of a leaf slot (0 = empty / internal)
//   w8..w19 qlo_x[8] qlo_y[8] qlo_z[8] qhi_x[8] qhi_y[8] qhi_z[8]
// Slot k's box decodes to lo = origin + scale * qlo, hi = origin + scale * qhi
// (an exact product and one rounded add); the builder chooses qlo / qhi so the
// decoded float box contains the box the reference stores for that subtree.
//
// Leaf triangles are stored as 3 x float4: (p0, vertexOffset) (p1-p0, index01)
// (p2-p0, index2_matId) -- the edges are the same rounded differences
// CollideTriangle computes, so the triangle test stays bit-identical.
//
// Box test: the reference's slab test divides by the direction; here it
// multiplies by 1/d and then widens near/far by a relative 2^-18, which covers
// the (<= 2^-21 relative) difference between the two forms. Together with the
// outward-rounded bounds, a child whose reference box test passes always
// passes here: the quantised traversal never loses a hit the binary one finds.
#pragma once
#include "common.cuh"
#include "trace_plain.cuh"

namespace timrt {

__device__ __forceinline__ float wdecode(float o, float sc, uint32_t word, uint32_t k) {
    const uint32_t q = (word >> (8u * k)) & 0xFFu;
    return o + sc * (float)q;
}

// Tests the 8 slots of wide node `ni` and returns the hit slots ordered by
// entry distance: bits 0..23 = slots (3 bits each, nearest first), bits 24..27 = count.
__device__ __forceinline__ uint32_t wide_visit(const SceneView& s, const TravState& st, float ix, float iy, float iz,
                                               uint32_t ni, WideHdr& h) {
    const uint4* np = s.wnodes + 5u * ni;
    const uint4 U0 = __ldg(np), U1 = __ldg(np + 1), U2 = __ldg(np + 2), U3 = __ldg(np + 3), U4 = __ldg(np + 4);
    h.imask = U0.w >> 24;
    h.child_base = U1.x;
    h.tri_base = U1.y;
    h.meta_lo = U1.z;
    h.meta_hi = U1.w;
    const float ox = __uint_as_float(U0.x), oy = __uint_as_float(U0.y), oz = __uint_as_float(U0.z);
    const float sx = __uint_as_float((U0.w & 0xFFu) << 23);
    const float sy = __uint_as_float(((U0.w >> 8) & 0xFFu) << 23);
    const float sz = __uint_as_float(((U0.w >> 16) & 0xFFu) << 23);
    const float tcur = st.t;
    uint32_t key[8];
#pragma unroll
    for (uint32_t k = 0; k < 8u; ++k) {
        const uint32_t wsel = k < 4u ? 0u : 1u, kk = k & 3u;
        const uint32_t meta = ((wsel ? h.meta_hi : h.meta_lo) >> (8u * kk)) & 0xFFu;
        const bool valid = ((h.imask >> k) & 1u) || meta != 0u;
        const float lx = wdecode(ox, sx, wsel ? U2.y : U2.x, kk);
        const float ly = wdecode(oy, sy, wsel ? U2.w : U2.z, kk);
        const float lz = wdecode(oz, sz, wsel ? U3.y : U3.x, kk);
        const float hx = wdecode(ox, sx, wsel ? U3.w : U3.z, kk);
        const float hy = wdecode(oy, sy, wsel ? U4.y : U4.x, kk);
        const float hz = wdecode(oz, sz, wsel ? U4.w : U4.z, kk);
        const float t0x = (lx - st.r.ox) * ix, t1x = (hx - st.r.ox) * ix;
        const float t0y = (ly - st.r.oy) * iy, t1y = (hy - st.r.oy) * iy;
        const float t0z = (lz - st.r.oz) * iz, t1z = (hz - st.r.oz) * iz;
        float nearv = fmaxf(fminf(t0x, t1x), fmaxf(fminf(t0y, t1y), fminf(t0z, t1z)));
        float farv = fminf(fmaxf(t0x, t1x), fminf(fmaxf(t0y, t1y), fmaxf(t0z, t1z)));
        // widen by a relative 2^-18; a product keeps +-inf (direction component 0)
        // infinite, where a subtraction of |x| * eps would turn inf into NaN
        nearv = nearv * (nearv > 0.0f ? 0.999996185302734375f : 1.000003814697265625f);
        farv = farv * (farv > 0.0f ? 1.000003814697265625f : 0.999996185302734375f);
        const float tmin = fmaxf(0.0f, nearv);
        const float tm = fminf(tcur, farv);
        const bool hit = valid && (tmin < tm);
        // non-negative floats order like their bit patterns; the low 3 bits carry the slot
        key[k] = hit ? ((__float_as_uint(tmin) & ~7u) | k) : 0xFFFFFFFFu;
    }
    // sorting network for 8 keys (Batcher odd-even merge, 19 compare-exchanges)
#define TIMRT_CX(a, b)                               \
    {                                                \
        const uint32_t lo_ = min(key[a], key[b]);    \
        const uint32_t hi_ = max(key[a], key[b]);    \
        key[a] = lo_;                                \
        key[b] = hi_;                                \
    }
    TIMRT_CX(0, 1) TIMRT_CX(2, 3) TIMRT_CX(4, 5) TIMRT_CX(6, 7)
    TIMRT_CX(0, 2) TIMRT_CX(1, 3) TIMRT_CX(4, 6) TIMRT_CX(5, 7)
    TIMRT_CX(1, 2) TIMRT_CX(5, 6) TIMRT_CX(0, 4) TIMRT_CX(3, 7)
    TIMRT_CX(1, 5) TIMRT_CX(2, 6)
    TIMRT_CX(1, 4) TIMRT_CX(3, 6)
    TIMRT_CX(2, 4) TIMRT_CX(3, 5)
    TIMRT_CX(3, 4)
#undef TIMRT_CX
    uint32_t order = 0, cnt = 0;
#pragma unroll
    for (uint32_t k = 0; k < 8u; ++k) {
        if (key[k] != 0xFFFFFFFFu) {
            order |= (key[k] & 7u) << (3u * cnt);
            ++cnt;
        }
    }
    return order | (cnt << 24);
}

__device__ __forceinline__ void wide_read_hdr(const SceneView& s, uint32_t ni, WideHdr& h) {
    const uint4* np = s.wnodes + 5u * ni;
    const uint4 U0 = __ldg(np), U1 = __ldg(np + 1);
    h.imask = U0.w >> 24;
    h.child_base = U1.x;
    h.tri_base = U1.y;
    h.meta_lo = U1.z;
    h.meta_hi = U1.w;
}

template <int BLOCK>
__device__ __forceinline__ void wide_leaf(const SceneView& s, TravState& st, const WideHdr& h, uint32_t slot) {
    const uint32_t below_lo = slot >= 4u ? h.meta_lo : (slot == 0u ? 0u : (h.meta_lo & ((1u << (8u * slot)) - 1u)));
    const uint32_t below_hi = slot <= 4u ? 0u : (h.meta_hi & ((1u << (8u * (slot - 4u))) - 1u));
    const uint32_t first = h.tri_base + __dp4a(below_lo, 0x01010101u, __dp4a(below_hi, 0x01010101u, 0u));
    const uint32_t cnt = ((slot < 4u ? h.meta_lo : h.meta_hi) >> (8u * (slot & 3u))) & 0xFFu;
    const float4* tp = s.wtris + 3u * first;
    st.c_leaf++;
    for (uint32_t i = 0; i < cnt; ++i, tp += 3) {
        st.c_tri++;
        const float4 A = __ldg(tp), B = __ldg(tp + 1), C = __ldg(tp + 2);
        float u, v;
        const float t = collide_triangle_e(st.r, A.x, A.y, A.z, B.x, B.y, B.z, C.x, C.y, C.z, st.t, u, v);
        if (t > 0.0f) {
            if (st.any) {
                st.hit = true;
                st.done = true;
                return;
            }
            st.t = t - kOffsetRayCollision;
            st.rec0 = __float_as_uint(A.w);
            st.rec1 = __float_as_uint(B.w);
            st.rec2 = __float_as_uint(C.w);
            st.nid = __ldg(s.wtri_nid + first + i);
            st.u = u;
            st.v = v;
            st.hit = true;
        }
    }
}

__device__ __forceinline__ void wide_init(const SceneView& s, TravState& st, uint32_t*) {
    st.ix = 1.0f / st.r.dx;
    st.iy = 1.0f / st.r.dy;
    st.iz = 1.0f / st.r.dz;
    st.sp = 0;
    st.done = false;
    st.hit = false;
    st.rec0 = st.rec1 = st.rec2 = 0u;
    st.nid = 0xFFFFFFFFu;
    st.u = st.v = 0.0f;
    st.node = 0u;
    st.c_node = st.c_leaf = st.c_tri = st.c_reload = 0u;
    if (s.num_wnodes == 0u) {
        st.done = true;
        return;
    }
    if (s.wide_root_is_leaf) {   // the reference intersects a single-leaf tree without a box test
        wide_read_hdr(s, 0u, st.h);
        st.order = 1u << 24;
    } else {
        st.c_node++;
        st.order = wide_visit(s, st, st.ix, st.iy, st.iz, 0u, st.h);
    }
}

// One step: walk slots nearest-first, descending into internal slots (the rest
// of the current node is pushed as one (node, order) entry), until one leaf
// slot has been tested or the traversal ends.
template <int BLOCK>
__device__ __forceinline__ void wide_step(const SceneView& s, TravState& st, uint32_t* stk, uint32_t* err) {
    for (;;) {
        const uint32_t cnt = st.order >> 24;
        if (cnt == 0u) {
            if (st.sp == 0) {
                st.done = true;
                return;
            }
            --st.sp;
            st.node = stk[(2 * st.sp) * BLOCK];
            st.order = stk[(2 * st.sp + 1) * BLOCK];
            wide_read_hdr(s, st.node, st.h);
            st.c_reload++;
            continue;
        }
        const uint32_t slot = st.order & 7u;
        st.order = ((st.order & 0xFFFFFFu) >> 3) | ((cnt - 1u) << 24);
        if ((st.h.imask >> slot) & 1u) {
            const uint32_t child = st.h.child_base + __popc(st.h.imask & ((1u << slot) - 1u));
            if ((st.order >> 24) != 0u) {
                if (st.sp >= kStackSize) {   // unreachable: wide depth <= binary depth <= 32
                    atomicOr(err, 1u);
                    st.done = true;
                    return;
                }
                stk[(2 * st.sp) * BLOCK] = st.node;
                stk[(2 * st.sp + 1) * BLOCK] = st.order;
                ++st.sp;
            }
            st.node = child;
            st.c_node++;
            st.order = wide_visit(s, st, st.ix, st.iy, st.iz, child, st.h);
        } else {
            wide_leaf<BLOCK>(s, st, st.h, slot);
            return;
        }
    }
}

}  // namespace timrt
