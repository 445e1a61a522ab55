// trace_wide.cuh -- traversal of the 8-wide BVH with 8-bit quantised child bounds.
//
// Node layout (80 B = 5 x 16 B, built by bvh_layout.cpp from the reference's
// binary tree; the compressed wide-node idea follows Ylitie, Karras & Laine,
// "Efficient Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs",
// HPG 2017, with a layout of our own):
//   w0..w2  origin o (float) of the quantisation grid
//   w3      ex | ey << 8 | ez << 16 | imask << 24   (scale per axis s = 2^(e-127);
//           imask bit k: slot k is an internal wide node)
//   w4      index of the first internal child node (internal children are contiguous)
//   w5      first triangle (in the leaf-triangle array) of this node's leaf slots
//   w6,w7   meta byte per slot: triangle count of a leaf slot (0 = empty / internal)
//   w8..w19 qlo_x[8] qlo_y[8] qlo_z[8] qhi_x[8] qhi_y[8] qhi_z[8]
// Slot k spans [o + s*qlo, o + s*qhi] per axis (real arithmetic); the builder
// rounds outward so this box contains the box the reference stores for the
// subtree.
//
// Leaf triangles are stored as 3 x float4: (p0, vertexOffset) (p1-p0, index01)
// (p2-p0, index2_matId) -- the edges are the same rounded differences
// CollideTriangle computes, so the triangle test stays bit-identical.
//
// Box test, and why it never rejects a child the reference accepts. Per node
// and axis the kernel forms A = RN(RN(o - r) * inv) and B = s * inv (exact: s is
// a power of two), with inv = RN(1/d), and evaluates every plane as one fused
// multiply-add t = RN(q * B' + A'), where A' and B' are A and B moved outward by
// 2^-18 of their magnitude (down for near planes, up for far planes). Against
// the exact distance T = (o + s*q - r)/d, A and q*B are within 3u|A| and u q|B|
// (u = 2^-24), the moves shift the sum by 2^-18 (|A| + q|B|) and the roundings
// of A', B' and the FMA add below 3u (|A| + q|B|); since |T| <= |A*| + q|B*| the
// shift exceeds all of that plus the 2u|T| the reference's own two roundings
// can take away. Near and far planes are picked from the sign of inv, which
// for d != 0 equals the min / max of the two slab distances. A zero direction
// component is replaced by +-2^-80 for this test only, which keeps all values
// finite. So, for rays whose direction components are at least 2^-60 and whose
// origin lies within 2^60, tmin_here <= tmin_reference and tmax_here >=
// tmax_reference for every child: the quantised traversal visits a superset of
// the binary traversal's leaves and never loses a hit. For other rays (a zero
// or tiny component, a far origin) the slab can come out narrower than the
// reference's, so their 8-wide answer, hit or miss, is not trusted
// (wide_trusted): they are traced again by the binary walk (a single-leaf
// tree, which both walks test without a box, excepted).
//
// Same hit as the binary walk, for every ray. The reference's closest-hit rule
// is order-dependent: a hit at t is accepted iff t < c, and then c = t - 1e-5,
// so of two hits less than 1e-5 apart the one visited first wins. The 8-wide
// walk visits leaves in another order, so it finds the smallest hit t1 exactly
// (every candidate below c = min(tmax, t1 + 1e-5 + 2^-20 t1 + 2^-30) is tested),
// tracks whether the second smallest t2 lies in its window, and keeps its answer
// only when the binary walk provably gives the same one:
//   (a) RN(t2 - 1e-5) > t1: no other hit can block the nearest one whatever the
//       order, and after it is accepted none can replace it; and
//   (b) its binary leaf is reached: the intersection E of the leaf's box and the
//       boxes of all its binary ancestors (per axis the largest lower and the
//       smallest upper plane, precomputed per leaf) passes CollideBox with
//       tmin <= t1. For a direction without zero components IEEE subtraction and
//       division are monotonic, so E's slab entry is the largest entry and its
//       exit the smallest exit of all those boxes: each of them then passes its
//       own test with any c > t1, which is every value c takes before the
//       nearest hit is accepted. (The reference builder's child boxes can stick
//       out of the parent's by an ulp, so the leaf box alone would not do.)
// Any-hit rays keep their first hit under (b) alone. A ray failing a test (a
// near-tie, a hit grazing its leaf box: about one ray in 10^5) is traced again
// from the root by the binary walk (binary_walk below), which reproduces the
// reference's order exactly.
#pragma once
#include "common.cuh"
#include "trace_plain.cuh"

namespace timrt {

constexpr float kWiden = 3.814697265625e-06f;   // 2^-18

// Three-input max / min (PTX max.f32 / min.f32 with three sources, sm_100). Used
// only where no operand can be NaN.
__device__ __forceinline__ float max3f(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Byte k of w0 and of w1 as the floats 2^23 + q (0x4B0000qq is exact), packed;
// sub2 with 2^23 then gives q.
__device__ __forceinline__ uint64_t qbytes2(uint32_t w0, uint32_t w1, uint32_t k) {
    uint64_t r;
    const uint32_t lo = __byte_perm(w0, 0x4B000000u, 0x7650u | k), hi = __byte_perm(w1, 0x4B000000u, 0x7650u | k);
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "r"(lo), "r"(hi));
    return r;
}

// Tests the 8 slots of wide node `ni` and returns the hit slots as a rank mask:
// bit r set = slot r ^ octant(ray) was hit. Visiting ranks in increasing order is
// roughly front to back because the builder placed each child in the slot of its
// direction from the node centre (bit a = + side of axis a) and the octant bit a
// is set for rays going towards -a.
__device__ __forceinline__ uint32_t wide_visit(const SceneView& s, const TravState& st, uint32_t ni, WideHdr& h,
                                               uint32_t& first) {
    const uint4* np = s.wnodes + 5u * ni;
    const uint4 U0 = __ldg(np), U1 = __ldg(np + 1), U2 = __ldg(np + 2), U3 = __ldg(np + 3), U4 = __ldg(np + 4);
    h.imask = U0.w >> 24;
    h.child_base = U1.x;
    h.tri_base = U1.y;
    h.meta_lo = U1.z;
    h.meta_hi = U1.w;
    const float ix = st.ix, iy = st.iy, iz = st.iz;
    // per-axis plane coefficients: t = q * B + A
    const float Bx = __uint_as_float((U0.w & 0xFFu) << 23) * ix;
    const float By = __uint_as_float(((U0.w >> 8) & 0xFFu) << 23) * iy;
    const float Bz = __uint_as_float(((U0.w >> 16) & 0xFFu) << 23) * iz;
    const float Ax = (__uint_as_float(U0.x) - st.r.ox) * ix;
    const float Ay = (__uint_as_float(U0.y) - st.r.oy) * iy;
    const float Az = (__uint_as_float(U0.z) - st.r.oz) * iz;
    const float Anx = __fmaf_rn(-fabsf(Ax), kWiden, Ax), Afx = __fmaf_rn(fabsf(Ax), kWiden, Ax);
    const float Any = __fmaf_rn(-fabsf(Ay), kWiden, Ay), Afy = __fmaf_rn(fabsf(Ay), kWiden, Ay);
    const float Anz = __fmaf_rn(-fabsf(Az), kWiden, Az), Afz = __fmaf_rn(fabsf(Az), kWiden, Az);
    const float Bnx = __fmaf_rn(-fabsf(Bx), kWiden, Bx), Bfx = __fmaf_rn(fabsf(Bx), kWiden, Bx);
    const float Bny = __fmaf_rn(-fabsf(By), kWiden, By), Bfy = __fmaf_rn(fabsf(By), kWiden, By);
    const float Bnz = __fmaf_rn(-fabsf(Bz), kWiden, Bz), Bfz = __fmaf_rn(fabsf(Bz), kWiden, Bz);
    // near / far plane words from the direction's sign
    const bool negx = __float_as_uint(ix) >> 31, negy = __float_as_uint(iy) >> 31, negz = __float_as_uint(iz) >> 31;
    const uint32_t nx0 = negx ? U3.z : U2.x, nx1 = negx ? U3.w : U2.y, fx0 = negx ? U2.x : U3.z, fx1 = negx ? U2.y : U3.w;
    const uint32_t ny0 = negy ? U4.x : U2.z, ny1 = negy ? U4.y : U2.w, fy0 = negy ? U2.z : U4.x, fy1 = negy ? U2.w : U4.y;
    const uint32_t nz0 = negz ? U4.z : U3.x, nz1 = negz ? U4.w : U3.y, fz0 = negz ? U3.x : U4.z, fz1 = negz ? U3.y : U4.w;
    const float tcur = st.t;
    // Slots k and k + 4 in one packed pair, one axis at a time: each plane of both
    // slots is one sub.f32x2 (byte to float) and one fma.f32x2, which round each
    // half exactly as the scalar FADD and FFMA do (IEEE round to nearest per
    // element), so every value is that of the scalar form of this test.
    const uint64_t magic = pack2f(8388608.0f, 8388608.0f);
    float tn[8], tf[8];   // running slab entry / exit per slot
#pragma unroll
    for (uint32_t kk = 0; kk < 4u; ++kk) {
        unpack2f(fma2(sub2(qbytes2(nx0, nx1, kk), magic), pack2f(Bnx, Bnx), pack2f(Anx, Anx)), tn[kk], tn[kk + 4u]);
        unpack2f(fma2(sub2(qbytes2(fx0, fx1, kk), magic), pack2f(Bfx, Bfx), pack2f(Afx, Afx)), tf[kk], tf[kk + 4u]);
    }
#pragma unroll
    for (uint32_t kk = 0; kk < 4u; ++kk) {
        float a, b, c, d;
        unpack2f(fma2(sub2(qbytes2(ny0, ny1, kk), magic), pack2f(Bny, Bny), pack2f(Any, Any)), a, b);
        unpack2f(fma2(sub2(qbytes2(fy0, fy1, kk), magic), pack2f(Bfy, Bfy), pack2f(Afy, Afy)), c, d);
        tn[kk] = fmaxf(tn[kk], a);
        tn[kk + 4u] = fmaxf(tn[kk + 4u], b);
        tf[kk] = fminf(tf[kk], c);
        tf[kk + 4u] = fminf(tf[kk + 4u], d);
    }
    uint32_t mask = 0, nearest = 0xFFFFFFFFu;
#pragma unroll
    for (uint32_t kk = 0; kk < 4u; ++kk) {
        float a[2], c[2];
        unpack2f(fma2(sub2(qbytes2(nz0, nz1, kk), magic), pack2f(Bnz, Bnz), pack2f(Anz, Anz)), a[0], a[1]);
        unpack2f(fma2(sub2(qbytes2(fz0, fz1, kk), magic), pack2f(Bfz, Bfz), pack2f(Afz, Afz)), c[0], c[1]);
#pragma unroll
        for (uint32_t h2 = 0; h2 < 2u; ++h2) {
            // empty slots carry the inverted box qlo = 255, qhi = 0 and fail this test
            // by themselves (if rounding ever lets one through, it is a leaf of 0 triangles)
            const uint32_t k = kk + 4u * h2;
            const float tmin = max3f(tn[k], a[h2], 0.0f);
            const float tm = min3f(tf[k], c[h2], tcur);
            const bool hit = tmin < tm;
            // slot k is visited at rank k ^ octant: children were placed by direction
            mask |= (hit ? 1u : 0u) << (k ^ st.oct);
            // the nearest hit slot goes first (non-negative floats order like their bits)
            nearest = min(nearest, hit ? ((__float_as_uint(tmin) & ~7u) | (k ^ st.oct)) : 0xFFFFFFFFu);
        }
    }
    first = nearest & 7u;
    return mask;
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

// Tests the triangles of leaf slot `slot` in their stored order (bvh_collide /
// bvh_collide_fast semantics, bvhCollision.glsl:177-284).
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
                st.t1 = t;
                st.nid = first + i;   // wide triangle; wide_finish turns it into the leaf nid
                return;
            }
            if (t < st.t1) {
                // the old nearest becomes the second nearest (it is <= any other hit)
                st.near2 = st.t1 - kOffsetRayCollision <= t;
                st.t1 = t;
                // test every hit that could still block or replace the nearest one
                // (c = t + 1e-5 + 2^-20 t + 2^-30: the margin exceeds the rounding of
                // RN(t2 - 1e-5) and of this sum, so every t2 that matters is below c)
                st.t = fminf(st.t0, t + (kOffsetRayCollision + (t * 9.5367431640625e-07f + 9.313225746154785e-10f)));
                st.rec0 = __float_as_uint(A.w);
                st.rec1 = __float_as_uint(B.w);
                st.rec2 = __float_as_uint(C.w);
                st.nid = first + i;
                // wide_finish reads this triangle's leaf record: start fetching it now
                asm volatile("prefetch.global.L1 [%0];" ::"l"(s.wtri_leaf + 2u * (first + i)));
                st.u = u;
                st.v = v;
                st.hit = true;
            } else {
                // A second reference to the nearest triangle itself -- the reference
                // builder copies a triangle into every leaf it straddles -- gives the
                // same record, t and barycentrics; whichever copy the binary walk meets
                // first, the other then fails t < c. Only the leaf id would differ, so
                // where the leaf id is not an output (dup_ok) it is no competing hit.
                const bool same_tri = st.dup_ok && t == st.t1 && __float_as_uint(A.w) == st.rec0 &&
                                      __float_as_uint(B.w) == st.rec1 && __float_as_uint(C.w) == st.rec2;
                st.near2 = st.near2 || (!same_tri && t - kOffsetRayCollision <= st.t1);
            }
        }
    }
}

// 1 / d for the quantised box test; a zero component becomes +-2^-80 (see above).
__device__ __forceinline__ float wide_inv(float d) { return 1.0f / (d == 0.0f ? copysignf(8.271806125530277e-25f, d) : d); }

__device__ __forceinline__ void wide_init(const SceneView& s, TravState& st, uint32_t*) {
    st.ix = wide_inv(st.r.dx);
    st.iy = wide_inv(st.r.dy);
    st.iz = wide_inv(st.r.dz);
    st.oct = (__float_as_uint(st.ix) >> 31) | ((__float_as_uint(st.iy) >> 31) << 1) | ((__float_as_uint(st.iz) >> 31) << 2);
    st.sp = 0;
    st.done = false;
    st.hit = false;
    st.rec0 = st.rec1 = st.rec2 = 0u;
    st.nid = 0xFFFFFFFFu;
    st.u = st.v = 0.0f;
    st.node = 0u;
    st.c_node = st.c_leaf = st.c_tri = st.c_reload = 0u;
    st.t1 = __int_as_float(0x7F800000);   // +inf (st.t0 = tmax is set by the caller)
    st.near2 = false;
    st.leaf = 8u;
    if (s.num_wnodes == 0u) {
        st.done = true;
        return;
    }
    if (s.wide_root_is_leaf) {   // the reference intersects a single-leaf tree without a box test
        wide_read_hdr(s, 0u, st.h);
        st.order = 1u << st.oct;   // slot 0
        st.first = 8u;
    } else {
        st.c_node++;
        st.order = wide_visit(s, st, 0u, st.h, st.first);
    }
}

// One advance of one lane: take the next hit slot in rank order (popping a
// pending node first when the current one is used up); an internal slot is
// visited (the rest of the current node is pushed as one (node << 8 | rank
// mask) entry), a leaf slot becomes the lane's pending leaf (st.leaf). At most
// one node visit per call, so that lanes calling it together visit together.
template <int BLOCK>
__device__ __forceinline__ void wide_advance(const SceneView& s, TravState& st, uint32_t* stk, uint32_t* err,
                                             int sdepth) {
    if (st.order == 0u) {
        if (st.sp == 0) {
            st.done = true;
            return;
        }
        --st.sp;
        const uint32_t e = stk[st.sp * BLOCK];
        st.node = e >> 8;
        st.order = e & 0xFFu;   // never 0: only non-empty remainders are pushed
        st.first = 8u;
        wide_read_hdr(s, st.node, st.h);
        st.c_reload++;
    }
    uint32_t r;
    if (st.first < 8u) {   // the nearest hit slot of a freshly visited node
        r = st.first;
        st.first = 8u;
    } else {
        r = (uint32_t)(__ffs(st.order) - 1);
    }
    st.order &= ~(1u << r);
    const uint32_t slot = r ^ st.oct;
    if ((st.h.imask >> slot) & 1u) {
        const uint32_t child = st.h.child_base + __popc(st.h.imask & ((1u << slot) - 1u));
        if (st.order != 0u) {
            if (st.sp >= sdepth) {   // unreachable: the stack holds the 8-wide tree depth
                atomicOr(err, 1u);
                st.done = true;
                return;
            }
            stk[st.sp * BLOCK] = (st.node << 8) | st.order;   // fewer than 2^24 nodes (checked at build)
            ++st.sp;
        }
        st.node = child;
        st.c_node++;
        st.order = wide_visit(s, st, child, st.h, st.first);
    } else {
        st.leaf = slot;
    }
}

// One traversal step of the whole warp, called by all 32 lanes (`active`: the
// lane has a ray): first the lanes advance, one node visit per round and all in
// the same rounds, until each has a pending leaf slot or has finished -- or until
// only `sw` lanes still need nodes while some lane holds a leaf (those few lanes
// go on in the next step instead of making the warp run near-empty rounds); then
// the lanes test their pending leaves together. Without this the node test and
// the triangle loop ran in many passes of a few lanes each, as lanes reached
// them at different iterations of a per-lane loop.
template <int BLOCK>
__device__ __forceinline__ void wide_step_warp(const SceneView& s, TravState& st, bool active, uint32_t* stk,
                                               uint32_t* err, int sdepth, uint32_t sw) {
    for (;;) {
        const bool need = active && !st.done && st.leaf >= 8u;
        const uint32_t nm = __ballot_sync(0xFFFFFFFFu, need);
        if (nm == 0u) break;
        if ((uint32_t)__popc(nm) <= sw && __any_sync(0xFFFFFFFFu, active && st.leaf < 8u)) break;
        if (need) wide_advance<BLOCK>(s, st, stk, err, sdepth);
    }
    if (active && st.leaf < 8u) {
        const uint32_t slot = st.leaf;
        st.leaf = 8u;
        wide_leaf<BLOCK>(s, st, st.h, slot);
    }
}

// Whether the 8-wide walk's answer for this ray may stand at all. The slab
// argument above needs finite plane distances that contain the reference's: a
// zero direction component is replaced by +-2^-80, which turns the reference's
// unbounded slab (origin strictly inside, 1/0 = inf) into a finite one that
// can end short of a hit when the origin lies within about 2^-80 tmax of the
// plane, and a component below 2^-126 overflows 1/d. Such a narrower slab can
// lose the nearest hit as well as every hit, so the walk's answer, a hit or a
// miss, counts only when every component is at least 2^-60 in magnitude and the
// origin within 2^60 (with scene coordinates below 2^60 every plane distance is
// then finite); other rays are traced again by the binary walk.
__device__ __forceinline__ bool wide_trusted(const Ray& r) {
    constexpr float dlo = 8.673617379884035e-19f, ohi = 1.152921504606847e18f;   // 2^-60, 2^60
    return fabsf(r.dx) >= dlo && fabsf(r.dy) >= dlo && fabsf(r.dz) >= dlo &&      // false for NaN too
           fabsf(r.ox) <= ohi && fabsf(r.oy) <= ohi && fabsf(r.oz) <= ohi;
}

// Called when the 8-wide walk of a ray ends: keeps its answer (binary leaf nid,
// closest t - 1e-5) when tests (a) and (b) above hold and returns true;
// otherwise returns false and the caller has the ray traced by the binary walk.
__device__ __forceinline__ bool wide_finish(const SceneView& s, TravState& st) {
    // the box test is conservative only for trusted rays (see wide_trusted): for
    // them, no hit below tmax anywhere means the binary walk finds none either
    const bool trusted = wide_trusted(st.r);
    if (!st.hit) return trusted;
    const uint4 lo = __ldg(s.wtri_leaf + 2u * st.nid), hi = __ldg(s.wtri_leaf + 2u * st.nid + 1u);
    bool same = hi.w == 1u;     // a single-leaf tree is intersected without a box test
    // an untrusted ray may have lost a nearer hit, and an empty E proves nothing:
    // binary walk (trusted rays have no zero direction component)
    if (hi.w == 0u && trusted) {
        const float lx = __uint_as_float(lo.x), ly = __uint_as_float(lo.y), lz = __uint_as_float(lo.z);
        const float hx = __uint_as_float(hi.x), hy = __uint_as_float(hi.y), hz = __uint_as_float(hi.z);
        // Fast proof first: with inv = RN(1/d) (d != 0 here), RN((p - o) * inv) is
        // within 2^-22 |t| of CollideBox's RN((p - o) / d), so moving every entry up
        // and every exit down by 2^-21 |t| bounds the reference's tmin from above and
        // its exit from below. (An infinite plane distance makes t +- |t| e NaN only
        // on the side fminf / fmaxf then ignore, which is the side that does not
        // constrain the reference either; the 2^-100 terms cover underflow.) Rays
        // this cannot settle take the exact test with the reference's divisions.
        constexpr float e = 4.76837158203125e-07f;   // 2^-21
        constexpr float a = 7.888609052210118e-31f;  // 2^-100
        const float ax = (lx - st.r.ox) * st.ix, bx = (hx - st.r.ox) * st.ix;
        const float ay = (ly - st.r.oy) * st.iy, by = (hy - st.r.oy) * st.iy;
        const float az = (lz - st.r.oz) * st.iz, bz = (hz - st.r.oz) * st.iz;
        const float sx = fminf(ax, bx), sy = fminf(ay, by), sz = fminf(az, bz);
        const float fx = fmaxf(ax, bx), fy = fmaxf(ay, by), fz = fmaxf(az, bz);
        const float up = fmaxf(0.0f, fmaxf(sx + fabsf(sx) * e, fmaxf(sy + fabsf(sy) * e, sz + fabsf(sz) * e))) + a;
        const float dn = fminf(fx - fabsf(fx) * e, fminf(fy - fabsf(fy) * e, fz - fabsf(fz) * e)) - a;
        same = up <= st.t1 && up < dn;
        if (!same) {
            const float d = collide_box(st.r, lx, ly, lz, hx, hy, hz, st.t0);
            same = d >= 0.0f && d <= st.t1;
        }
    }
    if (!st.any) same = same && !st.near2;
    if (same) {
        st.nid = lo.w;
        if (!st.any) st.t = st.t1 - kOffsetRayCollision;
        return true;
    }
    return false;
}

// The binary walk of one ray from the root to the end, for the rays wide_finish
// could not prove. Not inlined: its code and registers stay out of the 8-wide
// kernels' hot loop (inlined, even unexecuted, it slowed them by about 5%); the
// lane that calls it runs the whole walk while the warp's other lanes wait, which
// costs little at about one ray in 10^5, and other warps hide its latency.
struct BinaryResult {
    uint32_t rec0, rec1, rec2, nid;
    float t, u, v;
    uint32_t hit;
};

static __device__ __noinline__ BinaryResult binary_walk(const float4* nodes, const uint32_t* leaf, const float* pos,
                                                        const float* blas, uint32_t num_nodes, uint32_t leaf_words,
                                                        float ox, float oy, float oz, float dx, float dy, float dz,
                                                        float tmax, bool any, uint32_t* err) {
    SceneView v{};
    v.nodes = nodes;
    v.leaf = leaf;
    v.pos = pos;
    v.blas = blas;
    v.num_nodes = num_nodes;
    v.leaf_words = leaf_words;
    TravState st;
    st.r.ox = ox; st.r.oy = oy; st.r.oz = oz;
    st.r.dx = dx; st.r.dy = dy; st.r.dz = dz;
    st.t = tmax;
    st.any = any;
    trav_init(st, num_nodes == 1u ? kNidLeafBit : 0u);
    uint32_t stk[kStackSize];
    do {
        plain_step<1>(v, st, stk, err, kStackSize);
    } while (!st.done);
    return {st.rec0, st.rec1, st.rec2, st.nid, st.t, st.u, st.v, st.hit ? 1u : 0u};
}

// wide_finish, and the binary walk when it fails: afterwards st holds the
// reference's answer for the ray.
__device__ __forceinline__ void wide_finish_or_walk(const SceneView& s, TravState& st, uint32_t* err) {
    if (wide_finish(s, st)) return;
    const BinaryResult b = binary_walk(s.nodes, s.leaf, s.pos, s.blas, s.num_nodes, s.leaf_words, st.r.ox, st.r.oy,
                                       st.r.oz, st.r.dx, st.r.dy, st.r.dz, st.t0, st.any, err);
    st.rec0 = b.rec0; st.rec1 = b.rec1; st.rec2 = b.rec2; st.nid = b.nid;
    st.t = b.t; st.u = b.u; st.v = b.v;
    st.hit = b.hit != 0u;
}

}  // namespace timrt
