// common.cuh -- device-side layouts and the reference's intersection arithmetic.
//
// Floating-point policy (identical to the CPU restatement used as the parity
// checker): the library is compiled with --fmad=false, -prec-div=true and
// -prec-sqrt=true, so every a*b+c below is a rounded multiply followed by a
// rounded add, divisions and square roots are IEEE round-to-nearest, and GLSL
// min/max are fminf/fmaxf. Dot products sum left to right and cross() keeps
// GLSL component order; that is what makes hit ids and t bit-exact.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace timrt {

constexpr float kTMax = 100.0f;                 // struct_cpp.glsl:5 TMAX
constexpr float kEpsTri = 1e-7f;                // collision.glsl:62 (10e-8)
constexpr float kOffsetRayCollision = 1e-5f;    // system.glsl:45 (10e-6)
constexpr uint32_t kNidLeafBit = 0x80000000u;   // struct_cpp.glsl:52-55
constexpr uint32_t kNidMask = 0x3FFFFFFFu;
constexpr uint32_t kNidLeftLeafBit = 0x80000000u;
constexpr uint32_t kNidRightLeafBit = 0x40000000u;
constexpr uint32_t kTriBits = 12, kBlasBits = 8, kPrimBits = 8, kLightBits = 4;  // primitive_cpp.glsl:18-21
constexpr uint32_t kLightSphere = 1u;           // primitive_cpp.glsl:8
constexpr int kStackSize = 32;                  // the reference's bitstack is 32 bits wide

// Device view of one uploaded scene (reference layout).
struct SceneView {
    const float4* nodes;        // PackedBVHNode: nid, n0xy, n1xy, nz (primitive_cpp.glsl:80-86)
    const uint32_t* leaf;       // leaf-data words
    const float* pos;           // xyz per vertex
    const float* nrm;           // xyz per vertex (may be null)
    const float* lights;        // PackedLight, 14 words each (primitive_cpp.glsl:113-117)
    const float* blas;          // BlasHeader, 8 words each (primitive_cpp.glsl:88-94)
    const float* materials;     // Material, 12 words each (primitive_cpp.glsl:67-72)
    uint32_t num_nodes;
    uint32_t num_lights;
    uint32_t leaf_words;
    uint32_t num_vertex;
    uint32_t depth;             // binary tree depth (stack entries needed)
    uint32_t wide_depth;        // 8-wide tree depth
    // 8-wide quantised form (null when not built)
    const uint4* wnodes;        // WideNode, 5 x 16 B
    const float4* wtris;        // 3 x float4 per leaf triangle: (p0, vo) (e1, i01) (e2, i2m)
    const uint4* wtri_leaf;     // per wide triangle, its binary leaf: (E lo.xyz, nid), (E hi.xyz, flag)
    uint32_t num_wnodes;
    uint32_t wide_root_is_leaf; // scene is a single leaf
    // the plain form's leaf-triangle copy (null: read the reference's leaf data and
    // positions directly, as the allocation-free entry point does)
    const uint4* pleaf;         // per node: (first triangle, leaf header, leaf-data offset, 0)
    const float4* ptris;        // 3 x float4 per leaf triangle: (p0, vo) (e1, i01) (e2, i2m)
};

struct Ray {
    float ox, oy, oz, dx, dy, dz;
};

// Header words of the current 8-wide node (see trace_wide.cuh).
struct WideHdr {
    uint32_t imask, child_base, tri_base, meta_lo, meta_hi;
};

__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
    return ax * bx + ay * by + az * bz;
}

// collision.glsl:23-40 CollideBox with STORE_RAY_INVDIR = 0 (true division).
__device__ __forceinline__ float collide_box(const Ray& r, float mnx, float mny, float mnz, float mxx, float mxy,
                                             float mxz, float tmax) {
    const float t0x = (mnx - r.ox) / r.dx, t0y = (mny - r.oy) / r.dy, t0z = (mnz - r.oz) / r.dz;
    const float t1x = (mxx - r.ox) / r.dx, t1y = (mxy - r.oy) / r.dy, t1z = (mxz - r.oz) / r.dz;
    const float sx = fminf(t0x, t1x), sy = fminf(t0y, t1y), sz = fminf(t0z, t1z);
    const float bx = fmaxf(t0x, t1x), by = fmaxf(t0y, t1y), bz = fmaxf(t0z, t1z);
    const float tmin = fmaxf(0.0f, fmaxf(sx, fmaxf(sy, sz)));
    const float tm = fminf(tmax, fminf(bx, fminf(by, bz)));
    return (tmin < tm) ? tmin : -1.0f;
}

// collision.glsl:58-95 CollideTriangle on (p0, edge1, edge2); edge1 = p1 - p0 and
// edge2 = p2 - p0 are the same rounded values whether computed here or ahead of time.
__device__ __forceinline__ float collide_triangle_e(const Ray& r, float p0x, float p0y, float p0z, float e1x,
                                                    float e1y, float e1z, float e2x, float e2y, float e2z,
                                                    float tmax, float& uo, float& vo) {
    const float hx = r.dy * e2z - r.dz * e2y;
    const float hy = r.dz * e2x - r.dx * e2z;
    const float hz = r.dx * e2y - r.dy * e2x;
    const float a = dot3(e1x, e1y, e1z, hx, hy, hz);
    if (fabsf(a) < kEpsTri) return -1.0f;
    const float f = 1.0f / a;
    const float sx = r.ox - p0x, sy = r.oy - p0y, sz = r.oz - p0z;
    const float u = f * dot3(sx, sy, sz, hx, hy, hz);
    if (fminf(fmaxf(u, 0.0f), 1.0f) != u) return -1.0f;
    const float qx = sy * e1z - sz * e1y;
    const float qy = sz * e1x - sx * e1z;
    const float qz = sx * e1y - sy * e1x;
    const float v = f * dot3(r.dx, r.dy, r.dz, qx, qy, qz);
    if (v < 0.0f || u + v > 1.0f) return -1.0f;
    const float t = f * dot3(e2x, e2y, e2z, qx, qy, qz);
    if (t > kEpsTri && t < tmax) {
        uo = u;
        vo = v;
        return t;
    }
    return -1.0f;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Leaf header read; nodes whose packed count is 0 carry offset 0xFFFFFFFF
// (BVHBuilder.cpp:1515) and are treated as empty.
__device__ __forceinline__ uint32_t leaf_header(const SceneView& s, uint32_t off) {
    return (off == 0xFFFFFFFFu || off >= s.leaf_words) ? 0u : __ldg(s.leaf + off);
}

// Packed pairs of floats (sm_100 f32x2 arithmetic): lo in the low 32 bits.
__device__ __forceinline__ uint64_t pack2f(float lo, float hi) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void unpack2f(uint64_t v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}
__device__ __forceinline__ uint64_t sub2(uint64_t a, uint64_t b) {
    uint64_t r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ uint64_t mul2(uint64_t a, uint64_t b) {
    uint64_t r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}

}  // namespace timrt
