// trace.cu -- persistent ray-tracing kernels for sm_100a and their launchers.
//
// Every trace kernel here is the same persistent loop: a grid sized to fill
// the GPU (blocks per SM from the occupancy calculator x 148 SMs), in which
// each warp keeps all 32 lanes busy by refilling finished lanes with new work
// items from a global atomic counter (one atomicAdd per refill, issued by one
// elected lane). A policy object turns a work item into a ray (load) and
// writes the result (store): plain ray batches, camera pixels, secondary
// (shadow / probe-visibility / bounce) rays, probe rays.
#include <cuda_runtime.h>
#include <cstdio>
#include "common.cuh"
#include "trace_plain.cuh"
#include "trace_wide.cuh"
#include "kernels.h"
#include "../../include/tim_rt.h"

namespace timrt {

// -------------------------------------------------------------------- policies

struct BatchPolicy {
    const tim_rt_ray* rays;
    uint4* hit;
    uint32_t* nid;
    float2* bary;
    uint32_t mode;

    __device__ __forceinline__ bool load(const SceneView&, uint32_t i, TravState& st) const {
        const float4* rp = reinterpret_cast<const float4*>(rays + i);
        const float4 a = __ldg(rp), b = __ldg(rp + 1);
        st.r.ox = a.x; st.r.oy = a.y; st.r.oz = a.z;
        st.r.dx = b.x; st.r.dy = b.y; st.r.dz = b.z;
        st.t = a.w;
        const uint32_t fl = __float_as_uint(b.w);
        st.any = (mode == TIM_RT_MODE_ANY) || (mode == TIM_RT_MODE_PER_RAY && (fl & TIM_RT_RAY_ANY));
        return true;
    }
    __device__ __forceinline__ void store(const SceneView&, uint32_t i, const TravState& st, float tmax0) const {
        if (st.any) {
            hit[i] = make_uint4(st.hit ? 1u : 0u, 0u, 0u, __float_as_uint(tmax0));
            if (nid) nid[i] = 0xFFFFFFFFu;
            if (bary) bary[i] = make_float2(0.f, 0.f);
        } else {
            hit[i] = make_uint4(st.rec0, st.rec1, st.rec2, __float_as_uint(st.t));
            if (nid) nid[i] = st.hit ? st.nid : 0xFFFFFFFFu;
            if (bary) bary[i] = make_float2(st.u, st.v);
        }
    }
    __device__ __forceinline__ void skip(uint32_t) const {}
};

// cameraPass.comp:44-76: one work item per output pixel.
struct CameraPolicy {
    tim_rt_pass_data pd;
    uint32_t ngy16;         // 16 * ceil(H / 16)
    uint4* out;             // 2 x uint4 per pixel
    uint32_t* leaf_nid;     // per pixel, for the leaf-light shadow mask

    __device__ __forceinline__ bool load(const SceneView&, uint32_t pix, TravState& st) const {
        const uint32_t W = pd.frameSize[0];
        const uint32_t px = pix % W, py = pix / W;
        if (py == 0u) return false;   // never produced by the reference's row mapping
        const uint32_t gx = px, gy = ngy16 - py;
        const float fx = (float)gx, fy = (float)gy;
        const float swx = (pd.frustumCorner10[0] - pd.frustumCorner00[0]) * pd.invFrameSize[0];
        const float swy = (pd.frustumCorner10[1] - pd.frustumCorner00[1]) * pd.invFrameSize[0];
        const float swz = (pd.frustumCorner10[2] - pd.frustumCorner00[2]) * pd.invFrameSize[0];
        const float shx = (pd.frustumCorner01[0] - pd.frustumCorner00[0]) * pd.invFrameSize[1];
        const float shy = (pd.frustumCorner01[1] - pd.frustumCorner00[1]) * pd.invFrameSize[1];
        const float shz = (pd.frustumCorner01[2] - pd.frustumCorner00[2]) * pd.invFrameSize[1];
        const float tx = (pd.frustumCorner00[0] + swx * fx) + shx * fy;
        const float ty = (pd.frustumCorner00[1] + swy * fx) + shy * fy;
        const float tz = (pd.frustumCorner00[2] + swz * fx) + shz * fy;
        const float vx = tx - pd.cameraPos[0], vy = ty - pd.cameraPos[1], vz = tz - pd.cameraPos[2];
        const float len = sqrtf(dot3(vx, vy, vz, vx, vy, vz));
        st.r.ox = pd.cameraPos[0]; st.r.oy = pd.cameraPos[1]; st.r.oz = pd.cameraPos[2];
        st.r.dx = vx / len; st.r.dy = vy / len; st.r.dz = vz / len;
        st.t = kTMax;
        st.any = false;
        return true;
    }
    __device__ __forceinline__ void store(const SceneView&, uint32_t pix, const TravState& st, float) const {
        out[2u * pix] = make_uint4(st.rec0, st.rec1, st.rec2, __float_as_uint(st.t));
        out[2u * pix + 1u] = make_uint4(0u, 0u, 0u, 0u);
        leaf_nid[pix] = st.hit ? st.nid : 0xFFFFFFFFu;
    }
    __device__ __forceinline__ void skip(uint32_t pix) const {
        out[2u * pix] = make_uint4(0u, 0u, 0u, 0u);
        out[2u * pix + 1u] = make_uint4(0u, 0u, 0u, 0u);
        leaf_nid[pix] = 0xFFFFFFFFu;
    }
};

// Secondary rays generated from camera hits. ray.flags: bit 0 any-hit, bits
// 8..15 the mask bit, bits 16..17 the kind (0 shadow mask, 1 probe mask, 2 bounce).
struct SecondaryPolicy {
    const tim_rt_ray* rays;
    const uint32_t* pixel;
    uint32_t* out_words;    // tracingData as u32 words (8 per pixel)
    uint4* bounce_out;

    __device__ __forceinline__ bool load(const SceneView&, uint32_t i, TravState& st) const {
        const float4* rp = reinterpret_cast<const float4*>(rays + i);
        const float4 a = __ldg(rp), b = __ldg(rp + 1);
        st.r.ox = a.x; st.r.oy = a.y; st.r.oz = a.z;
        st.r.dx = b.x; st.r.dy = b.y; st.r.dz = b.z;
        st.t = a.w;
        st.any = (__float_as_uint(b.w) & 1u) != 0u;
        return true;
    }
    __device__ __forceinline__ void store(const SceneView&, uint32_t i, const TravState& st, float) const {
        const uint32_t fl = __float_as_uint(__ldg(reinterpret_cast<const float*>(rays + i) + 7));
        const uint32_t kind = (fl >> 16) & 3u, bit = (fl >> 8) & 0xFFu;
        const uint32_t p = __ldg(pixel + i);
        if (kind == 2u) {
            bounce_out[p] = make_uint4(st.rec0, st.rec1, st.rec2, __float_as_uint(st.t));
        } else if (st.hit) {
            atomicOr(out_words + 8u * p + 4u + kind, 1u << bit);
        }
    }
    __device__ __forceinline__ void skip(uint32_t) const {}
};

// -------------------------------------------------------------------- persistent loop

template <int BLOCK, bool WIDE, bool STATS, class Policy>
__global__ void __launch_bounds__(BLOCK) k_persistent(SceneView s, Policy P, uint32_t n_static,
                                                      const uint32_t* n_dev, uint32_t* counter, uint32_t* err,
                                                      unsigned long long* stats) {
    extern __shared__ uint32_t stack_mem[];   // (WIDE ? 2 : 1) * kStackSize * BLOCK words
    uint32_t* stk = stack_mem + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t n = n_dev ? *n_dev : n_static;
    const uint32_t root = s.num_nodes == 1u ? kNidLeafBit : 0u;   // baseRaytracingPass.glsl:20

    TravState st;
    st.done = true;
    bool active = false, exhausted = false;
    uint32_t idx = 0;
    float tmax0 = 0.f;
    for (;;) {
        if (!exhausted) {
            const uint32_t need = __ballot_sync(0xFFFFFFFFu, !active);
            if (need) {
                const int leader = __ffs(need) - 1;
                uint32_t base = 0;
                if ((int)lane == leader) base = atomicAdd(counter, (uint32_t)__popc(need));
                base = __shfl_sync(0xFFFFFFFFu, base, leader);
                if ((uint64_t)base + (uint32_t)__popc(need) >= n) exhausted = true;
                if (!active) {
                    const uint32_t my = base + __popc(need & lanemask_lt());
                    if (my < n) {
                        idx = my;
                        if (P.load(s, idx, st)) {
                            tmax0 = st.t;
                            if (WIDE) wide_init(s, st, stk);
                            else trav_init(st, root);
                            active = true;
                        } else {
                            P.skip(idx);
                        }
                    }
                }
            }
        }
        if (__ballot_sync(0xFFFFFFFFu, active) == 0u) {
            if (exhausted) break;
            continue;
        }
        if (active) {
            if (WIDE) wide_step<BLOCK>(s, st, stk, err);
            else plain_step<BLOCK>(s, st, stk, err);
            if (st.done) {
                P.store(s, idx, st, tmax0);
                if (STATS) {
                    atomicAdd(stats + 0, 1ull);
                    atomicAdd(stats + 1, (unsigned long long)st.c_node);
                    atomicAdd(stats + 2, (unsigned long long)st.c_leaf);
                    atomicAdd(stats + 3, (unsigned long long)st.c_tri);
                    atomicAdd(stats + 4, (unsigned long long)st.c_reload);
                }
                active = false;
            }
        }
    }
}

// -------------------------------------------------------------------- secondary ray generation

__device__ __forceinline__ uint32_t hash32(uint32_t x) {
    x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
    return x;
}
__device__ __forceinline__ float u01(uint32_t h) { return (float)(h >> 8) * (1.0f / 16777216.0f); }

// Cosine-weighted direction about unit normal (nx,ny,nz): Malley's method with
// a rejection-sampled disk point and the orthonormal basis of Duff et al.,
// "Building an Orthonormal Basis, Revisited" (JCGT 2017).
__device__ __forceinline__ void bounce_dir(float nx, float ny, float nz, uint32_t pixel, uint32_t seed, float& dx,
                                           float& dy, float& dz) {
    float x = 0.f, y = 0.f;
    for (uint32_t k = 0; k < 16u; ++k) {
        const uint32_t h0 = hash32(pixel * 2u + 0x9E3779B9u * (seed + 1u) + k * 0x85EBCA6Bu);
        const uint32_t h1 = hash32(h0 ^ 0x27D4EB2Fu);
        const float a = u01(h0) * 2.0f - 1.0f, b = u01(h1) * 2.0f - 1.0f;
        if (a * a + b * b < 1.0f) { x = a; y = b; break; }
    }
    const float z = sqrtf(fmaxf(0.0f, 1.0f - x * x - y * y));
    const float sign = copysignf(1.0f, nz);
    const float a = -1.0f / (sign + nz);
    const float b = nx * ny * a;
    const float b1x = 1.0f + sign * nx * nx * a, b1y = sign * b, b1z = -sign * nx;
    const float b2x = b, b2y = sign + ny * ny * a, b2z = -ny;
    dx = (b1x * x + b2x * y) + nx * z;
    dy = (b1y * x + b2y * y) + ny * z;
    dz = (b1z * x + b2z * y) + nz * z;
}

struct GenParams {
    tim_rt_pass_data pd;
    uint32_t flags;
    uint32_t seed;
    uint32_t ngy16;
    uint32_t tiles_x;
    const uint32_t* tile_counts;
    const uint32_t* tile_lists;
    uint32_t* out_words;
    const uint32_t* leaf_nid;
    uint4* bounce_out;
    tim_rt_ray* q_rays;
    uint32_t* q_pixel;
    uint32_t* q_count;
    uint32_t q_capacity;
};

__device__ __forceinline__ void lpf_position(const tim_rt_pass_data& pd, uint32_t cx, uint32_t cy, uint32_t cz,
                                             float& x, float& y, float& z) {
    // lightprobHelpers.glsl:63-69 getLightProbPosition
    const float stx = (pd.sceneMaxExtent[0] - pd.sceneMinExtent[0]) / (float)pd.lpfResolution[0];
    const float sty = (pd.sceneMaxExtent[1] - pd.sceneMinExtent[1]) / (float)pd.lpfResolution[1];
    const float stz = (pd.sceneMaxExtent[2] - pd.sceneMinExtent[2]) / (float)pd.lpfResolution[2];
    x = pd.sceneMinExtent[0] + stx * ((float)cx + 0.5f);
    y = pd.sceneMinExtent[1] + sty * ((float)cy + 0.5f);
    z = pd.sceneMinExtent[2] + stz * ((float)cz + 0.5f);
}

// For each camera hit, emit the rays of computeAdditionalHitData
// (baseRaytracingPass.glsl:85-97): the sun shadow ray and one ray per light of
// the hit leaf's list (bvhLighting.glsl:143-163) or of the pixel's tile list,
// the 8 probe-visibility segments (bvhLighting.glsl:165-184) and the bounce.
// Lights out of range set their bit directly (evalShadow returns true,
// bvhLighting.glsl:121-124).
__global__ void __launch_bounds__(256) k_gen_secondary(SceneView s, GenParams g) {
    const uint32_t W = g.pd.frameSize[0], H = g.pd.frameSize[1];
    const uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31u;
    tim_rt_ray local[1 + 16 + 8 + 1];
    uint32_t nr = 0;
    uint32_t direct_bits = 0;
    bool valid = pix < W * H;
    uint4 rec = make_uint4(0, 0, 0, 0);
    if (valid) rec = reinterpret_cast<const uint4*>(g.out_words)[2u * pix];
    const float t = __uint_as_float(rec.w);
    const uint32_t py = valid ? pix / W : 0u;
    if (valid && py != 0u && t < kTMax) {
        const uint32_t px = pix % W, gx = px, gy = g.ngy16 - py;
        // primary ray (same arithmetic as CameraPolicy::load)
        const tim_rt_pass_data& pd = g.pd;
        const float fx = (float)gx, fy = (float)gy;
        const float swx = (pd.frustumCorner10[0] - pd.frustumCorner00[0]) * pd.invFrameSize[0];
        const float swy = (pd.frustumCorner10[1] - pd.frustumCorner00[1]) * pd.invFrameSize[0];
        const float swz = (pd.frustumCorner10[2] - pd.frustumCorner00[2]) * pd.invFrameSize[0];
        const float shx = (pd.frustumCorner01[0] - pd.frustumCorner00[0]) * pd.invFrameSize[1];
        const float shy = (pd.frustumCorner01[1] - pd.frustumCorner00[1]) * pd.invFrameSize[1];
        const float shz = (pd.frustumCorner01[2] - pd.frustumCorner00[2]) * pd.invFrameSize[1];
        const float tx = (pd.frustumCorner00[0] + swx * fx) + shx * fy;
        const float ty = (pd.frustumCorner00[1] + swy * fx) + shy * fy;
        const float tz = (pd.frustumCorner00[2] + swz * fx) + shz * fy;
        const float vx = tx - pd.cameraPos[0], vy = ty - pd.cameraPos[1], vz = tz - pd.cameraPos[2];
        const float len = sqrtf(dot3(vx, vy, vz, vx, vy, vz));
        const float dx = vx / len, dy = vy / len, dz = vz / len;
        // baseRaytracingPass.glsl:91 hitPos = from + dir * t
        const float hx = pd.cameraPos[0] + dx * t, hy = pd.cameraPos[1] + dy * t, hz = pd.cameraPos[2] + dz * t;
        // sun ray (tmax = TMAX)
        {
            tim_rt_ray& r = local[nr++];
            r.o[0] = hx; r.o[1] = hy; r.o[2] = hz; r.tmax = kTMax;
            r.d[0] = -pd.sunDir[0]; r.d[1] = -pd.sunDir[1]; r.d[2] = -pd.sunDir[2];
            r.flags = 1u | (0u << 8) | (0u << 16);
        }
        // light list
        const uint32_t* list;
        uint32_t count;
        if (g.flags & TIM_RT_CAM_TILE_LIGHTS) {
            const uint32_t tile = (gy / 16u) * g.tiles_x + gx / 16u;
            list = g.tile_lists + 16u * tile;
            count = min(g.tile_counts[tile], 16u);
        } else {
            const uint32_t nid = g.leaf_nid[pix];
            const uint32_t off = __ldg(reinterpret_cast<const uint32_t*>(s.nodes + 4u * nid) + 3);
            const uint32_t hdr = leaf_header(s, off);
            uint32_t skip = 3u * (hdr & ((1u << kTriBits) - 1u));
            skip += (hdr >> kTriBits) & ((1u << kBlasBits) - 1u);
            skip += (hdr >> (kTriBits + kBlasBits)) & ((1u << kPrimBits) - 1u);
            count = (hdr >> (kTriBits + kBlasBits + kPrimBits)) & ((1u << kLightBits) - 1u);
            list = s.leaf + skip + 1u + off;
        }
        for (uint32_t i = 0; i < count; ++i) {
            const uint32_t li = __ldg(list + i);
            const float* L = s.lights + 14u * li;
            if (__float_as_uint(__ldg(L)) != kLightSphere) continue;   // evalShadow returns false
            const float lx = __ldg(L + 1) - hx, ly = __ldg(L + 2) - hy, lz = __ldg(L + 3) - hz;
            const float radius = __ldg(L + 4);
            const float rl = sqrtf(dot3(lx, ly, lz, lx, ly, lz));
            const uint32_t bit = li + 1u;
            if (bit >= 32u) continue;   // the 32-bit mask has no bit for this light
            if (rl < radius) {
                tim_rt_ray& r = local[nr++];
                r.o[0] = hx; r.o[1] = hy; r.o[2] = hz; r.tmax = rl;
                r.d[0] = lx / rl; r.d[1] = ly / rl; r.d[2] = lz / rl;
                r.flags = 1u | (bit << 8) | (0u << 16);
            } else {
                direct_bits |= 1u << bit;
            }
        }
        if (g.flags & TIM_RT_CAM_PROB_MASK) {
            // lightprobHelpers.glsl:71-77 getLightProbCoordUVW and bvhLighting.glsl:170-180
            const uint32_t* res = pd.lpfResolution;
            const float stx = (pd.sceneMaxExtent[0] - pd.sceneMinExtent[0]) / (float)res[0];
            const float sty = (pd.sceneMaxExtent[1] - pd.sceneMinExtent[1]) / (float)res[1];
            const float stz = (pd.sceneMaxExtent[2] - pd.sceneMinExtent[2]) / (float)res[2];
            float ux = (hx - pd.sceneMinExtent[0]) / stx - 0.5f;
            float uy = (hy - pd.sceneMinExtent[1]) / sty - 0.5f;
            float uz = (hz - pd.sceneMinExtent[2]) / stz - 0.5f;
            ux = fminf(fmaxf(ux, 0.0f), (float)res[0] - 1.0f);
            uy = fminf(fmaxf(uy, 0.0f), (float)res[1] - 1.0f);
            uz = fminf(fmaxf(uz, 0.0f), (float)res[2] - 1.0f);
            const uint32_t ix = (uint32_t)(int32_t)ux, iy = (uint32_t)(int32_t)uy, iz = (uint32_t)(int32_t)uz;
            const uint32_t cx = min(ix, res[0] - 2u), cy = min(iy, res[1] - 2u), cz = min(iz, res[2] - 2u);
            for (uint32_t i = 0; i < 8u; ++i) {
                float qx, qy, qz;
                lpf_position(pd, cx + (i & 1u), cy + ((i >> 1) & 1u), cz + ((i >> 2) & 1u), qx, qy, qz);
                tim_rt_ray& r = local[nr++];
                r.o[0] = hx; r.o[1] = hy; r.o[2] = hz; r.tmax = 1.0f;
                r.d[0] = qx - hx; r.d[1] = qy - hy; r.d[2] = qz - hz;
                r.flags = 1u | (i << 8) | (1u << 16);
            }
        }
        if (g.flags & TIM_RT_CAM_BOUNCE) {
            // geometric normal of the hit triangle, facing the incoming ray
            const uint32_t i0 = rec.x + (rec.y & 0xFFFFu), i1 = rec.x + (rec.y >> 16), i2 = rec.x + (rec.z & 0xFFFFu);
            const float p0x = s.pos[3u * i0], p0y = s.pos[3u * i0 + 1], p0z = s.pos[3u * i0 + 2];
            const float e1x = s.pos[3u * i1] - p0x, e1y = s.pos[3u * i1 + 1] - p0y, e1z = s.pos[3u * i1 + 2] - p0z;
            const float e2x = s.pos[3u * i2] - p0x, e2y = s.pos[3u * i2 + 1] - p0y, e2z = s.pos[3u * i2 + 2] - p0z;
            float nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
            const float nl = sqrtf(dot3(nx, ny, nz, nx, ny, nz));
            nx = nx / nl; ny = ny / nl; nz = nz / nl;
            if (dot3(nx, ny, nz, dx, dy, dz) > 0.0f) { nx = -nx; ny = -ny; nz = -nz; }
            float bx, by, bz;
            bounce_dir(nx, ny, nz, pix, g.seed, bx, by, bz);
            tim_rt_ray& r = local[nr++];
            r.o[0] = hx; r.o[1] = hy; r.o[2] = hz; r.tmax = kTMax;
            r.d[0] = bx; r.d[1] = by; r.d[2] = bz;
            r.flags = 0u | (0u << 8) | (2u << 16);
        }
    }
    if (valid) {
        g.out_words[8u * pix + 4u] = direct_bits;
        g.out_words[8u * pix + 5u] = 0u;
        if (g.bounce_out) g.bounce_out[pix] = make_uint4(0u, 0u, 0u, 0u);
    }
    // warp-aggregated append into the secondary queue
    uint32_t incl = nr;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if ((int)lane >= o) incl += v;
    }
    const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    uint32_t base = 0;
    if (lane == 31u && total) base = atomicAdd(g.q_count, total);
    base = __shfl_sync(0xFFFFFFFFu, base, 31);
    const uint32_t my = base + incl - nr;
    for (uint32_t k = 0; k < nr; ++k) {
        const uint32_t slot = my + k;
        if (slot < g.q_capacity) {
            g.q_rays[slot] = local[k];
            g.q_pixel[slot] = pix;
        }
    }
}

// Clamp the queue count to its capacity (the generator sizes the queue for the
// worst case, so this only guards the trace kernel's bounds).
__global__ void k_clamp_count(uint32_t* q_count, uint32_t cap) {
    if (*q_count > cap) *q_count = cap;
}

// Adds the frame's ray count (primary rays of rows 1..H-1 plus the secondary queue).
__global__ void k_add_ray_count(uint64_t* dst, uint64_t primary, const uint32_t* q_count) {
    *dst += primary + *q_count;
}

// -------------------------------------------------------------------- tile light culling

// cullFrustum.glsl:9-13 computePlan
__device__ __forceinline__ void compute_plan(float p1x, float p1y, float p1z, float p2x, float p2y, float p2z,
                                             float p3x, float p3y, float p3z, float4& pl) {
    const float ax = p1x - p2x, ay = p1y - p2y, az = p1z - p2z;
    const float bx = p3x - p2x, by = p3y - p2y, bz = p3z - p2z;
    float nx = ay * bz - az * by, ny = az * bx - ax * bz, nz = ax * by - ay * bx;
    const float l = sqrtf(dot3(nx, ny, nz, nx, ny, nz));
    nx = nx / l; ny = ny / l; nz = nz / l;
    pl = make_float4(nx, ny, nz, -dot3(nx, ny, nz, p2x, p2y, p2z));
}

// One warp per tile: lanes test lights lane, lane+32, ...; survivors are
// compacted with a ballot in ascending light order (cullFrustum.glsl:63-100,136-151,
// collision.glsl:219-227).
__global__ void __launch_bounds__(256) k_cull_lights(SceneView s, tim_rt_pass_data pd, uint32_t tiles_x,
                                                     uint32_t tiles_y, uint32_t* counts, uint32_t* lists) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (warp >= tiles_x * tiles_y) return;
    const uint32_t wx = warp % tiles_x, wy = warp / tiles_x;
    const float* c00 = pd.frustumCorner00;
    const float* c10 = pd.frustumCorner10;
    const float* c01 = pd.frustumCorner01;
    const float sxx = (c10[0] - c00[0]) / (float)tiles_x, sxy = (c10[1] - c00[1]) / (float)tiles_x,
                sxz = (c10[2] - c00[2]) / (float)tiles_x;
    const float syx = (c01[0] - c00[0]) / (float)tiles_y, syy = (c01[1] - c00[1]) / (float)tiles_y,
                syz = (c01[2] - c00[2]) / (float)tiles_y;
    const float fx0 = (float)wx, fx1 = (float)(wx + 1u), fy0 = (float)wy, fy1 = (float)(wy + 1u);
    float blx = (c00[0] + sxx * fx0) + syx * fy0, bly = (c00[1] + sxy * fx0) + syy * fy0, blz = (c00[2] + sxz * fx0) + syz * fy0;
    float brx = (c00[0] + sxx * fx1) + syx * fy0, bry = (c00[1] + sxy * fx1) + syy * fy0, brz = (c00[2] + sxz * fx1) + syz * fy0;
    float tlx = (c00[0] + sxx * fx0) + syx * fy1, tly = (c00[1] + sxy * fx0) + syy * fy1, tlz = (c00[2] + sxz * fx0) + syz * fy1;
    float trx = (c00[0] + sxx * fx1) + syx * fy1, try_ = (c00[1] + sxy * fx1) + syy * fy1, trz = (c00[2] + sxz * fx1) + syz * fy1;
    const float dxx = sxx * 0.25f, dxy = sxy * 0.25f, dxz = sxz * 0.25f;
    const float dyx = syx * 0.25f, dyy = syy * 0.25f, dyz = syz * 0.25f;
    blx = (blx - dxx) - dyx; bly = (bly - dxy) - dyy; blz = (blz - dxz) - dyz;
    brx = (brx + dxx) - dyx; bry = (bry + dxy) - dyy; brz = (brz + dxz) - dyz;
    tlx = (tlx - dxx) + dyx; tly = (tly - dxy) + dyy; tlz = (tlz - dxz) + dyz;
    trx = (trx + dxx) + dyx; try_ = (try_ + dxy) + dyy; trz = (trz + dxz) + dyz;
    const float cx = pd.cameraPos[0], cy = pd.cameraPos[1], cz = pd.cameraPos[2];
    float4 pl[4];
    compute_plan(cx, cy, cz, tlx, tly, tlz, blx, bly, blz, pl[0]);
    compute_plan(cx, cy, cz, brx, bry, brz, trx, try_, trz, pl[1]);
    compute_plan(cx, cy, cz, trx, try_, trz, tlx, tly, tlz, pl[2]);
    compute_plan(cx, cy, cz, blx, bly, blz, brx, bry, brz, pl[3]);
    uint32_t cnt = 0;
    uint32_t* lst = lists + 16u * warp;
    for (uint32_t base = 0; base < s.num_lights && cnt < 16u; base += 32u) {
        const uint32_t i = base + lane;
        bool inside = false;
        if (i < s.num_lights) {
            const float* L = s.lights + 14u * i;
            const float px = __ldg(L + 1), py = __ldg(L + 2), pz = __ldg(L + 3), r = __ldg(L + 4);
            inside = true;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (dot3(pl[k].x, pl[k].y, pl[k].z, px, py, pz) + pl[k].w < -r) inside = false;
        }
        const uint32_t m = __ballot_sync(0xFFFFFFFFu, inside);
        const uint32_t pos = cnt + __popc(m & lanemask_lt());
        if (inside && pos < 16u) lst[pos] = i;
        cnt += __popc(m);
    }
    cnt = min(cnt, 16u);
    if (lane >= cnt && lane < 16u) lst[lane] = 0xFFFFFFFFu;
    if (lane == 0) counts[warp] = cnt;
}

// -------------------------------------------------------------------- launchers

template <int BLOCK, bool WIDE>
constexpr size_t stack_bytes() {
    return sizeof(uint32_t) * (WIDE ? 2 : 1) * kStackSize * BLOCK;
}

// Grid of the persistent kernels: as many resident blocks as the occupancy
// calculator allows on every SM (the dynamic shared memory holds the stacks).
template <int BLOCK, bool WIDE, bool STATS, class Policy>
static int grid_for() {
    static int blocks = 0;
    if (!blocks) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaFuncSetAttribute(k_persistent<BLOCK, WIDE, STATS, Policy>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)stack_bytes<BLOCK, WIDE>());
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_persistent<BLOCK, WIDE, STATS, Policy>, BLOCK,
                                                      stack_bytes<BLOCK, WIDE>());
        blocks = sms * (per > 0 ? per : 1);
    }
    return blocks;
}

template <int BLOCK, bool WIDE, bool STATS, class Policy>
static void launch_block(const SceneView& s, const Policy& P, uint32_t n_static, const uint32_t* n_dev,
                         uint32_t* counter, uint32_t* err, unsigned long long* stats, cudaStream_t stream) {
    k_persistent<BLOCK, WIDE, STATS, Policy>
        <<<grid_for<BLOCK, WIDE, STATS, Policy>(), BLOCK, stack_bytes<BLOCK, WIDE>(), stream>>>(s, P, n_static, n_dev,
                                                                                            counter, err, stats);
}

template <bool WIDE, class Policy>
static cudaError_t launch_persistent(const SceneView& s, const Policy& P, uint32_t n_static, const uint32_t* n_dev,
                                     uint32_t* counter, uint32_t* err, cudaStream_t stream, const LaunchConfig& cfg) {
    if (cfg.stats) {
        launch_block<128, WIDE, true>(s, P, n_static, n_dev, counter, err, cfg.stats, stream);
        return cudaGetLastError();
    }
    switch (cfg.block) {
        case 64: launch_block<64, WIDE, false>(s, P, n_static, n_dev, counter, err, nullptr, stream); break;
        case 256: launch_block<256, WIDE, false>(s, P, n_static, n_dev, counter, err, nullptr, stream); break;
        default: launch_block<128, WIDE, false>(s, P, n_static, n_dev, counter, err, nullptr, stream); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_trace_batch(const SceneView& s, const tim_rt_ray* rays, uint32_t n, uint32_t mode, uint32_t* hit,
                               uint32_t* nid, float* bary, uint32_t* counter, uint32_t* err, cudaStream_t stream,
                               const LaunchConfig& cfg) {
    BatchPolicy P{rays, reinterpret_cast<uint4*>(hit), nid, reinterpret_cast<float2*>(bary), mode & 0xFFu};
    if (cfg.wide) return launch_persistent<true>(s, P, n, nullptr, counter, err, stream, cfg);
    return launch_persistent<false>(s, P, n, nullptr, counter, err, stream, cfg);
}

cudaError_t launch_camera(const SceneView& s, const tim_rt_pass_data& pd, uint32_t flags, uint32_t seed,
                          const uint32_t* tile_counts, const uint32_t* tile_lists, uint32_t* out, uint32_t* bounce_out,
                          uint32_t* leaf_nid, tim_rt_ray* q_rays, uint32_t* q_pixel, uint32_t q_capacity,
                          uint32_t* counters, uint32_t* err, uint64_t* d_ray_count, cudaStream_t stream,
                          const LaunchConfig& cfg) {
    const uint32_t W = pd.frameSize[0], H = pd.frameSize[1];
    const uint32_t npix = W * H;
    const uint32_t ngy16 = 16u * ((H + 15u) / 16u);
    CameraPolicy CP{pd, ngy16, reinterpret_cast<uint4*>(out), leaf_nid};
    if (cfg.phase_ev) cudaEventRecord(cfg.phase_ev[0], stream);
    cudaError_t e = cfg.wide ? launch_persistent<true>(s, CP, npix, nullptr, counters + 0, err, stream, cfg)
                             : launch_persistent<false>(s, CP, npix, nullptr, counters + 0, err, stream, cfg);
    if (e != cudaSuccess) return e;
    if (cfg.phase_ev) cudaEventRecord(cfg.phase_ev[1], stream);
    GenParams g;
    g.pd = pd;
    g.flags = flags;
    g.seed = seed;
    g.ngy16 = ngy16;
    g.tiles_x = (W + 15u) / 16u;
    g.tile_counts = tile_counts;
    g.tile_lists = tile_lists;
    g.out_words = out;
    g.leaf_nid = leaf_nid;
    g.bounce_out = reinterpret_cast<uint4*>(bounce_out);
    g.q_rays = q_rays;
    g.q_pixel = q_pixel;
    g.q_count = counters + 1;
    g.q_capacity = q_capacity;
    k_gen_secondary<<<(npix + 255u) / 256u, 256, 0, stream>>>(s, g);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_clamp_count<<<1, 1, 0, stream>>>(counters + 1, q_capacity);
    if (cfg.phase_ev) cudaEventRecord(cfg.phase_ev[2], stream);
    SecondaryPolicy SP{q_rays, q_pixel, out, reinterpret_cast<uint4*>(bounce_out)};
    e = cfg.wide ? launch_persistent<true>(s, SP, 0u, counters + 1, counters + 2, err, stream, cfg)
                 : launch_persistent<false>(s, SP, 0u, counters + 1, counters + 2, err, stream, cfg);
    if (cfg.phase_ev) cudaEventRecord(cfg.phase_ev[3], stream);
    if (e != cudaSuccess || !d_ray_count) return e;
    k_add_ray_count<<<1, 1, 0, stream>>>(d_ray_count, (uint64_t)W * (H - 1u), counters + 1);
    return cudaGetLastError();
}

cudaError_t launch_cull_lights(const SceneView& s, const tim_rt_pass_data& pd, uint32_t tiles_x, uint32_t tiles_y,
                               uint32_t* counts, uint32_t* lists, cudaStream_t stream) {
    const uint32_t warps = tiles_x * tiles_y;
    const uint32_t blocks = (warps * 32u + 255u) / 256u;
    k_cull_lights<<<blocks, 256, 0, stream>>>(s, pd, tiles_x, tiles_y, counts, lists);
    return cudaGetLastError();
}

}  // namespace timrt
