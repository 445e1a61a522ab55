// trace.cu -- persistent ray-tracing kernels for sm_100a and their launchers.
//
// Every trace kernel here is the same persistent loop: a grid sized to fill
// the GPU (blocks per SM from the occupancy calculator x 148 SMs), in which
// each warp keeps all 32 lanes busy by refilling finished lanes with new work
// items from a global atomic counter (one atomicAdd per refill, issued by one
// elected lane). A policy object turns a work item into a ray (load) and
// writes the result (store): plain ray batches, camera pixels, secondary
// (shadow / probe-visibility / bounce) rays.
//
// Coherence: camera work items walk the frame in 8x4-pixel tiles (32 pixels =
// one warp), and the secondary rays of those pixels are queued by kind -- sun,
// tile-light slot j, probe corner i, bounce -- in one segment per kind, so a
// warp traces 32 rays of the same kind from neighbouring pixels.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cstdio>
#include "common.cuh"
#include "trace_plain.cuh"
#include "trace_wide.cuh"
#include "kernels.h"
#include "../../include/tim_rt.h"

namespace timrt {

// Secondary-ray kinds, one queue segment each.
constexpr uint32_t kKindSun = 0, kKindLight0 = 1, kKindProbe0 = 17, kKindBounce = 25, kNumKinds = 26;

// The secondary queue split into bands of output rows (one band unless a camera
// trace is pipelined): band b's rays of kind k take cap[b] slots from
// base[b] + k * cap[b]; its counts and prefix entries are b * kNumKinds + k.
struct QueueBands {
    uint32_t n;
    uint32_t row[kMaxCamBands + 1];   // band b: output rows [row[b], row[b + 1])
    uint32_t base[kMaxCamBands];
    uint32_t cap[kMaxCamBands];
};

__device__ __forceinline__ uint32_t band_of_row(const QueueBands& q, uint32_t r) {
    uint32_t b = 0;
    for (uint32_t k = 1; k < q.n; ++k) b += r >= q.row[k] ? 1u : 0u;
    return b;
}

// Work item -> pixel in 8x4 tiles (row-major tiles over the frame).
__device__ __forceinline__ bool tile_pixel(uint32_t i, uint32_t W, uint32_t H, uint32_t& px, uint32_t& py) {
    const uint32_t tiles_x = (W + 7u) >> 3;
    const uint32_t tile = i >> 5, within = i & 31u;
    px = (tile % tiles_x) * 8u + (within & 7u);
    py = (tile / tiles_x) * 4u + (within >> 3);
    return px < W && py < H;
}

__host__ __device__ __forceinline__ uint32_t tiled_work_items(uint32_t W, uint32_t H) {
    return ((W + 7u) >> 3) * ((H + 3u) >> 2) * 32u;
}

// -------------------------------------------------------------------- policies

// The leaf kind a policy's rays take (kLeafOne unless the policy says otherwise).
template <class P, class = void>
struct leaf_kind { static constexpr int value = kLeafOne; };
template <class P>
struct leaf_kind<P, decltype((void)P::kLeaf)> { static constexpr int value = P::kLeaf; };
// Whether a policy wants its finished() hook called by the whole warp after each
// round of stores.
template <class P, class = void>
struct finishes { static constexpr bool value = false; };
template <class P>
struct finishes<P, decltype((void)P::kFinishes)> { static constexpr bool value = P::kFinishes; };

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
        st.dup_ok = nid == nullptr;
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

// Any-hit rays of a two-level scene (TIM_RT_TRACE_TLAS): traverseTlasFast
// (bvhTraversal_inline.glsl:83-151 with TLAS_COLLIDE) from the scene root.
struct TlasBatchPolicy : BatchPolicy {
    static constexpr int kLeaf = kLeafTlasTop;
};

// cameraPass.comp:44-76 pinhole ray of invocation (gx, gy) (cameraPass.comp:50-54).
__device__ __forceinline__ void camera_ray(const tim_rt_pass_data& pd, uint32_t gx, uint32_t gy, float& dx, float& dy,
                                           float& dz) {
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
    const float len = sqrtf(dot3(vx, vy, vz, vx, vy, vz));   // normalize(v) = v / sqrt(dot(v, v))
    dx = vx / len;
    dy = vy / len;
    dz = vz / len;
}

// One work item per pixel, tile order. Output row py is traced by invocation
// gy = 16*ceil(H/16) - py (cameraPass.comp:46), so row 0 is never traced.
struct CameraPolicy {
    tim_rt_pass_data pd;
    uint32_t ngy16;         // 16 * ceil(H / 16)
    uint4* out;             // 2 x uint4 per pixel
    uint32_t* leaf_nid;     // per pixel, for the leaf-light shadow mask
    uint32_t item0;         // first work item (8x4-pixel tile order) of this launch

    __device__ __forceinline__ bool load(const SceneView&, uint32_t i, TravState& st) const {
        uint32_t px, py;
        if (!tile_pixel(item0 + i, pd.frameSize[0], pd.frameSize[1], px, py) || py == 0u) return false;
        st.slot = py * pd.frameSize[0] + px;
        camera_ray(pd, px, ngy16 - py, st.r.dx, st.r.dy, st.r.dz);
        st.r.ox = pd.cameraPos[0]; st.r.oy = pd.cameraPos[1]; st.r.oz = pd.cameraPos[2];
        st.t = kTMax;
        st.any = false;
        st.dup_ok = false;   // the hit leaf's light list feeds the shadow rays
        return true;
    }
    __device__ __forceinline__ void store(const SceneView&, uint32_t, const TravState& st, float) const {
        const uint32_t pix = st.slot;
        out[2u * pix] = make_uint4(st.rec0, st.rec1, st.rec2, __float_as_uint(st.t));
        out[2u * pix + 1u] = make_uint4(0u, 0u, 0u, 0u);
        leaf_nid[pix] = st.hit ? st.nid : 0xFFFFFFFFu;
    }
    __device__ __forceinline__ void skip(uint32_t i) const {
        uint32_t px, py;
        if (!tile_pixel(item0 + i, pd.frameSize[0], pd.frameSize[1], px, py)) return;
        const uint32_t pix = py * pd.frameSize[0] + px;
        out[2u * pix] = make_uint4(0u, 0u, 0u, 0u);
        out[2u * pix + 1u] = make_uint4(0u, 0u, 0u, 0u);
        leaf_nid[pix] = 0xFFFFFFFFu;
    }
};

// Secondary rays queued by band and kind (QueueBands); prefix[b * kNumKinds + k] is
// the first work item of band b's kind k and prefix[n * kNumKinds] the total, so
// work items run band by band. ray.flags: bit 0 any-hit, bits 8..15 the mask
// bit, bits 16..17 the output (0 shadow mask, 1 probe mask, 2 bounce record).
// With done / flags (a pipelined camera trace), finished rays are counted per
// band and flags[b] is set once all of band b's rays are stored.
struct SecondaryPolicy {
    static constexpr bool kFinishes = true;
    const tim_rt_ray* rays;
    const uint32_t* pixel;
    const uint32_t* prefix;
    QueueBands qb;
    uint32_t* out_words;    // tracingData as u32 words (8 per pixel)
    uint4* bounce_out;
    uint32_t* done;         // finished rays per band, or null
    volatile uint32_t* flags;

    __device__ __forceinline__ bool load(const SceneView&, uint32_t i, TravState& st) const {
        uint32_t lo = 0, hi = qb.n * kNumKinds;   // largest segment k with prefix[k] <= i
        while (hi - lo > 1u) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(prefix + mid) <= i) lo = mid;
            else hi = mid;
        }
        const uint32_t band = lo / kNumKinds, kind = lo - band * kNumKinds;
        const uint32_t slot = qb.base[band] + kind * qb.cap[band] + (i - __ldg(prefix + lo));
        st.slot = slot;
        const float4* rp = reinterpret_cast<const float4*>(rays + slot);
        const float4 a = __ldg(rp), b = __ldg(rp + 1);
        st.r.ox = a.x; st.r.oy = a.y; st.r.oz = a.z;
        st.r.dx = b.x; st.r.dy = b.y; st.r.dz = b.z;
        st.t = a.w;
        st.any = (__float_as_uint(b.w) & 1u) != 0u;
        st.dup_ok = true;   // bounce rays store the hit record only
        st.slot2 = __ldg(pixel + slot);   // read now, used when the ray is stored
        return true;
    }
    // Called by all 32 lanes after a round of stores (`stored`: this lane stored
    // the ray in queue slot `slot`): one count per band and warp, after each
    // storing lane's release fence; the count that completes a band follows every
    // other count of the band in the counter's order, and raises the band's flag
    // after a system-scope fence.
    __device__ __forceinline__ void finished(bool stored, uint32_t slot) const {
        if (!done) return;
        uint32_t band = 0xFFFFFFFFu;
        if (stored) {
            band = 0;
            for (uint32_t k = 1; k < qb.n; ++k) band += slot >= qb.base[k] ? 1u : 0u;
            asm volatile("fence.acq_rel.gpu;" ::: "memory");   // this lane's stores before the warp's count
        }
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, band);
        __syncwarp();
        const uint32_t lane = threadIdx.x & 31u;
        if (stored && lane == (uint32_t)(__ffs(peers) - 1)) {
            const uint32_t total = __ldg(prefix + (band + 1u) * kNumKinds) - __ldg(prefix + band * kNumKinds);
            const uint32_t cnt = (uint32_t)__popc(peers);
            if (atomicAdd(done + band, cnt) + cnt == total) {
                __threadfence_system();
                flags[band] = 1u;
            }
        }
    }
    __device__ __forceinline__ void store(const SceneView&, uint32_t, const TravState& st, float) const {
        const uint32_t slot = st.slot;
        const uint32_t fl = __float_as_uint(__ldg(reinterpret_cast<const float*>(rays + slot) + 7));
        const uint32_t kind = (fl >> 16) & 3u, bit = (fl >> 8) & 0xFFu;
        const uint32_t p = st.slot2;
        if (kind == 2u) {
            bounce_out[p] = make_uint4(st.rec0, st.rec1, st.rec2, __float_as_uint(st.t));
        } else if (st.hit) {
            atomicOr(out_words + 8u * p + 4u + kind, 1u << bit);
        }
    }
    __device__ __forceinline__ void skip(uint32_t) const {}
};

// -------------------------------------------------------------------- persistent loop

// sdepth: traversal-stack entries per thread (the tree depth; <= 32). The stack
// lives in dynamic shared memory, entry k of thread t at [k * BLOCK + t]
// (binary form) or [(2k, 2k+1) * BLOCK + t] (8-wide form).
template <int BLOCK, bool WIDE, bool STATS, class Policy>
__global__ void __launch_bounds__(BLOCK, WIDE ? 896 / BLOCK : 1024 / BLOCK) k_persistent(SceneView s, Policy P, uint32_t n_static,
                                                      const uint32_t* n_dev, uint32_t* counter, uint32_t* err,
                                                      unsigned long long* stats, int sdepth, int knobs) {
    extern __shared__ uint32_t stack_mem[];
    // knobs: refill threshold (bits 0..7), phase-switch threshold (bits 8..15)
    const int refill_min = knobs & 0xFF;
    const uint32_t phase_sw = (uint32_t)(knobs >> 8) & 0xFFu;
    uint32_t* stk = stack_mem + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t n = n_dev ? *n_dev : n_static;
    const uint32_t root = s.num_nodes == 1u ? kNidLeafBit : 0u;   // baseRaytracingPass.glsl:20

    TravState st;
    st.done = true;
    // active: a ray is being traversed; pending: its traversal ended and its
    // result waits to be finished (8-wide proof) and stored. Pending lanes are
    // finished together when the warp refills, so that end-of-ray work runs
    // converged instead of once per lane as lanes end at different steps.
    bool active = false, pending = false, exhausted = false;
    uint32_t idx = 0;
    for (;;) {
        const uint32_t idle = __ballot_sync(0xFFFFFFFFu, !active);
        // refill once at least refill_min lanes are idle (32: whole-warp
        // batches, which keeps coherent rays of a batch in lockstep); after the
        // last ray was handed out, finish pending lanes as they come
        if (idle && (exhausted || __popc(idle) >= refill_min || idle == 0xFFFFFFFFu)) {
            const bool stored = pending;
            if (pending) {
                pending = false;
                if (WIDE) wide_finish_or_walk(s, st, err);
                P.store(s, idx, st, st.t0);
                if (STATS) {
                    atomicAdd(stats + 0, 1ull);
                    atomicAdd(stats + 1, (unsigned long long)st.c_node);
                    atomicAdd(stats + 2, (unsigned long long)st.c_leaf);
                    atomicAdd(stats + 3, (unsigned long long)st.c_tri);
                    atomicAdd(stats + 4, (unsigned long long)st.c_reload);
                }
            }
            if constexpr (finishes<Policy>::value) P.finished(stored, st.slot);
            if (!exhausted) {
                const uint32_t need = __ballot_sync(0xFFFFFFFFu, !active);
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
                            st.t0 = st.t;
                            st.err = err;
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
        if (__ballot_sync(0xFFFFFFFFu, active || pending) == 0u) {
            if (exhausted) break;
            continue;
        }
        if (WIDE) {
            wide_step_warp<BLOCK>(s, st, active, stk, err, sdepth, phase_sw);   // all lanes: warp-synchronous step
        } else {
            plain_step_warp<BLOCK, leaf_kind<Policy>::value>(s, st, active, stk, err, sdepth, phase_sw);
        }
        if (active && st.done) {
            active = false;
            pending = true;
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
    uint32_t* q_counts;     // counters [band][kind]
    QueueBands qb;
    uint32_t item0, item1;  // work items (8x4-pixel tile order) of this launch
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

// Appends one ray of `kind` to the warp's band (uniform across the warp) for the
// lanes with has == true: warp-aggregated atomic on the band's kind counter,
// lane order preserved inside the segment.
__device__ __forceinline__ void emit(const GenParams& g, uint32_t band, uint32_t kind, bool has, uint32_t pix,
                                     float ox, float oy, float oz, float tmax, float dx, float dy, float dz,
                                     uint32_t flags) {
    const uint32_t m = __ballot_sync(0xFFFFFFFFu, has);
    if (!m) return;
    const uint32_t lane = threadIdx.x & 31u;
    const int leader = __ffs(m) - 1;
    uint32_t base = 0;
    if ((int)lane == leader) base = atomicAdd(g.q_counts + band * kNumKinds + kind, (uint32_t)__popc(m));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    if (has) {
        const uint32_t off = base + __popc(m & lanemask_lt());
        const uint32_t cap = g.qb.cap[band];
        if (off < cap) {
            const uint64_t slot = (uint64_t)g.qb.base[band] + (uint64_t)kind * cap + off;
            float4* rp = reinterpret_cast<float4*>(g.q_rays + slot);
            rp[0] = make_float4(ox, oy, oz, tmax);
            rp[1] = make_float4(dx, dy, dz, __uint_as_float(flags));
            g.q_pixel[slot] = pix;
        }
    }
}

// For each camera hit, emit the rays of computeAdditionalHitData
// (baseRaytracingPass.glsl:85-97): the sun shadow ray and one ray per light of
// the hit leaf's list (bvhLighting.glsl:143-163) or of the pixel's tile list,
// the 8 probe-visibility segments (bvhLighting.glsl:165-184) and the bounce.
// Lights out of range set their bit directly (evalShadow returns true,
// bvhLighting.glsl:121-124). One thread per pixel, pixels in 8x4 tiles.
__global__ void __launch_bounds__(256) k_gen_secondary(SceneView s, GenParams g) {
    const tim_rt_pass_data& pd = g.pd;
    const uint32_t W = pd.frameSize[0], H = pd.frameSize[1];
    const uint32_t i = g.item0 + blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t px = 0, py = 0;
    const bool valid = i < g.item1 && tile_pixel(i, W, H, px, py);
    const uint32_t pix = py * W + px;
    // the warp's band: all its pixels lie in one 8x4 tile, bands end on tile rows
    const uint32_t band = band_of_row(g.qb, (i >> 5) / ((W + 7u) >> 3) * 4u);
    uint4 rec = make_uint4(0, 0, 0, 0);
    if (valid) rec = reinterpret_cast<const uint4*>(g.out_words)[2u * pix];
    const float t = __uint_as_float(rec.w);
    const bool hit = valid && py != 0u && t < kTMax;
    const uint32_t gx = px, gy = g.ngy16 - py;
    float dx = 0.f, dy = 0.f, dz = 0.f, hx = 0.f, hy = 0.f, hz = 0.f;
    if (hit) {
        camera_ray(pd, gx, gy, dx, dy, dz);
        // baseRaytracingPass.glsl:91 hitPos = from + dir * t
        hx = pd.cameraPos[0] + dx * t;
        hy = pd.cameraPos[1] + dy * t;
        hz = pd.cameraPos[2] + dz * t;
    }
    // sun ray, tmax = TMAX (bvhLighting.glsl:148-149)
    emit(g, band, kKindSun, hit, pix, hx, hy, hz, kTMax, -pd.sunDir[0], -pd.sunDir[1], -pd.sunDir[2], 1u);
    // light list of the tile or of the hit leaf
    const uint32_t* list = nullptr;
    uint32_t count = 0;
    if (hit) {
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
    }
    uint32_t direct_bits = 0;
    // lights past every lane's count emit nothing: the loop ends at the warp's
    // largest count (one 16x16 tile's list with tile lists, so usually uniform)
    const uint32_t jmax = __reduce_max_sync(0xFFFFFFFFu, count);
    for (uint32_t j = 0; j < jmax; ++j) {
        bool has = false;
        float rl = 1.f, dlx = 0.f, dly = 0.f, dlz = 0.f;
        uint32_t bit = 0;
        if (j < count) {
            const uint32_t li = __ldg(list + j);
            const float* L = s.lights + 14u * li;
            bit = li + 1u;
            if (__float_as_uint(__ldg(L)) == kLightSphere && bit < 32u) {   // evalShadow: sphere lights only
                const float lx = __ldg(L + 1) - hx;
                const float ly = __ldg(L + 2) - hy;
                const float lz = __ldg(L + 3) - hz;
                rl = sqrtf(dot3(lx, ly, lz, lx, ly, lz));
                if (rl < __ldg(L + 4)) {
                    has = true;
                    dlx = lx / rl;
                    dly = ly / rl;
                    dlz = lz / rl;
                } else {
                    direct_bits |= 1u << bit;   // out of range counts as masked
                }
            }
        }
        emit(g, band, kKindLight0 + j, has, pix, hx, hy, hz, rl, dlx, dly, dlz, 1u | (bit << 8));
    }
    if (g.flags & TIM_RT_CAM_PROB_MASK) {
        // lightprobHelpers.glsl:71-77 getLightProbCoordUVW and bvhLighting.glsl:170-180
        uint32_t cx = 0, cy = 0, cz = 0;
        if (hit) {
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
            cx = min(ix, res[0] - 2u);
            cy = min(iy, res[1] - 2u);
            cz = min(iz, res[2] - 2u);
        }
        for (uint32_t k = 0; k < 8u; ++k) {
            float qx = 0.f, qy = 0.f, qz = 0.f;
            if (hit) lpf_position(pd, cx + (k & 1u), cy + ((k >> 1) & 1u), cz + ((k >> 2) & 1u), qx, qy, qz);
            emit(g, band, kKindProbe0 + k, hit, pix, hx, hy, hz, 1.0f, qx - hx, qy - hy, qz - hz,
                 1u | (k << 8) | (1u << 16));
        }
    }
    if (g.flags & TIM_RT_CAM_BOUNCE) {
        float bx = 0.f, by = 0.f, bz = 0.f;
        if (hit) {
            // geometric normal of the hit triangle, facing the incoming ray
            const uint32_t i0 = rec.x + (rec.y & 0xFFFFu), i1 = rec.x + (rec.y >> 16), i2 = rec.x + (rec.z & 0xFFFFu);
            const float p0x = s.pos[3u * i0], p0y = s.pos[3u * i0 + 1], p0z = s.pos[3u * i0 + 2];
            const float e1x = s.pos[3u * i1] - p0x, e1y = s.pos[3u * i1 + 1] - p0y, e1z = s.pos[3u * i1 + 2] - p0z;
            const float e2x = s.pos[3u * i2] - p0x, e2y = s.pos[3u * i2 + 1] - p0y, e2z = s.pos[3u * i2 + 2] - p0z;
            float nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
            const float nl = sqrtf(dot3(nx, ny, nz, nx, ny, nz));
            nx = nx / nl; ny = ny / nl; nz = nz / nl;
            if (dot3(nx, ny, nz, dx, dy, dz) > 0.0f) { nx = -nx; ny = -ny; nz = -nz; }
            bounce_dir(nx, ny, nz, pix, g.seed, bx, by, bz);
        }
        emit(g, band, kKindBounce, hit, pix, hx, hy, hz, kTMax, bx, by, bz, 2u << 16);
    }
    if (valid) {
        g.out_words[8u * pix + 4u] = direct_bits;
        g.out_words[8u * pix + 5u] = 0u;
        if (g.bounce_out) g.bounce_out[pix] = make_uint4(0u, 0u, 0u, 0u);
    }
}

// prefix[b * kNumKinds + k] = first work item of band b's kind k over the
// (capacity-clamped) segment counts. A band without secondary rays is final
// already: its flag (when there are flags) is raised here.
__global__ void k_kind_prefix(const uint32_t* q_counts, uint32_t* prefix, QueueBands qb, volatile uint32_t* flags) {
    uint32_t acc = 0;
    for (uint32_t b = 0; b < qb.n; ++b) {
        const uint32_t first = acc;
        for (uint32_t k = 0; k < kNumKinds; ++k) {
            prefix[b * kNumKinds + k] = acc;
            acc += min(q_counts[b * kNumKinds + k], qb.cap[b]);
        }
        if (flags && acc == first) {
            __threadfence_system();
            flags[b] = 1u;
        }
    }
    prefix[qb.n * kNumKinds] = acc;
}

// Adds the frame's ray count (primary rays of rows 1..H-1 plus the secondary queue).
__global__ void k_add_ray_count(uint64_t* dst, uint64_t primary, const uint32_t* total) {
    *dst += primary + *total;
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
constexpr size_t stack_bytes(int depth) {
    return sizeof(uint32_t) * (size_t)depth * BLOCK;   // one word per entry in both forms
}

// Grid of the persistent kernels: as many resident blocks as the occupancy
// calculator allows on every SM for this stack depth (cached per device and depth).
template <int BLOCK, bool WIDE, bool STATS, class Policy>
static int grid_for(int depth) {
    static GridCache cache;
    return cache.get(depth, [depth](int dev) {
        int sms = 0, per = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaFuncSetAttribute(k_persistent<BLOCK, WIDE, STATS, Policy>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)stack_bytes<BLOCK, WIDE>(kStackSize));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_persistent<BLOCK, WIDE, STATS, Policy>, BLOCK,
                                                      stack_bytes<BLOCK, WIDE>(depth));
        return (sms > 0 ? sms : 1) * (per > 0 ? per : 1);
    });
}

template <int BLOCK, bool WIDE, bool STATS, class Policy>
static void launch_block(const SceneView& s, const Policy& P, uint32_t n_static, const uint32_t* n_dev,
                         uint32_t* counter, uint32_t* err, unsigned long long* stats, int depth, int refill,
                         cudaStream_t stream) {
    k_persistent<BLOCK, WIDE, STATS, Policy><<<grid_for<BLOCK, WIDE, STATS, Policy>(depth), BLOCK,
                                               stack_bytes<BLOCK, WIDE>(depth), stream>>>(s, P, n_static, n_dev,
                                                                                          counter, err, stats, depth,
                                                                                          refill);
}

template <bool WIDE, class Policy>
static cudaError_t launch_persistent(const SceneView& s, const Policy& P, uint32_t n_static, const uint32_t* n_dev,
                                     uint32_t* counter, uint32_t* err, cudaStream_t stream, const LaunchConfig& cfg) {
    int depth = WIDE ? (int)s.wide_depth : (int)s.depth;
    if (cfg.stack_depth > depth) depth = cfg.stack_depth;
    depth = depth < 1 ? 1 : (depth > kStackSize ? kStackSize : depth);
    const int refill = launch_knobs(cfg);
    if (cfg.stats) {
        launch_block<128, WIDE, true>(s, P, n_static, n_dev, counter, err, cfg.stats, depth, refill, stream);
        return cudaGetLastError();
    }
    switch (cfg.block) {
        case 64: launch_block<64, WIDE, false>(s, P, n_static, n_dev, counter, err, nullptr, depth, refill, stream); break;
        case 256: launch_block<256, WIDE, false>(s, P, n_static, n_dev, counter, err, nullptr, depth, refill, stream); break;
        default: launch_block<128, WIDE, false>(s, P, n_static, n_dev, counter, err, nullptr, depth, refill, stream); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_trace_batch(const SceneView& s, const tim_rt_ray* rays, uint32_t n, uint32_t mode, uint32_t* hit,
                               uint32_t* nid, float* bary, uint32_t* counter, uint32_t* err, cudaStream_t stream,
                               const LaunchConfig& cfg) {
    BatchPolicy P{rays, reinterpret_cast<uint4*>(hit), nid, reinterpret_cast<float2*>(bary), mode & 0xFFu};
    if (mode & TIM_RT_TRACE_TLAS) {   // any-hit only, binary form only (checked by the callers)
        TlasBatchPolicy T;
        static_cast<BatchPolicy&>(T) = P;
        return launch_persistent<false>(s, T, n, nullptr, counter, err, stream, cfg);
    }
    if (cfg.wide) return launch_persistent<true>(s, P, n, nullptr, counter, err, stream, cfg);
    return launch_persistent<false>(s, P, n, nullptr, counter, err, stream, cfg);
}

uint32_t camera_queue_segment(uint32_t W, uint32_t H) { return W * H; }
uint32_t camera_queue_kinds() { return kNumKinds; }
uint32_t probe_queue_kinds() { return kKindProbe0; }

cudaError_t launch_camera(const SceneView& s, const tim_rt_pass_data& pd, uint32_t flags, uint32_t seed,
                          const uint32_t* tile_counts, const uint32_t* tile_lists, uint32_t* out, uint32_t* bounce_out,
                          uint32_t* leaf_nid, tim_rt_ray* q_rays, uint32_t* q_pixel, uint32_t seg_cap,
                          uint32_t* counters, uint32_t* err, uint64_t* d_ray_count, cudaStream_t stream,
                          const LaunchConfig& cfg, uint32_t row_begin, uint32_t row_end, const CameraBands* bands) {
    const uint32_t W = pd.frameSize[0], H = pd.frameSize[1];
    // output rows [row_begin, row_end): whole rows of 8x4-pixel tiles (row_begin a multiple of 4)
    row_end = min(row_end, H);
    if (row_begin >= row_end) return cudaSuccess;
    // the queue's bands: one (the launch's rows, segments of seg_cap slots), or the
    // caller's bands of the whole frame (segments of each band's pixels)
    QueueBands qb{};
    qb.n = 1;
    qb.row[0] = row_begin;
    qb.row[1] = row_end;
    qb.cap[0] = seg_cap;
    if (bands && bands->n > 1u) {
        if (bands->n > kMaxCamBands || row_begin != 0u || row_end != H || seg_cap != W * H) return cudaErrorInvalidValue;
        qb.n = bands->n;
        for (uint32_t b = 0; b <= qb.n; ++b) qb.row[b] = bands->row[b];
        if (qb.row[0] != 0u || qb.row[qb.n] != H) return cudaErrorInvalidValue;
        for (uint32_t b = 0; b < qb.n; ++b) {
            if (qb.row[b + 1] <= qb.row[b] || qb.row[b] % 4u != 0u) return cudaErrorInvalidValue;
            qb.base[b] = kNumKinds * W * qb.row[b];
            qb.cap[b] = W * (qb.row[b + 1] - qb.row[b]);
        }
    }
    volatile uint32_t* flags_host = bands && bands->n > 1u ? bands->flags : nullptr;
    const uint32_t tiles_x = (W + 7u) >> 3;
    const uint32_t item0 = (row_begin >> 2) * tiles_x * 32u;
    const uint32_t item1 = min(tiled_work_items(W, H), ((row_end + 3u) >> 2) * tiles_x * 32u);
    const uint32_t items = item1 - item0;
    const uint32_t ngy16 = 16u * ((H + 15u) / 16u);
    // counters: [0] pixel work, [1] secondary work, then the bands' kind counts, their
    // prefix and the bands' finished rays
    uint32_t* q_counts = counters + 2;
    uint32_t* prefix = counters + 2 + kNumKinds * qb.n;
    uint32_t* done = prefix + kNumKinds * qb.n + 1u;
    CameraPolicy CP{pd, ngy16, reinterpret_cast<uint4*>(out), leaf_nid, item0};
    if (cfg.phase_ev) cudaEventRecord(cfg.phase_ev[0], stream);
    // primary rays: a warp refills only when all 32 lanes are idle, so it always
    // traces one whole 8x4-pixel tile together (measured fastest for these
    // coherent rays; the secondary launch keeps the configured threshold)
    LaunchConfig pcfg = cfg;
    pcfg.refill_min = 32;
    if (flags & TIM_RT_CAM_PRIMARY_BINARY) pcfg.wide = false;
    cudaError_t e = pcfg.wide ? launch_persistent<true>(s, CP, items, nullptr, counters + 0, err, stream, pcfg)
                              : launch_persistent<false>(s, CP, items, nullptr, counters + 0, err, stream, pcfg);
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
    g.q_counts = q_counts;
    g.qb = qb;
    g.item0 = item0;
    g.item1 = item1;
    k_gen_secondary<<<(items + 255u) / 256u, 256, 0, stream>>>(s, g);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_kind_prefix<<<1, 1, 0, stream>>>(q_counts, prefix, qb, flags_host);
    if (cfg.phase_ev) cudaEventRecord(cfg.phase_ev[2], stream);
    SecondaryPolicy SP{q_rays, q_pixel, prefix, qb, out, reinterpret_cast<uint4*>(bounce_out),
                       flags_host ? done : nullptr, flags_host};
    LaunchConfig cfg2 = cfg;   // the secondary kernel counts into stats[8..12]
    if (cfg.stats) cfg2.stats = cfg.stats + 8;
    const uint32_t* total = prefix + kNumKinds * qb.n;
    e = cfg.wide ? launch_persistent<true>(s, SP, 0u, total, counters + 1, err, stream, cfg2)
                 : launch_persistent<false>(s, SP, 0u, total, counters + 1, err, stream, cfg2);
    if (cfg.phase_ev) cudaEventRecord(cfg.phase_ev[3], stream);
    if (e != cudaSuccess || !d_ray_count) return e;
    // primary rays of the rows traced (output row 0 is never traced)
    const uint64_t primary = (uint64_t)W * (row_end - max(row_begin, 1u));
    k_add_ray_count<<<1, 1, 0, stream>>>(d_ray_count, primary, total);
    return cudaGetLastError();
}

cudaError_t launch_cull_lights(const SceneView& s, const tim_rt_pass_data& pd, uint32_t tiles_x, uint32_t tiles_y,
                               uint32_t* counts, uint32_t* lists, cudaStream_t stream) {
    const uint32_t warps = tiles_x * tiles_y;
    const uint32_t blocks = (warps * 32u + 255u) / 256u;
    k_cull_lights<<<blocks, 256, 0, stream>>>(s, pd, tiles_x, tiles_y, counts, lists);
    return cudaGetLastError();
}

// -------------------------------------------------------------------- light-probe field

// lightprobHelpers.glsl:33-61 getLightProbCoord (LP_TILE_RES = 4)
__device__ __forceinline__ void probe_coord(uint32_t index, const uint32_t* res, uint32_t& x, uint32_t& y, uint32_t& z) {
    const uint32_t trx = res[0] / 4u, try_ = res[1] / 4u;
    uint32_t tile = index / 64u;
    const uint32_t in = index % 64u;
    z = tile / (trx * try_);
    tile = tile % (trx * try_);
    y = tile / trx;
    x = tile % trx;
    x = x * 4u + in % 4u;
    y = y * 4u + (in / 4u) % 4u;
    z = z * 4u + (in / 16u) % 4u;
}

// lightprobHelpers.glsl:63-69 getLightProbPosition
__device__ __forceinline__ void probe_position(const ProbeArgs& d, uint32_t p, float& x, float& y, float& z) {
    uint32_t cx, cy, cz;
    probe_coord(p, d.res, cx, cy, cz);
    const float stx = (d.mx[0] - d.mn[0]) / (float)d.res[0];
    const float sty = (d.mx[1] - d.mn[1]) / (float)d.res[1];
    const float stz = (d.mx[2] - d.mn[2]) / (float)d.res[2];
    x = d.mn[0] + stx * ((float)cx + 0.5f);
    y = d.mn[1] + sty * ((float)cy + 0.5f);
    z = d.mn[2] + stz * ((float)cz + 0.5f);
}

// Work item i of the shadow-ray generator: probe-major (r = i % nd), so that a
// warp takes 32 consecutive directions of one probe and its shadow rays start
// close together; results are stored probe-major (sample = probe * nd + r) as
// genLightProbField.comp:47 indexes them.
__device__ __forceinline__ uint32_t probe_sample(const ProbeArgs& d, uint32_t i, uint32_t& pl, uint32_t& r) {
    r = i % d.nd;
    pl = i / d.nd;
    return pl * d.nd + r;
}

// Work item i of the probe-ray trace. It is probe-major like the generator,
// except under TIM_RT_PROBE_OCTA (the directions are the octahedral grid), where it
// is direction-major (r = i / np: a warp traces one direction from 32
// neighbouring probes; trace_dir_major is set from that flag). Measured
// per update on the 1M-triangle scene, 32x32x8 probes x 256 directions: the
// octahedral set takes 4.17 ms this way against 4.28 ms probe-major, the
// stratified set 3.71 ms probe-major against 3.85 ms direction-major.
__device__ __forceinline__ uint32_t probe_trace_item(const ProbeArgs& d, uint32_t i, uint32_t& pl, uint32_t& r) {
    if (!d.trace_dir_major) return probe_sample(d, i, pl, r);
    r = i / d.np;
    pl = i % d.np;
    return pl * d.nd + r;
}

struct ProbePolicy {
    ProbeArgs d;
    uint4* out;          // 2 x uint4 per sample (tracingData layout)
    uint32_t* leaf_nid;

    __device__ __forceinline__ bool load(const SceneView&, uint32_t i, TravState& st) const {
        uint32_t pl, r;
        st.slot = probe_trace_item(d, i, pl, r);
        probe_position(d, d.p0 + pl, st.r.ox, st.r.oy, st.r.oz);
        const float4 dir = __ldg(d.dirs + r);
        st.r.dx = dir.x; st.r.dy = dir.y; st.r.dz = dir.z;
        st.t = kTMax;
        st.any = false;
        st.dup_ok = false;   // the hit leaf's light list feeds the shadow rays
        return true;
    }
    __device__ __forceinline__ void store(const SceneView&, uint32_t, const TravState& st, float) const {
        out[2u * st.slot] = make_uint4(st.rec0, st.rec1, st.rec2, __float_as_uint(st.t));
        out[2u * st.slot + 1u] = make_uint4(0u, 0u, 0u, 0u);
        leaf_nid[st.slot] = st.hit ? st.nid : 0xFFFFFFFFu;
    }
    __device__ __forceinline__ void skip(uint32_t) const {}
};

// Shadow rays of the probe hits: the sun (tmax = TMAX) and the hit leaf's lights
// (computeAdditionalHitData / computeShadowMask, baseRaytracingPass.glsl:85-97,
// bvhLighting.glsl:143-163); the probe mask stays 0 (no USE_LPF_MASK).
__global__ void __launch_bounds__(256) k_probe_gen(SceneView s, ProbeArgs d, GenParams g, const uint32_t* leaf_nid) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < d.np * d.nd;
    uint32_t pl = 0, r = 0, sample = 0;
    if (valid) sample = probe_sample(d, i, pl, r);
    uint4 rec = make_uint4(0, 0, 0, 0);
    if (valid) rec = reinterpret_cast<const uint4*>(g.out_words)[2u * sample];
    const float t = __uint_as_float(rec.w);
    const bool hit = valid && t < kTMax;
    float hx = 0.f, hy = 0.f, hz = 0.f;
    if (hit) {
        float ox, oy, oz;
        probe_position(d, d.p0 + pl, ox, oy, oz);
        const float4 dir = __ldg(d.dirs + r);
        hx = ox + dir.x * t;
        hy = oy + dir.y * t;
        hz = oz + dir.z * t;
    }
    emit(g, 0u, kKindSun, hit, sample, hx, hy, hz, kTMax, -d.sun[0], -d.sun[1], -d.sun[2], 1u);
    const uint32_t* list = nullptr;
    uint32_t count = 0;
    if (hit) {
        const uint32_t nid = leaf_nid[sample];
        const uint32_t off = __ldg(reinterpret_cast<const uint32_t*>(s.nodes + 4u * nid) + 3);
        const uint32_t hdr = leaf_header(s, off);
        uint32_t skip = 3u * (hdr & ((1u << kTriBits) - 1u));
        skip += (hdr >> kTriBits) & ((1u << kBlasBits) - 1u);
        skip += (hdr >> (kTriBits + kBlasBits)) & ((1u << kPrimBits) - 1u);
        count = (hdr >> (kTriBits + kBlasBits + kPrimBits)) & ((1u << kLightBits) - 1u);
        list = s.leaf + skip + 1u + off;
    }
    uint32_t direct_bits = 0;
    const uint32_t jmax = min(__reduce_max_sync(0xFFFFFFFFu, count), 15u);   // lights past every lane's count emit nothing
    for (uint32_t j = 0; j < jmax; ++j) {
        bool has = false;
        float rl = 1.f, dlx = 0.f, dly = 0.f, dlz = 0.f;
        uint32_t bit = 0;
        if (j < count) {
            const uint32_t li = __ldg(list + j);
            const float* L = s.lights + 14u * li;
            bit = li + 1u;
            if (__float_as_uint(__ldg(L)) == kLightSphere && bit < 32u) {
                const float lx = __ldg(L + 1) - hx;
                const float ly = __ldg(L + 2) - hy;
                const float lz = __ldg(L + 3) - hz;
                rl = sqrtf(dot3(lx, ly, lz, lx, ly, lz));
                if (rl < __ldg(L + 4)) {
                    has = true;
                    dlx = lx / rl;
                    dly = ly / rl;
                    dlz = lz / rl;
                } else {
                    direct_bits |= 1u << bit;
                }
            }
        }
        emit(g, 0u, kKindLight0 + j, has, sample, hx, hy, hz, rl, dlx, dly, dlz, 1u | (bit << 8));
    }
    if (valid) {
        g.out_words[8u * sample + 4u] = direct_bits;
        g.out_words[8u * sample + 5u] = 0u;
    }
}

// core/lighting.glsl:16-20 computeAttenuation
__device__ __forceinline__ float attenuation(float dist, float radius) {
    const float att = (radius * radius + 1.0f) / (255.0f * dist * dist);
    return fminf(fmaxf(att - (1.0f / 255.0f), 0.0f), 1.0f);
}

// core/lighting.glsl:22-57 computeLighting (texColor = 1, no shadow ray on the fly)
// and 137-182 computePbrLighting; m = the Material record (12 words).
__device__ void compute_lighting(const float* m, float lcx, float lcy, float lcz, float px, float py, float pz,
                                 float Lx, float Ly, float Lz, float Nx, float Ny, float Nz, float ex, float ey,
                                 float ez, float att, float& ox, float& oy, float& oz) {
    const uint32_t type = __float_as_uint(__ldg(m));
    const float cr = __ldg(m + 4), cg = __ldg(m + 5), cb = __ldg(m + 6);
    if (type == 1u) { ox = cr; oy = cg; oz = cb; return; }            // Material_Emissive
    if (type == 4u) { ox = oy = oz = 0.0f; return; }                  // Material_Transparent
    float rx = 0.f, ry = 0.f, rz = 0.f;
    const float dotL = fminf(fmaxf(dot3(Nx, Ny, Nz, Lx, Ly, Lz), 0.0f), 1.0f);
    if (type == 5u) {                                                 // Material_PBR
        const float metal = __ldg(m + 8);
        float vx = ex - px, vy = ey - py, vz = ez - pz;
        const float vl = sqrtf(dot3(vx, vy, vz, vx, vy, vz));
        vx = vx / vl; vy = vy / vl; vz = vz / vl;
        float hx = vx + Lx, hy = vy + Ly, hz = vz + Lz;
        const float hl = sqrtf(dot3(hx, hy, hz, hx, hy, hz));
        hx = hx / hl; hy = hy / hl; hz = hz / hl;
        const float NoV = fabsf(dot3(Nx, Ny, Nz, vx, vy, vz)) + 1e-5f;
        const float NoL = fminf(fmaxf(dot3(Nx, Ny, Nz, Lx, Ly, Lz), 0.0f), 1.0f);
        const float NoH = fminf(fmaxf(dot3(Nx, Ny, Nz, hx, hy, hz), 0.0f), 1.0f);
        const float LoH = fminf(fmaxf(dot3(Lx, Ly, Lz, hx, hy, hz), 0.0f), 1.0f);
        const float rough = 0.02f * 0.02f;
        const float a2 = rough * rough;
        const float f = (NoH * a2 - NoH) * NoH + 1.0f;
        const float D = a2 / (3.141592f * f * f);
        const float f0x = 0.04f * (1.0f - metal) + cr * metal, f0y = 0.04f * (1.0f - metal) + cg * metal,
                    f0z = 0.04f * (1.0f - metal) + cb * metal;
        const float p5 = powf(1.0f - LoH, 5.0f);
        const float Fx = f0x + (1.0f - f0x) * p5, Fy = f0y + (1.0f - f0y) * p5, Fz = f0z + (1.0f - f0z) * p5;
        const float GGXL = NoV * sqrtf((-NoL * a2 + NoL) * NoL + a2);
        const float GGXV = NoL * sqrtf((-NoV * a2 + NoV) * NoV + a2);
        const float V = 0.5f / (GGXV + GGXL);
        const float DV = D * V;
        const float dx = cr * (1.0f - metal) / 3.141592f, dy = cg * (1.0f - metal) / 3.141592f,
                    dz = cb * (1.0f - metal) / 3.141592f;
        rx = ((dx + Fx * DV) * lcx) * NoL;
        ry = ((dy + Fy * DV) * lcy) * NoL;
        rz = ((dz + Fz * DV) * lcz) * NoL;
    } else if (type == 2u) {                                          // Material_Lambert
        rx = (lcx * dotL) * cr;
        ry = (lcy * dotL) * cg;
        rz = (lcz * dotL) * cb;
    }
    ox = rx * att;
    oy = ry * att;
    oz = rz * att;
}

// baseRaytracingPass.glsl:38-64 fillUvNormal, the normal: barycentric weights of
// the hit point in the hit triangle (record rec) and the interpolated vertex normal.
__device__ __forceinline__ void hit_normal(const SceneView& s, const uint4& rec, float px, float py, float pz,
                                           float& Nx, float& Ny, float& Nz) {
    const uint32_t i0 = rec.x + (rec.y & 0xFFFFu), i1 = rec.x + (rec.y >> 16), i2 = rec.x + (rec.z & 0xFFFFu);
    const float* P = s.pos;
    const float v0x = P[3 * i1] - P[3 * i0], v0y = P[3 * i1 + 1] - P[3 * i0 + 1], v0z = P[3 * i1 + 2] - P[3 * i0 + 2];
    const float v1x = P[3 * i2] - P[3 * i0], v1y = P[3 * i2 + 1] - P[3 * i0 + 1], v1z = P[3 * i2 + 2] - P[3 * i0 + 2];
    const float v2x = px - P[3 * i0], v2y = py - P[3 * i0 + 1], v2z = pz - P[3 * i0 + 2];
    const float d00 = dot3(v0x, v0y, v0z, v0x, v0y, v0z), d01 = dot3(v0x, v0y, v0z, v1x, v1y, v1z);
    const float d11 = dot3(v1x, v1y, v1z, v1x, v1y, v1z);
    const float d20 = dot3(v2x, v2y, v2z, v0x, v0y, v0z), d21 = dot3(v2x, v2y, v2z, v1x, v1y, v1z);
    const float denom = d00 * d11 - d01 * d01;
    const float v = (d11 * d20 - d01 * d21) / denom;
    const float w = (d00 * d21 - d01 * d20) / denom;
    const float u = 1.0f - v - w;
    const float* Nn = s.nrm;
    Nx = (Nn[3 * i0] * u + Nn[3 * i1] * v) + Nn[3 * i2] * w;
    Ny = (Nn[3 * i0 + 1] * u + Nn[3 * i1 + 1] * v) + Nn[3 * i2 + 1] * w;
    Nz = (Nn[3 * i0 + 2] * u + Nn[3 * i1 + 2] * v) + Nn[3 * i2 + 2] * w;
}

// bvhLighting.glsl:42-85 computeLighting, direct part (texColor 1): the lights whose
// shadow-mask bit is clear (evalLighting -> evalSphereLight; an out-of-range light
// adds nothing), then the sun (evalSunLight), summed in the shader's order.
__device__ void direct_lit(const SceneView& s, const float* m, float px, float py, float pz, float Nx, float Ny,
                           float Nz, float ex, float ey, float ez, uint32_t mask, const float* sun, const float* sunc,
                           float& lx, float& ly, float& lz) {
    lx = 0.f; ly = 0.f; lz = 0.f;
    for (uint32_t li = 0; li < s.num_lights && li < 31u; ++li) {
        if (mask & (1u << (li + 1u))) continue;
        const float* L = s.lights + 14u * li;
        if (__float_as_uint(__ldg(L)) != kLightSphere) continue;
        const float ax = __ldg(L + 1) - px, ay = __ldg(L + 2) - py, az = __ldg(L + 3) - pz;
        float dd = sqrtf(dot3(ax, ay, az, ax, ay, az));
        if (dd < __ldg(L + 4)) {
            const float Lx = ax / dd, Ly = ay / dd, Lz = az / dd;
            dd = fmaxf(0.01f, dd - __ldg(L + 8));
            float cx, cy, cz;
            compute_lighting(m, __ldg(L + 5), __ldg(L + 6), __ldg(L + 7), px, py, pz, Lx, Ly, Lz, Nx, Ny, Nz, ex, ey,
                             ez, attenuation(dd, __ldg(L + 4)), cx, cy, cz);
            lx = lx + cx; ly = ly + cy; lz = lz + cz;
        }
    }
    if ((mask & 1u) == 0u) {
        float cx, cy, cz;
        compute_lighting(m, sunc[0], sunc[1], sunc[2], px, py, pz, -sun[0], -sun[1], -sun[2], Nx, Ny, Nz, ex, ey, ez,
                         1.0f, cx, cy, cz);
        lx = lx + cx; ly = ly + cy; lz = lz + cz;
    }
}

// baseRaytracingPass.glsl:81: the colour of a miss, 0.3 * vec3(200, 220, 255) / 255.
__device__ __forceinline__ void sky_colour(float& lx, float& ly, float& lz) {
    lx = (0.3f * 200.0f) / 255.0f;
    ly = (0.3f * 220.0f) / 255.0f;
    lz = (0.3f * 255.0f) / 255.0f;
}

// Lit value of one probe ray: bvhLighting.glsl:42-85 computeLighting with NO_LPF
// (genLightProbField.comp:5), normal from baseRaytracingPass.glsl:38-64, sky
// colour on a miss (baseRaytracingPass.glsl:81).
__global__ void __launch_bounds__(256) k_probe_light(SceneView s, ProbeArgs d, const uint32_t* out_words, float* irr) {
    const uint32_t sample = blockIdx.x * blockDim.x + threadIdx.x;
    if (sample >= d.np * d.nd) return;
    const uint32_t pl = sample / d.nd, r = sample % d.nd;
    const uint4 rec = reinterpret_cast<const uint4*>(out_words)[2u * sample];
    const uint32_t mask = out_words[8u * sample + 4u];
    const float t = __uint_as_float(rec.w);
    float lx, ly, lz;
    if (!(t < kTMax)) {
        sky_colour(lx, ly, lz);
    } else {
        float ox, oy, oz;
        probe_position(d, d.p0 + pl, ox, oy, oz);
        const float4 dir = __ldg(d.dirs + r);
        const float px = ox + dir.x * t, py = oy + dir.y * t, pz = oz + dir.z * t;
        float Nx, Ny, Nz;
        hit_normal(s, rec, px, py, pz, Nx, Ny, Nz);
        const float* m = s.materials + 12u * (rec.z >> 16);
        direct_lit(s, m, px, py, pz, Nx, Ny, Nz, ox, oy, oz, mask, d.sun, d.sunc, lx, ly, lz);
    }
    irr[3u * sample] = lx;
    irr[3u * sample + 1u] = ly;
    irr[3u * sample + 2u] = lz;
}

// updateLightProbField.comp:33-64: one thread per probe, rays summed in order
// (j-th SH coefficient, r,g,b), x 4*pi/N, GLSL mix with the previous FP16 value,
// stored back as FP16 in storeSH9's channel layout; plus the octahedral texels.
__global__ void __launch_bounds__(128) k_probe_accum(ProbeArgs d, const float* irr, uint16_t* sh16, float* sh32,
                                                     float* octa, uint32_t side) {
    const uint32_t pl = blockIdx.x * blockDim.x + threadIdx.x;
    if (pl >= d.np) return;
    const uint32_t nd = d.nd;
    float acc[27];
#pragma unroll
    for (int q = 0; q < 27; ++q) acc[q] = 0.0f;
    const float* L = irr + 3ull * pl * nd;
    for (uint32_t r = 0; r < nd; ++r) {
        const float Lr = L[3 * r], Lg = L[3 * r + 1], Lb = L[3 * r + 2];
        const float* w = d.basis + 9u * r;
#pragma unroll
        for (int j = 0; j < 9; ++j) {
            const float wj = __ldg(w + j);
            acc[3 * j] = acc[3 * j] + Lr * wj;
            acc[3 * j + 1] = acc[3 * j + 1] + Lg * wj;
            acc[3 * j + 2] = acc[3 * j + 2] + Lb * wj;
        }
    }
    const float norm = (4.0f * 3.14159265358979323846f) / (float)nd;
    uint32_t cx, cy, cz;
    probe_coord(d.p0 + pl, d.res, cx, cy, cz);
    const uint64_t texel = ((uint64_t)cz * d.res[1] + cy) * d.res[0] + cx;
    const uint64_t img = (uint64_t)d.res[0] * d.res[1] * d.res[2];
    const float a = d.hyst;
#pragma unroll
    for (int j = 0; j < 9; ++j) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const uint32_t image = j == 0 ? 0u : (j <= 4 ? 1u + 2u * c : 2u + 2u * c);
            const uint32_t ch = j == 0 ? (uint32_t)c : (j <= 4 ? (uint32_t)(j - 1) : (uint32_t)(j - 5));
            uint16_t* h = sh16 + 4ull * (image * img + texel) + ch;
            const float prev = __half2float(__ushort_as_half(*h));
            const float nw = prev * (1.0f - a) + (acc[3 * j + c] * norm) * a;
            *h = __half_as_ushort(__float2half_rn(nw));
            if (sh32) sh32[27ull * pl + 3 * j + c] = nw;
        }
    }
    sh16[4ull * texel + 3] = 0;   // image 0 alpha (storeSH9 writes 0)
    if (octa) {
        const uint32_t per = (side / 8u) * (side / 8u);
        const float inv = 1.0f / (float)per;
        float* o = octa + 192ull * pl;
        for (uint32_t q = 0; q < 64u; ++q) {
            const uint32_t tx = q % 8u, ty = q / 8u, step = side / 8u;
            float sr = 0.f, sg = 0.f, sb = 0.f;
            for (uint32_t jj = ty * step; jj < (ty + 1u) * step; ++jj)
                for (uint32_t ii = tx * step; ii < (tx + 1u) * step; ++ii) {
                    const uint32_t k = jj * side + ii;
                    sr = sr + L[3 * k]; sg = sg + L[3 * k + 1]; sb = sb + L[3 * k + 2];
                }
            o[3 * q] = sr * inv;
            o[3 * q + 1] = sg * inv;
            o[3 * q + 2] = sb * inv;
        }
    }
}

// ------------------------------------------------------------ camera lighting step
__device__ __forceinline__ float mixf(float a, float b, float x) { return a * (1.0f - x) + b * x; }   // GLSL mix

// fetchSH_inline.glsl:82-118 sampleSH9 with the probe mask, for one image channel:
// v[x + 2y + 4z] are the corner values, mask bit (x + 2y + 4z) set = corner
// masked; the shader's lerp tree, so the shader's rounding.
__device__ __forceinline__ float masked_trilinear(const float (&v)[8], float fx, float fy, float fz, uint32_t mask) {
    const bool m0 = !(mask & 1u), m1 = !(mask & 2u), m2 = !(mask & 4u), m3 = !(mask & 8u);
    const bool m4 = !(mask & 16u), m5 = !(mask & 32u), m6 = !(mask & 64u), m7 = !(mask & 128u);
    float x0 = m0 && m1 ? mixf(v[0], v[1], fx) : (m0 ? v[0] : v[1]);
    float x1 = m2 && m3 ? mixf(v[2], v[3], fx) : (m2 ? v[2] : v[3]);
    const bool b00 = m0 || m1, b10 = m2 || m3;
    const float z0 = b00 && b10 ? mixf(x0, x1, fy) : (b00 ? x0 : x1);
    x0 = m4 && m5 ? mixf(v[4], v[5], fx) : (m4 ? v[4] : v[5]);
    x1 = m6 && m7 ? mixf(v[6], v[7], fx) : (m6 ? v[6] : v[7]);
    const bool b01 = m4 || m5, b11 = m6 || m7;
    const float z1 = b01 && b11 ? mixf(x0, x1, fy) : (b01 ? x0 : x1);
    const bool bxy0 = b00 || b10, bxy1 = b01 || b11;
    return bxy0 && bxy1 ? mixf(z0, z1, fz) : (bxy0 ? z0 : z1);
}

// bvhLighting.glsl:24-40 computeLPFLighting with USE_LPF_MASK: probe-grid uvw
// (lightprobHelpers.glsl:10-14,71-77), masked SH9 sample of the 7 RGBA16F images
// (fetchSH_inline.glsl:6-31 channel layout), evalSH (lightprobHelpers.glsl:90-101)
// and computeIndirectLighting (core/lighting.glsl:59-74, texColor 1).
__device__ void lpf_lit(const tim_rt_pass_data& pd, const uint2* sh16, const float* m, float px, float py, float pz,
                        float Nx, float Ny, float Nz, uint32_t mask, float& lx, float& ly, float& lz) {
    const uint32_t rx = pd.lpfResolution[0], ry = pd.lpfResolution[1], rz = pd.lpfResolution[2];
    const float sx = (pd.sceneMaxExtent[0] - pd.sceneMinExtent[0]) / (float)rx;
    const float sy = (pd.sceneMaxExtent[1] - pd.sceneMinExtent[1]) / (float)ry;
    const float sz = (pd.sceneMaxExtent[2] - pd.sceneMinExtent[2]) / (float)rz;
    float u = (px - pd.sceneMinExtent[0]) / sx - 0.5f;
    float v = (py - pd.sceneMinExtent[1]) / sy - 0.5f;
    float w = (pz - pd.sceneMinExtent[2]) / sz - 0.5f;
    u = fminf(fmaxf(u, 0.0f), (float)rx - 1.0f);
    v = fminf(fmaxf(v, 0.0f), (float)ry - 1.0f);
    w = fminf(fmaxf(w, 0.0f), (float)rz - 1.0f);
    // min(int(uvw), res - 2) in GLSL's int -> uint conversion
    const uint32_t ix = min((uint32_t)(int)u, rx - 2u), iy = min((uint32_t)(int)v, ry - 2u),
                   iz = min((uint32_t)(int)w, rz - 2u);
    const float fx = u - (float)(int)ix, fy = v - (float)(int)iy, fz = w - (float)(int)iz;
    const uint64_t img = (uint64_t)rx * ry * rz;
    float ch[7][4];
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        float c[4][8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const uint64_t texel = ((uint64_t)(iz + ((q >> 2) & 1)) * ry + (iy + ((q >> 1) & 1))) * rx + ix + (q & 1);
            const uint2 h = __ldg(sh16 + k * img + texel);
            c[0][q] = __half2float(__ushort_as_half((unsigned short)(h.x & 0xFFFFu)));
            c[1][q] = __half2float(__ushort_as_half((unsigned short)(h.x >> 16)));
            c[2][q] = __half2float(__ushort_as_half((unsigned short)(h.y & 0xFFFFu)));
            c[3][q] = __half2float(__ushort_as_half((unsigned short)(h.y >> 16)));
        }
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) ch[k][cc] = masked_trilinear(c[cc], fx, fy, fz, mask);
    }
    const float c1 = 0.429043f, c2 = 0.511664f, c3 = 0.743125f, c4 = 0.886227f, c5 = 0.247708f;
    float L[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        // SH9Color.w[j] from the storeSH9 layout: w0 = image 0; w1..4 = images 1/3/5, w5..8 = images 2/4/6
        const float w0 = ch[0][c], w1 = ch[1 + 2 * c][0], w2 = ch[1 + 2 * c][1], w3 = ch[1 + 2 * c][2];
        const float w4 = ch[1 + 2 * c][3], w5 = ch[2 + 2 * c][0], w6 = ch[2 + 2 * c][1], w7 = ch[2 + 2 * c][2];
        const float w8 = ch[2 + 2 * c][3];
        // SH_Y00 0, Y11 1, Y10 2, Y1_1 3, Y21 4, Y2_1 5, Y2_2 6, Y20 7, Y22 8 (lightprob/lightprob.glsl)
        const float t1 = (c1 * (Nx * Nx - Ny * Ny)) * w8;
        const float t2 = ((c3 * w7) * Nz) * Nz;
        const float t3 = c4 * w0;
        const float t4 = c5 * w7;
        const float t5 = (2.0f * c1) * (((w6 * Nx) * Ny + (w4 * Nx) * Nz) + (w5 * Ny) * Nz);
        const float t6 = (2.0f * c2) * ((w1 * Nx + w3 * Ny) + w2 * Nz);
        L[c] = ((((t1 + t2) + t3) - t4) + t5) + t6;
    }
    const uint32_t type = __float_as_uint(__ldg(m));
    const float cr = __ldg(m + 4), cg = __ldg(m + 5), cb = __ldg(m + 6);
    const float pi = 3.14159265359f;   // TIM_PI, core/math.glsl:4
    if (type == 5u) {                  // Material_PBR
        const float k = 1.0f - __ldg(m + 8);
        lx = ((k * cr) * L[0]) / pi; ly = ((k * cg) * L[1]) / pi; lz = ((k * cb) * L[2]) / pi;
    } else if (type == 2u) {           // Material_Lambert
        lx = (L[0] * cr) / pi; ly = (L[1] * cg) / pi; lz = (L[2] * cb) / pi;
    } else {
        lx = ly = lz = 0.0f;
    }
}

// cameraPass.comp:78-88, the lighting step (RayTracingPass::lightingPass,
// raytracingPass.cpp:113-135: USE_LPF, USE_LPF_MASK). One thread per output pixel
// in row-major order (coalesced record reads and image writes); the pixel's ray is
// the tracing step's (cameraPass.comp:46-56), output row 0 is never reached by the
// reference's dispatch and is written as 0.
__global__ void __launch_bounds__(256) k_shade_camera(SceneView s, tim_rt_pass_data pd, uint32_t flags,
                                                      const uint4* tracing, const uint2* sh16, uint2* out16,
                                                      float* out32) {
    const uint32_t W = pd.frameSize[0], H = pd.frameSize[1];
    const uint64_t pix = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= (uint64_t)W * H) return;
    const uint32_t px = (uint32_t)(pix % W), py = (uint32_t)(pix / W);
    float lx = 0.f, ly = 0.f, lz = 0.f;
    bool reached = py != 0u;
    if (reached) {
        const uint4 rec = __ldg(tracing + 2u * pix);
        const uint4 masks = __ldg(tracing + 2u * pix + 1u);
        const float t = __uint_as_float(rec.w);
        if (!(t < kTMax)) {
            sky_colour(lx, ly, lz);
        } else {
            const uint32_t ngy16 = 16u * ((H + 15u) / 16u);
            float dx, dy, dz;
            camera_ray(pd, px, ngy16 - py, dx, dy, dz);
            const float ex = pd.cameraPos[0], ey = pd.cameraPos[1], ez = pd.cameraPos[2];
            const float hx = ex + dx * t, hy = ey + dy * t, hz = ez + dz * t;
            float Nx, Ny, Nz;
            hit_normal(s, rec, hx, hy, hz, Nx, Ny, Nz);
            const float* m = s.materials + 12u * (rec.z >> 16);
            direct_lit(s, m, hx, hy, hz, Nx, Ny, Nz, ex, ey, ez, masks.x, pd.sunDir, pd.sunColor, lx, ly, lz);
            if (!(flags & TIM_RT_SHADE_NO_LPF)) {
                float ix, iy, iz;
                lpf_lit(pd, sh16, m, hx, hy, hz, Nx, Ny, Nz, masks.y, ix, iy, iz);
                lx = lx + ix; ly = ly + iy; lz = lz + iz;
            }
        }
    }
    const uint32_t hr = __half_as_ushort(__float2half_rn(lx)), hg = __half_as_ushort(__float2half_rn(ly));
    const uint32_t hb = __half_as_ushort(__float2half_rn(lz));
    const uint32_t ha = reached ? 0x3C00u : 0u;   // alpha 1
    out16[pix] = make_uint2(hr | (hg << 16), hb | (ha << 16));
    if (out32) {
        out32[3u * pix] = lx;
        out32[3u * pix + 1u] = ly;
        out32[3u * pix + 2u] = lz;
    }
}

cudaError_t launch_shade(const SceneView& s, const tim_rt_pass_data& pd, uint32_t flags, const uint32_t* tracing,
                         const uint16_t* sh16, uint16_t* out16, float* out32, cudaStream_t stream) {
    const uint64_t npix = (uint64_t)pd.frameSize[0] * pd.frameSize[1];
    if (npix == 0) return cudaSuccess;
    k_shade_camera<<<(unsigned)((npix + 255u) / 256u), 256, 0, stream>>>(
        s, pd, flags, reinterpret_cast<const uint4*>(tracing), reinterpret_cast<const uint2*>(sh16),
        reinterpret_cast<uint2*>(out16), out32);
    return cudaGetLastError();
}

cudaError_t launch_probes(const SceneView& s, const ProbeArgs& d, uint32_t* out, uint32_t* leaf_nid, tim_rt_ray* q_rays,
                          uint32_t* q_pixel, uint32_t* counters, uint32_t* err, float* irr, uint16_t* sh16, float* sh32,
                          float* octa, uint32_t side, cudaStream_t stream, const LaunchConfig& cfg) {
    const uint32_t n = d.np * d.nd;
    uint32_t* q_counts = counters + 2;
    uint32_t* prefix = counters + 2 + kNumKinds;
    ProbePolicy PP{d, reinterpret_cast<uint4*>(out), leaf_nid};
    if (cfg.phase_ev) cudaEventRecord(cfg.phase_ev[0], stream);
    const bool probe_wide = cfg.wide && !cfg.primary_binary;
    cudaError_t e = probe_wide ? launch_persistent<true>(s, PP, n, nullptr, counters + 0, err, stream, cfg)
                               : launch_persistent<false>(s, PP, n, nullptr, counters + 0, err, stream, cfg);
    if (e != cudaSuccess) return e;
    if (cfg.phase_ev) cudaEventRecord(cfg.phase_ev[1], stream);
    GenParams g{};
    g.out_words = out;
    g.q_rays = q_rays;
    g.q_pixel = q_pixel;
    g.q_counts = q_counts;
    g.qb.n = 1;
    g.qb.cap[0] = n;
    k_probe_gen<<<(n + 255u) / 256u, 256, 0, stream>>>(s, d, g, leaf_nid);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_kind_prefix<<<1, 1, 0, stream>>>(q_counts, prefix, g.qb, nullptr);
    if (cfg.phase_ev) cudaEventRecord(cfg.phase_ev[2], stream);
    SecondaryPolicy SP{q_rays, q_pixel, prefix, g.qb, out, nullptr, nullptr, nullptr};
    LaunchConfig cfg2 = cfg;
    if (cfg.stats) cfg2.stats = cfg.stats + 8;
    e = cfg.wide ? launch_persistent<true>(s, SP, 0u, prefix + kNumKinds, counters + 1, err, stream, cfg2)
                 : launch_persistent<false>(s, SP, 0u, prefix + kNumKinds, counters + 1, err, stream, cfg2);
    if (cfg.phase_ev) cudaEventRecord(cfg.phase_ev[3], stream);
    if (e != cudaSuccess) return e;
    k_probe_light<<<(n + 255u) / 256u, 256, 0, stream>>>(s, d, out, irr);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_probe_accum<<<(d.np + 127u) / 128u, 128, 0, stream>>>(d, irr, sh16, sh32, octa, side);
    return cudaGetLastError();
}

}  // namespace timrt
