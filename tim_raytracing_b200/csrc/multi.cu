// multi.cu -- batched multi-scene trace: one persistent launch over the rays of
// many jobs, each traced against its own resident scene, with an optional
// coherence sort of the rays (radix sort of a per-ray key) before the trace.
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include "common.cuh"
#include "trace_plain.cuh"
#include "trace_wide.cuh"
#include "kernels.h"
#include "../../include/tim_rt.h"

namespace timrt {

template <int BLOCK, bool WIDE>
constexpr size_t multi_stack_bytes(int depth) {
    return sizeof(uint32_t) * (size_t)depth * BLOCK;   // one word per entry in both forms
}

// -------------------------------------------------------------------- batched multi-scene trace

// Job of batch item i: the largest j with jobs[j].first <= i.
__device__ __forceinline__ uint32_t find_job(const MultiJob* __restrict__ jobs, uint32_t njobs, uint32_t i) {
    uint32_t lo = 0, hi = njobs;
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(&jobs[mid].first) <= i) lo = mid;
        else hi = mid;
    }
    return lo;
}

// 30-bit Morton code of a point quantised to 10 bits per axis.
__device__ __forceinline__ uint32_t spread10(uint32_t x) {
    x &= 0x3FFu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

__device__ __forceinline__ uint32_t quant10(float v, float lo, float scale) {
    const float q = (v - lo) * scale;
    return q <= 0.f ? 0u : (q >= 1023.f ? 1023u : (uint32_t)q);
}

// Sort key of every batch item: job index in the high word (rays never leave
// their job's range), then the direction octant and, for TIM_RT_SORT_MORTON,
// the Morton code of the origin in the scene's bounds. Values = item index.
__global__ void k_sort_keys(const MultiJob* __restrict__ jobs, uint32_t njobs, uint32_t total, int kind,
                            unsigned long long* __restrict__ keys, uint32_t* __restrict__ vals) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const uint32_t j = find_job(jobs, njobs, i);
        const MultiJob& J = jobs[j];
        const float4* rp = reinterpret_cast<const float4*>(J.rays + (i - J.first));
        const float4 a = __ldg(rp), b = __ldg(rp + 1);
        const uint32_t oct = (b.x < 0.f ? 1u : 0u) | (b.y < 0.f ? 2u : 0u) | (b.z < 0.f ? 4u : 0u);
        uint32_t low = oct << 29;
        if (kind == TIM_RT_SORT_MORTON) {
            const uint32_t m = spread10(quant10(a.x, J.lo[0], J.scale[0])) << 2 |
                               spread10(quant10(a.y, J.lo[1], J.scale[1])) << 1 |
                               spread10(quant10(a.z, J.lo[2], J.scale[2]));
            low |= m >> 1;
        }
        keys[i] = (unsigned long long)j << 32 | low;
        vals[i] = i;
    }
}

// One persistent launch over the rays of many jobs, each against its own
// resident scene. Work item i (or perm[i] when the rays were sorted) belongs to
// the job j with first[j] <= item < first[j+1]; a lane that refills looks its
// job up (binary search) and loads that job's scene view, so the lanes of one
// warp may trace different scenes.
template <int BLOCK, bool WIDE>
__global__ void __launch_bounds__(BLOCK, WIDE ? 768 / BLOCK : 1) k_multi(const SceneView* __restrict__ views, const MultiJob* __restrict__ jobs,
                                                 uint32_t njobs, uint32_t total, const uint32_t* __restrict__ perm,
                                                 uint32_t* counter, uint32_t* err, int sdepth, int knobs) {
    extern __shared__ uint32_t stack_mem[];
    // knobs: refill threshold (bits 0..7), phase-switch threshold (bits 8..15)
    const int refill_min = knobs & 0xFF;
    const uint32_t phase_sw = (uint32_t)(knobs >> 8) & 0xFFu;
    uint32_t* stk = stack_mem + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31u;
    TravState st;
    st.done = true;
    // the lane's scene: a pointer into the read-only view table, its fields loaded
    // where they are used (through L1) rather than held in registers
    const SceneView* svp = views;
    // active / pending as in k_persistent: lanes whose ray ended are finished
    // (8-wide proof, binary walk when it fails) and stored together when the warp
    // refills. The job's output pointers are read again at store time, so only
    // its index stays live during the traversal.
    bool active = false, pending = false, exhausted = false;
    uint32_t idx = 0, jidx = 0;
    for (;;) {
        const uint32_t idle = __ballot_sync(0xFFFFFFFFu, !active);
        if (idle && (exhausted || __popc(idle) >= refill_min || idle == 0xFFFFFFFFu)) {
            if (pending) {
                pending = false;
                if (WIDE) wide_finish_or_walk(*svp, st, err);
                const MultiJob& J = jobs[jidx];
                uint4* hit = J.hit;
                uint32_t* nid = J.nid;
                float2* bary = J.bary;
                if (st.any) {
                    hit[idx] = make_uint4(st.hit ? 1u : 0u, 0u, 0u, __float_as_uint(st.t0));
                    if (nid) nid[idx] = 0xFFFFFFFFu;
                    if (bary) bary[idx] = make_float2(0.f, 0.f);
                } else {
                    hit[idx] = make_uint4(st.rec0, st.rec1, st.rec2, __float_as_uint(st.t));
                    if (nid) nid[idx] = st.hit ? st.nid : 0xFFFFFFFFu;
                    if (bary) bary[idx] = make_float2(st.u, st.v);
                }
            }
            if (!exhausted) {
                const uint32_t need = __ballot_sync(0xFFFFFFFFu, !active);
                const int leader = __ffs(need) - 1;
                uint32_t base = 0;
                if ((int)lane == leader) base = atomicAdd(counter, (uint32_t)__popc(need));
                base = __shfl_sync(0xFFFFFFFFu, base, leader);
                if ((uint64_t)base + (uint32_t)__popc(need) >= total) exhausted = true;
                if (!active) {
                    const uint32_t my = base + __popc(need & lanemask_lt());
                    if (my < total) {
                        const uint32_t item = perm ? __ldg(perm + my) : my;
                        jidx = find_job(jobs, njobs, item);
                        const MultiJob& J = jobs[jidx];
                        svp = views + J.scene_slot;
                        idx = item - J.first;
                        const uint32_t mode = J.mode;
                        const float4* rp = reinterpret_cast<const float4*>(J.rays + idx);
                        const float4 a = __ldg(rp), b = __ldg(rp + 1);
                        st.r.ox = a.x; st.r.oy = a.y; st.r.oz = a.z;
                        st.r.dx = b.x; st.r.dy = b.y; st.r.dz = b.z;
                        st.t = a.w;
                        st.t0 = a.w;
                        st.any = (mode == TIM_RT_MODE_ANY) ||
                                 (mode == TIM_RT_MODE_PER_RAY && (__float_as_uint(b.w) & TIM_RT_RAY_ANY));
                        st.dup_ok = J.nid == nullptr;   // the leaf id is an output only with a nid buffer
                        if (WIDE) wide_init(*svp, st, stk);
                        else trav_init(st, svp->num_nodes == 1u ? kNidLeafBit : 0u);
                        active = true;
                    }
                }
            }
        }
        if (__ballot_sync(0xFFFFFFFFu, active || pending) == 0u) {
            if (exhausted) break;
            continue;
        }
        if (WIDE) {
            wide_step_warp<BLOCK>(*svp, st, active, stk, err, sdepth, phase_sw);   // all lanes: warp-synchronous step
        } else {
            plain_step_warp<BLOCK>(*svp, st, active, stk, err, sdepth, phase_sw);
        }
        if (active && st.done) {
            active = false;
            pending = true;
        }
    }
}

template <int BLOCK, bool WIDE>
static int grid_multi(int depth) {
    static GridCache cache;
    return cache.get(depth, [depth](int dev) {
        int sms = 0, per = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaFuncSetAttribute(k_multi<BLOCK, WIDE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)multi_stack_bytes<BLOCK, WIDE>(kStackSize));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_multi<BLOCK, WIDE>, BLOCK, multi_stack_bytes<BLOCK, WIDE>(depth));
        return (sms > 0 ? sms : 1) * (per > 0 ? per : 1);
    });
}

template <int BLOCK, bool WIDE>
static void launch_multi_block(const SceneView* views, const MultiJob* jobs, uint32_t njobs, uint32_t total,
                               const uint32_t* perm, uint32_t* counter, uint32_t* err, int depth, int refill,
                               cudaStream_t stream) {
    k_multi<BLOCK, WIDE><<<grid_multi<BLOCK, WIDE>(depth), BLOCK, multi_stack_bytes<BLOCK, WIDE>(depth), stream>>>(
        views, jobs, njobs, total, perm, counter, err, depth, refill);
}

static int key_bits(uint32_t njobs) {
    int b = 0;
    while ((1u << b) < njobs && b < 31) ++b;
    return 32 + (b < 1 ? 1 : b);
}

size_t multi_sort_temp_bytes(uint32_t total) {
    size_t bytes = 0;
    cub::DoubleBuffer<unsigned long long> kb(nullptr, nullptr);
    cub::DoubleBuffer<uint32_t> vb(nullptr, nullptr);
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, kb, vb, (int)total, 0, 64);
    return bytes;
}

cudaError_t launch_multi(const SceneView* views, const MultiJob* jobs, uint32_t njobs, uint32_t total, uint32_t* counter,
                         uint32_t* err, int depth, bool wide, const SortScratch* sort, cudaStream_t stream,
                         const LaunchConfig& cfg) {
    depth = depth < 1 ? 1 : (depth > kStackSize ? kStackSize : depth);
    const int refill = launch_knobs(cfg);
    const uint32_t* perm = nullptr;
    if (cfg.ray_sort != TIM_RT_SORT_NONE) {
        if (!sort) return cudaErrorInvalidValue;
        int sms = 0, dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        k_sort_keys<<<sms * 8, 256, 0, stream>>>(jobs, njobs, total, cfg.ray_sort, sort->keys[0], sort->vals[0]);
        size_t tb = sort->temp_bytes;
        cub::DoubleBuffer<unsigned long long> kb(sort->keys[0], sort->keys[1]);
        cub::DoubleBuffer<uint32_t> vb(sort->vals[0], sort->vals[1]);
        cudaError_t e = cub::DeviceRadixSort::SortPairs(sort->temp, tb, kb, vb, (int)total, 0, key_bits(njobs), stream);
        if (e != cudaSuccess) return e;
        perm = vb.Current();
    }
    cudaMemsetAsync(counter, 0, 4, stream);
    switch (cfg.block) {
        case 64:
            wide ? launch_multi_block<64, true>(views, jobs, njobs, total, perm, counter, err, depth, refill, stream)
                 : launch_multi_block<64, false>(views, jobs, njobs, total, perm, counter, err, depth, refill, stream);
            break;
        case 256:
            wide ? launch_multi_block<256, true>(views, jobs, njobs, total, perm, counter, err, depth, refill, stream)
                 : launch_multi_block<256, false>(views, jobs, njobs, total, perm, counter, err, depth, refill, stream);
            break;
        default:
            wide ? launch_multi_block<128, true>(views, jobs, njobs, total, perm, counter, err, depth, refill, stream)
                 : launch_multi_block<128, false>(views, jobs, njobs, total, perm, counter, err, depth, refill, stream);
            break;
    }
    return cudaGetLastError();
}

}  // namespace timrt
