// kernels.h -- host-side declarations of the kernel launchers (trace.cu, probes.cu).
#pragma once
#include <cstdint>
#include <mutex>
#include <cuda_runtime.h>
#include "common.cuh"
#include "../../include/tim_rt.h"

namespace timrt {

// Launch shape of the persistent trace kernels (chosen by the autotuner).
struct LaunchConfig {
    int block = 256;    // threads per block: 64, 128 or 256
    int stack_depth = 0;  // traversal-stack entries per thread; 0 = the scene's tree depth
    int refill_min = 16;  // a warp fetches new rays once this many lanes are idle (1..32)
    int ray_sort = 0;     // batched traces: TIM_RT_SORT_* key
    int phase_switch = 10;  // a warp's node rounds end once only this many lanes still need nodes (0..31)
    bool wide = false;  // 8-wide quantised BVH instead of the reference binary layout
    bool primary_binary = false;   // probe updates with `wide`: the probe rays take the binary walk
    // when set, a counting variant of the kernel adds per-ray work to
    // stats[0..4] = (rays, node visits, leaf visits, triangle tests, node reloads)
    unsigned long long* stats = nullptr;
    // when set, the camera launcher records ev[0..3] around its three phases
    cudaEvent_t* phase_ev = nullptr;
};

// Grid sizes of one persistent kernel, per device ordinal and stack depth: the
// occupancy calculator's resident blocks per SM times the device's SM count,
// computed on first use with the device current (which also sets the kernel's
// dynamic shared-memory limit in that device's context). Thread-safe.
struct GridCache {
    static constexpr int kDevices = 64;
    std::mutex mu;
    int blocks[kDevices][kStackSize + 1] = {};
    template <class F>
    int get(int depth, F compute) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDevices) {
            cudaGetLastError();
            dev = -1;
        }
        std::lock_guard<std::mutex> lock(mu);
        if (dev < 0) return compute(0);
        if (!blocks[dev][depth]) blocks[dev][depth] = compute(dev);
        return blocks[dev][depth];
    }
};

// The kernels' packed knob word: refill threshold (1..32) | phase switch (0..31) << 8.
inline int launch_knobs(const LaunchConfig& cfg) {
    const int refill = cfg.refill_min < 1 ? 1 : (cfg.refill_min > 32 ? 32 : cfg.refill_min);
    const int sw = cfg.phase_switch < 0 ? 0 : (cfg.phase_switch > 31 ? 31 : cfg.phase_switch);
    return refill | (sw << 8);
}

cudaError_t launch_trace_batch(const SceneView& s, const tim_rt_ray* rays, uint32_t n, uint32_t mode, uint32_t* hit,
                               uint32_t* nid, float* bary, uint32_t* counter, uint32_t* err, cudaStream_t stream,
                               const LaunchConfig& cfg);

// A camera trace whose results go down in bands of output rows while it runs:
// band b covers rows [row[b], row[b+1]) (row[0] = 0, row[n] = H, the others
// multiples of 4). Primary rays and their secondary rays are generated for the
// whole frame at once, each band's secondary rays in its own part of the queue,
// and the one secondary launch takes the bands in order, counting finished rays
// per band and setting flags[b] (host memory the device writes) once band b's
// records are final, so a host thread can start that band's copy.
constexpr uint32_t kMaxCamBands = 8;
struct CameraBands {
    uint32_t n;
    uint32_t row[kMaxCamBands + 1];
    volatile uint32_t* flags;   // device address of the host flags
};

// Secondary rays are queued in camera_queue_kinds() segments of seg_cap = W*H slots
// (with bands, band b's segments hold the band's pixels each). row_begin / row_end
// restrict a launch to a band of output rows (row_begin a multiple of 4; no bands);
// counters must be cleared before each launch. counters (nb bands, 1 without):
// [0] pixel work, [1] secondary work, [2, 2 + 26 nb) per-band per-kind counts,
// [2 + 26 nb, 3 + 52 nb) their prefix (the last entry = secondary rays traced),
// [3 + 52 nb, 3 + 53 nb) finished rays per band.
uint32_t camera_queue_kinds();
// Queue segments of a probe update (np*nd slots each): the sun and the 16 light
// slots, the only kinds its shadow-ray generator emits.
uint32_t probe_queue_kinds();
constexpr uint32_t cam_counter_words(uint32_t nb) { return 3u + 53u * nb; }
constexpr uint32_t kCamCounterWords = cam_counter_words(1), kCamTotalWord = 54;
cudaError_t launch_camera(const SceneView& s, const tim_rt_pass_data& pd, uint32_t flags, uint32_t seed,
                          const uint32_t* tile_counts, const uint32_t* tile_lists, uint32_t* out, uint32_t* bounce_out,
                          uint32_t* leaf_nid, tim_rt_ray* q_rays, uint32_t* q_pixel, uint32_t seg_cap,
                          uint32_t* counters, uint32_t* err, uint64_t* d_ray_count, cudaStream_t stream,
                          const LaunchConfig& cfg, uint32_t row_begin = 0, uint32_t row_end = 0xFFFFFFFFu,
                          const CameraBands* bands = nullptr);

// One job of a batched multi-scene trace (device table entry).
struct MultiJob {
    const tim_rt_ray* rays;
    uint4* hit;
    uint32_t* nid;
    float2* bary;
    uint32_t scene_slot;    // index into the context's device SceneView table
    uint32_t mode;          // TIM_RT_MODE_*
    uint32_t first;         // first work item of the job (prefix over the batch)
    uint32_t n;
    float lo[3];            // scene bounds, for the Morton ray-sort key
    float scale[3];         // 1024 / extent per axis
};
// Ray-sort scratch of a batch: two key/value buffers of `total` entries and the
// radix sort's temporary storage.
struct SortScratch {
    unsigned long long* keys[2];
    uint32_t* vals[2];
    void* temp;
    size_t temp_bytes;
};
size_t multi_sort_temp_bytes(uint32_t total);
// Resets `counter` and launches one persistent kernel over all jobs; with
// cfg.ray_sort != 0 the rays are first ordered by the coherence key.
cudaError_t launch_multi(const SceneView* views, const MultiJob* jobs, uint32_t njobs, uint32_t total, uint32_t* counter,
                         uint32_t* err, int depth, bool wide, const SortScratch* sort, cudaStream_t stream,
                         const LaunchConfig& cfg);

// Light-probe update of probes [p0, p0 + np), nd directions each.
struct ProbeArgs {
    float mn[3], mx[3];
    uint32_t res[3];
    float sun[3], sunc[3];
    float hyst;
    uint32_t nd, p0, np;
    uint32_t trace_dir_major;  // probe rays traced direction-major (TIM_RT_PROBE_OCTA; probe_trace_item)
    const float4* dirs;     // nd
    const float* basis;     // nd x 9
};
// out: np*nd*8 u32 trace records; leaf_nid: np*nd; the queue holds
// camera_queue_kinds() segments of np*nd slots; irr: np*nd*3; sh16: the whole
// field's 7 RGBA16F images (read and written for the updated probes); sh32 and
// octa optional; side: octahedral grid side (0 = no octahedral texels).
cudaError_t launch_probes(const SceneView& s, const ProbeArgs& d, uint32_t* out, uint32_t* leaf_nid, tim_rt_ray* q_rays,
                          uint32_t* q_pixel, uint32_t* counters, uint32_t* err, float* irr, uint16_t* sh16, float* sh32,
                          float* octa, uint32_t side, cudaStream_t stream, const LaunchConfig& cfg);

// Camera lighting step: tracing = W*H*8 u32 (tim_rt_trace_camera's output), sh16 =
// the 7 RGBA16F light-probe images of pd.lpfResolution (unused with
// TIM_RT_SHADE_NO_LPF), out16 = W*H*4 halves, out32 optional W*H*3 floats.
cudaError_t launch_shade(const SceneView& s, const tim_rt_pass_data& pd, uint32_t flags, const uint32_t* tracing,
                         const uint16_t* sh16, uint16_t* out16, float* out32, cudaStream_t stream);

cudaError_t launch_cull_lights(const SceneView& s, const tim_rt_pass_data& pd, uint32_t tiles_x, uint32_t tiles_y,
                               uint32_t* counts, uint32_t* lists, cudaStream_t stream);

}  // namespace timrt
