// context.h -- the context, scene and batch structures behind the opaque
// handles of include/tim_rt.h, shared by the C-ABI implementation files.
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include <map>
#include <memory>
#include <set>
#include <string>
#include <vector>
#include "internal.h"
#include "kernels.h"

namespace timrt {

struct DevBuf {
    void* ptr = nullptr;
    uint64_t bytes = 0;
};

struct Scene {
    DevBuf blob, pos, nrm, uv, wnodes, wtris, wnid;
    DevBuf ptris, pleaf;   // the plain form's leaf-triangle copy (build_leaf_tris)
    SceneView view{};
    uint32_t ranges[7][2];
    tim_rt_push_constants pc{};
    uint32_t depth = 0;
    bool has_wide = false;
    bool blas_roots_ok = true;              // every BLAS rootIndex is an inner node (TIM_RT_TRACE_TLAS)
    uint64_t bytes = 0;
    float bounds[6] = {0, 0, 0, 1, 1, 1};   // vertex bounds (ray-sort key)
    std::atomic<uint32_t> batch_refs{0};    // live batches and pending server requests on this scene
};

}  // namespace timrt

using namespace timrt;

struct tim_rt_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint64_t budget = 0;
    uint64_t used = 0;
    std::map<uint32_t, std::unique_ptr<Scene>> scenes;
    uint32_t next_id = 1;
    // scratch
    DevBuf rays, hits, nid, bary;
    DevBuf counters;            // [0..63] per-call work counters, [64] device error word, ring after
    uint32_t ring = 0;
    DevBuf cam_out, cam_bounce, cam_nid, q_rays, q_pixel, tiles_counts, tiles_lists;
    DevBuf dstats;              // [0..15] u64 work counters of the counting kernels, [16..20] verification
    DevBuf p_dirs, p_basis, p_out, p_nid, p_irr, p_sh16, p_sh32, p_octa;   // light-probe update
    DevBuf sh_out, sh_f32;      // camera lighting step
    DevBuf bld;                 // GPU BVH builder scratch (kept between builds)
    cudaEvent_t ev[4] = {};
    cudaEvent_t pev[4] = {};   // camera phases
    cudaStream_t cstream = nullptr;   // result copies overlapped with tracing (TIM_RT_CAM_PIPELINED)
    cudaEvent_t copy_ev = nullptr;    // the copies of a pipelined camera trace are done
    DevBuf band_ctr;                  // counters of a pipelined camera trace (cam_counter_words(kMaxCamBands))
    uint32_t* band_flags = nullptr;   // per band: records final (pinned host memory the device writes)
    uint32_t* band_flags_dev = nullptr;
    DevBuf ray_acc;                   // rays traced by a pipelined camera trace (u64)
    LaunchConfig cfg;
    std::set<tim_rt_batch*> batches;
    std::set<tim_rt_server*> servers;
};

struct tim_rt_batch {
    DevBuf table;               // SceneView per distinct scene, MultiJob per job, 16-B counter
    DevBuf sort;                // ray-sort keys/values and radix-sort temporary storage
    std::vector<uint32_t> scene_ids;
    uint32_t njobs = 0, total = 0;
    int depth = 1, wide_depth = 1;
    bool wide = false;
    SceneView* d_views = nullptr;
    MultiJob* d_jobs = nullptr;
    uint32_t* d_counter = nullptr;
    SortScratch ss{};
};


namespace timrt {

constexpr uint32_t kCounterWords = 64 + 1 + 4096;   // fixed counters, error word, trace_dev ring
constexpr uint32_t kErrWord = 64;
constexpr uint32_t kRingBase = 65, kRingSize = 4096;

// Device allocation admitted against the context's budget.
int dev_alloc(tim_rt_ctx* c, DevBuf& b, uint64_t bytes);
void dev_free(tim_rt_ctx* c, DevBuf& b);
// Makes the context's device current; TIM_RT_EINVAL for a null context.
int check_ctx(tim_rt_ctx* c);
Scene* find_scene(tim_rt_ctx* c, tim_rt_scene_id id);
// Stops a server's worker and releases its device memory (context teardown).
void server_shutdown(tim_rt_ctx* c, tim_rt_server* s);

// A validated light-probe update: kernel arguments (without the device
// direction / basis pointers), octahedral side (0 = no texels), rays and probes.
struct ProbePlan {
    ProbeArgs args{};
    uint32_t side = 0;
    uint64_t n = 0, total = 0;
};
// Checks a probe description and range against a scene (messages prefixed with
// `who`); TIM_RT_OK and *out filled, or an error code with the message set.
int probe_plan(Scene* s, const tim_rt_probe_desc* desc, uint32_t probe_begin, uint32_t probe_end, const char* who,
               ProbePlan* out);

}  // namespace timrt
