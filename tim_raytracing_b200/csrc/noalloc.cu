// noalloc.cu -- camera trace that allocates no memory.
//
// Some callers cannot allocate device memory when they trace: an engine whose
// allocator hands out every byte from a budget fixed at start-up, a plugin host
// that forbids allocation from its callbacks, or a frame loop that cannot afford
// cudaMalloc's implicit device synchronisation. tim_rt_trace_camera_noalloc
// serves them: the caller passes its own device copies of the BVH buffer, the
// vertex positions, the tile lists and the outputs, and the scratch memory the
// camera pipeline needs (work counters, the per-pixel hit-leaf ids and the
// secondary-ray queue) lives in one file-scope device array sized for frames
// of at most TIM_RT_NOALLOC_MAX_PIXELS pixels. The array exists on every GPU
// that loads the library, from load until process exit.
#include <cuda.h>   // driver types only: the entry points come from cudaGetDriverEntryPointByVersion
#include <cuda_runtime.h>
#include <mutex>
#include <string>
#include "internal.h"
#include "kernels.h"

namespace timrt {

namespace {

constexpr uint32_t kMaxPix = TIM_RT_NOALLOC_MAX_PIXELS;
constexpr uint32_t kKinds = 26;                 // secondary-ray kinds of the camera pipeline
constexpr uint32_t kHeaderWords = 128;          // counters [0, 55), error word [64]
constexpr uint32_t kNidWords = kMaxPix;
constexpr uint32_t kPixelWords = kKinds * kMaxPix;
constexpr uint32_t kRayWords = kKinds * kMaxPix * 8u;
constexpr uint32_t kScratchWords = kHeaderWords + kNidWords + kPixelWords + kRayWords;
static_assert((kHeaderWords + kNidWords + kPixelWords) % 4u == 0u, "ray records must stay 16-byte aligned");

// The scratch of every call on this device (3.85 MB). In host code this name is
// only a stand-in: its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) uint32_t g_noalloc_scratch[kScratchWords];

std::mutex g_mu;

// The array's device address is looked up once per device context: a context
// torn down by cudaDeviceReset (or a primary-context reset) unloads the module,
// and the next context may place the array elsewhere. Contexts are told apart by
// cuCtxGetId, whose ids are never reused within a process; the two driver calls
// are reached through the runtime's entry-point query, so the library does not
// link libcuda itself.
struct AddrCache {
    unsigned long long ctx_id = 0;   // 0: nothing cached
    void* addr = nullptr;
};
AddrCache g_cache[128];
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);
CtxGetCurrentFn g_get_current = nullptr;
CtxGetIdFn g_get_id = nullptr;
bool g_fns_looked_up = false;

// Id of the calling thread's current context, or 0 when the driver cannot say
// (then the address is looked up on every call instead of cached).
unsigned long long current_context_id() {
    if (!g_fns_looked_up) {
        g_fns_looked_up = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_get_current = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_get_id = reinterpret_cast<CtxGetIdFn>(f);
        cudaGetLastError();
    }
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (!g_get_current || !g_get_id || g_get_current(&c) != CUDA_SUCCESS || !c || g_get_id(c, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

// Set-up of a call: the device address of g_noalloc_scratch in the current
// device's context, looked up with that device current on the first call in
// each context (cudaGetSymbolAddress loads the module there if needed). A
// thread on which no runtime call has bound the context yet reports id 0 and
// takes the lookup, which binds it.
int scratch_address(uint32_t** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) {
        cudaGetLastError();
        set_error("tim_rt_trace_camera_noalloc: no current CUDA device");
        return TIM_RT_EDEVICE;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    const unsigned long long id = current_context_id();
    AddrCache& c = g_cache[dev];
    if (id == 0 || c.ctx_id != id || !c.addr) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            set_error(std::string("tim_rt_trace_camera_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
            return TIM_RT_EDEVICE;
        }
        // the lookup made the context current if it was not: read the id again
        c.ctx_id = id ? id : current_context_id();
        c.addr = p;
    }
    *out = static_cast<uint32_t*>(c.addr);
    return TIM_RT_OK;
}

}  // namespace
}  // namespace timrt

using namespace timrt;

extern "C" int tim_rt_trace_camera_noalloc(const void* d_bvh, const uint32_t ranges[7][2],
                                           const tim_rt_push_constants* pc, const float* d_pos, uint32_t num_vertex,
                                           uint32_t tree_depth, const tim_rt_pass_data* pd, uint32_t flags,
                                           uint32_t seed, const uint32_t* d_tile_counts, const uint32_t* d_tile_lists,
                                           uint32_t* d_out, uint32_t* d_bounce_out, void* cuda_stream) {
    if (!d_bvh || !ranges || !pc || !d_pos || !pd || !d_out || num_vertex == 0 || pc->numNodes == 0) {
        set_error("tim_rt_trace_camera_noalloc: null argument");
        return TIM_RT_EINVAL;
    }
    const uint64_t npix = (uint64_t)pd->frameSize[0] * pd->frameSize[1];
    if (npix == 0 || npix > kMaxPix) {
        set_error("tim_rt_trace_camera_noalloc: a frame of " + std::to_string(pd->frameSize[0]) + " x " +
                  std::to_string(pd->frameSize[1]) + " pixels exceeds the allocation-free limit of " +
                  std::to_string(kMaxPix) + " pixels");
        return TIM_RT_EINVAL;
    }
    if (flags & ~(uint32_t)(TIM_RT_CAM_PROB_MASK | TIM_RT_CAM_TILE_LIGHTS | TIM_RT_CAM_BOUNCE)) {
        set_error("tim_rt_trace_camera_noalloc: only PROB_MASK, TILE_LIGHTS and BOUNCE are available here");
        return TIM_RT_EUNSUPPORTED;
    }
    if (((flags & TIM_RT_CAM_TILE_LIGHTS) && (!d_tile_counts || !d_tile_lists)) ||
        ((flags & TIM_RT_CAM_BOUNCE) && !d_bounce_out)) {
        set_error("tim_rt_trace_camera_noalloc: TILE_LIGHTS needs tile lists, BOUNCE needs bounce_out");
        return TIM_RT_EINVAL;
    }
    if ((flags & TIM_RT_CAM_PROB_MASK) &&
        (pd->lpfResolution[0] < 2 || pd->lpfResolution[1] < 2 || pd->lpfResolution[2] < 2)) {
        set_error("tim_rt_trace_camera_noalloc: PROB_MASK needs lpfResolution >= 2 per axis");
        return TIM_RT_EINVAL;
    }
    // every range is read as 4-byte words (materials and lights as floats), the
    // nodes as 16-byte vectors
    bool misaligned = ranges[TIM_RT_RANGE_NODE][0] % 16u != 0u;
    for (int k = 0; k < 7; ++k) misaligned = misaligned || (ranges[k][0] % 4u != 0u);
    if (misaligned || tree_depth > 32u) {
        set_error("tim_rt_trace_camera_noalloc: misaligned range or tree depth above 32");
        return TIM_RT_EINVAL;
    }
    uint32_t* scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc) return rc;
    const uint8_t* b = static_cast<const uint8_t*>(d_bvh);
    SceneView v{};
    v.nodes = reinterpret_cast<const float4*>(b + ranges[TIM_RT_RANGE_NODE][0]);
    v.leaf = reinterpret_cast<const uint32_t*>(b + ranges[TIM_RT_RANGE_LEAF][0]);
    v.pos = d_pos;
    v.lights = reinterpret_cast<const float*>(b + ranges[TIM_RT_RANGE_LIGHT][0]);
    v.blas = reinterpret_cast<const float*>(b + ranges[TIM_RT_RANGE_BLAS][0]);
    v.materials = reinterpret_cast<const float*>(b + ranges[TIM_RT_RANGE_MAT][0]);
    v.num_nodes = pc->numNodes;
    v.num_lights = pc->numLights;
    v.leaf_words = ranges[TIM_RT_RANGE_LEAF][1] / 4u;
    v.num_vertex = num_vertex;
    v.depth = tree_depth ? tree_depth : 32u;
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    uint32_t* header = scratch;
    uint32_t* nid = scratch + kHeaderWords;
    uint32_t* qpix = nid + kNidWords;
    tim_rt_ray* qrays = reinterpret_cast<tim_rt_ray*>(qpix + kPixelWords);
    // counters and the error word must start at zero; the queue and leaf ids are
    // fully rewritten by each call
    cudaError_t e = cudaMemsetAsync(header, 0, 4u * kHeaderWords, st);
    if (e == cudaSuccess) {
        LaunchConfig cfg;
        e = launch_camera(v, *pd, flags, seed, d_tile_counts, d_tile_lists, d_out,
                          (flags & TIM_RT_CAM_BOUNCE) ? d_bounce_out : nullptr, nid, qrays, qpix, (uint32_t)npix,
                          header, header + 64, nullptr, st, cfg);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error(std::string("tim_rt_trace_camera_noalloc: launch failed: ") + cudaGetErrorString(e));
        return TIM_RT_EDEVICE;
    }
    return TIM_RT_OK;
}
