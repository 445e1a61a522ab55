// api.cpp -- the C ABI of include/tim_rt.h: contexts, scene upload, trace calls.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <vector>
#include "context.h"

namespace timrt {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }

#define TIMRT_CUDA(call)                                                                         \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) {                                                                 \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                       \
            return TIM_RT_EDEVICE;                                                               \
        }                                                                                        \
    } while (0)

}  // namespace timrt

using namespace timrt;

namespace timrt {

int dev_alloc(tim_rt_ctx* c, DevBuf& b, uint64_t bytes) {
    if (bytes == 0) bytes = 16;
    if (c->budget && c->used + bytes > c->budget) {
        set_error("device-memory budget exhausted: need " + std::to_string(bytes) + " B, " +
                  std::to_string(c->budget - c->used) + " B left");
        return TIM_RT_ENOMEM;
    }
    cudaError_t e = cudaMalloc(&b.ptr, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
        b.ptr = nullptr;
        return TIM_RT_ENOMEM;
    }
    b.bytes = bytes;
    c->used += bytes;
    return TIM_RT_OK;
}

void dev_free(tim_rt_ctx* c, DevBuf& b) {
    if (b.ptr) {
        cudaFree(b.ptr);
        c->used -= b.bytes;
    }
    b.ptr = nullptr;
    b.bytes = 0;
}

}  // namespace timrt

namespace {

// Grows a scratch buffer to at least `bytes` (contents not preserved).
int ensure(tim_rt_ctx* c, DevBuf& b, uint64_t bytes) {
    if (b.bytes >= bytes && b.ptr) return TIM_RT_OK;
    if (b.ptr) {
        cudaStreamSynchronize(c->stream);
        dev_free(c, b);
    }
    return dev_alloc(c, b, bytes);
}

}  // namespace

namespace timrt {

int check_ctx(tim_rt_ctx* c) {
    if (!c) {
        set_error("null context");
        return TIM_RT_EINVAL;
    }
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) {
        set_error(std::string("cudaSetDevice: ") + cudaGetErrorString(e));
        return TIM_RT_EDEVICE;
    }
    return TIM_RT_OK;
}

Scene* find_scene(tim_rt_ctx* c, tim_rt_scene_id id) {
    auto it = c->scenes.find(id);
    if (it == c->scenes.end()) {
        set_error("unknown scene id " + std::to_string(id));
        return nullptr;
    }
    return it->second.get();
}

}  // namespace timrt

namespace {

// Reads and clears the device error word; a set bit means a kernel guard fired.
int check_device_error(tim_rt_ctx* c) {
    uint32_t err = 0;
    uint32_t* ew = static_cast<uint32_t*>(c->counters.ptr) + kErrWord;
    if (cudaMemcpy(&err, ew, 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_error("reading the device error word failed");
        return TIM_RT_EDEVICE;
    }
    if (err) {
        cudaMemset(ew, 0, 4);
        set_error("a trace kernel overflowed its 32-entry traversal stack");
        return TIM_RT_EDEVICE;
    }
    return TIM_RT_OK;
}

LaunchConfig cfg_for(tim_rt_ctx* c, const Scene* s, bool wide, bool count = false) {
    LaunchConfig cfg = c->cfg;
    cfg.wide = wide && s->has_wide;
    cfg.stats = count ? static_cast<unsigned long long*>(c->dstats.ptr) : nullptr;
    return cfg;
}

}  // namespace

namespace timrt {

int probe_plan(Scene* s, const tim_rt_probe_desc* desc, uint32_t probe_begin, uint32_t probe_end, const char* who,
               ProbePlan* out) {
    const std::string w(who);
    if (!desc || desc->num_dirs == 0 || desc->num_dirs > 4096) {
        set_error(w + ": null description or num_dirs outside 1..4096");
        return TIM_RT_EINVAL;
    }
    const uint32_t* res = desc->resolution;
    if (res[0] == 0 || res[1] == 0 || res[2] == 0 || res[0] % 4u || res[1] % 4u || res[2] % 4u) {
        set_error(w + ": the probe resolution must be a positive multiple of 4 per axis "
                      "(4x4x4 probe tiles, lightprobHelpers.glsl:16-61)");
        return TIM_RT_EINVAL;
    }
    const uint64_t total = (uint64_t)res[0] * res[1] * res[2];
    if (probe_begin >= probe_end || probe_end > total || total > (1u << 24)) {
        set_error(w + ": bad probe range");
        return TIM_RT_EINVAL;
    }
    const uint32_t nd = desc->num_dirs, np = probe_end - probe_begin;
    const uint64_t n = (uint64_t)np * nd;
    if (n * probe_queue_kinds() > 0xFFFFFFFFull) {
        set_error(w + ": too many probe rays in one call");
        return TIM_RT_EINVAL;
    }
    uint32_t side = 0;
    if (desc->flags & TIM_RT_PROBE_OCTA) {
        while ((uint64_t)side * side < nd) ++side;
        if ((uint64_t)side * side != nd || side % 8u) {
            set_error(w + ": OCTA needs num_dirs = side^2 with side a multiple of 8");
            return TIM_RT_EINVAL;
        }
    }
    if ((desc->flags & TIM_RT_PROBE_WIDE) && !s->has_wide) {
        set_error(w + ": scene was uploaded without TIM_RT_UPLOAD_QUANT8");
        return TIM_RT_EUNSUPPORTED;
    }
    if (!s->nrm.ptr) {
        set_error(w + ": the lit value needs vertex normals (upload with nrm)");
        return TIM_RT_EINVAL;
    }
    ProbeArgs d{};
    for (int a = 0; a < 3; ++a) {
        d.mn[a] = desc->aabbMin[a];
        d.mx[a] = desc->aabbMax[a];
        d.res[a] = res[a];
        d.sun[a] = desc->sunDir[a];
        d.sunc[a] = desc->sunColor[a];
    }
    d.hyst = desc->hysteresis;
    d.nd = nd;
    d.p0 = probe_begin;
    d.np = np;
    d.trace_dir_major = side != 0u;
    out->args = d;
    out->side = side;
    out->n = n;
    out->total = total;
    return TIM_RT_OK;
}

}  // namespace timrt

namespace {

// Copies the counting kernels' totals into the caller's stats (after a sync).
void read_counts(tim_rt_ctx* c, tim_rt_stats* st) {
    unsigned long long v[16] = {};
    cudaMemcpy(v, c->dstats.ptr, sizeof(v), cudaMemcpyDeviceToHost);
    st->node_visits = v[1] + v[9];
    st->leaf_visits = v[2] + v[10];
    st->tri_tests = v[3] + v[11];
    st->node_reloads = v[4] + v[12];
    st->secondary_rays_counted = v[8];
    st->secondary_node_visits = v[9];
    st->secondary_leaf_visits = v[10];
    st->secondary_tri_tests = v[11];
    st->secondary_node_reloads = v[12];
}

}  // namespace

extern "C" {

const char* tim_rt_version(void) { return "tim-rt-b200 1.0 (sm_100a)"; }
const char* tim_rt_last_error(void) { return g_last_error.c_str(); }

int tim_rt_create(int device, uint64_t mem_budget_bytes, tim_rt_ctx** out) {
    if (!out) {
        set_error("null output pointer");
        return TIM_RT_EINVAL;
    }
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        set_error("no CUDA device " + std::to_string(device));
        return TIM_RT_EDEVICE;
    }
    TIMRT_CUDA(cudaSetDevice(device));
    auto c = std::make_unique<tim_rt_ctx>();
    c->device = device;
    c->budget = mem_budget_bytes;
    TIMRT_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    for (auto& e : c->ev) TIMRT_CUDA(cudaEventCreate(&e));
    for (auto& e : c->pev) TIMRT_CUDA(cudaEventCreate(&e));
    TIMRT_CUDA(cudaStreamCreateWithFlags(&c->cstream, cudaStreamNonBlocking));
    TIMRT_CUDA(cudaEventCreateWithFlags(&c->copy_ev, cudaEventDisableTiming));
    TIMRT_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&c->band_flags), 4ull * kMaxCamBands, cudaHostAllocMapped));
    TIMRT_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void**>(&c->band_flags_dev), c->band_flags, 0));
    int rc = dev_alloc(c.get(), c->counters, 4ull * kCounterWords);
    if (rc) return rc;
    if ((rc = dev_alloc(c.get(), c->dstats, 256))) return rc;   // 16 counter words + 16 verification words
    if ((rc = dev_alloc(c.get(), c->ray_acc, 16))) return rc;
    TIMRT_CUDA(cudaMemset(c->counters.ptr, 0, 4ull * kCounterWords));
    *out = c.release();
    return TIM_RT_OK;
}

int tim_rt_destroy(tim_rt_ctx* c) {
    if (!c) return TIM_RT_OK;
    cudaSetDevice(c->device);
    while (!c->servers.empty()) server_shutdown(c, *c->servers.begin());
    cudaStreamSynchronize(c->stream);
    for (tim_rt_batch* b : c->batches) {
        dev_free(c, b->table);
        dev_free(c, b->sort);
        delete b;
    }
    c->batches.clear();
    for (auto& kv : c->scenes) {
        Scene* s = kv.second.get();
        for (DevBuf* b : {&s->blob, &s->pos, &s->nrm, &s->uv, &s->wnodes, &s->wtris, &s->wnid, &s->ptris, &s->pleaf}) dev_free(c, *b);
    }
    c->scenes.clear();
    for (DevBuf* b : {&c->rays, &c->hits, &c->nid, &c->bary, &c->counters, &c->cam_out, &c->cam_bounce, &c->cam_nid,
                      &c->q_rays, &c->q_pixel, &c->tiles_counts, &c->tiles_lists, &c->dstats, &c->p_dirs, &c->p_basis,
                      &c->p_out, &c->p_nid, &c->p_irr, &c->p_sh16, &c->p_sh32, &c->p_octa, &c->sh_out, &c->sh_f32, &c->bld, &c->ray_acc,
                      &c->band_ctr})
        dev_free(c, *b);
    for (auto& e : c->ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : c->pev)
        if (e) cudaEventDestroy(e);
    if (c->copy_ev) cudaEventDestroy(c->copy_ev);
    if (c->band_flags) cudaFreeHost(c->band_flags);
    if (c->cstream) {
        cudaStreamSynchronize(c->cstream);
        cudaStreamDestroy(c->cstream);
    }
    cudaStreamDestroy(c->stream);
    delete c;
    return TIM_RT_OK;
}

int tim_rt_get_launch_config(tim_rt_ctx* c, tim_rt_launch_config* cfg) {
    if (!c || !cfg) {
        set_error("null argument");
        return TIM_RT_EINVAL;
    }
    cfg->block = (uint32_t)c->cfg.block;
    cfg->stack_depth = (uint32_t)c->cfg.stack_depth;
    cfg->refill_min = (uint32_t)c->cfg.refill_min;
    cfg->ray_sort = (uint32_t)c->cfg.ray_sort;
    cfg->phase_switch = (uint32_t)c->cfg.phase_switch;
    return TIM_RT_OK;
}

int tim_rt_set_launch_config(tim_rt_ctx* c, const tim_rt_launch_config* cfg) {
    if (!c || !cfg || (cfg->block != 64 && cfg->block != 128 && cfg->block != 256) || cfg->stack_depth > 32 ||
        cfg->refill_min < 1 || cfg->refill_min > 32 || cfg->ray_sort > TIM_RT_SORT_MORTON || cfg->phase_switch > 31) {
        set_error("tim_rt_set_launch_config: block must be 64/128/256, stack_depth <= 32, refill_min 1..32, "
                  "ray_sort 0..2, phase_switch 0..31");
        return TIM_RT_EINVAL;
    }
    c->cfg.block = (int)cfg->block;
    c->cfg.stack_depth = (int)cfg->stack_depth;
    c->cfg.refill_min = (int)cfg->refill_min;
    c->cfg.ray_sort = (int)cfg->ray_sort;
    c->cfg.phase_switch = (int)cfg->phase_switch;
    return TIM_RT_OK;
}

int tim_rt_memory_used(tim_rt_ctx* c, uint64_t* bytes) {
    if (!c || !bytes) {
        set_error("null argument");
        return TIM_RT_EINVAL;
    }
    *bytes = c->used;
    return TIM_RT_OK;
}

int tim_rt_upload_bvh(tim_rt_ctx* c, const void* bvh_bytes, uint64_t n_bytes, const uint32_t ranges[7][2],
                      const float* pos, const float* nrm, const float* uv, uint32_t max_vertex, uint32_t num_vertex,
                      const tim_rt_push_constants* pc, uint32_t flags, tim_rt_scene_id* out) {
    int rc = check_ctx(c);
    if (rc) return rc;
    if (!bvh_bytes || !ranges || !pos || !pc || !out || num_vertex == 0) {
        set_error("tim_rt_upload_bvh: null argument or no vertices");
        return TIM_RT_EINVAL;
    }
    if (max_vertex < num_vertex) max_vertex = num_vertex;
    const uint8_t* blob = static_cast<const uint8_t*>(bvh_bytes);
    std::string err;
    uint32_t depth = 0;
    if (!validate_bvh(blob, n_bytes, ranges, pc->numNodes, num_vertex, pc->numLights, pc->numBlas, &depth, err)) {
        set_error("tim_rt_upload_bvh: " + err);
        return TIM_RT_EINVAL;
    }
    auto s = std::make_unique<Scene>();
    std::memcpy(s->ranges, ranges, sizeof(s->ranges));
    s->pc = *pc;
    s->depth = depth;
    {   // whether a two-level walk may enter every BLAS root (validated: the header range holds numBlas records)
        const uint32_t* bh = reinterpret_cast<const uint32_t*>(blob + ranges[TIM_RT_RANGE_BLAS][0]);
        const uint32_t* nd = reinterpret_cast<const uint32_t*>(blob + ranges[TIM_RT_RANGE_NODE][0]);
        bool ok = true;
        for (uint32_t i = 0; i < pc->numBlas && ok; ++i) {
            const uint32_t root = bh[8ull * i + 7];
            ok = root < pc->numNodes && (nd[16ull * root + 2] & 0x3FFFFFFFu) != 0x3FFFFFFFu;
        }
        s->blas_roots_ok = ok;
    }
    for (int a = 0; a < 3; ++a) {
        float lo = pos[a], hi = pos[a];
        for (uint32_t i = 1; i < num_vertex; ++i) {
            lo = std::min(lo, pos[3ull * i + a]);
            hi = std::max(hi, pos[3ull * i + a]);
        }
        s->bounds[a] = lo;
        s->bounds[3 + a] = hi;
    }
    WideHost wh;
    if (flags & TIM_RT_UPLOAD_QUANT8) {
        if (pc->numBlas) {
            set_error("tim_rt_upload_bvh: the 8-wide form does not support BLAS instances");
            return TIM_RT_EUNSUPPORTED;
        }
        if (!build_wide(blob, ranges, pc->numNodes, pos, wh, err)) {
            set_error("tim_rt_upload_bvh: 8-wide build: " + err);
            return TIM_RT_EUNSUPPORTED;
        }
    }
    // the plain form's leaf-triangle copy (16-byte vector fetches instead of
    // scalar gathers of the records and vertex positions)
    RawVec<float> ptris;
    RawVec<uint32_t> pleaf;
    build_leaf_tris(blob, ranges, pc->numNodes, pos, ptris, pleaf);
    auto fail = [&](int code) {
        for (DevBuf* b : {&s->blob, &s->pos, &s->nrm, &s->uv, &s->wnodes, &s->wtris, &s->wnid, &s->ptris, &s->pleaf}) dev_free(c, *b);
        return code;
    };
    if ((rc = dev_alloc(c, s->blob, n_bytes))) return fail(rc);
    if ((rc = dev_alloc(c, s->pos, 12ull * max_vertex))) return fail(rc);
    if (nrm && (rc = dev_alloc(c, s->nrm, 12ull * max_vertex))) return fail(rc);
    if (uv && (rc = dev_alloc(c, s->uv, 8ull * max_vertex))) return fail(rc);
    if ((rc = dev_alloc(c, s->pleaf, 4ull * pleaf.size()))) return fail(rc);
    if (!ptris.empty() && (rc = dev_alloc(c, s->ptris, 4ull * ptris.size()))) return fail(rc);
    if (cudaMemcpyAsync(s->pleaf.ptr, pleaf.data(), 4ull * pleaf.size(), cudaMemcpyHostToDevice, c->stream) != cudaSuccess ||
        (!ptris.empty() &&
         cudaMemcpyAsync(s->ptris.ptr, ptris.data(), 4ull * ptris.size(), cudaMemcpyHostToDevice, c->stream) != cudaSuccess)) {
        set_error("tim_rt_upload_bvh: host-to-device copy of the leaf triangles failed");
        return fail(TIM_RT_EDEVICE);
    }
    if (cudaMemcpyAsync(s->blob.ptr, blob, n_bytes, cudaMemcpyHostToDevice, c->stream) != cudaSuccess ||
        cudaMemcpyAsync(s->pos.ptr, pos, 12ull * num_vertex, cudaMemcpyHostToDevice, c->stream) != cudaSuccess ||
        (nrm && cudaMemcpyAsync(s->nrm.ptr, nrm, 12ull * num_vertex, cudaMemcpyHostToDevice, c->stream) != cudaSuccess) ||
        (uv && cudaMemcpyAsync(s->uv.ptr, uv, 8ull * num_vertex, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)) {
        set_error("tim_rt_upload_bvh: host-to-device copy failed");
        return fail(TIM_RT_EDEVICE);
    }
    if (flags & TIM_RT_UPLOAD_QUANT8) {
        if ((rc = dev_alloc(c, s->wnodes, 4ull * wh.nodes.size()))) return fail(rc);
        if ((rc = dev_alloc(c, s->wtris, 4ull * wh.tris.size()))) return fail(rc);
        if ((rc = dev_alloc(c, s->wnid, 4ull * wh.tri_leaf.size()))) return fail(rc);
        if (cudaMemcpyAsync(s->wnodes.ptr, wh.nodes.data(), 4ull * wh.nodes.size(), cudaMemcpyHostToDevice, c->stream) ||
            (!wh.tris.empty() && cudaMemcpyAsync(s->wtris.ptr, wh.tris.data(), 4ull * wh.tris.size(), cudaMemcpyHostToDevice, c->stream)) ||
            (!wh.tri_leaf.empty() && cudaMemcpyAsync(s->wnid.ptr, wh.tri_leaf.data(), 4ull * wh.tri_leaf.size(), cudaMemcpyHostToDevice, c->stream))) {
            set_error("tim_rt_upload_bvh: host-to-device copy of the 8-wide form failed");
            return fail(TIM_RT_EDEVICE);
        }
        s->has_wide = true;
    }
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
        set_error("tim_rt_upload_bvh: stream synchronisation failed");
        return fail(TIM_RT_EDEVICE);
    }
    const uint8_t* d = static_cast<const uint8_t*>(s->blob.ptr);
    SceneView& v = s->view;
    v.nodes = reinterpret_cast<const float4*>(d + ranges[TIM_RT_RANGE_NODE][0]);
    v.leaf = reinterpret_cast<const uint32_t*>(d + ranges[TIM_RT_RANGE_LEAF][0]);
    v.pos = static_cast<const float*>(s->pos.ptr);
    v.nrm = static_cast<const float*>(s->nrm.ptr);
    v.lights = reinterpret_cast<const float*>(d + ranges[TIM_RT_RANGE_LIGHT][0]);
    v.blas = reinterpret_cast<const float*>(d + ranges[TIM_RT_RANGE_BLAS][0]);
    v.materials = reinterpret_cast<const float*>(d + ranges[TIM_RT_RANGE_MAT][0]);
    v.num_nodes = pc->numNodes;
    v.num_lights = pc->numLights;
    v.leaf_words = ranges[TIM_RT_RANGE_LEAF][1] / 4u;
    v.num_vertex = num_vertex;
    v.depth = depth;
    v.wide_depth = wh.max_depth;
    v.wnodes = static_cast<const uint4*>(s->wnodes.ptr);
    v.wtris = static_cast<const float4*>(s->wtris.ptr);
    v.wtri_leaf = static_cast<const uint4*>(s->wnid.ptr);
    v.num_wnodes = s->has_wide ? wh.num_nodes : 0u;
    v.wide_root_is_leaf = wh.root_is_leaf;
    v.pleaf = static_cast<const uint4*>(s->pleaf.ptr);
    v.ptris = static_cast<const float4*>(s->ptris.ptr);
    s->bytes = s->blob.bytes + s->pos.bytes + s->nrm.bytes + s->uv.bytes + s->wnodes.bytes + s->wtris.bytes + s->wnid.bytes +
               s->pleaf.bytes + s->ptris.bytes;
    const uint32_t id = c->next_id++;
    c->scenes[id] = std::move(s);
    *out = id;
    return TIM_RT_OK;
}

int tim_rt_validate_bvh(const void* bvh_bytes, uint64_t n_bytes, const uint32_t ranges[7][2],
                        const tim_rt_push_constants* pc, uint32_t num_vertex, uint32_t* depth) {
    if (!bvh_bytes || !ranges || !pc) {
        set_error("tim_rt_validate_bvh: null argument");
        return TIM_RT_EINVAL;
    }
    std::string err;
    if (!validate_bvh(static_cast<const uint8_t*>(bvh_bytes), n_bytes, ranges, pc->numNodes, num_vertex, pc->numLights,
                      pc->numBlas, depth, err)) {
        set_error("tim_rt_validate_bvh: " + err);
        return TIM_RT_EINVAL;
    }
    return TIM_RT_OK;
}

int tim_rt_free_scene(tim_rt_ctx* c, tim_rt_scene_id id) {
    int rc = check_ctx(c);
    if (rc) return rc;
    Scene* s = find_scene(c, id);
    if (!s) return TIM_RT_ENOTFOUND;
    if (s->batch_refs) {
        set_error("tim_rt_free_scene: scene " + std::to_string(id) + " is used by " + std::to_string(s->batch_refs) +
                  " live batch(es)");
        return TIM_RT_EINVAL;
    }
    cudaStreamSynchronize(c->stream);
    for (DevBuf* b : {&s->blob, &s->pos, &s->nrm, &s->uv, &s->wnodes, &s->wtris, &s->wnid, &s->ptris, &s->pleaf}) dev_free(c, *b);
    c->scenes.erase(id);
    return TIM_RT_OK;
}

int tim_rt_scene_bytes(tim_rt_ctx* c, tim_rt_scene_id id, uint64_t* bytes) {
    if (!c || !bytes) {
        set_error("null argument");
        return TIM_RT_EINVAL;
    }
    Scene* s = find_scene(c, id);
    if (!s) return TIM_RT_ENOTFOUND;
    *bytes = s->bytes;
    return TIM_RT_OK;
}

}  // extern "C"
namespace {
// TIM_RT_TRACE_TLAS: any-hit rays only (the reference's closest-hit two-level walk
// does not compile), the binary form, and an image whose BLAS roots are inner nodes.
int tlas_check(const Scene* s, uint32_t mode, const char* who) {
    if (!(mode & TIM_RT_TRACE_TLAS)) return TIM_RT_OK;
    if ((mode & 0xFFu) != TIM_RT_MODE_ANY || (mode & TIM_RT_TRACE_WIDE)) {
        set_error(std::string(who) + ": TIM_RT_TRACE_TLAS traces any-hit rays (TIM_RT_MODE_ANY) in the binary form only");
        return TIM_RT_EUNSUPPORTED;
    }
    if (!s->blas_roots_ok) {
        set_error(std::string(who) + ": TIM_RT_TRACE_TLAS needs every BLAS rootIndex to name an inner node of the image");
        return TIM_RT_EINVAL;
    }
    return TIM_RT_OK;
}

}  // namespace
extern "C" {

int tim_rt_trace_dev(tim_rt_ctx* c, tim_rt_scene_id id, const tim_rt_ray* d_rays, uint32_t n, uint32_t mode,
                     uint32_t* d_hit, uint32_t* d_nid, float* d_bary, void* cuda_stream) {
    int rc = check_ctx(c);
    if (rc) return rc;
    Scene* s = find_scene(c, id);
    if (!s) return TIM_RT_ENOTFOUND;
    if ((mode & 0xFFu) > TIM_RT_MODE_PER_RAY ||
        (mode & ~(0xFFu | TIM_RT_TRACE_WIDE | TIM_RT_TRACE_COUNT | TIM_RT_TRACE_TLAS)) || n > 0x7FFFFFFFu ||
        (n && (!d_rays || !d_hit))) {
        set_error("tim_rt_trace_dev: bad mode, size or null buffer");
        return TIM_RT_EINVAL;
    }
    if ((rc = tlas_check(s, mode, "tim_rt_trace_dev"))) return rc;
    if ((mode & TIM_RT_TRACE_WIDE) && !s->has_wide) {
        set_error("tim_rt_trace_dev: scene was uploaded without TIM_RT_UPLOAD_QUANT8");
        return TIM_RT_EUNSUPPORTED;
    }
    if (n == 0) return TIM_RT_OK;
    cudaStream_t st = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : c->stream;
    uint32_t* ctr = static_cast<uint32_t*>(c->counters.ptr) + kRingBase + (c->ring++ % kRingSize);
    uint32_t* err = static_cast<uint32_t*>(c->counters.ptr) + kErrWord;
    TIMRT_CUDA(cudaMemsetAsync(ctr, 0, 4, st));
    TIMRT_CUDA(launch_trace_batch(s->view, d_rays, n, mode, d_hit, d_nid, d_bary, ctr, err, st,
                                  cfg_for(c, s, (mode & TIM_RT_TRACE_WIDE) != 0)));
    return TIM_RT_OK;
}

int tim_rt_trace(tim_rt_ctx* c, tim_rt_scene_id id, const tim_rt_ray* rays, uint32_t n, uint32_t mode, uint32_t* hit,
                 uint32_t* leaf_nid, float* bary, tim_rt_stats* stats) {
    int rc = check_ctx(c);
    if (rc) return rc;
    Scene* s = find_scene(c, id);
    if (!s) return TIM_RT_ENOTFOUND;
    if ((mode & 0xFFu) > TIM_RT_MODE_PER_RAY ||
        (mode & ~(0xFFu | TIM_RT_TRACE_WIDE | TIM_RT_TRACE_COUNT | TIM_RT_TRACE_TLAS)) || n > 0x7FFFFFFFu ||
        (n && (!rays || !hit))) {
        set_error("tim_rt_trace: bad mode, size or null buffer");
        return TIM_RT_EINVAL;
    }
    if ((rc = tlas_check(s, mode, "tim_rt_trace"))) return rc;
    if ((mode & TIM_RT_TRACE_WIDE) && !s->has_wide) {
        set_error("tim_rt_trace: scene was uploaded without TIM_RT_UPLOAD_QUANT8");
        return TIM_RT_EUNSUPPORTED;
    }
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (n == 0) return TIM_RT_OK;
    if ((rc = ensure(c, c->rays, 32ull * n)) || (rc = ensure(c, c->hits, 16ull * n))) return rc;
    if (leaf_nid && (rc = ensure(c, c->nid, 4ull * n))) return rc;
    if (bary && (rc = ensure(c, c->bary, 8ull * n))) return rc;
    uint32_t* ctr = static_cast<uint32_t*>(c->counters.ptr);
    uint32_t* err = ctr + kErrWord;
    const bool count = (mode & TIM_RT_TRACE_COUNT) != 0;
    if (count) TIMRT_CUDA(cudaMemsetAsync(c->dstats.ptr, 0, 128, c->stream));
    TIMRT_CUDA(cudaEventRecord(c->ev[0], c->stream));
    TIMRT_CUDA(cudaMemcpyAsync(c->rays.ptr, rays, 32ull * n, cudaMemcpyHostToDevice, c->stream));
    TIMRT_CUDA(cudaMemsetAsync(ctr, 0, 4, c->stream));
    TIMRT_CUDA(cudaEventRecord(c->ev[1], c->stream));
    TIMRT_CUDA(launch_trace_batch(s->view, static_cast<const tim_rt_ray*>(c->rays.ptr), n, mode,
                                  static_cast<uint32_t*>(c->hits.ptr), leaf_nid ? static_cast<uint32_t*>(c->nid.ptr) : nullptr,
                                  bary ? static_cast<float*>(c->bary.ptr) : nullptr, ctr, err, c->stream,
                                  cfg_for(c, s, (mode & TIM_RT_TRACE_WIDE) != 0, count)));
    TIMRT_CUDA(cudaEventRecord(c->ev[2], c->stream));
    TIMRT_CUDA(cudaMemcpyAsync(hit, c->hits.ptr, 16ull * n, cudaMemcpyDeviceToHost, c->stream));
    if (leaf_nid) TIMRT_CUDA(cudaMemcpyAsync(leaf_nid, c->nid.ptr, 4ull * n, cudaMemcpyDeviceToHost, c->stream));
    if (bary) TIMRT_CUDA(cudaMemcpyAsync(bary, c->bary.ptr, 8ull * n, cudaMemcpyDeviceToHost, c->stream));
    TIMRT_CUDA(cudaEventRecord(c->ev[3], c->stream));
    TIMRT_CUDA(cudaStreamSynchronize(c->stream));
    if ((rc = check_device_error(c))) return rc;
    if (stats) {
        stats->rays = n;
        stats->primary_rays = n;
        cudaEventElapsedTime(&stats->kernel_ms, c->ev[1], c->ev[2]);
        cudaEventElapsedTime(&stats->total_ms, c->ev[0], c->ev[3]);
        if (count) read_counts(c, stats);
    }
    return TIM_RT_OK;
}

int tim_rt_cull_lights(tim_rt_ctx* c, tim_rt_scene_id id, const tim_rt_pass_data* pd, uint32_t tiles_x,
                       uint32_t tiles_y, uint32_t* out_counts, uint32_t* out_lists) {
    int rc = check_ctx(c);
    if (rc) return rc;
    Scene* s = find_scene(c, id);
    if (!s) return TIM_RT_ENOTFOUND;
    if (!pd || !out_counts || !out_lists || tiles_x == 0 || tiles_y == 0 || (uint64_t)tiles_x * tiles_y > (1u << 26)) {
        set_error("tim_rt_cull_lights: bad argument");
        return TIM_RT_EINVAL;
    }
    const uint64_t nt = (uint64_t)tiles_x * tiles_y;
    if ((rc = ensure(c, c->tiles_counts, 4ull * nt)) || (rc = ensure(c, c->tiles_lists, 64ull * nt))) return rc;
    TIMRT_CUDA(launch_cull_lights(s->view, *pd, tiles_x, tiles_y, static_cast<uint32_t*>(c->tiles_counts.ptr),
                                  static_cast<uint32_t*>(c->tiles_lists.ptr), c->stream));
    TIMRT_CUDA(cudaMemcpyAsync(out_counts, c->tiles_counts.ptr, 4ull * nt, cudaMemcpyDeviceToHost, c->stream));
    TIMRT_CUDA(cudaMemcpyAsync(out_lists, c->tiles_lists.ptr, 64ull * nt, cudaMemcpyDeviceToHost, c->stream));
    TIMRT_CUDA(cudaStreamSynchronize(c->stream));
    return TIM_RT_OK;
}

}  // extern "C"

namespace {

// Validates a camera call and sizes the context's scratch; shared by the host
// and device forms.
int camera_prepare(tim_rt_ctx* c, Scene* s, const tim_rt_pass_data* pd, uint32_t flags, bool have_tiles,
                   bool have_bounce, uint64_t* qcap_out) {
    if (!pd || pd->frameSize[0] == 0 || pd->frameSize[1] == 0 ||
        (uint64_t)pd->frameSize[0] * pd->frameSize[1] > (1ull << 26)) {
        set_error("trace_camera: bad pass data");
        return TIM_RT_EINVAL;
    }
    if ((flags & TIM_RT_CAM_TILE_LIGHTS) && !have_tiles) {
        set_error("trace_camera: TILE_LIGHTS needs tile_counts and tile_lists");
        return TIM_RT_EINVAL;
    }
    if ((flags & TIM_RT_CAM_BOUNCE) && !have_bounce) {
        set_error("trace_camera: BOUNCE needs bounce_out");
        return TIM_RT_EINVAL;
    }
    if ((flags & TIM_RT_CAM_PROB_MASK) &&
        (pd->lpfResolution[0] < 2 || pd->lpfResolution[1] < 2 || pd->lpfResolution[2] < 2)) {
        set_error("trace_camera: PROB_MASK needs lpfResolution >= 2 per axis");
        return TIM_RT_EINVAL;
    }
    if ((flags & TIM_RT_CAM_WIDE) && !s->has_wide) {
        set_error("trace_camera: scene was uploaded without TIM_RT_UPLOAD_QUANT8");
        return TIM_RT_EUNSUPPORTED;
    }
    const uint64_t npix = (uint64_t)pd->frameSize[0] * pd->frameSize[1];
    const uint64_t qcap = npix * camera_queue_kinds();   // one segment of W*H slots per secondary-ray kind
    if (qcap > 0xFFFFFFFFull) {
        set_error("trace_camera: frame too large");
        return TIM_RT_EINVAL;
    }
    int rc;
    if ((rc = ensure(c, c->cam_nid, 4ull * npix)) || (rc = ensure(c, c->q_rays, 32ull * qcap)) ||
        (rc = ensure(c, c->q_pixel, 4ull * qcap)))
        return rc;
    *qcap_out = npix;
    return TIM_RT_OK;
}

}  // namespace

extern "C" {

int tim_rt_cull_lights_dev(tim_rt_ctx* c, tim_rt_scene_id id, const tim_rt_pass_data* pd, uint32_t tiles_x,
                           uint32_t tiles_y, uint32_t* d_counts, uint32_t* d_lists, void* cuda_stream) {
    int rc = check_ctx(c);
    if (rc) return rc;
    Scene* s = find_scene(c, id);
    if (!s) return TIM_RT_ENOTFOUND;
    if (!pd || !d_counts || !d_lists || tiles_x == 0 || tiles_y == 0 || (uint64_t)tiles_x * tiles_y > (1u << 26)) {
        set_error("tim_rt_cull_lights_dev: bad argument");
        return TIM_RT_EINVAL;
    }
    cudaStream_t st = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : c->stream;
    TIMRT_CUDA(launch_cull_lights(s->view, *pd, tiles_x, tiles_y, d_counts, d_lists, st));
    return TIM_RT_OK;
}

// tim_rt_trace_camera_dev over output rows [row_begin, row_end) (the whole frame: 0, H).
static int camera_dev_rows(tim_rt_ctx* c, tim_rt_scene_id id, const tim_rt_pass_data* pd, uint32_t flags, uint32_t seed,
                           uint32_t row_begin, uint32_t row_end, const uint32_t* d_tile_counts,
                           const uint32_t* d_tile_lists, uint32_t* d_out, uint32_t* d_bounce_out, uint64_t* d_ray_count,
                           void* cuda_stream, const char* who) {
    int rc = check_ctx(c);
    if (rc) return rc;
    Scene* s = find_scene(c, id);
    if (!s) return TIM_RT_ENOTFOUND;
    if (!d_out) {
        set_error(std::string(who) + ": null output");
        return TIM_RT_EINVAL;
    }
    if (flags & TIM_RT_CAM_DEVICE_CULL) {
        set_error(std::string(who) + ": TIM_RT_CAM_DEVICE_CULL is for tim_rt_trace_camera (cull with "
                                     "tim_rt_cull_lights_dev on the same stream instead)");
        return TIM_RT_EINVAL;
    }
    uint64_t qcap = 0;
    if ((rc = camera_prepare(c, s, pd, flags, d_tile_counts && d_tile_lists, d_bounce_out != nullptr, &qcap))) return rc;
    if (row_begin % 4u != 0u || row_begin >= row_end || row_end > pd->frameSize[1]) {
        set_error(std::string(who) + ": rows [" + std::to_string(row_begin) + ", " + std::to_string(row_end) +
                  ") must be a non-empty range inside the frame starting at a multiple of 4");
        return TIM_RT_EINVAL;
    }
    cudaStream_t st = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : c->stream;
    uint32_t* ctr = static_cast<uint32_t*>(c->counters.ptr);
    TIMRT_CUDA(cudaMemsetAsync(ctr, 0, 4 * kCamCounterWords, st));
    TIMRT_CUDA(launch_camera(s->view, *pd, flags, seed, d_tile_counts, d_tile_lists, d_out,
                             (flags & TIM_RT_CAM_BOUNCE) ? d_bounce_out : nullptr, static_cast<uint32_t*>(c->cam_nid.ptr),
                             static_cast<tim_rt_ray*>(c->q_rays.ptr), static_cast<uint32_t*>(c->q_pixel.ptr),
                             (uint32_t)qcap, ctr, ctr + kErrWord, d_ray_count, st,
                             cfg_for(c, s, (flags & TIM_RT_CAM_WIDE) != 0), row_begin, row_end));
    return TIM_RT_OK;
}

int tim_rt_trace_camera_dev(tim_rt_ctx* c, tim_rt_scene_id id, const tim_rt_pass_data* pd, uint32_t flags,
                            uint32_t seed, const uint32_t* d_tile_counts, const uint32_t* d_tile_lists, uint32_t* d_out,
                            uint32_t* d_bounce_out, uint64_t* d_ray_count, void* cuda_stream) {
    return camera_dev_rows(c, id, pd, flags, seed, 0u, pd ? pd->frameSize[1] : 0u, d_tile_counts, d_tile_lists, d_out,
                           d_bounce_out, d_ray_count, cuda_stream, "tim_rt_trace_camera_dev");
}

int tim_rt_trace_camera_rows_dev(tim_rt_ctx* c, tim_rt_scene_id id, const tim_rt_pass_data* pd, uint32_t flags,
                                 uint32_t seed, uint32_t row_begin, uint32_t row_end, const uint32_t* d_tile_counts,
                                 const uint32_t* d_tile_lists, uint32_t* d_out, uint32_t* d_bounce_out,
                                 uint64_t* d_ray_count, void* cuda_stream) {
    return camera_dev_rows(c, id, pd, flags, seed, row_begin, row_end, d_tile_counts, d_tile_lists, d_out,
                           d_bounce_out, d_ray_count, cuda_stream, "tim_rt_trace_camera_rows_dev");
}

// Checks of tim_rt_shade_camera(_dev): frame size, light-probe resolution, normals.
static int shade_check(Scene* s, const tim_rt_pass_data* pd, uint32_t flags, const void* tracing, const void* sh16,
                       const void* out16, const char* who) {
    const std::string w(who);
    if (!pd || !tracing || !out16 || (!(flags & TIM_RT_SHADE_NO_LPF) && !sh16) || (flags & ~TIM_RT_SHADE_NO_LPF)) {
        set_error(w + ": null argument or unknown flag");
        return TIM_RT_EINVAL;
    }
    const uint64_t npix = (uint64_t)pd->frameSize[0] * pd->frameSize[1];
    if (pd->frameSize[0] == 0 || pd->frameSize[1] == 0 || npix > (1ull << 30)) {
        set_error(w + ": frame size must be 1..2^30 pixels");
        return TIM_RT_EINVAL;
    }
    if (!(flags & TIM_RT_SHADE_NO_LPF)) {
        const uint32_t* r = pd->lpfResolution;
        if (r[0] < 2 || r[1] < 2 || r[2] < 2 || (uint64_t)r[0] * r[1] * r[2] > (1ull << 24)) {
            set_error(w + ": light-probe resolution must be 2..2^24 probes with at least 2 per axis "
                          "(sampleSH9 interpolates between neighbours)");
            return TIM_RT_EINVAL;
        }
    }
    if (!s->nrm.ptr) {
        set_error(w + ": the lit value needs vertex normals (upload with nrm)");
        return TIM_RT_EINVAL;
    }
    return TIM_RT_OK;
}

int tim_rt_shade_camera(tim_rt_ctx* c, tim_rt_scene_id id, const tim_rt_pass_data* pd, uint32_t flags,
                        const uint32_t* tracing, const uint16_t* sh9_fp16, uint16_t* out_rgba16, float* out_rgb32,
                        tim_rt_stats* stats) {
    int rc = check_ctx(c);
    if (rc) return rc;
    Scene* s = find_scene(c, id);
    if (!s) return TIM_RT_ENOTFOUND;
    if ((rc = shade_check(s, pd, flags, tracing, sh9_fp16, out_rgba16, "tim_rt_shade_camera"))) return rc;
    const uint64_t npix = (uint64_t)pd->frameSize[0] * pd->frameSize[1];
    const bool lpf = !(flags & TIM_RT_SHADE_NO_LPF);
    const uint64_t field = lpf ? 56ull * pd->lpfResolution[0] * pd->lpfResolution[1] * pd->lpfResolution[2] : 0;
    if ((rc = ensure(c, c->cam_out, 32ull * npix)) || (rc = ensure(c, c->sh_out, 8ull * npix)) ||
        (lpf && (rc = ensure(c, c->p_sh16, field))) || (out_rgb32 && (rc = ensure(c, c->sh_f32, 12ull * npix))))
        return rc;
    TIMRT_CUDA(cudaEventRecord(c->ev[0], c->stream));
    TIMRT_CUDA(cudaMemcpyAsync(c->cam_out.ptr, tracing, 32ull * npix, cudaMemcpyHostToDevice, c->stream));
    if (lpf) TIMRT_CUDA(cudaMemcpyAsync(c->p_sh16.ptr, sh9_fp16, field, cudaMemcpyHostToDevice, c->stream));
    TIMRT_CUDA(cudaEventRecord(c->ev[1], c->stream));
    TIMRT_CUDA(launch_shade(s->view, *pd, flags, static_cast<const uint32_t*>(c->cam_out.ptr),
                            lpf ? static_cast<const uint16_t*>(c->p_sh16.ptr) : nullptr,
                            static_cast<uint16_t*>(c->sh_out.ptr), out_rgb32 ? static_cast<float*>(c->sh_f32.ptr) : nullptr,
                            c->stream));
    TIMRT_CUDA(cudaEventRecord(c->ev[2], c->stream));
    TIMRT_CUDA(cudaMemcpyAsync(out_rgba16, c->sh_out.ptr, 8ull * npix, cudaMemcpyDeviceToHost, c->stream));
    if (out_rgb32) TIMRT_CUDA(cudaMemcpyAsync(out_rgb32, c->sh_f32.ptr, 12ull * npix, cudaMemcpyDeviceToHost, c->stream));
    TIMRT_CUDA(cudaEventRecord(c->ev[3], c->stream));
    TIMRT_CUDA(cudaStreamSynchronize(c->stream));
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        cudaEventElapsedTime(&stats->kernel_ms, c->ev[1], c->ev[2]);
        cudaEventElapsedTime(&stats->total_ms, c->ev[0], c->ev[3]);
    }
    return TIM_RT_OK;
}

int tim_rt_shade_camera_dev(tim_rt_ctx* c, tim_rt_scene_id id, const tim_rt_pass_data* pd, uint32_t flags,
                            const uint32_t* d_tracing, const uint16_t* d_sh9_fp16, uint16_t* d_out_rgba16,
                            float* d_out_rgb32, void* cuda_stream) {
    int rc = check_ctx(c);
    if (rc) return rc;
    Scene* s = find_scene(c, id);
    if (!s) return TIM_RT_ENOTFOUND;
    if ((rc = shade_check(s, pd, flags, d_tracing, d_sh9_fp16, d_out_rgba16, "tim_rt_shade_camera_dev"))) return rc;
    cudaStream_t st = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : c->stream;
    TIMRT_CUDA(launch_shade(s->view, *pd, flags, d_tracing, d_sh9_fp16, d_out_rgba16, d_out_rgb32, st));
    return TIM_RT_OK;
}

int tim_rt_update_probes(tim_rt_ctx* c, tim_rt_scene_id id, const tim_rt_probe_desc* desc, const float* dirs,
                         const float* sh_basis, uint32_t probe_begin, uint32_t probe_end, uint32_t* trace_out,
                         float* irradiance, uint16_t* sh9_fp16, float* sh9_fp32, float* octa, tim_rt_stats* stats) {
    int rc = check_ctx(c);
    if (rc) return rc;
    Scene* s = find_scene(c, id);
    if (!s) return TIM_RT_ENOTFOUND;
    if (!dirs || !sh_basis || !sh9_fp16) {
        set_error("tim_rt_update_probes: null argument");
        return TIM_RT_EINVAL;
    }
    ProbePlan P;
    if ((rc = probe_plan(s, desc, probe_begin, probe_end, "tim_rt_update_probes", &P))) return rc;
    const uint32_t nd = P.args.nd, np = P.args.np, side = P.side;
    const uint64_t n = P.n, total = P.total;
    if ((rc = ensure(c, c->p_dirs, 16ull * nd)) || (rc = ensure(c, c->p_basis, 36ull * nd)) ||
        (rc = ensure(c, c->p_out, 32ull * n)) || (rc = ensure(c, c->p_nid, 4ull * n)) ||
        (rc = ensure(c, c->p_irr, 12ull * n)) || (rc = ensure(c, c->p_sh16, 56ull * total)) ||
        (rc = ensure(c, c->q_rays, 32ull * n * probe_queue_kinds())) ||
        (rc = ensure(c, c->q_pixel, 4ull * n * probe_queue_kinds())))
        return rc;
    if (sh9_fp32 && (rc = ensure(c, c->p_sh32, 108ull * np))) return rc;
    if (octa && side && (rc = ensure(c, c->p_octa, 768ull * np))) return rc;
    ProbeArgs d = P.args;
    d.dirs = static_cast<const float4*>(c->p_dirs.ptr);
    d.basis = static_cast<const float*>(c->p_basis.ptr);
    uint32_t* ctr = static_cast<uint32_t*>(c->counters.ptr);
    TIMRT_CUDA(cudaEventRecord(c->ev[0], c->stream));
    TIMRT_CUDA(cudaMemcpyAsync(c->p_dirs.ptr, dirs, 16ull * nd, cudaMemcpyHostToDevice, c->stream));
    TIMRT_CUDA(cudaMemcpyAsync(c->p_basis.ptr, sh_basis, 36ull * nd, cudaMemcpyHostToDevice, c->stream));
    TIMRT_CUDA(cudaMemcpyAsync(c->p_sh16.ptr, sh9_fp16, 56ull * total, cudaMemcpyHostToDevice, c->stream));
    TIMRT_CUDA(cudaMemsetAsync(ctr, 0, 4 * kCamCounterWords, c->stream));
    TIMRT_CUDA(cudaEventRecord(c->ev[1], c->stream));
    LaunchConfig cfg = cfg_for(c, s, (desc->flags & TIM_RT_PROBE_WIDE) != 0);
    cfg.primary_binary = (desc->flags & TIM_RT_PROBE_PRIMARY_BINARY) != 0;
    cfg.phase_ev = c->pev;
    TIMRT_CUDA(launch_probes(s->view, d, static_cast<uint32_t*>(c->p_out.ptr), static_cast<uint32_t*>(c->p_nid.ptr),
                             static_cast<tim_rt_ray*>(c->q_rays.ptr), static_cast<uint32_t*>(c->q_pixel.ptr), ctr,
                             ctr + kErrWord, static_cast<float*>(c->p_irr.ptr), static_cast<uint16_t*>(c->p_sh16.ptr),
                             sh9_fp32 ? static_cast<float*>(c->p_sh32.ptr) : nullptr,
                             (octa && side) ? static_cast<float*>(c->p_octa.ptr) : nullptr, side, c->stream, cfg));
    TIMRT_CUDA(cudaEventRecord(c->ev[2], c->stream));
    TIMRT_CUDA(cudaMemcpyAsync(sh9_fp16, c->p_sh16.ptr, 56ull * total, cudaMemcpyDeviceToHost, c->stream));
    if (trace_out) TIMRT_CUDA(cudaMemcpyAsync(trace_out, c->p_out.ptr, 32ull * n, cudaMemcpyDeviceToHost, c->stream));
    if (irradiance) TIMRT_CUDA(cudaMemcpyAsync(irradiance, c->p_irr.ptr, 12ull * n, cudaMemcpyDeviceToHost, c->stream));
    if (sh9_fp32) TIMRT_CUDA(cudaMemcpyAsync(sh9_fp32, c->p_sh32.ptr, 108ull * np, cudaMemcpyDeviceToHost, c->stream));
    if (octa && side) TIMRT_CUDA(cudaMemcpyAsync(octa, c->p_octa.ptr, 768ull * np, cudaMemcpyDeviceToHost, c->stream));
    uint32_t qn = 0;
    TIMRT_CUDA(cudaMemcpyAsync(&qn, ctr + kCamTotalWord, 4, cudaMemcpyDeviceToHost, c->stream));
    TIMRT_CUDA(cudaEventRecord(c->ev[3], c->stream));
    TIMRT_CUDA(cudaStreamSynchronize(c->stream));
    if ((rc = check_device_error(c))) return rc;
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->primary_rays = n;
        stats->shadow_rays = qn;
        stats->rays = n + qn;
        cudaEventElapsedTime(&stats->kernel_ms, c->ev[1], c->ev[2]);
        cudaEventElapsedTime(&stats->total_ms, c->ev[0], c->ev[3]);
        cudaEventElapsedTime(&stats->primary_ms, c->pev[0], c->pev[1]);
        cudaEventElapsedTime(&stats->gen_ms, c->pev[1], c->pev[2]);
        cudaEventElapsedTime(&stats->secondary_ms, c->pev[2], c->pev[3]);
    }
    return TIM_RT_OK;
}

int tim_rt_trace_camera(tim_rt_ctx* c, tim_rt_scene_id id, const tim_rt_pass_data* pd, uint32_t flags, uint32_t seed,
                        const uint32_t* tile_counts, const uint32_t* tile_lists, uint32_t* out, uint32_t* bounce_out,
                        tim_rt_stats* stats) {
    int rc = check_ctx(c);
    if (rc) return rc;
    Scene* s = find_scene(c, id);
    if (!s) return TIM_RT_ENOTFOUND;
    if (!out) {
        set_error("tim_rt_trace_camera: null output");
        return TIM_RT_EINVAL;
    }
    const bool device_cull = (flags & TIM_RT_CAM_DEVICE_CULL) != 0;
    if (device_cull && !(flags & TIM_RT_CAM_TILE_LIGHTS)) {
        set_error("tim_rt_trace_camera: TIM_RT_CAM_DEVICE_CULL needs TIM_RT_CAM_TILE_LIGHTS");
        return TIM_RT_EINVAL;
    }
    uint64_t qcap = 0;
    if ((rc = camera_prepare(c, s, pd, flags, device_cull || (tile_counts && tile_lists), bounce_out != nullptr, &qcap)))
        return rc;
    const uint32_t W = pd->frameSize[0], H = pd->frameSize[1];
    const uint64_t npix = (uint64_t)W * H;
    const uint64_t tiles = (uint64_t)((W + 15) / 16) * ((H + 15) / 16);
    if ((rc = ensure(c, c->cam_out, 32ull * npix))) return rc;
    if ((flags & TIM_RT_CAM_BOUNCE) && (rc = ensure(c, c->cam_bounce, 16ull * npix))) return rc;
    if ((flags & TIM_RT_CAM_TILE_LIGHTS) &&
        ((rc = ensure(c, c->tiles_counts, 4ull * tiles)) || (rc = ensure(c, c->tiles_lists, 64ull * tiles))))
        return rc;
    uint32_t* ctr = static_cast<uint32_t*>(c->counters.ptr);
    TIMRT_CUDA(cudaEventRecord(c->ev[0], c->stream));
    if (device_cull) {
        TIMRT_CUDA(launch_cull_lights(s->view, *pd, (W + 15u) / 16u, (H + 15u) / 16u,
                                      static_cast<uint32_t*>(c->tiles_counts.ptr),
                                      static_cast<uint32_t*>(c->tiles_lists.ptr), c->stream));
    } else if (flags & TIM_RT_CAM_TILE_LIGHTS) {
        TIMRT_CUDA(cudaMemcpyAsync(c->tiles_counts.ptr, tile_counts, 4ull * tiles, cudaMemcpyHostToDevice, c->stream));
        TIMRT_CUDA(cudaMemcpyAsync(c->tiles_lists.ptr, tile_lists, 64ull * tiles, cudaMemcpyHostToDevice, c->stream));
    }
    const bool count = (flags & TIM_RT_CAM_COUNT) != 0;
    if (count) TIMRT_CUDA(cudaMemsetAsync(c->dstats.ptr, 0, 128, c->stream));
    LaunchConfig cam_cfg = cfg_for(c, s, (flags & TIM_RT_CAM_WIDE) != 0, count);
    // TIM_RT_CAM_PIPELINED: bands of output rows (equal, at least 64 rows each, up to
    // 8). The frame traces as one launch sequence whose secondary trace takes the
    // bands in order and raises each band's host flag once its records are final;
    // this thread starts each band's copy as soon as its flag is up, so the copies
    // run while the later bands trace.
    const uint32_t tile_rows = (H + 3u) / 4u;
    const uint32_t bands = (flags & TIM_RT_CAM_PIPELINED) ? std::min<uint32_t>(kMaxCamBands, std::max<uint32_t>(1u, tile_rows / 16u))
                                                           : 1u;
    CameraBands cb{};
    cb.n = bands;
    for (uint32_t b = 0; b < bands; ++b) cb.row[b] = 4u * (uint32_t)((uint64_t)tile_rows * b / bands);
    cb.row[bands] = H;
    uint32_t* cctr = ctr;
    if (bands > 1u) {
        if ((rc = ensure(c, c->band_ctr, 4ull * cam_counter_words(kMaxCamBands)))) return rc;
        cctr = static_cast<uint32_t*>(c->band_ctr.ptr);
        for (uint32_t b = 0; b < kMaxCamBands; ++b) c->band_flags[b] = 0u;   // no kernel of this context runs
        cb.flags = c->band_flags_dev;
    }
    cam_cfg.phase_ev = c->pev;
    uint64_t* acc = static_cast<uint64_t*>(c->ray_acc.ptr);
    TIMRT_CUDA(cudaMemsetAsync(acc, 0, 8, c->stream));
    TIMRT_CUDA(cudaMemsetAsync(cctr, 0, 4ull * cam_counter_words(bands), c->stream));
    TIMRT_CUDA(cudaEventRecord(c->ev[1], c->stream));
    TIMRT_CUDA(launch_camera(s->view, *pd, flags, seed, static_cast<const uint32_t*>(c->tiles_counts.ptr),
                             static_cast<const uint32_t*>(c->tiles_lists.ptr), static_cast<uint32_t*>(c->cam_out.ptr),
                             (flags & TIM_RT_CAM_BOUNCE) ? static_cast<uint32_t*>(c->cam_bounce.ptr) : nullptr,
                             static_cast<uint32_t*>(c->cam_nid.ptr), static_cast<tim_rt_ray*>(c->q_rays.ptr),
                             static_cast<uint32_t*>(c->q_pixel.ptr), (uint32_t)qcap, cctr, ctr + kErrWord, acc,
                             c->stream, cam_cfg, 0u, H, &cb));
    TIMRT_CUDA(cudaEventRecord(c->ev[2], c->stream));
    if (bands == 1u) {
        TIMRT_CUDA(cudaMemcpyAsync(out, c->cam_out.ptr, 32ull * npix, cudaMemcpyDeviceToHost, c->stream));
        if (flags & TIM_RT_CAM_BOUNCE)
            TIMRT_CUDA(cudaMemcpyAsync(bounce_out, c->cam_bounce.ptr, 16ull * npix, cudaMemcpyDeviceToHost, c->stream));
    } else {
        // Band b's copy starts when its flag is up. Should the trace end without a
        // flag (an error ended a kernel early), the remaining copies wait for its end.
        // The flag is polled in host memory; the trace's end event (a driver call)
        // only every 64th poll.
        bool ended = false;
        uint32_t polls = 0;
        for (uint32_t b = 0; b < bands;) {
            if (!ended && !reinterpret_cast<volatile uint32_t*>(c->band_flags)[b]) {
                if (++polls % 64u != 0u) continue;
                const cudaError_t q = cudaEventQuery(c->ev[2]);
                if (q == cudaErrorNotReady) continue;
                ended = true;
                TIMRT_CUDA(cudaStreamWaitEvent(c->cstream, c->ev[2], 0));
            }
            const uint64_t p0 = (uint64_t)W * cb.row[b], np = (uint64_t)W * (cb.row[b + 1] - cb.row[b]);
            TIMRT_CUDA(cudaMemcpyAsync(out + 8ull * p0, static_cast<uint32_t*>(c->cam_out.ptr) + 8ull * p0, 32ull * np,
                                       cudaMemcpyDeviceToHost, c->cstream));
            if (flags & TIM_RT_CAM_BOUNCE)
                TIMRT_CUDA(cudaMemcpyAsync(bounce_out + 4ull * p0, static_cast<uint32_t*>(c->cam_bounce.ptr) + 4ull * p0,
                                           16ull * np, cudaMemcpyDeviceToHost, c->cstream));
            ++b;
        }
        TIMRT_CUDA(cudaEventRecord(c->copy_ev, c->cstream));
        TIMRT_CUDA(cudaStreamWaitEvent(c->stream, c->copy_ev, 0));
    }
    uint64_t traced = 0;
    TIMRT_CUDA(cudaMemcpyAsync(&traced, acc, 8, cudaMemcpyDeviceToHost, c->stream));
    TIMRT_CUDA(cudaEventRecord(c->ev[3], c->stream));
    TIMRT_CUDA(cudaStreamSynchronize(c->stream));
    if ((rc = check_device_error(c))) return rc;
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        const uint64_t primary = (uint64_t)W * (H - 1u);
        stats->primary_rays = primary;
        stats->rays = traced;
        stats->shadow_rays = traced - primary;   // all secondary rays (shadow, probe-visibility, bounce)
        cudaEventElapsedTime(&stats->kernel_ms, c->ev[1], c->ev[2]);
        cudaEventElapsedTime(&stats->total_ms, c->ev[0], c->ev[3]);
        cudaEventElapsedTime(&stats->primary_ms, c->pev[0], c->pev[1]);
        cudaEventElapsedTime(&stats->gen_ms, c->pev[1], c->pev[2]);
        cudaEventElapsedTime(&stats->secondary_ms, c->pev[2], c->pev[3]);
        if (count) read_counts(c, stats);
    }
    return TIM_RT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- batched multi-scene trace

namespace {

// Sort scratch of a batch: keys[2] (8 B per ray each), vals[2] (4 B per ray each),
// then the radix sort's temporary storage, each part 256-byte aligned.
int batch_sort_scratch(tim_rt_ctx* c, tim_rt_batch* b) {
    if (b->sort.ptr) return TIM_RT_OK;
    auto up = [](uint64_t x) { return (x + 255ull) & ~255ull; };
    const uint64_t n = b->total;
    const uint64_t o_k1 = up(8 * n), o_v0 = o_k1 + up(8 * n), o_v1 = o_v0 + up(4 * n), o_t = o_v1 + up(4 * n);
    const size_t tb = multi_sort_temp_bytes(b->total);
    int rc = dev_alloc(c, b->sort, o_t + tb);
    if (rc) return rc;
    uint8_t* base = static_cast<uint8_t*>(b->sort.ptr);
    b->ss.keys[0] = reinterpret_cast<unsigned long long*>(base);
    b->ss.keys[1] = reinterpret_cast<unsigned long long*>(base + o_k1);
    b->ss.vals[0] = reinterpret_cast<uint32_t*>(base + o_v0);
    b->ss.vals[1] = reinterpret_cast<uint32_t*>(base + o_v1);
    b->ss.temp = base + o_t;
    b->ss.temp_bytes = tb;
    return TIM_RT_OK;
}

bool live_batch(tim_rt_ctx* c, const tim_rt_batch* b) {
    if (b && c->batches.count(const_cast<tim_rt_batch*>(b))) return true;
    set_error("unknown batch");
    return false;
}

int batch_run(tim_rt_ctx* c, tim_rt_batch* b, const LaunchConfig& cfg, bool wide, cudaStream_t st) {
    if (b->total == 0) return TIM_RT_OK;
    int rc;
    if (cfg.ray_sort != TIM_RT_SORT_NONE && (rc = batch_sort_scratch(c, b))) return rc;
    int depth = wide ? b->wide_depth : b->depth;
    if (cfg.stack_depth > depth) depth = cfg.stack_depth;
    uint32_t* err = static_cast<uint32_t*>(c->counters.ptr) + kErrWord;
    TIMRT_CUDA(launch_multi(b->d_views, b->d_jobs, b->njobs, b->total, b->d_counter, err, depth, wide,
                            cfg.ray_sort != TIM_RT_SORT_NONE ? &b->ss : nullptr, st, cfg));
    return TIM_RT_OK;
}

}  // namespace

extern "C" {

int tim_rt_batch_create(tim_rt_ctx* c, const tim_rt_job* jobs, uint32_t num_jobs, uint32_t flags,
                        tim_rt_batch** out) {
    int rc = check_ctx(c);
    if (rc) return rc;
    if (!out || (num_jobs && !jobs) || (flags & ~TIM_RT_BATCH_WIDE)) {
        set_error("tim_rt_batch_create: null argument or unknown flag");
        return TIM_RT_EINVAL;
    }
    *out = nullptr;
    const bool wide = (flags & TIM_RT_BATCH_WIDE) != 0;
    std::map<uint32_t, uint32_t> slot_of;
    std::vector<SceneView> views;
    std::vector<MultiJob> table;
    auto b = std::make_unique<tim_rt_batch>();
    uint64_t total = 0;
    for (uint32_t j = 0; j < num_jobs; ++j) {
        const tim_rt_job& J = jobs[j];
        Scene* s = find_scene(c, J.scene);
        if (!s) return TIM_RT_ENOTFOUND;
        if (J.mode > TIM_RT_MODE_PER_RAY || (J.n && (!J.d_rays || !J.d_hit)) ||
            (reinterpret_cast<uintptr_t>(J.d_rays) & 15u) || (reinterpret_cast<uintptr_t>(J.d_hit) & 15u) ||
            (reinterpret_cast<uintptr_t>(J.d_bary) & 7u) || (reinterpret_cast<uintptr_t>(J.d_leaf_nid) & 3u)) {
            set_error("tim_rt_batch_create: job " + std::to_string(j) + ": bad mode, null or misaligned buffer");
            return TIM_RT_EINVAL;
        }
        if (wide && !s->has_wide) {
            set_error("tim_rt_batch_create: scene " + std::to_string(J.scene) +
                      " was uploaded without TIM_RT_UPLOAD_QUANT8");
            return TIM_RT_EUNSUPPORTED;
        }
        if (J.n == 0) continue;
        auto it = slot_of.find(J.scene);
        if (it == slot_of.end()) {
            it = slot_of.emplace(J.scene, (uint32_t)views.size()).first;
            views.push_back(s->view);
            b->scene_ids.push_back(J.scene);
            b->depth = std::max(b->depth, (int)s->depth);
            b->wide_depth = std::max(b->wide_depth, (int)s->view.wide_depth);
        }
        MultiJob m{};
        m.rays = J.d_rays;
        m.hit = reinterpret_cast<uint4*>(J.d_hit);
        m.nid = J.d_leaf_nid;
        m.bary = reinterpret_cast<float2*>(J.d_bary);
        m.scene_slot = it->second;
        m.mode = J.mode;
        m.first = (uint32_t)total;
        m.n = J.n;
        for (int a = 0; a < 3; ++a) {
            m.lo[a] = s->bounds[a];
            const float ext = s->bounds[3 + a] - s->bounds[a];
            m.scale[a] = ext > 0.f ? 1024.0f / ext : 0.f;
        }
        table.push_back(m);
        total += J.n;
        if (total > 0x7FFFFFFFull) {
            set_error("tim_rt_batch_create: more than 2^31 - 1 rays in one batch");
            return TIM_RT_EINVAL;
        }
    }
    b->njobs = (uint32_t)table.size();
    b->total = (uint32_t)total;
    b->wide = wide;
    const uint64_t vb = (sizeof(SceneView) * views.size() + 15ull) & ~15ull;
    const uint64_t jb = (sizeof(MultiJob) * table.size() + 15ull) & ~15ull;
    if ((rc = dev_alloc(c, b->table, vb + jb + 16))) return rc;
    uint8_t* base = static_cast<uint8_t*>(b->table.ptr);
    b->d_views = reinterpret_cast<SceneView*>(base);
    b->d_jobs = reinterpret_cast<MultiJob*>(base + vb);
    b->d_counter = reinterpret_cast<uint32_t*>(base + vb + jb);
    if ((!views.empty() && cudaMemcpy(b->d_views, views.data(), sizeof(SceneView) * views.size(),
                                      cudaMemcpyHostToDevice) != cudaSuccess) ||
        (!table.empty() && cudaMemcpy(b->d_jobs, table.data(), sizeof(MultiJob) * table.size(),
                                      cudaMemcpyHostToDevice) != cudaSuccess)) {
        dev_free(c, b->table);
        set_error("tim_rt_batch_create: host-to-device copy of the job table failed");
        return TIM_RT_EDEVICE;
    }
    for (uint32_t id : b->scene_ids) c->scenes[id]->batch_refs++;
    *out = b.release();
    c->batches.insert(*out);
    return TIM_RT_OK;
}

int tim_rt_batch_launch(tim_rt_ctx* c, tim_rt_batch* b, void* cuda_stream) {
    int rc = check_ctx(c);
    if (rc) return rc;
    if (!live_batch(c, b)) return TIM_RT_EINVAL;
    cudaStream_t st = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : c->stream;
    LaunchConfig cfg = c->cfg;
    cfg.stats = nullptr;
    return batch_run(c, b, cfg, b->wide, st);
}

int tim_rt_batch_info(tim_rt_ctx* c, const tim_rt_batch* b, uint64_t* rays, uint64_t* bytes) {
    if (!c || !live_batch(c, b)) return TIM_RT_EINVAL;
    if (rays) *rays = b->total;
    if (bytes) *bytes = b->table.bytes + b->sort.bytes;
    return TIM_RT_OK;
}

int tim_rt_batch_destroy(tim_rt_ctx* c, tim_rt_batch* b) {
    int rc = check_ctx(c);
    if (rc) return rc;
    if (!b) return TIM_RT_OK;
    if (!live_batch(c, b)) return TIM_RT_EINVAL;
    cudaStreamSynchronize(c->stream);
    cudaDeviceSynchronize();   // launches may have gone to caller streams
    for (uint32_t id : b->scene_ids) {
        auto it = c->scenes.find(id);
        if (it != c->scenes.end() && it->second->batch_refs) it->second->batch_refs--;
    }
    dev_free(c, b->table);
    dev_free(c, b->sort);
    c->batches.erase(b);
    delete b;
    return TIM_RT_OK;
}

int tim_rt_autotune_batch(tim_rt_ctx* c, tim_rt_batch* b, uint32_t flags, uint32_t reps, tim_rt_tune_result* res) {
    int rc = check_ctx(c);
    if (rc) return rc;
    if (!live_batch(c, b) || !res || (flags & ~TIM_RT_TUNE_WIDTH)) {
        if (!res) set_error("tim_rt_autotune_batch: null result");
        return TIM_RT_EINVAL;
    }
    std::memset(res, 0, sizeof(*res));
    reps = reps == 0 ? 3 : std::min(reps, 50u);
    bool can_wide = true;
    for (uint32_t id : b->scene_ids) can_wide = can_wide && c->scenes[id]->has_wide;
    cudaEvent_t e0, e1;
    TIMRT_CUDA(cudaEventCreate(&e0));
    TIMRT_CUDA(cudaEventCreate(&e1));
    int err = TIM_RT_OK;
    uint32_t tried = 0;
    // median device time of one launch under (cfg, wide); negative on error
    auto time_cfg = [&](const LaunchConfig& cfg, bool wide) -> float {
        // a ray-sort key whose scratch does not fit the budget is not a candidate
        if (cfg.ray_sort != TIM_RT_SORT_NONE && batch_sort_scratch(c, b) != TIM_RT_OK) return -1.f;
        ++tried;
        std::vector<float> ms;
        for (uint32_t r = 0; r <= reps; ++r) {
            cudaEventRecord(e0, c->stream);
            int rc2 = batch_run(c, b, cfg, wide, c->stream);
            cudaEventRecord(e1, c->stream);
            if (rc2 || cudaEventSynchronize(e1) != cudaSuccess) {
                err = rc2 ? rc2 : TIM_RT_EDEVICE;
                return -1.f;
            }
            float t = 0.f;
            cudaEventElapsedTime(&t, e0, e1);
            if (r) ms.push_back(t);   // launch 0 is the warm-up
        }
        std::sort(ms.begin(), ms.end());
        return ms[ms.size() / 2];
    };
    LaunchConfig best = c->cfg;
    best.stats = nullptr;
    best.phase_ev = nullptr;
    bool best_wide = b->wide;
    float best_ms = time_cfg(best, best_wide);
    res->start_ms = best_ms;
    auto consider = [&](LaunchConfig cand, bool wide) {
        if (err) return;
        const float t = time_cfg(cand, wide);
        if (t >= 0.f && t < best_ms) {
            best_ms = t;
            best = cand;
            best_wide = wide;
        }
    };
    for (int pass = 0; pass < 2 && !err; ++pass) {
        for (int blk : {64, 128, 256}) {
            LaunchConfig cand = best;
            if (cand.block == blk) continue;
            cand.block = blk;
            consider(cand, best_wide);
        }
        for (int refill : {1, 2, 4, 8, 12, 16, 20, 24, 28, 32}) {
            LaunchConfig cand = best;
            if (cand.refill_min == refill) continue;
            cand.refill_min = refill;
            consider(cand, best_wide);
        }
        for (int srt : {0, 1, 2}) {
            LaunchConfig cand = best;
            if (cand.ray_sort == srt) continue;
            cand.ray_sort = srt;
            consider(cand, best_wide);
        }
        for (int sw : {0, 4, 8, 12, 16}) {
            LaunchConfig cand = best;
            if (cand.phase_switch == sw) continue;
            cand.phase_switch = sw;
            consider(cand, best_wide);
        }
        for (int sd : {0, 32}) {
            LaunchConfig cand = best;
            if (cand.stack_depth == sd) continue;
            cand.stack_depth = sd;
            consider(cand, best_wide);
        }
        if ((flags & TIM_RT_TUNE_WIDTH) && can_wide) consider(best, !best_wide);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err) return err;
    c->cfg.block = best.block;
    c->cfg.refill_min = best.refill_min;
    c->cfg.ray_sort = best.ray_sort;
    c->cfg.stack_depth = best.stack_depth;
    c->cfg.phase_switch = best.phase_switch;
    b->wide = best_wide;
    res->best.block = (uint32_t)best.block;
    res->best.stack_depth = (uint32_t)best.stack_depth;
    res->best.refill_min = (uint32_t)best.refill_min;
    res->best.ray_sort = (uint32_t)best.ray_sort;
    res->best.phase_switch = (uint32_t)best.phase_switch;
    res->wide = best_wide ? 1u : 0u;
    res->tried = tried;
    res->best_ms = best_ms;
    return TIM_RT_OK;
}

}  // extern "C"
