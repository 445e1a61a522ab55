// server.cu -- the serving loop of include/tim_rt.h (tim_rt_server_*): admission
// of trace and probe-update requests against a device arena, continuous batching
// of trace-request chunks into batched multi-scene launches (launch_multi),
// probe updates (launch_probes) on a stream of their own beside those launches,
// asynchronous result copies and latency statistics.
//
// Threads: callers submit and wait; one worker thread per server issues every
// CUDA call; CUDA host functions (cudaLaunchHostFunc) report step and request
// completion. The worker never holds the server mutex across a CUDA call, so a
// host function waiting for the mutex cannot stall a stream the worker waits on.
#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <set>
#include <thread>
#include <vector>
#include "context.h"

namespace timrt {
namespace {

using Clock = std::chrono::steady_clock;

inline uint64_t round256(uint64_t x) { return (x + 255ull) & ~255ull; }

// First-fit allocator over the server's device arena (offsets, 256-byte granules).
struct Arena {
    uint64_t size = 0, used = 0, peak = 0;
    std::map<uint64_t, uint64_t> free_;   // offset -> bytes
    void init(uint64_t n) {
        size = n;
        used = peak = 0;
        free_.clear();
        free_[0] = n;
    }
    bool alloc(uint64_t n, uint64_t& off) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            off = it->first;
            const uint64_t rest = it->second - n;
            free_.erase(it);
            if (rest) free_[off + n] = rest;
            used += n;
            peak = std::max(peak, used);
            return true;
        }
        return false;
    }
    void release(uint64_t off, uint64_t n) {
        used -= n;
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

struct Req {
    uint64_t ticket = 0;
    tim_rt_request r{};
    Scene* scene = nullptr;
    uint64_t off = 0, bytes = 0;
    uint64_t rays = 0;            // rays the request traces (probe updates: the probe rays)
    tim_rt_ray* d_rays = nullptr;
    uint4* d_hit = nullptr;
    uint32_t* d_nid = nullptr;
    float2* d_bary = nullptr;
    uint32_t issued = 0;          // rays handed to steps so far (worker only)
    bool first_chunk = true;      // the next step must wait for the upload
    bool last_planned = false;    // a planned step traces its last rays (under the server mutex)
    bool cancel = false;          // tim_rt_server_cancel took it back (under the server mutex)
    uint32_t planned = 0;         // rays assigned to planned steps (under the server mutex)
    Clock::time_point t_submit, t_admit;
    cudaEvent_t uploaded = nullptr;
    // probe-field update requests
    bool probe = false;
    tim_rt_probe_request pr{};
    tim_rt_probe_desc pdesc{};
    ProbePlan plan;
    cudaEvent_t ran = nullptr;
    float4* d_dirs = nullptr;
    float* d_basis = nullptr;
    uint32_t* d_out = nullptr;
    uint32_t* d_pnid = nullptr;
    float* d_irr = nullptr;
    uint16_t* d_sh16 = nullptr;
    tim_rt_ray* d_qrays = nullptr;
    uint32_t* d_qpix = nullptr;
    uint32_t* d_ctr = nullptr;
    float* d_octa = nullptr;
};

// Device staging of a probe-update request, in arena order (256-byte aligned parts).
struct ProbeStaging {
    uint64_t dirs, basis, out, nid, irr, sh16, qrays, qpix, ctr, octa;
    uint64_t total() const { return dirs + basis + out + nid + irr + sh16 + qrays + qpix + ctr + octa; }
};
inline ProbeStaging probe_staging(const ProbePlan& P, bool octa) {
    const uint64_t n = P.n, nd = P.args.nd, kinds = probe_queue_kinds();
    ProbeStaging b;
    b.dirs = round256(16 * nd);
    b.basis = round256(36 * nd);
    b.out = round256(32 * n);
    b.nid = round256(4 * n);
    b.irr = round256(12 * n);
    b.sh16 = round256(56 * P.total);
    b.qrays = round256(32 * n * kinds);
    b.qpix = round256(4 * n * kinds);
    b.ctr = round256(4ull * kCamCounterWords);
    b.octa = (octa && P.side) ? round256(768ull * P.args.np) : 0;
    return b;
}

struct Slot {
    DevBuf dev;                   // SceneView[max_jobs], MultiJob[max_jobs], counter
    void* host = nullptr;         // pinned staging of the two tables (mapped into the device's address space)
    const void* host_dev = nullptr;   // its device address
    SceneView* d_views = nullptr;
    MultiJob* d_jobs = nullptr;
    uint32_t* d_counter = nullptr;
    cudaEvent_t done = nullptr;
    cudaEvent_t t_begin = nullptr, t_end = nullptr;   // around the step's kernel, for the GPU-busy time
    bool timing_pending = false;   // t_begin / t_end hold a step not yet added to gpu_busy_ms (under the mutex)
};

// Copies a step's tables from the mapped pinned staging into device memory. A
// kernel, not a copy: host-to-device copies of all streams share the copy
// engine's queue, so a table copy on the compute stream would wait behind every
// ray upload queued before it.
__global__ void k_stage_tables(uint32_t* dv, const uint32_t* sv, uint32_t nv, uint32_t* dj, const uint32_t* sj,
                               uint32_t nj) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nv + nj; i += gridDim.x * blockDim.x) {
        if (i < nv) dv[i] = sv[i];
        else dj[i - nv] = sj[i - nv];
    }
}

}  // namespace
}  // namespace timrt

using namespace timrt;

struct tim_rt_server {
    tim_rt_ctx* ctx = nullptr;
    tim_rt_server_params p{};
    bool wide = false;
    DevBuf arena_buf;
    Arena arena;                  // worker-only
    cudaStream_t up = nullptr, comp = nullptr, down = nullptr;
    cudaStream_t probe = nullptr;      // probe updates, beside the trace steps
    std::vector<Slot> slots;

    std::mutex m;
    std::condition_variable cv;        // wakes the worker
    std::condition_variable cv_done;   // wakes waiters
    std::deque<Req*> waiting;          // submitted, not admitted
    std::vector<Req*> finished;        // completed by a host function, resources not yet released
    std::vector<int> free_slots;
    std::map<uint64_t, Req*> pending;  // every request not yet completed
    uint64_t next_ticket = 1;
    bool stop = false;
    int error = TIM_RT_OK;
    std::string error_msg;
    // statistics (under m)
    std::vector<float> lat_ms, queue_ms;
    uint64_t submitted = 0, completed = 0, rays_completed = 0, steps = 0;
    uint64_t cancelled = 0, step_requests = 0;
    uint32_t max_step_requests = 0, max_inflight = 0;
    double gpu_busy_ms = 0.0;
    std::vector<Req*> cancel_q;        // admitted requests taken back, for the worker
    std::set<uint64_t> cancelled_tickets;   // completed by cancellation (tim_rt_server_wait reports it)
    bool t0_set = false;
    Clock::time_point t0;

    std::deque<Req*> active;           // worker-only: admitted, rays left to issue
    int last_slot = -1;                // worker-only: slot of the step issued last
    bool last_started = true;          // worker-only: that step has begun on the GPU
    std::thread worker;
};

namespace {

struct DoneMsg {
    tim_rt_server* s;
    std::vector<Req*> reqs;
};

struct SlotMsg {
    tim_rt_server* s;
    int slot;
};

void CUDART_CB on_requests_done(void* p) {
    DoneMsg* msg = static_cast<DoneMsg*>(p);
    tim_rt_server* s = msg->s;
    const Clock::time_point now = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->m);
        for (Req* r : msg->reqs) {
            s->lat_ms.push_back(std::chrono::duration<float, std::milli>(now - r->t_submit).count());
            s->queue_ms.push_back(std::chrono::duration<float, std::milli>(r->t_admit - r->t_submit).count());
            s->completed++;
            s->rays_completed += r->rays;
            s->pending.erase(r->ticket);
            s->finished.push_back(r);
        }
    }
    s->cv.notify_all();
    s->cv_done.notify_all();
    delete msg;
}

// Runs on the compute stream after every step that traced part of the cancelled
// requests: they complete without results.
void CUDART_CB on_requests_cancelled(void* p) {
    DoneMsg* msg = static_cast<DoneMsg*>(p);
    tim_rt_server* s = msg->s;
    {
        std::lock_guard<std::mutex> lk(s->m);
        for (Req* r : msg->reqs) {
            s->cancelled++;
            s->cancelled_tickets.insert(r->ticket);
            s->pending.erase(r->ticket);
            s->finished.push_back(r);
        }
    }
    s->cv.notify_all();
    s->cv_done.notify_all();
    delete msg;
}

void CUDART_CB on_slot_free(void* p) {
    SlotMsg* msg = static_cast<SlotMsg*>(p);
    {
        std::lock_guard<std::mutex> lk(msg->s->m);
        msg->s->free_slots.push_back(msg->slot);
    }
    msg->s->cv.notify_all();
    delete msg;
}

// One planned step: request chunks and the requests whose last chunk it traces.
struct Plan {
    int slot = -1;
    std::vector<std::pair<Req*, uint32_t>> chunks;   // (request, rays)
    std::vector<Req*> finishing;
};

void fail_all(tim_rt_server* s, int code, const std::string& msg) {
    std::lock_guard<std::mutex> lk(s->m);
    if (s->error == TIM_RT_OK) {
        s->error = code;
        s->error_msg = msg;
    }
    s->cv_done.notify_all();
}

// A request's rays are on the device (its upload has completed, or an earlier
// step already traced part of it).
bool uploaded(const Req* r) {
    if (!r->first_chunk) return true;
    return r->uploaded && cudaEventQuery(r->uploaded) == cudaSuccess;
}

// Plans the next step under the mutex: an equal share of max_rays_per_step for
// every admitted request with rays left, then the rest in admission order. Only
// requests whose rays are already on the device take part, so a step never waits
// for uploads that later admissions queued; when none is ready, the oldest request
// alone (its upload was queued first; the step waits for it on the device).
void plan_step(tim_rt_server* s, Plan& P) {
    const uint32_t cap = s->p.max_rays_per_step;
    std::vector<Req*> cand;
    for (Req* r : s->active) {
        if (cand.size() >= s->p.max_jobs_per_step) break;
        if (uploaded(r)) cand.push_back(r);
    }
    if (cand.empty()) cand.push_back(s->active.front());   // its upload was queued first
    const size_t k = cand.size();
    std::vector<uint32_t> take(k, 0);
    const uint32_t share = std::max<uint32_t>(1u, cap / (uint32_t)k);
    uint64_t used = 0;
    for (size_t i = 0; i < k; ++i) {
        Req* r = cand[i];
        take[i] = std::min<uint32_t>(r->r.n - r->planned, share);
        used += take[i];
    }
    for (size_t i = 0; i < k && used < cap; ++i) {
        Req* r = cand[i];
        const uint32_t extra = (uint32_t)std::min<uint64_t>(r->r.n - r->planned - take[i], cap - used);
        take[i] += extra;
        used += extra;
    }
    for (size_t i = 0; i < k; ++i) {
        if (!take[i]) continue;
        P.chunks.push_back({cand[i], take[i]});
        cand[i]->planned += take[i];
        if (cand[i]->planned == cand[i]->r.n) cand[i]->last_planned = true;
    }
}

int issue_step(tim_rt_server* s, Plan& P) {
    Slot& sl = s->slots[P.slot];
    const uint32_t maxj = s->p.max_jobs_per_step;
    SceneView* hv = static_cast<SceneView*>(sl.host);
    MultiJob* hj = reinterpret_cast<MultiJob*>(static_cast<uint8_t*>(sl.host) + round256(sizeof(SceneView) * maxj));
    std::map<Scene*, uint32_t> slot_of;
    int depth = 1;
    uint32_t total = 0, nj = 0;
    for (auto& ch : P.chunks) {
        Req* r = ch.first;
        auto it = slot_of.find(r->scene);
        if (it == slot_of.end()) {
            it = slot_of.emplace(r->scene, (uint32_t)slot_of.size()).first;
            hv[it->second] = r->scene->view;
            depth = std::max(depth, s->wide ? (int)r->scene->view.wide_depth : (int)r->scene->depth);
        }
        MultiJob& J = hj[nj++];
        std::memset(&J, 0, sizeof(J));
        J.rays = r->d_rays + r->issued;
        J.hit = r->d_hit + r->issued;
        J.nid = r->d_nid ? r->d_nid + r->issued : nullptr;
        J.bary = r->d_bary ? r->d_bary + r->issued : nullptr;
        J.scene_slot = it->second;
        J.mode = r->r.mode;
        J.first = total;
        J.n = ch.second;
        total += ch.second;
        if (r->first_chunk) {
            if (cudaStreamWaitEvent(s->comp, r->uploaded, 0) != cudaSuccess) return TIM_RT_EDEVICE;
            r->first_chunk = false;
        }
        r->issued += ch.second;
    }
    const uint64_t vb = round256(sizeof(SceneView) * maxj);
    static_assert(sizeof(SceneView) % 4 == 0 && sizeof(MultiJob) % 4 == 0, "tables are copied in 4-byte words");
    const uint32_t nvw = (uint32_t)(sizeof(SceneView) * slot_of.size() / 4), njw = (uint32_t)(sizeof(MultiJob) * nj / 4);
    const uint32_t* hd = static_cast<const uint32_t*>(sl.host_dev);
    k_stage_tables<<<4, 256, 0, s->comp>>>(reinterpret_cast<uint32_t*>(sl.d_views), hd, nvw,
                                           reinterpret_cast<uint32_t*>(sl.d_jobs), hd + vb / 4, njw);
    if (cudaGetLastError() != cudaSuccess) return TIM_RT_EDEVICE;
    LaunchConfig cfg = s->ctx->cfg;
    cfg.stats = nullptr;
    cfg.phase_ev = nullptr;
    cfg.ray_sort = TIM_RT_SORT_NONE;
    if (cfg.stack_depth > depth) depth = cfg.stack_depth;
    uint32_t* err = static_cast<uint32_t*>(s->ctx->counters.ptr) + kErrWord;
    if (cudaEventRecord(sl.t_begin, s->comp) != cudaSuccess ||
        launch_multi(sl.d_views, sl.d_jobs, nj, total, sl.d_counter, err, depth, s->wide, nullptr, s->comp, cfg) !=
            cudaSuccess ||
        cudaEventRecord(sl.t_end, s->comp) != cudaSuccess)
        return TIM_RT_EDEVICE;
    {
        std::lock_guard<std::mutex> lk(s->m);
        sl.timing_pending = true;
    }
    if (cudaLaunchHostFunc(s->comp, on_slot_free, new SlotMsg{s, P.slot}) != cudaSuccess) return TIM_RT_EDEVICE;
    if (!P.finishing.empty()) {
        if (cudaEventRecord(sl.done, s->comp) || cudaStreamWaitEvent(s->down, sl.done, 0)) return TIM_RT_EDEVICE;
        for (Req* r : P.finishing) {
            const uint64_t n = r->r.n;
            if (cudaMemcpyAsync(r->r.hit, r->d_hit, 16ull * n, cudaMemcpyDeviceToHost, s->down) ||
                (r->d_nid && cudaMemcpyAsync(r->r.leaf_nid, r->d_nid, 4ull * n, cudaMemcpyDeviceToHost, s->down)) ||
                (r->d_bary && cudaMemcpyAsync(r->r.bary, r->d_bary, 8ull * n, cudaMemcpyDeviceToHost, s->down)))
                return TIM_RT_EDEVICE;
        }
        if (cudaLaunchHostFunc(s->down, on_requests_done, new DoneMsg{s, P.finishing}) != cudaSuccess)
            return TIM_RT_EDEVICE;
    }
    return TIM_RT_OK;
}

// Uploads nothing: the request's inputs were queued on the probe stream at
// admission. Runs the probe update on the probe stream, beside the trace steps
// (its small launches fill the SMs a step's tail leaves idle), then copies the
// FP16 field (and the texels) back and completes the request.
int issue_probe(tim_rt_server* s, Req* r) {
    ProbeArgs d = r->plan.args;
    d.dirs = r->d_dirs;
    d.basis = r->d_basis;
    LaunchConfig cfg = s->ctx->cfg;
    cfg.stats = nullptr;
    cfg.phase_ev = nullptr;
    cfg.wide = (r->pdesc.flags & TIM_RT_PROBE_WIDE) != 0 && r->scene->has_wide;
    cfg.primary_binary = (r->pdesc.flags & TIM_RT_PROBE_PRIMARY_BINARY) != 0;
    uint32_t* err = static_cast<uint32_t*>(s->ctx->counters.ptr) + kErrWord;
    if (cudaMemsetAsync(r->d_ctr, 0, 4ull * kCamCounterWords, s->probe) ||
        launch_probes(r->scene->view, d, r->d_out, r->d_pnid, r->d_qrays, r->d_qpix, r->d_ctr, err, r->d_irr,
                      r->d_sh16, nullptr, r->d_octa, r->d_octa ? r->plan.side : 0, s->probe, cfg) != cudaSuccess ||
        cudaEventCreateWithFlags(&r->ran, cudaEventDisableTiming) || cudaEventRecord(r->ran, s->probe) ||
        cudaStreamWaitEvent(s->down, r->ran, 0) ||
        cudaMemcpyAsync(r->pr.sh9_fp16, r->d_sh16, 56ull * r->plan.total, cudaMemcpyDeviceToHost, s->down) ||
        (r->d_octa && cudaMemcpyAsync(r->pr.octa, r->d_octa, 768ull * r->plan.args.np, cudaMemcpyDeviceToHost, s->down)))
        return TIM_RT_EDEVICE;
    if (cudaLaunchHostFunc(s->down, on_requests_done, new DoneMsg{s, {r}}) != cudaSuccess) return TIM_RT_EDEVICE;
    return TIM_RT_OK;
}

// Points a probe request's staging into its arena block and queues its uploads
// (a few hundred KB) on the probe stream, right ahead of the update itself:
// queued on the upload stream they would wait behind every ray upload admitted
// before them.
int stage_probe(tim_rt_server* s, Req* r, uint8_t* p) {
    const ProbeStaging b = probe_staging(r->plan, r->pr.octa != nullptr);
    r->d_dirs = reinterpret_cast<float4*>(p);
    p += b.dirs;
    r->d_basis = reinterpret_cast<float*>(p);
    p += b.basis;
    r->d_out = reinterpret_cast<uint32_t*>(p);
    p += b.out;
    r->d_pnid = reinterpret_cast<uint32_t*>(p);
    p += b.nid;
    r->d_irr = reinterpret_cast<float*>(p);
    p += b.irr;
    r->d_sh16 = reinterpret_cast<uint16_t*>(p);
    p += b.sh16;
    r->d_qrays = reinterpret_cast<tim_rt_ray*>(p);
    p += b.qrays;
    r->d_qpix = reinterpret_cast<uint32_t*>(p);
    p += b.qpix;
    r->d_ctr = reinterpret_cast<uint32_t*>(p);
    p += b.ctr;
    r->d_octa = b.octa ? reinterpret_cast<float*>(p) : nullptr;
    const uint64_t nd = r->plan.args.nd;
    if (cudaEventCreateWithFlags(&r->uploaded, cudaEventDisableTiming) ||
        cudaMemcpyAsync(r->d_dirs, r->pr.dirs, 16 * nd, cudaMemcpyHostToDevice, s->probe) ||
        cudaMemcpyAsync(r->d_basis, r->pr.sh_basis, 36 * nd, cudaMemcpyHostToDevice, s->probe) ||
        cudaMemcpyAsync(r->d_sh16, r->pr.sh9_fp16, 56ull * r->plan.total, cudaMemcpyHostToDevice, s->probe) ||
        cudaEventRecord(r->uploaded, s->probe))
        return TIM_RT_EDEVICE;
    return TIM_RT_OK;
}

void release_req(Req* r) {
    r->scene->batch_refs--;
    if (r->uploaded) cudaEventDestroy(r->uploaded);
    if (r->ran) cudaEventDestroy(r->ran);
    delete r;
}

// Adds a completed step's kernel time to gpu_busy_ms (caller holds the mutex; the
// slot is free, so its end event has completed and the query does not wait).
void account_slot(tim_rt_server* s, Slot& sl) {
    if (!sl.timing_pending) return;
    sl.timing_pending = false;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, sl.t_begin, sl.t_end) == cudaSuccess) s->gpu_busy_ms += ms;
    else cudaGetLastError();
}

// Cancelled requests that were admitted: after the upload and every step that
// traced part of them, they complete without results (on_requests_cancelled).
int issue_cancels(tim_rt_server* s, std::vector<Req*>& cancels) {
    if (cancels.empty()) return TIM_RT_OK;
    for (Req* r : cancels)
        if (r->uploaded && cudaStreamWaitEvent(s->comp, r->uploaded, 0) != cudaSuccess) return TIM_RT_EDEVICE;
    if (cudaLaunchHostFunc(s->comp, on_requests_cancelled, new DoneMsg{s, cancels}) != cudaSuccess)
        return TIM_RT_EDEVICE;
    return TIM_RT_OK;
}

// A step is planned when a slot is free and the step issued before it has begun
// on the GPU, so that at most one step waits behind a running one and each plan
// takes every request uploaded while the previous step ran (planning as soon as a
// slot frees would leave the second slot with whatever little had arrived since).
// Whether the last step has begun is polled (its begin event, outside the mutex)
// every 20 us while the worker waits.
void worker_main(tim_rt_server* s) {
    cudaSetDevice(s->ctx->device);
    for (;;) {
        std::vector<Req*> release, admitted, cancels;
        Plan P;
        if (!s->last_started) {
            const cudaError_t q = cudaEventQuery(s->slots[s->last_slot].t_begin);
            if (q != cudaErrorNotReady) {
                s->last_started = true;
                if (q != cudaSuccess) cudaGetLastError();   // a failed step reports itself on the stream
            }
        }
        {
            std::unique_lock<std::mutex> lk(s->m);
            auto ready = [&] {
                if (s->stop || !s->finished.empty()) return true;
                if (s->error) return false;
                if (!s->cancel_q.empty()) return true;
                if (!s->waiting.empty()) {
                    // admissible once the head fits in the free arena
                    uint64_t off;
                    Arena probe = s->arena;
                    if (probe.alloc(s->waiting.front()->bytes, off)) return true;
                }
                return !s->active.empty() && !s->free_slots.empty() && s->last_started;
            };
            if (s->last_started) {
                s->cv.wait(lk, ready);
            } else if (!s->cv.wait_for(lk, std::chrono::microseconds(20), ready)) {
                continue;   // poll the last step's begin event again
            }
            // stop once everything completed (or, after a device error, at once:
            // teardown waits for the streams and releases what is left)
            if (s->stop && (s->error || (s->pending.empty() && s->finished.empty()))) break;
            release.swap(s->finished);
            for (Req* r : release) s->arena.release(r->off, r->bytes);
            // admitted requests taken back leave the active list before planning
            cancels.swap(s->cancel_q);
            if (!cancels.empty())
                s->active.erase(std::remove_if(s->active.begin(), s->active.end(), [](Req* r) { return r->cancel; }),
                                s->active.end());
            if (!s->error) {
                while (!s->waiting.empty()) {
                    Req* r = s->waiting.front();
                    uint64_t off;
                    if (!s->arena.alloc(r->bytes, off)) break;
                    r->off = off;
                    r->t_admit = Clock::now();
                    s->waiting.pop_front();
                    admitted.push_back(r);
                    if (!r->probe) s->active.push_back(r);
                }
                if (!s->active.empty() && !s->free_slots.empty() && s->last_started) {
                    P.slot = s->free_slots.back();
                    s->free_slots.pop_back();
                    account_slot(s, s->slots[P.slot]);
                    plan_step(s, P);
                    s->steps++;
                    s->step_requests += P.chunks.size();
                    s->max_step_requests = std::max<uint32_t>(s->max_step_requests, (uint32_t)P.chunks.size());
                    // steps queued on the GPU and not yet completed, this one included
                    s->max_inflight = std::max<uint32_t>(
                        s->max_inflight, (uint32_t)(s->slots.size() - s->free_slots.size()));
                    // requests whose last rays this step traces leave the active list
                    for (auto& ch : P.chunks)
                        if (ch.first->last_planned) P.finishing.push_back(ch.first);
                    s->active.erase(std::remove_if(s->active.begin(), s->active.end(),
                                                   [](Req* r) { return r->last_planned; }),
                                    s->active.end());
                }
            }
        }
        for (Req* r : release) release_req(r);
        int rc = TIM_RT_OK;
        uint8_t* base = static_cast<uint8_t*>(s->arena_buf.ptr);
        for (Req* r : admitted) {
            if (r->probe) {
                if (stage_probe(s, r, base + r->off) != TIM_RT_OK) rc = TIM_RT_EDEVICE;
                continue;
            }
            const uint64_t n = r->r.n;
            uint8_t* p = base + r->off;
            r->d_rays = reinterpret_cast<tim_rt_ray*>(p);
            p += round256(32ull * n);
            r->d_hit = reinterpret_cast<uint4*>(p);
            p += round256(16ull * n);
            if (r->r.leaf_nid) {
                r->d_nid = reinterpret_cast<uint32_t*>(p);
                p += round256(4ull * n);
            }
            if (r->r.bary) r->d_bary = reinterpret_cast<float2*>(p);
            if (cudaEventCreateWithFlags(&r->uploaded, cudaEventDisableTiming) ||
                cudaMemcpyAsync(r->d_rays, r->r.rays, 32ull * n, cudaMemcpyHostToDevice, s->up) ||
                cudaEventRecord(r->uploaded, s->up))
                rc = TIM_RT_EDEVICE;
        }
        // admitted probe updates run on the probe stream, beside the trace steps
        for (Req* r : admitted)
            if (r->probe && rc == TIM_RT_OK) rc = issue_probe(s, r);
        if (P.slot >= 0 && rc == TIM_RT_OK) {
            rc = issue_step(s, P);
            s->last_slot = P.slot;
            s->last_started = false;
        }
        if (rc == TIM_RT_OK) rc = issue_cancels(s, cancels);
        if (rc != TIM_RT_OK) fail_all(s, rc, std::string("serving step failed: ") + cudaGetErrorString(cudaGetLastError()));
    }
}

int server_teardown(tim_rt_server* s) {
    {
        std::lock_guard<std::mutex> lk(s->m);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->ctx->device);
    for (cudaStream_t st : {s->up, s->comp, s->down, s->probe})
        if (st) cudaStreamSynchronize(st);
    // requests left behind (only after a device error or a failed create)
    std::set<Req*> left(s->finished.begin(), s->finished.end());
    for (auto& kv : s->pending) left.insert(kv.second);
    for (Req* r : left) release_req(r);
    s->finished.clear();
    s->pending.clear();
    s->waiting.clear();
    for (Slot& sl : s->slots) {
        dev_free(s->ctx, sl.dev);
        if (sl.host) cudaFreeHost(sl.host);
        if (sl.done) cudaEventDestroy(sl.done);
        if (sl.t_begin) cudaEventDestroy(sl.t_begin);
        if (sl.t_end) cudaEventDestroy(sl.t_end);
    }
    dev_free(s->ctx, s->arena_buf);
    for (cudaStream_t st : {s->up, s->comp, s->down, s->probe})
        if (st) cudaStreamDestroy(st);
    s->ctx->servers.erase(s);
    delete s;
    return TIM_RT_OK;
}

float percentile(std::vector<float> v, double q) {
    if (v.empty()) return 0.f;
    const size_t k = std::min(v.size() - 1, (size_t)(q * (double)(v.size() - 1) + 0.5));
    std::nth_element(v.begin(), v.begin() + k, v.end());
    return v[k];
}

}  // namespace

namespace timrt {
void server_shutdown(tim_rt_ctx*, tim_rt_server* s) { server_teardown(s); }
}  // namespace timrt

extern "C" {

int tim_rt_server_create(tim_rt_ctx* c, const tim_rt_server_params* params, tim_rt_server** out) {
    int rc = check_ctx(c);
    if (rc) return rc;
    if (!out || !params || (params->flags & ~TIM_RT_BATCH_WIDE) || params->max_inflight_steps > 8) {
        set_error("tim_rt_server_create: null argument, unknown flag or more than 8 in-flight steps");
        return TIM_RT_EINVAL;
    }
    *out = nullptr;
    auto s = std::make_unique<tim_rt_server>();
    s->ctx = c;
    s->p = *params;
    if (!s->p.memory_budget_bytes) s->p.memory_budget_bytes = 1ull << 30;
    if (!s->p.max_rays_per_step) s->p.max_rays_per_step = 4u << 20;
    if (!s->p.max_inflight_steps) s->p.max_inflight_steps = 2;
    if (!s->p.max_jobs_per_step) s->p.max_jobs_per_step = 256;
    s->p.memory_budget_bytes = round256(s->p.memory_budget_bytes);
    s->wide = (params->flags & TIM_RT_BATCH_WIDE) != 0;
    if ((rc = dev_alloc(c, s->arena_buf, s->p.memory_budget_bytes))) return rc;
    s->arena.init(s->p.memory_budget_bytes);
    const uint32_t maxj = s->p.max_jobs_per_step;
    const uint64_t vb = round256(sizeof(SceneView) * maxj), jb = round256(sizeof(MultiJob) * maxj);
    s->slots.resize(s->p.max_inflight_steps);
    bool ok = cudaStreamCreateWithFlags(&s->up, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&s->comp, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&s->down, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&s->probe, cudaStreamNonBlocking) == cudaSuccess;
    for (size_t i = 0; ok && i < s->slots.size(); ++i) {
        Slot& sl = s->slots[i];
        if (dev_alloc(c, sl.dev, vb + jb + 256) != TIM_RT_OK ||
            cudaHostAlloc(&sl.host, vb + jb, cudaHostAllocMapped) != cudaSuccess ||
            cudaHostGetDevicePointer(const_cast<void**>(&sl.host_dev), sl.host, 0) != cudaSuccess ||
            cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreate(&sl.t_begin) != cudaSuccess || cudaEventCreate(&sl.t_end) != cudaSuccess) {
            ok = false;
            break;
        }
        uint8_t* d = static_cast<uint8_t*>(sl.dev.ptr);
        sl.d_views = reinterpret_cast<SceneView*>(d);
        sl.d_jobs = reinterpret_cast<MultiJob*>(d + vb);
        sl.d_counter = reinterpret_cast<uint32_t*>(d + vb + jb);
        s->free_slots.push_back((int)i);
    }
    tim_rt_server* raw = s.release();
    c->servers.insert(raw);
    if (!ok) {
        std::string msg = "tim_rt_server_create: stream, pinned table or event creation failed";
        server_teardown(raw);
        set_error(msg);
        return TIM_RT_ENOMEM;
    }
    raw->worker = std::thread(worker_main, raw);
    *out = raw;
    return TIM_RT_OK;
}

int tim_rt_server_submit(tim_rt_server* s, const tim_rt_request* req, uint64_t* ticket) {
    if (!s || !req || !ticket || req->n == 0 || req->n > 0x7FFFFFFFu || !req->rays || !req->hit ||
        req->mode > TIM_RT_MODE_PER_RAY) {
        set_error("tim_rt_server_submit: null argument, empty request or bad mode");
        return TIM_RT_EINVAL;
    }
    const uint64_t n = req->n;
    const uint64_t bytes = round256(32 * n) + round256(16 * n) + (req->leaf_nid ? round256(4 * n) : 0) +
                           (req->bary ? round256(8 * n) : 0);
    if (bytes > s->p.memory_budget_bytes) {
        set_error("tim_rt_server_submit: request needs " + std::to_string(bytes) + " B, the arena holds " +
                  std::to_string(s->p.memory_budget_bytes));
        return TIM_RT_ENOMEM;
    }
    std::unique_lock<std::mutex> lk(s->m);
    if (s->error) {
        set_error(s->error_msg);
        return s->error;
    }
    if (s->stop) {
        set_error("tim_rt_server_submit: server is stopping");
        return TIM_RT_EINVAL;
    }
    Scene* sc = find_scene(s->ctx, req->scene);
    if (!sc) return TIM_RT_ENOTFOUND;
    if (s->wide && !sc->has_wide) {
        set_error("tim_rt_server_submit: scene was uploaded without TIM_RT_UPLOAD_QUANT8");
        return TIM_RT_EUNSUPPORTED;
    }
    Req* r = new Req;
    r->ticket = s->next_ticket++;
    r->r = *req;
    r->rays = req->n;
    r->scene = sc;
    r->bytes = bytes;
    r->t_submit = Clock::now();
    sc->batch_refs++;
    if (!s->t0_set) {
        s->t0 = r->t_submit;
        s->t0_set = true;
    }
    s->submitted++;
    s->pending[r->ticket] = r;
    s->waiting.push_back(r);
    *ticket = r->ticket;
    lk.unlock();
    s->cv.notify_all();
    return TIM_RT_OK;
}

int tim_rt_server_submit_probes(tim_rt_server* s, const tim_rt_probe_request* req, uint64_t* ticket) {
    if (!s || !req || !ticket || !req->desc || !req->dirs || !req->sh_basis || !req->sh9_fp16) {
        set_error("tim_rt_server_submit_probes: null argument");
        return TIM_RT_EINVAL;
    }
    std::unique_lock<std::mutex> lk(s->m);
    if (s->error) {
        set_error(s->error_msg);
        return s->error;
    }
    if (s->stop) {
        set_error("tim_rt_server_submit_probes: server is stopping");
        return TIM_RT_EINVAL;
    }
    Scene* sc = find_scene(s->ctx, req->scene);
    if (!sc) return TIM_RT_ENOTFOUND;
    ProbePlan plan;
    int rc = probe_plan(sc, req->desc, req->probe_begin, req->probe_end, "tim_rt_server_submit_probes", &plan);
    if (rc) return rc;
    const uint64_t bytes = probe_staging(plan, req->octa != nullptr).total();
    if (bytes > s->p.memory_budget_bytes) {
        set_error("tim_rt_server_submit_probes: request needs " + std::to_string(bytes) + " B, the arena holds " +
                  std::to_string(s->p.memory_budget_bytes));
        return TIM_RT_ENOMEM;
    }
    Req* r = new Req;
    r->ticket = s->next_ticket++;
    r->probe = true;
    r->pr = *req;
    r->pdesc = *req->desc;
    r->pr.desc = &r->pdesc;
    r->plan = plan;
    r->rays = plan.n;
    r->scene = sc;
    r->bytes = bytes;
    r->t_submit = Clock::now();
    sc->batch_refs++;
    if (!s->t0_set) {
        s->t0 = r->t_submit;
        s->t0_set = true;
    }
    s->submitted++;
    s->pending[r->ticket] = r;
    s->waiting.push_back(r);
    *ticket = r->ticket;
    lk.unlock();
    s->cv.notify_all();
    return TIM_RT_OK;
}

int tim_rt_server_wait(tim_rt_server* s, uint64_t ticket, uint32_t timeout_ms) {
    if (!s) {
        set_error("null server");
        return TIM_RT_EINVAL;
    }
    std::unique_lock<std::mutex> lk(s->m);
    if (ticket == 0 || ticket >= s->next_ticket) {
        set_error("tim_rt_server_wait: unknown ticket");
        return TIM_RT_EINVAL;
    }
    auto pred = [&] { return s->error || !s->pending.count(ticket); };
    if (timeout_ms) {
        if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred)) {
            set_error("tim_rt_server_wait: request still pending");
            return TIM_RT_ETIMEOUT;
        }
    } else {
        s->cv_done.wait(lk, pred);
    }
    if (s->pending.count(ticket)) {
        set_error(s->error_msg);
        return s->error;
    }
    if (s->cancelled_tickets.erase(ticket)) {
        set_error("tim_rt_server_wait: the request was cancelled");
        return TIM_RT_ECANCELLED;
    }
    return TIM_RT_OK;
}

int tim_rt_server_cancel(tim_rt_server* s, uint64_t ticket) {
    if (!s) {
        set_error("null server");
        return TIM_RT_EINVAL;
    }
    std::unique_lock<std::mutex> lk(s->m);
    if (s->error) {
        set_error(s->error_msg);
        return s->error;
    }
    auto it = s->pending.find(ticket);
    if (it == s->pending.end()) {
        set_error("tim_rt_server_cancel: unknown or completed request");
        return TIM_RT_ENOTFOUND;
    }
    Req* r = it->second;
    if (r->cancel) return TIM_RT_OK;
    auto w = std::find(s->waiting.begin(), s->waiting.end(), r);
    if (w != s->waiting.end()) {
        // not admitted: nothing of it reached the device
        s->waiting.erase(w);
        s->pending.erase(it);
        s->cancelled++;
        s->cancelled_tickets.insert(ticket);
        r->scene->batch_refs--;
        delete r;
        lk.unlock();
        s->cv.notify_all();
        s->cv_done.notify_all();
        return TIM_RT_OK;
    }
    if (r->probe || r->last_planned) {
        set_error("tim_rt_server_cancel: the request's work is already on the GPU; it completes normally");
        return TIM_RT_EBUSY;
    }
    r->cancel = true;
    s->cancel_q.push_back(r);
    lk.unlock();
    s->cv.notify_all();
    return TIM_RT_OK;
}

int tim_rt_server_drain(tim_rt_server* s, uint32_t timeout_ms) {
    if (!s) {
        set_error("null server");
        return TIM_RT_EINVAL;
    }
    std::unique_lock<std::mutex> lk(s->m);
    auto pred = [&] { return s->error || s->pending.empty(); };
    if (timeout_ms) {
        if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred)) {
            set_error("tim_rt_server_drain: requests still pending");
            return TIM_RT_ETIMEOUT;
        }
    } else {
        s->cv_done.wait(lk, pred);
    }
    if (!s->pending.empty()) {
        set_error(s->error_msg);
        return s->error;
    }
    return TIM_RT_OK;
}

int tim_rt_server_stats_get(tim_rt_server* s, tim_rt_server_stats* st, int reset) {
    if (!s || !st) {
        set_error("null argument");
        return TIM_RT_EINVAL;
    }
    std::lock_guard<std::mutex> lk(s->m);
    std::memset(st, 0, sizeof(*st));
    st->submitted = s->submitted;
    st->completed = s->completed;
    st->rays_completed = s->rays_completed;
    st->steps = s->steps;
    st->arena_bytes = s->p.memory_budget_bytes;
    st->arena_peak_bytes = s->arena.peak;
    st->p50_ms = percentile(s->lat_ms, 0.50);
    st->p99_ms = percentile(s->lat_ms, 0.99);
    double sum = 0;
    for (float v : s->lat_ms) {
        sum += v;
        st->max_ms = std::max(st->max_ms, v);
    }
    st->mean_ms = s->lat_ms.empty() ? 0.f : (float)(sum / s->lat_ms.size());
    st->queue_p50_ms = percentile(s->queue_ms, 0.50);
    st->queue_p99_ms = percentile(s->queue_ms, 0.99);
    st->wall_s = s->t0_set ? std::chrono::duration<float>(Clock::now() - s->t0).count() : 0.f;
    for (int k : s->free_slots) account_slot(s, s->slots[k]);   // completed steps not yet counted
    st->cancelled = s->cancelled;
    st->step_requests = s->step_requests;
    st->max_step_requests = s->max_step_requests;
    st->max_inflight_steps = s->max_inflight;
    st->gpu_busy_ms = (float)s->gpu_busy_ms;
    if (reset) {
        s->lat_ms.clear();
        s->queue_ms.clear();
        s->submitted = s->completed = s->rays_completed = s->steps = 0;
        s->cancelled = s->step_requests = 0;
        s->max_step_requests = s->max_inflight = 0;
        s->gpu_busy_ms = 0.0;
        s->arena.peak = s->arena.used;
        s->t0_set = false;
    }
    return TIM_RT_OK;
}

int tim_rt_server_destroy(tim_rt_server* s) {
    if (!s) return TIM_RT_OK;
    tim_rt_server_drain(s, 0);
    return server_teardown(s);
}

}  // extern "C"
