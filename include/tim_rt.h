/*
 * tim_rt.h -- C ABI of the B200 (sm_100a) ray-tracing path.
 *
 * Drop-in replacement for the compute dispatch of TIM_Raytracing's hot path:
 * the V-EZ/Vulkan `IRenderContext::Dispatch(DrawArguments, gx, gy, gz)` calls
 * (src/rtDevice/public/IRenderContext.h:70, src/rtDevice/private/RenderContext.cpp:71-104)
 * made by RayTracingPass and LightProbFieldPass, and the BVH upload made by
 * BVHData::build (src/Renderer/BVHData.cpp:28-49).
 *
 * The entry points consume the reference's own byte layouts unchanged:
 *   - the BVH buffer written by BVHBuilder::fillGpuBuffer
 *     (src/Renderer/BVHBuilder.cpp:1319-1534) with its seven sub-ranges,
 *   - PackedBVHNode (64 B), inlined leaf Triangle records (12 B), PackedLight,
 *     BlasHeader (src/Shaders/core/primitive_cpp.glsl:50-117),
 *   - the BVHGeometry vertex arrays (src/Renderer/BVHGeometry.cpp:69-85),
 *   - PassData and PushConstants (src/Shaders/struct_cpp.glsl:10-37),
 *   - the tracingData hit-record layout (src/Shaders/cameraPass.comp:69-75).
 *
 * Conventions: every function returns an int status (TIM_RT_OK = 0); no C++
 * exception crosses the ABI; tim_rt_last_error() describes the last failure of
 * the calling thread. Host pointers are borrowed for the duration of a call.
 * Device memory is owned by the context and released by tim_rt_free_scene /
 * tim_rt_destroy. A context is used by one host thread at a time; its calls
 * are ordered on the context's CUDA stream. The *_dev variants take device
 * pointers and a CUDA stream (NULL = the context stream) and do not
 * synchronise.
 */
#ifndef TIM_RT_H
#define TIM_RT_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TIM_RT_ABI_VERSION 1

/* Status codes. The reference returns no errors (TIM_VK_VERIFY aborts in Debug,
 * src/rtDevice/private/Common.h:6-17); these are new. */
#define TIM_RT_OK 0
#define TIM_RT_EINVAL 1       /* bad argument or malformed BVH ranges */
#define TIM_RT_ENOMEM 2       /* device-memory budget or allocation exhausted */
#define TIM_RT_ETIMEOUT 3     /* a bounded device-side wait gave up */
#define TIM_RT_EDEVICE 4      /* CUDA error */
#define TIM_RT_ENOTFOUND 5    /* unknown scene id */
#define TIM_RT_EUNSUPPORTED 6 /* feature not available for this scene */
#define TIM_RT_ECANCELLED 7   /* the serving request was cancelled (tim_rt_server_cancel) */
#define TIM_RT_EBUSY 8        /* too late to cancel: the serving request completes normally */

/* Sub-range indices of the BVH buffer, in fillGpuBuffer's memory order
 * (BVHBuilder.cpp:1326-1500): {offset bytes, size bytes}. */
#define TIM_RT_RANGE_BLAS 0
#define TIM_RT_RANGE_TRI 1
#define TIM_RT_RANGE_PRIM 2
#define TIM_RT_RANGE_MAT 3
#define TIM_RT_RANGE_LIGHT 4
#define TIM_RT_RANGE_NODE 5
#define TIM_RT_RANGE_LEAF 6

typedef struct tim_rt_ctx tim_rt_ctx;
typedef uint32_t tim_rt_scene_id;

/* PushConstants, src/Shaders/struct_cpp.glsl:30-37 (filled at raytracingPass.cpp:156). */
typedef struct {
    uint32_t numTriangles, numBlas, numPrimitives, numLights, numNodes;
} tim_rt_push_constants;

/* PassData, src/Shaders/struct_cpp.glsl:10-28 (C++ layout of the reference, 240 bytes). */
typedef struct {
    uint32_t frameSize[2]; float invFrameSize[2];
    float cameraPos[4]; float cameraDir[4];
    float frustumCorner00[4]; float frustumCorner10[4]; float frustumCorner01[4];
    float invProjView[16];
    float sunDir[4]; float sunColor[4];
    float sceneMinExtent[4]; float sceneMaxExtent[4];
    uint32_t lpfResolution[4];
} tim_rt_pass_data;

/* One ray of a batch (32 bytes): origin, tmax, direction, flags.
 * flags bit 0: any-hit (occlusion) ray when the batch mode is TIM_RT_MODE_PER_RAY.
 * The reference's closest-hit rays start at tmax = TMAX = 100 (struct_cpp.glsl:5). */
typedef struct { float o[3]; float tmax; float d[3]; uint32_t flags; } tim_rt_ray;
#define TIM_RT_RAY_ANY 1u

/* Trace modes and options (low byte = mode, higher bits = options). */
#define TIM_RT_MODE_CLOSEST 0u   /* traverseBvh, bvhTraversal_inline.glsl:5-78 */
#define TIM_RT_MODE_ANY 1u       /* traverseBvhFast, bvhTraversal_inline.glsl:83-151 */
#define TIM_RT_MODE_PER_RAY 2u   /* ray.flags bit 0 selects any-hit */
#define TIM_RT_TRACE_WIDE 0x100u /* trace the 8-wide quantised BVH (needs TIM_RT_UPLOAD_QUANT8) */
#define TIM_RT_TRACE_COUNT 0x400u /* run the counting kernel variant and fill the work counters of tim_rt_stats */
#define TIM_RT_TRACE_TLAS 0x800u  /* with TIM_RT_MODE_ANY: the two-level walk of USE_TRAVERSE_TLAS scenes
                                     (traverseTlasFast + tlas_collide_fast, bvhCollision.glsl:321-348) over an
                                     image from tim_rt_build_bvh_tlas; binary form only. The reference's
                                     closest-hit two-level walk does not compile (HitBox and Hit exist only
                                     commented out, collision.glsl:175-195): TIM_RT_EUNSUPPORTED */

/* Upload flags. */
#define TIM_RT_UPLOAD_QUANT8 0x2u /* also build the 8-wide BVH with 8-bit quantised child bounds */

/* Per-call statistics (optional output). */
typedef struct {
    uint64_t rays;            /* rays traced by the call (all kinds) */
    uint64_t primary_rays, shadow_rays, probe_rays, bounce_rays;
    float kernel_ms;          /* device time of the trace kernels (CUDA events) */
    float total_ms;           /* device time of the whole call incl. copies */
    /* work counters, filled only with TIM_RT_TRACE_COUNT / TIM_RT_CAM_COUNT:
     * inner-node fetches (binary: 64-B node, 8-wide: 80-B node), leaf visits,
     * triangle tests, node-header reloads (8-wide: 32 B when a pending node is popped) */
    uint64_t node_visits, leaf_visits, tri_tests, node_reloads;
    /* camera calls: device time of the primary trace, the secondary-ray
     * generation and the secondary trace kernels (CUDA events) */
    float primary_ms, gen_ms, secondary_ms;
    /* camera calls with TIM_RT_CAM_COUNT: the secondary-trace kernel's share of the counters */
    uint64_t secondary_rays_counted, secondary_node_visits, secondary_leaf_visits, secondary_tri_tests,
        secondary_node_reloads;
} tim_rt_stats;

/* ---------------------------------------------------------------- context */
const char *tim_rt_version(void);
/* Message of the last failed call on this thread ("" if none). */
const char *tim_rt_last_error(void);

/* Creates a context on CUDA device `device`, owning one CUDA stream. Device
 * allocations made by the context are admitted against `mem_budget_bytes`
 * (0 = no budget). New: the reference's device is created by
 * VezRenderer::Init (src/rtDevice/private/VezRenderer.cpp:54-188). */
int tim_rt_create(int device, uint64_t mem_budget_bytes, tim_rt_ctx **out);
int tim_rt_destroy(tim_rt_ctx *ctx);
/* Device bytes currently held by the context (scenes + scratch). */
int tim_rt_memory_used(tim_rt_ctx *ctx, uint64_t *bytes);

/* Launch shape of the persistent trace kernels (the knobs the autotuner picks). */
typedef struct {
    uint32_t block;        /* threads per block: 64, 128 or 256 (default 256) */
    uint32_t stack_depth;  /* traversal-stack entries per thread; 0 = the scene's tree depth (<= 32) */
    uint32_t refill_min;   /* a warp fetches new rays once this many of its 32 lanes are idle (1..32);
                              camera primary rays always refill whole warps (one 8x4-pixel tile) */
    uint32_t ray_sort;     /* batched traces: TIM_RT_SORT_* coherence key the rays are reordered by */
    uint32_t phase_switch; /* 0..31 (default 10): a warp stops its lockstep node rounds and tests the leaves
                              its lanes hold once only this many lanes still need nodes */
} tim_rt_launch_config;
#define TIM_RT_SORT_NONE 0u     /* trace in input order */
#define TIM_RT_SORT_OCTANT 1u   /* group each job's rays by direction octant (stable) */
#define TIM_RT_SORT_MORTON 2u   /* octant, then 30-bit Morton code of the origin in the scene's bounds */
int tim_rt_get_launch_config(tim_rt_ctx *ctx, tim_rt_launch_config *cfg);
int tim_rt_set_launch_config(tim_rt_ctx *ctx, const tim_rt_launch_config *cfg);

/* Measures L2 read bandwidth (GB/s) on `device` by reading a `bytes`-sized
 * buffer (1..64 MiB, i.e. L2-resident) `passes` times. A measurement utility for
 * roofline reporting; no counterpart in the reference. */
int tim_rt_measure_l2_bandwidth(int device, uint64_t bytes, int passes, float *gbs);

/* ---------------------------------------------------------------- BVH upload */
/* Replaces BVHData::build's CreateBuffer + UploadBuffer (src/Renderer/BVHData.cpp:43-48)
 * and BVHGeometry::flush (src/Renderer/BVHGeometry.cpp:69-78).
 * bvh_bytes/ranges: BVHBuilder::fillGpuBuffer output. pos/nrm/uv: vertex arrays
 * (xyz, xyz, uv per vertex; nrm and uv may be NULL). pc: the scene's PushConstants.
 * The buffers are validated (ranges inside the buffer, node children and leaf
 * offsets in range, vertex indices < num_vertex) before anything is launched;
 * a malformed buffer returns TIM_RT_EINVAL. */
int tim_rt_upload_bvh(tim_rt_ctx *ctx, const void *bvh_bytes, uint64_t n_bytes, const uint32_t ranges[7][2],
                      const float *pos, const float *nrm, const float *uv, uint32_t max_vertex, uint32_t num_vertex,
                      const tim_rt_push_constants *pc, uint32_t flags, tim_rt_scene_id *out);
/* Host-only check of a fillGpuBuffer image, the same one tim_rt_upload_bvh runs
 * before uploading: ranges inside the buffer and aligned, child ids above their
 * parent's id and in range, leaf data inside the leaf range, vertex / light /
 * blas ids in range, tree depth <= 32. Writes the tree depth. No GPU needed.
 * New: the reference uploads without any check (BVHData.cpp:43-48). */
int tim_rt_validate_bvh(const void *bvh_bytes, uint64_t n_bytes, const uint32_t ranges[7][2],
                        const tim_rt_push_constants *pc, uint32_t num_vertex, uint32_t *depth);
/* Host-only check of the 8-wide quantised form that tim_rt_upload_bvh builds with
 * TIM_RT_UPLOAD_QUANT8 (no GPU needed). New: the reference has no wide form. The
 * call validates the image (as tim_rt_validate_bvh), builds the 8-wide form on the
 * host exactly as the upload does, and checks it against the binary tree: every
 * used slot's 8-bit box contains the box the reference stores for that subtree,
 * empty slots are empty, internal slots reach every wide node once, and every
 * binary leaf's triangles appear once, in order, with the reference's records,
 * vertices and rounded edges bit for bit. Returns TIM_RT_EINVAL with the first
 * violation in tim_rt_last_error(); the report is zeroed first and filled as far
 * as the check got. */
typedef struct {
    uint32_t nodes;              /* 8-wide nodes */
    uint32_t depth;              /* levels of 8-wide nodes */
    uint32_t triangles;          /* leaf triangles (each binary leaf's triangles once) */
    uint32_t leaf_slots;         /* slots holding a binary leaf */
    uint32_t internal_slots;     /* slots pointing at a child node */
    uint32_t slot_histogram[9];  /* nodes by number of used slots, 0..8 */
    uint32_t reserved[2];
    uint64_t device_bytes;       /* bytes of the 8-wide arrays on the device */
} tim_rt_wide_report;
int tim_rt_wide_check(const void *bvh_bytes, uint64_t n_bytes, const uint32_t ranges[7][2],
                      const tim_rt_push_constants *pc, const float *pos, uint32_t num_vertex,
                      tim_rt_wide_report *report);
/* Replaces BVHData::~BVHData / BVHGeometry::~BVHGeometry (DestroyBuffer). */
int tim_rt_free_scene(tim_rt_ctx *ctx, tim_rt_scene_id scene);
/* Device bytes held by one scene. */
int tim_rt_scene_bytes(tim_rt_ctx *ctx, tim_rt_scene_id scene, uint64_t *bytes);

/* ---------------------------------------------------------------- tracing */
/* Batched closest-hit / any-hit trace of n rays; replaces the trace half of the
 * reference's compute dispatches (rayTrace, baseRaytracingPass.glsl:16-27, and
 * traverseForShadow, bvhLighting.glsl:100-108).
 * hit[4i..4i+3]: closest hit -> (vertexOffset, index01, index2_matId, bits(t)),
 *   t = t_hit - 1e-5 on a hit (bvhCollision.glsl:210) and t = ray.tmax on a
 *   miss with xyz = 0; any-hit -> (1 if occluded else 0, 0, 0, bits(ray.tmax)).
 * leaf_nid (optional): masked id of the leaf whose triangle was accepted,
 *   0xFFFFFFFF on a miss or for any-hit rays.
 * bary (optional): (u, v) of the accepted Moller-Trumbore hit, (0, 0) otherwise. */
int tim_rt_trace(tim_rt_ctx *ctx, tim_rt_scene_id scene, const tim_rt_ray *rays, uint32_t n, uint32_t mode,
                 uint32_t *hit, uint32_t *leaf_nid, float *bary, tim_rt_stats *stats);
/* Device-pointer form of tim_rt_trace; stream-ordered, no synchronisation. */
int tim_rt_trace_dev(tim_rt_ctx *ctx, tim_rt_scene_id scene, const tim_rt_ray *d_rays, uint32_t n, uint32_t mode,
                     uint32_t *d_hit, uint32_t *d_leaf_nid, float *d_bary, void *cuda_stream);

/* Verification (not in the reference, and never on the trace path): re-runs the
 * Moller-Trumbore test of each closest-hit record's triangle in FP64 and reports
 * the largest |(t + 1e-5) - t_fp64| (absolute and relative to t_fp64) over the
 * records with a hit, the records without one (t = ray tmax), and hits the FP64
 * test does not confirm (u, v outside [-1e-6, 1 + 1e-6] or t <= 0: grazing hits
 * accepted by the FP32 arithmetic). The only FP64 arithmetic on the GPU.
 * d_hit: closest-hit records of d_rays (tim_rt_trace_dev layout). Synchronous. */
typedef struct {
    uint64_t hits_checked, misses, fp64_misses;
    double max_abs_t_err, max_rel_t_err;
} tim_rt_verify_result;
int tim_rt_verify_hits(tim_rt_ctx *ctx, tim_rt_scene_id scene, const tim_rt_ray *d_rays, uint32_t n,
                       const uint32_t *d_hit, tim_rt_verify_result *result);

/* ---------------------------------------------------------------- batched multi-scene trace */
/* Not in the reference, which dispatches one scene per compute pass. A batch is
 * a device-resident table of jobs, each a ray buffer traced against one resident
 * scene; tim_rt_batch_launch traces all of them in ONE persistent kernel launch
 * whose warps take rays from any job (a lane loads its job's scene when it
 * fetches a ray), so scenes of very uneven size share the GPU without a tail of
 * small launches. Each job's outputs are exactly those of tim_rt_trace_dev on the
 * same scene, rays and mode (same layouts), whatever the launch configuration and
 * ray-sort key. The launch issues only memsets and kernels on the given stream
 * (no host<->device copies, no allocation once the sort scratch exists), so it
 * can be captured in a CUDA graph and replayed; the job table is fixed at create
 * time but the ray buffers' contents may change between launches. Scenes used by
 * a live batch cannot be freed (TIM_RT_EINVAL). Launches of one batch must not
 * overlap on the GPU (they share the batch's work counter). */
typedef struct {
    tim_rt_scene_id scene;
    uint32_t mode;             /* TIM_RT_MODE_CLOSEST / ANY / PER_RAY */
    uint32_t n;                /* rays */
    uint32_t reserved;
    const tim_rt_ray *d_rays;  /* device, 32 B per ray, 16-byte aligned */
    uint32_t *d_hit;           /* device, 4 u32 per ray */
    uint32_t *d_leaf_nid;      /* device, optional */
    float *d_bary;             /* device, optional, 2 floats per ray */
} tim_rt_job;
typedef struct tim_rt_batch tim_rt_batch;
#define TIM_RT_BATCH_WIDE 0x100u   /* trace the 8-wide quantised BVHs (all scenes need TIM_RT_UPLOAD_QUANT8) */
int tim_rt_batch_create(tim_rt_ctx *ctx, const tim_rt_job *jobs, uint32_t num_jobs, uint32_t flags,
                        tim_rt_batch **out);
/* Traces every job of the batch with the context's launch configuration. The
 * first launch with a ray-sort key allocates the batch's sort scratch (24 B per
 * ray plus the radix sort's temporary storage): make it before capturing. */
int tim_rt_batch_launch(tim_rt_ctx *ctx, tim_rt_batch *batch, void *cuda_stream);
/* Rays in the batch and its device bytes (job table + sort scratch). */
int tim_rt_batch_info(tim_rt_ctx *ctx, const tim_rt_batch *batch, uint64_t *rays, uint64_t *bytes);
int tim_rt_batch_destroy(tim_rt_ctx *ctx, tim_rt_batch *batch);

/* Autotuner (not in the reference, whose launch shape is fixed at 16x16 tiles).
 * Times the batch's launch under candidate launch configurations (threads per
 * block, refill threshold, stack depth, ray-sort key and, with TIM_RT_TUNE_WIDTH,
 * node width) by coordinate descent, each candidate the median of `reps` timed
 * launches (CUDA events on the context's stream, after one warm-up launch), and
 * installs the fastest as the context's launch configuration (node width: the
 * batch's). Synchronous. Results do not depend on the configuration, except that
 * the two node widths may resolve exact near-ties of t differently, which is why
 * width is only tried when asked for. */
typedef struct {
    tim_rt_launch_config best;
    uint32_t wide;          /* node width of the fastest configuration: 1 = 8-wide */
    uint32_t tried;         /* configurations timed */
    float best_ms;          /* median device time of one launch, best configuration */
    float start_ms;         /* the same for the configuration in force before tuning */
} tim_rt_tune_result;
#define TIM_RT_TUNE_WIDTH 1u
int tim_rt_autotune_batch(tim_rt_ctx *ctx, tim_rt_batch *batch, uint32_t flags, uint32_t reps,
                          tim_rt_tune_result *result);

/* ---------------------------------------------------------------- serving loop */
/* Not in the reference (a single-user renderer). A server owns a worker thread
 * that traces requests from any number of submitting threads against the
 * context's resident scenes, with continuous batching:
 *   - admission: a request is admitted once its device staging (rays, hit
 *     records and the optional outputs it asks for) fits in the server's device
 *     arena of memory_budget_bytes (FIFO; a request larger than the whole arena
 *     is refused at submit with TIM_RT_ENOMEM); its rays are then copied to the
 *     device on an upload stream;
 *   - steps: each step is one batched multi-scene launch (the kernel of
 *     tim_rt_batch_launch) over chunks of the admitted requests, at most
 *     max_rays_per_step rays: first an equal share for every admitted request,
 *     then the unused capacity in admission order, so small requests finish in
 *     their first step while large ones span several; up to max_inflight_steps
 *     steps are queued on the GPU, and requests that arrive meanwhile join the
 *     next step;
 *   - completion: when a request's last chunk has been traced its results are
 *     copied to the caller's host buffers on a download stream and the request
 *     completes; its latency is measured from submit to the end of that copy.
 * Each request's outputs are exactly those of tim_rt_trace on the same scene,
 * rays and mode (closest / any / per-ray), whatever else is in flight. Host
 * buffers should be pinned (cudaHostAlloc / cudaHostRegister) for the copies to
 * overlap; they must stay valid until the request completes. Scenes with pending
 * requests cannot be freed. While a server runs, the context may be used from
 * other threads only through tim_rt_server_* calls, which are thread-safe. */
typedef struct tim_rt_server tim_rt_server;
typedef struct {
    uint64_t memory_budget_bytes;  /* device arena for admitted requests; 0 = 1 GiB */
    uint32_t max_rays_per_step;    /* 0 = 4M */
    uint32_t max_inflight_steps;   /* 1..8; 0 = 2 */
    uint32_t max_jobs_per_step;    /* request chunks per step; 0 = 256 */
    uint32_t flags;                /* TIM_RT_BATCH_WIDE: trace the 8-wide BVHs */
} tim_rt_server_params;
typedef struct {
    tim_rt_scene_id scene;
    uint32_t mode;             /* TIM_RT_MODE_CLOSEST / ANY / PER_RAY */
    uint32_t n;                /* rays, >= 1 */
    uint32_t reserved;
    const tim_rt_ray *rays;    /* host */
    uint32_t *hit;             /* host, 4 u32 per ray */
    uint32_t *leaf_nid;        /* host, optional */
    float *bary;               /* host, optional */
} tim_rt_request;
typedef struct {
    uint64_t submitted, completed, rays_completed, steps;
    uint64_t arena_bytes, arena_peak_bytes;   /* arena size and the most of it ever admitted */
    float p50_ms, p99_ms, mean_ms, max_ms;   /* request latency, submit -> results on the host */
    float queue_p50_ms, queue_p99_ms;        /* submit -> admission */
    float wall_s;                            /* seconds since the first submit after the last reset */
    uint64_t cancelled;                      /* requests completed by tim_rt_server_cancel */
    uint64_t step_requests;                  /* sum over trace steps of the requests each step traced */
    uint32_t max_step_requests;              /* most requests one trace step traced */
    uint32_t max_inflight_steps;             /* most trace steps queued on the GPU at once */
    float gpu_busy_ms;                       /* device time of the trace steps' kernels (CUDA events) */
} tim_rt_server_stats;
int tim_rt_server_create(tim_rt_ctx *ctx, const tim_rt_server_params *params, tim_rt_server **out);
/* Queues a request; never blocks on the GPU. *ticket identifies it. */
int tim_rt_server_submit(tim_rt_server *srv, const tim_rt_request *req, uint64_t *ticket);
/* A light-probe field update as a server request: the work and outputs of
 * tim_rt_update_probes (declared below) on probes [probe_begin, probe_end) of a
 * resident scene, with the same validation. sh9_fp16 (the whole field, host) is
 * read when the request is admitted and rewritten when it completes; octa is
 * optional (TIM_RT_PROBE_OCTA). Admission counts its whole device staging
 * (directions, basis, the FP16 field, per-ray records, lit values, the shadow-ray
 * queue and the optional texels) against the same arena as trace requests, in the
 * same FIFO. Once admitted it runs as one probe-update launch sequence on a
 * server stream of its own, beside the batched trace steps; the outputs equal
 * those of tim_rt_update_probes on the same inputs. */
typedef struct tim_rt_probe_desc tim_rt_probe_desc;
typedef struct {
    tim_rt_scene_id scene;
    uint32_t probe_begin, probe_end;
    uint32_t reserved;
    const tim_rt_probe_desc *desc;  /* copied at submit */
    const float *dirs;              /* host, 4 floats per direction */
    const float *sh_basis;          /* host, 9 floats per direction */
    uint16_t *sh9_fp16;             /* host, in/out: [7][res_z][res_y][res_x][4] */
    float *octa;                    /* host, optional: [probes][64][3] */
} tim_rt_probe_request;
int tim_rt_server_submit_probes(tim_rt_server *srv, const tim_rt_probe_request *req, uint64_t *ticket);
/* Waits until the request completes (timeout_ms 0 = no limit): TIM_RT_OK,
 * TIM_RT_ECANCELLED for a cancelled request, or TIM_RT_ETIMEOUT with the request
 * still pending. */
int tim_rt_server_wait(tim_rt_server *srv, uint64_t ticket, uint32_t timeout_ms);
/* Takes a request back. TIM_RT_OK: none of its remaining rays will be traced and
 * its output buffers are not written; a request not yet admitted is gone at once,
 * an admitted one completes once its upload and the steps already tracing part of
 * it have finished -- tim_rt_server_wait then returns TIM_RT_ECANCELLED, after
 * which its host buffers may be reused. TIM_RT_EBUSY: too late (its last rays
 * are already in a queued step, or it is an admitted probe update); it completes
 * normally. TIM_RT_ENOTFOUND: unknown or already completed ticket. Thread-safe.
 * The reference has no request queue to cancel from: its passes run once per
 * frame (src/Renderer/raytracingPass.cpp:89-110). */
int tim_rt_server_cancel(tim_rt_server *srv, uint64_t ticket);
/* Waits until every submitted request has completed. */
int tim_rt_server_drain(tim_rt_server *srv, uint32_t timeout_ms);
/* Statistics over the requests completed since the last reset (reset != 0 clears them afterwards). */
int tim_rt_server_stats_get(tim_rt_server *srv, tim_rt_server_stats *stats, int reset);
/* Drains, stops the worker and frees the arena. */
int tim_rt_server_destroy(tim_rt_server *srv);

/* Camera trace step: cameraPass.comp with TRACING_STEP (src/Shaders/cameraPass.comp:44-76),
 * dispatched by RayTracingPass::tracePass (src/Renderer/raytracingPass.cpp:89-110).
 * out: W*H*8 u32 = tracingData[2*pix] (hit record) and tracingData[2*pix+1]
 * (shadowMask, probMask, 0, 0). Pixel rows never produced by the reference's
 * row mapping (cameraPass.comp:46) are written as zeros.
 * flags: TIM_RT_CAM_PROB_MASK = USE_LPF_MASK; TIM_RT_CAM_TILE_LIGHTS = shadow
 * rays to the tile-culled lights (tile_counts/tile_lists from
 * tim_rt_cull_lights over ceil(W/16) x ceil(H/16) tiles) instead of the hit
 * leaf's light list; TIM_RT_CAM_BOUNCE = one cosine-weighted diffuse bounce
 * ray per hit, its hit record written to bounce_out (W*H*4 u32). */
#define TIM_RT_CAM_PROB_MASK 1u
#define TIM_RT_CAM_TILE_LIGHTS 2u
#define TIM_RT_CAM_BOUNCE 4u
#define TIM_RT_CAM_WIDE 0x100u   /* use the quantised 8-wide BVH */
#define TIM_RT_CAM_COUNT 0x200u  /* counting kernel variant; fills the work counters of tim_rt_stats */
#define TIM_RT_CAM_PIPELINED 0x800u /* tim_rt_trace_camera only: copy the results to the host in up to 8 bands of
                                       rows while the frame traces: the secondary rays are traced band by band and
                                       each band's copy starts as soon as its records are final (same results) */
#define TIM_RT_CAM_PRIMARY_BINARY 0x400u /* with TIM_RT_CAM_WIDE: primary rays take the binary walk (faster for
                                          coherent camera rays here; both walks give identical results) */
#define TIM_RT_CAM_DEVICE_CULL 0x1000u /* tim_rt_trace_camera only, with TIM_RT_CAM_TILE_LIGHTS: the call culls the
                                         lights itself on the device (the lists tim_rt_cull_lights returns, over
                                         ceil(W/16) x ceil(H/16) tiles) right before the trace, as the reference's
                                         culling feeds its camera pass on the GPU; tile_counts / tile_lists are not
                                         read and may be NULL (same results) */
int tim_rt_trace_camera(tim_rt_ctx *ctx, tim_rt_scene_id scene, const tim_rt_pass_data *pd, uint32_t flags,
                        uint32_t seed, const uint32_t *tile_counts, const uint32_t *tile_lists,
                        uint32_t *out, uint32_t *bounce_out, tim_rt_stats *stats);

/* Device-pointer form of tim_rt_trace_camera (pd is read on the host at call
 * time). Stream-ordered, no synchronisation, capturable in a CUDA graph after a
 * first call has sized the context's scratch buffers. If d_ray_count is not
 * NULL, the number of rays the frame traced (primary + secondary) is ADDED to
 * *d_ray_count on the device. One camera call per context may be in flight. */
int tim_rt_trace_camera_dev(tim_rt_ctx *ctx, tim_rt_scene_id scene, const tim_rt_pass_data *pd, uint32_t flags,
                            uint32_t seed, const uint32_t *d_tile_counts, const uint32_t *d_tile_lists,
                            uint32_t *d_out, uint32_t *d_bounce_out, uint64_t *d_ray_count, void *cuda_stream);

/* tim_rt_trace_camera_dev restricted to the output rows [row_begin, row_end) of
 * the frame (row_begin a multiple of 4, the height of the kernels' 8x4-pixel
 * tiles; row_end <= H): the unit by which one frame is split across GPUs, each
 * GPU tracing its contiguous band against its own copy of the scene. d_out and
 * d_bounce_out are the whole frame's arrays (W*H*8 and W*H*4 u32, same pixel
 * indexing as tim_rt_trace_camera_dev); only the band's pixels are written, so
 * the band's records are the contiguous words [row_begin*W*8, row_end*W*8) of
 * d_out. The results of all bands equal those of one whole-frame call. Same
 * tile lists (of the whole frame), flags, scratch and stream rules as
 * tim_rt_trace_camera_dev. No counterpart in the reference: its one renderer
 * dispatches the whole frame on one device (RayTracingPass::tracePass,
 * src/Renderer/raytracingPass.cpp:89-110). */
int tim_rt_trace_camera_rows_dev(tim_rt_ctx *ctx, tim_rt_scene_id scene, const tim_rt_pass_data *pd, uint32_t flags,
                                 uint32_t seed, uint32_t row_begin, uint32_t row_end,
                                 const uint32_t *d_tile_counts, const uint32_t *d_tile_lists, uint32_t *d_out,
                                 uint32_t *d_bounce_out, uint64_t *d_ray_count, void *cuda_stream);

/* Camera trace that allocates nothing. It has no counterpart in the reference.
 * For callers that may not allocate device memory while they trace (a fixed
 * device budget owned by their engine, a plugin host that forbids allocation
 * from its callbacks, or a frame loop that cannot take cudaMalloc's implicit
 * synchronisation): the caller passes its own device copies of the BVH buffer
 * (fillGpuBuffer image), the vertex positions, the tile lists and the outputs;
 * the scratch (counters, hit-leaf ids, secondary-ray queue) is a static device
 * array inside the library, which holds it on every GPU that loads it until the
 * process exits (3.85 MB). Frames are limited to TIM_RT_NOALLOC_MAX_PIXELS
 * pixels; larger ones return TIM_RT_EINVAL. Same results as
 * tim_rt_trace_camera_dev on the binary form (flags PROB_MASK, TILE_LIGHTS,
 * BOUNCE only). The buffer must have passed tim_rt_validate_bvh, since this call
 * reads device memory it cannot check; every range offset must be a multiple of
 * 4 bytes and the node range's of 16 (else TIM_RT_EINVAL). tree_depth is the
 * depth tim_rt_validate_bvh reports, or 0 for the maximum (32): a value below
 * the tree's real depth lets a ray's traversal stack run out, which ends that
 * ray early with its hits so far, and the device error word that records it is
 * not reported by this call -- pass 0 when unsure. The first call in each device
 * context (again after a cudaDeviceReset) looks up the scratch array's address
 * with cudaGetSymbolAddress, with that device current, and should come before
 * any stream capture on the device. All calls share the one scratch array, and
 * each call clears its counters before use: calls whose kernels overlap on the
 * GPU (different streams, no ordering) race. Stream-ordered, no synchronisation. */
#define TIM_RT_NOALLOC_MAX_PIXELS 4096u
int tim_rt_trace_camera_noalloc(const void *d_bvh, const uint32_t ranges[7][2], const tim_rt_push_constants *pc,
                                const float *d_pos, uint32_t num_vertex, uint32_t tree_depth,
                                const tim_rt_pass_data *pd, uint32_t flags, uint32_t seed,
                                const uint32_t *d_tile_counts, const uint32_t *d_tile_lists,
                                uint32_t *d_out, uint32_t *d_bounce_out, void *cuda_stream);

/* Tile light-frustum culling, cullWithFrustumTile's light section
 * (src/Shaders/cullFrustum.glsl:63-100,136-151). One list of at most 16 light
 * ids per tile, ascending (the reference's order is atomic-arrival order). */
int tim_rt_cull_lights(tim_rt_ctx *ctx, tim_rt_scene_id scene, const tim_rt_pass_data *pd,
                       uint32_t tiles_x, uint32_t tiles_y, uint32_t *out_counts, uint32_t *out_lists);
/* Device-pointer form of tim_rt_cull_lights; stream-ordered, no synchronisation. */
int tim_rt_cull_lights_dev(tim_rt_ctx *ctx, tim_rt_scene_id scene, const tim_rt_pass_data *pd,
                           uint32_t tiles_x, uint32_t tiles_y, uint32_t *d_counts, uint32_t *d_lists, void *cuda_stream);

/* Lighting step of the camera pass: cameraPass.comp without TRACING_STEP, as
 * RayTracingPass::lightingPass dispatches it (src/Renderer/raytracingPass.cpp:113-135:
 * USE_LPF, USE_LPF_MASK; cameraPass.comp:78-88). Per pixel, from the tracing step's
 * output (tracing: W*H*8 u32 as tim_rt_trace_camera writes it): the hit point and
 * interpolated normal (baseRaytracingPass.glsl:38-82); direct light of the lights
 * whose shadow-mask bit is clear and of the sun (bvhLighting.glsl:42-85, a light
 * out of range adds nothing); unless TIM_RT_SHADE_NO_LPF, the light-probe term:
 * the probe-masked trilinear SH9 sample of the 7 RGBA16F images that
 * tim_rt_update_probes writes (resolution pd->lpfResolution, at least 2 per axis,
 * over pd->sceneMinExtent..sceneMaxExtent; fetchSH_inline.glsl:82-118), evalSH and
 * computeIndirectLighting; the sky colour on a miss. Materials are taken as
 * untextured (texColor 1). out_rgba16: W*H*4 halves (lit rgb, alpha 1), written
 * for every pixel, output row 0 (which the reference's dispatch never reaches) as
 * 0; out_rgb32: optional W*H*3 floats before the FP16 rounding. */
#define TIM_RT_SHADE_NO_LPF 1u
int tim_rt_shade_camera(tim_rt_ctx *ctx, tim_rt_scene_id scene, const tim_rt_pass_data *pd, uint32_t flags,
                        const uint32_t *tracing, const uint16_t *sh9_fp16, uint16_t *out_rgba16, float *out_rgb32,
                        tim_rt_stats *stats);
int tim_rt_shade_camera_dev(tim_rt_ctx *ctx, tim_rt_scene_id scene, const tim_rt_pass_data *pd, uint32_t flags,
                            const uint32_t *d_tracing, const uint16_t *d_sh9_fp16, uint16_t *d_out_rgba16,
                            float *d_out_rgb32, void *cuda_stream);

/* ---------------------------------------------------------------- light-probe field */
/* Probe field update: genLightProbField.comp (trace step and lighting step,
 * src/Shaders/genLightProbField.comp:41-81) followed by updateLightProbField.comp
 * (src/Shaders/updateLightProbField.comp:33-64), dispatched by
 * LightProbFieldPass::traceLightProbField / updateLightProbField
 * (src/Renderer/lightProbFieldPass.cpp:81-149).
 *   - probe p (tiled 4x4x4 order, lightprobHelpers.glsl:33-61) sits at
 *     aabbMin + (aabbMax - aabbMin) / resolution * (coord + 0.5); resolution must
 *     be divisible by 4 on every axis;
 *   - ray r of probe p goes along dirs[r].xyz (the caller's directions, e.g.
 *     LightProbFieldPass::sampleRays or an octahedral grid), closest hit, then the
 *     sun (direction -sunDir, not normalised, as lightProbFieldPass.cpp:29 passes it)
 *     and leaf-light shadow mask; the probe-visibility mask is 0;
 *   - lit value: computeLighting with NO_LPF (bvhLighting.glsl:42-85) with texColor 1,
 *     the sky colour 0.3 * (200, 220, 255) / 255 on a miss (baseRaytracingPass.glsl:81);
 *   - SH9: sum_r L_r * sh_basis[r][j] * 4*pi/num_dirs, new = prev * (1 - h) + sh * h
 *     (GLSL mix), where prev is read from and new written to sh9_fp16: 7 RGBA16F
 *     3-D images [7][res_z][res_y][res_x][4] in the channel layout of storeSH9
 *     (lightprob/storeSH_inline.glsl:6-18);
 *   - octa (TIM_RT_PROBE_OCTA): dirs form a side x side octahedral grid in row-major
 *     order (side^2 = num_dirs, side a multiple of 8); texel (i*8/side, j*8/side)
 *     of probe p holds the mean radiance of its rays, FP32 [probes][64][3]. Not in
 *     the reference.
 * Outputs of probes [probe_begin, probe_end) only; all optional except sh9_fp16.
 * trace_out: [probes][num_dirs][8] u32 tracingData; irradiance: [probes][num_dirs][3];
 * sh9_fp32: the new SH9 before FP16 rounding, [probes][9][3]. */
struct tim_rt_probe_desc {
    float aabbMin[4]; float aabbMax[4];
    uint32_t resolution[4];
    float sunDir[4]; float sunColor[4];
    float hysteresis;          /* 0.03 in the reference */
    uint32_t num_dirs;
    uint32_t flags;            /* TIM_RT_PROBE_* */
    uint32_t reserved;
};
#define TIM_RT_PROBE_OCTA 1u
#define TIM_RT_PROBE_WIDE 0x100u
#define TIM_RT_PROBE_PRIMARY_BINARY 0x400u /* with TIM_RT_PROBE_WIDE: the probe rays take the binary walk and
                                            only their shadow rays the 8-wide one (identical results) */
/* Probe ray directions (4 floats each) and, when sh_basis is not NULL, their SH9
 * basis weights (9 floats each, the constants and order of LightProbFieldPass::
 * sampleRays, lightProbFieldPass.cpp:186-199) for count = side^2 rays (1..4096):
 *   TIM_RT_DIRS_STRATIFIED: sampleRays' jittered stratified sphere directions
 *     (lightProbFieldPass.cpp:151-185), drawn from a std::mt19937 seeded with
 *     `seed` (the reference uses std::random_device, not reproducible);
 *   TIM_RT_DIRS_OCTAHEDRAL: the cell centres of a side x side octahedral grid in the
 *     order TIM_RT_PROBE_OCTA bins (index j * side + i). Host only. */
#define TIM_RT_DIRS_STRATIFIED 0u
#define TIM_RT_DIRS_OCTAHEDRAL 1u
int tim_rt_probe_directions(uint32_t count, uint32_t kind, uint64_t seed, float *dirs, float *sh_basis);
int tim_rt_update_probes(tim_rt_ctx *ctx, tim_rt_scene_id scene, const tim_rt_probe_desc *desc, const float *dirs,
                         const float *sh_basis, uint32_t probe_begin, uint32_t probe_end, uint32_t *trace_out,
                         float *irradiance, uint16_t *sh9_fp16, float *sh9_fp32, float *octa, tim_rt_stats *stats);

/* ---------------------------------------------------------------- product-side BVH builder */
/* Builds a BVH over triangle records and writes it in the reference's
 * fillGpuBuffer layout (BVHBuilder.cpp:1319-1534), so its output can be passed
 * to tim_rt_upload_bvh. Binned-SAH object splits (no spatial splits), leaves of
 * at most max_leaf_size triangles, depth at most max_depth (<= 32, the width of
 * the reference's traversal bitstack), leaf light lists of at most 15 lights
 * (sphere vs leaf box, as BVHBuilder.cpp:749-756; 15 avoids the 4-bit count
 * wrap at 16). tri_records: 3 u32 per triangle (Triangle, primitive_cpp.glsl:50-55).
 * materials: Material records (48 B each); lights: PackedLight records (56 B each). */
typedef struct {
    uint32_t max_leaf_size;   /* default 4 */
    uint32_t max_depth;       /* default 30 */
    float traversal_cost;     /* GPU builder: surface-area cost of a node, default 1 */
    float intersection_cost;  /* GPU builder: surface-area cost of a triangle, default 0.4 */
    uint32_t num_threads;     /* 0 = all hardware threads */
} tim_rt_build_params;
typedef struct tim_rt_bvh_blob tim_rt_bvh_blob;
void tim_rt_build_params_default(tim_rt_build_params *p);
int tim_rt_build_bvh(const float *pos, uint32_t num_vertex, const uint32_t *tri_records, uint32_t num_tris,
                     const void *materials, uint32_t num_materials, const void *lights, uint32_t num_lights,
                     const tim_rt_build_params *params, tim_rt_bvh_blob **out);
/* The same output (layout, node numbering scheme, light lists) built on the
 * context's GPU: a linear BVH over 63-bit Morton codes of the triangle centroids
 * (radix tree over single triangles split at the highest differing bit, Karras
 * 2012), then four passes of treelet restructuring (7-leaf treelets rebuilt for
 * the least surface-area cost, Karras & Aila 2013) that also choose which
 * subtrees of at most max_leaf_size triangles become leaves, by the cost
 * traversal_cost * area per node against intersection_cost * area per triangle
 * (both positive and finite, else TIM_RT_EINVAL). A leaf's triangles are stored
 * in tree order. Builds in milliseconds where the binned-SAH host builder takes
 * tens to hundreds, and its trees trace within about 10% of the host builder's.
 * num_threads is not used. A restructured tree deeper than max_depth falls back to
 * the Morton-code tree with its subtrees of at most max_leaf_size triangles as
 * leaves; TIM_RT_EUNSUPPORTED when that is deeper too (max_depth at most 32, the
 * reference traversal's bitstack); scenes of at most max_leaf_size triangles are
 * built by tim_rt_build_bvh. The host builder (tim_rt_build_bvh) splits down to
 * max_leaf_size by binned SAH and does not use the two costs. */
int tim_rt_build_bvh_gpu(tim_rt_ctx *ctx, const float *pos, uint32_t num_vertex, const uint32_t *tri_records,
                         uint32_t num_tris, const void *materials, uint32_t num_materials, const void *lights,
                         uint32_t num_lights, const tim_rt_build_params *params, tim_rt_bvh_blob **out);
/* A two-level image for the reference's TLAS/BLAS traversal (USE_TRAVERSE_TLAS,
 * src/Shaders/bvh/bvhCollision.glsl:286-349), in the layout fillGpuBuffer gives a
 * top-level builder holding BLAS instances (src/Renderer/BVHBuilder.cpp:1441-1457,
 * 1521-1533; BVHBuilder::addBlas, :292-301): instance i is the BLAS over
 * triangles [inst_first[i], inst_first[i] + inst_count[i]) of tri_records (at
 * least 2; it is built with tim_rt_build_bvh, its root an inner node), the top
 * level a binned-SAH tree over the instance boxes with at most tlas_max_leaf
 * (1..255) instances per leaf; lights go into the top-level leaves' lists. The
 * reference's own builder cannot write this image: with its inlined triangles
 * (INLINE_TRIANGLES, BVHBuilder.cpp:13) fillGpuBuffer copies the BLAS leaves'
 * triangles out of the top-level builder's own, empty, triangle array
 * (BVHBuilder.cpp:1490-1495, under a TIM_ASSERT(!m_isTlas) that release builds
 * drop). Trace it with TIM_RT_TRACE_TLAS. */
int tim_rt_build_bvh_tlas(const float *pos, uint32_t num_vertex, const uint32_t *tri_records, uint32_t num_tris,
                          const uint32_t *inst_first, const uint32_t *inst_count, uint32_t num_instances,
                          const void *materials, uint32_t num_materials, const void *lights, uint32_t num_lights,
                          const tim_rt_build_params *params, uint32_t tlas_max_leaf, tim_rt_bvh_blob **out);
int tim_rt_bvh_blob_info(const tim_rt_bvh_blob *blob, const uint8_t **bytes, uint64_t *size,
                         uint32_t ranges[7][2], tim_rt_push_constants *pc, float aabb[6]);
void tim_rt_bvh_blob_free(tim_rt_bvh_blob *blob);

/* ---------------------------------------------------------------- on-disk BVH file */
/* Not in the reference (BVHData::build rebuilds every run, BVHData.cpp:28-49, and
 * its threaded builder is not deterministic, BVHBuilder.cpp:851-894). A versioned
 * file holding a fillGpuBuffer image (bytes, seven ranges, push constants, bounds)
 * and the BVHGeometry vertex arrays (positions; normals and uvs when given), with
 * an FNV-1a 64 checksum. Writing validates the BVH first and replaces the file
 * atomically; reading checks magic, version, sizes, checksum and the BVH, and
 * returns TIM_RT_EINVAL (corrupt) or TIM_RT_EUNSUPPORTED (other version). */
typedef struct tim_rt_bvh_file tim_rt_bvh_file;
int tim_rt_bvh_file_write(const char *path, const void *bvh_bytes, uint64_t n_bytes, const uint32_t ranges[7][2],
                          const tim_rt_push_constants *pc, const float aabb[6], const float *pos, const float *nrm,
                          const float *uv, uint32_t max_vertex, uint32_t num_vertex);
int tim_rt_bvh_file_read(const char *path, tim_rt_bvh_file **out);
/* Pointers stay valid until tim_rt_bvh_file_free; nrm / uv are NULL when absent. */
int tim_rt_bvh_file_info(const tim_rt_bvh_file *file, const uint8_t **bytes, uint64_t *size, uint32_t ranges[7][2],
                         tim_rt_push_constants *pc, float aabb[6], const float **pos, const float **nrm,
                         const float **uv, uint32_t *max_vertex, uint32_t *num_vertex);
void tim_rt_bvh_file_free(tim_rt_bvh_file *file);
/* tim_rt_bvh_file_read followed by tim_rt_upload_bvh with `flags`. */
int tim_rt_upload_bvh_file(tim_rt_ctx *ctx, const char *path, uint32_t flags, tim_rt_scene_id *out);

#ifdef __cplusplus
}
#endif
#endif
