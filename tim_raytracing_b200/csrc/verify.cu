// verify.cu -- FP64 re-intersection of reported hits (tim_rt_verify_hits).
//
// A verification utility, never called by the trace path: for every closest-hit
// record with a hit it re-runs the Moller-Trumbore test of the recorded triangle
// in FP64 and reduces the largest absolute and relative difference between the
// record's t (the accepted t_hit minus the 1e-5 shrink, bvhCollision.glsl:210)
// plus 1e-5 and the FP64 t. It is the only FP64 arithmetic on the GPU.
#include <cuda_runtime.h>
#include <cstring>
#include "context.h"

namespace timrt {
namespace {

// Non-negative doubles order like their bit patterns, so atomicMax on the bits
// is a max on the values.
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* p, double v) {
    atomicMax(p, (unsigned long long)__double_as_longlong(v));
}

// out[0] hits checked, [1] misses, [2] records the FP64 test does not hit,
// [3] max |dt| bits, [4] max |dt| / t64 bits
__global__ void k_verify(const float* __restrict__ pos, uint32_t num_vertex, const float4* __restrict__ rays,
                         uint32_t n, const uint4* __restrict__ hit, unsigned long long* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = __ldg(rays + 2u * i), b = __ldg(rays + 2u * i + 1u);
    const uint4 rec = __ldg(hit + i);
    const float t32 = __uint_as_float(rec.w);
    if (t32 == a.w) {   // a miss keeps t = tmax
        atomicAdd(out + 1, 1ull);
        return;
    }
    const uint32_t i0 = rec.x + (rec.y & 0xFFFFu), i1 = rec.x + (rec.y >> 16), i2 = rec.x + (rec.z & 0xFFFFu);
    if (i0 >= num_vertex || i1 >= num_vertex || i2 >= num_vertex) {
        atomicAdd(out + 2, 1ull);
        return;
    }
    const double p0x = pos[3u * i0], p0y = pos[3u * i0 + 1], p0z = pos[3u * i0 + 2];
    const double e1x = pos[3u * i1] - p0x, e1y = pos[3u * i1 + 1] - p0y, e1z = pos[3u * i1 + 2] - p0z;
    const double e2x = pos[3u * i2] - p0x, e2y = pos[3u * i2 + 1] - p0y, e2z = pos[3u * i2 + 2] - p0z;
    const double dx = b.x, dy = b.y, dz = b.z;
    const double hx = dy * e2z - dz * e2y, hy = dz * e2x - dx * e2z, hz = dx * e2y - dy * e2x;
    const double det = e1x * hx + e1y * hy + e1z * hz;
    const double sx = (double)a.x - p0x, sy = (double)a.y - p0y, sz = (double)a.z - p0z;
    const double qx = sy * e1z - sz * e1y, qy = sz * e1x - sx * e1z, qz = sx * e1y - sy * e1x;
    const double u = (sx * hx + sy * hy + sz * hz) / det;
    const double v = (dx * qx + dy * qy + dz * qz) / det;
    const double t64 = (e2x * qx + e2y * qy + e2z * qz) / det;
    atomicAdd(out + 0, 1ull);
    // the FP32 test accepts hits on the boundary; allow a relative 1e-6 there
    if (!(u >= -1e-6 && v >= -1e-6 && u + v <= 1.0 + 1e-6 && t64 > 0.0)) atomicAdd(out + 2, 1ull);
    const double dt = fabs(((double)t32 + 1e-5) - t64);
    atomic_max_nonneg(out + 3, dt);
    atomic_max_nonneg(out + 4, t64 > 0.0 ? dt / t64 : 0.0);
}

}  // namespace
}  // namespace timrt

using namespace timrt;

extern "C" int tim_rt_verify_hits(tim_rt_ctx* c, tim_rt_scene_id id, const tim_rt_ray* d_rays, uint32_t n,
                                  const uint32_t* d_hit, tim_rt_verify_result* result) {
    int rc = check_ctx(c);
    if (rc) return rc;
    Scene* s = find_scene(c, id);
    if (!s) return TIM_RT_ENOTFOUND;
    if (!result || (n && (!d_rays || !d_hit))) {
        set_error("tim_rt_verify_hits: null argument");
        return TIM_RT_EINVAL;
    }
    *result = tim_rt_verify_result{};
    if (n == 0) return TIM_RT_OK;
    unsigned long long* out = static_cast<unsigned long long*>(c->dstats.ptr) + 16;   // words 16..20
    unsigned long long h[5] = {};
    if (cudaMemsetAsync(out, 0, sizeof(h), c->stream) != cudaSuccess) {
        set_error("tim_rt_verify_hits: memset failed");
        return TIM_RT_EDEVICE;
    }
    k_verify<<<(n + 255u) / 256u, 256, 0, c->stream>>>(s->view.pos, s->view.num_vertex,
                                                       reinterpret_cast<const float4*>(d_rays), n,
                                                       reinterpret_cast<const uint4*>(d_hit), out);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess) {
        set_error("tim_rt_verify_hits: kernel or copy failed");
        return TIM_RT_EDEVICE;
    }
    result->hits_checked = h[0];
    result->misses = h[1];
    result->fp64_misses = h[2];
    std::memcpy(&result->max_abs_t_err, &h[3], 8);
    std::memcpy(&result->max_rel_t_err, &h[4], 8);
    return TIM_RT_OK;
}
