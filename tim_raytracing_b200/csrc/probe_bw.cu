// probe_bw.cu -- L2 read-bandwidth probe used as the roofline denominator for
// kernels whose working set is L2-resident (the measured peaks in MEASURED_PEAKS.json cover
// HBM and tensor throughput only).
//
// A buffer well below the L2 size is first touched, then read `passes` times
// by a grid of 4 blocks of 512 threads per SM with 16-byte loads; the reads go through L1 with
// the evict-first hint so each pass is served by L2. Bytes read / device time.
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include "internal.h"
#include "../../include/tim_rt.h"

namespace timrt {

__global__ void __launch_bounds__(512) k_l2_read(const uint4* __restrict__ p, size_t n16, int passes,
                                                 unsigned int* sink) {
    uint32_t acc = 0;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (int r = 0; r < passes; ++r) {
        for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += stride) {
            uint4 v;
            asm volatile("ld.global.L1::evict_first.v4.u32 {%0,%1,%2,%3}, [%4];"
                         : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                         : "l"(p + i));
            acc ^= v.x ^ v.y ^ v.z ^ v.w;
        }
    }
    if (acc == 0x9E3779B9u) atomicAdd(sink, 1u);   // keeps the loads alive
}

}  // namespace timrt

using namespace timrt;

extern "C" int tim_rt_measure_l2_bandwidth(int device, uint64_t bytes, int passes, float* gbs) {
    if (!gbs || bytes < (1u << 20) || bytes > (64ull << 20) || passes < 1) {
        set_error("tim_rt_measure_l2_bandwidth: bytes must be 1..64 MiB, passes >= 1");
        return TIM_RT_EINVAL;
    }
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        set_error("tim_rt_measure_l2_bandwidth: bad device");
        return TIM_RT_EDEVICE;
    }
    void* buf = nullptr;
    unsigned int* sink = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    int rc = TIM_RT_OK;
    const size_t n16 = bytes / 16u;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (cudaMalloc(&buf, bytes) != cudaSuccess || cudaMalloc(&sink, 4) != cudaSuccess ||
        cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
        cudaGetLastError();
        set_error("tim_rt_measure_l2_bandwidth: allocation failed");
        rc = TIM_RT_ENOMEM;
    } else {
        cudaMemset(buf, 1, bytes);
        k_l2_read<<<sms * 4, 512>>>(static_cast<const uint4*>(buf), n16, 1, sink);   // warm L2
        cudaEventRecord(a);
        k_l2_read<<<sms * 4, 512>>>(static_cast<const uint4*>(buf), n16, passes, sink);
        cudaEventRecord(b);
        if (cudaEventSynchronize(b) != cudaSuccess) {
            set_error("tim_rt_measure_l2_bandwidth: kernel failed");
            rc = TIM_RT_EDEVICE;
        } else {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, a, b);
            *gbs = (float)((double)bytes * passes / (ms * 1e-3) / 1e9);
        }
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (buf) cudaFree(buf);
    if (sink) cudaFree(sink);
    return rc;
}
