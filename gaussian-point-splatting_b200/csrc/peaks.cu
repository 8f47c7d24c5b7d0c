// Measured device peaks that bound the splat: the rate of 64-bit atomicMin (RED.MIN.U64, no
// return value) on random addresses, which is the splat's unit of work.  The splat's roofline
// is this rate, not HBM bandwidth: every live sample that passes the pre-test is one such
// operation on a random slot of the splat buffer.
#include <cstdint>
#include <string>
#include <cuda_runtime.h>
#include "../../include/gps_b200.h"
#include "host_io.hpp"

namespace gps {
namespace {

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

// Each thread issues `per_thread` atomicMins to pseudo-random slots of buf[0, entries) with
// pseudo-random values (so that some lower the slot and some do not, as in the splat).
__global__ void __launch_bounds__(256) atomic_min_rate_kernel(unsigned long long* __restrict__ buf, uint64_t entries,
                                                              uint32_t per_thread, uint32_t salt) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t h = mix32(t ^ salt);
    for (uint32_t i = 0; i < per_thread; ++i) {
        h = mix32(h + 0x9E3779B9u);
        const uint64_t slot = ((uint64_t)h * entries) >> 32;
        const uint32_t v = mix32(h ^ 0x85ebca6bu);
        atomicMin(buf + slot, ((unsigned long long)v << 32) | h);
    }
}

__global__ void fill_u64(unsigned long long* __restrict__ buf, uint64_t n, unsigned long long v) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        buf[i] = v;
}

}  // namespace
}  // namespace gps

extern "C" gps_status gps_measure_atomic_min_rate(uint64_t* d_buf, uint64_t entries, int32_t repeats,
                                                  double* atomics_per_second, void* stream) {
    using namespace gps;
    if (!d_buf || !atomics_per_second || entries == 0 || entries >= (1ull << 32) || repeats < 1) {
        set_last_error("gps_measure_atomic_min_rate: bad argument");
        return GPS_ERR_INVALID_ARGUMENT;
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = sms * 8;
    const uint32_t per_thread = 256;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fill_u64<<<sms * 4, 256, 0, st>>>(reinterpret_cast<unsigned long long*>(d_buf), entries, ~0ull);
    atomic_min_rate_kernel<<<grid, 256, 0, st>>>(reinterpret_cast<unsigned long long*>(d_buf), entries, per_thread, 1u);
    float best = 0.0f;
    for (int r = 0; r < repeats; ++r) {
        cudaEventRecord(e0, st);
        atomic_min_rate_kernel<<<grid, 256, 0, st>>>(reinterpret_cast<unsigned long long*>(d_buf), entries, per_thread,
                                                     (uint32_t)r + 2u);
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (r == 0 || ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_last_error(std::string("gps_measure_atomic_min_rate: ") + cudaGetErrorString(e));
        return GPS_ERR_CUDA;
    }
    *atomics_per_second = (double)grid * 256.0 * per_thread / (best * 1e-3);
    return GPS_OK;
}
