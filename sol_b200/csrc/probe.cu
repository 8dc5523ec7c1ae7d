// Probes (bench and tests only; nothing on the rendering path uses them).
//
// Memory probe for the roofline: L2 read bandwidth of this GPU, measured on
// a buffer that L2 holds (the path tracer's scene is mostly served from L2, so
// its achieved L2 bytes per second are reported against this figure).
//
// The probe reads a `bytes`-long buffer `passes` times in one launch with
// 16-byte loads that bypass L1 (ld.global.cg), one grid-stride sweep per pass,
// after an untimed sweep that brings the buffer into L2.
//
// Math probe: the shared pow_ of core/math.h evaluated on the device, compiled
// with the library's flags, so that a test can compare its bits with the host
// build of the same source.  Built as its own small library (libsol_probe.so).
#include <cuda_runtime.h>
#include <stdint.h>

#include "core/math.h"

namespace {

__global__ void __launch_bounds__(256) l2_read(const uint4* __restrict__ buf, size_t n, int passes,
                                               unsigned int* __restrict__ sink) {
    unsigned int acc = 0;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (int p = 0; p < passes; ++p) {
        for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += stride) {
            const uint4 v = __ldcg(buf + i);
            acc ^= v.x ^ v.y ^ v.z ^ v.w;
        }
    }
    if (acc == 0x9e3779b9u) sink[0] = acc;   // keeps the loads; never true for a zero buffer
}

__global__ void pow_probe(const float* __restrict__ x, const float* __restrict__ y, float* __restrict__ out,
                          uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = sol_b200::pow_(x[i], y[i]);
}

}  // namespace

extern "C" {

/// out[i] = pow_(x[i], y[i]) on the current device for device arrays of n
/// floats; returns the CUDA error code of the launch (0 on success).
int sol_probe_pow(const float* x, const float* y, float* out, uint32_t n) {
    if (n == 0) return 0;
    pow_probe<<<(n + 255) / 256, 256>>>(x, y, out, n);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return (int)e;
}

/// L2 read bandwidth in GB/s over a `bytes` buffer read `passes` times (best of
/// `reps` timed launches); returns a negative value on a CUDA error.
double sol_probe_l2_read_gbs(uint64_t bytes, int passes, int reps) {
    uint4* buf = nullptr;
    unsigned int* sink = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    double best = -1.0;
    const size_t n = bytes / sizeof(uint4);
    int sms = 0, dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaMalloc(&buf, n * sizeof(uint4));
    if (e == cudaSuccess) e = cudaMalloc(&sink, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemset(buf, 0, n * sizeof(uint4));
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    const int grid = sms * 8;
    if (e == cudaSuccess) {
        l2_read<<<grid, 256>>>(buf, n, 1, sink);   // bring the buffer into L2
        e = cudaDeviceSynchronize();
    }
    for (int r = 0; r < reps && e == cudaSuccess; ++r) {
        cudaEventRecord(a);
        l2_read<<<grid, 256>>>(buf, n, passes, sink);
        cudaEventRecord(b);
        e = cudaEventSynchronize(b);
        float ms = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
        if (e == cudaSuccess && ms > 0.0f) {
            const double gbs = (double)n * sizeof(uint4) * passes / (ms * 1e-3) / 1e9;
            if (gbs > best) best = gbs;
        }
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    cudaFree(buf);
    cudaFree(sink);
    return e == cudaSuccess ? best : -1.0;
}

}  // extern "C"
