// rtw_probe.cu - issue-rate microbenchmarks for the roofline denominators of
// the trace kernel (FP32 FMA, FP64 FMA, MUFU ex2). Each thread runs 8
// independent dependency chains so the pipes, not latency, bound the rate.
#include <cuda_runtime.h>
#include "rtw_internal.h"

namespace rtw {

__global__ void probe_fma32(int iters, float* sink) {
    float a[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = threadIdx.x * 1e-3f + i;
    const float m = 0.999f, c = 1e-3f;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = fmaf(a[i], m, c);
        }
    }
    float s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += a[i];
    if (s == 12345.678f) sink[0] = s;
}

__global__ void probe_fma64(int iters, float* sink) {
    double a[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = threadIdx.x * 1e-3 + i;
    const double m = 0.999, c = 1e-3;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = fma(a[i], m, c);
        }
    }
    double s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += a[i];
    if (s == 12345.678) sink[0] = (float)s;
}

__global__ void probe_ex2(int iters, float* sink) {
    float a[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = -1e-3f * (threadIdx.x & 7) - 0.1f * i;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = exp2f(a[i]) - 1.0f;
        }
    }
    float s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += a[i];
    if (s == 12345.678f) sink[0] = s;
}

cudaError_t launch_peak_probe(int which, int grid, int block, int iters, float* sink, cudaStream_t stream) {
    if (which == 0) probe_fma32<<<grid, block, 0, stream>>>(iters, sink);
    else if (which == 1) probe_fma64<<<grid, block, 0, stream>>>(iters, sink);
    else probe_ex2<<<grid, block, 0, stream>>>(iters, sink);
    return cudaGetLastError();
}

}  // namespace rtw
