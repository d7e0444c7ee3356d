// rtw_launch.cuh - launcher template for one scene kind; each rtw_kind*.cu
// instantiates it once so the four scene kinds compile in parallel.
#pragma once

#include "rtw_trace.cuh"

namespace rtw {

template <int KIND, bool MIXED>
static const void* trace_fn(int bpl) {
    switch (bpl) {
    case 1: return (const void*)trace_kernel<KIND, MIXED, 1>;
    case 2: return (const void*)trace_kernel<KIND, MIXED, 2>;
    default: return (const void*)trace_kernel<KIND, MIXED, 4>;
    }
}

template <int KIND>
const void* trace_kernel_ptr(int precision, int np) {
    const int bpl = np / 32;
    return precision == RTW_PREC_MIXED ? trace_fn<KIND, true>(bpl) : trace_fn<KIND, false>(bpl);
}

template <int KIND>
cudaError_t launch_kind(const KParams& p, int precision, int grid, int block, cudaStream_t stream) {
    const void* fn = trace_kernel_ptr<KIND>(precision, p.np);
    void* args[] = {(void*)&p};
    return cudaLaunchKernel(fn, dim3(grid), dim3(block), args, trace_dyn_smem(precision, p.np, block / 32), stream);
}

}  // namespace rtw

#define RTW_INSTANTIATE_KIND(KIND)                                                                         \
    namespace rtw {                                                                                       \
    cudaError_t launch_kind_##KIND(const KParams& p, int precision, int grid, int block, cudaStream_t st) { \
        return launch_kind<KIND>(p, precision, grid, block, st);                                          \
    }                                                                                                     \
    const void* kernel_ptr_##KIND(int precision, int np) { return trace_kernel_ptr<KIND>(precision, np); } \
    }
