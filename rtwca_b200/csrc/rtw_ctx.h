// rtw_ctx.h - the context behind the opaque rtw_ctx handle and the host
// helpers shared by the C-ABI translation units (not part of the public ABI).
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <string>
#include <utility>
#include <vector>

#include "rtw_internal.h"

namespace rtw {
struct TorusBuffers;  // rtw_torus.cu
void torus_free(TorusBuffers* b);
}  // namespace rtw

using rtw::TorusBuffers;

struct rtw_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    void* d_frames = nullptr;
    size_t frames_cap = 0;
    double* d_bins = nullptr;
    unsigned long long* d_ctl = nullptr;  // [0] work counter, then DevStats
    void* d_spec = nullptr;
    size_t spec_cap = 0;
    void* d_tail = nullptr;  // FP32-mixed tail queue: records, then spectral rows
    size_t tail_bytes = 0;
    long long last_tail_cap = 0;
    void* d_out = nullptr;
    size_t out_cap = 0;
    float* d_sink = nullptr;
    unsigned long long* d_fclock = nullptr;  // per-frame timing, 3 words per frame
    size_t fclock_cap = 0;
    int last_frames = 0;
    // autotuner results: (kind, precision, np, integrator) -> (warps, refill_min)
    std::vector<std::pair<std::array<int, 4>, std::array<int, 2>>> tuned;
    // captured launch sequence and the pinned staging it reads the frame and
    // bin tables from
    cudaGraphExec_t gexec = nullptr;
    std::vector<unsigned char> gkey;
    void* h_stage = nullptr;
    size_t stage_cap = 0;
    int last_grid = 0, last_warps = 0, last_refill = 0, last_replayed = 0, last_launches = 0;
    // synchrotron torus renders and adjoints (rtw_torus.cu)
    TorusBuffers* torus = nullptr;
    std::string err;
    rtw_stats last{};
    bool have_last = false;
};

namespace rtw {

inline rtw_status fail(rtw_ctx* ctx, rtw_status st, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return st;
}

inline rtw_status cuda_fail(rtw_ctx* ctx, cudaError_t e, const char* what) {
    return fail(ctx, RTW_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define RTW_CUDA(call, what)                              \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, what); \
    } while (0)

inline rtw_status ensure(rtw_ctx* ctx, void** ptr, size_t* cap, size_t need) {
    if (need <= *cap && *ptr) return RTW_OK;
    if (*ptr) cudaFree(*ptr);
    *ptr = nullptr;
    *cap = 0;
    cudaError_t e = cudaMalloc(ptr, need);
    if (e != cudaSuccess) {
        *ptr = nullptr;
        return fail(ctx, RTW_ERR_OOM, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
    }
    *cap = need;
    return RTW_OK;
}


// Spatial R2 L R of a camera, row-major (rtw_capi.cu).
void bundle_basis(const rtw_camera& cam, double m3[9]);

// rtw_render of a RTW_SCENE_KERR_SYNCHRO_TORUS scene (rtw_torus.cu).
rtw_status torus_render(rtw_ctx* ctx, const rtw_scene* scene, const rtw_camera* cams, int32_t n_cams,
                        const rtw_render_params* prm, rtw_outputs* out);

}  // namespace rtw
