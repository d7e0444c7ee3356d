// rtw_noalloc.cu - rtw_render_noalloc: the trace kernel for callers that
// cannot allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is not allowed or not
// wanted - inside a host that pre-plans all device memory (a pool owned by
// another runtime, a real-time loop that must not block in the allocator, a
// process whose memory budget is fixed up front) - or callers that have no
// rtw_ctx (creating one allocates its buffers). This entry point allocates
// nothing: its scratch (the per-warp spectral state), the frame table, the
// bin table and the work counter live in file-scope __device__ arrays that
// every GPU which loads the library holds until the process exits.
//
// Limits (RTW_NOALLOC_* in include/rtw.h): at most RTW_NOALLOC_MAX_FRAMES
// cameras per call and RTW_NOALLOC_SCRATCH_BYTES of spectral scratch, which
// caps the number of resident warps (fewer than rtw_render uses, so it is
// slower); outputs must be device pointers (on_device = 1). Larger requests
// are rejected with RTW_ERR_INVALID_PARAM and a message.
//
// Every call shares the arrays: calls that overlap on the GPU (two streams,
// two host threads) race and corrupt each other; serialise them. Each call
// zeroes the work counter and the counters and rewrites the frame and bin
// tables before its trace launch; the kernel initialises a ray's spectral row
// when it starts the ray.
//
// The tables reach the device as the by-value parameters of a one-CTA upload
// kernel (a launch copies its parameters when it is enqueued), so the call
// reads no host memory after it returns.
//
// The first call on a device looks up the device addresses of the arrays
// (cudaGetSymbolAddress, with that device current) and caches them; make that
// first call before any stream capture. The cached addresses belong to the
// device's primary context as it was then: after cudaDeviceReset the module
// may load elsewhere, so this entry point must not be used again in that
// process.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "rtw_internal.h"

namespace rtw {
cudaError_t launch_kind_0(const KParams&, int, int, int, cudaStream_t);
const void* kernel_ptr_0(int, int);
const void* kernel_ptr_1(int, int);
const void* kernel_ptr_2(int, int);
const void* kernel_ptr_3(int, int);
}  // namespace rtw

extern "C" rtw_status rtw_prepare_frames(const rtw_scene* scene, const rtw_camera* cams, int32_t n_cams,
                                         void* frames_out, int64_t* total_out);

using namespace rtw;

static __device__ __align__(256) unsigned char g_noalloc_scratch[RTW_NOALLOC_SCRATCH_BYTES];
static __device__ __align__(256) FrameDesc g_noalloc_frames[RTW_NOALLOC_MAX_FRAMES];
static __device__ __align__(256) double g_noalloc_bins[4 * RTW_MAX_BINS];
// [0] work counter, [1..] DevStats
static __device__ __align__(256) unsigned long long g_noalloc_ctl[32];

// What one call uploads: the frame table (first n_frames entries used) and
// the bin table. About 20 KB, within the 32 KB kernel-parameter limit.
struct NoallocTables {
    FrameDesc frames[RTW_NOALLOC_MAX_FRAMES];
    double bins[4 * RTW_MAX_BINS];
    int n_frames;
};
static_assert(sizeof(NoallocTables) <= 32000, "upload tables exceed the kernel-parameter limit");

// One CTA: copies the tables into the arrays and zeroes the work counter and
// the counters.
__global__ void __launch_bounds__(256) noalloc_upload(__grid_constant__ const NoallocTables t) {
    const int i = threadIdx.x;
    if (i < t.n_frames) g_noalloc_frames[i] = t.frames[i];
    for (int k = i; k < 4 * RTW_MAX_BINS; k += blockDim.x) g_noalloc_bins[k] = t.bins[k];
    if (i < 32) g_noalloc_ctl[i] = 0ull;
}

namespace {

constexpr int kMaxDevices = 64;

struct Symbols {
    bool ready = false;
    void* scratch = nullptr;
    void* frames = nullptr;
    void* bins = nullptr;
    void* ctl = nullptr;
    int num_sms = 0;
};

std::mutex g_mu;
Symbols g_sym[kMaxDevices];

const void* noalloc_kernel(int kind, int precision, int np) {
    switch (kind) {
    case 0: return kernel_ptr_0(precision, np);
    case 1: return kernel_ptr_1(precision, np);
    case 2: return kernel_ptr_2(precision, np);
    default: return kernel_ptr_3(precision, np);
    }
}

thread_local char g_err[256];

rtw_status fail(rtw_status st, const char* msg) {
    std::strncpy(g_err, msg, sizeof(g_err) - 1);
    g_err[sizeof(g_err) - 1] = 0;
    return st;
}

// Device addresses of this file's arrays on the current device (once per device).
rtw_status symbols(int dev, Symbols*& out) {
    if (dev < 0 || dev >= kMaxDevices) return fail(RTW_ERR_INVALID_PARAM, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_mu);
    Symbols& s = g_sym[dev];
    if (!s.ready) {
        if (cudaGetSymbolAddress(&s.scratch, g_noalloc_scratch) != cudaSuccess ||
            cudaGetSymbolAddress(&s.frames, g_noalloc_frames) != cudaSuccess ||
            cudaGetSymbolAddress(&s.bins, g_noalloc_bins) != cudaSuccess ||
            cudaGetSymbolAddress(&s.ctl, g_noalloc_ctl) != cudaSuccess) {
            cudaGetLastError();
            return fail(RTW_ERR_CUDA, "cudaGetSymbolAddress failed for the no-alloc arrays");
        }
        if (cudaDeviceGetAttribute(&s.num_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return fail(RTW_ERR_CUDA, "cudaDeviceGetAttribute failed");
        s.ready = true;
    }
    out = &s;
    return RTW_OK;
}

}  // namespace

extern "C" const char* rtw_noalloc_last_error(void) { return g_err; }

extern "C" rtw_status rtw_render_noalloc(const rtw_scene* scene, const rtw_camera* cams, int32_t n_cams,
                                         const rtw_render_params* prm, rtw_outputs* out) {
    g_err[0] = 0;
    if (!scene || !cams || !prm || !out) return fail(RTW_ERR_INVALID_PARAM, "null argument");
    if (!out->on_device) return fail(RTW_ERR_INVALID_PARAM, "rtw_render_noalloc needs device output pointers");
    if (n_cams <= 0 || n_cams > RTW_NOALLOC_MAX_FRAMES)
        return fail(RTW_ERR_INVALID_PARAM, "n_cams must be 1..RTW_NOALLOC_MAX_FRAMES");
    if (prm->n_colors <= 0 || prm->n_colors > RTW_MAX_BINS || !prm->colors_nm)
        return fail(RTW_ERR_INVALID_PARAM, "n_colors must be 1..128 with colors_nm set");
    if (prm->ray_bundles) return fail(RTW_ERR_UNSUPPORTED, "ray bundles are built for the skybox scenes only");
    if (scene->ref_precision) return fail(RTW_ERR_UNSUPPORTED, "ref_precision is an oracle-only switch");
    if (prm->graph || prm->autotune || prm->trace_ray >= 0)
        return fail(RTW_ERR_UNSUPPORTED, "graph, autotune and trace_ray need an rtw_ctx (use rtw_render)");
    if (prm->precision != RTW_PREC_FP64 && prm->precision != RTW_PREC_MIXED) return fail(RTW_ERR_INVALID_PARAM, "precision");
    if (prm->integrator != RTW_DP45_REF_COMPAT && prm->integrator != RTW_DP45_FSAL)
        return fail(RTW_ERR_INVALID_PARAM, "integrator");
    if (scene->kind < 0 || scene->kind > RTW_SCENE_KERR_THICK_DISK) return fail(RTW_ERR_INVALID_PARAM, "scene kind");
    if (!(prm->max_dt_scale > 0)) return fail(RTW_ERR_INVALID_PARAM, "max_dt_scale must be > 0");
    const bool kerr = scene->kind == RTW_SCENE_KERR_DISK || scene->kind == RTW_SCENE_KERR_THICK_DISK;
    if (kerr && !(std::fabs(scene->spin) < scene->mass)) return fail(RTW_ERR_INVALID_PARAM, "Kerr spin must satisfy |a| < M");
    if (!(scene->mass > 0)) return fail(RTW_ERR_INVALID_PARAM, "mass must be > 0");

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(RTW_ERR_NO_DEVICE, "no current CUDA device");
    Symbols* sym = nullptr;
    rtw_status st = symbols(dev, sym);
    if (st != RTW_OK) return st;

    // host-side tables (on the stack; they travel as the upload kernel's parameters)
    NoallocTables tab;
    std::memset(&tab, 0, sizeof(tab));
    tab.n_frames = n_cams;
    int64_t total = 0;
    st = rtw_prepare_frames(scene, cams, n_cams, tab.frames, &total);
    if (st == RTW_ERR_INVALID_CAMERA) return fail(st, "a camera is on a coordinate singularity");
    if (st != RTW_OK) return fail(st, "camera parameters invalid or non-finite");
    const int N = prm->n_colors;
    double* bins = tab.bins;
    double wx[RTW_MAX_BINS], wy[RTW_MAX_BINS], wz[RTW_MAX_BINS], fac[RTW_MAX_BINS];
    if (rtw_cie_weights(prm->colors_nm, N, wx, wy, wz, fac) != RTW_OK)
        return fail(RTW_ERR_INVALID_PARAM, "colors_nm must be positive");
    for (int c = 0; c < N; ++c) {
        bins[c] = 1.0 / prm->colors_nm[c];
        bins[RTW_MAX_BINS + c] = fac[c] * wx[c];
        bins[2 * RTW_MAX_BINS + c] = fac[c] * wy[c];
        bins[3 * RTW_MAX_BINS + c] = fac[c] * wz[c];
    }
    const int np = N <= 32 ? 32 : (N <= 64 ? 64 : 128);

    // launch shape: as many warps as the kernel keeps resident (or ctas_per_sm
    // CTAs per SM when given), capped by the scratch
    const int warps = prm->block_warps > 0 ? (prm->block_warps < 4 ? prm->block_warps : 4) : 4;
    const int block = 32 * warps;
    if (trace_allow_smem(scene->kind, prm->precision, np) != cudaSuccess)
        return fail(RTW_ERR_CUDA, "kernel shared-memory attribute failed");
    int occ = prm->ctas_per_sm;
    if (occ <= 0 &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, noalloc_kernel(scene->kind, prm->precision, np), block,
                                                      trace_dyn_smem(prm->precision, np, warps)) != cudaSuccess)
        return fail(RTW_ERR_CUDA, "occupancy query failed");
    const size_t per_warp = spec_bytes_per_warp(prm->precision, np);
    const long long fit = (long long)(RTW_NOALLOC_SCRATCH_BYTES / (per_warp * warps));
    long long grid = (long long)sym->num_sms * (occ > 0 ? occ : 1);
    if (grid > fit) grid = fit;
    if (grid < 1) return fail(RTW_ERR_INVALID_PARAM, "spectral scratch of one CTA exceeds RTW_NOALLOC_SCRATCH_BYTES");

    KParams p;
    std::memset(&p, 0, sizeof(p));
    make_dev_scene(*scene, p.sc);
    p.frames = static_cast<const FrameDesc*>(sym->frames);
    p.n_frames = n_cams;
    p.n_bins = N;
    p.total_rays = total;
    p.max_dt_scale = prm->max_dt_scale;
    const double pdr = prm->promote_dr < 0 ? -1.0 : (prm->promote_dr > 0 ? prm->promote_dr : 1e-3);
    const double psn = prm->promote_sin < 0 ? 0.0 : (prm->promote_sin > 0 ? (prm->promote_sin < 1 ? prm->promote_sin : 1.0) : 2e-3);
    p.promote_dr = pdr * scene->mass;
    p.promote_theta = std::asin(psn);
    p.fsal = prm->integrator == RTW_DP45_FSAL;
    p.pixel_order = prm->pixel_order;
    double* b = static_cast<double*>(sym->bins);
    p.bin_nu = b;
    p.bin_fx = b + RTW_MAX_BINS;
    p.bin_fy = b + 2 * RTW_MAX_BINS;
    p.bin_fz = b + 3 * RTW_MAX_BINS;
    p.spec = sym->scratch;
    p.np = np;
    unsigned long long* ctl = static_cast<unsigned long long*>(sym->ctl);
    p.counter = ctl;
    p.stats = reinterpret_cast<DevStats*>(ctl + 1);
    p.xyz = out->xyz;
    p.cls = out->term_class;
    p.steps = out->steps;
    p.spectrum = out->spectrum;
    p.final_state = out->final_state;
    p.tau = out->tau;
    p.trace = nullptr;
    p.trace_gid = -1;
    p.trace_cap = 0;
    // compaction interval as rtw_render takes it (0: 1)
    p.refill_min = prm->refill_min > 0 ? (prm->refill_min < 32 ? prm->refill_min : 32) : 1;

    cudaStream_t stream = static_cast<cudaStream_t>(prm->stream);
    noalloc_upload<<<1, 256, 0, stream>>>(tab);
    if (cudaGetLastError() != cudaSuccess) return fail(RTW_ERR_CUDA, "upload of the frame / bin tables failed");
    if (launch_trace(p, prm->precision, (int)grid, block, stream) != cudaSuccess)
        return fail(RTW_ERR_CUDA, "trace kernel launch failed");
    // wait only when the caller gave no stream
    if (!prm->stream && cudaStreamSynchronize(stream) != cudaSuccess) return fail(RTW_ERR_CUDA, "trace kernel failed");
    return RTW_OK;
}
