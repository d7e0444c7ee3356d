// rtw_internal.h - types shared by the host side of the C ABI and the trace
// kernels (not part of the public ABI).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/rtw.h"

// FP32-mixed trace kernel with up to 64 bins: the spectral phase's intensity
// and carried-slope rows in shared memory (1), or in the global scratch (0).
// Measured on the Kerr disk at 1024^2 (reference step, tail pass on): 390 ms
// with the rows in shared memory, 335 ms without (FSAL: 167 / 131 ms): the
// 64 KB per CTA leave the L1 too small for the kernel's local memory.
#ifndef RTW_SPEC_SHARED
#define RTW_SPEC_SHARED 0
#endif

namespace rtw {

// One frame (camera) of a batched render: the FP64 camera transform of
// initialize_camera (initialization.jl:190-331) reduced to what a pixel needs.
struct FrameDesc {
    double pos[4];       // camera 4-position
    double M[16];        // row-major e * R2 * L * R (initialization.jl:254-260,327)
    double W, H;         // canvas half extents tan(fov/2)
    double rh, rv;       // inverse pixel densities (initialization.jl:202-203)
    double tol;          // abs_tol = rel_tol
    double r_term;       // horizon termination radius (1 + 10 tol) r_horizon
    double thick;        // -log(tol): optically thick threshold
    long long ray_begin; // first global ray id of this frame
    long long max_steps;
    int xp, yp;          // the frame's (window's) pixels
    int i0, j0;          // the window's origin in the whole image
};

// Scene constants in the form the device functors use.
struct DevScene {
    int kind;
    int refprec;
    double M, a, rs, r_ev;
    double r_in, r_out, th_lo, th_hi;
    double T, anu, esc, wind;
    double rho_r0, rho_h, rho_idx, t_idx;
    double sqrtM;
    double r_pm;  // r+ - r- (Kerr), rs (Schwarzschild: Delta/r = r - rs), 0 (flat)
};

// Counters one render accumulates on the device (rtw_stats).
struct DevStats {
    unsigned long long step_attempts;
    unsigned long long rejected_steps;
    unsigned long long promoted_steps;
    unsigned long long spectral_steps;
    unsigned long long emitting_steps;
    unsigned long long escape_substeps;
    unsigned long long nan_rays;
    unsigned long long rays;
    // RTW_PHASE_CLOCKS builds only: SM cycles per phase, summed over warps
    unsigned long long cyc_refill, cyc_geo, cyc_spec, cyc_commit;
    // rays handed to the FP64 tail pass (slots asked for; the pass takes at
    // most the queue's capacity), and the tail pass's work counter
    unsigned long long tail_rays, tail_counter;
};

// A ray handed from the main pass of the FP32-mixed trace kernel to its tail
// pass, at the start of an attempt: the lane state, exactly. Its spectral row
// (intensity, carried slope, Kahan low part, np values each) is stored apart.
struct TailRec {
    double x[9];
    double h, tol, r_term, thick;
    long long gid, nsteps, max_steps;
    float k1[9];
    int fi, prev_rej, spec_live;
};

struct KParams {
    DevScene sc;
    const FrameDesc* frames;
    int n_frames;
    int n_bins;
    long long total_rays;
    double max_dt_scale;
    double promote_dr;     // MIXED: FP64 stages while r - r_horizon < promote_dr
    double promote_theta;  // MIXED: FP64 stages while theta < promote_theta or > pi - promote_theta
    int fsal;
    int pixel_order;
    // per-bin tables, [n_bins]: observed frequency (nm^-1) and the factors
    // nu^3 c / lambda^2 * W_{X,Y,Z} of the XYZ epilogue
    const double* bin_nu;
    const double* bin_fx;
    const double* bin_fy;
    const double* bin_fz;
    // spectral scratch: per warp [32 rays][np] for each field
    void* spec;
    int np;                      // padded bins per ray row (32 * bins per lane)
    unsigned long long* counter; // work queue head
    DevStats* stats;
    // outputs (device pointers; may be null)
    float* xyz;
    uint8_t* cls;
    uint32_t* steps;
    float* spectrum;
    double* final_state;
    float* tau;
    // step trace of one ray (RTW_TRACE_FIELDS doubles per attempt)
    double* trace;
    long long trace_gid;
    int trace_cap;
    // a warp refills its empty lanes once at least refill_min are empty (or
    // all are), so that fresh rays start together
    int refill_min;
    // per-frame timing (may be null): [n_frames] finished-ray counters, then
    // [n_frames] global-timer ns when the frame's first ray started, then
    // [n_frames] when its last ray finished
    unsigned long long* frame_clock;
    // FP32-mixed kernel: rays within promote_dr of the horizon at the start
    // of an attempt leave the main pass (tail_mode 0) for the queue `tail`
    // (tail_cap records, spectral rows in tail_spec [tail_cap][3][np]); the
    // tail pass (tail_mode 1) traces them with whole warps of such rays.
    // tail NULL: every ray stays in its lane.
    TailRec* tail;
    float* tail_spec;
    long long tail_cap;
    int tail_mode;
};

// Scene constants of the device functors from the public scene struct.
void make_dev_scene(const rtw_scene& scene, DevScene& d);

// Launches the trace kernel for p.sc.kind / precision on `stream`.
// Returns cudaSuccess or the launch error.
cudaError_t launch_trace(const KParams& p, int precision, int grid, int block, cudaStream_t stream);
// Launches the plain FP64 one-thread-per-pixel kernel (RTW_PREC_FP64_PLAIN).
cudaError_t launch_plain(const KParams& p, int grid, int block, cudaStream_t stream);
// Bytes of spectral scratch per warp for a precision and padded bin count.
size_t spec_bytes_per_warp(int precision, int np);
// Dynamic shared memory of a trace-kernel CTA of `warps` warps (the spectral
// rows kept in shared memory: FP32-mixed, np <= 64), and the kernel attribute
// that allows it (call before a launch or an occupancy query).
size_t trace_dyn_smem(int precision, int np, int warps);
cudaError_t trace_allow_smem(int kind, int precision, int np);
// Registers / max threads of the kernel that launch_trace would run.
cudaError_t trace_attributes(int kind, int precision, int np, cudaFuncAttributes* attr);

// Issue-rate microbenchmarks (rtw_measure_peaks).
cudaError_t launch_peak_probe(int which, int grid, int block, int iters, float* sink, cudaStream_t stream);

}  // namespace rtw
