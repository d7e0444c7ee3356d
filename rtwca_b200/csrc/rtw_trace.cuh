// rtw_trace.cuh - the persistent trace kernel.
//
// Work decomposition (B200-first, not the reference's one-thread-per-pixel
// grid-stride loop of 5P.jl:73-99):
//  * A persistent grid; each warp owns 32 ray slots, one per lane. Lanes whose
//    ray terminated take the next rays from a global work counter with one
//    warp-aggregated atomic (ballot + popc), so warps stay full until the
//    queue drains (compaction by refill).
//  * Geodesic phase, one lane per ray: one adaptive Dormand-Prince attempt
//    (RKDP_Step_w_buffer!, integrators_LttM.jl:54-224) over the 8 geodesic
//    components plus the common optical depth tau (the emitters are grey, so
//    every tau slot of the reference's state is the same number). The stages
//    run as a rolled loop over one inlined right-hand side; the tableau sums
//    are shifted accumulators, so no register array is indexed dynamically
//    and the hot code stays small enough for the instruction cache. The
//    emitter numbers (A, X) of every stage go to shared memory.
//  * Spectral phase, warp-cooperative: for every ray of the warp whose
//    spectral slots change in this attempt (emission in a stage, or a
//    nonzero carried slope), the 32 lanes split its spectral bins, compute
//    the five new stage slopes of each bin, the 5th-order update and the
//    embedded error, reduce the error over the warp, and commit the bins if
//    the attempt is accepted. The per-bin state (intensity, carried slope)
//    lives in a per-warp scratch area [32 rays][np], read and written
//    coalesced along the bins.
//  * The step controller, termination test and the XYZ epilogue (a warp
//    reduction over bins) follow.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include "rtw_internal.h"
#include "rtw_scenes.cuh"

namespace rtw {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kMaxWarps = 4;  // warps per CTA (launch bound 128 threads)
// Lanes that share one ray's bins in a pass of the spectral phase (32, 16 or
// 8): a pass serves 32 / RTW_SPEC_LANES rays at once, each lane taking
// BPL * 32 / RTW_SPEC_LANES of its ray's bins. 32 serves one ray per pass.
// Measured on the Kerr disk at 1024^2 (64 bins, FP32-mixed, reference step):
// 32 lanes 385 ms, 16 lanes 376 ms, 8 lanes 405 ms (fewer passes, but each
// pass's chain is longer and the register demand spills into the geodesic
// phase); the spectral pass is bound by its dependency chain, not by the
// number of passes.
#ifndef RTW_SPEC_LANES
#define RTW_SPEC_LANES 16
#endif
constexpr int kSpecLanes = RTW_SPEC_LANES;
static_assert(kSpecLanes == 32 || kSpecLanes == 16 || kSpecLanes == 8 || kSpecLanes == 4, "RTW_SPEC_LANES");
constexpr int kSpecGroups = 32 / kSpecLanes;

// FP32-mixed with up to 64 bins: the intensity and carried-slope rows of the
// spectral phase live in shared memory (2 x 32 x np floats per warp, dynamic);
// the Kahan low parts, which the error reduction does not wait for, stay in the
// global scratch. RTW_SPEC_SHARED (rtw_internal.h, 0 by default: measured
// slower) 0 keeps every row in global memory.
template <bool MIXED, int BPL>
RTW_HD constexpr bool spec_in_shared() { return RTW_SPEC_SHARED && MIXED && BPL <= 2; }

// Dormand-Prince coefficients (64BitConstants.jl:28-37): a_sl, b_l (= a_7l), b*_l.
constexpr double a21 = 1.0 / 5;
constexpr double a31 = 3.0 / 40, a32 = 9.0 / 40;
constexpr double a41 = 44.0 / 45, a42 = -56.0 / 15, a43 = 32.0 / 9;
constexpr double a51 = 19372.0 / 6561, a52 = -25360.0 / 2187, a53 = 64448.0 / 6561, a54 = -212.0 / 729;
constexpr double a61 = 9017.0 / 3168, a62 = -355.0 / 33, a63 = 46732.0 / 5247, a64 = 49.0 / 176,
                 a65 = -5103.0 / 18656;
constexpr double b1 = 35.0 / 384, b3 = 500.0 / 1113, b4 = 125.0 / 192, b5 = -2187.0 / 6784, b6 = 11.0 / 84;
constexpr double bs1 = 5179.0 / 57600, bs3 = 7571.0 / 16695, bs4 = 393.0 / 640, bs5 = -92097.0 / 339200,
                 bs6 = 187.0 / 2100, bs7 = 1.0 / 40;
constexpr double e1 = b1 - bs1, e3 = b3 - bs3, e4 = b4 - bs4, e5 = b5 - bs5, e6 = b6 - bs6, e7 = -bs7;

// Shifted-accumulator form of the tableau. S[j] holds the partial sum
// sum_l a_{t,l} k_l of stage t = s + j while stage s is evaluated; after k_s,
// S[j] <- S[j+1] + kCoef[s-2][j] k_s with kCoef[s-2][j] = a_{s+1+j, s}
// (zero past stage 7). init_coef(j) = a_{2+j, 1}; the error weights are b_s - b*_s.
#define RTW_COEF_TABLE                 \
    {{a32, a42, a52, a62, 0.0},        \
     {a43, a53, a63, b3, 0.0},         \
     {a54, a64, b4, 0.0, 0.0},         \
     {a65, b5, 0.0, 0.0, 0.0},         \
     {b6, 0.0, 0.0, 0.0, 0.0},         \
     {0.0, 0.0, 0.0, 0.0, 0.0}}
#define RTW_ERR_TABLE {e1, 0.0, e3, e4, e5, e6, e7}
__constant__ double c_coef_d[6][5] = RTW_COEF_TABLE;
__constant__ float c_coef_f[6][5] = RTW_COEF_TABLE;
__constant__ double c_err_d[7] = RTW_ERR_TABLE;
__constant__ float c_err_f[7] = RTW_ERR_TABLE;
static const double h_coef[6][5] = RTW_COEF_TABLE;
static const double h_err[7] = RTW_ERR_TABLE;
RTW_HD constexpr double init_coef(int j) {
    return j == 0 ? a21 : j == 1 ? a31 : j == 2 ? a41 : j == 3 ? a51 : j == 4 ? a61 : b1;
}

template <class R>
RTW_HD R dp_coef(int it, int j) {
#ifdef __CUDA_ARCH__
    if constexpr (sizeof(R) == 4) return R(c_coef_f[it][j]);
    else return R(c_coef_d[it][j]);
#else
    return R(h_coef[it][j]);
#endif
}
template <class R>
RTW_HD R dp_err(int s1) {
#ifdef __CUDA_ARCH__
    if constexpr (sizeof(R) == 4) return R(c_err_f[s1]);
    else return R(c_err_d[s1]);
#else
    return R(h_err[s1]);
#endif
}

// Spectral scratch layout of one warp: for each field, [32 rays][np] values of
// type SR. Fields: 0 = intensity (high part), 1 = carried slope k1,
// 2 = intensity low part (MIXED only: Kahan compensation).
template <bool MIXED>
struct SpecTraits;
template <>
struct SpecTraits<false> {
    typedef double SR;
    static constexpr int kFields = 2;
};
template <>
struct SpecTraits<true> {
    typedef float SR;
    static constexpr int kFields = 3;
};

// Intensity slope of a bin: -A / (exp(X nu) - 1), X2 = X log2(e). The PTX
// approximations directly (ex2.approx.ftz: 2^v, rcp.approx.ftz: 1/v), one
// MUFU op each; exp(X nu) >= 1, so flushing subnormals changes nothing. (The
// same two MUFU ops as exp2f and __fdividef, without their range wrappers:
// measured identical results, 14% less kernel time on the Kerr disk.)
__device__ __forceinline__ float ex2_ftz(float v) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(v));
    return r;
}
__device__ __forceinline__ float rcp_ftz(float v) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(v));
    return r;
}
__device__ __forceinline__ float bin_slope(float A, float X2, float nu) {
    return (A == 0.0f) ? 0.0f : -A * rcp_ftz(ex2_ftz(X2 * nu) - 1.0f);
}
__device__ __forceinline__ double bin_slope(double A, double X, double nu) {
    return (A == 0.0) ? 0.0 : -A / (exp(X * nu) - 1.0);
}
__device__ __forceinline__ float x_for_bins(float X) { return X * 1.4426950408889634f; }
__device__ __forceinline__ double x_for_bins(double X) { return X; }

__device__ __forceinline__ float rabs(float v) { return fabsf(v); }
__device__ __forceinline__ double rabs(double v) { return fabs(v); }
__device__ __forceinline__ float rmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double rmax(double a, double b) { return fmax(a, b); }

// Compensated (TwoSum) add into hi/lo.
__device__ __forceinline__ void kahan_add(float& hi, float& lo, float t) {
    const float s = hi + t;
    const float bp = s - hi;
    const float err = (hi - (s - bp)) + (t - bp);
    hi = s;
    lo += err;
}

// Step controller of RKDP_Step_w_buffer! (integrators_LttM.jl:185-224). CT is
// the arithmetic of the error norm: double on the FP64 path, float on the
// mixed path (err^(-1/5) then via the MUFU log2/exp2 pair).
__device__ __forceinline__ double err_pow(double err) { return pow(1.0 / err, 1.0 / 5); }
__device__ __forceinline__ double err_pow(float err) { return (double)exp2f(-0.2f * __log2f(err)); }

template <class CT>
__device__ __forceinline__ void decide(CT err2, int L, double h, double max_dt, bool prev_rej, bool& accept,
                                       double& hnext) {
    const CT err = sqrt(err2 / CT(L));
    double hn = 0.9 * h * err_pow(err);
    if (fabs(hn) > max_dt) hn = -max_dt;
    if (err == CT(0) || !isfinite(hn)) {
        accept = true;
        hnext = h;
    } else if (err > CT(1)) {
        if (prev_rej && fabs(hn) >= fabs(h)) hn = h / 2;
        accept = false;
        hnext = hn;
    } else {
        if (fabs(hn) > 5 * fabs(h)) hn = 5 * h;
        accept = true;
        hnext = hn;
    }
}

// One Dormand-Prince attempt of the geodesic + tau components in arithmetic R.
// x: FP64 state (8 geodesic + tau); k1: carried slope. Outputs the 5th-order
// slope ns = sum_l b_l k_l (the new state is x + h ns), the slope carried to
// the next step (ns, or k7 with FSAL), the emitter numbers of stages 2..7
// (A[j * stride], X[j * stride]) and the un-normalised squared error
// (arithmetic CT) of the geodesic and tau components (the tau term counted
// once per bin). Stage vectors carry a 10th entry, r - r_horizon, formed from
// the FP64 state. With R = double the stage points are the reference's
// Ray + h * sum(a k) and the 7th stage is evaluated at y = Ray + h * ns.
template <class SC, class R, class K, class SR, class CT>
RTW_HD void dp45_attempt(const DevScene& s, const double* x, const K* k1in, double h, double tol, int nbins,
                         bool fsal, K* ns_out, K* nk1, SR* A, SR* X, int stride, CT& err2, bool& emit) {
    // Components that enter the right-hand side (r, theta, k^mu, tau) carry the
    // six shifted stage sums; t and phi (indices 0, 3) enter no right-hand side,
    // so only their b-weighted sum (the 5th-order slope) is kept.
    constexpr int kC = 7;
    constexpr int kIdx[kC] = {1, 2, 4, 5, 6, 7, 8};
    R S[6][kC], es[9], k[9], z[10], xr[kC], nt, np3;
    Emit<R> em;
    const R hr = R(h);
    const R d0 = R(x[1] - s.r_ev);
#pragma unroll
    for (int c = 0; c < kC; ++c) {
        xr[c] = R(x[kIdx[c]]);
        const R k1 = R(k1in[kIdx[c]]);
#pragma unroll
        for (int j = 0; j < 6; ++j) S[j][c] = R(init_coef(j)) * k1;
    }
    nt = R(b1) * R(k1in[0]);
    np3 = R(b1) * R(k1in[3]);
#pragma unroll
    for (int i = 0; i < 9; ++i) es[i] = R(e1) * R(k1in[i]);
    z[0] = R(0);
    z[3] = R(0);
    emit = false;
#pragma unroll 1
    for (int it = 0; it < 6; ++it) {
#pragma unroll
        for (int c = 0; c < kC; ++c) z[kIdx[c]] = xr[c] + hr * S[0][c];
        z[9] = d0 + hr * S[0][0];
        SC::template rhs<R>(s, z, k, em);
        A[it * stride] = SR(em.A);
        X[it * stride] = SR(em.X);
        if (it > 0) emit = emit || (em.A != R(0));  // stage 2 has no weight in the bin update
        // Zero tableau entries (b2 = b*2 = 0, stages past 7) enter as 0 * k,
        // which is an exact 0 for any finite slope.
        const R ew = dp_err<R>(it + 1);
#pragma unroll
        for (int i = 0; i < 9; ++i) es[i] = es[i] + ew * k[i];
        if (it < 5) {
            // b_{it+2} is the coefficient into stage 7 (column 4 - it)
            const R bw = dp_coef<R>(it, 4 - it);
            nt = nt + bw * k[0];
            np3 = np3 + bw * k[3];
#pragma unroll
            for (int j = 0; j < 5; ++j) {
                const R cf = dp_coef<R>(it, j);
#pragma unroll
                for (int c = 0; c < kC; ++c) S[j][c] = S[j + 1][c] + cf * k[kIdx[c]];
            }
        }
    }
    // after the 7th stage: z holds y (r, theta, k, tau), S[0] the 5th-order slope
#pragma unroll
    for (int c = 0; c < kC; ++c) ns_out[kIdx[c]] = K(S[0][c]);
    ns_out[0] = K(nt);
    ns_out[3] = K(np3);
    if (fsal) {
#pragma unroll
        for (int i = 0; i < 9; ++i) nk1[i] = K(k[i]);
    } else {
#pragma unroll
        for (int i = 0; i < 9; ++i) nk1[i] = ns_out[i];
    }
    z[0] = R(x[0]) + hr * nt;
    z[3] = R(x[3]) + hr * np3;
    CT acc = CT(0);
    const CT hc = CT(h), tc = CT(tol);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const CT d = hc * CT(es[i]);
        const CT xa = (i == 0 || i == 3) ? CT(x[i]) : CT(xr[i < 3 ? i - 1 : i - 2]);
        const CT tl = tc + cmax(cabs(xa), cabs(CT(z[i]))) * tc;
        const CT q = cdiv(d, tl);
        acc += (i < 8 ? CT(1) : CT(nbins)) * q * q;
    }
    err2 = acc;
}

// Outputs of one attempt, returned by value from the out-of-line FP64 attempt
// so that no lane array of the hot path has its address taken.
template <class K, class CT>
struct AttemptOut {
    K ns[9];
    K nk1[9];
    CT err2;
    bool emit;
};

// The promoted (FP64-stage) attempt of the mixed path, kept out of line so
// that its register demand does not set the register budget of the hot FP32
// path; it runs for few rays.
template <class SC, class K, class SR, class CT>
__device__ __noinline__ AttemptOut<K, CT> dp45_attempt_fp64(const DevScene& s, const double* x, const K* k1in,
                                                             double h, double tol, int nbins, bool fsal, SR* A,
                                                             SR* X, int stride) {
    AttemptOut<K, CT> o;
    dp45_attempt<SC, double, K, SR, CT>(s, x, k1in, h, tol, nbins, fsal, o.ns, o.nk1, A, X, stride, o.err2, o.emit);
    return o;
}

// FP64 right-hand side, out of line (initial slope, polar escape).
template <class SC>
__device__ __noinline__ void rhs_fp64(const DevScene& s, const double* x9, double* k, Emit<double>* em) {
    double z[10];
#pragma unroll
    for (int i = 0; i < 9; ++i) z[i] = x9[i];
    z[9] = x9[1] - s.r_ev;
    SC::template rhs<double>(s, z, k, *em);
}

// Camera ray of pixel (i, j) of a frame (initialization.jl:213-240,327), FP64.
__device__ __forceinline__ void camera_ray(const FrameDesc& f, int i, int j, double* x) {
    // (i, j): the pixel in the frame's window; the direction is that of pixel
    // (i0 + i, j0 + j) of the whole image
    const double w = f.rh * ((f.i0 + i + 1) - 0.5) - f.W;
    const double hh = f.rv * ((f.j0 + j + 1) - 0.5) - f.H;
    const double th = atan(sqrt(w * w + hh * hh));
    double ph;
    if (w > 0) ph = atan(hh / w);
    else if (w < 0 && hh >= 0) ph = atan(hh / w) + kPi;
    else if (w < 0 && hh < 0) ph = atan(hh / w) - kPi;
    else if (w == 0 && hh > 0) ph = kPi / 2;
    else if (w == 0 && hh < 0) ph = -kPi / 2;
    else ph = 0;
    double st, ct, sp, cp;
    sincos(th, &st, &ct);
    sincos(ph, &sp, &cp);
    const double v[4] = {1.0, -st * cp, -st * sp, -ct};
#pragma unroll
    for (int k = 0; k < 4; ++k) x[k] = f.pos[k];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        double sacc = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) sacc += f.M[4 * r + k] * v[k];
        x[4 + r] = sacc;
    }
    x[8] = 0.0;
}

// Pixel (i, j) of the local ray id of a frame. Order 0: row order. Order 1:
// 8x4 tiles in row-major tile order; the columns right of the last full tile
// form a narrower tile, rows below the last full tile row are in row order.
__device__ __forceinline__ void pixel_of(int order, long long local, int xp, int yp, int& pi, int& pj) {
    if (order != 1) {
        pi = (int)(local % xp);
        pj = (int)(local / xp);
        return;
    }
    const int tw = 8, th = 4;
    const int full_rows = yp / th;
    const long long per_row = (long long)th * xp;
    const long long trow = local / per_row;
    if (trow < full_rows) {
        const long long rem = local - trow * per_row;
        const int full_cols = xp / tw;
        const long long in_full = (long long)full_cols * tw * th;
        if (rem < in_full) {
            const int tc = (int)(rem / (tw * th));
            const int w = (int)(rem % (tw * th));
            pi = tc * tw + (w % tw);
            pj = (int)trow * th + w / tw;
        } else {
            const int w = (int)(rem - in_full);
            const int rw = xp - full_cols * tw;
            pi = full_cols * tw + (w % rw);
            pj = (int)trow * th + w / rw;
        }
    } else {
        const long long rem = local - (long long)full_rows * per_row;
        pi = (int)(rem % xp);
        pj = full_rows * th + (int)(rem / xp);
    }
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return __shfl_sync(kFull, v, 0);  // one association order for every lane
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return __shfl_sync(kFull, v, 0);
}

// Device-wide nanosecond clock (PTX %globaltimer).
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Polar / origin escape (integrators_LttM.jl:62-105): 37 explicit Euler steps
// of size temp through the coordinate singularity, FP64; the spectral slots of
// this ray (its row of the warp's scratch) are updated by this lane.
// x and k1 (copies of the lane state) are updated in place. Returns whether
// the ray terminated inside the escape; otherwise k1 is the slope at the new
// position and spec_live tells whether any bin slope is nonzero.
struct EscapeOut {
    bool terminated;
    bool spec_live;
    unsigned substeps;
};
template <int KIND, bool MIXED>
__device__ __noinline__ EscapeOut polar_escape(const KParams& p, double* x, typename SpecTraits<MIXED>::SR* k1,
                                               double temp, double r_term, double thick,
                                               typename SpecTraits<MIXED>::SR* rI,
                                               typename SpecTraits<MIXED>::SR* rK,
                                               typename SpecTraits<MIXED>::SR* rL, bool spec_live_in) {
    EscapeOut out;
    out.terminated = false;
    out.spec_live = spec_live_in;
    out.substeps = 0;
    typedef typename SceneOf<KIND>::type SC;
    typedef typename SpecTraits<MIXED>::SR SR;
    const int N = p.n_bins;
    const DevScene& s = p.sc;
    auto euler_spec = [&]() {
        for (int c = 0; c < N; ++c) {
            const SR t = SR(-temp) * rK[c];
            if constexpr (MIXED) {
                float hi = rI[c], lo = rL[c];
                kahan_add(hi, lo, t);
                rI[c] = hi;
                rL[c] = lo;
            } else {
                rI[c] = rI[c] + t;
            }
        }
    };
    auto slope_all = [&]() {
        double kd[9];
        Emit<double> e;
        rhs_fp64<SC>(s, x, kd, &e);
        for (int i = 0; i < 9; ++i) k1[i] = SR(kd[i]);
        const SR Ae = SR(e.A), Xe = x_for_bins(SR(e.X));
        bool nz = false;
        for (int c = 0; c < N; ++c) {
            const SR v = bin_slope(Ae, Xe, SR(p.bin_nu[c]));
            rK[c] = v;
            nz |= v != SR(0);
        }
        out.spec_live = nz;
    };
    for (int i = 0; i < 9; ++i) x[i] -= temp * double(k1[i]);
    euler_spec();
    keep_in_bounds<KIND>(x);
    ++out.substeps;
    for (int it = 0; it < 36; ++it) {
        if (!terminate_geo<KIND>(s, x, r_term, thick)) {
            slope_all();
            for (int i = 0; i < 9; ++i) x[i] -= temp * double(k1[i]);
            euler_spec();
            keep_in_bounds<KIND>(x);
            ++out.substeps;
        }
    }
    if (terminate_geo<KIND>(s, x, r_term, thick)) {
        out.terminated = true;
        return out;
    }
    slope_all();
    return out;
}

// A new ray: its frame (binary search over the frame offsets), pixel, FP64
// initial state, first step size and slope, and the frame-start stamp. Runs
// once per ray, so it is kept out of line: its FP64 atan, sincos and 64-bit
// divisions would otherwise sit between the hot phases of the loop (measured
// 1-3 % faster, identical results).
template <class K>
struct FreshRay {
    double x[9];
    K k1[9];
    long long gid, max_steps;
    double tol, r_term, thick, h, A, X;
    int fi;
};
template <int KIND, class K, class CT>
__device__ __noinline__ FreshRay<K> fresh_ray(const KParams& p, long long id) {
    typedef typename SceneOf<KIND>::type SC;
    FreshRay<K> o;
    int lo = 0, hi = p.n_frames - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (p.frames[mid].ray_begin <= id) lo = mid; else hi = mid - 1;
    }
    const FrameDesc& f = p.frames[lo];
    o.fi = lo;
    if (p.frame_clock && id == f.ray_begin) p.frame_clock[p.n_frames + lo] = global_ns();
    int pi, pj;
    pixel_of(p.pixel_order, id - f.ray_begin, f.xp, f.yp, pi, pj);
    o.gid = f.ray_begin + pi + (long long)f.xp * pj;
    camera_ray(f, pi, pj, o.x);
    o.tol = f.tol;
    o.r_term = f.r_term;
    o.thick = f.thick;
    o.max_steps = f.max_steps;
    o.h = -pad_max_dt<KIND, CT>(p.sc, o.x, p.max_dt_scale);
    double kd[9];
    Emit<double> em;
    rhs_fp64<SC>(p.sc, o.x, kd, &em);
    for (int i = 0; i < 9; ++i) o.k1[i] = K(kd[i]);
    o.A = em.A;
    o.X = em.X;
    return o;
}

// The tail queue's record of a ray, written and read out of line (both run
// once per queued ray; inline, their state copies raised the hot loop's
// spills).
template <class K>
__device__ __noinline__ void tail_store(TailRec* t, const double* x, const K* k1, double h, double tol, double r_term,
                                        double thick, long long gid, long long nsteps, long long max_steps, int fi,
                                        bool prev_rej, bool spec_live) {
    for (int i = 0; i < 9; ++i) {
        t->x[i] = x[i];
        t->k1[i] = float(k1[i]);
    }
    t->h = h;
    t->tol = tol;
    t->r_term = r_term;
    t->thick = thick;
    t->gid = gid;
    t->nsteps = nsteps;
    t->max_steps = max_steps;
    t->fi = fi;
    t->prev_rej = prev_rej ? 1 : 0;
    t->spec_live = spec_live ? 1 : 0;
}
template <class T>
__device__ __noinline__ T tail_load(const T* t) { return *t; }

// Launch bounds: 128 threads per CTA; RTW_MIXED_MIN_CTAS resident CTAs per SM
// for the mixed kernel (3: 168 registers per thread, measured faster than 4
// with spills or 2), 2 for the FP64 kernel.
#ifndef RTW_MIXED_MIN_CTAS
#define RTW_MIXED_MIN_CTAS 3
#endif
// The spectral rows of the rays that entered the warp in this iteration (the
// lanes in fm): intensity 0 and the carried slope at the camera (main pass;
// A and X of the ray's first slope in its lane), or the rows the ray left the
// main pass with (tail pass; tail_id its queue record). Out of line, like the
// epilogue: once per ray.
template <bool MIXED, int BPL>
__device__ __noinline__ void init_rows(const KParams& p, typename SpecTraits<MIXED>::SR* sI,
                                       typename SpecTraits<MIXED>::SR* sK, typename SpecTraits<MIXED>::SR* sL,
                                       int np, int N, int lane, unsigned fm, bool tail_pass, long long tail_id,
                                       double A, double X) {
    typedef typename SpecTraits<MIXED>::SR SR;
    while (fm) {
        const int r = __ffs(fm) - 1;
        fm &= fm - 1;
        if (tail_pass) {
            const float* row = p.tail_spec + __shfl_sync(kFull, tail_id, r) * (long long)SpecTraits<MIXED>::kFields * np;
#pragma unroll
            for (int b = 0; b < BPL; ++b) {
                const int c = lane + 32 * b;
                if (c < N) {
                    sI[r * np + c] = row[c];
                    sK[r * np + c] = row[np + c];
                    if constexpr (MIXED) sL[r * np + c] = row[2 * np + c];
                }
            }
        } else {
            const SR A0 = SR(__shfl_sync(kFull, A, r));
            const SR X0 = x_for_bins(SR(__shfl_sync(kFull, X, r)));
#pragma unroll
            for (int b = 0; b < BPL; ++b) {
                const int c = lane + 32 * b;
                if (c < N) {
                    sI[r * np + c] = SR(0);
                    sK[r * np + c] = bin_slope(A0, X0, SR(p.bin_nu[c]));
                    if constexpr (MIXED) sL[r * np + c] = SR(0);
                }
            }
        }
    }
}

// FP32-mixed main pass: the lanes in hm (want set) hand their rays to the tail
// pass's queue, state (on copies) and spectral rows; returns whether this
// lane's ray went (slots past the queue's capacity keep their ray). Out of line.
template <int BPL, class K>
__device__ __noinline__ bool tail_hand_off(const KParams& p, unsigned hm, bool want, const double* xe, const K* ke,
                                           double h, double tol, double r_term, double thick, long long gid,
                                           long long nsteps, long long max_steps, int fi, bool prev_rej,
                                           bool spec_live, const float* sI, const float* sK, const float* sL, int np,
                                           int N, int lane) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(&p.stats->tail_rays, (unsigned long long)__popc(hm));
    base = __shfl_sync(kFull, base, 0);
    const long long slot = (long long)base + __popc(hm & ((1u << lane) - 1u));
    const bool go = want && slot < p.tail_cap;
    if (go)
        tail_store<K>(p.tail + slot, xe, ke, h, tol, r_term, thick, gid, nsteps, max_steps, fi, prev_rej, spec_live);
    unsigned gm = __ballot_sync(kFull, go);
    while (gm) {
        const int r = __ffs(gm) - 1;
        gm &= gm - 1;
        float* row = p.tail_spec + __shfl_sync(kFull, slot, r) * (long long)SpecTraits<true>::kFields * np;
#pragma unroll
        for (int b = 0; b < BPL; ++b) {
            const int c = lane + 32 * b;
            if (c < N) {
                row[c] = sI[r * np + c];
                row[np + c] = sK[r * np + c];
                row[2 * np + c] = sL[r * np + c];
            }
        }
    }
    return go;
}

// The epilogue of the rays that finished in this iteration (the lanes in fm):
// their XYZ by a warp reduction over the bins, and their spectra. Out of line:
// it runs once per ray, not per attempt, and its code stays out of the hot
// loop's (measured 4-5 % faster on the Kerr disk).
template <bool MIXED, int BPL>
__device__ __noinline__ void xyz_epilogue(const KParams& p, const typename SpecTraits<MIXED>::SR* sI,
                                          const typename SpecTraits<MIXED>::SR* sL, int np, int N, int lane,
                                          unsigned fm, long long gid) {
    while (fm) {
        const int r = __ffs(fm) - 1;
        fm &= fm - 1;
        const long long og = __shfl_sync(kFull, gid, r);
        float X_ = 0, Y_ = 0, Z_ = 0;
#pragma unroll
        for (int b = 0; b < BPL; ++b) {
            const int c = lane + 32 * b;
            if (c < N) {
                double I = (double)sI[r * np + c];
                if constexpr (MIXED) I += (double)sL[r * np + c];
                X_ += (float)(I * p.bin_fx[c]);
                Y_ += (float)(I * p.bin_fy[c]);
                Z_ += (float)(I * p.bin_fz[c]);
                if (p.spectrum) p.spectrum[og * N + c] = (float)I;
            }
        }
        X_ = warp_sum(X_);
        Y_ = warp_sum(Y_);
        Z_ = warp_sum(Z_);
        if (lane == r && p.xyz) {
            p.xyz[3 * og + 0] = X_;
            p.xyz[3 * og + 1] = Y_;
            p.xyz[3 * og + 2] = Z_;
        }
    }
}

template <int KIND, bool MIXED, int BPL>
__global__ void __launch_bounds__(128, MIXED ? RTW_MIXED_MIN_CTAS : 2) trace_kernel(const KParams p) {
    typedef typename SceneOf<KIND>::type SC;
    typedef SpecTraits<MIXED> ST;
    typedef typename ST::SR SR;
    typedef typename ST::SR K;  // carried slope and 5th-order increment
    typedef typename ST::SR R;  // stage arithmetic (promoted to double per ray)
    typedef typename ST::SR CT; // step-controller arithmetic

    // per-lane emitter numbers of stages 2..7, read by the spectral phase
    __shared__ SR s_ax[kMaxWarps][2][6][32];

    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const long long warp_id = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int N = p.n_bins;
    const int np = p.np;
    const int L = 8 + 2 * N;
    const DevScene& s = p.sc;
    SR* spec = reinterpret_cast<SR*>(p.spec) + warp_id * (long long)ST::kFields * 32 * np;
    extern __shared__ __align__(16) unsigned char s_rows[];
    constexpr bool kShRows = spec_in_shared<MIXED, BPL>();
    SR* sI = kShRows ? reinterpret_cast<SR*>(s_rows) + wib * 2 * 32 * np : spec;  // [32][np]
    SR* sK = sI + 32 * np;                                                       // [32][np]
    SR* sL = spec + 2 * 32 * np;    // [32][np] (MIXED only)
    SR* myA = &s_ax[wib][0][0][lane];
    SR* myX = &s_ax[wib][1][0][lane];

    // the lane's bins in a spectral pass (c = sub + kSpecLanes * b)
    constexpr int kBL = BPL * kSpecGroups;
    const int grp = lane / kSpecLanes, sub = lane % kSpecLanes;
    SR nus[kBL];
#pragma unroll
    for (int b = 0; b < kBL; ++b) {
        const int c = sub + kSpecLanes * b;
        nus[b] = c < N ? SR(p.bin_nu[c]) : SR(0);
    }

    // lane ray state
    bool active = false, dry = false;
    long long gid = 0;  // global output index
    int fi = 0;         // frame of the lane's ray
    double x[9];
    K k1[9];
    double h = 0, tol = 0, r_term = 0, thick = 0;
    long long max_steps = 0;
    long long nsteps = 0;
    bool prev_rej = false, spec_live = false;
    // local counters
    unsigned c_att = 0, c_rej = 0, c_pro = 0, c_spec = 0, c_emit = 0, c_esc = 0, c_nan = 0, c_rays = 0;

#ifdef RTW_PHASE_CLOCKS
    // profiling build: cycles each warp spends per phase (lane 0 records)
    unsigned long long cy_ref = 0, cy_geo = 0, cy_spec = 0, cy_com = 0;
    long long t_mark = clock64();
#define RTW_PHASE(acc)                       \
    do {                                     \
        const long long t_now = clock64();   \
        acc += (unsigned long long)(t_now - t_mark); \
        t_mark = t_now;                      \
    } while (0)
#else
#define RTW_PHASE(acc) do {} while (0)
#endif
    // the tail pass takes the queued rays (at most tail_cap), with its own counter
    const bool tail_pass = MIXED && p.tail_mode;
    const long long total_rays =
        tail_pass ? (long long)min(*(volatile unsigned long long*)&p.stats->tail_rays, (unsigned long long)p.tail_cap)
                  : p.total_rays;
    unsigned long long* const work_counter = tail_pass ? &p.stats->tail_counter : p.counter;
    long long tail_id = -1;  // tail pass: the queue record of the lane's ray
    for (;;) {
        // ---------------- refill -----------------------------------------
        const unsigned empty = __ballot_sync(kFull, !active);
        bool fresh = false;
        Emit<double> em0;
        em0.A = 0; em0.X = 0; em0.ktau = 0;
        if (empty && !dry && (__popc(empty) >= p.refill_min || empty == kFull)) {
            unsigned long long base = 0;
            const unsigned n = __popc(empty);
            if (lane == 0) base = atomicAdd(work_counter, (unsigned long long)n);
            base = __shfl_sync(kFull, base, 0);
            if ((long long)(base + n) >= total_rays) dry = true;
            if (!active && tail_pass) {
                const long long id = (long long)base + __popc(empty & ((1u << lane) - 1u));
                if (id < total_rays) {
                    const TailRec t = tail_load(p.tail + id);
#pragma unroll
                    for (int i = 0; i < 9; ++i) {
                        x[i] = t.x[i];
                        k1[i] = K(t.k1[i]);
                    }
                    gid = t.gid;
                    fi = t.fi;
                    tol = t.tol;
                    r_term = t.r_term;
                    thick = t.thick;
                    max_steps = t.max_steps;
                    h = t.h;
                    nsteps = t.nsteps;
                    prev_rej = t.prev_rej != 0;
                    spec_live = t.spec_live != 0;
                    tail_id = id;
                    active = true;
                    fresh = true;
                }
            } else if (!active) {
                const long long id = (long long)base + __popc(empty & ((1u << lane) - 1u));
                if (id < total_rays) {
                    const FreshRay<K> fr = fresh_ray<KIND, K, CT>(p, id);
#pragma unroll
                    for (int i = 0; i < 9; ++i) {
                        x[i] = fr.x[i];
                        k1[i] = fr.k1[i];
                    }
                    gid = fr.gid;
                    fi = fr.fi;
                    tol = fr.tol;
                    r_term = fr.r_term;
                    thick = fr.thick;
                    max_steps = fr.max_steps;
                    h = fr.h;
                    em0.A = fr.A;
                    em0.X = fr.X;
                    nsteps = 0;
                    prev_rej = false;
                    spec_live = em0.A != 0.0;
                    active = true;
                    fresh = true;
                    ++c_rays;
                }
            }
        }
        // spectral init of fresh rays: I = 0, k1 = slope at the camera (tail
        // pass: the row the ray left the main pass with)
        {
            const unsigned fm = __ballot_sync(kFull, fresh);
            if (fm) init_rows<MIXED, BPL>(p, sI, sK, sL, np, N, lane, fm, tail_pass, tail_id, em0.A, em0.X);
        }
        const unsigned act = __ballot_sync(kFull, active);
        if (!act) break;
        __syncwarp();
        RTW_PHASE(cy_ref);

        // ---------------- hand-off to the tail pass (FP32-mixed) ---------
        // A ray within promote_dr of the horizon leaves the lane here, at the
        // start of an attempt, with its whole state; the tail pass resumes
        // this attempt. Such a ray is inside the photon sphere moving inwards
        // and falls in from there, so it would run FP64 attempts (about 400)
        // for the rest of its path in a lane of an otherwise FP32 warp. Rays
        // near a pole stay: they leave the pole's FP64 zone again, and their
        // remaining paths (thousands of steps along the axis) would set the
        // length of the tail pass. Slots past the queue's capacity keep their ray.
        if constexpr (MIXED) {
            if (p.tail && !tail_pass) {
                const bool want = active && (x[1] - s.r_ev < p.promote_dr);
                const unsigned hm = __ballot_sync(kFull, want);
                if (hm) {
                    // out of line on copies, so that x and k1 stay in registers
                    double xe[9];
                    K ke[9];
#pragma unroll
                    for (int i = 0; i < 9; ++i) {
                        xe[i] = x[i];
                        ke[i] = k1[i];
                    }
                    const bool go = tail_hand_off<BPL, K>(p, hm, want, xe, ke, h, tol, r_term, thick, gid, nsteps,
                                                          max_steps, fi, prev_rej, spec_live, sI, sK, sL, np, N, lane);
                    if (go) active = false;
                    __syncwarp();
                }
            }
        }

        // ---------------- geodesic phase ---------------------------------
        K ns[9];   // 5th-order slope: the new state is x + h ns
        K nk1[9];  // slope carried to the next attempt
        CT err2 = 0;
        double max_dt = 0, hnext = h;
        bool emit = false, esc_done = false, decided = false, accept = false, traced_promote = false;
        if (active) {
            ++c_att;
            max_dt = pad_max_dt<KIND, CT>(s, x, p.max_dt_scale);
            double temp;
            if (near_singularity<KIND>(x, h, tol, &temp)) {
                // out of line on copies, so that x and k1 stay in registers
                double xe[9];
                K ke[9];
#pragma unroll
                for (int i = 0; i < 9; ++i) {
                    xe[i] = x[i];
                    ke[i] = k1[i];
                }
                const EscapeOut eo = polar_escape<KIND, MIXED>(p, xe, ke, temp, r_term, thick, sI + lane * np,
                                                               sK + lane * np, sL + lane * np, spec_live);
#pragma unroll
                for (int i = 0; i < 9; ++i) {
                    x[i] = xe[i];
                    k1[i] = ke[i];
                }
                spec_live = eo.spec_live;
                c_esc += eo.substeps;
                if (eo.terminated) {
                    esc_done = true;
                    decided = true;
                    accept = true;
                    hnext = h;
                } else {
                    h = -pad_max_dt<KIND, CT>(s, x, p.max_dt_scale);
                }
            }
            if (!esc_done) {
                bool promote = false;
                if (MIXED) {
                    promote = (x[1] - s.r_ev < p.promote_dr) || (x[2] < p.promote_theta) ||
                              (x[2] > kPi - p.promote_theta);
                }
                traced_promote = promote;
                if (promote) {
                    ++c_pro;
                    double xe[9];
                    K ke[9];
#pragma unroll
                    for (int i = 0; i < 9; ++i) {
                        xe[i] = x[i];
                        ke[i] = k1[i];
                    }
                    const AttemptOut<K, CT> o =
                        dp45_attempt_fp64<SC, K, SR, CT>(s, xe, ke, h, tol, N, p.fsal != 0, myA, myX, 32);
#pragma unroll
                    for (int i = 0; i < 9; ++i) {
                        ns[i] = o.ns[i];
                        nk1[i] = o.nk1[i];
                    }
                    err2 = o.err2;
                    emit = o.emit;
                } else {
                    dp45_attempt<SC, R, K, SR, CT>(s, x, k1, h, tol, N, p.fsal != 0, ns, nk1, myA, myX, 32, err2,
                                                   emit);
                }
                if (emit) ++c_emit;
            }
        }
        __syncwarp();
        RTW_PHASE(cy_geo);

        // ---------------- spectral phase (warp-cooperative) --------------
        // Each pass serves the next kSpecGroups rays of the warp that need
        // bin work; kSpecLanes consecutive lanes split one ray's bins (bin
        // c = sub + kSpecLanes * b). A ray's arithmetic and the association
        // order of its error sum depend on kSpecLanes only, not on which
        // rays share its pass or which lane traces it.
        const bool need = active && !esc_done && (emit || spec_live);
        unsigned nm = __ballot_sync(kFull, need);
        if (need) ++c_spec;
        while (nm) {
            const unsigned pass_rays = nm;
            // this group's ray: the (grp+1)-th set bit of nm
            unsigned mg = nm;
#pragma unroll
            for (int g = 0; g < kSpecGroups - 1; ++g)
                if (g < grp) mg &= mg - 1u;
            const bool vg = mg != 0u;
            const int r = vg ? __ffs(mg) - 1 : __ffs(nm) - 1;  // an empty group repeats the first ray, discarded
#pragma unroll
            for (int g = 0; g < kSpecGroups; ++g) nm &= nm - 1u;
            SR Ar[5], Xr[5];
#pragma unroll
            for (int j = 0; j < 5; ++j) {  // stages 3..7
                Ar[j] = s_ax[wib][0][j + 1][r];
                Xr[j] = x_for_bins(s_ax[wib][1][j + 1][r]);
            }
            const SR hs = SR(__shfl_sync(kFull, h, r));
            const SR ts = SR(__shfl_sync(kFull, tol, r));
            SR yv[kBL], yl[kBL], nk[kBL];
            SR acc = 0;
            bool nz = false;
            // Branch-free over the lane's bins: a row holds np >= N slots, so
            // every load is in bounds; slots past N only feed discarded values.
#pragma unroll
            for (int b = 0; b < kBL; ++b) {
                const int c = sub + kSpecLanes * b;
                const bool ok = c < N;
                const SR I = sI[r * np + c];
                const SR kk1 = sK[r * np + c];
                const SR nuc = nus[b];
                const SR kk3 = bin_slope(Ar[0], Xr[0], nuc);
                const SR kk4 = bin_slope(Ar[1], Xr[1], nuc);
                const SR kk5 = bin_slope(Ar[2], Xr[2], nuc);
                const SR kk6 = bin_slope(Ar[3], Xr[3], nuc);
                const SR kk7 = bin_slope(Ar[4], Xr[4], nuc);
                // (k2 has zero weight in both the 5th-order update and the
                // error estimate, and the intensity slopes do not depend on
                // the intensity, so stage 2 needs no bin work.)
                const SR ns = kk1 * SR(b1) + kk3 * SR(b3) + kk4 * SR(b4) + kk5 * SR(b5) + kk6 * SR(b6);
                const SR es = kk1 * SR(e1) + kk3 * SR(e3) + kk4 * SR(e4) + kk5 * SR(e5) + kk6 * SR(e6) +
                              kk7 * SR(e7);
                SR yy, ylo = 0;
                if constexpr (MIXED) {
                    float hi = I, lo = sL[r * np + c];
                    kahan_add(hi, lo, hs * ns);
                    yy = hi;
                    ylo = lo;
                } else {
                    yy = I + hs * ns;
                }
                const SR d = hs * es;
                const SR tl = ts + rmax(rabs(I), rabs(yy)) * ts;
                const SR q = cdiv(d, tl);
                acc += ok ? q * q : SR(0);
                yv[b] = yy;
                yl[b] = ylo;
                nk[b] = p.fsal ? kk7 : ns;
                nz |= ok && nk[b] != SR(0);
            }
            // the group's sum, in one association order, in every lane of the group
#pragma unroll
            for (int o = kSpecLanes / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
            acc = __shfl_sync(kFull, acc, grp * kSpecLanes);
            // the lane that owns a ray of this pass decides its attempt
            const int rank = __popc(pass_rays & ((1u << lane) - 1u));
            const bool own = ((pass_rays >> lane) & 1u) && rank < kSpecGroups;
            const SR aown = __shfl_sync(kFull, acc, own ? rank * kSpecLanes : 0);
            int dec = 0;
            if (own) {
                decide<CT>(err2 + CT(aown), L, h, max_dt, prev_rej, accept, hnext);
                decided = true;
                dec = accept ? 1 : 0;
            }
            // every lane takes part in each collective (a full-mask shuffle
            // skipped by some lanes is undefined)
            const int dsrc = __shfl_sync(kFull, dec, r);
            const bool dg = vg && dsrc != 0;
            if (dg) {
#pragma unroll
                for (int b = 0; b < kBL; ++b) {
                    const int c = sub + kSpecLanes * b;
                    if (c < N) {
                        sI[r * np + c] = yv[b];
                        sK[r * np + c] = nk[b];
                        if constexpr (MIXED) sL[r * np + c] = yl[b];
                    }
                }
            }
            const unsigned nzb = __ballot_sync(kFull, vg && nz);
            constexpr unsigned kGroupMask = kSpecLanes == 32 ? kFull : ((1u << kSpecLanes) - 1u);
            if (own && dec) spec_live = ((nzb >> (rank * kSpecLanes)) & kGroupMask) != 0u;
        }
        __syncwarp();
        RTW_PHASE(cy_spec);

        // ---------------- controller + commit ----------------------------
        int cls = 0;
        if (active) {
            if (!decided) decide<CT>(err2, L, h, max_dt, prev_rej, accept, hnext);
            if (!esc_done) {
                if (accept) {
                    double y[9];
#pragma unroll
                    for (int i = 0; i < 9; ++i) y[i] = x[i] + h * double(ns[i]);
                    keep_in_bounds<KIND>(y);
#pragma unroll
                    for (int i = 0; i < 9; ++i) {
                        x[i] = y[i];
                        k1[i] = nk1[i];
                    }
                    prev_rej = false;
                } else {
                    keep_in_bounds<KIND>(x);
                    prev_rej = true;
                    ++c_rej;
                }
                h = hnext;
            } else {
                prev_rej = false;
            }
            ++nsteps;
            if (gid == p.trace_gid && nsteps <= p.trace_cap) {
                double* tr = p.trace + (nsteps - 1) * RTW_TRACE_FIELDS;
                tr[0] = (double)nsteps;
                tr[1] = h;
                tr[2] = accept ? 1.0 : 0.0;
                tr[3] = traced_promote ? 1.0 : 0.0;
                tr[4] = esc_done ? 1.0 : 0.0;
                tr[5] = (double)err2;
#pragma unroll
                for (int i = 0; i < 9; ++i) tr[6 + i] = x[i];
            }
            if (nsteps >= max_steps) cls = RTW_CLASS_MAXSTEPS;
            else cls = terminate_geo<KIND>(s, x, r_term, thick);
            if (cls) {
                bool fin = true;
#pragma unroll
                for (int i = 0; i < 8; ++i) fin &= isfinite(x[i]);
                if (!fin) {
                    cls = RTW_CLASS_NAN;
                    ++c_nan;
                }
            }
        }

        // ---------------- epilogue: XYZ, outputs -------------------------
        const bool fin = active && cls != 0;
        const unsigned fm = __ballot_sync(kFull, fin);
        if (fm) xyz_epilogue<MIXED, BPL>(p, sI, sL, np, N, lane, fm, gid);
        if (fin) {
            if (p.cls) p.cls[gid] = (uint8_t)cls;
            if (p.steps) p.steps[gid] = (uint32_t)nsteps;
            if (p.final_state) {
#pragma unroll
                for (int i = 0; i < 8; ++i) p.final_state[8 * gid + i] = x[i];
            }
            if (p.tau) p.tau[gid] = (float)x[8];
            if (p.frame_clock) {
                const unsigned long long done = atomicAdd(&p.frame_clock[fi], 1ull) + 1ull;
                if (done == (unsigned long long)p.frames[fi].xp * (unsigned long long)p.frames[fi].yp)
                    p.frame_clock[2 * p.n_frames + fi] = global_ns();
            }
            active = false;
        }
        __syncwarp();
        RTW_PHASE(cy_com);
    }
#ifdef RTW_PHASE_CLOCKS
    if (lane == 0) {
        atomicAdd(&p.stats->cyc_refill, cy_ref);
        atomicAdd(&p.stats->cyc_geo, cy_geo);
        atomicAdd(&p.stats->cyc_spec, cy_spec);
        atomicAdd(&p.stats->cyc_commit, cy_com);
    }
#endif

    // counters
    atomicAdd(&p.stats->step_attempts, (unsigned long long)c_att);
    atomicAdd(&p.stats->rejected_steps, (unsigned long long)c_rej);
    atomicAdd(&p.stats->promoted_steps, (unsigned long long)c_pro);
    atomicAdd(&p.stats->spectral_steps, (unsigned long long)c_spec);
    atomicAdd(&p.stats->emitting_steps, (unsigned long long)c_emit);
    atomicAdd(&p.stats->escape_substeps, (unsigned long long)c_esc);
    atomicAdd(&p.stats->nan_rays, (unsigned long long)c_nan);
    atomicAdd(&p.stats->rays, (unsigned long long)c_rays);
}

}  // namespace rtw
