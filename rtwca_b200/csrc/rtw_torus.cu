// rtw_torus.cu - the synchrotron torus: forward render (FP32-mixed or FP64,
// FSAL Dormand-Prince, per-bin optical depth) and its discrete adjoint.
//
// Forward: one lane per ray, rays taken from a global queue one at a time
// (per-lane refill; the lanes of a warp do not cooperate here). Per attempt
// the seven geodesic stages run first (scene functor of rtw_scenes.cuh) and
// leave six emitter-number sets (cj, nus, Theta, g) in local memory; then
// each bin runs its own seven tau / I stages from those numbers in registers.
// The error norm is the reference's RMS over all 8 + 2N components
// (integrators_LttM.jl:185-224).
//
// Adjoint: one recording forward pass gives the image and, per ray, a chain
// of chunks taken from a pool by an atomic counter, each chunk one segment:
// the state before it and the sizes and kinds of its `ck_every` accepted
// steps (and polar escapes). Rays with a polar escape whose gradient is
// wanted are recorded again, alone, with their state before every event.
// The reverse pass, one lane per ray in FP64, walks the segments backwards:
// it replays a segment's geodesic from its checkpoint, then reverses each
// step through its stages with vector-Jacobian products of the right-hand
// side built from dual numbers (rtw_dual.cuh), running the optical depths
// back from the segment's end.
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <cmath>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "rtw_ctx.h"
#include "rtw_trace.cuh"
#include "rtw_torus.cuh"

extern "C" rtw_status rtw_cie_weights(const double* colors_nm, int32_t n_colors, double* w_x, double* w_y,
                                      double* w_z, double* i_lambda_factor);
extern "C" rtw_status rtw_prepare_frames(const rtw_scene* scene, const rtw_camera* cams, int32_t n_cams,
                                         void* frames_out, int64_t* total_out);

namespace rtw {

// FSAL Dormand-Prince: stage s point = y + h sum_{j<s} A[s][j] K_j (row 6 =
// the 5th-order weights b, whose point is the new state), error weights E.
#define RTW_TORUS_A                                        \
    {{0, 0, 0, 0, 0, 0},                                   \
     {a21, 0, 0, 0, 0, 0},                                 \
     {a31, a32, 0, 0, 0, 0},                               \
     {a41, a42, a43, 0, 0, 0},                             \
     {a51, a52, a53, a54, 0, 0},                           \
     {a61, a62, a63, a64, a65, 0},                         \
     {b1, 0, b3, b4, b5, b6}}
#define RTW_TORUS_E {e1, 0, e3, e4, e5, e6, e7}
__constant__ double c_tA[7][6] = RTW_TORUS_A;
__constant__ double c_tE[7] = RTW_TORUS_E;
static const double h_tA[7][6] = RTW_TORUS_A;
static const double h_tE[7] = RTW_TORUS_E;
RTW_HD double tA(int s, int j) {
#ifdef __CUDA_ARCH__
    return c_tA[s][j];
#else
    return h_tA[s][j];
#endif
}
RTW_HD double tE(int s) {
#ifdef __CUDA_ARCH__
    return c_tE[s];
#else
    return h_tE[s];
#endif
}

// Everything a right-hand side needs.
struct TorusModel {
    DevScene geo;  // Kerr geodesic functor (its thin disk switched off)
    TorusDev tor;
    PowehiDev pw;
    SynchroDev sy;
    WormholeDev wh;
    TorusBin bins[kTorusMaxBins];
    int n;         // bins
    int emitter;   // 0: synchrotron torus, 1: Powehi (disk + jet), 2: Synchro_Test cylinder, 3: none (wormhole),
                   // 4: the Cartesian blackbody sphere, 5: the bremsstrahlung torus
    int geom;      // geometry: 0 Kerr (Boyer-Lindquist), 1 Minkowski (Cartesian), 2 Dneg wormhole
    SphereDev sp;
    BremsDev br;
};

// The scene's emitter at a stage point z (x^mu, k^mu) and the slopes of bin c.
// (EM: the emitter, -1 the model's at run time; the kernels instantiate one
// emitter each, so the others' code stays out of their hot loops)
template <class R, int EM = -1>
RTW_HD TorusPt<R> em_point(const TorusModel& m, const R* z) {
    if (EM == 3 || (EM == -1 && m.emitter == 3)) {  // the wormhole: empty space everywhere
        TorusPt<R> o;
        o.on = false;
        o.zone = 0;
        o.cj = R(0.0); o.nus = R(0.0); o.th = R(1.0); o.g = R(1.0);
        return o;
    }
    if (EM == 4 || (EM == -1 && m.emitter == 4)) return sphere_point<R>(m.sp, z);
    if (EM == 5 || (EM == -1 && m.emitter == 5))
        return brems_point<R>(m.tor, m.br, R(m.tor.a), R(m.tor.n0), R(m.tor.Th0), z[1], z[2], z[4], z[7]);
    if (EM == 2 || (EM == -1 && m.emitter == 2)) return synchro_point<R>(m.sy, z);
    if (EM == 1 || (EM == -1 && m.emitter == 1)) return powehi_point<R>(m.pw, z);
    return torus_point<R>(m.tor, R(m.tor.a), R(m.tor.n0), R(m.tor.B0), R(m.tor.Th0), z[1], z[2], z[4], z[7]);
}
template <class R, int EM = -1>
RTW_HD void em_bin(const TorusModel& m, const TorusPt<R>& S, int c, R& ft, R& fi) {
    if (EM == 4 || (EM == -1 && m.emitter == 4)) sphere_bin<R>(m.sp, S, m.bins[c].nu_nm, ft, fi);
    else if (EM == 5 || (EM == -1 && m.emitter == 5)) brems_bin<R>(m.br, S, m.bins[c], ft, fi);
    else if (EM > 0 || (EM == -1 && m.emitter != 0)) powehi_bin<R>(m.pw, S, m.bins[c].nu_nm, ft, fi);
    else torus_bin<R>(S.cj, S.nus, S.th, S.g, m.bins[c], ft, fi);
}

// The geodesic part of the right-hand side (8 components of y).
RTW_HD void torus_geo_rhs(const TorusModel& m, const double* y, double* f) {
    if (m.geom == 2) {
        wormhole_rhs<double>(m.wh, y, f);
        return;
    }
    if (m.geom == 1) {  // straight lines (Synchro_Test.source/source_geometry.jl:55-66 and the Cartesian sphere's)
        for (int i = 0; i < 4; ++i) {
            f[i] = y[4 + i];
            f[4 + i] = 0;
        }
        return;
    }
    double z[10], k[9];
    for (int i = 0; i < 8; ++i) z[i] = y[i];
    z[8] = 0;
    z[9] = y[1] - m.geo.r_ev;
    Emit<double> em;
    KerrScene<false>::rhs<double>(m.geo, z, k, em);
    for (int i = 0; i < 8; ++i) f[i] = k[i];
}

// FP64 right-hand side on a state y[8 + 2N] = (x^mu, k^mu, tau_c, I_c)
// (EM: the emitter as in em_point; the forward kernels pass their own).
template <int EM = -1>
RTW_HD void torus_f64(const TorusModel& m, const double* y, double* f) {
    const int N = m.n;
    torus_geo_rhs(m, y, f);
    const TorusPt<double> S = em_point<double, EM>(m, y);
    for (int c = 0; c < N; ++c) {
        double ft = 0, fi = 0;
        if (S.on) em_bin<double, EM>(m, S, c, ft, fi);
        f[8 + c] = ft;
        f[8 + N + c] = fi * exp(-y[8 + c]);
    }
}

// mu += J^T kap and pb += (d f / d(a, -, n0, b0, th0))^T kap at state y.
RTW_HD void torus_vjp(const TorusModel& m, const double* y, const double* kap, double* mu, double* pb) {
    const int N = m.n;
    // dx^mu / dl = k^mu
    for (int i = 0; i < 4; ++i) mu[4 + i] += kap[i];
    {
        typedef Dual<double, 7> D7;  // r, theta, k^t, k^r, k^theta, k^phi, a
        const D7 r = D7::var(y[1], 0), th = D7::var(y[2], 1), a = D7::var(m.tor.a, 6);
        D7 k[4], acc[4];
        for (int i = 0; i < 4; ++i) k[i] = D7::var(y[4 + i], 2 + i);
        kerr_accel<D7>(m.tor.M, a, r, th, k, acc);
        for (int i = 0; i < 4; ++i) {
            const double c = kap[4 + i];
            if (c == 0) continue;
            mu[1] += c * acc[i].d[0];
            mu[2] += c * acc[i].d[1];
            for (int q = 0; q < 4; ++q) mu[4 + q] += c * acc[i].d[2 + q];
            pb[0] += c * acc[i].d[6];
        }
    }
    typedef Dual<double, 8> D8;  // r, theta, k^t, k^phi, a, n0, b0, th0
    const TorusPt<D8> S = torus_point<D8>(m.tor, D8::var(m.tor.a, 4), D8::var(m.tor.n0, 5), D8::var(m.tor.B0, 6),
                                          D8::var(m.tor.Th0, 7), D8::var(y[1], 0), D8::var(y[2], 1),
                                          D8::var(y[4], 2), D8::var(y[7], 3));
    if (!S.on) return;
    double sb[4] = {0, 0, 0, 0};  // cotangent of (cj, nus, Theta, g)
    for (int c = 0; c < N; ++c) {
        double ft, fi, dft[4], dfi[4];
        torus_bin_grad(S.cj.v, S.nus.v, S.th.v, S.g.v, m.bins[c], ft, fi, dft, dfi);
        const double e = exp(-y[8 + c]);
        const double kt = kap[8 + c], ki = kap[8 + N + c];
        for (int q = 0; q < 4; ++q) sb[q] += kt * dft[q] + ki * e * dfi[q];
        mu[8 + c] += -ki * fi * e;  // d (fi exp(-tau)) / d tau
    }
    const D8* comp[4] = {&S.cj, &S.nus, &S.th, &S.g};
    double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int q = 0; q < 4; ++q)
        for (int t = 0; t < 8; ++t) v[t] += sb[q] * comp[q]->d[t];
    mu[1] += v[0];
    mu[2] += v[1];
    mu[4] += v[2];
    mu[7] += v[3];
    pb[0] += v[4];
    pb[2] += v[5];
    pb[3] += v[6];
    pb[4] += v[7];
}

// keepinbounds! (Kerr source_geometry.jl:275-301) on a full state; returns
// whether theta was reflected (theta and k^theta change sign, phi shifts).
RTW_HD bool torus_keep(double* x) {
    bool refl = false;
    if (x[2] < 0) {
        x[2] = -x[2];
        x[3] -= kPi;
        x[6] = -x[6];
        refl = !refl;
    }
    if (!(x[2] < 2 * kPi)) {
        double r = fmod(x[2], 2 * kPi);
        if (r < 0) r += 2 * kPi;
        x[2] = r;
    }
    if (x[2] >= kPi) {
        x[2] = 2 * kPi - x[2];
        x[3] += kPi;
        x[6] = -x[6];
        refl = !refl;
    }
    return refl;
}

// pad_max_dt of the Kerr scene (source_model.jl:86-103, the scale cast to
// Float32) over a generic scalar, for the derivative of the step sizes it sets:
// x2 = theta, vr, vth, vph = k^r, k^theta, k^phi.
template <class T>
RTW_HD T torus_pad(const T& x2, const T& vr, const T& vth, const T& vph, double scale_d) {
    typedef decltype(val(x2)) B;
    const double scale = (double)(float)scale_d;
    const double th = (double)val(x2);
    const double eps = (th < kPi / 8 || th > 7 * kPi / 8) ? fmin(scale, (double)1e-1f) : scale;
    auto tab = [](const T& v) { return val(v) < 0 ? -v : v; };
    const T first = tab(vr) * B(1.0 / eps) + B(kNoDivZero);
    const T pole = th <= kPi - th ? x2 : T(B(kPi)) - x2;
    const T second = T(B(1.0)) / (pole * B(eps) / (tab(vth) + B(kNoDivZero)) + B(kNoDivZero));
    const T third = T(B(1.0)) / (T(B(eps)) / (tab(vph) + B(kNoDivZero)) + B(kNoDivZero));
    const T m = T(B(1.0)) / (first + second + third + B(kNoDivZero));
    if (val(m) > 0.5) return T(B(0.5));
    if (val(m) < (double)1e-12f) return T(B((double)1e-12f));
    return m;
}

// d(-pad_max_dt)/dy at y, added to lam with weight w
RTW_HD void torus_pad_vjp(const double* y, double scale, double w, double* lam) {
    typedef Dual<double, 4> D4;
    const D4 m = torus_pad<D4>(D4::var(y[2], 0), D4::var(y[5], 1), D4::var(y[6], 2), D4::var(y[7], 3), scale);
    lam[2] -= w * m.d[0];
    lam[5] -= w * m.d[1];
    lam[6] -= w * m.d[2];
    lam[7] -= w * m.d[3];
}

// n_events word: the count, a flag for rays with a polar escape (re-recorded
// with their state before every event: near the pole the FP64 replay of
// FP32-stage steps would drift by more than the distance to the axis), and a
// flag for rays with more segments than their region of the pool holds
constexpr uint32_t kDenseCheckpoints = 0x80000000u;
constexpr uint32_t kOverflow = 0x40000000u;
constexpr uint32_t kEventCount = 0x3fffffffu;
constexpr int kTorusMaxCk = 16;  // recorded steps per checkpoint

// A recording chunk: one segment of ck_every events: the geodesic state and
// the optical depths before it ([8 + N] doubles; the reverse sweep needs no
// intensities), the step sizes ([ck_every] doubles) and the event kinds
// ([ck_every] bytes). A ray's chunks are contiguous: chunk base + segment.
RTW_HD int torus_chunk_bytes(int N, int kc) { return (8 * (8 + N) + 8 * kc + kc + 7) & ~7; }

struct TorusKP {
    TorusModel m;
    FrameDesc frame;
    long long total_rays;          // rays of this launch: pixels ray0 + k ray_stride, k < total_rays
    long long ray0, ray_stride;
    double max_dt_scale, promote_dr, promote_theta;
    unsigned long long* counter;
    DevStats* stats;
    float* spectrum;  // [P][N]
    float* xyz;       // [P][3]
    double* final_state;  // [P][8] (may be null)
    const float* sky[2];  // the wormhole's skyboxes (cross-layout cube maps) or null
    int sky_h[2];         // pixels per face edge
    int bundles;          // 1: Gaussian ray-bundle lookup of the skyboxes
    double bundle_m[9];   // row-major R2 L R of the camera, spatial blocks (initialization.jl:273-275)
    uint8_t* cls;
    uint32_t* steps;
    const uint32_t* ray_list;          // [total_rays] indices into the subset (dense re-record) or null
    // recording
    int record;                        // 0: none, 1: dense (offsets from counts), 2: chunks
    uint32_t* n_events;                // [P] (chunk pass writes, dense pass checks)
    const unsigned long long* ev_off;  // [P] first event of a ray
    const unsigned long long* ck_off;  // [P] first checkpoint of a ray
    double* ev_h;                      // [E] step size (DP step) or escape sub-step size
    uint8_t* ev_kind;                  // [E] 0: DP step with a controller step size, 0x41 / 0x42: DP
                                       // step of -pad_max_dt of the previous / its own start state,
                                       // 1 + n: polar escape of n sub-steps
    double* ck;                        // [C][8 + 2N] states
    int ck_every;
    int fsal;                          // 1: FSAL Dormand-Prince, 0: the reference's step
    unsigned int* err_flag;            // bit 0: record pass diverged from the count pass
    // chunked recording (record 2). Chunk index i lives in pool at i < split,
    // in pool2 at i - split above. A ray's chunks start at sub * region (first
    // pass, at most region of them: more sets kOverflow), or at chunk_base[loc]
    // (region 0: the pass over the overflowed rays, sized exactly). No atomics:
    // a shared allocation counter cost this kernel a third of its speed.
    char* pool;
    char* pool2;
    unsigned long long split;
    int chunk_bytes;
    unsigned int region;
    unsigned long long region_bytes;       // a ray's region in pool: an odd number of 128-byte lines
    const unsigned long long* chunk_base;  // [total_rays] (region 0)
    double* fin;                           // [P][D] final states
};

template <class R>
struct TorusStages {
    double ns[8];        // 5th-order slope of the geodesic components
    double es[8];        // error slope sum_j E_j K_j
    R k7[8];             // slope at the new state (carried, FSAL)
    TorusPt<R> S[7];     // emitter numbers of stage points 1..6 (index 0 unused)
};

// The seven geodesic stages of one attempt in arithmetic R from the FP64
// state x and the carried slope k1.
template <class R, class K, int EM>
__device__ void torus_geo_stages(const TorusModel& m, const double* x, const K* k1, double h, TorusStages<R>& o) {
    constexpr bool FLAT = EM == 2 || EM == 4;
    R Kg[7][8];
    for (int i = 0; i < 8; ++i) Kg[0][i] = R(k1[i]);
    const R hr = R(h);
    const R d0 = R(x[1] - m.geo.r_ev);
#pragma unroll 1
    for (int s = 1; s < 7; ++s) {
        R acc[8];
        for (int i = 0; i < 8; ++i) acc[i] = R(0);
        for (int j = 0; j < s; ++j) {
            const R w = R(tA(s, j));
            for (int i = 0; i < 8; ++i) acc[i] += w * Kg[j][i];
        }
        R z[10], kk[9];
        for (int i = 0; i < 8; ++i) z[i] = R(x[i]) + hr * acc[i];
        z[8] = R(0);
        z[9] = d0 + hr * acc[1];
        if constexpr (FLAT) {
            for (int i = 0; i < 4; ++i) {
                kk[i] = z[4 + i];
                kk[4 + i] = R(0);
            }
        } else if constexpr (EM == 3) {
            wormhole_rhs<R>(m.wh, z, kk);
        } else {
            Emit<R> em;
            KerrScene<false>::rhs<R>(m.geo, z, kk, em);
        }
        for (int i = 0; i < 8; ++i) Kg[s][i] = kk[i];
        o.S[s] = em_point<R, EM>(m, z);
        if (s == 6)
            for (int i = 0; i < 8; ++i) o.ns[i] = (double)acc[i];
    }
    for (int i = 0; i < 8; ++i) {
        R e = R(0);
        for (int j = 0; j < 7; ++j) e += R(tE(j)) * Kg[j][i];
        o.es[i] = (double)e;
        o.k7[i] = Kg[6][i];
    }
}

// promoted (FP64-stage) geodesic part of the mixed path, out of line
template <class K, int EM>
__device__ __noinline__ void torus_geo_stages_fp64(const TorusModel& m, const double* x, const K* k1, double h,
                                                   TorusStages<double>* o) {
    torus_geo_stages<double, K, EM>(m, x, k1, h, *o);
}

// The ray bundle of pixel (pi, pj) of the frame's window (initialization.jl:
// 198-204, 241-249, 262-325): its size |beamscale cos theta| (beamscale =
// atan(rho_hor) / 2) and the rates (du, dv, dg, dh) = (a.J (1 + E), b.J (1 +
// E), a.J (1 - E), b.J (1 - E)) / 2 of its shape, with E = 1 / (|n_z| +
// no_div_zero), J = n x (0, 0, -1) (or (0, -1, 0) when that is short) and n
// the ray's direction on the canvas, both taken through R2 L R (spatial blocks)
// and normalised, and (a, b) the basis normal to n of the reference (each
// divided by its squared length). The reference gives the 11 bundle components
// zero slope (integrators_LttM.jl:43-46) and leaves them out of the step's
// error norm (:180-185), so they reach the skybox as the camera set them: the
// bundle is a function of the pixel. Out: d[0..3] = du, dv, dg, dh; d[4] = size.
__device__ void bundle_shape(const TorusKP& p, int pi, int pj, double* d) {
    const FrameDesc& f = p.frame;
    const double w = f.rh * ((f.i0 + pi + 1) - 0.5) - f.W;
    const double hh = f.rv * ((f.j0 + pj + 1) - 0.5) - f.H;
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
    double n[3] = {-st * cp, -st * sp, -ct};
    d[4] = fabs(atan(f.rh) / 2 * n[2]);
    const double E = 1.0 / (fabs(n[2]) + 1e-24);
    double J[3] = {-n[1], n[0], 0.0};
    if (J[0] * J[0] + J[1] * J[1] + J[2] * J[2] < 1e-3) {
        J[0] = 0;
        J[1] = -1;
        J[2] = 0;
    }
    double Jr[3], nr[3];
    for (int r = 0; r < 3; ++r) {
        Jr[r] = p.bundle_m[3 * r] * J[0] + p.bundle_m[3 * r + 1] * J[1] + p.bundle_m[3 * r + 2] * J[2];
        nr[r] = p.bundle_m[3 * r] * n[0] + p.bundle_m[3 * r + 1] * n[1] + p.bundle_m[3 * r + 2] * n[2];
    }
    const double jn = sqrt(Jr[0] * Jr[0] + Jr[1] * Jr[1] + Jr[2] * Jr[2]);
    const double nn = sqrt(nr[0] * nr[0] + nr[1] * nr[1] + nr[2] * nr[2]);
    for (int r = 0; r < 3; ++r) {
        Jr[r] /= jn;
        nr[r] /= nn;
    }
    double A[3], B[3];
    if (!(fabs(1 - nr[0]) < 1e-3)) {
        const double q = 1 - nr[0];
        A[0] = nr[1]; A[1] = 1 - nr[1] * nr[1] / q; A[2] = -nr[1] * nr[2] / q;
        B[0] = nr[2]; B[1] = -nr[1] * nr[2] / q; B[2] = 1 - nr[2] * nr[2] / q;
        const double aa = A[0] * A[0] + A[1] * A[1] + A[2] * A[2], bb = B[0] * B[0] + B[1] * B[1] + B[2] * B[2];
        for (int r = 0; r < 3; ++r) {
            A[r] /= aa;
            B[r] /= bb;
        }
    } else {
        A[0] = 0; A[1] = -1; A[2] = 0;
        B[0] = 0; B[1] = 0; B[2] = -1;
    }
    const double aJ = A[0] * Jr[0] + A[1] * Jr[1] + A[2] * Jr[2];
    const double bJ = B[0] * Jr[0] + B[1] * Jr[1] + B[2] * Jr[2];
    d[0] = aJ * (1 + E) / 2;
    d[1] = bJ * (1 + E) / 2;
    d[2] = aJ * (1 - E) / 2;
    d[3] = bJ * (1 - E) / 2;
}

// skybox_handling! (Wormhole.source/source_model.jl:393-443) at a ray's end
// x: beyond r(l) = 50 the ray looks up the skybox on its side of the throat
// in the direction it points (calc_skybox_coord :175-263 with R_sph_to_cart,
// gen_geometry.jl:110-122) and adds, per bin, the spectrum of the texel
// colours (skybox_I_nu_calc :150-172: three Gaussian lines for R, G, B) x
// exp(-tau) / f^3 at f = nu_c k^t. Without ray bundles the colours are those
// of the texel hit (cubemap_coord_calc); with them (calc_skybox_I_nu_beam!
// :266-358) a Gaussian footprint weighs the texels within h <= 10 of it
// across face edges: the pixel's bundle, scaled by k^t, as major/minor axes
// and orientation (distort_gauss, my_special_functions.jl:40-52, by the
// inverse texel size atan(2 / (h_sky + 1)) / 2 on both axes), D2_Gauss
// (:28-34) as the weight of texel offset (k, l). The spectrum is linear in
// the colours, so the weighted colours are summed first and the bins take one
// spectrum: the reference's sum, reassociated. Texels whose wrapped
// coordinates fall off the map (maps under 10 texels a face: the reference
// stops with an index error there) are skipped.
// The Cartesian sphere (EM 4; Minkowski_Sphere_Cartesian.source/
// source_model.jl:175-431) runs the same lookup at every ray's end, in skybox
// 1, with the direction (k^x, k^y, k^z) as it is.
template <int EM>
__device__ void wormhole_skybox(const TorusKP& p, const double* x, int N, double* I, const double* tau, int pi,
                                int pj) {
    int k = 0;
    double vx, vy, vz;
    if constexpr (EM == 4) {
        vx = x[5];
        vy = x[6];
        vz = x[7];
    } else {
        const WormholeDev& W = p.m.wh;
        const double rl = wormhole_r<double>(W, x[1]);
        if (!(rl > 50) || x[1] == 0) return;
        k = x[1] > 0 ? 0 : 1;
        double st, ct, sp, cp;
        sincos(x[2], &st, &ct);
        sincos(x[3], &sp, &cp);
        const double e1 = x[5], e2 = rl * x[6], e3 = rl * st * x[7];
        vx = st * cp * e1 + ct * cp * e2 - sp * e3;
        vy = st * sp * e1 + ct * sp * e2 + cp * e3;
        vz = ct * e1 - st * e2;
    }
    if (!p.sky[k]) return;
    const int H = p.sky_h[k];
    const double nv = sqrt(vx * vx + vy * vy + vz * vz);
    const double X = vx / nv, Y = vy / nv, Z = vz / nv;
    const double ax = fabs(X), ay = fabs(Y), az = fabs(Z);
    int face;
    if (ax >= ay && ax >= az) face = X > 0 ? 1 : 3;
    else if (ay >= ax && ay >= az) face = Y > 0 ? 4 : 2;
    else face = Z > 0 ? 6 : 5;
    double u, v;
    switch (face) {
    case 1: u = -Y / ax; v = Z / ax; break;
    case 2: u = -X / ay; v = Z / ay; break;
    case 3: u = Y / ax; v = Z / ax; break;
    case 4: u = X / ay; v = Z / ay; break;
    case 5: u = -X / az; v = -Y / az; break;
    default: u = -X / az; v = Y / az; break;
    }
    int i = (int)min((double)H, floor(H * (u + 1) / 2) + 1), j = (int)min((double)H, floor(H * (v + 1) / 2) + 1);
    if (i < 1) i = 1;  // (u, v) in [-1, 1]: rounding only
    if (j < 1) j = 1;
    const float* map = p.sky[k];
    const long long H4 = 4LL * H;
    double cr, cg, cb;  // weighted texel colours
    if (!p.bundles) {
        sky_cross(face, H, i, j);
        const float* t = map + ((3LL * H - j) * H4 + (i - 1)) * 3;
        cr = (double)t[0];
        cg = (double)t[1];
        cb = (double)t[2];
    } else {
        double d[5];
        bundle_shape(p, pi, pj, d);
        const double dp = d[4] * x[4];
        const double ra = sqrt(d[0] * d[0] + d[1] * d[1]), rb = sqrt(d[2] * d[2] + d[3] * d[3]);
        const double dmaj = dp * (ra + rb), dmin = dp * (ra - rb);
        const double mu = atan2(d[0] * d[3] + d[1] * d[2], d[0] * d[2] - d[1] * d[3]) / 2;
        const double sc = 1.0 / (atan(2.0 / (H + 1)) / 2 + 1e-24);
        double sm, cm;
        sincos(mu, &sm, &cm);
        const double sxx = sc * sc * (dmaj * dmaj * cm * cm + dmin * dmin * sm * sm);
        const double syy = sc * sc * (dmaj * dmaj * sm * sm + dmin * dmin * cm * cm);
        const double sxy = sc * sc * (dmaj * dmaj - dmin * dmin) * sin(2 * mu) / 2;
        const double root = sqrt((sxx - syy) * (sxx - syy) + 4 * sxy * sxy);
        const double sx = sqrt((sxx + syy + root) / 2), sy = sqrt((sxx + syy - root) / 2);
        const double tn = atan2(2 * sxy, sxx - syy) / 2;
        // a footprint the reference cannot form (a NaN width, where it stops
        // with an error) adds nothing
        if (!(sx > 0 && sy > 0 && isfinite(sx) && isfinite(sy))) return;
        const int hw = (int)min(10.0, ceil(fmax(sx, sy)));
        double stn, ctn;
        sincos(tn, &stn, &ctn);
        const double ga = ctn * ctn / (2 * sx * sx) + stn * stn / (2 * sy * sy);
        const double gb = -stn * ctn / (2 * sx * sx) + stn * ctn / (2 * sy * sy);
        const double gc = stn * stn / (2 * sx * sx) + ctn * ctn / (2 * sy * sy);
        const double gn = 1.0 / (2 * kPi * sx * sy);
        cr = cg = cb = 0;
        for (int kk = -hw; kk <= hw; ++kk)
            for (int ll = -hw; ll <= hw; ++ll) {
                int i2 = i, j2 = j, F2 = face;
                sky_wrap(i2, j2, F2, kk, ll, H);
                sky_cross(F2, H, i2, j2);
                if (i2 < 1 || i2 > 4 * H || j2 < 1 || j2 > 3 * H) continue;
                const double wgt = gn * exp(-(ga * kk * kk + 2 * gb * kk * ll + gc * ll * ll));
                const float* t = map + ((3LL * H - j2) * H4 + (i2 - 1)) * 3;
                cr += wgt * (double)t[0];
                cg += wgt * (double)t[1];
                cb += wgt * (double)t[2];
            }
    }
    const double R = 1.0 * cr, G = 0.843 * cg, B = 0.914 * cb;
    const double inv = 1.0 / sqrt(2 * kPi);
    for (int c = 0; c < N; ++c) {
        const double f = p.m.bins[c].nu_nm * x[4];
        const double d1 = f - 0.001587, d2 = f - 0.001879, d3 = f - 0.002141;
        const double s = 1e-12 * inv *
                         (R * exp(-d1 * d1 / (2 * 5e-5 * 5e-5)) / 5e-5 + G * exp(-d2 * d2 / (2 * 7e-5 * 7e-5)) / 7e-5 +
                          B * exp(-d3 * d3 / (2 * 9e-5 * 9e-5)) / 9e-5);
        I[c] += s * exp(-tau[c]) / (f * f * f);
    }
}

// pad_max_dt of the wormhole (Wormhole.source/source_model.jl:88-110): the
// Kerr form with |k^l| for |k^r|, a tenfold smaller epsilon within 100 a of
// the throat, and the reference's Float32 literals
RTW_HD double wormhole_max_dt(const WormholeDev& W, const double* x, double scale) {
    const double th = x[2];
    double eps = (th < kPi / 8 || th > 7 * kPi / 8) ? fmin(scale, (double)1e-1f) : scale;
    if (fabs(x[1]) < 100 * W.a_wh) eps = eps / 10;
    const double a = fabs(1.0 / (eps / (fabs(x[5]) + kNoDivZero)) + kNoDivZero);
    const double b = fabs(1.0 / (eps * fmin(th, kPi - th) / (fabs(x[6]) + kNoDivZero) + kNoDivZero));
    const double c = fabs(1.0 / (eps / (fabs(x[7]) + kNoDivZero) + kNoDivZero));
    double m = fmin(1.0 / (a + b + c + kNoDivZero), 0.5);
    return fmax(m, (double)1e-12f);
}

// pad_max_dt of the geometry: Kerr (source_model.jl:86-103), Synchro_Test's
// max_dt_scale (1 + |x| + |y|) (source_model.jl:241-244), the Cartesian
// sphere's max_dt_scale (1 + |x| + |y| + |z|) (source_model.jl:130-132) or the
// wormhole's
template <int EM, class SR>
__device__ __forceinline__ double torus_max_dt(const TorusKP& p, const double* x) {
    if constexpr (EM == 2)
        return p.max_dt_scale * (1 + fabs(x[1]) + fabs(x[2]));
    else if constexpr (EM == 4)
        return p.max_dt_scale * (1 + fabs(x[1]) + fabs(x[2]) + fabs(x[3]));
    else if constexpr (EM == 3)
        return wormhole_max_dt(p.m.wh, x, p.max_dt_scale);
    else
        return pad_max_dt<RTW_SCENE_KERR_DISK, SR>(p.m.geo, x, p.max_dt_scale);
}

// near_singularity of the geometry: Kerr (source_geometry.jl:249-269), none
// in flat Cartesian space, the wormhole's within 5 tol of a pole
// (Wormhole.source/source_geometry.jl:156-171)
template <int EM>
__device__ __forceinline__ bool torus_near_singularity(const double* x, double h, double tol, double* temp) {
    if constexpr (EM == 2 || EM == 4) {
        return false;
    } else if constexpr (EM == 3) {
        const double th_new = x[2] + h * x[6];
        if (fabs(th_new) <= 5 * tol) {
            *temp = 2 * fabs(x[2]) / (fabs(x[6] * 37) + kNoDivZero);
            return true;
        }
        if (fabs(th_new - kPi) <= 5 * tol) {
            *temp = 2 * fabs((x[2] - kPi) / (fabs(x[6] * 37) + kNoDivZero));
            return true;
        }
        *temp = h;
        return false;
    } else {
        return near_singularity<RTW_SCENE_KERR_DISK>(x, h, tol, temp);
    }
}

// calc_terminate without the step-count predicate; THICK when every bin's
// tau has reached -log(tol). With ray bundles the reference's test also sees
// the bundle slots, which are 0 or small and keep it from firing: no THICK.
template <class SR, int EM>
__device__ __forceinline__ int torus_terminate(const TorusKP& p, const double* x, const SR* tau, int N) {
    if constexpr (EM == 2 || EM == 4) {
        // Synchro_Test.source/source_model.jl:258-275, the sphere's :158-172
        if (sqrt(x[1] * x[1] + x[2] * x[2] + x[3] * x[3]) > p.m.geo.esc) return RTW_CLASS_ESCAPE;
    } else if constexpr (EM == 3) {
        // Wormhole.source/source_model.jl:134-147: r(l) beyond the escape radius, phi winding
        if (wormhole_r<double>(p.m.wh, x[1]) > p.m.geo.esc) return RTW_CLASS_ESCAPE;
        if (x[3] > p.m.geo.wind) return RTW_CLASS_WINDING;
    } else {
        if (x[1] > p.m.geo.esc) return RTW_CLASS_ESCAPE;
        if (x[1] <= p.frame.r_term) return RTW_CLASS_HORIZON;
        if (x[3] > p.m.geo.wind) return RTW_CLASS_WINDING;
    }
    if constexpr (EM >= 3)
        if (p.bundles) return 0;
    for (int c = 0; c < N; ++c)
        if ((double)tau[c] < p.frame.thick) return 0;
    return RTW_CLASS_THICK;
}

// Recording of one ray (record 1: dense offsets, 2: chunks). One kernel
// instance serves renders and recording passes, so that both take
// bit-identical steps; the per-segment work is out of line and the per-event
// work is two stores into a buffer, so that a render does not pay for it.
struct TorusRec {
    unsigned long long eo, co;  // dense: first event and checkpoint
    uint32_t ev_cap, kc;        // dense: event count from the first pass; segment length
    unsigned long long base;    // chunks: the ray's first chunk
    uint32_t seg;               // chunks: segments opened so far
    uint32_t ovf;               // chunks: more segments than the region holds
    uint32_t bad;               // dense: more events than the first pass
    double hb[kTorusMaxCk];     // chunks: the current segment's events, written out whole
    uint8_t kb[kTorusMaxCk];
};

// Chunk i: in pool (i < split), ray i / region's region, segment i % region;
// the regions are an odd number of 128-byte lines apart, so that the lanes'
// concurrent chunks do not alias onto the same memory channels (a stride
// that was a multiple of 4 KB cost the reverse sweep about 10 %).
RTW_HD char* torus_chunk(const TorusKP& p, unsigned long long i) {
    if (i < p.split) {
        const unsigned long long ray = i / p.region, seg = i - ray * p.region;
        return p.pool + ray * p.region_bytes + seg * (unsigned long long)p.chunk_bytes;
    }
    return p.pool2 + (i - p.split) * (unsigned long long)p.chunk_bytes;
}

// write the first m buffered events of the current segment (streaming
// stores: this kernel does not read them again)
__device__ void torus_rec_flush(const TorusKP& p, const TorusRec* r, uint32_t m) {
    if (r->ovf || r->seg == 0 || m == 0) return;
    const int N = p.m.n;
    char* chunk = torus_chunk(p, r->base + r->seg - 1);
    double* h = (double*)(chunk + 8 * (8 + N));
    uint8_t* k = (uint8_t*)(chunk + 8 * (8 + N) + 8 * r->kc);
    for (uint32_t j = 0; j < m; ++j) {
        __stcs(h + j, r->hb[j]);
        k[j] = r->kb[j];
    }
}

__device__ __noinline__ void torus_rec_begin(const TorusKP& p, long long loc, long long sub, TorusRec* r) {
    r->seg = r->ovf = r->bad = 0;
    r->kc = (uint32_t)p.ck_every;
    r->ev_cap = 0;
    r->eo = r->co = 0;
    r->base = 0;
    if (p.record == 1) {
        const uint32_t w = p.n_events[loc];
        r->ev_cap = w & kEventCount;
        r->kc = (w & kDenseCheckpoints) ? 1u : (uint32_t)p.ck_every;
        r->eo = p.ev_off[loc];
        r->co = p.ck_off[loc];
    } else if (p.record == 2) {
        r->base = p.region ? (unsigned long long)sub * p.region : p.chunk_base[loc];
    }
}

template <class SR, bool MIXED>
__device__ void torus_save_state(int N, double* c, const double* x, const SR* tau, const SR* ihi, const SR* ilo,
                                 bool with_i) {
    for (int i = 0; i < 8; ++i) __stcs(c + i, x[i]);
    for (int q = 0; q < N; ++q) __stcs(c + 8 + q, (double)tau[q]);
    if (with_i)
        for (int q = 0; q < N; ++q) __stcs(c + 8 + N + q, (double)ihi[q] + (MIXED ? (double)ilo[q] : 0.0));
}

// the state before event n (n a multiple of kc): a checkpoint row (dense) or
// the ray's next chunk
template <class SR, bool MIXED>
__device__ __noinline__ void torus_rec_checkpoint(const TorusKP& p, TorusRec* r, uint32_t n, const double* x,
                                                  const SR* tau, const SR* ihi, const SR* ilo) {
    const int N = p.m.n, D = 8 + 2 * N;
    if (p.record == 1) {
        if (n < r->ev_cap)
            torus_save_state<SR, MIXED>(N, p.ck + (r->co + n / r->kc) * (unsigned long long)D, x, tau, ihi, ilo, true);
        return;
    }
    if (r->ovf) return;
    if (n > 0) torus_rec_flush(p, r, r->kc);  // the previous segment is complete
    if (p.region && r->seg >= p.region) {
        r->ovf = 1;
        return;
    }
    torus_save_state<SR, MIXED>(N, (double*)torus_chunk(p, r->base + r->seg), x, tau, ihi, ilo, false);
    ++r->seg;
}

// the end of a ray: the last segment's events and the final state (chunks),
// counts and flags
template <class SR, bool MIXED>
__device__ __noinline__ void torus_rec_end(const TorusKP& p, TorusRec* r, long long loc, long long sub, uint32_t n,
                                           bool escaped, const double* x, const SR* tau, const SR* ihi, const SR* ilo) {
    const int N = p.m.n, D = 8 + 2 * N;
    if (p.record == 2) {
        if (n > 0) torus_rec_flush(p, r, n - (n - 1) / r->kc * r->kc);
        torus_save_state<SR, MIXED>(N, p.fin + sub * (long long)D, x, tau, ihi, ilo, true);
        p.n_events[sub] = n | (escaped ? kDenseCheckpoints : 0u) | (r->ovf ? kOverflow : 0u);
    }
    if (p.record == 1 && (r->bad || n != r->ev_cap)) atomicOr(p.err_flag, 1u);
}

// Forward kernel. SR: arithmetic of the bins and of the stages (float on the
// mixed path, with Kahan intensities and per-ray FP64 stages near the horizon
// and the poles; double on the FP64 path).
// (FP32-mixed: 3 CTAs/SM, 168 registers, measured 7-13 % faster than 2 CTAs at
// 255; FP64 stays at 2, where 3 was 8-20 % slower)
// The FP64 right-hand side at the forward kernel's rare sites (a ray's start,
// polar escapes, pole reflections), kept out of line so that its per-bin loop
// stays out of the hot loop's code.
template <int KEM>
__device__ __noinline__ void torus_f64_cold(const TorusModel& m, const double* y, double* f) {
    torus_f64<KEM>(m, y, f);
}

// CTAs per SM the FP32-mixed per-bin forward is compiled for, per emitter
// (measured at 512^2 / 1024 x 645): the thermal tori (synchrotron, brems) at 4
// (128 registers: 478 against 500 ms, 0.501 against 0.489 Mrays/s), the others
// at 3 (168 registers: Powehi 4.56 against 4.32, the wormhole 3.48 against
// 3.11 Mrays/s at 4)
#ifndef RTW_FWD_MIN_CTAS
#define RTW_FWD_MIN_CTAS 4
#endif
template <bool MIXED, int EM>
__global__ void __launch_bounds__(128, MIXED ? ((EM == 0 || EM == 5) ? RTW_FWD_MIN_CTAS : 3) : 2)
    torus_forward(__grid_constant__ const TorusKP p) {
    constexpr bool FLAT = EM == 2 || EM == 4;  // Synchro_Test, the sphere: flat Cartesian geometry
    // the FP64 slope at a ray's start and after escapes: the instance's own
    // emitter on the mixed path (ptxas: the torus, Powehi and wormhole
    // instances then spill 32-124 B per thread instead of 318-326 with the
    // run-time dispatch), the run-time dispatch on the FP64 path (where the
    // instance's own emitter raised Synchro_Test's spills from 132 B to 496 B)
    constexpr int KEM = MIXED ? EM : -1;
    typedef typename SpecTraits<MIXED>::SR SR;
    const int N = p.m.n;
    const int D = 8 + 2 * N;
    unsigned c_att = 0, c_rej = 0, c_pro = 0, c_esc = 0, c_rays = 0, c_nan = 0;
    for (;;) {
        const long long loc = (long long)atomicAdd(p.counter, 1ull);  // index in the ray subset (list)
        if (loc >= p.total_rays) break;
        const long long sub = p.ray_list ? (long long)p.ray_list[loc] : loc;
        const long long id = p.ray0 + sub * p.ray_stride;              // pixel
        ++c_rays;
        const int pi = (int)(id % p.frame.xp), pj = (int)(id / p.frame.xp);
        double x[9];
        camera_ray(p.frame, pi, pj, x);
        SR tau[kTorusMaxBins], ihi[kTorusMaxBins], ilo[kTorusMaxBins], kt1[kTorusMaxBins], ki1[kTorusMaxBins];
        SR k1[8];
        {
            double y[8 + 2 * kTorusMaxBins], f[8 + 2 * kTorusMaxBins];
            for (int i = 0; i < 8; ++i) y[i] = x[i];
            for (int i = 8; i < D; ++i) y[i] = 0;
            torus_f64_cold<KEM>(p.m, y, f);
            for (int i = 0; i < 8; ++i) k1[i] = SR(f[i]);
            for (int c = 0; c < N; ++c) {
                tau[c] = 0; ihi[c] = 0; ilo[c] = 0;
                kt1[c] = SR(f[8 + c]);
                ki1[c] = SR(f[8 + N + c]);
            }
        }
        // some carried bin slope is nonzero: with no emitting stage point and
        // every carried slope zero, an attempt leaves every bin exactly as it
        // is (all its tau / I slopes are 0), so the bins' loop is skipped
        auto slopes_live = [&]() {
            bool nz = false;
            for (int c = 0; c < N; ++c) nz |= kt1[c] != SR(0) || ki1[c] != SR(0);
            return nz;
        };
        bool live = slopes_live();
        double h = -torus_max_dt<EM, SR>(p, x);
        // where h came from: 0 the controller (held fixed by the adjoint),
        // 1 -pad_max_dt of the previous accepted step's start state, 2 -pad_max_dt
        // of the current state
        uint8_t hsrc = 2;
        const double tol = p.frame.tol;
        bool prev_rej = false;
        long long nsteps = 0;
        uint32_t n_ev = 0;
        bool escaped = false;  // a ray with a polar escape stores its state at every step
        TorusRec rec;
        if (p.record) torus_rec_begin(p, loc, sub, &rec);
        // the state before event n_ev when it starts a segment (recording)
        auto checkpoint = [&]() {
            if (p.record && (n_ev % rec.kc) == 0u) torus_rec_checkpoint<SR, MIXED>(p, &rec, n_ev, x, tau, ihi, ilo);
        };
        // event n_ev: its step size (or escape sub-step size) and kind
        auto push = [&](uint8_t kind, double hv) {
            if (p.record == 1) {
                if (n_ev >= rec.ev_cap) {
                    rec.bad = 1;
                } else {
                    p.ev_h[rec.eo + n_ev] = hv;
                    p.ev_kind[rec.eo + n_ev] = kind;
                }
            } else if (p.record == 2) {
                const uint32_t j = n_ev % rec.kc;
                rec.hb[j] = hv;
                rec.kb[j] = kind;
            }
            ++n_ev;
        };
        int cls = 0;
        for (;;) {
            ++c_att;
            const double max_dt = torus_max_dt<EM, SR>(p, x);
            double temp;
            bool done = false;
            if (torus_near_singularity<EM>(x, h, tol, &temp)) {
                // polar escape (integrators_LttM.jl:62-105) in FP64 on the full state
                checkpoint();
                double y[8 + 2 * kTorusMaxBins], f[8 + 2 * kTorusMaxBins];
                for (int i = 0; i < 8; ++i) {
                    y[i] = x[i];
                    f[i] = (double)k1[i];
                }
                for (int q = 0; q < N; ++q) {
                    y[8 + q] = (double)tau[q];
                    y[8 + N + q] = (double)ihi[q] + (MIXED ? (double)ilo[q] : 0.0);
                    f[8 + q] = (double)kt1[q];
                    f[8 + N + q] = (double)ki1[q];
                }
                int nsub = 0;
                for (int it = 0; it < 37; ++it) {
                    if (it > 0) {
                        if (torus_terminate<double, EM>(p, y, y + 8, N)) continue;
                        torus_f64_cold<KEM>(p.m, y, f);
                    }
                    for (int i = 0; i < D; ++i) y[i] -= temp * f[i];
                    torus_keep(y);
                    ++nsub;
                }
                c_esc += nsub;
                escaped = true;
                push((uint8_t)(1 + nsub), temp);
                for (int i = 0; i < 8; ++i) x[i] = y[i];
                for (int q = 0; q < N; ++q) {
                    tau[q] = SR(y[8 + q]);
                    ihi[q] = SR(y[8 + N + q]);
                    ilo[q] = MIXED ? SR(y[8 + N + q] - (double)ihi[q]) : SR(0);
                }
                if (torus_terminate<double, EM>(p, y, y + 8, N)) {
                    done = true;
                    prev_rej = false;
                } else {
                    torus_f64_cold<KEM>(p.m, y, f);
                    for (int i = 0; i < 8; ++i) k1[i] = SR(f[i]);
                    for (int q = 0; q < N; ++q) {
                        kt1[q] = SR(f[8 + q]);
                        ki1[q] = SR(f[8 + N + q]);
                    }
                    live = slopes_live();
                    h = -torus_max_dt<EM, SR>(p, x);
                    hsrc = 2;
                }
            }
            if (!done) {
                // geodesic stages
                TorusStages<SR> st;
                bool promote = false;
                if (MIXED && EM == 3)  // the wormhole: the poles only (no horizon)
                    promote = (x[2] < p.promote_theta) || (x[2] > kPi - p.promote_theta);
                else if (MIXED && !FLAT)
                    promote = (x[1] - p.m.geo.r_ev < p.promote_dr) || (x[2] < p.promote_theta) ||
                              (x[2] > kPi - p.promote_theta);
                if (promote) {
                    ++c_pro;
                    TorusStages<double> sd;
                    torus_geo_stages_fp64<SR, EM>(p.m, x, k1, h, &sd);
                    for (int i = 0; i < 8; ++i) {
                        st.ns[i] = sd.ns[i];
                        st.es[i] = sd.es[i];
                        st.k7[i] = SR(sd.k7[i]);
                    }
                    for (int s = 1; s < 7; ++s) {
                        st.S[s].cj = SR(sd.S[s].cj);
                        st.S[s].nus = SR(sd.S[s].nus);
                        st.S[s].th = SR(sd.S[s].th);
                        st.S[s].g = SR(sd.S[s].g);
                        st.S[s].on = sd.S[s].on;
                        st.S[s].zone = sd.S[s].zone;
                    }
                } else {
                    torus_geo_stages<SR, SR, EM>(p.m, x, k1, h, st);
                }
                if constexpr (MIXED && EM == 0)
                    for (int s = 1; s < 7; ++s)
                        if (st.S[s].on) torus_bin_stage<SR>(st.S[s]);
                double y[8];
                double err2 = 0;
                for (int i = 0; i < 8; ++i) {
                    y[i] = x[i] + h * st.ns[i];
                    const double d = h * st.es[i];
                    const double tl = tol + fmax(fabs(x[i]), fabs(y[i])) * tol;
                    err2 += (d / tl) * (d / tl);
                }
                // bins: seven tau / I stages each
                SR c_t[kTorusMaxBins], c_h[kTorusMaxBins], c_l[kTorusMaxBins], c_kt[kTorusMaxBins],
                    c_ki[kTorusMaxBins];
                const SR hs = SR(h), ts = SR(tol);
                SR ebins = 0;
                bool run_bins = live, nz = false;
                for (int s = 1; s < 7; ++s) run_bins |= st.S[s].on;
                for (int c = 0; c < (run_bins ? N : 0); ++c) {
                    SR kt[7], ki[7];
                    kt[0] = kt1[c];
                    ki[0] = ki1[c];
                    const SR t0 = tau[c];
                    SR tp = t0;
#pragma unroll
                    for (int s = 1; s < 7; ++s) {
                        SR a = 0;
#pragma unroll
                        for (int j = 0; j < s; ++j) a += SR(tA(s, j)) * kt[j];
                        tp = t0 + hs * a;
                        SR ft = 0, fi = 0;
                        if (st.S[s].on) {
                            if constexpr (MIXED && EM == 0)
                                torus_bin_fast<SR>(st.S[s], p.m.bins[c], ft, fi);
                            else
                                em_bin<SR, EM>(p.m, st.S[s], c, ft, fi);
                        }
                        kt[s] = ft;
                        ki[s] = fi * (MIXED && EM == 0 ? BinMath<SR>::ex(-tp) : texp(-tp));
                    }
                    // tp is now the new tau (row 6 of A is b)
                    SR nsI = 0, nsT = 0, et = 0, ei = 0;
#pragma unroll
                    for (int j = 0; j < 7; ++j) {
                        if (j < 6) {
                            nsI += SR(tA(6, j)) * ki[j];
                            nsT += SR(tA(6, j)) * kt[j];
                        }
                        et += SR(tE(j)) * kt[j];
                        ei += SR(tE(j)) * ki[j];
                    }
                    SR yh = ihi[c], yl = MIXED ? ilo[c] : SR(0);
                    if constexpr (MIXED) {
                        kahan_add(yh, yl, hs * nsI);
                    } else {
                        yh = yh + hs * nsI;
                    }
                    const SR i0 = ihi[c];
                    const SR dt_ = hs * et, di = hs * ei;
                    const SR tlt = ts + rmax(rabs(t0), rabs(tp)) * ts;
                    const SR tli = ts + rmax(rabs(i0), rabs(yh)) * ts;
                    // (FP32-mixed: the hardware reciprocal, 2 ulp, for the error norm)
                    const SR qt = MIXED ? dt_ * rinv(tlt) : dt_ / tlt, qi = MIXED ? di * rinv(tli) : di / tli;
                    ebins += qt * qt + qi * qi;
                    c_t[c] = tp;
                    c_h[c] = yh;
                    c_l[c] = yl;
                    // slopes carried to the next attempt: k7 (FSAL) or the
                    // reference's sum b_i k_i
                    c_kt[c] = p.fsal ? kt[6] : nsT;
                    c_ki[c] = p.fsal ? ki[6] : nsI;
                    nz |= c_kt[c] != SR(0) || c_ki[c] != SR(0);
                }
                err2 += (double)ebins;
                bool accept;
                double hnext;
                decide<double>(err2, D, h, max_dt, prev_rej, accept, hnext);
                const uint8_t next_src = hnext == -max_dt ? (accept ? 1 : 2) : 0;
                if (accept) {
                    checkpoint();
                    push(hsrc ? (uint8_t)(0x40 | hsrc) : (uint8_t)0, h);
                    for (int i = 0; i < 8; ++i) {
                        x[i] = y[i];
                        k1[i] = p.fsal ? st.k7[i] : SR(st.ns[i]);
                    }
                    if (run_bins) {
                        for (int c = 0; c < N; ++c) {
                            tau[c] = c_t[c];
                            ihi[c] = c_h[c];
                            ilo[c] = c_l[c];
                            kt1[c] = c_kt[c];
                            ki1[c] = c_ki[c];
                        }
                        live = nz;
                    }
                    if (!FLAT && torus_keep(x) && p.fsal) {
                        // reflected through the pole: the carried slope belongs to
                        // the unreflected point, so take f at the new state (FSAL;
                        // the reference's step keeps its carried sum)
                        double yy[8 + 2 * kTorusMaxBins], ff[8 + 2 * kTorusMaxBins];
                        for (int i = 0; i < 8; ++i) yy[i] = x[i];
                        for (int q = 0; q < N; ++q) {
                            yy[8 + q] = (double)tau[q];
                            yy[8 + N + q] = (double)ihi[q] + (MIXED ? (double)ilo[q] : 0.0);
                        }
                        torus_f64_cold<KEM>(p.m, yy, ff);
                        for (int i = 0; i < 8; ++i) k1[i] = SR(ff[i]);
                        for (int q = 0; q < N; ++q) {
                            kt1[q] = SR(ff[8 + q]);
                            ki1[q] = SR(ff[8 + N + q]);
                        }
                        live = slopes_live();
                    }
                    prev_rej = false;
                } else {
                    if (!FLAT) torus_keep(x);
                    prev_rej = true;
                    ++c_rej;
                }
                h = hnext;
                hsrc = next_src;
            }
            ++nsteps;
            if (nsteps >= p.frame.max_steps) cls = RTW_CLASS_MAXSTEPS;
            else cls = torus_terminate<SR, EM>(p, x, tau, N);
            if (cls) break;
        }
        bool fin = true;
        for (int i = 0; i < 8; ++i) fin &= isfinite(x[i]);
        if (!fin) {
            cls = RTW_CLASS_NAN;
            ++c_nan;
        }
        if constexpr (EM == 3 || EM == 4) {
            if (fin && (p.sky[0] || p.sky[1])) {
                double I[kTorusMaxBins], tv[kTorusMaxBins];
                for (int c = 0; c < N; ++c) {
                    I[c] = (double)ihi[c] + (MIXED ? (double)ilo[c] : 0.0);
                    tv[c] = (double)tau[c];
                }
                wormhole_skybox<EM>(p, x, N, I, tv, pi, pj);
                for (int c = 0; c < N; ++c) {
                    ihi[c] = SR(I[c]);
                    ilo[c] = MIXED ? SR(I[c] - (double)ihi[c]) : SR(0);
                }
            }
        }
        if (p.spectrum || p.xyz) {
            double X = 0, Y = 0, Z = 0;
            for (int c = 0; c < N; ++c) {
                const double I = (double)ihi[c] + (MIXED ? (double)ilo[c] : 0.0);
                if (p.spectrum) p.spectrum[id * N + c] = (float)I;
                X += I * p.m.bins[c].fx;
                Y += I * p.m.bins[c].fy;
                Z += I * p.m.bins[c].fz;
            }
            if (p.xyz) {
                p.xyz[3 * id + 0] = (float)X;
                p.xyz[3 * id + 1] = (float)Y;
                p.xyz[3 * id + 2] = (float)Z;
            }
        }
        if (p.cls) p.cls[id] = (uint8_t)cls;
        if (p.steps) p.steps[id] = (uint32_t)nsteps;
        if (p.final_state)
            for (int i = 0; i < 8; ++i) p.final_state[8 * id + i] = x[i];
        if (p.record) torus_rec_end<SR, MIXED>(p, &rec, loc, sub, n_ev, escaped, x, tau, ihi, ilo);
    }
    atomicAdd(&p.stats->step_attempts, (unsigned long long)c_att);
    atomicAdd(&p.stats->rejected_steps, (unsigned long long)c_rej);
    atomicAdd(&p.stats->promoted_steps, (unsigned long long)c_pro);
    atomicAdd(&p.stats->escape_substeps, (unsigned long long)c_esc);
    atomicAdd(&p.stats->nan_rays, (unsigned long long)c_nan);
    atomicAdd(&p.stats->rays, (unsigned long long)c_rays);
}

struct TorusRP {
    TorusKP f;
    FrameDesc dframe[2];  // d frame / d a, d frame / d inclination (pos and M; the rest as frame)
    const float* target;
    const float* spectrum;
    double* out;                 // [1 + 5 + 2]: loss, gradient, escapes carried as identity, rays with escapes
    double* per_ray;             // [P][5] per-ray gradients (may be null)
    int skip_escape_rays;        // 1: rays with a polar escape give no gradient
    unsigned long long* counter;
    const uint32_t* esc_index;   // [P] a ray's index among the densely re-recorded rays
    const unsigned long long* rbase;  // [P] a ray's first chunk
    const uint32_t* order;       // [P] the rays by decreasing recorded steps (the queue's order)
};

// One recorded step of a ray, replayed in FP64: y_out = keep(step(y_in)).
RTW_HD bool torus_is_dp(uint8_t kind) { return kind == 0 || (kind & 0x40); }

// The six stage slopes K[s][D] of one recorded FSAL step of size h from y
// (the replay's arithmetic). Y: [D] scratch. Returns y' in y_out unless null.
RTW_HD void torus_dp_stages(const TorusModel& m, const double* y, double h, double* K, double* Y, double* y_out) {
    const int D = 8 + 2 * m.n;
    torus_f64(m, y, K);
    for (int s = 1; s < 6; ++s) {
        for (int i = 0; i < D; ++i) {
            double acc = 0;
            for (int j = 0; j < s; ++j) acc += tA(s, j) * K[j * D + i];
            Y[i] = y[i] + h * acc;
        }
        torus_f64(m, Y, K + s * D);
    }
    if (y_out)
        for (int i = 0; i < D; ++i) {
            double acc = 0;
            for (int j = 0; j < 6; ++j) acc += tA(6, j) * K[j * D + i];
            y_out[i] = y[i] + h * acc;
        }
}

__device__ bool torus_replay(const TorusModel& m, const double* y_in, uint8_t kind, double hv, double* y_out,
                             double* K, double* Y) {
    const int N = m.n, D = 8 + 2 * N;
    if (torus_is_dp(kind)) {
        // K: [6][D] stage slopes, Y: [D] a stage point
        torus_dp_stages(m, y_in, hv, K, Y, y_out);
        return torus_keep(y_out);
    }
    for (int i = 0; i < D; ++i) y_out[i] = y_in[i];
    bool refl = false;
    for (int it = 0; it < (int)kind - 1; ++it) {
        torus_f64(m, y_out, K);
        for (int i = 0; i < D; ++i) y_out[i] -= hv * K[i];
        refl = torus_keep(y_out);
    }
    return refl;  // (the reverse pass replays escapes sub-step by sub-step)
}

// Sub-step size of the polar escape from y (near_singularity, Kerr
// source_geometry.jl:249-269): 2 |theta - pole| / (37 |k^theta|), the pole
// nearer to theta.
RTW_HD double torus_escape_temp(const double* y) {
    const double dth = y[2] < 0.5 * kPi ? y[2] : y[2] - kPi;
    return 2 * fabs(dth) / (fabs(y[6] * 37) + kNoDivZero);
}

// End state of a polar escape of n sub-steps z <- keep(z - temp f(z)) from y.
RTW_HD void torus_escape_end(const TorusModel& m, const double* y, int nsub, double* z, double* K) {
    const int D = 8 + 2 * m.n;
    const double temp = torus_escape_temp(y);
    for (int i = 0; i < D; ++i) z[i] = y[i];
    for (int s = 0; s < nsub; ++s) {
        torus_f64(m, z, K);
        for (int i = 0; i < D; ++i) z[i] -= temp * K[i];
        torus_keep(z);
    }
}

// Vector-Jacobian product of a polar escape of n sub-steps from y with
// sub-step size temp (the recorded value, = torus_escape_temp(y)): lam (the
// cotangent of the end state) becomes that of y and pb gains the parameter
// part. The sub-step size depends on y and is differentiated too. Returns
// false when the escape amplified the geodesic cotangent by more than 1e3
// (sum |lambda_i y_i|): such an escape passed so close to the axis that its
// local derivative is a spike narrower than any parameter change, and it is
// carried as the identity (the state is continuous across the pole) with the
// exact per-bin tau -> I coupling. Scratch: W [4][D], mu, tmp [D].
RTW_HD bool torus_escape_vjp(const TorusModel& m, const double* y, int nsub, double temp, double* lam,
                             double* pb, double* W, double* mu, double* tmp) {
    const int N = m.n, D = 8 + 2 * N;
    double* z = W;             // sub-step state
    double* lin = W + D;       // the cotangent of the end state
    double* zl = W + 2 * D;    // one sub-step ahead
    double pbe[kTorusParams] = {0, 0, 0, 0, 0};
    for (int i = 0; i < D; ++i) lin[i] = lam[i];
    double gtemp = 0;  // d loss / d temp
    for (int s = nsub - 1; s >= 0; --s) {
        // z_s by replay from y (the sub-steps are few and the escapes rare)
        for (int i = 0; i < D; ++i) z[i] = y[i];
        for (int t = 0; t < s; ++t) {
            torus_f64(m, z, tmp);
            for (int i = 0; i < D; ++i) z[i] -= temp * tmp[i];
            torus_keep(z);
        }
        torus_f64(m, z, tmp);
        // sub-step s: z_{s+1} = keep(z_s - temp f(z_s))
        for (int i = 0; i < D; ++i) zl[i] = z[i] - temp * tmp[i];
        if (torus_keep(zl)) {
            lam[2] = -lam[2];
            lam[6] = -lam[6];
        }
        for (int i = 0; i < D; ++i) gtemp -= lam[i] * tmp[i];
        for (int i = 0; i < D; ++i) {
            zl[i] = -temp * lam[i];
            mu[i] = 0;
        }
        torus_vjp(m, z, zl, mu, pbe);
        for (int i = 0; i < D; ++i) lam[i] += mu[i];
    }
    const double dth = y[2] < 0.5 * kPi ? y[2] : y[2] - kPi;
    const double den = fabs(y[6] * 37) + kNoDivZero;
    lam[2] += gtemp * 2 * (dth >= 0 ? 1.0 : -1.0) / den;
    lam[6] += gtemp * (-2 * fabs(dth) * 37 * (y[6] >= 0 ? 1.0 : -1.0) / (den * den));
    double na = 0, nb = 0;
    for (int i = 1; i < 8; ++i) {
        if (i == 3) continue;
        na += fabs(lam[i] * y[i]);
        nb += fabs(lin[i] * y[i]);
    }
    for (int c = 0; c < N; ++c) nb += fabs(lin[8 + N + c] * y[8 + N + c]);
    if (!(na <= 1e3 * nb + 1e-300)) {
        for (int i = 0; i < D; ++i) lam[i] = lin[i];
        torus_escape_end(m, y, nsub, z, tmp);
        for (int c = 0; c < N; ++c) lam[8 + c] -= lin[8 + N + c] * (z[8 + N + c] - y[8 + N + c]);
        return false;
    }
    for (int q = 0; q < kTorusParams; ++q) pb[q] += pbe[q];
    return true;
}

// The geodesic part of one recorded FSAL step alone (bit-identical to the
// geodesic components of torus_dp_stages: the bins never enter them).
// Kg [6][8] the stage slopes; g_out = keep(g + h sum b Kg); returns whether
// keep reflected theta through the pole.
RTW_HD bool torus_geo_step(const TorusModel& m, const double* g, double h, double* Kg, double* g_out) {
    double Y[8];
    for (int t = 0; t < 6; ++t) {
        for (int i = 0; i < 8; ++i) {
            double acc = 0;
            for (int s = 0; s < t; ++s) acc += tA(t, s) * Kg[s * 8 + i];
            Y[i] = g[i] + h * acc;
        }
        torus_geo_rhs(m, Y, Kg + t * 8);
    }
    for (int i = 0; i < 8; ++i) {
        double acc = 0;
        for (int s = 0; s < 6; ++s) acc += tA(6, s) * Kg[s * 8 + i];
        g_out[i] = g[i] + h * acc;
    }
    return torus_keep(g_out);
}

// Reverse of one step y' = y + h sum_s b_s K_s, K_s = f(Y_s), Y_s = y + h
// sum_{j<s} A_sj K_j, written over the whole state with the generic VJP
// (the reference form the structured torus_dp_vjp is checked against).
// lam: the cotangent of y' in, of y out; returns d loss / d h.
// Scratch: Yst, kac [6][D], mu [D].
RTW_HD double torus_dp_vjp_generic(const TorusModel& m, const double* y, const double* K, double h, double* lam,
                                   double* pb, double* Yst, double* kac, double* mu) {
    const int D = 8 + 2 * m.n;
    for (int i = 0; i < D; ++i) Yst[i] = y[i];
    for (int s = 1; s < 6; ++s)
        for (int i = 0; i < D; ++i) {
            double acc = 0;
            for (int j = 0; j < s; ++j) acc += tA(s, j) * K[j * D + i];
            Yst[s * D + i] = y[i] + h * acc;
        }
    double hbar = 0;
    for (int i = 0; i < D; ++i) {
        double bk = 0;
        for (int s = 0; s < 6; ++s) bk += tA(6, s) * K[s * D + i];
        hbar += lam[i] * bk;
    }
    for (int s = 0; s < 6; ++s)
        for (int i = 0; i < D; ++i) kac[s * D + i] = h * tA(6, s) * lam[i];
    for (int t = 5; t >= 0; --t) {
        for (int i = 0; i < D; ++i) mu[i] = 0;
        torus_vjp(m, Yst + t * D, kac + t * D, mu, pb);
        for (int i = 0; i < D; ++i) lam[i] += mu[i];
        for (int i = 0; i < D && t > 0; ++i) {
            double ak = 0;
            for (int s = 0; s < t; ++s) ak += tA(t, s) * K[s * D + i];
            hbar += mu[i] * ak;
        }
        for (int s = 0; s < t; ++s) {
            const double w = h * tA(t, s);
            if (w != 0)
                for (int i = 0; i < D; ++i) kac[s * D + i] += w * mu[i];
        }
    }
    return hbar;
}

// The same reverse step, structured: the bins' (tau, I) cotangents never
// depend on the geodesic ones (d f_geo / d bins = 0 and each bin's block
// couples only to itself), so (1) the emitter numbers of the six stage points
// and their tangents are formed once, (2) each bin re-forms its twelve stage
// slopes from them (the closed-form partials return the values too) and runs
// its six-stage recursion in registers, adding to the cotangents of the
// emitter numbers, (3) the eight geodesic components run theirs. Only the
// step's geodesic start state yg [8], its geodesic stage slopes Kg [6][8] and
// the bins' optical depths tau [N] are read: same result as
// torus_dp_vjp_generic at a fraction of its memory traffic. The tau slopes
// depend on the geodesic alone (tau' = ft(emitter numbers)), so with
// tau_at_end the step is run backwards for tau: tau holds the depths at the
// end of the step on entry and those at its start on return (the intensities
// enter no slope, so the reverse sweep never needs them). BT: arithmetic of
// the bins' partials (double, or float for the FP32-mixed adjoint); the
// cotangents accumulate in FP64 either way.
// mu += (d accel / d(r, theta, k))^T cw and pb[0] += (d accel / d a)^T cw at
// the stage point Yt, by the acceleration's reverse mode (kerr_accel_vjp) in T
template <class T>
RTW_HD void torus_accel_vjp(const TorusModel& m, const double* Yt, const double* cw4, double* mu, double* pb) {
    if (cw4[0] == 0 && cw4[1] == 0 && cw4[2] == 0 && cw4[3] == 0) return;
    const T k[4] = {T(Yt[4]), T(Yt[5]), T(Yt[6]), T(Yt[7])};
    const T cw[4] = {T(cw4[0]), T(cw4[1]), T(cw4[2]), T(cw4[3])};
    T br, bth, ba, bk[4];
    kerr_accel_vjp<T>(m.tor.M, T(m.tor.a), T(Yt[1]), T(Yt[2]), k, cw, br, bth, ba, bk);
    mu[1] += (double)br;
    mu[2] += (double)bth;
    for (int q = 0; q < 4; ++q) mu[4 + q] += (double)bk[q];
    pb[0] += (double)ba;
}

#ifdef __CUDA_ARCH__
// the FP64 Jacobian of the FP32-mixed sweep (near the horizon and the poles;
// rare), out of line
__device__ __noinline__ void torus_accel_vjp_f64_cold(const TorusModel& m, const double* Yt, const double* cw4,
                                                      double* mu, double* pb) {
    torus_accel_vjp<double>(m, Yt, cw4, mu, pb);
}
#endif

template <class BT>
RTW_HD double torus_dp_vjp(const TorusModel& m, const double* y, const double* Kg, double* tau, bool tau_at_end,
                           double h, double* lam, double* pb, bool geo64 = true) {
    const int N = m.n;
    // the emitter numbers and their tangents in the partials' precision BT
    typedef Dual<BT, 8> D8;  // r, theta, k^t, k^phi, a, n0, b0, th0
    double Yg[6][8];
    for (int t = 0; t < 6; ++t)
        for (int i = 0; i < 8; ++i) {
            double acc = 0;
            for (int s = 0; s < t; ++s) acc += tA(t, s) * Kg[s * 8 + i];
            Yg[t][i] = y[i] + h * acc;
        }
    BT dS[6][4][8];
    double Sbar[6][4];
    TorusBinPre pre[6];
    bool on[6];
    for (int t = 0; t < 6; ++t) {
        const TorusPt<D8> S = torus_point<D8>(m.tor, D8::var(BT(m.tor.a), 4), D8::var(BT(m.tor.n0), 5),
                                              D8::var(BT(m.tor.B0), 6), D8::var(BT(m.tor.Th0), 7),
                                              D8::var(BT(Yg[t][1]), 0), D8::var(BT(Yg[t][2]), 1),
                                              D8::var(BT(Yg[t][4]), 2), D8::var(BT(Yg[t][7]), 3));
        on[t] = S.on;
        if (S.on) pre[t] = torus_bin_pre_t<BT>(S.cj.v, S.nus.v, S.th.v, S.g.v);
        const D8* comp[4] = {&S.cj, &S.nus, &S.th, &S.g};
        for (int q = 0; q < 4; ++q) {
            Sbar[t][q] = 0;
            for (int u = 0; u < 8; ++u) dS[t][q][u] = comp[q]->d[u];
        }
    }
    double hbar = 0;
    // (2) bins. The partials of a bin's slopes are linear in (DX, Dy) with
    // per-stage factors (torus_bin_core), so each stage's cotangent of the
    // emitter numbers is formed from three sums over the bins, with
    // U = kappa_tau ft and V = kappa_I e fi:
    //   W0 = sum (U + V), WX = sum (U + V) DX, WY = sum U Dy;
    //   Sbar = (W0 / cj, (W0 - WX) / nus, -WY / th, (WX - 4 W0 + WY) / g).
    // The per-stage arrays of a bin are kept in BT (their values' own
    // precision), so that the loop's live set stays in registers.
    double W0[6] = {0, 0, 0, 0, 0, 0}, WX[6] = {0, 0, 0, 0, 0, 0}, WY[6] = {0, 0, 0, 0, 0, 0};
    // no emitting stage point: every bin's slopes are 0 in this step, so it
    // adds nothing to any cotangent and leaves the optical depths as they are
    bool any_on = false;
    for (int t = 0; t < 6; ++t) any_on |= on[t];
    for (int c = 0; c < (any_on ? N : 0); ++c) {
        const int it = 8 + c, ii = 8 + N + c;
        BT Kt[6], fi[6], ex[6], DX[6], Dy[6], av[6];
        double kt[6];
        const double lt = lam[it], li = lam[ii];
        double bkt = 0, bki = 0;
#pragma unroll
        for (int t = 0; t < 6; ++t) {
            Kt[t] = fi[t] = DX[t] = Dy[t] = BT(0);
            if (on[t]) torus_bin_core<BT>(pre[t], m.bins[c], Kt[t], fi[t], DX[t], Dy[t]);
            bkt += tA(6, t) * (double)Kt[t];
        }
        double t0 = tau[c];
        if (tau_at_end) {
            t0 -= h * bkt;
            tau[c] = t0;
        }
        // the stage depth offsets sum_s a_ts Kt_s in BT (the FP32-mixed
        // forward forms its stage depths so), kept for the step-size term below
        const BT t0b = BT(t0), hb = BT(h);
#pragma unroll
        for (int t = 0; t < 6; ++t) {
            BT acc = 0;
#pragma unroll
            for (int s = 0; s < t; ++s) acc += BT(tA(t, s)) * Kt[s];
            av[t] = acc;
            ex[t] = on[t] ? BinMath<BT>::ex(-(t0b + hb * acc)) : BT(0);
            bki += tA(6, t) * (double)fi[t] * (double)ex[t];
            kt[t] = h * tA(6, t) * lt;
        }
        hbar += lt * bkt + li * bki;
        double msum = 0;
#pragma unroll
        for (int t = 5; t >= 0; --t) {
            if (!on[t]) continue;  // no emitter: the bin's slopes are 0 there
            const double ki = h * tA(6, t) * li, e = (double)ex[t];
            const double U = kt[t] * (double)Kt[t], V = ki * e * (double)fi[t];
            W0[t] += U + V;
            WX[t] += (U + V) * (double)DX[t];
            WY[t] += U * (double)Dy[t];
            const double mt = -ki * (double)fi[t] * e;  // d (fi exp(-tau)) / d tau
            msum += mt;
#pragma unroll
            for (int s = 0; s < t; ++s) kt[s] += h * tA(t, s) * mt;
            hbar += mt * (double)av[t];
        }
        lam[it] = lt + msum;
    }
    for (int t = 0; t < 6; ++t) {
        if (!on[t]) continue;
        Sbar[t][0] = W0[t] * pre[t].icj;
        Sbar[t][1] = (W0[t] - WX[t]) * pre[t].inus;
        Sbar[t][2] = -WY[t] * pre[t].ith;
        Sbar[t][3] = (WX[t] - 4 * W0[t] + WY[t]) * pre[t].ig;
    }
    // (3) geodesic components
    double kg[6][8], lg[8];
    for (int i = 0; i < 8; ++i) {
        double bk = 0;
        for (int s = 0; s < 6; ++s) bk += tA(6, s) * Kg[s * 8 + i];
        hbar += lam[i] * bk;
        lg[i] = lam[i];
        for (int s = 0; s < 6; ++s) kg[s][i] = h * tA(6, s) * lam[i];
    }
    for (int t = 5; t >= 0; --t) {
        double mu[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int i = 0; i < 4; ++i) mu[4 + i] += kg[t][i];
        // the geodesic Jacobian: FP32 where the FP32-mixed forward ran FP32
        // stages (away from the horizon and the poles), FP64 elsewhere
        if (sizeof(BT) == 4 && !geo64)
            torus_accel_vjp<float>(m, Yg[t], kg[t] + 4, mu, pb);
#ifdef __CUDA_ARCH__
        else if (sizeof(BT) == 4)
            torus_accel_vjp_f64_cold(m, Yg[t], kg[t] + 4, mu, pb);
#endif
        else
            torus_accel_vjp<double>(m, Yg[t], kg[t] + 4, mu, pb);
        if (on[t]) {
            double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            for (int q = 0; q < 4; ++q)
                for (int u = 0; u < 8; ++u) v[u] += Sbar[t][q] * (double)dS[t][q][u];
            mu[1] += v[0];
            mu[2] += v[1];
            mu[4] += v[2];
            mu[7] += v[3];
            pb[0] += v[4];
            pb[2] += v[5];
            pb[3] += v[6];
            pb[4] += v[7];
        }
        for (int i = 0; i < 8; ++i) {
            lg[i] += mu[i];
            double ak = 0;
            for (int s = 0; s < t; ++s) {
                ak += tA(t, s) * Kg[s * 8 + i];
                kg[s][i] += h * tA(t, s) * mu[i];
            }
            hbar += mu[i] * ak;
        }
    }
    for (int i = 0; i < 8; ++i) lam[i] = lg[i];
    return hbar;
}

constexpr int kTorusMaxD = 8 + 2 * kTorusMaxBins;  // state components

// Reverse kernel (FP64), one lane per ray. A ray without a polar escape walks
// its chunks backwards: replays each segment's geodesic from the chunk's
// checkpoint (G [ck_every + 1][8] states, Kgs [ck_every][6][8] stage slopes)
// and runs the bins' optical depths backwards from the segment's end state
// (the next chunk's checkpoint; the last segment ends at the ray's final
// state); a ray with a polar escape was re-recorded with its full state
// before every event (Ys [2][D], Kw [6][D] stage slopes, Ze [4][D] escape
// evaluations). The arrays live in local memory,
// whose layout interleaves the lanes of a warp (same-index accesses coalesce).
// The reverse kernel's path for rays with a polar escape (re-recorded with
// their full state before every event; rare), kept out of line.
__device__ __noinline__ bool torus_replay_cold(const TorusModel& m, const double* y_in, uint8_t kind, double hv,
                                               double* y_out, double* K, double* Y) {
    return torus_replay(m, y_in, kind, hv, y_out, K, Y);
}
__device__ __noinline__ bool torus_escape_vjp_cold(const TorusModel& m, const double* y, int nsub, double temp,
                                                   double* lam, double* pb, double* W, double* mu, double* tmp) {
    return torus_escape_vjp(m, y, nsub, temp, lam, pb, W, mu, tmp);
}

#ifndef RTW_REV_MIN_CTAS
#define RTW_REV_MIN_CTAS 2  // CTAs per SM the reverse kernel is compiled for (255 registers)
#endif
template <bool MIXED>
__global__ void __launch_bounds__(128, RTW_REV_MIN_CTAS) torus_reverse(__grid_constant__ const TorusRP p) {
    const TorusModel& m = p.f.m;
    const int N = m.n, D = 8 + 2 * N;
    double G[(kTorusMaxCk + 1) * 8], Kgs[kTorusMaxCk * 48], taus[kTorusMaxBins];
    double Ys[2 * kTorusMaxD], Kw[6 * kTorusMaxD], Ze[4 * kTorusMaxD];
    double lam[kTorusMaxD], mu[kTorusMaxD], tmp[kTorusMaxD];
    unsigned n_cut = 0;
    for (;;) {
        const long long k = (long long)atomicAdd(p.counter, 1ull);
        if (k >= p.f.total_rays) break;
        // longest first: the last rays taken are short, so the grid's lanes end together
        const long long loc = p.order ? (long long)p.order[k] : k;
        const long long id = p.f.ray0 + loc * p.f.ray_stride;
        double loss = 0;
        bool fin = true;
        for (int i = 0; i < D; ++i) lam[i] = 0;
        for (int c = 0; c < N; ++c) {
            const double d = (double)p.spectrum[id * N + c] - (double)p.target[id * N + c];
            fin &= isfinite(d);
            lam[8 + N + c] = 2 * d;
            loss += d * d;
        }
        const bool escaped = (p.f.n_events[loc] & kDenseCheckpoints) != 0;
        if (escaped) atomicAdd(&p.out[2 + kTorusParams], 1.0);
        if (!fin || (escaped && p.skip_escape_rays)) {
            if (fin) atomicAdd(&p.out[0], loss);
            if (p.per_ray)
                for (int q = 0; q < kTorusParams; ++q) p.per_ray[id * kTorusParams + q] = 0;
            continue;
        }
        double pb[kTorusParams] = {0, 0, 0, 0, 0};
        double pend = 0;  // d loss / d h of a step whose h was set at the previous step's start
        const uint32_t n_ev = p.f.n_events[loc] & kEventCount;
        const int KC = escaped ? 1 : p.f.ck_every;
        const int nseg = (int)((n_ev + (uint32_t)KC - 1) / (uint32_t)KC);
        // the reverse of one DP step from geodesic start state g
        auto dp_step = [&](const double* g, const double* Kg, uint8_t kind, double hv, bool refl, bool tau_at_end) {
            if (refl) {
                lam[2] = -lam[2];
                lam[6] = -lam[6];
            }
            const bool geo64 = !MIXED || (g[1] - m.geo.r_ev < p.f.promote_dr) || (g[2] < p.f.promote_theta) ||
                               (g[2] > kPi - p.f.promote_theta);
            const double hbar = torus_dp_vjp<typename std::conditional<MIXED, float, double>::type>(
                m, g, Kg, taus, tau_at_end, hv, lam, pb, geo64);
            // a pending step-size term of the next step lands on this state
            if (pend != 0) torus_pad_vjp(g, p.f.max_dt_scale, pend, lam);
            pend = 0;
            if (kind == 0x42) torus_pad_vjp(g, p.f.max_dt_scale, hbar, lam);
            if (kind == 0x41) pend = hbar;
        };
        if (!escaped) {
            const unsigned long long base = p.rbase[loc];
            const double* c1 = p.f.fin + loc * (long long)D;  // the state after the segment
            for (int seg = nseg - 1; seg >= 0; --seg) {
                const int e0 = seg * KC;
                const int e1 = min(e0 + KC, (int)n_ev);
                const char* ch = torus_chunk(p.f, base + (unsigned long long)seg);
                const double* c0 = (const double*)ch;
                const double* hs = (const double*)(ch + 8 * (8 + N));
                const uint8_t* ks = (const uint8_t*)(ch + 8 * (8 + N) + 8 * KC);
                for (int i = 0; i < 8; ++i) G[i] = c0[i];
                unsigned refl = 0;
                for (int e = e0; e < e1; ++e)
                    if (torus_geo_step(m, G + (e - e0) * 8, hs[e - e0], Kgs + (e - e0) * 48, G + (e - e0 + 1) * 8))
                        refl |= 1u << (e - e0);
                for (int c = 0; c < N; ++c) taus[c] = c1[8 + c];
                for (int e = e1 - 1; e >= e0; --e)
                    dp_step(G + (e - e0) * 8, Kgs + (e - e0) * 48, ks[e - e0], hs[e - e0], (refl >> (e - e0)) & 1u,
                            true);
                c1 = c0;
            }
        } else {
            const uint32_t j = p.esc_index[loc];
            const unsigned long long eo = p.f.ev_off[j], co = p.f.ck_off[j];
            for (int e = (int)n_ev - 1; e >= 0; --e) {
                const double* c0 = p.f.ck + (co + (unsigned long long)e) * (unsigned long long)D;
                for (int i = 0; i < D; ++i) Ys[i] = c0[i];
                const uint8_t kind = p.f.ev_kind[eo + e];
                const double hv = p.f.ev_h[eo + e];
                if (torus_is_dp(kind)) {
                    const bool r = torus_replay_cold(m, Ys, kind, hv, Ys + D, Kw, tmp);
                    for (int st = 0; st < 6; ++st)
                        for (int i = 0; i < 8; ++i) Kgs[st * 8 + i] = Kw[st * D + i];
                    for (int c = 0; c < N; ++c) taus[c] = Ys[8 + c];
                    dp_step(Ys, Kgs, kind, hv, r, false);
                } else {
                    if (!torus_escape_vjp_cold(m, Ys, (int)kind - 1, hv, lam, pb, Ze, mu, tmp)) ++n_cut;
                }
            }
        }
        // the camera initial data: d y0 / d(a, inclination)
        const int pi = (int)(id % p.f.frame.xp), pj = (int)(id / p.f.frame.xp);
        for (int q = 0; q < 2; ++q) {
            double dy[9];
            camera_ray(p.dframe[q], pi, pj, dy);
            double s = 0;
            for (int i = 0; i < 8; ++i) s += lam[i] * dy[i];
            pb[q] += s;
        }
        atomicAdd(&p.out[0], loss);
        for (int q = 0; q < kTorusParams; ++q) atomicAdd(&p.out[1 + q], pb[q]);
        if (p.per_ray)
            for (int q = 0; q < kTorusParams; ++q) p.per_ray[id * kTorusParams + q] = pb[q];
    }
    if (n_cut) atomicAdd(&p.out[1 + kTorusParams], (double)n_cut);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct TorusBuffers {
    void* ctl = nullptr;  // counters + stats + err flag + out
    size_t ctl_cap = 0;
    void* out = nullptr;  // spectrum, class, steps
    size_t out_cap = 0;
    void* nev = nullptr;  // n_events, ev_off, ck_off
    size_t nev_cap = 0;
    void* evh = nullptr;
    size_t evh_cap = 0;
    void* evk = nullptr;
    size_t evk_cap = 0;
    void* ck = nullptr;
    size_t ck_cap = 0;
    void* work = nullptr;
    size_t work_cap = 0;
    void* pool = nullptr;  // recording chunks (the rays' regions)
    size_t pool_cap = 0;
    void* pool2 = nullptr;  // recording chunks (the overflowed rays)
    size_t pool2_cap = 0;
    void* sky = nullptr;    // the wormhole's skyboxes
    size_t sky_cap = 0;
    void* gaunt = nullptr;  // the bremsstrahlung torus's Gaunt-factor table
    size_t gaunt_cap = 0;
    void* fin = nullptr;   // final states
    size_t fin_cap = 0;
    void* tgt = nullptr;
    size_t tgt_cap = 0;
};

void torus_free(TorusBuffers* b) {
    if (!b) return;
    for (void* q : {b->ctl, b->out, b->nev, b->evh, b->evk, b->ck, b->work, b->tgt, b->pool, b->pool2, b->fin, b->sky,
                    b->gaunt})
        if (q) cudaFree(q);
    delete b;
}

namespace {

constexpr double kE = 4.80320425e-10;          // esu
constexpr double kCcgs = 2.99792458e10;        // cm/s
constexpr double kMe = 9.1093837015e-28;       // g
constexpr double kHcgs = 6.62607015e-27;       // erg s
constexpr double kMec2 = kMe * kCcgs * kCcgs;  // erg
constexpr double kRydbergErg = 2.1798723611035e-11;  // Rydberg energy (CODATA 2018), erg

// Powehi.source constants (source_model.jl:7-35, source_geometry.jl:7-34)
constexpr double kPowehiP = 2.5, kPowehiGmin = 30.0, kPowehiGmax = 1e9;
constexpr double kPowehiFitC = 7.951834e-01, kPowehiFitD = 9.832989e-01, kPowehiFitE = -5.752283e-01;

void powehi_model(const rtw_scene& s, const DevScene& geo, PowehiDev& w) {
    w.M = s.mass;
    w.a = s.spin;
    w.rs = 2 * s.mass;
    w.r_ev = geo.r_ev;
    w.disk_r_in = s.r_in;
    w.disk_r_out = s.r_out;
    w.disk_th_lo = s.theta_lo;
    w.disk_th_hi = s.theta_hi;
    w.disk_a = s.a_nu;
    w.disk_T = s.temperature;
    w.r_nozzle = 10;
    w.gamma_min = 1.2;
    w.gamma_max = 10;
    w.nozzle_acc = (10.0 - 1.2) / (75.0 - 10.0);
    w.omega_jet = 0.5 * s.spin / (w.rs * w.r_ev);
    w.jet_th_lo = 0.087263889;
    w.jet_th_hi = 3.054236111;
    w.axis_lo = 1e-3;
    w.axis_hi = 3.1406;
    w.b_phi = s.b_0;
    // synch_em = 7.694e-37 map_scale 2.8e7, synch_ab = 2.8173e-24 map_scale
    // (map_scale in metres), times the electron-distribution constants of
    // calc_radiative_coefficients (Marszewski 2021 forms)
    const double ms = s.length_cm / 100.0, p = kPowehiP;
    const double gdiff = std::pow(kPowehiGmin, 1 - p) - std::pow(kPowehiGmax, 1 - p);
    const double cj = std::pow(3.0, p / 2) * (p - 1) / (2 * (p + 1) * gdiff) * std::tgamma((3 * p - 1) / 12) *
                      std::tgamma((3 * p + 19) / 12);
    const double ca = std::pow(3.0, (p + 1) / 2) * (p - 1) / (4 * gdiff) * std::tgamma((3 * p + 2) / 12) *
                      std::tgamma((3 * p + 22) / 12);
    w.j_scale = s.n_e0 * (7.694e-37 * ms * 2.8e7) * cj;
    w.a_scale = s.n_e0 * (2.8173e-24 * ms) * ca;
    w.p_index = p;
    w.inv_p_synch = 1.0 / (std::exp(kPowehiFitC + kPowehiFitE * p) * std::pow(p, kPowehiFitD * p));
}

rtw_status torus_model(const rtw_scene& s, const double* colors_nm, int N, TorusModel& m, std::string& why) {
    std::memset(&m, 0, sizeof(m));
    if (N <= 0 || N > kTorusMaxBins || !colors_nm) {
        why = "the per-bin scenes take 1..32 bins";
        return RTW_ERR_INVALID_PARAM;
    }
    const bool powehi = s.kind == RTW_SCENE_KERR_POWEHI, synchro = s.kind == RTW_SCENE_SYNCHRO_TEST,
               wormhole = s.kind == RTW_SCENE_WORMHOLE, sphere = s.kind == RTW_SCENE_MINKOWSKI_CART_SPHERE,
               brems = s.kind == RTW_SCENE_KERR_BREMS_TORUS;
    if (brems) {
        if (!(s.mass > 0) || !(std::fabs(s.spin) < s.mass) || !(s.length_cm > 0) || !(s.n_e0 >= 0)) {
            why = "scene parameters out of range";
            return RTW_ERR_INVALID_PARAM;
        }
    } else if (sphere) {
        if (!(s.r_out > 0) || !(s.temperature > 0) || !(s.a_nu >= 0) || !(s.escape_radius > 0)) {
            why = "sphere radius, temperature and escape radius must be > 0, a_nu >= 0";
            return RTW_ERR_INVALID_PARAM;
        }
    } else if (wormhole) {
        if (!(s.r_in > 0) || !(s.edge_in >= 0) || !(s.edge_out > 0) || !(s.escape_radius > s.r_in)) {
            why = "wormhole parameters out of range";
            return RTW_ERR_INVALID_PARAM;
        }
    } else if (!(s.mass > 0) || !(std::fabs(s.spin) < s.mass) || !(s.b_0 > 0) || !(s.length_cm > 0) ||
               !(s.n_e0 >= 0)) {
        why = "scene parameters out of range";
        return RTW_ERR_INVALID_PARAM;
    }
    if (synchro && !(s.r_out > 0 && s.escape_radius > 0)) {
        why = "cylinder radius and escape radius must be > 0";
        return RTW_ERR_INVALID_PARAM;
    }
    if (!powehi && !synchro && !wormhole && !sphere && (!(s.r_in > 0) || !(s.r_out >= s.r_in) || !(s.edge_in > 0) || !(s.edge_out > 0) ||
                    !(s.theta_e0 > 0) || !(s.rho_h > 0))) {
        why = "torus parameters out of range";
        return RTW_ERR_INVALID_PARAM;
    }
    rtw_scene g = s;
    g.r_in = 1;  // the geodesic functor's thin disk stays empty
    g.r_out = 0;
    make_dev_scene(g, m.geo);
    TorusDev& t = m.tor;
    t.M = s.mass;
    t.a = s.spin;
    t.r_in = s.r_in;
    t.r_out = s.r_out;
    t.edge_in = s.edge_in;
    t.edge_out = s.edge_out;
    t.cut_in = std::max(s.r_in - 4 * s.edge_in, 1.01 * m.geo.r_ev);
    t.cut_out = s.r_out + 4 * s.edge_out;
    t.h_ratio = s.rho_h;
    t.ne_idx = s.rho_index;
    t.b_idx = s.b_index;
    t.t_idx = s.t_index;
    t.n0 = s.n_e0;
    t.B0 = s.b_0;
    t.Th0 = s.theta_e0;
    t.cj_unit = std::sqrt(2.0) * kPi * kE * kE / (3 * kCcgs) * s.length_cm;
    t.nuc_unit = kE / (2 * kPi * kMe * kCcgs);
    double wx[kTorusMaxBins], wy[kTorusMaxBins], wz[kTorusMaxBins], fac[kTorusMaxBins];
    if (rtw_cie_weights(colors_nm, N, wx, wy, wz, fac) != RTW_OK) {
        why = "colors_nm must be positive";
        return RTW_ERR_INVALID_PARAM;
    }
    for (int c = 0; c < N; ++c) {
        const double lam = colors_nm[c];
        m.bins[c].fx = fac[c] * wx[c];
        m.bins[c].fy = fac[c] * wy[c];
        m.bins[c].fz = fac[c] * wz[c];
        const double nu = kLightC * 1e9 / lam;  // Hz
        m.bins[c].nu_nm = 1.0 / lam;
        m.bins[c].nu_hz = nu;
        m.bins[c].inv_nu_nm3 = lam * lam * lam;
        m.bins[c].b0 = 2 * kHcgs * nu * nu * nu / (kCcgs * kCcgs);
        m.bins[c].hk = kHcgs * nu / kMec2;
        m.bins[c].ln_nu = std::log(nu);
        m.bins[c].inv_b0 = 1.0 / m.bins[c].b0;
        m.bins[c].nu16 = std::pow(nu, 1.0 / 6.0);
    }
    m.n = N;
    m.emitter = powehi ? 1 : synchro ? 2 : wormhole ? 3 : sphere ? 4 : brems ? 5 : 0;
    if (brems) {
        m.br.lut = nullptr;  // set where the table is placed (device or host)
        m.br.cj_unit = kCYarCgs * s.length_cm;
        m.br.ry_mec2 = kRydbergErg / kMec2;
    }
    m.geom = synchro || sphere ? 1 : wormhole ? 2 : 0;
    if (sphere) {
        m.sp.r_sph = s.r_out;
        m.sp.a_nu = s.a_nu;
        m.sp.es = kEmissionScale;
        m.sp.ff_T = kFFactor / s.temperature;
    }
    if (wormhole) {
        // Wormhole.source/source_geometry.jl:7-15: M = W / W_over_M
        const double c = kPi / (2 * std::sqrt(2.0));
        m.wh.rho = s.r_in;
        m.wh.a_wh = s.edge_in;
        m.wh.M = s.edge_out / (-std::log(1 / std::cos(c)) + c * std::tan(c));
    }
    if (powehi || synchro) powehi_model(s, m.geo, m.pw);  // the power-law constants
    if (synchro) {
        m.sy.b_z = s.b_0;
        m.sy.r_cyl = s.r_out;
        m.sy.j_scale = m.pw.j_scale;
        m.sy.a_scale = m.pw.a_scale;
        m.sy.p_index = m.pw.p_index;
        m.sy.inv_p_synch = m.pw.inv_p_synch;
    }
    return RTW_OK;
}

// the forward kernel instance: precision x emitter (0 torus, 1 Powehi, 2
// Synchro_Test in flat Cartesian geometry, 3 none in the wormhole's geometry,
// 4 the blackbody sphere in flat Cartesian geometry, 5 the bremsstrahlung
// torus)
const void* forward_fn(bool mixed, int emitter) {
    static const void* const fn[2][6] = {
        {(const void*)torus_forward<false, 0>, (const void*)torus_forward<false, 1>, (const void*)torus_forward<false, 2>,
         (const void*)torus_forward<false, 3>, (const void*)torus_forward<false, 4>, (const void*)torus_forward<false, 5>},
        {(const void*)torus_forward<true, 0>, (const void*)torus_forward<true, 1>, (const void*)torus_forward<true, 2>,
         (const void*)torus_forward<true, 3>, (const void*)torus_forward<true, 4>, (const void*)torus_forward<true, 5>}};
    return fn[mixed ? 1 : 0][emitter >= 0 && emitter <= 5 ? emitter : 0];
}

// launch shape of the torus kernels: 128 threads, occupancy-limited CTAs
template <class F>
int torus_grid(rtw_ctx* ctx, F fn) {
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 128, 0);
    return ctx->num_sms * std::max(1, occ);
}

struct TorusRun {
    TorusKP kp;
    int grid = 0;
    long long P = 0;
};

// validation, model, frame, buffers and kernel parameters of a torus render
rtw_status torus_setup(rtw_ctx* ctx, const rtw_scene* scene, const rtw_camera* cam, const rtw_render_params* prm,
                       TorusRun& run) {
    if (!scene || !cam || !prm) return fail(ctx, RTW_ERR_INVALID_PARAM, "null argument");
    if (prm->precision != RTW_PREC_FP64 && prm->precision != RTW_PREC_MIXED)
        return fail(ctx, RTW_ERR_INVALID_PARAM, "precision");
    if (prm->integrator != RTW_DP45_FSAL && prm->integrator != RTW_DP45_REF_COMPAT)
        return fail(ctx, RTW_ERR_INVALID_PARAM, "integrator");
    // the bundle enters only the skybox lookups; in the reference its slots
    // also hold off the opacity stop (the all-slots tau test of
    // calc_terminate), which the skybox scenes follow and the others do not
    if (prm->ray_bundles && scene->kind != RTW_SCENE_WORMHOLE && scene->kind != RTW_SCENE_MINKOWSKI_CART_SPHERE)
        return fail(ctx, RTW_ERR_UNSUPPORTED, "ray bundles are built for the skybox scenes only");
    if (!(prm->max_dt_scale > 0)) return fail(ctx, RTW_ERR_INVALID_PARAM, "max_dt_scale must be > 0");
    std::string why;
    TorusKP& p = run.kp;
    std::memset(&p, 0, sizeof(p));
    rtw_status st = torus_model(*scene, prm->colors_nm, prm->n_colors, p.m, why);
    if (st != RTW_OK) return fail(ctx, st, why);
    int64_t total = 0;
    st = rtw_prepare_frames(scene, cam, 1, &p.frame, &total);
    if (st == RTW_ERR_INVALID_CAMERA) return fail(ctx, st, "camera is on a coordinate singularity");
    if (st != RTW_OK) return fail(ctx, st, "camera parameters invalid or non-finite");
    run.P = total;
    if (prm->ray_bundles) {
        p.bundles = 1;
        bundle_basis(*cam, p.bundle_m);
    }
    p.total_rays = total;
    p.ray0 = 0;
    p.ray_stride = 1;
    p.max_dt_scale = prm->max_dt_scale;
    const double pdr = prm->promote_dr < 0 ? -1.0 : (prm->promote_dr > 0 ? prm->promote_dr : 1e-3);
    // pole promotion: default sin(theta) < 1e-2; Powehi's jet lies within 5 deg
    // of the axis, where FP32 stages lose accuracy, so there the default covers it
    const double psn_default = scene->kind == RTW_SCENE_KERR_POWEHI ? 0.1 : 1e-2;
    const double psn =
        prm->promote_sin < 0 ? 0.0 : (prm->promote_sin > 0 ? std::min(prm->promote_sin, 1.0) : psn_default);
    p.promote_dr = pdr * scene->mass;
    p.promote_theta = std::asin(psn);
    p.ck_every = 16;
    p.fsal = prm->integrator == RTW_DP45_FSAL;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, RTW_ERR_CUDA, "cudaSetDevice");
    if (!ctx->torus) ctx->torus = new TorusBuffers();
    TorusBuffers* b = ctx->torus;
    // control block: counter, stats, err flag, out[6]
    if ((st = ensure(ctx, &b->ctl, &b->ctl_cap, 1024)) != RTW_OK) return st;
    unsigned long long* ctl = (unsigned long long*)b->ctl;
    p.counter = ctl;
    p.stats = (DevStats*)(ctl + 1);
    p.err_flag = (unsigned int*)(ctl + 32);
    run.grid = torus_grid(ctx, forward_fn(prm->precision == RTW_PREC_MIXED, p.m.emitter));
    return RTW_OK;
}

cudaError_t launch_forward(const TorusKP& p, bool mixed, int grid, cudaStream_t st) {
    void* args[] = {(void*)&p};
    return cudaLaunchKernel(forward_fn(mixed, p.m.emitter), dim3(grid), dim3(128), args, 0, st);
}

}  // namespace

rtw_status torus_render(rtw_ctx* ctx, const rtw_scene* scene, const rtw_camera* cams, int32_t n_cams,
                        const rtw_render_params* prm, rtw_outputs* out) {
    if (n_cams != 1) return fail(ctx, RTW_ERR_UNSUPPORTED, "the synchrotron torus renders one camera per call");
    TorusRun run;
    rtw_status st = torus_setup(ctx, scene, cams, prm, run);
    if (st != RTW_OK) return st;
    TorusKP& p = run.kp;
    TorusBuffers* b = ctx->torus;
    const int N = p.m.n;
    const long long P = run.P;
    cudaStream_t s = prm->stream ? (cudaStream_t)prm->stream : ctx->stream;
    float* spec = out->spectrum;
    uint8_t* cls = out->term_class;
    uint32_t* steps = out->steps;
    float* xyz = out->xyz;
    double* fst = out->final_state;
    if (!out->on_device) {
        auto up = [](size_t v) { return (v + 255) & ~(size_t)255; };
        const size_t o_steps = up((size_t)P * N * 4), o_cls = o_steps + up((size_t)P * 4),
                     o_xyz = o_cls + up((size_t)P), o_fst = o_xyz + up((size_t)P * 12),
                     need = o_fst + up((size_t)P * 64);
        if ((st = ensure(ctx, &b->out, &b->out_cap, need)) != RTW_OK) return st;
        char* base = (char*)b->out;
        spec = out->spectrum ? (float*)base : nullptr;
        steps = out->steps ? (uint32_t*)(base + o_steps) : nullptr;
        cls = out->term_class ? (uint8_t*)(base + o_cls) : nullptr;
        xyz = out->xyz ? (float*)(base + o_xyz) : nullptr;
        fst = out->final_state ? (double*)(base + o_fst) : nullptr;
    }
    p.final_state = fst;
    p.spectrum = spec;
    // the skyboxes: host cube maps uploaded for this render
    if (scene->kind == RTW_SCENE_WORMHOLE || scene->kind == RTW_SCENE_MINKOWSKI_CART_SPHERE) {
        size_t off[2] = {0, 0}, need = 0;
        for (int k = 0; k < 2; ++k)
            if (prm->skybox[k]) {
                if (prm->skybox_h[k] < 1) return fail(ctx, RTW_ERR_INVALID_PARAM, "skybox_h must be >= 1");
                off[k] = need;
                need += ((size_t)12 * prm->skybox_h[k] * prm->skybox_h[k] * 3 * sizeof(float) + 255) & ~(size_t)255;
            }
        if (need) {
            if ((st = ensure(ctx, &b->sky, &b->sky_cap, need)) != RTW_OK) return st;
            for (int k = 0; k < 2; ++k)
                if (prm->skybox[k]) {
                    const size_t bytes = (size_t)12 * prm->skybox_h[k] * prm->skybox_h[k] * 3 * sizeof(float);
                    RTW_CUDA(cudaMemcpyAsync((char*)b->sky + off[k], prm->skybox[k], bytes, cudaMemcpyHostToDevice, s),
                             "skybox H2D");
                    p.sky[k] = (const float*)((char*)b->sky + off[k]);
                    p.sky_h[k] = prm->skybox_h[k];
                }
        }
    }
    // the bremsstrahlung torus's Gaunt-factor table, uploaded for this render
    if (scene->kind == RTW_SCENE_KERR_BREMS_TORUS) {
        if (!prm->gaunt_lut) return fail(ctx, RTW_ERR_INVALID_PARAM, "the bremsstrahlung torus needs gaunt_lut");
        const size_t bytes = sizeof(float) * kGauntRows * kGauntCols;
        if ((st = ensure(ctx, &b->gaunt, &b->gaunt_cap, bytes)) != RTW_OK) return st;
        RTW_CUDA(cudaMemcpyAsync(b->gaunt, prm->gaunt_lut, bytes, cudaMemcpyHostToDevice, s), "Gaunt table H2D");
        p.m.br.lut = (const float*)b->gaunt;
    }
    p.cls = cls;
    p.steps = steps;
    p.xyz = xyz;
    // the context's counter and stats block, so that rtw_get_stats reads them
    p.counter = ctx->d_ctl;
    p.stats = (DevStats*)(ctx->d_ctl + 1);
    RTW_CUDA(cudaEventRecord(ctx->ev[0], s), "event");
    RTW_CUDA(cudaMemsetAsync(ctx->d_ctl, 0, sizeof(unsigned long long) + sizeof(DevStats), s), "reset counters");
    RTW_CUDA(cudaEventRecord(ctx->ev[1], s), "event");
    RTW_CUDA(launch_forward(p, prm->precision == RTW_PREC_MIXED, run.grid, s), "torus kernel launch");
    RTW_CUDA(cudaEventRecord(ctx->ev[2], s), "event");
    if (!out->on_device) {
        if (out->spectrum)
            RTW_CUDA(cudaMemcpyAsync(out->spectrum, spec, sizeof(float) * N * P, cudaMemcpyDeviceToHost, s), "D2H");
        if (out->steps) RTW_CUDA(cudaMemcpyAsync(out->steps, steps, 4 * P, cudaMemcpyDeviceToHost, s), "D2H");
        if (out->term_class) RTW_CUDA(cudaMemcpyAsync(out->term_class, cls, P, cudaMemcpyDeviceToHost, s), "D2H");
    }
    if (out->xyz && !out->on_device)
        RTW_CUDA(cudaMemcpyAsync(out->xyz, xyz, sizeof(float) * 3 * P, cudaMemcpyDeviceToHost, s), "xyz D2H");
    if (out->final_state && !out->on_device)
        RTW_CUDA(cudaMemcpyAsync(out->final_state, fst, sizeof(double) * 8 * P, cudaMemcpyDeviceToHost, s),
                 "state D2H");
    RTW_CUDA(cudaEventRecord(ctx->ev[3], s), "event");
    ctx->have_last = true;
    ctx->last_frames = 0;
    ctx->last_grid = run.grid;
    ctx->last_warps = 4;
    ctx->last_refill = 1;
    ctx->last_replayed = 0;
    ctx->last_launches = 1;
    ctx->last_tail_cap = 0;
    if (!prm->stream) RTW_CUDA(cudaStreamSynchronize(s), "torus kernel");
    return RTW_OK;
}

}  // namespace rtw

using namespace rtw;

extern "C" {

rtw_status rtw_adjoint(rtw_ctx* ctx, const rtw_scene* scene, const rtw_camera* cam, const rtw_render_params* prm,
                       const rtw_adjoint_params* adj, rtw_outputs* out, rtw_adjoint_result* res) {
    if (!ctx) return RTW_ERR_INVALID_PARAM;
    ctx->err.clear();
    if (!scene || !cam || !prm || !adj || !res || !adj->target) return fail(ctx, RTW_ERR_INVALID_PARAM, "null argument");
    if (scene->kind != RTW_SCENE_KERR_SYNCHRO_TORUS)
        return fail(ctx, RTW_ERR_UNSUPPORTED, "the adjoint is built for the synchrotron torus");
    if (prm->integrator != RTW_DP45_FSAL)
        return fail(ctx, RTW_ERR_UNSUPPORTED, "the adjoint needs the FSAL integrator (each step a function of its start state)");
    TorusRun run;
    rtw_status st = torus_setup(ctx, scene, cam, prm, run);
    if (st != RTW_OK) return st;
    TorusKP& p = run.kp;
    TorusBuffers* b = ctx->torus;
    const int N = p.m.n, D = 8 + 2 * N;
    const long long P = run.P;
    // the ray subset: pixels ray_begin + k ray_stride, k < ray_count
    const long long rs = adj->ray_stride > 0 ? adj->ray_stride : 1;
    const long long r0 = adj->ray_begin;
    const long long Q = adj->ray_count > 0 ? adj->ray_count : (r0 < P ? (P - r0 + rs - 1) / rs : 0);
    if (r0 < 0 || Q <= 0 || r0 + (Q - 1) * rs >= P)
        return fail(ctx, RTW_ERR_INVALID_PARAM, "ray subset outside the image");
    p.ray0 = r0;
    p.ray_stride = rs;
    p.total_rays = Q;
    const int KC = adj->checkpoint_every > 0 ? std::min(adj->checkpoint_every, kTorusMaxCk) : 16;
    p.ck_every = KC;
    const double dl = adj->camera_delta > 0 ? adj->camera_delta : 1e-6;
    const bool mixed = prm->precision == RTW_PREC_MIXED;
    cudaStream_t s = ctx->stream;
    std::memset(res, 0, sizeof(*res));

    // derivative of the camera transform in a and the inclination
    TorusRP rp;
    std::memset(&rp, 0, sizeof(rp));
    for (int q = 0; q < 2; ++q) {
        rtw_scene sp = *scene, sm = *scene;
        rtw_camera cp = *cam, cm = *cam;
        if (q == 0) {
            sp.spin += dl;
            sm.spin -= dl;
        } else {
            cp.position[2] += dl;
            cm.position[2] -= dl;
        }
        FrameDesc fp, fm;
        int64_t tp = 0, tm = 0;
        if (rtw_prepare_frames(&sp, &cp, 1, &fp, &tp) != RTW_OK || rtw_prepare_frames(&sm, &cm, 1, &fm, &tm) != RTW_OK)
            return fail(ctx, RTW_ERR_INVALID_PARAM, "camera transform not differentiable here");
        FrameDesc d = p.frame;
        for (int i = 0; i < 4; ++i) d.pos[i] = (fp.pos[i] - fm.pos[i]) / (2 * dl);
        for (int i = 0; i < 16; ++i) d.M[i] = (fp.M[i] - fm.M[i]) / (2 * dl);
        rp.dframe[q] = d;
    }

    // buffers: outputs, event counts and offsets
    const size_t spec_b = ((size_t)P * N * 4 + 255) & ~(size_t)255;
    if ((st = ensure(ctx, &b->out, &b->out_cap, spec_b + 2 * (((size_t)P * 4 + 255) & ~(size_t)255))) != RTW_OK)
        return st;
    float* spec = (float*)b->out;
    uint32_t* steps = (uint32_t*)((char*)b->out + spec_b);
    uint8_t* cls = (uint8_t*)((char*)b->out + spec_b + (((size_t)P * 4 + 255) & ~(size_t)255));
    // per-ray words: n_events, dense index, the lists of the second passes
    // (dense re-record, overflowed rays) with their counts, offsets and chunk
    // bases, and every ray's first chunk
    const size_t q4 = ((size_t)Q * 4 + 255) & ~(size_t)255;
    const size_t nev_b = 6 * q4 + 4 * (size_t)Q * 8;
    if ((st = ensure(ctx, &b->nev, &b->nev_cap, nev_b)) != RTW_OK) return st;
    uint32_t* nev = (uint32_t*)b->nev;
    uint32_t* esc_index = (uint32_t*)((char*)b->nev + q4);
    uint32_t* ray_list = (uint32_t*)((char*)b->nev + 2 * q4);
    uint32_t* nev_d = (uint32_t*)((char*)b->nev + 3 * q4);
    uint32_t* list2 = (uint32_t*)((char*)b->nev + 4 * q4);
    uint32_t* order = (uint32_t*)((char*)b->nev + 5 * q4);
    unsigned long long* ev_off = (unsigned long long*)((char*)b->nev + 6 * q4);  // [Q] events, then [Q] rows
    unsigned long long* base2 = ev_off + 2 * Q;
    unsigned long long* rbase = ev_off + 3 * Q;
    if ((st = ensure(ctx, &b->fin, &b->fin_cap, std::max<size_t>((size_t)Q * D * 8, 256))) != RTW_OK) return st;
    if ((st = ensure(ctx, &b->tgt, &b->tgt_cap, (size_t)P * N * 4)) != RTW_OK) return st;
    if (adj->target_on_device)
        RTW_CUDA(cudaMemcpyAsync(b->tgt, adj->target, (size_t)P * N * 4, cudaMemcpyDeviceToDevice, s), "target");
    else
        RTW_CUDA(cudaMemcpyAsync(b->tgt, adj->target, (size_t)P * N * 4, cudaMemcpyHostToDevice, s), "target H2D");
    p.spectrum = spec;
    p.cls = cls;
    p.steps = steps;
    p.n_events = nev;

    cudaEvent_t ev[6];
    for (auto& e : ev) RTW_CUDA(cudaEventCreate(&e), "event");
    struct EvGuard {
        cudaEvent_t* e;
        ~EvGuard() {
            for (int i = 0; i < 6; ++i) cudaEventDestroy(e[i]);
        }
    } guard{ev};

    // 1. forward pass, recording: image, step counts, and per ray its chunks
    // (one per segment of KC accepted steps) in a region of R0 chunks of the
    // pool; R0 from the memory there is (at most 256: 4096 steps at KC 16).
    const int cb = torus_chunk_bytes(N, KC);
    unsigned long long R0 = 256;
    {
        size_t fr = 0, tot = 0;
        RTW_CUDA(cudaMemGetInfo(&fr, &tot), "memory info");
        const double avail = 0.6 * (double)(fr + b->pool_cap);
        R0 = std::min<unsigned long long>(R0, (unsigned long long)(avail / ((double)Q * cb)));
        R0 = std::min<unsigned long long>(R0, (unsigned long long)(2 * p.frame.max_steps + KC - 1) / KC + 1);
        if (R0 < 4) return fail(ctx, RTW_ERR_OOM, "not enough device memory for the adjoint's records");
    }
    // (allocated before the timed region, like the other buffers)
    unsigned long long region_bytes = (R0 * cb + 127) / 128 * 128;
    if ((region_bytes / 128) % 2 == 0) region_bytes += 128;
    if ((st = ensure(ctx, &b->pool, &b->pool_cap, (size_t)Q * region_bytes)) != RTW_OK) return st;
    {
        // and the reverse sweep's per-thread local memory (the driver would
        // otherwise grow its reservation, GBs, at the sweep's first launch)
        const void* rfn = mixed ? (const void*)torus_reverse<true> : (const void*)torus_reverse<false>;
        cudaFuncAttributes fa;
        size_t cur = 0;
        RTW_CUDA(cudaFuncGetAttributes(&fa, rfn), "reverse attributes");
        RTW_CUDA(cudaDeviceGetLimit(&cur, cudaLimitStackSize), "stack limit");
        if (fa.localSizeBytes > cur) RTW_CUDA(cudaDeviceSetLimit(cudaLimitStackSize, fa.localSizeBytes), "stack limit");
    }
    p.record = 2;
    p.chunk_bytes = cb;
    p.pool = (char*)b->pool;
    p.split = (unsigned long long)Q * R0;
    p.region_bytes = region_bytes;
    p.region = (unsigned int)R0;
    p.fin = (double*)b->fin;
    std::vector<uint32_t> h_nev(Q);
    RTW_CUDA(cudaEventRecord(ev[0], s), "event");
    RTW_CUDA(cudaMemsetAsync(b->out, 0, b->out_cap, s), "clear outputs");
    RTW_CUDA(cudaMemsetAsync(b->ctl, 0, 1024, s), "reset counters");
    RTW_CUDA(launch_forward(p, mixed, run.grid, s), "torus forward");
    RTW_CUDA(cudaMemcpyAsync(h_nev.data(), nev, 4 * Q, cudaMemcpyDeviceToHost, s), "counts D2H");
    RTW_CUDA(cudaStreamSynchronize(s), "forward");
    RTW_CUDA(cudaEventRecord(ev[1], s), "event");
    // 1b. rays with more segments than R0 (and no polar escape): recorded
    // again, alone, into pool2 at exact offsets
    std::vector<uint32_t> h_l2;
    std::vector<unsigned long long> h_b2, h_rb(Q);
    unsigned long long used = p.split, extra = 0;
    for (long long i = 0; i < Q; ++i) {
        h_rb[i] = (unsigned long long)i * R0;
        if ((h_nev[i] & kOverflow) && !(h_nev[i] & kDenseCheckpoints)) {
            const unsigned long long nseg = ((h_nev[i] & kEventCount) + KC - 1) / KC;
            h_rb[i] = p.split + extra;
            h_l2.push_back((uint32_t)i);
            h_b2.push_back(h_rb[i]);
            extra += nseg;
        }
    }
    used += extra;
    const long long n2 = (long long)h_l2.size();
    RTW_CUDA(cudaEventRecord(ev[2], s), "event");
    if (n2 > 0) {
        if ((st = ensure(ctx, &b->pool2, &b->pool2_cap, (size_t)extra * cb)) != RTW_OK) return st;
        RTW_CUDA(cudaMemcpyAsync(list2, h_l2.data(), 4 * n2, cudaMemcpyHostToDevice, s), "list H2D");
        RTW_CUDA(cudaMemcpyAsync(base2, h_b2.data(), 8 * n2, cudaMemcpyHostToDevice, s), "bases H2D");
        TorusKP p2 = p;
        p2.pool2 = (char*)b->pool2;
        p2.region = 0;
        p2.chunk_base = base2;
        p2.ray_list = list2;
        p2.total_rays = n2;
        p2.spectrum = nullptr;  // the first pass's image stays
        p2.xyz = nullptr;
        p2.cls = nullptr;
        p2.steps = nullptr;
        RTW_CUDA(cudaMemsetAsync(b->ctl, 0, 8, s), "reset queue");
        RTW_CUDA(launch_forward(p2, mixed, run.grid, s), "torus record of long rays");
        p.pool2 = p2.pool2;
    }
    RTW_CUDA(cudaMemcpyAsync(rbase, h_rb.data(), 8 * Q, cudaMemcpyHostToDevice, s), "chunk bases H2D");
    // the reverse sweep's queue: rays by decreasing recorded steps (rays left
    // out of the gradient cost nothing and go last)
    std::vector<uint32_t> h_order(Q);
    {
        std::vector<uint64_t> key(Q);
        for (long long i = 0; i < Q; ++i) {
            const bool skip = (h_nev[i] & kDenseCheckpoints) && adj->escape_rays == 1;
            key[i] = ((uint64_t)(skip ? 0u : (h_nev[i] & kEventCount)) << 32) | (uint64_t)(0xffffffffu - (uint32_t)i);
        }
        std::sort(key.begin(), key.end(), std::greater<uint64_t>());
        for (long long i = 0; i < Q; ++i) h_order[i] = 0xffffffffu - (uint32_t)(key[i] & 0xffffffffu);
    }
    RTW_CUDA(cudaMemcpyAsync(order, h_order.data(), 4 * Q, cudaMemcpyHostToDevice, s), "order H2D");
    // 2. rays with a polar escape whose gradient is wanted: a second recording
    // pass over them alone, with the full state before every event
    unsigned long long E = 0, C = 0;
    std::vector<uint32_t> h_list, h_nd, h_esc(Q, 0xffffffffu);
    for (long long i = 0; i < Q; ++i) {
        E += h_nev[i] & kEventCount;
        if ((h_nev[i] & kDenseCheckpoints) && adj->escape_rays != 1) {
            h_esc[i] = (uint32_t)h_list.size();
            h_list.push_back((uint32_t)i);
            h_nd.push_back(h_nev[i]);
        }
    }
    const long long nB = (long long)h_list.size();
    std::vector<unsigned long long> h_off(2 * std::max<long long>(nB, 1));
    unsigned long long Ed = 0;
    for (long long j = 0; j < nB; ++j) {
        h_off[j] = Ed;
        h_off[nB + j] = C;
        const uint32_t n = h_nd[j] & kEventCount;
        Ed += n;
        C += n + 1;  // one row before every event + the final state
    }
    if ((st = ensure(ctx, &b->evh, &b->evh_cap, std::max<size_t>(8 * Ed, 256))) != RTW_OK) return st;
    if ((st = ensure(ctx, &b->evk, &b->evk_cap, std::max<size_t>(Ed, 256))) != RTW_OK) return st;
    if ((st = ensure(ctx, &b->ck, &b->ck_cap, std::max<size_t>(8 * C * (size_t)D, 256))) != RTW_OK) return st;
    RTW_CUDA(cudaMemcpyAsync(esc_index, h_esc.data(), 4 * Q, cudaMemcpyHostToDevice, s), "dense index H2D");
    p.ev_h = (double*)b->evh;
    p.ev_kind = (uint8_t*)b->evk;
    p.ck = (double*)b->ck;
    p.ev_off = ev_off;
    p.ck_off = ev_off + nB;
    if (nB > 0) {
        RTW_CUDA(cudaMemcpyAsync(ray_list, h_list.data(), 4 * nB, cudaMemcpyHostToDevice, s), "list H2D");
        RTW_CUDA(cudaMemcpyAsync(nev_d, h_nd.data(), 4 * nB, cudaMemcpyHostToDevice, s), "counts H2D");
        RTW_CUDA(cudaMemcpyAsync(ev_off, h_off.data(), 16 * nB, cudaMemcpyHostToDevice, s), "offsets H2D");
        TorusKP pd = p;
        pd.record = 1;
        pd.ray_list = ray_list;
        pd.total_rays = nB;
        pd.n_events = nev_d;
        pd.spectrum = nullptr;  // the first pass's image stays
        pd.xyz = nullptr;
        pd.cls = nullptr;
        pd.steps = nullptr;
        RTW_CUDA(cudaMemsetAsync(b->ctl, 0, 8, s), "reset queue");
        RTW_CUDA(launch_forward(pd, mixed, run.grid, s), "torus dense record");
    }
    RTW_CUDA(cudaEventRecord(ev[3], s), "event");
    // 3. reverse pass
    int occ = 0;
    const void* rev_fn = mixed ? (const void*)torus_reverse<true> : (const void*)torus_reverse<false>;
    RTW_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, rev_fn, 128, 0), "occupancy");
    const int rgrid = ctx->num_sms * std::max(1, occ);
    // local-memory work area of the reverse kernel (per resident thread)
    const size_t work_b = (size_t)rgrid * 128 *
                          ((size_t)(2 + 6 + 4 + 3) * kTorusMaxD + (kTorusMaxCk + 1) * 8 + kTorusMaxCk * 48 + kTorusMaxBins) * 8;
    const size_t per_ray_b = adj->per_ray_grad ? (size_t)P * kTorusParams * 8 : 0;
    if ((st = ensure(ctx, &b->work, &b->work_cap, std::max<size_t>(per_ray_b, 256))) != RTW_OK) return st;
    rp.f = p;
    rp.f.spectrum = spec;
    rp.esc_index = esc_index;
    rp.rbase = rbase;
    rp.order = order;
    rp.target = (const float*)b->tgt;
    rp.spectrum = spec;
    rp.per_ray = adj->per_ray_grad ? (double*)b->work : nullptr;
    rp.skip_escape_rays = adj->escape_rays == 1;
    unsigned long long* ctl = (unsigned long long*)b->ctl;
    rp.out = (double*)(ctl + 40);
    rp.counter = ctl + 39;
    if (rp.per_ray) RTW_CUDA(cudaMemsetAsync(rp.per_ray, 0, per_ray_b, s), "clear per-ray gradients");
    RTW_CUDA(cudaEventRecord(ev[4], s), "event");
    {
        void* args[] = {(void*)&rp};
        RTW_CUDA(cudaLaunchKernel(rev_fn, dim3(rgrid), dim3(128), args, 0, s), "torus reverse");
    }
    RTW_CUDA(cudaEventRecord(ev[5], s), "event");
    double h_out[3 + kTorusParams];
    unsigned int flag = 0;
    RTW_CUDA(cudaMemcpyAsync(h_out, rp.out, sizeof(h_out), cudaMemcpyDeviceToHost, s), "result D2H");
    RTW_CUDA(cudaMemcpyAsync(&flag, p.err_flag, 4, cudaMemcpyDeviceToHost, s), "flag D2H");
    if (rp.per_ray)
        RTW_CUDA(cudaMemcpyAsync(adj->per_ray_grad, rp.per_ray, per_ray_b, cudaMemcpyDeviceToHost, s), "per-ray D2H");
    if (out) {
        if (out->on_device) {
            if (out->spectrum) RTW_CUDA(cudaMemcpyAsync(out->spectrum, spec, 4 * N * P, cudaMemcpyDeviceToDevice, s), "D2D");
            if (out->steps) RTW_CUDA(cudaMemcpyAsync(out->steps, steps, 4 * P, cudaMemcpyDeviceToDevice, s), "D2D");
            if (out->term_class) RTW_CUDA(cudaMemcpyAsync(out->term_class, cls, P, cudaMemcpyDeviceToDevice, s), "D2D");
        } else {
            if (out->spectrum) RTW_CUDA(cudaMemcpyAsync(out->spectrum, spec, 4 * N * P, cudaMemcpyDeviceToHost, s), "D2H");
            if (out->steps) RTW_CUDA(cudaMemcpyAsync(out->steps, steps, 4 * P, cudaMemcpyDeviceToHost, s), "D2H");
            if (out->term_class) RTW_CUDA(cudaMemcpyAsync(out->term_class, cls, P, cudaMemcpyDeviceToHost, s), "D2H");
        }
    }
    RTW_CUDA(cudaStreamSynchronize(s), "adjoint");
    if (flag) return fail(ctx, RTW_ERR_CUDA, "record pass diverged from the forward pass");
    float t01 = 0, t23 = 0, t45 = 0, t05 = 0;
    cudaEventElapsedTime(&t01, ev[0], ev[1]);
    cudaEventElapsedTime(&t23, ev[2], ev[3]);
    cudaEventElapsedTime(&t45, ev[4], ev[5]);
    cudaEventElapsedTime(&t05, ev[0], ev[5]);
    res->loss = h_out[0];
    for (int q = 0; q < kTorusParams; ++q) res->grad[q] = h_out[1 + q];
    res->forward_ms = t01;
    res->record_ms = t23;
    res->reverse_ms = t45;
    res->total_ms = t05;
    res->events = E;
    res->checkpoints = used + C;  // chunk slots (the first pass's regions whole) + dense rows
    res->escape_cuts = (uint64_t)h_out[1 + kTorusParams];
    res->escape_rays = (uint64_t)h_out[2 + kTorusParams];
    res->scratch_bytes = (size_t)used * cb + (size_t)Q * D * 8 + 9 * Ed + 8 * C * (size_t)D + work_b + nev_b;
    ctx->have_last = false;
    return RTW_OK;
}

static rtw_status torus_rhs_host(const rtw_scene* scene, const double* colors_nm, int32_t n_colors, int32_t form,
                                 const float* gaunt_lut, const double* state, double* slope) {
    TorusModel m;
    std::string why;
    if (torus_model(*scene, colors_nm, n_colors, m, why) != RTW_OK) return RTW_ERR_INVALID_PARAM;
    m.br.lut = gaunt_lut;
    const int N = n_colors, D = 8 + 2 * N;
    std::vector<double> y(D), f(D);
    for (int i = 0; i < 8; ++i) y[i] = state[i];
    for (int c = 0; c < N; ++c) {
        y[8 + N + c] = state[8 + 2 * c];  // I
        y[8 + c] = state[9 + 2 * c];      // tau
    }
    torus_f64(m, y.data(), f.data());
    if (form == 1) {
        double acc[4];
        const double k[4] = {y[4], y[5], y[6], y[7]};
        kerr_accel<double>(m.tor.M, m.tor.a, y[1], y[2], k, acc);
        for (int i = 0; i < 4; ++i) f[4 + i] = acc[i];
    }
    for (int i = 0; i < 8; ++i) slope[i] = f[i];
    for (int c = 0; c < N; ++c) {
        slope[8 + 2 * c] = f[8 + N + c];
        slope[9 + 2 * c] = f[8 + c];
    }
    return RTW_OK;
}

rtw_status rtw_torus_rhs(const rtw_scene* scene, const double* colors_nm, int32_t n_colors, int32_t form,
                         const double* state, double* slope) {
    if (!scene || !state || !slope ||
        (scene->kind != RTW_SCENE_KERR_SYNCHRO_TORUS && scene->kind != RTW_SCENE_KERR_POWEHI &&
         scene->kind != RTW_SCENE_SYNCHRO_TEST && scene->kind != RTW_SCENE_WORMHOLE &&
         scene->kind != RTW_SCENE_MINKOWSKI_CART_SPHERE))
        return RTW_ERR_INVALID_PARAM;
    return torus_rhs_host(scene, colors_nm, n_colors, form, nullptr, state, slope);
}

rtw_status rtw_brems_rhs(const rtw_scene* scene, const double* colors_nm, int32_t n_colors, const float* gaunt_lut,
                         const double* state, double* slope) {
    if (!scene || !state || !slope || !gaunt_lut || scene->kind != RTW_SCENE_KERR_BREMS_TORUS)
        return RTW_ERR_INVALID_PARAM;
    return torus_rhs_host(scene, colors_nm, n_colors, 0, gaunt_lut, state, slope);
}

float rtw_gaunt_lookup(const float* lut, double gam2, double u) {
    if (!lut) return 1.2f;
    return gaunt_van_hoof(lut, rlog10f_(gam2), rlog10f_(u));
}

rtw_status rtw_torus_escape_vjp(const rtw_scene* scene, const double* colors_nm, int32_t n_colors,
                                const double* state, int32_t n_sub, const double* cot, double* end_state,
                                double* mu, double* pbar) {
    if (!scene || !state || !cot || !mu || !pbar || !end_state || n_sub < 1 || n_sub > 37 ||
        scene->kind != RTW_SCENE_KERR_SYNCHRO_TORUS)
        return RTW_ERR_INVALID_PARAM;
    TorusModel m;
    std::string why;
    if (torus_model(*scene, colors_nm, n_colors, m, why) != RTW_OK) return RTW_ERR_INVALID_PARAM;
    const int N = n_colors, D = 8 + 2 * N;
    std::vector<double> y(D), lam(D), W(4 * D), mu_(D), tmp(D), e(D);
    for (int i = 0; i < 8; ++i) {
        y[i] = state[i];
        lam[i] = cot[i];
    }
    for (int c = 0; c < N; ++c) {
        y[8 + N + c] = state[8 + 2 * c];
        y[8 + c] = state[9 + 2 * c];
        lam[8 + N + c] = cot[8 + 2 * c];
        lam[8 + c] = cot[9 + 2 * c];
    }
    torus_escape_end(m, y.data(), n_sub, e.data(), tmp.data());
    double pb[kTorusParams] = {0, 0, 0, 0, 0};
    const bool ok = torus_escape_vjp(m, y.data(), n_sub, torus_escape_temp(y.data()), lam.data(), pb, W.data(),
                                     mu_.data(), tmp.data());
    for (int i = 0; i < 8; ++i) {
        mu[i] = lam[i];
        end_state[i] = e[i];
    }
    for (int c = 0; c < N; ++c) {
        mu[8 + 2 * c] = lam[8 + N + c];
        mu[9 + 2 * c] = lam[8 + c];
        end_state[8 + 2 * c] = e[8 + N + c];
        end_state[9 + 2 * c] = e[8 + c];
    }
    for (int q = 0; q < kTorusParams; ++q) pbar[q] = pb[q];
    return ok ? RTW_OK : RTW_ERR_NAN;
}

rtw_status rtw_skybox_wrap(int32_t i, int32_t j, int32_t face, int32_t x, int32_t y, int32_t n, int32_t* out) {
    if (!out || n < 1 || face < 1 || face > 6) return RTW_ERR_INVALID_PARAM;
    int a = i, b = j, F = face;
    sky_wrap(a, b, F, x, y, n);
    out[0] = a;
    out[1] = b;
    out[2] = F;
    return RTW_OK;
}

rtw_status rtw_torus_step_vjp(const rtw_scene* scene, const double* colors_nm, int32_t n_colors,
                              const double* state, double h, const double* cot, int32_t form, double* mu,
                              double* pbar, double* hbar) {
    if (!scene || !state || !cot || !mu || !pbar || !hbar || scene->kind != RTW_SCENE_KERR_SYNCHRO_TORUS)
        return RTW_ERR_INVALID_PARAM;
    TorusModel m;
    std::string why;
    if (torus_model(*scene, colors_nm, n_colors, m, why) != RTW_OK) return RTW_ERR_INVALID_PARAM;
    const int N = n_colors, D = 8 + 2 * N;
    std::vector<double> y(D), lam(D), K(6 * D), Y(D), Yst(6 * D), kac(6 * D), tmp(D);
    for (int i = 0; i < 8; ++i) {
        y[i] = state[i];
        lam[i] = cot[i];
    }
    for (int c = 0; c < N; ++c) {
        y[8 + N + c] = state[8 + 2 * c];
        y[8 + c] = state[9 + 2 * c];
        lam[8 + N + c] = cot[8 + 2 * c];
        lam[8 + c] = cot[9 + 2 * c];
    }
    torus_dp_stages(m, y.data(), h, K.data(), Y.data(), nullptr);
    double pb[kTorusParams] = {0, 0, 0, 0, 0};
    double Kg[48], taus[kTorusMaxBins];
    for (int st = 0; st < 6; ++st)
        for (int i = 0; i < 8; ++i) Kg[st * 8 + i] = K[st * D + i];
    if (form == 1) {
        *hbar = torus_dp_vjp_generic(m, y.data(), K.data(), h, lam.data(), pb, Yst.data(), kac.data(), tmp.data());
    } else {
        // form 2 starts from the depths at the end of the step
        std::vector<double> y1(D);
        torus_dp_stages(m, y.data(), h, K.data(), Y.data(), y1.data());
        for (int c = 0; c < N; ++c) taus[c] = form >= 2 ? y1[8 + c] : y[8 + c];
        *hbar = form == 3 ? torus_dp_vjp<float>(m, y.data(), Kg, taus, true, h, lam.data(), pb, false)
                          : torus_dp_vjp<double>(m, y.data(), Kg, taus, form == 2, h, lam.data(), pb);
    }
    for (int i = 0; i < 8; ++i) mu[i] = lam[i];
    for (int c = 0; c < N; ++c) {
        mu[8 + 2 * c] = lam[8 + N + c];
        mu[9 + 2 * c] = lam[8 + c];
    }
    for (int q = 0; q < kTorusParams; ++q) pbar[q] = pb[q];
    return RTW_OK;
}

rtw_status rtw_torus_vjp(const rtw_scene* scene, const double* colors_nm, int32_t n_colors, const double* state,
                         const double* cot, double* mu, double* pbar) {
    if (!scene || !state || !cot || !mu || !pbar || scene->kind != RTW_SCENE_KERR_SYNCHRO_TORUS)
        return RTW_ERR_INVALID_PARAM;
    TorusModel m;
    std::string why;
    if (torus_model(*scene, colors_nm, n_colors, m, why) != RTW_OK) return RTW_ERR_INVALID_PARAM;
    const int N = n_colors, D = 8 + 2 * N;
    std::vector<double> y(D), k(D), u(D, 0.0);
    for (int i = 0; i < 8; ++i) {
        y[i] = state[i];
        k[i] = cot[i];
    }
    for (int c = 0; c < N; ++c) {
        y[8 + N + c] = state[8 + 2 * c];
        y[8 + c] = state[9 + 2 * c];
        k[8 + N + c] = cot[8 + 2 * c];
        k[8 + c] = cot[9 + 2 * c];
    }
    double pb[kTorusParams] = {0, 0, 0, 0, 0};
    torus_vjp(m, y.data(), k.data(), u.data(), pb);
    for (int i = 0; i < 8; ++i) mu[i] = u[i];
    for (int c = 0; c < N; ++c) {
        mu[8 + 2 * c] = u[8 + N + c];
        mu[9 + 2 * c] = u[8 + c];
    }
    for (int q = 0; q < kTorusParams; ++q) pbar[q] = pb[q];
    return RTW_OK;
}

}  // extern "C"
