// rtw_scenes.cuh - the reference's ".source" scene contract as compile-time
// device functors, templated on the arithmetic type R of the right-hand side.
//
// Each scene provides, for a stage point z = (t, r, theta, phi, k^t, k^r,
// k^theta, k^phi, tau):
//   * the geodesic slopes dx^mu = k^mu, dk^mu = -Gamma^mu_{ab} k^a k^b
//     (calc_christoffel_udd! + the contraction of calc_ray_derivative!,
//     integrators_LttM.jl:12-30), with the symmetric Christoffel pairs summed
//     once and doubled;
//   * the emitter at z (is_fire, get_source_velocity!, calc_freq_shift,
//     calc_fluid_params!, calc_radiative_coefficients; integrators_LttM.jl:33-42)
//     reduced to three numbers, because every emitter on this path is grey
//     (a_nu does not depend on nu) and blackbody:
//         A    = a_nu * emission_scale * exp(-tau) / g      (>= 0)
//         X    = f_factor * g / T
//         ktau = -a_nu / g
//     so that the intensity slope of bin c is  dI_c = -A / (exp(X nu_c) - 1)
//     and every tau slot has the same slope ktau. With j_nu = a_nu B_nu(T) and
//     nu = g nu_c this is the reference's -inv(g) j_nu exp(-tau) / nu^3 with
//     the nu^3 of the Planck function cancelled.
// Outside every emitter A = X = ktau = 0 and no metric, velocity or redshift
// is evaluated (the reference's slopes are exactly zero there too).
#pragma once

#include <cuda_runtime.h>
#include <cmath>
#include "rtw_internal.h"

#define RTW_HD __host__ __device__ __forceinline__

namespace rtw {

constexpr double kPi = 3.141592653589793;
constexpr double kNoDivZero = 1e-24;
constexpr double kLightC = 299792458.0;
// 64BitConstants.jl:22-25 (nu in nm^-1)
constexpr double kEmissionScale = 2 * 6.62607015e-34 * 299792458.0 * 1e27;
constexpr double kFFactor = 6.62607015e-34 * 299792458.0 * 1e9 / 1.380649e-23;

template <class R>
struct Emit {
    R A, X, ktau;
};

// FP32 stages use the MUFU forms (absolute error ~5e-7 on [0, pi]); within
// sin(theta) < promote_sin of a pole the mixed path runs FP64 stages.
// (Host versions exist only for the operation-count instantiation.)
RTW_HD void rsincos(float x, float* s, float* c) {
#ifdef __CUDA_ARCH__
    __sincosf(x, s, c);
#else
    *s = std::sin(x); *c = std::cos(x);
#endif
}
RTW_HD void rsincos(double x, double* s, double* c) {
#ifdef __CUDA_ARCH__
    sincos(x, s, c);
#else
    *s = std::sin(x); *c = std::cos(x);
#endif
}
RTW_HD float rsqrt_(float x) { return sqrtf(x); }
RTW_HD double rsqrt_(double x) { return sqrt(x); }
RTW_HD float rexp_(float x) {
#ifdef __CUDA_ARCH__
    return __expf(x);
#else
    return std::exp(x);
#endif
}
RTW_HD double rexp_(double x) { return exp(x); }
RTW_HD float rpow_(float x, float y) { return powf(x, y); }
RTW_HD double rpow_(double x, double y) { return pow(x, y); }
RTW_HD double rinv(double x) { return 1.0 / x; }
RTW_HD float rinv(float x) {
#ifdef __CUDA_ARCH__
    return __fdividef(1.0f, x);
#else
    return 1.0f / x;
#endif
}

// Blackbody grey emitter at redshift factor g with temperature T and
// absorption a_nu (calc_planck + calc_radiative_coefficients).
// exp(-tau) of a stage point. A stage that enters an absorber mid-step can
// carry a large negative stage tau (the tableau has negative coefficients);
// in FP32, exp(-tau) would overflow to inf and turn the embedded error into
// NaN, which the reference's controller accepts. The FP32 form saturates at
// exp(40) (so a_nu emission_scale exp(-tau) / g and the squared error stay
// finite in FP32): the slope stays huge, the error rejects the step, as the
// FP64 form does.
RTW_HD float attenuation(float tau) { return rexp_(fminf(-tau, 40.0f)); }
RTW_HD double attenuation(double tau) { return rexp_(-tau); }
template <class R>
RTW_HD R attenuation(R tau) { return rexp_(-tau); }

template <class R>
RTW_HD Emit<R> bb_emit(R a_nu, R T, R g, R tau) {
    Emit<R> e;
    const R ig = rinv(g);
    e.A = a_nu * R(kEmissionScale) * attenuation(tau) * ig;
    e.X = R(kFFactor) * g / T;
    e.ktau = -a_nu * ig;
    return e;
}

// ---------------------------------------------------------------------------
// Minkowski space, spherical coordinates; emitting sphere r <= r_out.
// Minkowski_Sphere_Spherical.source/source_geometry.jl:93-108, source_model.jl:60-117
// ---------------------------------------------------------------------------
struct MinkowskiSphere {
    template <class R>
    static RTW_HD void rhs(const DevScene& s, const R z[10], R k[9], Emit<R>& em) {
        const R r = z[1], kt = z[4], kr = z[5], kth = z[6], kph = z[7];
        R sn, cs;
        rsincos(z[2], &sn, &cs);
        const R ir = rinv(r + R(kNoDivZero));
        const R cot = cs * rinv(sn);
        k[0] = kt; k[1] = kr; k[2] = kth; k[3] = kph;
        k[4] = R(0);
        k[5] = r * kth * kth + r * sn * sn * kph * kph;
        k[6] = -R(2) * ir * kr * kth + sn * cs * kph * kph;
        k[7] = -R(2) * ir * kr * kph - R(2) * cot * kth * kph;
        if (r <= R(s.r_out)) {
            // u = (1,0,0,0), g_tt = -1: g = k^t
            em = bb_emit<R>(R(s.anu), R(s.T), kt, z[8]);
        } else {
            em.A = R(0); em.X = R(0); em.ktau = R(0);
        }
        k[8] = em.ktau;
    }
};

// ---------------------------------------------------------------------------
// Schwarzschild, Boyer-Lindquist; wedge disk, circular-orbit emitter.
// Schwarzschild_Simple_Disk_Spherical.source/source_geometry.jl:109-128,
// source_model.jl:57-133
// ---------------------------------------------------------------------------
struct SchwarzschildDisk {
    template <class R>
    static RTW_HD void rhs(const DevScene& s, const R z[10], R k[9], Emit<R>& em) {
        const R r = z[1], th = z[2], kt = z[4], kr = z[5], kth = z[6], kph = z[7];
        const R rs = R(s.rs);
        R sn, cs;
        rsincos(th, &sn, &cs);
        const R ir = rinv(r);
        // r - rs: FP64 stages form it from r as the reference does; FP32 stages
        // take z[9] = r - r_horizon, carried from the FP64 state without the
        // cancellation of subtracting two nearly equal FP32 numbers.
        const R rmrs = sizeof(R) == 4 ? z[9] : r - rs;
        const R q = rs * R(0.5) * ir * rinv(rmrs);  // rs / (2 r (r - rs))
        const R cot = cs * rinv(sn);
        k[0] = kt; k[1] = kr; k[2] = kth; k[3] = kph;
        k[4] = -R(2) * q * kt * kr;
        k[5] = -(rs * rmrs * R(0.5) * ir * ir * ir * kt * kt - q * kr * kr - rmrs * kth * kth -
                 rmrs * sn * sn * kph * kph);
        k[6] = -(R(2) * ir * kr * kth - sn * cs * kph * kph);
        k[7] = -(R(2) * ir * kr * kph + R(2) * cot * kth * kph);
        if (R(s.r_in) <= r && r <= R(s.r_out) && R(s.th_lo) <= th && th <= R(s.th_hi)) {
            const R M = R(s.M);
            const R ut = rinv(rsqrt_(R(1) - R(3) * M * ir));
            const R uph = ut * rsqrt_(M * ir * ir * ir);
            const R gtt = -(R(1) - rs * ir);
            const R gpp = (r * sn) * (r * sn);
            const R g = -(ut * gtt * kt + uph * gpp * kph);
            em = bb_emit<R>(R(s.anu), R(s.T), g, z[8]);
        } else {
            em.A = R(0); em.X = R(0); em.ktau = R(0);
        }
        k[8] = em.ktau;
    }
};

// ---------------------------------------------------------------------------
// Kerr, Boyer-Lindquist. Geodesic part: Kerr.source/source_geometry.jl:55-75,195-243.
// THICK = false: wedge disk with Keplerian emitter (Kerr.source/source_model.jl:57-137).
// THICK = true: thickened optically thin disk, alpha = a_nu rho, j = alpha B_nu(T),
//   rho = (r/r0)^rho_index exp(-z^2 / 2 (h r)^2), T = T0 (r/r0)^t_index,
//   r_in <= r <= r_out, the same Keplerian velocity of radius r.
// ---------------------------------------------------------------------------
template <bool THICK>
struct KerrScene {
    template <class R>
    static RTW_HD void rhs(const DevScene& s, const R z[10], R k[9], Emit<R>& em) {
        const R r = z[1], th = z[2], kt = z[4], kr = z[5], kth = z[6], kph = z[7];
        const R a = R(s.a), rs = R(s.rs);
        R sn, cs;
        rsincos(th, &sn, &cs);
        const R r2 = r * r, a2 = a * a, s2 = sn * sn;
        const R ac2 = a2 * cs * cs, as2 = a2 * s2;  // a^2 cos^2, a^2 sin^2
        const R Sig = r2 + ac2;
        // Delta = r^2 - rs r + a^2 = (r - r+)(r - r-). FP32 stages use the
        // factored form with z[9] = r - r+ carried from the FP64 state, which
        // stays accurate down to the horizon stop (1 + 10 tol) r+.
        const R Del = sizeof(R) == 4 ? z[9] * (z[9] + R(s.r_pm)) : r2 - rs * r + a2;
        const R ra2 = r2 + a2;
        const R Aa = ra2 * Sig + rs * r * as2;
        const R iS = rinv(Sig), iD = rinv(Del), cot = cs * rinv(sn);
        const R iS2 = iS * iS;
        const R P = rs * iS2;             // rs / Sig^2
        const R Q = R(0.5) * P * iD;      // rs / (2 Sig^2 Del)
        const R iS3h = R(0.5) * iS2 * iS; // 1 / (2 Sig^3)
        const R sc = sn * cs;             // sin(2 theta) / 2
        const R dr = r2 - ac2;            // r^2 - a^2 cos^2
        // The 30 nonzero Christoffel symbols of Kerr.source/source_geometry.jl:203-240,
        // written around shared factors (Gamma^t_tr = Q (r^2+a^2) dr,
        // Gamma^phi_tr = Q a dr, Gamma^r_tphi = -a sin^2 Gamma^r_tt,
        // Gamma^theta_tt = Gamma^t_ttheta / Sig, Gamma^theta_thth = Gamma^r_rth,
        // Gamma^theta_rr = -Gamma^r_rth / Delta, ...).
        const R Gt_tth = -P * a2 * r * sc;
        const R Gt_thph = -Gt_tth * a * s2;
        const R Gt_rph = Q * a * s2 * (ac2 * (a2 - r2) - r2 * (a2 + R(3) * r2));
        const R Gp_tth = -P * a * r * cot;
        const R Gp_rph = r * iD + Q * (as2 * ac2 - r2 * (Sig + ra2));
        const R Gp_thph = cot * (R(1) + P * r * as2);
        const R Gr_tt = rs * Del * dr * iS3h;
        const R Gr_rth = -a2 * sc * iS;
        const R Gr_rr = (r * as2 - R(0.5) * rs * dr) * iS * iD;
        const R Gr_thth = -r * Del * iS;
        const R Gr_phph = Del * s2 * (rs * as2 * dr - R(2) * r * Sig * Sig) * iS3h;
        const R Gh_tt = Gt_tth * iS;
        const R Gh_tph = P * iS * a * r * ra2 * sc;
        const R Gh_rr = -Gr_rth * iD;
        const R Gh_rth = r * iS;
        const R Gh_phph = -R(2) * sc * (Aa * Sig + ra2 * rs * r * as2) * iS3h;
        const R Qdr_ktkr = Q * dr * kt * kr;

        k[0] = kt; k[1] = kr; k[2] = kth; k[3] = kph;
        k[4] = -R(2) * (Qdr_ktkr * ra2 + Gt_tth * kt * kth + Gt_rph * kr * kph + Gt_thph * kth * kph);
        k[5] = -(Gr_tt * (kt * kt - R(2) * a * s2 * kt * kph) + Gr_rr * kr * kr + R(2) * Gr_rth * kr * kth +
                 Gr_thth * kth * kth + Gr_phph * kph * kph);
        k[6] = -(Gh_tt * kt * kt + R(2) * Gh_tph * kt * kph + Gh_rr * kr * kr + R(2) * Gh_rth * kr * kth +
                 Gr_rth * kth * kth + Gh_phph * kph * kph);
        k[7] = -R(2) * (Qdr_ktkr * a + Gp_tth * kt * kth + Gp_rph * kr * kph + Gp_thph * kth * kph);

        bool fire;
        if (THICK)
            fire = R(s.r_in) <= r && r <= R(s.r_out);
        else
            fire = R(s.r_in) <= r && r <= R(s.r_out) && R(s.th_lo) <= th && th <= R(s.th_hi);
        if (fire) {
            // prograde circular orbit (Kerr.source/source_model.jl:110-120)
            const R sM = R(s.sqrtM), M = R(s.M);
            const R sr = rsqrt_(r);
            const R r32 = r * sr;
            const R Om = sM * rinv(r32 + a * sM);
            const R D = r32 - R(3) * M * sr + R(2) * a * sM;
            const R ut = (r32 + a * sM) * rinv(rsqrt_(r32) * rsqrt_(D));
            const R uph = ut * Om;
            // lower metric (source_geometry.jl:66-75)
            const R gtt = -(R(1) - rs * r * iS);
            const R gtp = -rs * a * r * s2 * iS;
            const R gpp = Aa * iS * s2;
            const R g = -(ut * (gtt * kt + gtp * kph) + uph * (gtp * kt + gpp * kph));
            R anu = R(s.anu), T = R(s.T);
            if (THICK) {
                const R x = r * rinv(R(s.rho_r0));
                const R zc = r * cs;
                const R hz = R(s.rho_h) * r;
                const R rho = rpow_(x, R(s.rho_idx)) * rexp_(-(zc * zc) * rinv(R(2) * hz * hz));
                anu = anu * rho;
                T = T * rpow_(x, R(s.t_idx));
            }
            em = bb_emit<R>(anu, T, g, z[8]);
        } else {
            em.A = R(0); em.X = R(0); em.ktau = R(0);
        }
        k[8] = em.ktau;
    }
};

template <int KIND> struct SceneOf;
template <> struct SceneOf<RTW_SCENE_MINKOWSKI_SPHERE> { typedef MinkowskiSphere type; };
template <> struct SceneOf<RTW_SCENE_SCHWARZSCHILD_DISK> { typedef SchwarzschildDisk type; };
template <> struct SceneOf<RTW_SCENE_KERR_DISK> { typedef KerrScene<false> type; };
template <> struct SceneOf<RTW_SCENE_KERR_THICK_DISK> { typedef KerrScene<true> type; };

// ---------------------------------------------------------------------------
// Per-step scene functions evaluated in FP64 on the accepted state.
// ---------------------------------------------------------------------------

// pad_max_dt: Kerr model :86-103 (scale cast to Float32), Schwarzschild :86-106
// (photon-sphere slowdown), Minkowski :89-105.
// CT: arithmetic of the step controller (double for the FP64 path, float for
// the mixed path; the bound only needs a few digits).
RTW_HD double cdiv(double a, double b) { return a / b; }
RTW_HD float cdiv(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fdividef(a, b);
#else
    return a / b;
#endif
}
RTW_HD float cabs(float a) { return fabsf(a); }
RTW_HD double cabs(double a) { return fabs(a); }
RTW_HD float cmin(float a, float b) { return fminf(a, b); }
RTW_HD double cmin(double a, double b) { return fmin(a, b); }
RTW_HD float cmax(float a, float b) { return fmaxf(a, b); }
RTW_HD double cmax(double a, double b) { return fmax(a, b); }

template <int KIND, class CT = double>
__device__ __forceinline__ double pad_max_dt(const DevScene& s, const double* xd, double scale_d) {
    constexpr bool kerr = KIND == RTW_SCENE_KERR_DISK || KIND == RTW_SCENE_KERR_THICK_DISK;
    CT scale = (CT)(kerr ? (double)(float)scale_d : scale_d);
    const CT vr = (CT)xd[5], vth = (CT)xd[6], vph = (CT)xd[7];
    const CT ndz = (CT)kNoDivZero;
    CT eps;
    if (xd[2] < kPi / 8 || xd[2] > 7 * kPi / 8)
        eps = cmin(scale, (CT)1e-1f);
    else if (KIND == RTW_SCENE_SCHWARZSCHILD_DISK && xd[1] <= 1.5 * (3 * s.M))
        eps = scale / CT(10);
    else
        eps = scale;
    CT first;
    if (kerr)
        first = cabs(cdiv(CT(1), cdiv(eps, cabs(vr)))) + ndz;
    else
        first = cabs(cdiv(CT(1), cdiv(eps, cabs(vr) + ndz))) + ndz;
    // distance to the nearer pole in FP64: in FP32, pi - theta is 0 within
    // 1.2e-7 of the pole, which would freeze a ray crossing the axis
    const CT pole = CT(fmin(xd[2], kPi - xd[2]));
    const CT second = cabs(cdiv(CT(1), cdiv(eps * pole, cabs(vth) + ndz) + ndz));
    const CT third = cabs(cdiv(CT(1), cdiv(eps, cabs(vph) + ndz) + ndz));
    CT m = cmin(cdiv(CT(1), first + second + third + ndz), (CT)0.5);
    return (double)cmax(m, (CT)1e-12f);
}

// near_singularity: Kerr :249-269 (= Schwarzschild :134-154), Minkowski :114-132.
template <int KIND>
__device__ __forceinline__ bool near_singularity(const double* x, double h, double tol, double* temp) {
    const double th_new = x[2] + h * x[6];
    const double r_new = x[1] + h * x[5];
    double lim = tol;
    if (KIND == RTW_SCENE_MINKOWSKI_SPHERE) lim = 10 * tol / fabs(r_new + kNoDivZero);
    if (fabs(th_new) <= lim) {
        *temp = 2 * fabs(x[2]) / (fabs(x[6] * 37) + kNoDivZero);
        return true;
    }
    if (fabs(th_new - kPi) <= lim) {
        *temp = 2 * fabs((x[2] - kPi) / (fabs(x[6] * 37) + kNoDivZero));
        return true;
    }
    if (KIND == RTW_SCENE_MINKOWSKI_SPHERE && fabs(r_new) <= 100 * tol) {
        *temp = 2 * tol / (fabs(x[5] * 37) + kNoDivZero);
        return true;
    }
    return false;
}

__device__ __forceinline__ double jl_mod(double x, double y) {
    double r = fmod(x, y);
    if (r != 0 && ((r < 0) != (y < 0))) r += y;
    return r;
}

// keepinbounds!: Kerr :275-301, Minkowski :138-163 (adds the r <= 0 reflection).
template <int KIND>
__device__ __forceinline__ void keep_in_bounds(double* x) {
    if (KIND == RTW_SCENE_MINKOWSKI_SPHERE && x[1] <= 0) {
        x[1] = -x[1] + kNoDivZero;
        x[5] = -x[5];
        x[2] -= kPi;
        x[6] = -x[6];
    }
    if (x[2] < 0) {
        x[2] = -x[2];
        x[3] -= kPi;
        x[6] = -x[6];
    }
    // mod(theta, 2 pi) is the identity on [0, 2 pi)
    if (!(x[2] < 2 * kPi)) x[2] = jl_mod(x[2], 2 * kPi);
    if (x[2] >= kPi) {
        x[2] = 2 * kPi - x[2];
        x[3] += kPi;
        x[6] = -x[6];
    }
}

// calc_terminate without the step-count predicate (the polar escape calls it
// with max_steps = 2, step_count = 1). tau is the common value of all tau slots.
template <int KIND>
__device__ __forceinline__ int terminate_geo(const DevScene& s, const double* x, double r_term, double thick) {
    if (x[1] > s.esc) return RTW_CLASS_ESCAPE;
    if (KIND != RTW_SCENE_MINKOWSKI_SPHERE && x[1] <= r_term) return RTW_CLASS_HORIZON;
    if (x[3] > s.wind) return RTW_CLASS_WINDING;
    if (x[8] >= thick) return RTW_CLASS_THICK;
    return 0;
}

}  // namespace rtw
