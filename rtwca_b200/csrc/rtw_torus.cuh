// rtw_torus.cuh - the thermal synchrotron torus emitter (a new .source
// emitter behind the reference's RT slot contract, integrators_LttM.jl:33-42:
// slope[I_c] = -inv(g) j_nu exp(-tau_c) / nu^3, slope[tau_c] = -inv(g) a_nu,
// nu = g nu_c the source-frame frequency in nm^-1), written once over a
// generic scalar T so that the forward kernels run it as float or double and
// the adjoint as dual numbers. Also the Kerr geodesic acceleration in a
// generic form for the adjoint (from metric derivatives; the forward kernels
// use the scene functor of rtw_scenes.cuh for the same quantity).
#pragma once

#include "rtw_dual.cuh"
#include "rtw_scenes.cuh"

namespace rtw {

constexpr int kTorusMaxBins = 32;
constexpr int kTorusParams = 5;  // a, inclination, n_e0, b_0, theta_e0

// Torus constants (FP64 on the host; the kernels cast what they need).
struct TorusDev {
    double M, a;
    double r_in, r_out, edge_in, edge_out, cut_in, cut_out;
    double h_ratio, ne_idx, b_idx, t_idx;
    double n0, B0, Th0;
    double cj_unit;  // sqrt(2) pi e^2 / (3 c) * length_cm (cgs)
    double nuc_unit; // e / (2 pi m_e c): cyclotron frequency per gauss, Hz
};

// Per-bin constants of the observed frequency nu_c.
struct TorusBin {
    double nu_nm;       // nu_c in nm^-1
    double nu_hz;       // nu_c in Hz
    double inv_nu_nm3;  // 1 / (nu_c in nm^-1)^3
    double b0;          // 2 h nu_c^3 / c^2 (cgs)
    double hk;          // h nu_c / (m_e c^2)
    double fx, fy, fz;  // nu^3 c / lambda^2 * CIE trapezoid weights (XYZ epilogue)
    double ln_nu;       // log(nu_c in Hz)
    double inv_b0;      // 1 / b0
    double nu16;        // (nu_c in Hz)^(1/6)
};

// Emitter numbers at a point, shared by every bin: j_nu = cj nus F(nu / nus)
// (per map unit), nus = (2/9) nu_cyc Theta^2 sin(theta_B), Theta = kT_e / m_e
// c^2, g = -u.k. on = false outside the emitter (every slope is then 0).
// The Powehi emitter (powehi_point) uses the same record with zone 1 (disk:
// cj = a_nu, nus = T) or zone 2 (jet: cj = J0, nus = A0, th = 1/(nu_c sin
// theta_B)).
template <class T>
struct TorusPt {
    T cj, nus, th, g;
    bool on;
    int zone;
};

// K_2(1/theta) by the trapezoid rule on K_2(x) = int_0^inf exp(-x cosh t)
// cosh 2t dt, step 1/4 up to t = 8 (relative error below 1e-13 for
// x in [0.04, 3]: the integrand decays double-exponentially).
__device__ __constant__ double c_k2_cosh[33] = {1.0, 1.0314130998795732, 1.1276259652063807, 1.2946832846768448, 1.5430806348152437, 1.8884238771610158, 2.352409615243247, 2.9641883097280877, 3.7621956910836314, 4.796567530460195, 6.132289479663686, 7.853279872697439, 10.067661995777765, 12.914557062512392, 16.572824671057315, 21.272299872959398, 27.308232836016487, 35.05983829029843, 45.014120148530026, 57.79646811119539, 74.20994852478785, 95.28575798851459, 122.34800951782942, 157.09692153324536, 201.7156361224559, 259.00737756123914, 332.5715682417774, 427.02996670288616, 548.3170351552121, 704.0527791895422, 904.0214837702167, 1160.7864226767986, 1490.479161252178};
__device__ __constant__ double c_k2_cosh2[33] = {1.0, 1.1276259652063807, 1.5430806348152437, 2.352409615243247, 3.7621956910836314, 6.132289479663686, 10.067661995777765, 16.572824671057315, 27.308232836016487, 45.014120148530026, 74.20994852478785, 122.34800951782942, 201.7156361224559, 332.5715682417774, 548.3170351552121, 904.0214837702167, 1490.479161252178, 2457.384521883752, 4051.542025492594, 6679.863452256851, 11013.232920103323, 18157.751350891544, 29937.07086594976, 49357.885510445296, 81377.39571257407, 134168.64326230055, 221206.6960055904, 364708.18492453615, 601302.1420828041, 991379.6317690365, 1634508.6862362083, 2694849.238141599, 4443055.260253993};
static const double h_k2_cosh[33] = {1.0, 1.0314130998795732, 1.1276259652063807, 1.2946832846768448, 1.5430806348152437, 1.8884238771610158, 2.352409615243247, 2.9641883097280877, 3.7621956910836314, 4.796567530460195, 6.132289479663686, 7.853279872697439, 10.067661995777765, 12.914557062512392, 16.572824671057315, 21.272299872959398, 27.308232836016487, 35.05983829029843, 45.014120148530026, 57.79646811119539, 74.20994852478785, 95.28575798851459, 122.34800951782942, 157.09692153324536, 201.7156361224559, 259.00737756123914, 332.5715682417774, 427.02996670288616, 548.3170351552121, 704.0527791895422, 904.0214837702167, 1160.7864226767986, 1490.479161252178};
static const double h_k2_cosh2[33] = {1.0, 1.1276259652063807, 1.5430806348152437, 2.352409615243247, 3.7621956910836314, 6.132289479663686, 10.067661995777765, 16.572824671057315, 27.308232836016487, 45.014120148530026, 74.20994852478785, 122.34800951782942, 201.7156361224559, 332.5715682417774, 548.3170351552121, 904.0214837702167, 1490.479161252178, 2457.384521883752, 4051.542025492594, 6679.863452256851, 11013.232920103323, 18157.751350891544, 29937.07086594976, 49357.885510445296, 81377.39571257407, 134168.64326230055, 221206.6960055904, 364708.18492453615, 601302.1420828041, 991379.6317690365, 1634508.6862362083, 2694849.238141599, 4443055.260253993};

// The FP32 paths' rule: step 0.4 up to t = 7.6 (20 points; relative error
// below 2e-8 for x in [0.02, 3], under FP32's rounding), cosh(0.4 i) and
// cosh(0.8 i).
__device__ __constant__ double c_k2f_cosh[20] = {1.0, 1.0810723718384547, 1.3374349463048447, 1.8106555673243752, 2.5774644711948853, 3.7621956910836314, 5.556947166965509, 8.252728416861135, 12.28664620054386, 18.31277908306264, 27.308232836016487, 40.73157300243561, 60.75932363289199, 90.63887921978599, 135.21505264493462, 201.7156361224559, 300.9233497146777, 448.9242027127831, 669.7157554901132, 999.0981977777762};
__device__ __constant__ double c_k2f_cosh2[20] = {1.0, 1.3374349463048447, 2.5774644711948853, 5.556947166965509, 12.28664620054386, 27.308232836016487, 60.75932363289199, 135.21505264493462, 300.9233497146777, 669.7157554901132, 1490.479161252178, 3317.1220785054825, 7382.3908166530155, 16429.812852437903, 36565.22092354488, 81377.39571257407, 181108.72480700444, 403064.87956261594, 897037.3863033862, 1996393.417605601};
static const double h_k2f_cosh[20] = {1.0, 1.0810723718384547, 1.3374349463048447, 1.8106555673243752, 2.5774644711948853, 3.7621956910836314, 5.556947166965509, 8.252728416861135, 12.28664620054386, 18.31277908306264, 27.308232836016487, 40.73157300243561, 60.75932363289199, 90.63887921978599, 135.21505264493462, 201.7156361224559, 300.9233497146777, 448.9242027127831, 669.7157554901132, 999.0981977777762};
static const double h_k2f_cosh2[20] = {1.0, 1.3374349463048447, 2.5774644711948853, 5.556947166965509, 12.28664620054386, 27.308232836016487, 60.75932363289199, 135.21505264493462, 300.9233497146777, 669.7157554901132, 1490.479161252178, 3317.1220785054825, 7382.3908166530155, 16429.812852437903, 36565.22092354488, 81377.39571257407, 181108.72480700444, 403064.87956261594, 897037.3863033862, 1996393.417605601};

template <class T>
RTW_HD T bessel_k2_inv(const T& theta) {
    if constexpr (sizeof(decltype(val(theta))) == 4) {
        const T x = T(1.0) / theta;
        T s = T(0.0);
        for (int i = 0; i < 20; ++i) {
#ifdef __CUDA_ARCH__
            const double ch = c_k2f_cosh[i], ch2 = c_k2f_cosh2[i];
#else
            const double ch = h_k2f_cosh[i], ch2 = h_k2f_cosh2[i];
#endif
            const double w = i == 0 ? 0.2 : 0.4;
            s = s + texp(x * decltype(val(x))(-ch)) * decltype(val(x))(w * ch2);
        }
        return s;
    }
    const T x = T(1.0) / theta;
    T s = T(0.0);
    for (int i = 0; i < 33; ++i) {
#ifdef __CUDA_ARCH__
        const double ch = c_k2_cosh[i], ch2 = c_k2_cosh2[i];
#else
        const double ch = h_k2_cosh[i], ch2 = h_k2_cosh2[i];
#endif
        const double w = i == 0 ? 0.125 : 0.25;
        s = s + texp(x * decltype(val(x))(-ch)) * decltype(val(x))(w * ch2);
    }
    return s;
}

// Dual argument: the value and dK_2/dx as two plain trapezoid sums, then one
// chain-rule step (dK_2(x)/dx = -int cosh t cosh 2t exp(-x cosh t) dt).
template <class T, int K>
RTW_HD Dual<T, K> bessel_k2_inv(const Dual<T, K>& theta) {
    // (in the tangents' precision T: FP32 for the FP32-mixed adjoint's
    // emitter tangents, FP64 otherwise)
    const T x = T(1.0) / theta.v;
    T s = T(0), ds = T(0);
    if constexpr (sizeof(T) == 4) {
        for (int i = 0; i < 20; ++i) {
#ifdef __CUDA_ARCH__
            const double ch = c_k2f_cosh[i], ch2 = c_k2f_cosh2[i];
#else
            const double ch = h_k2f_cosh[i], ch2 = h_k2f_cosh2[i];
#endif
            const T w = T((i == 0 ? 0.2 : 0.4) * ch2) * texp(-x * T(ch));
            s += w;
            ds -= w * T(ch);
        }
        return chain(theta, s, ds * (-x * x));
    }
    for (int i = 0; i < 33; ++i) {
#ifdef __CUDA_ARCH__
        const double ch = c_k2_cosh[i], ch2 = c_k2_cosh2[i];
#else
        const double ch = h_k2_cosh[i], ch2 = h_k2_cosh2[i];
#endif
        const T w = T((i == 0 ? 0.125 : 0.25) * ch2) * texp(-x * T(ch));
        s += w;
        ds -= w * T(ch);
    }
    // d/dtheta = dK/dx * (-1 / theta^2)
    return chain(theta, s, ds * (-x * x));
}

// Emitter numbers at (r, theta) for a ray with k^t, k^phi (the Keplerian
// 4-velocity and the toroidal field have only t and phi components, so k^r
// and k^theta do not enter). a, n0, b0, th0 are the differentiable parameters.
template <class T>
RTW_HD TorusPt<T> torus_point(const TorusDev& P, const T& a, const T& n0, const T& b0, const T& th0, const T& r,
                              const T& th, const T& kt, const T& kph) {
    typedef decltype(val(r)) B;  // float or double
    TorusPt<T> o;
    o.on = false;
    o.zone = 0;
    o.cj = T(0.0); o.nus = T(0.0); o.th = T(1.0); o.g = T(1.0);
    const double rv = (double)val(r);
    if (!(rv >= P.cut_in && rv <= P.cut_out)) return o;
    const T x = r * B(1.0 / P.r_in);
    T taper = T(1.0);
    if (rv < P.r_in) {
        const T q = (T(B(P.r_in)) - r) * B(1.0 / P.edge_in);
        taper = texp(-(q * q));
    } else if (rv > P.r_out) {
        const T q = (r - B(P.r_out)) * B(1.0 / P.edge_out);
        taper = texp(-(q * q));
    }
    const T sn = tsin(th), cs = tcos(th);
    const T lx = tlog(x);
    // n_e with the Gaussian in z = r cos(theta) of width h_ratio r
    const T gz = cs * cs * B(-0.5 / (P.h_ratio * P.h_ratio));
    const T ne = n0 * texp(lx * B(P.ne_idx) + gz) * taper;
    const T bf = b0 * texp(lx * B(P.b_idx));
    const T tht = th0 * texp(lx * B(P.t_idx));
    // Kerr metric (Boyer-Lindquist), t-phi block
    const B M = B(P.M);
    const T r2 = r * r, a2 = a * a, s2 = sn * sn;
    const T Sig = r2 + a2 * cs * cs;
    const T f = B(2.0) * M * r / Sig;  // 2 M r / Sigma
    const T gtt = f - B(1.0);
    const T gtp = -(f * a * s2);
    const T gpp = (r2 + a2 + f * a2 * s2) * s2;
    // prograde Keplerian angular velocity at r, normalised 4-velocity
    const B sM = B(sqrt(P.M));
    const T Om = T(sM) / (r * tsqrt(r) + a * sM);
    const T n2 = -(gtt + B(2.0) * Om * gtp + Om * Om * gpp);
    if (!(val(n2) > 0)) return o;
    const T ut = T(1.0) / tsqrt(n2);
    const T u_t = ut * (gtt + Om * gtp);
    const T u_p = ut * (gtp + Om * gpp);
    const T g = -(u_t * kt + u_p * kph);
    // toroidal field along the projection of d/dphi orthogonal to u:
    // b = d_phi + u_phi u, b.b = g_phph + u_phi^2, b.k = k_phi - u_phi g
    const T kph_low = gtp * kt + gpp * kph;
    const T bb = gpp + u_p * u_p;
    const T bk = kph_low - u_p * g;
    if (!(val(bb) > 0) || !(val(g) > 0)) return o;
    const T cth2 = bk * bk / (bb * g * g);
    const double s2v = 1.0 - (double)val(cth2);
    if (!(s2v > 1e-12)) return o;
    const T sinb = tsqrt(T(1.0) - cth2);
    o.nus = bf * tht * tht * sinb * B(2.0 / 9.0 * P.nuc_unit);
    o.cj = ne * B(P.cj_unit) / bessel_k2_inv(tht);
    o.th = tht;
    o.g = g;
    o.on = true;
    return o;
}

// Intensity and optical-depth slopes of one bin without the exp(-tau) factor:
// slope[tau] = ft, slope[I] = fi exp(-tau). Thermal synchrotron fit of Leung,
// Gammie & Noble 2011 (ApJ 737, 21):
//   j_nu = n_e sqrt(2) pi e^2 nus / (3 K_2(1/Theta) c)
//          (X^1/2 + 2^(11/12) X^1/6)^2 exp(-X^1/3),   X = nu / nus,
// alpha_nu = j_nu / B_nu(T_e) (Kirchhoff), B_nu = 2 h nu^3 / c^2 / expm1(h nu / kT).
template <class T>
RTW_HD void torus_bin(const T& cj, const T& nus, const T& th, const T& g, const TorusBin& bn, T& ft, T& fi) {
    typedef decltype(val(g)) B;
    const T nu = g * B(bn.nu_hz);
    const T X = nu / nus;
    const double xv = (double)val(X);
    if (!(xv > 0) || xv > 2.0e5) {  // exp(-X^1/3) < 1e-25: no emission
        ft = T(0.0);
        fi = T(0.0);
        return;
    }
    const T lx = tlog(X);
    const T x12 = texp(lx * B(0.5));
    const T x16 = texp(lx * B(1.0 / 6.0));
    const T x13 = texp(lx * B(1.0 / 3.0));
    const T p = x12 + x16 * B(1.8877486253633868);  // 2^(11/12)
    const T j = cj * nus * p * p * texp(-x13);
    const T g2 = g * g;
    const T g4 = g2 * g2;
    // -inv(g) j / nu^3 with nu = g nu_c in nm^-1
    fi = -(j * B(bn.inv_nu_nm3) / g4);
    // -inv(g) alpha, alpha = j expm1(h nu / k T) / (2 h nu^3 / c^2)
    const T em1 = texpm1(g * B(bn.hk) / th);
    ft = -(j * em1 / (g4 * B(bn.b0)));
}

// exp and expm1 in the arithmetic of the bins' slopes and partials: FP64, or
// FP32 with the hardware exponential (the FP32-mixed forward and adjoint)
template <class T>
struct BinMath;
template <>
struct BinMath<double> {
    static RTW_HD double ex(double x) { return exp(x); }
    static RTW_HD double em1(double x) { return expm1(x); }
};
template <>
struct BinMath<float> {
#ifdef __CUDA_ARCH__
    static __device__ float ex(float x) { return __expf(x); }
#else
    static float ex(float x) { return std::exp(x); }
#endif
    static RTW_HD float em1(float x) { return expm1f(x); }
};

// torus_bin in two parts, for the FP32-mixed forward. Per stage point, the
// bin-independent factors replace the emitter numbers in place:
//   (cj, nus, th, g) -> (cj nus, (g / nus)^(1/6), g / th, 1 / g^4),
// so that per bin X^(1/6) = (g nu_c / nus)^(1/6) = (g / nus)^(1/6) nu_c^(1/6)
// is one multiply, X^(1/3) and X^(1/2) its square and cube, and the bin
// spends one exponential (exp(-X^(1/3))). expm1(h nu / k T) is its Taylor
// polynomial to the fifth power below 1e-2 (relative error < 2e-11; the
// argument is 1e-9..1e-5 at 230 GHz over the torus), expm1 above.
template <class R>
RTW_HD void torus_bin_stage(TorusPt<R>& S) {
    const R r = S.g / S.nus;
    if (!(r > R(0))) {  // X <= 0 in every bin: no emission
        S.cj = S.nus = S.th = S.g = R(0);
        return;
    }
    const R g2 = S.g * S.g;
    const R cjnus = S.cj * S.nus;
    const R gt = S.g / S.th;
    S.nus = texp(tlog(r) * R(1.0 / 6.0));
    S.cj = cjnus;
    S.th = gt;
    S.g = R(1) / (g2 * g2);
}

template <class R>
RTW_HD void torus_bin_fast(const TorusPt<R>& S, const TorusBin& bn, R& ft, R& fi) {
    const R x16 = S.nus * R(bn.nu16);
    if (!(x16 <= R(7.647244913317299))) {  // X > 2e5 ((2e5)^(1/6)): exp(-X^1/3) < 1e-25, no emission
        ft = fi = R(0);
        return;
    }
    const R x13 = x16 * x16, x12 = x13 * x16;
    const R p = x12 + x16 * R(1.8877486253633868);  // 2^(11/12)
    const R j = S.cj * p * p * BinMath<R>::ex(-x13);
    fi = -(j * R(bn.inv_nu_nm3) * S.g);
    const R y = S.th * R(bn.hk);
    const R em1 = y < R(1e-2) ? y * (R(1) + y * (R(0.5) + y * (R(1.0 / 6.0) + y * (R(1.0 / 24.0) + y * R(1.0 / 120.0)))))
                              : texpm1(y);
    ft = -(j * (em1 * R(bn.inv_b0)) * S.g);  // em1 / b0 first: j em1 alone can fall below FP32's normal range
}

// ---------------------------------------------------------------------------
// The Powehi scene (Powehi.source, the reference's M87* model): Kerr a = 0.9
// with a blackbody wedge disk (zone 1) and a rotating conical jet (zone 2)
// radiating power-law synchrotron; source_model.jl:186-317.
// ---------------------------------------------------------------------------
struct PowehiDev {
    double M, a, r_ev, rs;
    double disk_r_in, disk_r_out, disk_th_lo, disk_th_hi, disk_a, disk_T;  // zone 1
    double r_nozzle, gamma_min, gamma_max, nozzle_acc, omega_jet;        // zone 2 geometry
    double jet_th_lo, jet_th_hi, axis_lo, axis_hi;                         // zone 2 polar limits
    double b_phi;        // global field component B^phi (gauss)
    double j_scale;      // ne_0 synch_em * (p-dependent constants): j = j_scale |b| sin Phi s^-(p-1)/2
    double a_scale;      // ne_0 synch_ab * (p-dependent constants): a = a_scale Phi / nu s^-(p+2)/2
    double p_index;      // electron power-law index p
    double inv_p_synch;  // 1 / Approx_P_synch(p)
};

// Emitter numbers at a stage point z = (t, r, theta, phi, k^t, k^r, k^theta,
// k^phi) (region_calc, get_source_velocity!, calc_freq_shift,
// calc_fluid_params!, transform_B_b, calc_b_angle; source_model.jl:60-317).
template <class T>
RTW_HD TorusPt<T> powehi_point(const PowehiDev& P, const T* z) {
    typedef decltype(val(z[1])) B;
    TorusPt<T> o;
    o.on = false;
    o.zone = 0;
    o.cj = T(0.0); o.nus = T(0.0); o.th = T(1.0); o.g = T(1.0);
    const double rv = (double)val(z[1]), thv = (double)val(z[2]);
    int zone = 3;
    if (P.disk_r_in <= rv && rv <= P.disk_r_out && P.disk_th_lo <= thv && thv <= P.disk_th_hi)
        zone = 1;
    else if (rv >= P.r_nozzle && !(P.jet_th_lo <= thv && thv <= P.jet_th_hi) && (P.axis_lo <= thv && thv <= P.axis_hi))
        zone = 2;
    if (zone == 3) return o;
    const T r = z[1], th = z[2], kt = z[4], kr = z[5], kth = z[6], kph = z[7];
    const B a = B(P.a), M = B(P.M);
    const T sn = tsin(th), cs = tcos(th);
    const T r2 = r * r, s2 = sn * sn;
    const T Sig = r2 + a * a * cs * cs;
    const T Del = r2 - B(2.0) * M * r + a * a;
    const T Aa = (r2 + a * a) * (r2 + a * a) - Del * a * a * s2;
    const T gtt = -(T(B(1.0)) - B(2.0) * M * r / Sig);
    const T gtp = -(B(2.0) * M * a * r * s2 / Sig);
    const T gpp = Aa / Sig * s2;
    const T grr = Sig / Del;
    const T ghh = Sig;
    T ut, ur = T(B(0.0)), up;
    if (zone == 1) {
        // prograde equatorial circular orbit
        const T sr = tsqrt(r);
        const T r32 = r * sr;
        const B sM = B(sqrt(P.M));
        const T Om = T(sM) / (r32 + a * sM);
        const T D = r32 - B(3.0) * M * sr + B(2.0) * a * sM;
        ut = (r32 + a * sM) / (tsqrt(r32) * tsqrt(D));
        up = ut * Om;
    } else {
        // rotating conical jet accelerating through the nozzle
        const T w = -(gtp / (gpp + B(kNoDivZero)));
        T Om = B(0.9) / (sn * r);
        if ((double)val(Om) > P.omega_jet) Om = T(B(P.omega_jet));
        const T inv_lapse = tsqrt(Aa / (Sig * Del));
        T acc = (r - B(P.r_nozzle)) * B(P.nozzle_acc);
        if ((double)val(acc) > P.gamma_max) acc = T(B(P.gamma_max));
        const T G = acc + B(P.gamma_min);
        ut = G * inv_lapse;
        const T dw = Om - w;
        const T ur2 = (G * G - B(1.0) - gpp * ut * ut * dw * dw) / grr;
        if (!((double)val(ur2) > 0)) return o;  // the reference's sqrt of a negative: no emitter here
        ur = tsqrt(ur2);
        up = ut * Om;
    }
    const T u_t = gtt * ut + gtp * up, u_r = grr * ur, u_p = gtp * ut + gpp * up;
    const T g = -(u_t * kt + u_r * kr + u_p * kph);
    o.g = g;
    if (zone == 1) {
        o.cj = T(B(P.disk_a));
        o.nus = T(B(P.disk_T));
        o.zone = 1;
        o.on = true;
        return o;
    }
    // field: global B = (0, 0, B^phi) into the fluid frame (transform_B_b),
    // with the reference's magnitude sum_mu (sum_i g_{i mu}) b_mu^2
    const T b1 = u_p * B(P.b_phi);
    const T b2 = b1 * ur / ut;
    const T b4 = (T(B(P.b_phi)) + b1 * up) / ut;
    T bmag2 = (gtt + gtp) * b1 * b1 + grr * b2 * b2 + (gtp + gpp) * b4 * b4;
    if ((double)val(bmag2) < 1e-12) bmag2 = T(B(1e-12));
    // cos^2 of the field-ray angle (calc_b_angle) + no_div_zero
    const T bk = b1 * (gtt * kt + gtp * kph) + b2 * (grr * kr) + b4 * (gtp * kt + gpp * kph);
    T c2 = bk * bk / (bmag2 * g * g);
    if ((double)val(c2) > 1.0) c2 = T(B(1.0));
    c2 = c2 + B(kNoDivZero);
    T s2b = T(B(1.0)) - c2;
    if ((double)val(s2b) < 1e-12) s2b = T(B(1e-12));
    const T sinb = tsqrt(s2b);
    const T bmag = tsqrt(bmag2);
    const T nuc = bmag * B(9.34e-11);  // cyclotron frequency, nm^-1
    // anisotropy Phi = (1 - 0.99 cos^2)^(-p/2) / Approx_P_synch(p)
    const T phi = texp(tlog(T(B(1.0)) - B(0.99) * c2) * B(-0.5 * P.p_index)) * B(P.inv_p_synch);
    o.cj = bmag * sinb * phi * B(P.j_scale);  // J0
    o.nus = phi * B(P.a_scale);               // A0
    o.th = T(B(1.0)) / (nuc * sinb);           // 1 / (nu_c sin theta_B)
    o.zone = 2;
    o.on = true;
    return o;
}

// ---------------------------------------------------------------------------
// Synchro_Test.source, the reference's flat-space synchrotron test: Cartesian
// Minkowski space, a static cylinder around the z axis in a uniform field
// B^z radiating the power-law synchrotron of the Powehi jet
// (source_model.jl:18-244). Its emitter numbers use the Powehi zone-2 record,
// so powehi_bin gives its slopes.
// ---------------------------------------------------------------------------
struct SynchroDev {
    double b_z;          // global field B^z, gauss
    double r_cyl;        // cylinder radius (map units)
    double j_scale, a_scale, p_index, inv_p_synch;  // as PowehiDev
};

// Emitter numbers at a stage point z = (t, x, y, z, k^t, k^x, k^y, k^z)
// (is_fire :229-236, get_source_velocity! :250-256, calc_freq_shift,
// calc_fluid_params! :152-172, transform_B_b :60-108, calc_b_angle :114-146).
// With u = (1, 0, 0, 0) and g = diag(-1, 1, 1, 1): the frequency shift is
// k^t, the fluid-frame field b = (0, 0, 0, B^z) with the reference's
// magnitude sum_mu (sum_i g_{i mu}) b_mu^2 = B^z^2, and cos^2 of the
// field-ray angle (k^z / k^t)^2.
template <class T>
RTW_HD TorusPt<T> synchro_point(const SynchroDev& Y, const T* z) {
    typedef decltype(val(z[1])) B;
    TorusPt<T> o;
    o.on = false;
    o.zone = 0;
    o.cj = T(0.0); o.nus = T(0.0); o.th = T(1.0); o.g = T(1.0);
    const double xv = (double)val(z[1]), yv = (double)val(z[2]);
    if (!(sqrt(xv * xv + yv * yv) <= Y.r_cyl)) return o;
    const T g = z[4];
    o.g = g;
    const T c2 = z[7] * z[7] / (g * g);
    const T s2b = T(B(1.0)) - c2;
    // a ray along the field: the reference's j is 0 * inf there
    if (!((double)val(s2b) > 0)) return o;
    const T sinb = tsqrt(s2b);
    const B bmag = B(fabs(Y.b_z));
    const T phi = texp(tlog(T(B(1.0)) - B(0.99) * c2) * B(-0.5 * Y.p_index)) * B(Y.inv_p_synch);
    o.cj = sinb * phi * B(Y.j_scale * fabs(Y.b_z));   // J0
    o.nus = phi * B(Y.a_scale);                        // A0
    o.th = T(B(1.0)) / (sinb * B(9.34e-11) * bmag);    // 1 / (nu_c sin theta_B)
    o.zone = 2;
    o.on = true;
    return o;
}

// ---------------------------------------------------------------------------
// Wormhole.source, the reference's Dneg wormhole (Interstellar's): coordinates
// (t, l, theta, phi), metric -dt^2 + dl^2 + r(l)^2 dOmega^2, throat radius rho,
// half-length a, lensing width W = M W_over_M (source_geometry.jl:7-150). No
// emitter anywhere (source_model.jl:54-86).
// ---------------------------------------------------------------------------
struct WormholeDev {
    double rho, a_wh, M;  // throat radius, half-length, lensing mass parameter
};

// r(l) (source_geometry.jl:22-31)
template <class T>
RTW_HD T wormhole_r(const WormholeDev& W, const T& l) {
    typedef decltype(val(l)) B;
    const double lv = (double)val(l);
    if (!(fabs(lv) > W.a_wh)) return T(B(W.rho));
    const T al = lv < 0 ? T(B(0)) - l : l;
    const T x = (al - B(W.a_wh)) * B(2.0 / (kPi * W.M));
    return T(B(W.rho)) + B(W.M) * (x * tatan(x) - tlog(T(B(1)) + x * x) * B(0.5));
}

// dr/dl as the reference writes it (source_geometry.jl:34-41): 2 sign(l)
// (atan x + (x - 1) / (1 + x^2)) / pi. (The derivative of its r(l) is
// 2 sign(l) atan(x) / pi; the extra term is the reference's, kept for parity.)
template <class T>
RTW_HD T wormhole_drdl(const WormholeDev& W, const T& l) {
    typedef decltype(val(l)) B;
    const double lv = (double)val(l);
    if (!(fabs(lv) > W.a_wh)) return T(B(0));
    const T al = lv < 0 ? T(B(0)) - l : l;
    const T x = (al - B(W.a_wh)) * B(2.0 / (kPi * W.M));
    const T d = (tatan(x) + (x - B(1)) / (T(B(1)) + x * x)) * B(2.0 / kPi);
    return lv < 0 ? T(B(0)) - d : d;
}

// the geodesic right-hand side from the Christoffel symbols of
// calc_christoffel_udd! (source_geometry.jl:131-150): z = (t, l, theta, phi,
// k^t, k^l, k^theta, k^phi)
template <class T>
RTW_HD void wormhole_rhs(const WormholeDev& W, const T* z, T* k) {
    typedef decltype(val(z[1])) B;
    const T r = wormhole_r<T>(W, z[1]), rp = wormhole_drdl<T>(W, z[1]);
    const T sn = tsin(z[2]), cs = tcos(z[2]);
    const T kl = z[5], kth = z[6], kph = z[7];
    const T rpr = rp / r;
    for (int i = 0; i < 4; ++i) k[i] = z[4 + i];
    k[4] = T(B(0));
    k[5] = r * rp * kth * kth + r * rp * sn * sn * kph * kph;
    k[6] = B(-2) * rpr * kl * kth + sn * cs * kph * kph;
    k[7] = B(-2) * rpr * kl * kph - B(2) * (cs / sn) * kth * kph;
}

// ---------------------------------------------------------------------------
// Minkowski_Sphere_Cartesian.source: flat space in Cartesian (t, x, y, z) and
// a static blackbody sphere of radius 1 centred on the origin (is_fire
// :82-90), T = 5778 K (calc_fluid_params! :51-55), a_nu = 1 / map_scale and
// j_nu = a_nu calc_planck(T, nu) (calc_radiative_coefficients :66-77), at
// rest (get_source_velocity! :138-145): the frequency shift is k^t.
// ---------------------------------------------------------------------------
struct SphereDev {
    double r_sph;   // radius (map units)
    double a_nu;    // absorption coefficient (1 / map unit)
    double es;      // emission_scale
    double ff_T;    // f_factor / T (nm)
};

template <class T>
RTW_HD TorusPt<T> sphere_point(const SphereDev& S, const T* z) {
    TorusPt<T> o;
    o.on = false;
    o.zone = 0;
    o.cj = T(0.0); o.nus = T(0.0); o.th = T(1.0); o.g = T(1.0);
    const double xv = (double)val(z[1]), yv = (double)val(z[2]), zv = (double)val(z[3]);
    if (!(sqrt(xv * xv + yv * yv + zv * zv) <= S.r_sph)) return o;
    o.g = z[4];
    o.zone = 1;
    o.on = true;
    return o;
}

// Slopes of bin c without exp(-tau), nu = g nu_c (nm^-1): tau' = -a / g and
// I' = -(a / g) emission_scale / (exp(f_factor nu / T) - 1) (calc_planck :26-29
// over nu^3, calc_ray_derivative! integrators_LttM.jl:37-42)
template <class T>
RTW_HD void sphere_bin(const SphereDev& S, const TorusPt<T>& P, double nu_nm, T& ft, T& fi) {
    typedef decltype(val(P.g)) B;
    const T ag = T(B(S.a_nu)) / P.g;
    ft = -ag;
    fi = -(ag * B(S.es)) / (texp(P.g * B(S.ff_T * nu_nm)) - B(1.0));
}

// ---------------------------------------------------------------------------
// Thermal bremsstrahlung torus (RTW_SCENE_KERR_BREMS_TORUS): the synchrotron
// torus's fluid (n_e, Theta_e, tapers, Keplerian 4-velocity) radiating
// free-free emission with the van Hoof Gaunt factor of the reference's
// gaunt_ei_therm_van_Hoof (emission_functions.jl:54-78).
// ---------------------------------------------------------------------------
constexpr int kGauntRows = 146;  // constant log10 u: -16, -15.8, ...
constexpr int kGauntCols = 81;   // constant log10 gamma^2: -6, -5.8, ...
constexpr double kCYarCgs = 7.089314638783696e-44;  // emission_functions.jl:19

struct BremsDev {
    const float* lut;  // [kGauntRows][kGauntCols] row-major (device memory in the kernels)
    double cj_unit;    // C_Yar_cgs * length_cm
    double ry_mec2;    // Ry / (m_e c^2)
};

// IEEE single-precision steps without contraction (the reference's Float32
// arithmetic, which does not fuse a multiply and an add)
RTW_HD float f32_add(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}
RTW_HD float f32_mul(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
RTW_HD float f32_div(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fdiv_rn(a, b);
#else
    return a / b;
#endif
}

// gaunt_ei_therm_van_Hoof (emission_functions.jl:54-78) at log10 gamma^2 and
// log10 u (each already rounded to Float32, as Float32(log10(.)) there).
// Kept as the reference writes it: the fractional indices (log + 16) / 0.2 and
// (log + 6) / 0.2 address the 1-based table directly, so the lookup sits one
// grid step (0.2 dex) away from the table's own abscissae, and the upper
// index is ceil(frac + 1e-3), so just below an integer the two weights add up
// to 2. Outside the table, and for a non-finite argument (where the
// reference's floor(Int32, .) throws), the Gaunt factor is 1.2.
RTW_HD float gaunt_van_hoof(const float* lut, float loggam, float logu) {
    const float frac_i = f32_div(f32_add(logu, 16.0f), 0.2f);
    const float frac_j = f32_div(f32_add(loggam, 6.0f), 0.2f);
    if (!(frac_i >= 1.0f && frac_i < 200.0f && frac_j >= 1.0f && frac_j < 200.0f)) return 1.2f;
    const float fi = floorf(frac_i), ci = ceilf(f32_add(frac_i, 1e-3f));
    const float fj = floorf(frac_j), cj = ceilf(f32_add(frac_j, 1e-3f));
    if (!(ci <= (float)kGauntRows && cj <= (float)kGauntCols)) return 1.2f;
    const int i0 = (int)fi - 1, i1 = (int)ci - 1, j0 = (int)fj - 1, j1 = (int)cj - 1;
    const float wi0 = ci - frac_i, wi1 = frac_i - fi;  // exact: integers and frac_i are Float32
    const float g1 = f32_add(f32_mul(wi0, lut[i0 * kGauntCols + j0]), f32_mul(wi1, lut[i1 * kGauntCols + j0]));
    const float g2 = f32_add(f32_mul(wi0, lut[i0 * kGauntCols + j1]), f32_mul(wi1, lut[i1 * kGauntCols + j1]));
    return f32_add(f32_mul(cj - frac_j, g1), f32_mul(frac_j - fj, g2));
}
RTW_HD float rlog10f_(float x) { return log10f(x); }
RTW_HD float rlog10f_(double x) { return (float)log10(x); }

// The fluid at (r, theta) for a ray with k^t, k^phi: cj = C n_e^2 length_cm,
// th = Theta_e, g = -u.k (the synchrotron torus's profiles and 4-velocity).
template <class T>
RTW_HD TorusPt<T> brems_point(const TorusDev& P, const BremsDev& Bd, const T& a, const T& n0, const T& th0,
                              const T& r, const T& th, const T& kt, const T& kph) {
    typedef decltype(val(r)) B;
    TorusPt<T> o;
    o.on = false;
    o.zone = 0;
    o.cj = T(0.0); o.nus = T(1.0); o.th = T(1.0); o.g = T(1.0);
    const double rv = (double)val(r);
    if (!(rv >= P.cut_in && rv <= P.cut_out)) return o;
    const T x = r * B(1.0 / P.r_in);
    T taper = T(1.0);
    if (rv < P.r_in) {
        const T q = (T(B(P.r_in)) - r) * B(1.0 / P.edge_in);
        taper = texp(-(q * q));
    } else if (rv > P.r_out) {
        const T q = (r - B(P.r_out)) * B(1.0 / P.edge_out);
        taper = texp(-(q * q));
    }
    const T sn = tsin(th), cs = tcos(th);
    const T lx = tlog(x);
    const T gz = cs * cs * B(-0.5 / (P.h_ratio * P.h_ratio));
    const T ne = n0 * texp(lx * B(P.ne_idx) + gz) * taper;
    const T tht = th0 * texp(lx * B(P.t_idx));
    const B M = B(P.M);
    const T r2 = r * r, a2 = a * a, s2 = sn * sn;
    const T Sig = r2 + a2 * cs * cs;
    const T f = B(2.0) * M * r / Sig;
    const T gtt = f - B(1.0);
    const T gtp = -(f * a * s2);
    const T gpp = (r2 + a2 + f * a2 * s2) * s2;
    const B sM = B(sqrt(P.M));
    const T Om = T(sM) / (r * tsqrt(r) + a * sM);
    const T n2 = -(gtt + B(2.0) * Om * gtp + Om * Om * gpp);
    if (!(val(n2) > 0)) return o;
    const T ut = T(1.0) / tsqrt(n2);
    const T g = -(ut * (gtt + Om * gtp) * kt + ut * (gtp + Om * gpp) * kph);
    if (!(val(g) > 0)) return o;
    o.cj = ne * ne * B(Bd.cj_unit);
    o.th = tht;
    o.g = g;
    o.on = true;
    return o;
}

// Slopes of one bin without the exp(-tau) factor (slope[tau] = ft,
// slope[I] = fi exp(-tau)): j_nu = cj Theta^-1/2 exp(-u) g_ff(gamma^2, u),
// u = h nu / (Theta m_e c^2) with nu = g nu_c, gamma^2 = Ry / (Theta m_e c^2),
// alpha_nu = j_nu / B_nu(T_e) = j_nu expm1(u) / (2 h nu^3 / c^2).
template <class T>
RTW_HD void brems_bin(const BremsDev& Bd, const TorusPt<T>& S, const TorusBin& bn, T& ft, T& fi) {
    typedef decltype(val(S.g)) B;
    const T u = S.g * B(bn.hk) / S.th;
    if (!(val(u) > 0)) {
        ft = T(0.0);
        fi = T(0.0);
        return;
    }
    const T gam2 = T(B(Bd.ry_mec2)) / S.th;
    const float gff = gaunt_van_hoof(Bd.lut, rlog10f_(val(gam2)), rlog10f_(val(u)));
    const T j = S.cj / tsqrt(S.th) * texp(-u) * B(gff);
    const T g2 = S.g * S.g;
    const T g4 = g2 * g2;
    fi = -(j * B(bn.inv_nu_nm3) / g4);
    ft = -(j * texpm1(u) / (g4 * B(bn.b0)));
}

// Cube-map neighbours (cube_wrap, gen_geometry.jl:128-344). Texel (i, j) of
// face F, 1-based with n texels per face edge, moved by x texels along i and
// y along j. A move that leaves the face enters the face across that edge,
// re-oriented as the reference's table says; its formulas are kept as they
// are, so some moves land outside [1, n] (face 6's low i edge gives j = n - s)
// and, in cross-layout coordinates, on another region of the map, as there.
RTW_HD int sky_mod1(int s, int n) {
    int r = (s - 1) % n;
    if (r < 0) r += n;
    return r + 1;
}

RTW_HD void sky_move_i(int& i, int& j, int& F, int x, int n) {
    const int s = i + x;
    if (s >= 1 && s <= n) {
        i = s;
        return;
    }
    const bool hi = s > n;
    const int m = sky_mod1(s, n);
    switch (F) {
    case 1: i = m; F = hi ? 2 : 4; break;
    case 2: i = m; F = hi ? 3 : 1; break;
    case 3: i = m; F = hi ? 4 : 2; break;
    case 4: i = m; F = hi ? 1 : 3; break;
    case 5:
        if (hi) { i = n - j + 1; j = m; F = 3; }
        else { i = j; j = 1 - s; F = 1; }
        break;
    case 6:
        if (hi) { i = j; j = n - m + 1; F = 3; }
        else { i = n - j + 1; j = n - s; F = 1; }
        break;
    default: break;
    }
}

RTW_HD void sky_move_j(int& i, int& j, int& F, int y, int n) {
    const int t = j + y;
    if (t >= 1 && t <= n) {
        j = t;
        return;
    }
    const bool hi = t > n;
    const int m = sky_mod1(t, n);
    switch (F) {
    case 1:
        if (hi) { j = n + 1 - i; i = m; F = 6; }
        else { j = i; i = 1 - t; F = 5; }
        break;
    case 2: j = m; F = hi ? 6 : 5; break;
    case 3:
        if (hi) { j = i; i = n - m + 1; F = 6; }
        else { j = n - i + 1; i = n + t; F = 5; }
        break;
    case 4:
        i = n - i + 1;
        if (hi) { j = n - m + 1; F = 6; }
        else { j = 1 - t; F = 5; }
        break;
    case 5:
        if (hi) { j = m; F = 2; }
        else { i = n - i + 1; j = 1 - t; F = 4; }
        break;
    case 6:
        if (hi) { i = n - i + 1; j = n - m + 1; F = 4; }
        else { j = m; F = 2; }
        break;
    default: break;
    }
}

// A diagonal move is an i move, then a j move; on faces 5 and 6 an i move
// that leaves the face continues as an i move on the new face (by -y or +y).
RTW_HD void sky_wrap(int& i, int& j, int& F, int x, int y, int n) {
    if (x == 0 || y == 0) {
        if (x != 0) sky_move_i(i, j, F, x, n);
        else sky_move_j(i, j, F, y, n);
        return;
    }
    const int s = i + x, F0 = F;
    sky_move_i(i, j, F, x, n);
    if (F0 == 6 && s < 1) sky_move_i(i, j, F, -y, n);
    else if (F0 == 6 && s > n) sky_move_i(i, j, F, y, n);
    else if (F0 == 5 && s > n) sky_move_i(i, j, F, -y, n);
    else if (F0 == 5 && s < 1) sky_move_i(i, j, F, y, n);
    else sky_move_j(i, j, F, y, n);
}

// Face-local texel (i, j) of face F to cross-layout coordinates
// (cubemap_coord_calc, gen_geometry.jl:347-370): faces 1-4 in the middle row
// of four squares, 5 below face 2, 6 above it.
RTW_HD void sky_cross(int F, int n, int& i, int& j) {
    switch (F) {
    case 1: j += n; break;
    case 2: i += n; j += n; break;
    case 3: i += 2 * n; j += n; break;
    case 4: i += 3 * n; j += n; break;
    case 5: i += n; break;
    default: i += n; j += 2 * n; break;
    }
}

// Slopes of one bin without exp(-tau) (as torus_bin): nu = g nu_c in nm^-1.
// Disk: a = a_nu, j = a B_nu(T); jet: j = J0 s^-(p-1)/2, a = A0 / nu s^-(p+2)/2,
// s = nu / (nu_cyc sin theta_B) (calc_radiative_coefficients).
template <class T>
RTW_HD void powehi_bin(const PowehiDev& P, const TorusPt<T>& S, double nu_nm, T& ft, T& fi) {
    typedef decltype(val(S.g)) B;
    const T g = S.g;
    if (S.zone == 1) {
        const T x = g * B(kFFactor * nu_nm) / S.nus;
        ft = -(S.cj / g);
        fi = ft * B(kEmissionScale) / texpm1(x);
        return;
    }
    const T nu = g * B(nu_nm);
    const T ls = tlog(nu * S.th);
    const T j = S.cj * texp(ls * B(-0.5 * (P.p_index - 1.0)));
    const T an = S.nus / nu * texp(ls * B(-0.5 * (P.p_index + 2.0)));
    fi = -(j / (g * nu * nu * nu));
    ft = -(an / g);
}

// torus_bin in FP64 with its partial derivatives in (cj, nus, Theta, g), from
// the closed-form log-derivatives of the fit: with X = g nu_c / nus,
//   D_X = dln(P^2 e^{-X^1/3}) / dln X = (X^1/2 + 2^(11/12)/3 X^1/6) / P - X^1/3 / 3
//   D_y = dln expm1(y) / dln y = y e^y / expm1(y),   y = g hk / Theta
// ln|fi| = ln cj + ln nus + ln(P^2 e^..)(X) - 4 ln g + const,
// ln|ft| = ln|fi| + ln expm1(y) + const.
// The bin-independent part of torus_bin_grad at one emitter point: X = nu_c
// r with r = g / nus, so log X = log r + log nu_c; reciprocals shared by all
// bins.
struct TorusBinPre {
    double L, gt, cjnus, ig4, icj, inus, ig, ith;
    double e6;  // (g / nus)^(1/6) = exp(L / 6)
    bool ok;
};

RTW_HD TorusBinPre torus_bin_pre(double cj, double nus, double th, double g) {
    TorusBinPre q;
    const double r = g / nus;
    q.ok = r > 0;
    q.L = q.ok ? log(r) : 0.0;
    q.e6 = q.ok ? exp(q.L * (1.0 / 6.0)) : 0.0;
    q.gt = g / th;
    q.cjnus = cj * nus;
    const double g2 = g * g;
    q.ig4 = 1.0 / (g2 * g2);
    q.icj = 1.0 / cj;
    q.inus = 1.0 / nus;
    q.ig = 1.0 / g;
    q.ith = 1.0 / th;
    return q;
}

// The same in the bins' arithmetic BT: FP64 as above, or FP32 for the
// FP32-mixed adjoint, whose partials read these factors in FP32 (X^(1/6)'s
// stage factor then comes out as the forward's torus_bin_stage forms it).
template <class BT>
RTW_HD TorusBinPre torus_bin_pre_t(BT cj, BT nus, BT th, BT g) {
    if constexpr (sizeof(BT) == 8) {
        return torus_bin_pre(cj, nus, th, g);
    } else {
        TorusBinPre q;
        const BT r = g / nus;
        q.ok = r > BT(0);
        const BT L = q.ok ? tlog(r) : BT(0);
        q.L = L;
        q.e6 = q.ok ? (double)texp(L * BT(1.0 / 6.0)) : 0.0;
        q.gt = g / th;
        q.cjnus = cj * nus;
        const BT g2 = g * g;
        q.ig4 = BT(1) / (g2 * g2);
        q.icj = BT(1) / cj;
        q.inus = BT(1) / nus;
        q.ig = BT(1) / g;
        q.ith = BT(1) / th;
        return q;
    }
}


// torus_bin_grad from the shared part, in arithmetic T: the bin's slopes
// (ft, fi) and the two numbers their partials are linear in,
//   d ft / d(cj, nus, th, g) = ft (1/cj, (1 - DX)/nus, -Dy/th, (DX - 4 + Dy)/g),
//   d fi / d(cj, nus, th, g) = fi (1/cj, (1 - DX)/nus, 0, (DX - 4)/g),
// with DX = d log(P^2 exp(-X^1/3)) / d log X (P = X^1/2 + 2^(11/12) X^1/6, the
// emissivity's X dependence) and Dy = y e^y / expm1(y). FP64: X^1/6 by one
// exponential, X^1/3 and X^1/2 as its square and cube. FP32: the factorized
// form of torus_bin_fast (X^(1/6) = (g / nus)^(1/6) nu_c^(1/6); expm1(y) and
// y e^y / expm1(y) as Taylor polynomials below 1e-2, relative error < 2e-11).
template <class T>
RTW_HD void torus_bin_core(const TorusBinPre& q, const TorusBin& bn, T& ft, T& fi, T& DX, T& Dy) {
    const T c = T(1.8877486253633868);  // 2^(11/12)
    T x16;
    if constexpr (sizeof(T) == 4) {
        x16 = T(q.e6) * T(bn.nu16);
        if (!q.ok || !(x16 <= T(7.647244913317299))) {  // X > 2e5 ((2e5)^(1/6)): no emission
            ft = fi = DX = Dy = T(0);
            return;
        }
    } else {
        const double lxd = q.L + bn.ln_nu;
        if (!q.ok || !(lxd <= 12.206072645530174)) {  // X > 2e5: exp(-X^1/3) < 1e-25, no emission
            ft = fi = DX = Dy = T(0);
            return;
        }
        x16 = BinMath<T>::ex(T(lxd) * T(1.0 / 6.0));
    }
    const T x13 = x16 * x16, x12 = x13 * x16;
    const T P = x12 + c * x16;
    const T j = T(q.cjnus) * P * P * BinMath<T>::ex(-x13);
    const T ig4 = T(q.ig4);
    fi = -(j * T(bn.inv_nu_nm3) * ig4);
    T em1;
    if constexpr (sizeof(T) == 4) {
        const T y = T(q.gt) * T(bn.hk);
        if (y < T(1e-2)) {
            em1 = y * (T(1) + y * (T(0.5) + y * (T(1.0 / 6.0) + y * (T(1.0 / 24.0) + y * T(1.0 / 120.0)))));
            Dy = T(1) + y * (T(0.5) + y * (T(1.0 / 12.0) - y * y * T(1.0 / 720.0)));
        } else {
            em1 = BinMath<T>::em1(y);
            Dy = y * (em1 + T(1)) / em1;
        }
        ft = -(j * (em1 * T(bn.inv_b0)) * ig4);  // em1 / b0 first: j em1 alone can fall below FP32's normal range
    } else {
        const T y = T(q.gt * bn.hk);
        em1 = BinMath<T>::em1(y);
        Dy = y * (em1 + T(1)) / em1;
        ft = -(j * em1 * ig4 * T(bn.inv_b0));
    }
    DX = (x12 + c * T(1.0 / 3.0) * x16) / P - x13 * T(1.0 / 3.0);
}

// The bin's slopes and their partials d(ft, fi) / d(cj, nus, th, g).
template <class T>
RTW_HD void torus_bin_grad_pre(const TorusBinPre& q, const TorusBin& bn, T& ft, T& fi, T* dft, T* dfi) {
    T DX, Dy;
    torus_bin_core<T>(q, bn, ft, fi, DX, Dy);
    const T icj = T(q.icj), inus = T(q.inus), ig = T(q.ig);
    dfi[0] = fi * icj;
    dfi[1] = fi * (T(1) - DX) * inus;
    dfi[2] = 0;
    dfi[3] = fi * (DX - T(4)) * ig;
    dft[0] = ft * icj;
    dft[1] = ft * (T(1) - DX) * inus;
    dft[2] = -ft * Dy * T(q.ith);
    dft[3] = ft * (DX - T(4) + Dy) * ig;
}

RTW_HD void torus_bin_grad(double cj, double nus, double th, double g, const TorusBin& bn, double& ft, double& fi,
                           double* dft, double* dfi) {
    for (int q = 0; q < 4; ++q) {
        dft[q] = 0;
        dfi[q] = 0;
    }
    ft = 0;
    fi = 0;
    const double X = g * bn.nu_hz / nus;
    if (!(X > 0) || X > 2.0e5) return;
    const double lx = log(X);
    const double x12 = exp(0.5 * lx), x16 = exp(lx / 6.0), x13 = exp(lx / 3.0);
    const double c = 1.8877486253633868;  // 2^(11/12)
    const double P = x12 + c * x16;
    const double j = cj * nus * P * P * exp(-x13);
    const double g2 = g * g, g4 = g2 * g2;
    fi = -(j * bn.inv_nu_nm3 / g4);
    const double y = g * bn.hk / th;
    const double em1 = expm1(y);
    ft = -(j * em1 / (g4 * bn.b0));
    const double DX = (x12 + c / 3.0 * x16) / P - x13 / 3.0;
    const double Dy = y * (em1 + 1.0) / em1;
    // d/dS = F * dlnF/dlnS / S
    dfi[0] = fi / cj;
    dfi[1] = fi * (1.0 - DX) / nus;
    dfi[2] = 0;
    dfi[3] = fi * (DX - 4.0) / g;
    dft[0] = ft / cj;
    dft[1] = ft * (1.0 - DX) / nus;
    dft[2] = -ft * Dy / th;
    dft[3] = ft * (DX - 4.0 + Dy) / g;
}

// Kerr geodesic acceleration a^mu = -g^{mu nu} T_nu with
// T_nu = (k^a d_a g_{nu b}) k^b - (1/2) d_nu g_{ab} k^a k^b (the metric
// depends on r and theta only). Generic in T for the adjoint's derivatives
// (including d/da); k = (k^t, k^r, k^theta, k^phi).
template <class T>
RTW_HD void kerr_accel(double Md, const T& a, const T& r, const T& th, const T* k, T* acc) {
    typedef decltype(val(r)) B;
    const B M = B(Md);
    const T sn = tsin(th), cs = tcos(th);
    const T r2 = r * r, a2 = a * a, s2 = sn * sn, c2 = cs * cs, sc = sn * cs;
    const T Sig = r2 + a2 * c2;
    const T Del = r2 - B(2.0) * M * r + a2;
    const T iS = T(1.0) / Sig;
    const T Sr = B(2.0) * r, St = B(-2.0) * a2 * sc;  // d Sigma / dr, / dtheta
    const T f = B(2.0) * M * r * iS;                    // 2 M r / Sigma
    const T fr = B(2.0) * M * iS - f * Sr * iS;         // d f / dr
    const T ft = -(f * St * iS);                        // d f / dtheta
    // metric
    const T gtt = f - B(1.0);
    const T gtp = -(f * a * s2);
    const T gpp = (r2 + a2) * s2 + f * a2 * s2 * s2;
    const T grr = Sig / Del;
    // derivatives
    const T gtt_r = fr, gtt_t = ft;
    const T gtp_r = -(fr * a * s2), gtp_t = -(a * (ft * s2 + f * B(2.0) * sc));
    const T gpp_r = B(2.0) * r * s2 + fr * a2 * s2 * s2;
    const T gpp_t = (r2 + a2) * B(2.0) * sc + a2 * (ft * s2 * s2 + f * B(4.0) * s2 * sc);
    const T grr_r = (Sr * Del - Sig * (B(2.0) * r - B(2.0) * M)) / (Del * Del);
    const T grr_t = St / Del;
    const T ghh_r = Sr, ghh_t = St;
    const T kt = k[0], kr = k[1], kh = k[2], kp = k[3];
    // T_t, T_phi: only the advective part
    const T Tt = (kr * gtt_r + kh * gtt_t) * kt + (kr * gtp_r + kh * gtp_t) * kp;
    const T Tp = (kr * gtp_r + kh * gtp_t) * kt + (kr * gpp_r + kh * gpp_t) * kp;
    const T Qr = gtt_r * kt * kt + B(2.0) * gtp_r * kt * kp + gpp_r * kp * kp + grr_r * kr * kr + ghh_r * kh * kh;
    const T Qt = gtt_t * kt * kt + B(2.0) * gtp_t * kt * kp + gpp_t * kp * kp + grr_t * kr * kr + ghh_t * kh * kh;
    const T Tr = (kr * grr_r + kh * grr_t) * kr - B(0.5) * Qr;
    const T Th = (kr * ghh_r + kh * ghh_t) * kh - B(0.5) * Qt;
    // inverse metric: (t, phi) block, det = gtt gpp - gtp^2
    const T det = gtt * gpp - gtp * gtp;
    const T idet = T(1.0) / det;
    acc[0] = -((gpp * Tt - gtp * Tp) * idet);
    acc[3] = -((gtt * Tp - gtp * Tt) * idet);
    acc[1] = -(Tr / grr);
    acc[2] = -(Th * iS);
}

// Reverse mode of kerr_accel: given the cotangent cw of acc, the cotangents
// of r, theta, a and k (db_r, db_th, db_a, db_k[4]), by the chain rule through
// kerr_accel's own intermediates in reverse order (about three times the
// acceleration's arithmetic, against eight for a 7-tangent dual pass).
template <class T>
RTW_HD void kerr_accel_vjp(double Md, T a, T r, T th, const T* k, const T* cw, T& db_r, T& db_th, T& db_a,
                           T* db_k) {
    const T M = T(Md);
    const T sn = tsin(th), cs = tcos(th);
    const T r2 = r * r, a2 = a * a, s2 = sn * sn, c2 = cs * cs, sc = sn * cs;
    const T Sig = r2 + a2 * c2;
    const T Del = r2 - T(2.0) * M * r + a2;
    const T iS = T(1.0) / Sig;
    const T Sr = T(2.0) * r, St = T(-2.0) * a2 * sc;
    const T f = T(2.0) * M * r * iS;
    const T fr = T(2.0) * M * iS - f * Sr * iS;
    const T ft = -(f * St * iS);
    const T gtt = f - T(1.0);
    const T gtp = -(f * a * s2);
    const T gpp = (r2 + a2) * s2 + f * a2 * s2 * s2;
    const T iD = T(1.0) / Del;
    const T grr = Sig * iD;
    const T gtt_r = fr, gtt_t = ft;
    const T gtp_r = -(fr * a * s2), gtp_t = -(a * (ft * s2 + f * T(2.0) * sc));
    const T gpp_r = T(2.0) * r * s2 + fr * a2 * s2 * s2;
    const T gpp_t = (r2 + a2) * T(2.0) * sc + a2 * (ft * s2 * s2 + f * T(4.0) * s2 * sc);
    const T Nr = Sr * Del - Sig * (T(2.0) * r - T(2.0) * M);
    const T grr_r = Nr * iD * iD;
    const T grr_t = St * iD;
    const T ghh_r = Sr, ghh_t = St;
    const T kt = k[0], kr = k[1], kh = k[2], kp = k[3];
    const T A1 = kr * gtt_r + kh * gtt_t, A2 = kr * gtp_r + kh * gtp_t, A3 = kr * gpp_r + kh * gpp_t;
    const T Tt = A1 * kt + A2 * kp;
    const T Tp = A2 * kt + A3 * kp;
    const T Tr = (kr * grr_r + kh * grr_t) * kr - T(0.5) * (gtt_r * kt * kt + T(2.0) * gtp_r * kt * kp +
                                                            gpp_r * kp * kp + grr_r * kr * kr + ghh_r * kh * kh);
    const T Th = (kr * ghh_r + kh * ghh_t) * kh - T(0.5) * (gtt_t * kt * kt + T(2.0) * gtp_t * kt * kp +
                                                            gpp_t * kp * kp + grr_t * kr * kr + ghh_t * kh * kh);
    const T det = gtt * gpp - gtp * gtp;
    const T idet = T(1.0) / det;
    const T N0 = gpp * Tt - gtp * Tp, N3 = gtt * Tp - gtp * Tt;
    // acc0 = -N0 idet, acc3 = -N3 idet, acc1 = -Tr / grr, acc2 = -Th iS
    const T bN0 = -cw[0] * idet, bN3 = -cw[3] * idet;
    const T bdet = (cw[0] * N0 + cw[3] * N3) * idet * idet;  // d/d det of -(N0 c0 + N3 c3) / det
    const T igrr = T(1.0) / grr;
    const T bTr = -cw[1] * igrr, bTh = -cw[2] * iS;
    T bgrr = cw[1] * Tr * igrr * igrr;
    T biS = -cw[2] * Th;
    // N0, N3, det
    T bgpp = bN0 * Tt + bdet * gtt;
    T bgtt = bN3 * Tp + bdet * gpp;
    T bgtp = -bN0 * Tp - bN3 * Tt - T(2.0) * bdet * gtp;
    const T bTt = bN0 * gpp - bN3 * gtp;
    const T bTp = -bN0 * gtp + bN3 * gtt;
    // Tr, Th (with Qr, Qt)
    const T bQr = T(-0.5) * bTr, bQt = T(-0.5) * bTh;
    T bkt = T(0), bkr = T(0), bkh = T(0), bkp = T(0);
    T bgrr_r = bTr * kr * kr + bQr * kr * kr;
    T bgrr_t = bTr * kh * kr + bQt * kr * kr;
    T bghh_r = bTh * kr * kh + bQr * kh * kh;
    T bghh_t = bTh * kh * kh + bQt * kh * kh;
    bkr += bTr * (T(2.0) * kr * grr_r + kh * grr_t) + bTh * ghh_r * kh;
    bkh += bTr * grr_t * kr + bTh * (kr * ghh_r + T(2.0) * kh * ghh_t);
    T bgtt_r = bQr * kt * kt, bgtp_r = bQr * T(2.0) * kt * kp, bgpp_r = bQr * kp * kp;
    T bgtt_t = bQt * kt * kt, bgtp_t = bQt * T(2.0) * kt * kp, bgpp_t = bQt * kp * kp;
    bkt += bQr * (T(2.0) * gtt_r * kt + T(2.0) * gtp_r * kp) + bQt * (T(2.0) * gtt_t * kt + T(2.0) * gtp_t * kp);
    bkp += bQr * (T(2.0) * gtp_r * kt + T(2.0) * gpp_r * kp) + bQt * (T(2.0) * gtp_t * kt + T(2.0) * gpp_t * kp);
    bkr += bQr * T(2.0) * grr_r * kr + bQt * T(2.0) * grr_t * kr;
    bkh += bQr * T(2.0) * ghh_r * kh + bQt * T(2.0) * ghh_t * kh;
    // Tt = A1 kt + A2 kp, Tp = A2 kt + A3 kp
    const T bA1 = bTt * kt, bA2 = bTt * kp + bTp * kt, bA3 = bTp * kp;
    bkt += bTt * A1 + bTp * A2;
    bkp += bTt * A2 + bTp * A3;
    bgtt_r += bA1 * kr;
    bgtt_t += bA1 * kh;
    bgtp_r += bA2 * kr;
    bgtp_t += bA2 * kh;
    bgpp_r += bA3 * kr;
    bgpp_t += bA3 * kh;
    bkr += bA1 * gtt_r + bA2 * gtp_r + bA3 * gpp_r;
    bkh += bA1 * gtt_t + bA2 * gtp_t + bA3 * gpp_t;
    // the metric and its derivatives
    T br = T(0), ba = T(0), br2 = T(0), ba2 = T(0), bs2 = T(0), bc2 = T(0), bsc = T(0);
    T bSig = T(0), bDel = T(0), bSr = bghh_r, bSt = bghh_t;
    // grr_t = St iD, grr_r = Nr iD^2, grr = Sig iD
    bSt += bgrr_t * iD;
    const T bNr = bgrr_r * iD * iD;
    bDel += -bgrr_t * grr_t * iD - T(2.0) * bgrr_r * grr_r * iD - bgrr * grr * iD + bNr * Sr;
    bSr += bNr * Del;
    bSig += -bNr * (T(2.0) * r - T(2.0) * M) + bgrr * iD;
    br += T(-2.0) * bNr * Sig;
    // gpp_t, gpp_r, gtp_t, gtp_r
    T bft = bgtt_t, bfr = bgtt_r, bf = bgtt;
    br2 += bgpp_t * T(2.0) * sc + bgpp * s2;
    ba2 += bgpp_t * (T(2.0) * sc + ft * s2 * s2 + T(4.0) * f * s2 * sc) + bgpp_r * fr * s2 * s2 +
           bgpp * (s2 + f * s2 * s2);
    bsc += bgpp_t * (T(2.0) * (r2 + a2) + T(4.0) * a2 * f * s2) - bgtp_t * T(2.0) * a * f;
    bft += bgpp_t * a2 * s2 * s2 - bgtp_t * a * s2;
    bs2 += bgpp_t * a2 * (T(2.0) * ft * s2 + T(4.0) * f * sc) + bgpp_r * (T(2.0) * r + T(2.0) * fr * a2 * s2) -
           bgtp_t * a * ft - bgtp_r * fr * a + bgpp * ((r2 + a2) + T(2.0) * f * a2 * s2) - bgtp * f * a;
    bf += bgpp_t * T(4.0) * a2 * s2 * sc - bgtp_t * T(2.0) * a * sc + bgpp * a2 * s2 * s2 - bgtp * a * s2;
    br += bgpp_r * T(2.0) * s2;
    bfr += bgpp_r * a2 * s2 * s2 - bgtp_r * a * s2;
    ba += -bgtp_t * (ft * s2 + T(2.0) * f * sc) - bgtp_r * fr * s2 - bgtp * f * s2;
    // ft = -f St iS, fr = 2 M iS - f Sr iS, f = 2 M r iS
    bf += -bft * St * iS - bfr * Sr * iS;
    bSt += -bft * f * iS;
    bSr += -bfr * f * iS;
    biS += -bft * f * St + bfr * (T(2.0) * M - f * Sr) + bf * T(2.0) * M * r;
    br += bf * T(2.0) * M * iS;
    // St = -2 a2 sc, Sr = 2 r, iS = 1 / Sig
    ba2 += T(-2.0) * bSt * sc;
    bsc += T(-2.0) * bSt * a2;
    br += T(2.0) * bSr;
    bSig += -biS * iS * iS;
    // Del = r2 - 2 M r + a2, Sig = r2 + a2 c2
    br2 += bDel + bSig;
    br += T(-2.0) * M * bDel;
    ba2 += bDel + bSig * c2;
    bc2 += bSig * a2;
    // sc = sn cs, c2 = cs^2, s2 = sn^2, a2 = a^2, r2 = r^2
    const T bsn = bsc * cs + T(2.0) * sn * bs2;
    const T bcs = bsc * sn + T(2.0) * cs * bc2;
    ba += T(2.0) * a * ba2;
    br += T(2.0) * r * br2;
    db_r = br;
    db_th = bsn * cs - bcs * sn;
    db_a = ba;
    db_k[0] = bkt;
    db_k[1] = bkr;
    db_k[2] = bkh;
    db_k[3] = bkp;
}

}  // namespace rtw
