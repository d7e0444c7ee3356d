// rtw_oracle.cpp - TEST INFRASTRUCTURE ONLY (the checker; never the product).
//
// A plain C++17 FP64 restatement of the reference's CPU ("LttM") render path,
// used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg to
// check and time the CUDA library. Nothing in the product path (rtwca_b200/,
// librtw_b200.so) links, loads or calls this file.
//
// Parity status: parity unpinned against the reference itself. The reference
// is Julia, Julia is not installed on any machine of this build, and the
// reference's own tests pin no numerical results (its "tests" are timing runs
// that write PNGs that are not in the repository). This restatement is pinned
// instead against analytic known answers (flat-space straight lines, null-norm
// and Killing-constant conservation, the Schwarzschild critical impact
// parameter, an opaque blackbody sphere, a uniform slab, the CIE fit) in
// tests/test_oracle_physics.py, and against committed golden fixtures that it
// produced (tests/golden/).
//
// What it restates, file:line within the reference project:
//   integrate_ray / ray_kernel / gen_image   main/Iterators/LttM/LttM.jl:11-80,104-176
//   calc_ray_derivative! / RKDP_Step_w_buffer!  main/Iterators/LttM/integrators_LttM.jl:9-224
//   initialize_camera                        main/initialization.jl:190-331
//   rotation / boost matrices                main/gen_geometry.jl:9-103
//   calc_freq_shift                          main/gen_geometry.jl:373-390
//   constants, DP_Butcher                    main/64BitConstants.jl:6-38
//   CIE fit, weights, I_lambda               main/color_theory.jl:11-108
//   Heaviside                                main/my_special_functions.jl:9-15
//   scenes: main/Minkowski_Sphere_Spherical.source/, main/Schwarzschild_Simple_
//           Disk_Spherical.source/, main/Kerr.source/, main/Powehi.source/,
//           main/Synchro_Test.source/ (geometry + model files).
//
// Deliberate differences from the reference, shared with the CUDA library:
//  * Scene constants (spin, disk extent, temperature, a_nu, escape radius) are
//    runtime values of rtw_scene instead of per-scene `const`s.
//  * Outside every emitter (a_nu = j_nu = 0) both RT slopes are exactly 0. The
//    reference computes -inv(g)*0*exp(-tau)/nu^3, which is NaN when a stage
//    point lies inside the horizon (sqrt of a negative in the ZAMO velocity);
//    the reference's CPU path throws a DomainError there instead.
//  * CIE trapezoid weights use the local bin widths; for the reference's
//    uniform `colors` they equal precompute_CIE_weights (color_theory.jl:79-91).
//  * The Kerr Christoffel symbols are FP64 unless scene.ref_precision = 1,
//    which computes them in FP32 as the reference's CPU path does
//    (Kerr.source/source_geometry.jl:196-197).
//  * The termination class is the first predicate of calc_terminate that holds,
//    in the reference's order; RTW_CLASS_NAN marks a non-finite final state.
//
// The synchrotron torus (RTW_SCENE_KERR_SYNCHRO_TORUS) has no reference
// counterpart: it is a new emitter behind the same RT slot contract, restated
// here independently of the library (K_2 from std::cyl_bessel_k, powers from
// std::pow, the normalised Keplerian velocity and the toroidal-field angle
// written out in plain FP64), so that the library's generic-scalar emitter
// is checked against a second implementation. Its formulas: thermal
// synchrotron emissivity of Leung, Gammie & Noble 2011 (ApJ 737, 21) with
// alpha = j / B_nu(T_e).

#include "../include/rtw.h"

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <omp.h>

namespace {

// Float64(pi) as the reference rebinds it in CPU mode (initialization.jl:61-62).
constexpr double kPi = 3.141592653589793;
// 64BitConstants.jl:13-25
constexpr double kPlanckH = 6.62607015e-34;
constexpr double kLightC = 299792458.0;
constexpr double kBoltzmann = 1.380649e-23;
constexpr double kNoDivZero = 1e-24;
const double kEmissionScale = 2 * kPlanckH * kLightC * 1e27;
const double kFFactor = kPlanckH * kLightC * 1e9 / kBoltzmann;

// Dormand-Prince tableau (64BitConstants.jl:28-37): rows 2..6 stage
// coefficients (column 1 is c_i), row 7 = b, row 9 = b*.
struct Tableau {
    double a[10][9];
    Tableau() {
        std::memset(a, 0, sizeof(a));
        a[2][1] = 1.0 / 5;  a[2][2] = 1.0 / 5;
        a[3][1] = 3.0 / 10; a[3][2] = 3.0 / 40; a[3][3] = 9.0 / 40;
        a[4][1] = 4.0 / 5;  a[4][2] = 44.0 / 45; a[4][3] = -56.0 / 15; a[4][4] = 32.0 / 9;
        a[5][1] = 8.0 / 9;  a[5][2] = 19372.0 / 6561; a[5][3] = -25360.0 / 2187;
        a[5][4] = 64448.0 / 6561; a[5][5] = -212.0 / 729;
        a[6][1] = 1; a[6][2] = 9017.0 / 3168; a[6][3] = -355.0 / 33; a[6][4] = 46732.0 / 5247;
        a[6][5] = 49.0 / 176; a[6][6] = -5103.0 / 18656;
        a[7][1] = 1; a[7][2] = 35.0 / 384; a[7][3] = 0; a[7][4] = 500.0 / 1113;
        a[7][5] = 125.0 / 192; a[7][6] = -2187.0 / 6784; a[7][7] = 11.0 / 84;
        a[9][2] = 5179.0 / 57600; a[9][4] = 7571.0 / 16695; a[9][5] = 393.0 / 640;
        a[9][6] = -92097.0 / 339200; a[9][7] = 187.0 / 2100; a[9][8] = 1.0 / 40;
    }
};
const Tableau kDP;

// Julia's mod(x, y) for floats: result has the sign of y.
inline double jl_mod(double x, double y) {
    double r = std::fmod(x, y);
    if (r != 0 && ((r < 0) != (y < 0))) r += y;
    return r;
}

inline double sq(double x) { return x * x; }

// ----------------------------------------------------------------------------
// Forward-mode derivatives: a dual number with five tangents (spin,
// inclination, n_e0, b_0, theta_e0 of the synchrotron torus). The oracle's
// torus path below is written once over the scalar type and instantiated
// with double (the oracle itself) and with D5 (its forward-mode derivative,
// in the role ForwardDiff plays for the reference's CPU integrator).
// Comparisons and branches use the value, as ForwardDiff's do.
// ----------------------------------------------------------------------------
constexpr int kTan = 5;
struct D5 {
    double v = 0;
    double d[kTan] = {0, 0, 0, 0, 0};
    D5() = default;
    D5(double x) : v(x) {}  // NOLINT: constants enter with zero tangents
};
inline double val(double x) { return x; }
inline double val(const D5& x) { return x.v; }
template <class F>
inline D5 chain(const D5& a, double f, double df) {  // f(a), f'(a)
    D5 r(f);
    for (int i = 0; i < kTan; ++i) r.d[i] = df * a.d[i];
    return r;
}
inline D5 operator-(const D5& a) { D5 r(-a.v); for (int i = 0; i < kTan; ++i) r.d[i] = -a.d[i]; return r; }
inline D5 operator+(const D5& a, const D5& b) { D5 r(a.v + b.v); for (int i = 0; i < kTan; ++i) r.d[i] = a.d[i] + b.d[i]; return r; }
inline D5 operator-(const D5& a, const D5& b) { D5 r(a.v - b.v); for (int i = 0; i < kTan; ++i) r.d[i] = a.d[i] - b.d[i]; return r; }
inline D5 operator*(const D5& a, const D5& b) {
    D5 r(a.v * b.v);
    for (int i = 0; i < kTan; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
inline D5 operator/(const D5& a, const D5& b) {
    D5 r(a.v / b.v);
    for (int i = 0; i < kTan; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) / b.v;
    return r;
}
inline D5 operator+(const D5& a, double b) { D5 r = a; r.v += b; return r; }
inline D5 operator+(double a, const D5& b) { return b + a; }
inline D5 operator-(const D5& a, double b) { D5 r = a; r.v -= b; return r; }
inline D5 operator-(double a, const D5& b) { return -(b - a); }
inline D5 operator*(const D5& a, double b) { D5 r(a.v * b); for (int i = 0; i < kTan; ++i) r.d[i] = a.d[i] * b; return r; }
inline D5 operator*(double a, const D5& b) { return b * a; }
inline D5 operator/(const D5& a, double b) { D5 r(a.v / b); for (int i = 0; i < kTan; ++i) r.d[i] = a.d[i] / b; return r; }
inline D5 operator/(double a, const D5& b) { return D5(a) / b; }
inline D5& operator+=(D5& a, const D5& b) { a = a + b; return a; }
inline D5& operator-=(D5& a, const D5& b) { a = a - b; return a; }
inline bool operator<(const D5& a, const D5& b) { return a.v < b.v; }
inline bool operator>(const D5& a, const D5& b) { return a.v > b.v; }
inline bool operator<=(const D5& a, const D5& b) { return a.v <= b.v; }
inline bool operator>=(const D5& a, const D5& b) { return a.v >= b.v; }
inline bool operator==(const D5& a, const D5& b) { return a.v == b.v; }
inline bool operator!=(const D5& a, const D5& b) { return a.v != b.v; }
inline D5 sin(const D5& a) { return chain<D5>(a, std::sin(a.v), std::cos(a.v)); }
inline D5 cos(const D5& a) { return chain<D5>(a, std::cos(a.v), -std::sin(a.v)); }
inline D5 tan(const D5& a) { const double t = std::tan(a.v); return chain<D5>(a, t, 1 + t * t); }
inline D5 atan(const D5& a) { return chain<D5>(a, std::atan(a.v), 1 / (1 + a.v * a.v)); }
inline D5 sqrt(const D5& a) { const double s = std::sqrt(a.v); return chain<D5>(a, s, 0.5 / s); }
inline D5 exp(const D5& a) { const double e = std::exp(a.v); return chain<D5>(a, e, e); }
inline D5 expm1(const D5& a) { return chain<D5>(a, std::expm1(a.v), std::exp(a.v)); }
inline D5 log(const D5& a) { return chain<D5>(a, std::log(a.v), 1 / a.v); }
inline D5 pow(const D5& a, double e) { return chain<D5>(a, std::pow(a.v, e), e * std::pow(a.v, e - 1)); }
inline D5 fabs(const D5& a) { return a.v < 0 ? -a : a; }
inline bool isfinite(const D5& a) { return std::isfinite(a.v); }
// K_nu(x) and dK_nu/dx = -(K_{nu-1}(x) + K_{nu+1}(x)) / 2
inline D5 cyl_bessel_k(double nu, const D5& x) {
    return chain<D5>(x, std::cyl_bessel_k(nu, x.v),
                     -0.5 * (std::cyl_bessel_k(nu - 1, x.v) + std::cyl_bessel_k(nu + 1, x.v)));
}
template <class T>
inline T sqT(const T& x) { return x * x; }

// ----------------------------------------------------------------------------
// Counting scalar: a double value and, per thread, the operations the
// oracle's arithmetic performs on it, so that the algorithmic work of the
// reference's form is counted by running the oracle itself: add/sub/mul = 1
// flop; div/sqrt/exp/log/sin/cos = 1 flop + 1 transcendental; pow = 2 + 2
// (the convention of the library's rtw_get_op_counts). Sign flips and
// fabs/min/max are not counted. Comparisons and branches use the value, so a
// counting run takes the double run's path exactly.
// ----------------------------------------------------------------------------
struct OpTally {
    long long flops = 0, special = 0;
};
inline OpTally& tally() {
    static thread_local OpTally t;
    return t;
}
struct Cnt {
    double v = 0;
    Cnt() = default;
    Cnt(double x) : v(x) {}  // NOLINT: constants enter uncounted
};
inline double val(const Cnt& x) { return x.v; }
inline Cnt cnt_op(double r, int f, int sp) {
    OpTally& t = tally();
    t.flops += f;
    t.special += sp;
    return Cnt(r);
}
inline Cnt operator-(const Cnt& a) { return Cnt(-a.v); }
inline Cnt operator+(const Cnt& a, const Cnt& b) { return cnt_op(a.v + b.v, 1, 0); }
inline Cnt operator-(const Cnt& a, const Cnt& b) { return cnt_op(a.v - b.v, 1, 0); }
inline Cnt operator*(const Cnt& a, const Cnt& b) { return cnt_op(a.v * b.v, 1, 0); }
inline Cnt operator/(const Cnt& a, const Cnt& b) { return cnt_op(a.v / b.v, 1, 1); }
inline Cnt operator+(const Cnt& a, double b) { return cnt_op(a.v + b, 1, 0); }
inline Cnt operator+(double a, const Cnt& b) { return cnt_op(a + b.v, 1, 0); }
inline Cnt operator-(const Cnt& a, double b) { return cnt_op(a.v - b, 1, 0); }
inline Cnt operator-(double a, const Cnt& b) { return cnt_op(a - b.v, 1, 0); }
inline Cnt operator*(const Cnt& a, double b) { return cnt_op(a.v * b, 1, 0); }
inline Cnt operator*(double a, const Cnt& b) { return cnt_op(a * b.v, 1, 0); }
inline Cnt operator/(const Cnt& a, double b) { return cnt_op(a.v / b, 1, 1); }
inline Cnt operator/(double a, const Cnt& b) { return cnt_op(a / b.v, 1, 1); }
inline Cnt& operator+=(Cnt& a, const Cnt& b) { return a = a + b; }
inline Cnt& operator-=(Cnt& a, const Cnt& b) { return a = a - b; }
inline Cnt& operator*=(Cnt& a, const Cnt& b) { return a = a * b; }
inline bool operator<(const Cnt& a, const Cnt& b) { return a.v < b.v; }
inline bool operator>(const Cnt& a, const Cnt& b) { return a.v > b.v; }
inline bool operator<=(const Cnt& a, const Cnt& b) { return a.v <= b.v; }
inline bool operator>=(const Cnt& a, const Cnt& b) { return a.v >= b.v; }
inline bool operator==(const Cnt& a, const Cnt& b) { return a.v == b.v; }
inline bool operator!=(const Cnt& a, const Cnt& b) { return a.v != b.v; }
inline bool operator<(const Cnt& a, double b) { return a.v < b; }
inline bool operator>(const Cnt& a, double b) { return a.v > b; }
inline bool operator<=(const Cnt& a, double b) { return a.v <= b; }
inline bool operator>=(const Cnt& a, double b) { return a.v >= b; }
inline bool operator==(const Cnt& a, double b) { return a.v == b; }
inline bool operator!=(const Cnt& a, double b) { return a.v != b; }
inline bool operator<(double a, const Cnt& b) { return a < b.v; }
inline bool operator>(double a, const Cnt& b) { return a > b.v; }
inline bool operator<=(double a, const Cnt& b) { return a <= b.v; }
inline bool operator>=(double a, const Cnt& b) { return a >= b.v; }
inline Cnt sin(const Cnt& a) { return cnt_op(std::sin(a.v), 1, 1); }
inline Cnt cos(const Cnt& a) { return cnt_op(std::cos(a.v), 1, 1); }
inline Cnt tan(const Cnt& a) { return cnt_op(std::tan(a.v), 1, 1); }
inline Cnt atan(const Cnt& a) { return cnt_op(std::atan(a.v), 1, 1); }
inline Cnt sqrt(const Cnt& a) { return cnt_op(std::sqrt(a.v), 1, 1); }
inline Cnt exp(const Cnt& a) { return cnt_op(std::exp(a.v), 1, 1); }
inline Cnt expm1(const Cnt& a) { return cnt_op(std::expm1(a.v), 1, 1); }
inline Cnt log(const Cnt& a) { return cnt_op(std::log(a.v), 1, 1); }
inline Cnt pow(const Cnt& a, double e) { return cnt_op(std::pow(a.v, e), 2, 2); }
inline Cnt pow(const Cnt& a, const Cnt& e) { return cnt_op(std::pow(a.v, e.v), 2, 2); }
inline Cnt fabs(const Cnt& a) { return Cnt(std::fabs(a.v)); }
inline bool isfinite(const Cnt& a) { return std::isfinite(a.v); }
inline Cnt jl_mod(const Cnt& x, double y) { return cnt_op(jl_mod(x.v, y), 1, 0); }
inline Cnt max(const Cnt& a, const Cnt& b) { return a.v < b.v ? b : a; }
inline Cnt min(const Cnt& a, const Cnt& b) { return b.v < a.v ? b : a; }
inline Cnt max(const Cnt& a, double b) { return a.v < b ? Cnt(b) : a; }
inline Cnt min(const Cnt& a, double b) { return b < a.v ? Cnt(b) : a; }


// ----------------------------------------------------------------------------
// Scenes (".source" plugins), restated with runtime constants.
// ----------------------------------------------------------------------------
struct OScene {
    int kind = 0;
    bool refprec = false;
    double M = 1, a = 0, rs = 2, r_ev = 2, r_in = 6, r_out = 12, th_lo = 0, th_hi = kPi;
    double T = 5778, anu = 1, esc = 100, wind = 8 * kPi;
    double rho_r0 = 6, rho_h = 0.1, rho_idx = -2, t_idx = -0.75;
    double n0 = 0, b0 = 0, th0 = 0, b_idx = 0, edge_in = 1, edge_out = 1, length_cm = 1;
    // gen_image's ray_bundles: 11 more ray components, which calc_terminate's
    // all-slots opacity test also reads (they are 0 or small: it never holds)
    bool bundles = false;

    explicit OScene(const rtw_scene& s) {
        kind = s.kind;
        refprec = s.ref_precision != 0;
        M = s.mass;
        a = s.spin;
        r_in = s.r_in; r_out = s.r_out; th_lo = s.theta_lo; th_hi = s.theta_hi;
        T = s.temperature; anu = s.a_nu; esc = s.escape_radius; wind = s.winding_limit;
        rho_r0 = s.rho_r0; rho_h = s.rho_h; rho_idx = s.rho_index; t_idx = s.t_index;
        n0 = s.n_e0; b0 = s.b_0; th0 = s.theta_e0; b_idx = s.b_index;
        edge_in = s.edge_in; edge_out = s.edge_out; length_cm = s.length_cm;
        if (kind == RTW_SCENE_SCHWARZSCHILD_DISK) a = 0;
        if (refprec) {
            // the reference's Float32 literals (Kerr source_geometry.jl:7,13,
            // source_model.jl:44,60)
            a = (double)(float)a;
            anu = (double)(float)anu;
            T = (double)(float)T;
        }
        rs = 2 * M;
        if (is_kerr()) {
            // Kerr source_geometry.jl:17
            if (refprec) {
                float rsf = (float)rs, af = (float)a;
                r_ev = (double)(rsf / 2 + std::sqrt((rsf * rsf / 4) - af * af));
            } else {
                r_ev = rs / 2 + std::sqrt((rs * rs / 4) - a * a);
            }
        } else {
            r_ev = rs;
        }
    }

    bool is_kerr() const {
        return kind == RTW_SCENE_KERR_DISK || kind == RTW_SCENE_KERR_THICK_DISK || kind == RTW_SCENE_KERR_SYNCHRO_TORUS ||
               kind == RTW_SCENE_KERR_BREMS_TORUS ||
               kind == RTW_SCENE_KERR_POWEHI;
    }
    // Synchro_Test.source and Minkowski_Sphere_Cartesian.source: Minkowski
    // space in Cartesian (t, x, y, z) (the two geometry files differ in
    // whitespace only)
    bool is_cart() const { return kind == RTW_SCENE_SYNCHRO_TEST || kind == RTW_SCENE_MINKOWSKI_CART_SPHERE; }
    // Wormhole.source: the Dneg wormhole in (t, l, theta, phi)
    bool is_wh() const { return kind == RTW_SCENE_WORMHOLE; }
    // source_geometry.jl:7-41: M = W / W_over_M, r(l), and dr/dl as the
    // reference writes it (with its extra (x - 1) / (1 + x^2) term)
    double wh_M() const {
        const double c = kPi / (2 * std::sqrt(2.0));
        return edge_out / (-std::log(1 / std::cos(c)) + c * std::tan(c));
    }
    double wh_r(double l) const {
        if (!(std::fabs(l) > edge_in)) return r_in;
        const double M = wh_M(), x = 2 * (std::fabs(l) - edge_in) / (kPi * M);
        return r_in + M * (x * std::atan(x) - std::log(1 + x * x) / 2);
    }
    double wh_drdl(double l) const {
        if (!(std::fabs(l) > edge_in)) return 0.0;
        const double M = wh_M(), x = 2 * (std::fabs(l) - edge_in) / (kPi * M);
        const double d = 2 * (std::atan(x) + (x - 1) / (1 + x * x)) / kPi;
        return l < 0 ? -d : d;
    }

    // --- geometry -----------------------------------------------------------
    // Kerr calc_metric_params, source_geometry.jl:55-60
    void kerr_params(double r, double th, double& Sig, double& Del, double& A) const {
        Sig = r * r + sq(a * std::cos(th));
        Del = r * r - r * rs + a * a;
        A = (r * r + a * a) * Sig + rs * r * sq(a * std::sin(th));
    }

    // Kerr calc_lower_metric! (source_geometry.jl:66-75) over the scalar type,
    // spin al (the metric entries not written are left as they are)
    template <class T>
    void kerr_metric_t(const T& r, const T& th, const T& al, T g[4][4]) const {
        using std::cos;
        using std::sin;
        const T Sig = r * r + sqT(al * cos(th));
        const T Del = r * r - r * rs + al * al;
        const T A = (r * r + al * al) * Sig + rs * r * sqT(al * sin(th));
        g[0][0] = -(1.0 - rs * r / Sig);
        g[0][3] = -rs * al * r * sqT(sin(th)) / Sig;
        g[3][0] = g[0][3];
        g[1][1] = Sig / Del;
        g[2][2] = Sig;
        g[3][3] = (A / Sig) * sqT(sin(th));
    }

    // calc_lower_metric!: Kerr :66-75, Schwarzschild :15-21, Minkowski :10-16
    // (over the scalar F: double, or Cnt for the thin-disk scenes' op counts)
    template <class F>
    void lower_metric(const F* x, F g[4][4]) const {
        using std::sin;
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) g[i][j] = (i == j) ? 1.0 : 0.0;
        const F r = x[1], th = x[2];
        if (is_cart()) {  // Synchro_Test source_geometry.jl:7-16
            g[0][0] = -1.0;
        } else if (is_wh()) {  // Wormhole source_geometry.jl:44-51
            if constexpr (std::is_same<F, double>::value) {
                g[0][0] = -1.0;
                g[2][2] = sq(wh_r(r));
                g[3][3] = sq(wh_r(r) * std::sin(th));
            }
        } else if (is_kerr()) {
            kerr_metric_t<F>(r, th, F(a), g);
        } else if (kind == RTW_SCENE_SCHWARZSCHILD_DISK) {
            g[0][0] = -(1.0 - rs / r);
            g[1][1] = 1.0 / (1.0 - rs / r);
            g[2][2] = r * r;
            g[3][3] = sqT(r * sin(th));
        } else {
            g[0][0] = -1.0;
            g[1][1] = 1.0;
            g[2][2] = r * r;
            g[3][3] = sqT(r * sin(th));
        }
    }

    // calc_inv_vierbein: Kerr :112-121, Schwarzschild :53-60, Minkowski :45-50
    void inv_vierbein(const double* x, double e[4][4]) const {
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) e[i][j] = (i == j) ? 1.0 : 0.0;
        if (is_cart()) return;  // Synchro_Test source_geometry.jl:44-50
        const double r = x[1], th = x[2];
        if (is_wh()) {  // Wormhole source_geometry.jl:83-90
            e[2][2] = 1.0 / wh_r(r);
            e[3][3] = 1.0 / (wh_r(r) * std::sin(th) + kNoDivZero);
            return;
        }
        if (is_kerr()) {
            double Sig, Del, A;
            kerr_params(r, th, Sig, Del, A);
            e[0][0] = std::sqrt(A / (Sig * Del));
            e[3][0] = (rs * a * r / A) * e[0][0];
            e[1][1] = std::sqrt(Del / Sig);
            e[2][2] = 1.0 / std::sqrt(Sig);
            e[3][3] = std::sqrt(Sig / A) / std::sin(th);
        } else if (kind == RTW_SCENE_SCHWARZSCHILD_DISK) {
            e[0][0] = 1.0 / std::sqrt(1.0 - rs / r);
            e[1][1] = std::sqrt(1.0 - rs / r);
            e[2][2] = 1.0 / r;
            e[3][3] = 1.0 / (r * std::sin(th) + kNoDivZero);
        } else {
            e[2][2] = 1.0 / (r + kNoDivZero);
            e[3][3] = 1.0 / (r * std::sin(th) + kNoDivZero);
        }
    }

    template <class F, class GT>
    void kerr_christoffel(F r, F th, F al, F rsv, GT G[4][4][4]) const {
        using std::cos;
        using std::sin;
        const F two = 2;
        const F Sig = r * r + (al * cos(th)) * (al * cos(th));
        const F Del = r * r - r * rsv + al * al;
        const F A = (r * r + al * al) * Sig + rsv * r * (al * sin(th)) * (al * sin(th));
        const F s = sin(th), c = cos(th), s2t = sin(two * th);
        const F cot = c / s;  // cot(theta)
        const F ac2 = (al * c) * (al * c), as2 = (al * s) * (al * s);
        const F Sig2 = Sig * Sig, Sig3 = Sig * Sig * Sig;
        // Kerr source_geometry.jl:203-240
        G[0][0][1] = rsv * (r * r + al * al) * (r * r - ac2) / (two * Sig2 * Del);
        G[0][1][0] = G[0][0][1];
        G[0][0][2] = -rsv * al * al * r * s2t / (two * Sig2);
        G[0][2][0] = G[0][0][2];
        G[0][1][3] = rsv * al * s * s * (ac2 * (al * al - r * r) - r * r * (al * al + 3 * r * r)) / (two * Sig2 * Del);
        G[0][3][1] = G[0][1][3];
        G[0][2][3] = rsv * al * al * al * r * s * s * s * c / Sig2;
        G[0][3][2] = G[0][2][3];
        G[1][0][0] = rsv * Del * (r * r - al * al * c * c) / (two * Sig3);
        G[1][0][3] = -Del * rsv * al * s * s * (r * r - ac2) / (two * Sig3);
        G[1][3][0] = G[1][0][3];
        G[1][1][1] = (two * r * as2 - rsv * (r * r - ac2)) / (two * Sig * Del);
        G[1][1][2] = -al * al * s2t / (two * Sig);
        G[1][2][1] = G[1][1][2];
        G[1][2][2] = -r * Del / Sig;
        G[1][3][3] = Del * s * s * (-two * r * Sig2 + rsv * as2 * (r * r - ac2)) / (two * Sig3);
        G[2][0][0] = -rsv * al * al * r * s2t / (two * Sig3);
        G[2][0][3] = rsv * al * r * (r * r + al * al) * s2t / (two * Sig3);
        G[2][3][0] = G[2][0][3];
        G[2][1][1] = al * al * s2t / (two * Sig * Del);
        G[2][1][2] = r / Sig;
        G[2][2][1] = G[2][1][2];
        G[2][2][2] = -al * al * s2t / (two * Sig);
        G[2][3][3] = -s2t * (A * Sig + (r * r + al * al) * rsv * r * as2) / (two * Sig3);
        G[3][0][1] = rsv * al * (r * r - ac2) / (two * Sig2 * Del);
        G[3][1][0] = G[3][0][1];
        G[3][0][2] = -rsv * al * r * cot / Sig2;
        G[3][2][0] = G[3][0][2];
        const F hs = al * al * s2t / two;
        G[3][1][3] = (two * r * Sig2 + rsv * (hs * hs - r * r * (Sig + r * r + al * al))) / (two * Sig2 * Del);
        G[3][3][1] = G[3][1][3];
        G[3][2][3] = cot * (Sig2 + rsv * r * as2) / Sig2;
        G[3][3][2] = G[3][2][3];
    }

    // calc_christoffel_udd!: Kerr :195-243, Schwarzschild :109-128, Minkowski :93-108
    template <class F>
    void christoffel(const F* x, F G[4][4][4]) const {
        using std::cos;
        using std::sin;
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j)
                for (int k = 0; k < 4; ++k) G[i][j][k] = 0.0;
        if (is_cart()) return;  // Synchro_Test source_geometry.jl:53-66
        const F r = x[1], th = x[2];
        if constexpr (!std::is_same<F, double>::value) {
            // the counting run: the thin-disk scenes (FP64 Christoffel symbols)
            if (is_kerr()) {
                kerr_christoffel<F, F>(r, th, F(a), F(rs), G);
                return;
            }
        } else if (is_wh()) {  // Wormhole source_geometry.jl:131-150
            const double rl = wh_r(r), drdl = wh_drdl(r);
            G[1][2][2] = -rl * drdl;
            G[1][3][3] = -rl * drdl * sq(std::sin(th));
            G[2][1][2] = drdl / rl;
            G[2][2][1] = G[2][1][2];
            G[2][3][3] = -std::sin(th) * std::cos(th);
            G[3][1][3] = drdl / rl;
            G[3][3][1] = G[3][1][3];
            G[3][2][3] = std::cos(th) / std::sin(th);
            G[3][3][2] = G[3][2][3];
            return;
        }
        if constexpr (std::is_same<F, double>::value) {
            if (is_kerr()) {
                if (refprec)
                    kerr_christoffel<float, double>((float)r, (float)th, (float)a, (float)rs, G);
                else
                    kerr_christoffel<double, double>(r, th, a, rs, G);
                return;
            }
        }
        if (kind == RTW_SCENE_SCHWARZSCHILD_DISK) {
            G[0][0][1] = rs / (2 * r * (r - rs));
            G[0][1][0] = G[0][0][1];
            G[1][0][0] = rs * (r - rs) / (2 * r * r * r);
            G[1][1][1] = -rs / (2 * r * (r - rs));
            G[1][2][2] = -(r - rs);
            G[1][3][3] = -(r - rs) * sqT(sin(th));
            G[2][1][2] = 1.0 / r;
            G[2][2][1] = G[2][1][2];
            G[2][3][3] = -sin(th) * cos(th);
            G[3][1][3] = 1.0 / r;
            G[3][3][1] = G[3][1][3];
            G[3][2][3] = cos(th) / sin(th);
            G[3][3][2] = G[3][2][3];
        } else {
            G[1][2][2] = -r;
            G[1][3][3] = -r * sqT(sin(th));
            G[2][1][2] = 1.0 / (r + kNoDivZero);
            G[2][2][1] = G[2][1][2];
            G[2][3][3] = -sin(th) * cos(th);
            G[3][1][3] = 1.0 / (r + kNoDivZero);
            G[3][3][1] = G[3][1][3];
            G[3][2][3] = cos(th) / sin(th);
            G[3][3][2] = G[3][2][3];
        }
    }

    // near_singularity: Kerr :249-269 (= Schwarzschild :134-154), Minkowski :114-132
    bool near_singularity(const double* x, double h, double tol, double* temp) const {
        if (is_cart()) {  // Synchro_Test source_geometry.jl:69-73
            *temp = h;
            return false;
        }
        if (is_wh()) {  // Wormhole source_geometry.jl:156-171: within 5 tol of a pole
            const double th_w = x[2] + h * x[6];
            if (std::fabs(th_w) <= 5 * tol) {
                *temp = 2 * std::fabs(x[2]) / (std::fabs(x[6] * 37) + kNoDivZero);
                return true;
            } else if (std::fabs(th_w - kPi) <= 5 * tol) {
                *temp = 2 * std::fabs((x[2] - kPi) / (std::fabs(x[6] * 37) + kNoDivZero));
                return true;
            }
            *temp = h;
            return false;
        }
        const double th_new = x[2] + h * x[6];
        const double r_new = x[1] + h * x[5];
        if (kind == RTW_SCENE_MINKOWSKI_SPHERE) {
            const double lim = 10 * tol / std::fabs(r_new + kNoDivZero);
            if (std::fabs(th_new) <= lim) {
                *temp = 2 * std::fabs(x[2]) / (std::fabs(x[6] * 37) + kNoDivZero);
                return true;
            } else if (std::fabs(th_new - kPi) <= lim) {
                *temp = 2 * std::fabs((x[2] - kPi) / (std::fabs(x[6] * 37) + kNoDivZero));
                return true;
            } else if (std::fabs(r_new) <= 100 * tol) {
                *temp = 2 * tol / (std::fabs(x[5] * 37) + kNoDivZero);
                return true;
            }
            *temp = h;
            return false;
        }
        if (std::fabs(th_new) <= tol) {
            *temp = 2 * std::fabs(x[2]) / (std::fabs(x[6] * 37) + kNoDivZero);
            return true;
        } else if (std::fabs(th_new - kPi) <= tol) {
            *temp = 2 * std::fabs((x[2] - kPi) / (std::fabs(x[6] * 37) + kNoDivZero));
            return true;
        }
        *temp = h;
        return false;
    }

    // keepinbounds!: Kerr :275-301 (= Schwarzschild :160-186), Minkowski :138-163
    template <class F>
    void keepinbounds(F* x) const {
        if (is_cart()) return;  // Synchro_Test source_geometry.jl:76-80
        if (kind == RTW_SCENE_MINKOWSKI_SPHERE && x[1] <= 0) {
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
        x[2] = jl_mod(x[2], 2 * kPi);
        if (x[2] >= kPi) {
            x[2] = 2 * kPi - x[2];
            x[3] += kPi;
            x[6] = -x[6];
        }
    }

    // is_singularity: Kerr :307-315 and the other scenes
    bool is_singularity(const double* pos) const {
        if (is_cart()) return false;  // Synchro_Test source_geometry.jl:84-88
        if (is_wh())  // Wormhole source_geometry.jl:197-205: the poles only
            return std::fabs(pos[2]) <= (double)1e-32f || std::fabs(pos[2] - kPi) <= (double)1e-32f;
        if (std::fabs(pos[1]) <= (double)1e-32f) return true;
        if (std::fabs(pos[2]) <= (double)1e-32f || std::fabs(pos[2] - kPi) <= 1e-32) return true;
        return false;
    }

    // --- model --------------------------------------------------------------
    // is_fire: Kerr model :73-80, Schwarzschild :73-80, Minkowski :76-83
    template <class F>
    bool is_fire(const F* x) const {
        using std::sqrt;
        const F r = x[1], th = x[2];
        switch (kind) {
        case RTW_SCENE_MINKOWSKI_SPHERE: return r <= r_out;
        case RTW_SCENE_MINKOWSKI_CART_SPHERE:  // Minkowski_Sphere_Cartesian model :82-90
            return sqrt(x[1] * x[1] + x[2] * x[2] + x[3] * x[3]) <= r_out;
        case RTW_SCENE_SCHWARZSCHILD_DISK:
        case RTW_SCENE_KERR_DISK:
            return r_in <= r && r <= r_out && th_lo <= th && th <= th_hi;
        case RTW_SCENE_KERR_THICK_DISK: return r_in <= r && r <= r_out;
        }
        return false;
    }

    // get_source_velocity!: Kerr model :109-137, Schwarzschild :112-133, Minkowski :111-117
    template <class F>
    void source_velocity(const F* x, F u[4]) const {
        using std::cos;
        using std::pow;
        using std::sin;
        using std::sqrt;
        const F r = x[1], th = x[2];
        u[0] = 1; u[1] = 0; u[2] = 0; u[3] = 0;
        if (kind == RTW_SCENE_MINKOWSKI_SPHERE || kind == RTW_SCENE_MINKOWSKI_CART_SPHERE) return;
        if (kind == RTW_SCENE_SCHWARZSCHILD_DISK) {
            if (is_fire(x)) {
                u[0] = 1.0 / sqrt(1 - 3 * M / r);
                u[3] = (1.0 / sqrt(1 - 3 * M / r)) * sqrt(M / (r * r * r));
            } else {
                u[0] = 1.0 / sqrt(1 - 2 * M / r);
            }
            return;
        }
        if (is_fire(x)) {
            const F r32 = pow(r, 1.5);
            const F Om = sqrt(F(M)) / (r32 + a * sqrt(F(M)));
            const F D = r32 - 3 * M * sqrt(r) + 2 * a * sqrt(F(M));
            const F ut = (r32 + a * sqrt(F(M))) / (pow(r, 0.75) * sqrt(D));
            u[0] = ut;
            u[3] = ut * Om;
        } else {
            const F Aa = sqrt(r * r + sqT(a * cos(th)));
            const F B = r * r + a * a - 2 * M * r;
            const F C = sqT(r * r + a * a) - B * sqT(a * sin(th));
            const F ut = sqrt(C) / (Aa * sqrt(B));
            const F Om = 2 * a * M * r / C;
            u[0] = ut;
            u[3] = ut * Om;
        }
    }

    // calc_radiative_coefficients + calc_planck (Kerr model :18-21,57-67 and
    // the other scenes). fluid: temperature (and density for the thick disk).
    template <class F>
    void radiative(const F* x, F nu, F* a_nu, F* j_nu) const {
        using std::cos;
        using std::exp;
        using std::pow;
        if (!is_fire(x)) {
            *a_nu = 0;
            *j_nu = 0;
            return;
        }
        F Tl = T, al = anu;
        if (kind == RTW_SCENE_KERR_THICK_DISK) {
            const F r = x[1];
            const F z = r * cos(x[2]);
            const F hz = rho_h * r;
            const F rho = pow(r / rho_r0, rho_idx) * exp(-(z * z) / (2 * hz * hz));
            Tl = T * pow(r / rho_r0, t_idx);
            al = anu * rho;
        }
        *a_nu = al;
        *j_nu = al * (kEmissionScale * (nu * nu * nu) / (exp(kFFactor * nu / Tl) - 1));
    }

    // pad_max_dt: Kerr model :86-103, Schwarzschild :86-106, Minkowski :89-105
    double pad_max_dt(const double* x, double scale) const {
        if (kind == RTW_SCENE_MINKOWSKI_CART_SPHERE)  // Minkowski_Sphere_Cartesian model :130-132
            return scale * (1 + std::fabs(x[1]) + std::fabs(x[2]) + std::fabs(x[3]));
        if (is_cart()) return scale * (1 + std::fabs(x[1]) + std::fabs(x[2]));  // Synchro_Test model :241-244
        if (is_wh()) {  // Wormhole model :88-110
            double e = (x[2] < kPi / 8 || x[2] > 7 * kPi / 8) ? std::min(scale, (double)1e-1f) : scale;
            if (std::fabs(x[1]) < 100 * edge_in) e = e / 10;
            const double a = std::fabs(1.0 / (e / (std::fabs(x[5]) + kNoDivZero)) + kNoDivZero);
            const double b = std::fabs(1.0 / (e * std::min(x[2], kPi - x[2]) / (std::fabs(x[6]) + kNoDivZero) + kNoDivZero));
            const double c = std::fabs(1.0 / (e / (std::fabs(x[7]) + kNoDivZero) + kNoDivZero));
            return std::max(std::min(1.0 / (a + b + c + kNoDivZero), 0.5), (double)1e-12f);
        }
        double eps;
        // Kerr casts the scale to Float32 (Kerr model :92-96); the other scenes
        // keep it in Float64 except for the Float32 literal 1f-1.
        if (is_kerr()) scale = (double)(float)scale;
        if (x[2] < kPi / 8 || x[2] > 7 * kPi / 8) {
            eps = std::min(scale, (double)1e-1f);
        } else if (kind == RTW_SCENE_SCHWARZSCHILD_DISK && x[1] <= 1.5 * (3 * M)) {
            eps = scale / 10;
        } else {
            eps = scale;
        }
        double first;
        if (is_kerr())
            first = std::fabs(1.0 / (eps / std::fabs(x[5]))) + kNoDivZero;
        else
            first = std::fabs(1.0 / (eps / (std::fabs(x[5]) + kNoDivZero))) + kNoDivZero;
        const double second =
            std::fabs(1.0 / (eps * std::min(x[2], kPi - x[2]) / (std::fabs(x[6]) + kNoDivZero) + kNoDivZero));
        const double third = std::fabs(1.0 / (eps / (std::fabs(x[7]) + kNoDivZero) + kNoDivZero));
        double m = std::min(1.0 / (first + second + third + kNoDivZero), 0.5);
        m = std::max(m, (double)1e-12f);
        return m;
    }

    // calc_terminate: Kerr model :168-182, Schwarzschild :156-170, Minkowski :131-145.
    // Returns the class of the first predicate that holds, or 0.
    int terminate(const double* ray, int L, double tol, long long max_steps, long long step_count) const {
        if ((double)step_count >= (double)max_steps) return RTW_CLASS_MAXSTEPS;
        if (is_wh()) {  // Wormhole model :134-147
            if (wh_r(ray[1]) > esc) return RTW_CLASS_ESCAPE;
            if (ray[3] > wind) return RTW_CLASS_WINDING;
            if (bundles) return 0;  // the bundle slots are in the opacity test too
            const double thick = -std::log(tol);
            for (int i = 9; i < L; i += 2)
                if (ray[i] < thick) return 0;
            return RTW_CLASS_THICK;
        }
        if (is_cart()) {  // Synchro_Test model :258-275, Minkowski_Sphere_Cartesian :158-172
            if (std::sqrt(ray[1] * ray[1] + ray[2] * ray[2] + ray[3] * ray[3]) > esc) return RTW_CLASS_ESCAPE;
            if (bundles) return 0;
            const double thick = -std::log(tol);
            for (int i = 9; i < L; i += 2)
                if (ray[i] < thick) return 0;
            return RTW_CLASS_THICK;
        }
        if (ray[1] > esc) return RTW_CLASS_ESCAPE;
        if (kind != RTW_SCENE_MINKOWSKI_SPHERE && ray[1] <= (1 + 10 * tol) * r_ev) return RTW_CLASS_HORIZON;
        if (ray[3] > wind) return RTW_CLASS_WINDING;
        const double thick = -std::log(tol);
        for (int i = 9; i < L; i += 2)
            if (ray[i] < thick) return 0;
        return RTW_CLASS_THICK;
    }
};

// ----------------------------------------------------------------------------
// Integrator (integrators_LttM.jl), one ray's buffers.
// ----------------------------------------------------------------------------
// (over the scalar F: double, or Cnt for the thin-disk scenes' op counts)
template <class F>
struct RayWorkT {
    int L = 0, N = 0;
    const double* freq = nullptr;  // colors_freq, nm^-1
    double tol = 1e-4;
    double scale = 0.1;
    bool fsal = false;
    std::vector<F> last_slope, next_slope, buffer, y, k2, k3, k4, k5, k6, k7;
    std::vector<double> plain;  // the state as doubles, for the scene's control functions
    F G[4][4][4];
    F g[4][4];
    F u[4];
    void init(int N_, const double* f, double tol_, double scale_, bool fsal_) {
        N = N_;
        L = 8 + 2 * N;
        freq = f;
        tol = tol_;
        scale = scale_;
        fsal = fsal_;
        for (auto* v : {&last_slope, &next_slope, &buffer, &y, &k2, &k3, &k4, &k5, &k6, &k7}) v->assign(L, F(0.0));
        plain.assign(L, 0.0);
    }
};
using RayWork = RayWorkT<double>;

// The state's values as doubles (the scene's step-size cap, polar-escape
// test and termination test read values only): R itself for double.
inline const double* plain_state(RayWork&, const double* R) { return R; }
template <class F>
const double* plain_state(RayWorkT<F>& w, const F* R) {
    for (int i = 0; i < w.L; ++i) w.plain[i] = val(R[i]);
    return w.plain.data();
}

// RT slopes of the synchrotron torus (no reference counterpart; the formulas
// are listed in the file header), over the scalar type: spin al and the
// emission parameters n0, b0, th0 are arguments so that forward-mode tangents
// can enter through them. slope[8 + 2c] = dI_c, slope[9 + 2c] = dtau_c.
template <class T>
void torus_bins_t(const OScene& sc, const T& al, const T& n0, const T& b0, const T& th0, const double* freq, int N,
                  const T* R, T* slope) {
    using std::cos;
    using std::cyl_bessel_k;
    using std::exp;
    using std::expm1;
    using std::pow;
    using std::sqrt;
    for (int c = 0; c < N; ++c) {
        slope[8 + 2 * c] = 0;
        slope[9 + 2 * c] = 0;
    }
    const T r = R[1], th = R[2];
    const double cut_in = std::max(sc.r_in - 4 * sc.edge_in, 1.01 * sc.r_ev);
    const double cut_out = sc.r_out + 4 * sc.edge_out;
    if (!(val(r) >= cut_in && val(r) <= cut_out)) return;
    T taper = 1;
    if (r < sc.r_in) taper = exp(-sqT((sc.r_in - r) / sc.edge_in));
    else if (r > sc.r_out) taper = exp(-sqT((r - sc.r_out) / sc.edge_out));
    const T x = r / sc.r_in;
    const T z = r * cos(th), hz = sc.rho_h * r;
    const T ne = n0 * pow(x, sc.rho_idx) * exp(-z * z / (2 * hz * hz)) * taper;
    const T B = b0 * pow(x, sc.b_idx);
    const T Th = th0 * pow(x, sc.t_idx);
    T g[4][4];
    sc.kerr_metric_t<T>(r, th, al, g);
    const T Om = std::sqrt(sc.M) / (pow(r, 1.5) + al * std::sqrt(sc.M));
    const T n2 = -(g[0][0] + 2 * Om * g[0][3] + Om * Om * g[3][3]);
    if (!(val(n2) > 0)) return;
    const T ut = 1 / sqrt(n2);
    const T u_t = ut * (g[0][0] + Om * g[0][3]);
    const T u_p = ut * (g[0][3] + Om * g[3][3]);
    const T gs = -(u_t * R[4] + u_p * R[7]);
    const T kph_low = g[0][3] * R[4] + g[3][3] * R[7];
    const T bb = g[3][3] + u_p * u_p;
    const T bk = kph_low - u_p * gs;
    if (!(val(bb) > 0) || !(val(gs) > 0)) return;
    const T c2 = bk * bk / (bb * gs * gs);
    if (!(val(1 - c2) > 1e-12)) return;
    const T sinb = sqrt(1 - c2);
    constexpr double e = 4.80320425e-10, cc = 2.99792458e10, me = 9.1093837015e-28, h = 6.62607015e-27;
    const T nus = 2.0 / 9.0 * (e * B / (2 * kPi * me * cc)) * Th * Th * sinb;
    const T k2 = cyl_bessel_k(2.0, 1 / Th);
    for (int c = 0; c < N; ++c) {
        const T nu = gs * kLightC * 1e9 * freq[c];  // Hz in the fluid frame
        const T X = nu / nus;
        if (!(val(X) > 0) || val(X) > 2.0e5) continue;
        const T j = ne * std::sqrt(2.0) * kPi * e * e * nus / (3 * cc * k2) *
                    sqT(sqrt(X) + std::pow(2.0, 11.0 / 12) * pow(X, 1.0 / 6)) * exp(-pow(X, 1.0 / 3));
        const T bnu = 2 * h * nu * nu * nu / (cc * cc) / expm1(h * nu / (Th * me * cc * cc));
        const T j_u = j * sc.length_cm, a_u = j / bnu * sc.length_cm;
        const T nu_nm = gs * freq[c];
        slope[8 + 2 * c] = -(1 / gs) * j_u * exp(-R[9 + 2 * c]) / (nu_nm * nu_nm * nu_nm);
        slope[9 + 2 * c] = -(1 / gs) * a_u;
    }
}

void torus_bins(const OScene& sc, RayWork& w, const double* R, double* slope) {
    torus_bins_t<double>(sc, sc.a, sc.n0, sc.b0, sc.th0, w.freq, w.N, R, slope);
}

// The van Hoof merged Gaunt-factor table of the bremsstrahlung torus
// ([146][81] float32 row-major: rows of constant log10 u from -16, columns of
// constant log10 gamma^2 from -6, 0.2 dex apart), set by oracle_set_gaunt.
static const float* g_gaunt = nullptr;

// gaunt_ei_therm_van_Hoof (emission_functions.jl:54-78), Float32 as there:
// loggam, logu rounded to Float32; frac = (log + offset) / 0.2f0 used as the
// 1-based index; floor / ceil(frac + 1f-3) neighbours; bilinear weights
// (ceil - frac), (frac - floor); 1.2 outside [1, 146] x [1, 81]. A non-finite
// argument (floor(Int32, .) would throw there) also gives 1.2.
float gaunt_van_hoof_oracle(double gam2, double u) {
    if (!g_gaunt) return 1.2f;
    const float loggam = (float)std::log10(gam2);
    const float logu = (float)std::log10(u);
    const float frac_i = (logu + 16.0f) / 0.2f;
    const float frac_j = (loggam + 6.0f) / 0.2f;
    if (!std::isfinite(frac_i) || !std::isfinite(frac_j)) return 1.2f;
    const double floor_i = std::floor((double)frac_i), floor_j = std::floor((double)frac_j);
    const double ceil_i = std::ceil((double)(frac_i + 1e-3f)), ceil_j = std::ceil((double)(frac_j + 1e-3f));
    if (!(1 <= floor_i && 1 <= floor_j && ceil_i <= 146 && ceil_j <= 81)) return 1.2f;
    auto L = [](double i, double j) { return g_gaunt[((long)i - 1) * 81 + ((long)j - 1)]; };
    const float a_i = (float)ceil_i - frac_i, b_i = frac_i - (float)floor_i;
    const float gaunt1 = a_i * L(floor_i, floor_j) + b_i * L(ceil_i, floor_j);
    const float gaunt2 = a_i * L(floor_i, ceil_j) + b_i * L(ceil_i, ceil_j);
    return ((float)ceil_j - frac_j) * gaunt1 + (frac_j - (float)floor_j) * gaunt2;
}

// RT slopes of the bremsstrahlung torus (RTW_SCENE_KERR_BREMS_TORUS; no
// reference scene, the reference's parts are C_Yar_cgs (emission_functions.jl:
// 19) and the Gaunt factor): the synchrotron torus's n_e, Theta_e, tapers and
// Keplerian velocity; j_nu = C_Yar n_e^2 Theta_e^(-1/2) exp(-u) g_ff,
// u = h nu / (Theta_e m_e c^2), gamma^2 = Ry / (Theta_e m_e c^2),
// alpha_nu = j_nu / B_nu(T_e).
void brems_bins(const OScene& sc, RayWork& w, const double* R, double* slope) {
    for (int c = 0; c < w.N; ++c) {
        slope[8 + 2 * c] = 0;
        slope[9 + 2 * c] = 0;
    }
    const double r = R[1], th = R[2];
    if (!(r >= std::max(sc.r_in - 4 * sc.edge_in, 1.01 * sc.r_ev) && r <= sc.r_out + 4 * sc.edge_out)) return;
    double taper = 1;
    if (r < sc.r_in) taper = std::exp(-sq((sc.r_in - r) / sc.edge_in));
    else if (r > sc.r_out) taper = std::exp(-sq((r - sc.r_out) / sc.edge_out));
    const double x = r / sc.r_in;
    const double zz = r * std::cos(th), hz = sc.rho_h * r;
    const double ne = sc.n0 * std::pow(x, sc.rho_idx) * std::exp(-zz * zz / (2 * hz * hz)) * taper;
    const double Th = sc.th0 * std::pow(x, sc.t_idx);
    sc.lower_metric(R, w.g);
    const double Om = std::sqrt(sc.M) / (std::pow(r, 1.5) + sc.a * std::sqrt(sc.M));
    const double n2 = -(w.g[0][0] + 2 * Om * w.g[0][3] + Om * Om * w.g[3][3]);
    if (!(n2 > 0)) return;
    const double ut = 1 / std::sqrt(n2);
    const double gs = -(ut * (w.g[0][0] + Om * w.g[0][3]) * R[4] + ut * (w.g[0][3] + Om * w.g[3][3]) * R[7]);
    if (!(gs > 0)) return;
    constexpr double cc = 2.99792458e10, me = 9.1093837015e-28, h = 6.62607015e-27;
    constexpr double ry = 2.1798723611035e-11, c_yar = 7.089314638783696e-44;
    const double kT = Th * me * cc * cc;
    for (int c = 0; c < w.N; ++c) {
        const double nu = gs * kLightC * 1e9 * w.freq[c];  // Hz in the fluid frame
        const double u = h * nu / kT;
        if (!(u > 0)) continue;
        const double gff = (double)gaunt_van_hoof_oracle(ry / kT, u);
        const double j = c_yar * ne * ne / std::sqrt(Th) * std::exp(-u) * gff;
        const double bnu = 2 * h * nu * nu * nu / (cc * cc) / std::expm1(u);
        const double nu_nm = gs * w.freq[c];
        slope[8 + 2 * c] = -(1 / gs) * j * sc.length_cm * std::exp(-R[9 + 2 * c]) / (nu_nm * nu_nm * nu_nm);
        slope[9 + 2 * c] = -(1 / gs) * j / bnu * sc.length_cm;
    }
}

// RT slopes of Powehi.source (the reference's M87* model, source_model.jl:
// region_calc :229-241, get_source_velocity! :269-317, transform_B_b :60-113,
// calc_b_angle :115-146, calc_fluid_params! :152-176,
// calc_radiative_coefficients :186-225), with the reference's constants.
// Where the jet's u^r would be the square root of a negative number (the
// reference's CPU path would throw) there is no emission.
void powehi_bins(const OScene& sc, RayWork& w, const double* R, double* slope) {
    for (int c = 0; c < w.N; ++c) {
        slope[8 + 2 * c] = 0;
        slope[9 + 2 * c] = 0;
    }
    const double r = R[1], th = R[2], M = sc.M, a = sc.a;
    int zone = 3;
    if (sc.r_in <= r && r <= sc.r_out && sc.th_lo <= th && th <= sc.th_hi) zone = 1;
    else if (r >= 10.0 && !(0.087263889 <= th && th <= 3.054236111) && (1e-3 <= th && th <= 3.1406)) zone = 2;
    if (zone == 3) return;
    sc.lower_metric(R, w.g);
    const double (*g)[4] = w.g;
    double u[4] = {0, 0, 0, 0};
    if (zone == 1) {
        const double Om = std::sqrt(M) / (std::pow(r, 1.5) + a * std::sqrt(M));
        const double D = std::pow(r, 1.5) - 3 * M * std::sqrt(r) + 2 * a * std::sqrt(M);
        u[0] = (std::pow(r, 1.5) + a * std::sqrt(M)) / (std::pow(r, 0.75) * std::sqrt(D));
        u[3] = u[0] * Om;
    } else {
        const double omega = -g[0][3] / (g[3][3] + kNoDivZero);
        const double omega_jet = 0.5 * a / (sc.rs * sc.r_ev);
        const double Om = std::min(0.9 / std::sin(th) / r, omega_jet);
        double Sig, Del, A;
        sc.kerr_params(r, th, Sig, Del, A);
        const double inv_lapse = std::sqrt(A / (Sig * Del));
        const double Gam = 1.2 + std::min((10.0 - 1.2) / (75.0 - 10.0) * (r - 10.0), 10.0);
        const double ur2 = (Gam * Gam - 1 - g[3][3] * sq(Gam * inv_lapse) * sq(Om - omega)) / g[1][1];
        if (!(ur2 > 0)) return;
        u[0] = Gam * inv_lapse;
        u[1] = std::sqrt(ur2);
        u[3] = u[0] * Om;
    }
    double fs = 0;  // calc_freq_shift
    for (int j = 0; j < 4; ++j) {
        double ps = 0;
        for (int i = 0; i < 4; ++i) ps += g[i][j] * R[i + 4];
        fs -= u[j] * ps;
    }
    if (zone == 1) {
        for (int c = 0; c < w.N; ++c) {
            const double nu = w.freq[c] * fs;
            const double a_nu = sc.anu;
            const double j_nu = a_nu * (kEmissionScale * nu * nu * nu / (std::exp(kFFactor * nu / sc.T) - 1));
            slope[8 + 2 * c] = -(1 / fs) * j_nu * std::exp(-R[9 + 2 * c]) / (nu * nu * nu);
            slope[9 + 2 * c] = -(1 / fs) * a_nu;
        }
        return;
    }
    // fluid-frame field from the global (0, 0, B^phi)
    const double B[4] = {0, 0, 0, sc.b0};
    double b[4];
    b[0] = 0;
    for (int col = 1; col < 4; ++col) {
        double ps = 0;
        for (int i = 0; i < 4; ++i) ps += g[i][col] * u[i];
        b[0] += B[col] * ps;
    }
    for (int mu = 1; mu < 4; ++mu) b[mu] = (B[mu] + b[0] * u[mu]) / u[0];
    double bmag2 = 0;
    for (int mu = 0; mu < 4; ++mu) {
        double cs = 0;
        for (int i = 0; i < 4; ++i) cs += g[i][mu];
        bmag2 += cs * b[mu] * b[mu];
    }
    bmag2 = std::max(1e-12, bmag2);
    double bk = 0;
    for (int mu = 0; mu < 4; ++mu) {
        double ps = 0;
        for (int i = 0; i < 4; ++i) ps += g[i][mu] * R[i + 4];
        bk += b[mu] * ps;
    }
    const double cos2 = std::min(bk * bk / (bmag2 * fs * fs), 1.0) + kNoDivZero;
    const double p = 2.5, gmin = 30.0, gmax = 1e9, ne0 = sc.n0, map_scale = sc.length_cm / 100.0;
    const double synch_em = 7.694e-37 * map_scale * 2.8e7, synch_ab = 2.8173e-24 * map_scale;
    const double nuc = 9.34e-11 * std::sqrt(bmag2);
    const double sinth = std::sqrt(std::max(1e-12, 1 - cos2));
    const double pfit = std::exp(7.951834e-01 + (-5.752283e-01) * p) * std::pow(p, 9.832989e-01 * p);
    const double Phi = (1 / pfit) * std::pow(1 - 0.99 * cos2, -p / 2);
    const double gd = std::pow(gmin, 1 - p) - std::pow(gmax, 1 - p);
    for (int c = 0; c < w.N; ++c) {
        const double nu = w.freq[c] * fs;
        double j_nu = ne0 * synch_em * (nuc / 9.34e-11);
        double a_nu = ne0 * synch_ab / nu;
        j_nu *= std::pow(3.0, p / 2) * (p - 1) * sinth / (2 * (p + 1) * gd);
        j_nu *= std::tgamma((3 * p - 1) / 12) * std::tgamma((3 * p + 19) / 12) * std::pow(nu / (nuc * sinth), -(p - 1) / 2);
        a_nu *= std::pow(3.0, (p + 1) / 2) * (p - 1) / (4 * gd);
        a_nu *= std::tgamma((3 * p + 2) / 12) * std::tgamma((3 * p + 22) / 12) * std::pow(nu / (nuc * sinth), -(p + 2) / 2);
        j_nu *= Phi;
        a_nu *= Phi;
        slope[8 + 2 * c] = -(1 / fs) * j_nu * std::exp(-R[9 + 2 * c]) / (nu * nu * nu);
        slope[9 + 2 * c] = -(1 / fs) * a_nu;
    }
}

// RT slopes of Synchro_Test.source (the reference's flat-space synchrotron
// test, source_model.jl: is_fire :229-236, static fluid :250-256,
// calc_B_field :47-54, transform_B_b :60-108, calc_b_angle :114-146,
// calc_fluid_params! :152-172, calc_radiative_coefficients :186-224), with
// the reference's constants, written over the general metric-contraction
// forms (g = diag(-1, 1, 1, 1), u = (1, 0, 0, 0)). A ray along the field
// (sin theta_B = 0, where the reference's j is 0 * inf) gets no emission.
void synchro_bins(const OScene& sc, RayWork& w, const double* R, double* slope) {
    for (int c = 0; c < w.N; ++c) {
        slope[8 + 2 * c] = 0;
        slope[9 + 2 * c] = 0;
    }
    if (!(std::sqrt(R[1] * R[1] + R[2] * R[2]) <= sc.r_out)) return;
    sc.lower_metric(R, w.g);
    const double (*g)[4] = w.g;
    const double u[4] = {1, 0, 0, 0};
    double fs = 0;  // calc_freq_shift
    for (int j = 0; j < 4; ++j) {
        double ps = 0;
        for (int i = 0; i < 4; ++i) ps += g[i][j] * R[i + 4];
        fs -= u[j] * ps;
    }
    const double B[4] = {0, 0, 0, sc.b0};  // (B^x, B^y, B^z) = (0, 0, 10 G)
    double b[4];
    b[0] = 0;
    for (int col = 1; col < 4; ++col) {
        double ps = 0;
        for (int i = 0; i < 4; ++i) ps += g[i][col] * u[i];
        b[0] += B[col] * ps;
    }
    for (int mu = 1; mu < 4; ++mu) b[mu] = (B[mu] + b[0] * u[mu]) / u[0];
    double bmag2 = 0;
    for (int mu = 0; mu < 4; ++mu) {
        double cs = 0;
        for (int i = 0; i < 4; ++i) cs += g[i][mu];
        bmag2 += cs * b[mu] * b[mu];
    }
    double bk = 0;
    for (int mu = 0; mu < 4; ++mu) {
        double ps = 0;
        for (int i = 0; i < 4; ++i) ps += g[i][mu] * R[i + 4];
        bk += b[mu] * ps;
    }
    const double cos2 = bk * bk / (bmag2 * fs * fs);
    if (!(1 - cos2 > 0)) return;
    const double p = 2.5, gmin = 30.0, gmax = 1e9, ne0 = sc.n0, map_scale = sc.length_cm / 100.0;
    const double synch_em = 7.694e-37 * map_scale * 2.8e7, synch_ab = 2.8173e-24 * map_scale;
    const double nuc = 9.34e-11 * std::sqrt(bmag2);
    const double sinth = std::sqrt(1 - cos2);
    const double pfit = std::exp(7.951834e-01 + (-5.752283e-01) * p) * std::pow(p, 9.832989e-01 * p);
    const double Phi = (1 / pfit) * std::pow(1 - 0.99 * cos2, -p / 2);
    const double gd = std::pow(gmin, 1 - p) - std::pow(gmax, 1 - p);
    for (int c = 0; c < w.N; ++c) {
        const double nu = w.freq[c] * fs;
        double j_nu = ne0 * synch_em * (nuc / 9.34e-11);
        double a_nu = ne0 * synch_ab / nu;
        j_nu *= std::pow(3.0, p / 2) * (p - 1) * sinth / (2 * (p + 1) * gd);
        j_nu *= std::tgamma((3 * p - 1) / 12) * std::tgamma((3 * p + 19) / 12) * std::pow(nu / (nuc * sinth), -(p - 1) / 2);
        a_nu *= std::pow(3.0, (p + 1) / 2) * (p - 1) / (4 * gd);
        a_nu *= std::tgamma((3 * p + 2) / 12) * std::tgamma((3 * p + 22) / 12) * std::pow(nu / (nuc * sinth), -(p + 2) / 2);
        j_nu *= Phi;
        a_nu *= Phi;
        slope[8 + 2 * c] = -(1 / fs) * j_nu * std::exp(-R[9 + 2 * c]) / (nu * nu * nu);
        slope[9 + 2 * c] = -(1 / fs) * a_nu;
    }
}

// calc_ray_derivative!, integrators_LttM.jl:9-48
// (over the scalar F: double; Cnt runs the thin-disk scenes only)
template <class F>
void rhs(const OScene& sc, RayWorkT<F>& w, const F* R, F* slope) {
    using std::exp;
    for (int i = 0; i < 4; ++i) slope[i] = R[i + 4];
    sc.christoffel(R, w.G);
    for (int i = 0; i < 4; ++i) {
        F acc = 0;
        for (int j = 0; j < 4; ++j)
            for (int k = 0; k < 4; ++k) acc -= w.G[i][j][k] * R[4 + j] * R[4 + k];
        slope[4 + i] = acc;
    }
    if constexpr (std::is_same<F, double>::value) {
        if (sc.kind == RTW_SCENE_KERR_SYNCHRO_TORUS) {
            torus_bins(sc, w, R, slope);
            return;
        }
        if (sc.kind == RTW_SCENE_KERR_BREMS_TORUS) {
            brems_bins(sc, w, R, slope);
            return;
        }
        if (sc.kind == RTW_SCENE_KERR_POWEHI) {
            powehi_bins(sc, w, R, slope);
            return;
        }
        if (sc.kind == RTW_SCENE_SYNCHRO_TEST) {
            synchro_bins(sc, w, R, slope);
            return;
        }
    }
    sc.lower_metric(R, w.g);
    sc.source_velocity(R, w.u);
    // calc_freq_shift, gen_geometry.jl:373-390
    F fs = 0;
    for (int j = 0; j < 4; ++j) {
        F ps = 0;
        for (int i = 0; i < 4; ++i) ps += w.g[i][j] * R[i + 4];
        fs -= w.u[j] * ps;
    }
    for (int c = 0; c < w.N; ++c) {
        const F nu = w.freq[c] * fs;
        F a_nu, j_nu;
        sc.radiative(R, nu, &a_nu, &j_nu);
        if (a_nu == 0 && j_nu == 0) {
            slope[8 + 2 * c] = 0;
            slope[9 + 2 * c] = 0;
        } else {
            slope[8 + 2 * c] = -(1.0 / fs) * j_nu * exp(-R[9 + 2 * c]) / (nu * nu * nu);
            slope[9 + 2 * c] = -(1.0 / fs) * a_nu;
        }
    }
}

// RKDP_Step_w_buffer!, integrators_LttM.jl:54-224. Returns the new step size;
// *rejected is the reject flag. counters[0] counts polar Euler sub-steps.
// (over the scalar F: double, or Cnt for the thin-disk scenes' op counts)
template <class F>
F dp45_step(const OScene& sc, RayWorkT<F>& w, F* R, F h, bool prev_rejected, bool* rejected,
            long long* escape_substeps) {
    using std::fabs;
    using std::isfinite;
    using std::max;
    using std::pow;
    using std::sqrt;
    const int L = w.L;
    F* k1 = w.last_slope.data();
    const double max_dt = sc.pad_max_dt(plain_state(w, R), w.scale);
    double temp;
    if (sc.near_singularity(plain_state(w, R), val(h), w.tol, &temp)) {
        for (int i = 0; i < L; ++i) R[i] -= temp * k1[i];
        sc.keepinbounds(R);
        if (escape_substeps) ++*escape_substeps;
        for (int it = 0; it < 36; ++it) {
            if (!sc.terminate(plain_state(w, R), L, w.tol, 2, 1)) {
                rhs(sc, w, R, k1);
                for (int j = 0; j < L; ++j) R[j] -= temp * k1[j];
                sc.keepinbounds(R);
                if (escape_substeps) ++*escape_substeps;
            }
        }
        if (sc.terminate(plain_state(w, R), L, w.tol, 2, 1)) {
            *rejected = false;
            return h;
        }
        rhs(sc, w, R, k1);
        h = -sc.pad_max_dt(plain_state(w, R), w.scale);
    }
    const auto& A = kDP.a;
    F* buf = w.buffer.data();
    F *k2 = w.k2.data(), *k3 = w.k3.data(), *k4 = w.k4.data(), *k5 = w.k5.data(), *k6 = w.k6.data(),
      *k7 = w.k7.data();
    for (int i = 0; i < L; ++i) buf[i] = R[i] + h * k1[i] * A[2][2];
    rhs(sc, w, buf, k2);
    for (int i = 0; i < L; ++i) buf[i] = R[i] + h * (k1[i] * A[3][2] + k2[i] * A[3][3]);
    rhs(sc, w, buf, k3);
    for (int i = 0; i < L; ++i) buf[i] = R[i] + h * (k1[i] * A[4][2] + k2[i] * A[4][3] + k3[i] * A[4][4]);
    rhs(sc, w, buf, k4);
    for (int i = 0; i < L; ++i)
        buf[i] = R[i] + h * (k1[i] * A[5][2] + k2[i] * A[5][3] + k3[i] * A[5][4] + k4[i] * A[5][5]);
    rhs(sc, w, buf, k5);
    for (int i = 0; i < L; ++i)
        buf[i] = R[i] + h * (k1[i] * A[6][2] + k2[i] * A[6][3] + k3[i] * A[6][4] + k4[i] * A[6][5] + k5[i] * A[6][6]);
    rhs(sc, w, buf, k6);
    F* ns = w.next_slope.data();
    for (int i = 0; i < L; ++i)
        ns[i] = k1[i] * A[7][2] + k3[i] * A[7][4] + k4[i] * A[7][5] + k5[i] * A[7][6] + k6[i] * A[7][7];
    for (int i = 0; i < L; ++i) buf[i] = R[i] + h * ns[i];
    rhs(sc, w, buf, k7);
    F* y = w.y.data();
    for (int i = 0; i < L; ++i) y[i] = R[i] + h * ns[i];
    for (int i = 0; i < L; ++i)
        buf[i] = y[i] - R[i] -
                 h * (k1[i] * A[9][2] + k3[i] * A[9][4] + k4[i] * A[9][5] + k5[i] * A[9][6] + k6[i] * A[9][7] +
                      k7[i] * A[9][8]);
    F err = 0;
    for (int i = 0; i < L; ++i) {
        const F tol = w.tol + max(fabs(R[i]), fabs(y[i])) * w.tol;
        err += sqT(buf[i] / tol);
    }
    err = sqrt(err / L);
    F hn = 0.9 * h * pow(1.0 / err, 1.0 / 5);
    if (fabs(hn) > max_dt) hn = -max_dt;
    const F* newk1 = w.fsal ? k7 : ns;
    if (err == 0 || !isfinite(hn)) {
        const double th_before = val(y[2]);
        sc.keepinbounds(y);
        for (int i = 0; i < L; ++i) {
            k1[i] = newk1[i];
            R[i] = y[i];
        }
        if ((sc.kind == RTW_SCENE_KERR_SYNCHRO_TORUS || sc.kind == RTW_SCENE_KERR_POWEHI ||
             sc.kind == RTW_SCENE_KERR_BREMS_TORUS) && w.fsal && val(y[2]) != th_before)
        rhs(sc, w, R, k1);
        *rejected = false;
        return h;
    } else if (err > 1) {
        if (prev_rejected && fabs(hn) >= fabs(h)) hn = h / 2;
        sc.keepinbounds(R);
        *rejected = true;
        return hn;
    }
    if (fabs(hn) > 5 * fabs(h)) hn = 5 * h;
    const double th_before = val(y[2]);
    sc.keepinbounds(y);
    for (int i = 0; i < L; ++i) {
        k1[i] = newk1[i];
        R[i] = y[i];
    }
    // per-bin scenes (torus, Powehi) with the FSAL step: a step reflected
    // through the pole re-evaluates the carried slope at the new state, so that
    // each step depends on its start state alone, as the library's per-bin
    // kernels do (the reference's own step keeps its carried slope)
    if ((sc.kind == RTW_SCENE_KERR_SYNCHRO_TORUS || sc.kind == RTW_SCENE_KERR_POWEHI ||
             sc.kind == RTW_SCENE_KERR_BREMS_TORUS) && w.fsal && val(y[2]) != th_before)
        rhs(sc, w, R, k1);
    *rejected = false;
    return hn;
}

// integrate_ray, LttM.jl:11-59: one ray from its initial state to its
// termination class (over the scalar F, as dp45_step); counts its step
// attempts, rejections, polar sub-steps and equatorial crossings.
template <class F>
int integrate_ray(const OScene& sc, RayWorkT<F>& w, F* ray, double max_dt_scale, double tol, long long max_steps,
                  long long* step_count, long long* rej, long long* esc, int* crossings) {
    const int L = w.L;
    F dt = -sc.pad_max_dt(plain_state(w, ray), max_dt_scale);
    rhs(sc, w, ray, w.last_slope.data());
    w.next_slope = w.last_slope;
    bool rejected = false;
    while (true) {
        bool rj = false;
        const double side = val(ray[2]) - kPi / 2;
        dt = dp45_step(sc, w, ray, dt, rejected, &rj, esc);
        if ((side < 0) != (val(ray[2]) - kPi / 2 < 0)) ++*crossings;
        rejected = rj;
        *rej += rj ? 1 : 0;
        ++*step_count;
        const int klass = sc.terminate(plain_state(w, ray), L, tol, max_steps, *step_count);
        if (klass) return klass;
    }
}

// ----------------------------------------------------------------------------
// Camera (initialization.jl:190-331, gen_geometry.jl:9-103)
// ----------------------------------------------------------------------------
typedef double Mat4[4][4];

void matmul(const Mat4 A, const Mat4 B, Mat4 C) {
    Mat4 t;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double s = 0;
            for (int k = 0; k < 4; ++k) s += A[i][k] * B[k][j];
            t[i][j] = s;
        }
    std::memcpy(C, t, sizeof(Mat4));
}

// gen_intrinsic_rotation_matrix, gen_geometry.jl:9-40
void intrinsic_rotation(const double p[3], Mat4 R) {
    Mat4 Rx = {{0}}, Ry = {{0}}, Rz = {{0}};
    Rx[0][0] = 1; Rx[1][1] = 1;
    Rx[2][2] = std::cos(p[0]); Rx[3][2] = std::sin(p[0]); Rx[2][3] = -std::sin(p[0]); Rx[3][3] = std::cos(p[0]);
    Ry[0][0] = 1;
    Ry[1][1] = std::cos(p[1]); Ry[3][1] = -std::sin(p[1]); Ry[2][2] = 1; Ry[1][3] = std::sin(p[1]);
    Ry[3][3] = std::cos(p[1]);
    Rz[0][0] = 1;
    Rz[1][1] = std::cos(p[2]); Rz[2][1] = std::sin(p[2]); Rz[1][2] = -std::sin(p[2]); Rz[2][2] = std::cos(p[2]);
    Rz[3][3] = 1;
    Mat4 t;
    matmul(Rz, Ry, t);
    matmul(t, Rx, R);
}

// gen_final_rotation_matrix, gen_geometry.jl:47-87
void final_rotation(const double dir[2], Mat4 R) {
    const double d[3] = {std::sin(dir[0]) * std::cos(dir[1]), std::sin(dir[0]) * std::sin(dir[1]), std::cos(dir[0])};
    double k[3] = {0.0 * d[2] - 1.0 * d[1], 1.0 * d[0] - 0.0 * d[2], 0.0 * d[1] - 0.0 * d[0]};
    const double mag = std::sqrt(k[0] * k[0] + k[1] * k[1] + k[2] * k[2]);
    const double yaw[3] = {0, 0, kPi / 2 + dir[1]};
    Mat4 Ri;
    intrinsic_rotation(yaw, Ri);
    if (mag > 0) {
        for (double& v : k) v /= mag;
        double K[3][3] = {{0, -k[2], k[1]}, {k[2], 0, -k[0]}, {-k[1], k[0], 0}};
        double KK[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double s = 0;
                for (int m = 0; m < 3; ++m) s += K[i][m] * K[m][j];
                KK[i][j] = s;
            }
        Mat4 R4 = {{0}};
        R4[0][0] = 1;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                R4[1 + i][1 + j] = (i == j ? 1.0 : 0.0) + std::sin(dir[0]) * K[i][j] + (1 - std::cos(dir[0])) * KK[i][j];
        Mat4 T;
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) T[i][j] = R4[j][i];
        matmul(T, Ri, R);
    } else {
        std::memcpy(R, Ri, sizeof(Mat4));
    }
}

// lorentz_boost_z, gen_geometry.jl:93-103
void boost_z(double beta, Mat4 L) {
    std::memset(L, 0, sizeof(Mat4));
    const double gamma = 1 / std::sqrt(1 - beta * beta);
    L[0][0] = gamma; L[3][0] = -beta * gamma; L[0][3] = -beta * gamma;
    L[1][1] = 1; L[2][2] = 1; L[3][3] = gamma;
}

struct CameraGeom {
    int xp = 0, yp = 0;
    double W = 0, H = 0, rh = 0, rv = 0;
    Mat4 M;  // e * R2 * L * R
    double B3[3][3];  // R2[2:4,2:4] * L[2:4,2:4] * R[2:4,2:4] (ray bundles)
};

bool camera_geom(const OScene& sc, const rtw_camera& cam, CameraGeom& cg) {
    const double fh = kPi * cam.fov_hor / 180, fv = kPi * cam.fov_vert / 180;
    cg.W = std::tan(fh / 2);
    cg.H = std::tan(fv / 2);
    cg.xp = cam.x_pix;
    cg.yp = (int)std::nearbyint(cam.x_pix * cg.H / cg.W);
    cg.rh = 2 * cg.W / (cg.xp + 1);
    cg.rv = 2 * cg.H / (cg.yp + 1);
    Mat4 R, L, R2, e, t1, t2;
    intrinsic_rotation(cam.pointing, R);
    boost_z(-cam.speed, L);
    final_rotation(cam.direction, R2);
    sc.inv_vierbein(cam.position, e);
    matmul(e, R2, t1);
    matmul(t1, L, t2);
    matmul(t2, R, cg.M);
    double RL[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            RL[a][b] = 0;
            for (int c = 0; c < 3; ++c) RL[a][b] += R2[1 + a][1 + c] * L[1 + c][1 + b];
        }
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            cg.B3[a][b] = 0;
            for (int c = 0; c < 3; ++c) cg.B3[a][b] += RL[a][c] * R[1 + c][1 + b];
        }
    return true;
}

// The ray-bundle components of pixel (i, j), 0-based, as initialize_camera
// sets them (initialization.jl:198-204, 244-249, 262-324), in the order
// b = (chi, du, dv, dg, dh, size): the shape parameters u, v, g, h, chi and
// dchi start at 0, the rates of u, v, g, h come from the bundle's major axis
// J = n x d (d = (0, 0, -1); (0, -1, 0) if |J|^2 < 1e-3) and the basis (a, b)
// normal to the ray, both after R2 L R, and the size is |beamscale n_z| with
// beamscale = atan(rho_hor) / 2. Their slopes are zero (integrators_LttM.jl:
// 43-46), so these are also their values at the ray's end.
void camera_bundle(const CameraGeom& cg, int i, int j, double* bo) {
    const double w = cg.rh * ((i + 1) - 0.5) - cg.W;
    const double h = cg.rv * ((j + 1) - 0.5) - cg.H;
    const double th = std::atan(std::sqrt(w * w + h * h));
    double ph;
    if (w > 0) ph = std::atan(h / w);
    else if (w < 0 && h >= 0) ph = std::atan(h / w) + kPi;
    else if (w < 0 && h < 0) ph = std::atan(h / w) - kPi;
    else if (w == 0 && h > 0) ph = kPi / 2;
    else if (w == 0 && h < 0) ph = -kPi / 2;
    else ph = 0;
    double n[3] = {-std::sin(th) * std::cos(ph), -std::sin(th) * std::sin(ph), -std::cos(th)};
    const double beamscale = std::atan(cg.rh) / 2;
    const double size = std::fabs(beamscale * n[2]);
    const double d[3] = {0.0, 0.0, -1.0};
    const double E = 1.0 / (std::fabs(n[2]) + kNoDivZero);
    double J[3] = {n[1] * d[2] - n[2] * d[1], n[2] * d[0] - n[0] * d[2], n[0] * d[1] - n[1] * d[0]};
    if (J[0] * J[0] + J[1] * J[1] + J[2] * J[2] < 1e-3) {
        J[0] = 0.0; J[1] = -1.0; J[2] = 0.0;
    }
    double J2[3], n2[3];
    for (int a = 0; a < 3; ++a) {
        J2[a] = cg.B3[a][0] * J[0] + cg.B3[a][1] * J[1] + cg.B3[a][2] * J[2];
        n2[a] = cg.B3[a][0] * n[0] + cg.B3[a][1] * n[1] + cg.B3[a][2] * n[2];
    }
    const double jj = std::sqrt(J2[0] * J2[0] + J2[1] * J2[1] + J2[2] * J2[2]);
    const double nn = std::sqrt(n2[0] * n2[0] + n2[1] * n2[1] + n2[2] * n2[2]);
    for (int a = 0; a < 3; ++a) {
        J2[a] = J2[a] / jj;
        n2[a] = n2[a] / nn;
    }
    double av[3], bv[3];
    if (!(std::fabs(1 - n2[0]) < 1e-3)) {
        av[0] = n2[1]; av[1] = 1 - n2[1] * n2[1] / (1 - n2[0]); av[2] = -n2[1] * n2[2] / (1 - n2[0]);
        const double aa = av[0] * av[0] + av[1] * av[1] + av[2] * av[2];
        for (double& v : av) v = v / aa;
        bv[0] = n2[2]; bv[1] = -n2[1] * n2[2] / (1 - n2[0]); bv[2] = 1 - n2[2] * n2[2] / (1 - n2[0]);
        const double bb = bv[0] * bv[0] + bv[1] * bv[1] + bv[2] * bv[2];
        for (double& v : bv) v = v / bb;
    } else {
        av[0] = 0.0; av[1] = -1.0; av[2] = 0.0;
        bv[0] = 0.0; bv[1] = 0.0; bv[2] = -1.0;
    }
    const double aJ = av[0] * J2[0] + av[1] * J2[1] + av[2] * J2[2];
    const double bJ = bv[0] * J2[0] + bv[1] * J2[1] + bv[2] * J2[2];
    bo[0] = 0;
    bo[1] = aJ * (1 + E) / 2;
    bo[2] = bJ * (1 + E) / 2;
    bo[3] = aJ * (1 - E) / 2;
    bo[4] = bJ * (1 - E) / 2;
    bo[5] = size;
}

// Initial state of pixel (i, j), 0-based (initialization.jl:213-240,327).
void camera_ray(const CameraGeom& cg, const rtw_camera& cam, int i, int j, double* S) {
    const double w = cg.rh * ((i + 1) - 0.5) - cg.W;
    const double h = cg.rv * ((j + 1) - 0.5) - cg.H;
    const double th = std::atan(std::sqrt(w * w + h * h));
    double ph;
    if (w > 0) ph = std::atan(h / w);
    else if (w < 0 && h >= 0) ph = std::atan(h / w) + kPi;
    else if (w < 0 && h < 0) ph = std::atan(h / w) - kPi;
    else if (w == 0 && h > 0) ph = kPi / 2;
    else if (w == 0 && h < 0) ph = -kPi / 2;
    else ph = 0;
    const double v[4] = {1, -std::sin(th) * std::cos(ph), -std::sin(th) * std::sin(ph), -std::cos(th)};
    for (int k = 0; k < 4; ++k) S[k] = cam.position[k];
    for (int r = 0; r < 4; ++r) {
        double s = 0;
        for (int k = 0; k < 4; ++k) s += cg.M[r][k] * v[k];
        S[4 + r] = s;
    }
}

// ----------------------------------------------------------------------------
// The synchrotron torus's render over the scalar type T (double: the same
// arithmetic as the render loop above; D5: forward-mode tangents). Restates,
// for the Kerr torus only: calc_ray_derivative! (integrators_LttM.jl:9-48),
// RKDP_Step_w_buffer! with the FSAL step (integrators_LttM.jl:54-224),
// pad_max_dt (Kerr model :86-103), near_singularity (Kerr geometry :249-269),
// keepinbounds! (:275-301) and the camera (initialization.jl:190-331) with
// the Kerr inverse vierbein (:112-121).
//
// Step sizes: mode 1 carries tangents through every step size, the
// controller's err^(-1/5) included (what forward-mode differentiation of the
// whole program gives). Mode 0 keeps a step size's tangent only where it is
// -pad_max_dt (the first step, after a polar escape, and where the
// controller's proposal is capped by max_dt) and holds the controller's own
// choices fixed: the convention of the discrete adjoint.
// ----------------------------------------------------------------------------
template <class T>
struct TorusFwd {
    const OScene& sc;
    T al, n0, b0, th0;  // spin and the emission parameters, with their tangents
    const double* freq;
    int N, L;
    double tol, scale;
    int mode;
    std::vector<T> k1, buf, y, k2, k3, k4, k5, k6, k7, ns;

    TorusFwd(const OScene& s, int n, const double* f, double tol_, double scale_, int mode_)
        : sc(s), freq(f), N(n), L(8 + 2 * n), tol(tol_), scale(scale_), mode(mode_) {
        for (auto* v : {&k1, &buf, &y, &k2, &k3, &k4, &k5, &k6, &k7, &ns}) v->assign(L, T(0));
    }

    void rhs(const T* R, T* slope) const {
        for (int i = 0; i < 4; ++i) slope[i] = R[i + 4];
        T G[4][4][4];
        for (auto& a : G)
            for (auto& b : a)
                for (auto& c : b) c = 0;
        sc.kerr_christoffel<T, T>(R[1], R[2], al, T(sc.rs), G);
        for (int i = 0; i < 4; ++i) {
            T acc = 0;
            for (int j = 0; j < 4; ++j)
                for (int k = 0; k < 4; ++k) acc -= G[i][j][k] * R[4 + j] * R[4 + k];
            slope[4 + i] = acc;
        }
        torus_bins_t<T>(sc, al, n0, b0, th0, freq, N, R, slope);
    }

    static T tmin(const T& a, const T& b) { return val(b) < val(a) ? b : a; }
    static T tmax(const T& a, const T& b) { return val(a) < val(b) ? b : a; }

    T pad_max_dt(const T* x) const {
        using std::fabs;
        const double sc32 = (double)(float)scale;
        double eps;
        if (val(x[2]) < kPi / 8 || val(x[2]) > 7 * kPi / 8) eps = std::min(sc32, (double)1e-1f);
        else eps = sc32;
        const T first = fabs(1.0 / (eps / fabs(x[5]))) + kNoDivZero;
        const T second = fabs(1.0 / (eps * tmin(x[2], kPi - x[2]) / (fabs(x[6]) + kNoDivZero) + kNoDivZero));
        const T third = fabs(1.0 / (eps / (fabs(x[7]) + kNoDivZero) + kNoDivZero));
        T m = tmin(1.0 / (first + second + third + kNoDivZero), T(0.5));
        return tmax(m, T((double)1e-12f));
    }

    bool near_singularity(const T* x, const T& h, T* temp) const {
        using std::fabs;
        const T th_new = x[2] + h * x[6];
        if (val(fabs(th_new)) <= tol) {
            *temp = 2 * fabs(x[2]) / (fabs(x[6] * 37) + kNoDivZero);
            return true;
        } else if (val(fabs(th_new - kPi)) <= tol) {
            *temp = 2 * fabs((x[2] - kPi) / (fabs(x[6] * 37) + kNoDivZero));
            return true;
        }
        *temp = h;
        return false;
    }

    void keepinbounds(T* x) const {
        if (val(x[2]) < 0) {
            x[2] = -x[2];
            x[3] = x[3] - kPi;
            x[6] = -x[6];
        }
        const double m = jl_mod(val(x[2]), 2 * kPi);
        x[2] = x[2] + (m - val(x[2]));  // mod(theta, 2 pi): the shift carries no tangent
        if (val(x[2]) >= kPi) {
            x[2] = 2 * kPi - x[2];
            x[3] = x[3] + kPi;
            x[6] = -x[6];
        }
    }

    int terminate(const T* R, long long max_steps, long long step_count) const {
        std::vector<double> v(L);
        for (int i = 0; i < L; ++i) v[i] = val(R[i]);
        return sc.terminate(v.data(), L, tol, max_steps, step_count);
    }

    // a step size the controller chose: mode 0 keeps the tangent of -max_dt only
    T held(const T& hn, const T& max_dt) const {
        if (mode == 1) return hn;
        if (val(hn) == val(-max_dt)) return -max_dt;
        return T(val(hn));
    }

    // one call of RKDP_Step_w_buffer! with the FSAL step (the torus's)
    T step(T* R, T h, bool prev_rejected, bool* rejected, long long* esc) {
        using std::fabs;
        using std::pow;
        using std::sqrt;
        const T max_dt = pad_max_dt(R);
        T temp;
        if (near_singularity(R, h, &temp)) {
            for (int i = 0; i < L; ++i) R[i] = R[i] - temp * k1[i];
            keepinbounds(R);
            ++*esc;
            for (int it = 0; it < 36; ++it) {
                if (!terminate(R, 2, 1)) {
                    rhs(R, k1.data());
                    for (int j = 0; j < L; ++j) R[j] = R[j] - temp * k1[j];
                    keepinbounds(R);
                    ++*esc;
                }
            }
            if (terminate(R, 2, 1)) {
                *rejected = false;
                return h;
            }
            rhs(R, k1.data());
            h = -pad_max_dt(R);
        }
        const auto& A = kDP.a;
        for (int i = 0; i < L; ++i) buf[i] = R[i] + h * k1[i] * A[2][2];
        rhs(buf.data(), k2.data());
        for (int i = 0; i < L; ++i) buf[i] = R[i] + h * (k1[i] * A[3][2] + k2[i] * A[3][3]);
        rhs(buf.data(), k3.data());
        for (int i = 0; i < L; ++i) buf[i] = R[i] + h * (k1[i] * A[4][2] + k2[i] * A[4][3] + k3[i] * A[4][4]);
        rhs(buf.data(), k4.data());
        for (int i = 0; i < L; ++i)
            buf[i] = R[i] + h * (k1[i] * A[5][2] + k2[i] * A[5][3] + k3[i] * A[5][4] + k4[i] * A[5][5]);
        rhs(buf.data(), k5.data());
        for (int i = 0; i < L; ++i)
            buf[i] = R[i] + h * (k1[i] * A[6][2] + k2[i] * A[6][3] + k3[i] * A[6][4] + k4[i] * A[6][5] +
                                 k5[i] * A[6][6]);
        rhs(buf.data(), k6.data());
        for (int i = 0; i < L; ++i)
            ns[i] = k1[i] * A[7][2] + k3[i] * A[7][4] + k4[i] * A[7][5] + k5[i] * A[7][6] + k6[i] * A[7][7];
        for (int i = 0; i < L; ++i) buf[i] = R[i] + h * ns[i];
        rhs(buf.data(), k7.data());
        for (int i = 0; i < L; ++i) y[i] = R[i] + h * ns[i];
        T err = 0;
        for (int i = 0; i < L; ++i) {
            const T d = y[i] - R[i] -
                        h * (k1[i] * A[9][2] + k3[i] * A[9][4] + k4[i] * A[9][5] + k5[i] * A[9][6] +
                             k6[i] * A[9][7] + k7[i] * A[9][8]);
            const T tl = tol + tmax(fabs(R[i]), fabs(y[i])) * tol;
            err = err + sqT(d / tl);
        }
        err = sqrt(err / L);
        T hn = 0.9 * h * pow(1.0 / err, 1.0 / 5);
        if (val(fabs(hn)) > val(max_dt)) hn = -max_dt;
        if (val(err) == 0 || !std::isfinite(val(hn))) {
            const double th_before = val(y[2]);
            keepinbounds(y.data());
            for (int i = 0; i < L; ++i) {
                k1[i] = k7[i];
                R[i] = y[i];
            }
            if (val(y[2]) != th_before) rhs(R, k1.data());
            *rejected = false;
            return held(h, max_dt);
        } else if (val(err) > 1) {
            if (prev_rejected && val(fabs(hn)) >= val(fabs(h))) hn = h / 2;
            keepinbounds(R);
            *rejected = true;
            return held(hn, max_dt);
        }
        if (val(fabs(hn)) > 5 * val(fabs(h))) hn = 5 * h;
        const double th_before = val(y[2]);
        keepinbounds(y.data());
        for (int i = 0; i < L; ++i) {
            k1[i] = k7[i];
            R[i] = y[i];
        }
        if (val(y[2]) != th_before) rhs(R, k1.data());
        *rejected = false;
        return held(hn, max_dt);
    }
};

// ----------------------------------------------------------------------------
// CIE (color_theory.jl)
// ----------------------------------------------------------------------------
const double kCie[4][7] = {
    {0.362, 1.056, -0.065, 0.821, 0.286, 1.217, 0.681},
    {442.0, 599.8, 501.1, 568.8, 530.9, 437.0, 459.0},
    {0.0624, 0.0264, 0.0490, 0.0213, 0.0613, 0.0845, 0.0385},
    {0.0374, 0.0323, 0.0382, 0.0247, 0.0322, 0.0278, 0.0725}};

inline double heaviside(double x) { return x >= 0 ? 1.0 : 0.0; }
inline double selector(double x, double y, double z) { return y * (1 - heaviside(x)) + z * heaviside(x); }
double cie_lobes(double wl, int first, int n) {
    double s = 0;
    for (int i = first; i < first + n; ++i) {
        const double d = wl - kCie[1][i];
        s = s + kCie[0][i] * std::exp((-1.0 / 2) * sq(d * selector(d, kCie[2][i], kCie[3][i])));
    }
    return s;
}

void cie_weights(const double* colors, int n, double* wx, double* wy, double* wz, double* fac) {
    for (int i = 0; i < n; ++i) {
        double w;
        if (n == 1) w = 1.0;
        else if (i == 0) w = (colors[1] - colors[0]) / 2;
        else if (i == n - 1) w = (colors[n - 1] - colors[n - 2]) / 2;
        else w = (colors[i + 1] - colors[i - 1]) / 2;
        wx[i] = cie_lobes(colors[i], 0, 3) * w;
        wy[i] = cie_lobes(colors[i], 3, 2) * w;
        wz[i] = cie_lobes(colors[i], 5, 2) * w;
        const double f = 1.0 / colors[i];
        fac[i] = f * f * f * kLightC / (colors[i] * colors[i]);
    }
}

}  // namespace

// ----------------------------------------------------------------------------
// C API for tests (ctypes). Outputs are double precision.
// ----------------------------------------------------------------------------
// Skyboxes of the wormhole (set by oracle_set_skybox): cube maps in the
// reference's cross layout, 3h rows x 4h columns x RGB, row 0 at the top.
static const float* g_sky[2] = {nullptr, nullptr};
static int g_sky_h[2] = {0, 0};
static int g_bundles = 0;
// per-pixel diagnostics of the next oracle_render (NULL: not recorded): the
// number of accepted steps and polar escapes that carry the ray across the
// equatorial plane theta = pi/2, and the polar Euler sub-steps it took
static int* g_diag_cross = nullptr;
static int* g_diag_escape = nullptr;

inline double normal_gauss(double x, double s, double m) {  // my_special_functions.jl:20-22
    return std::exp(-(x - m) * (x - m) / (2 * s * s)) / (s * std::sqrt(2 * kPi));
}

// cube_wrap (gen_geometry.jl:128-344), branch by branch: face, then the
// axis of a one-axis move, then the side it leaves by; a diagonal move is two
// one-axis moves in the reference's order.
void cube_wrap(int i1, int j1, int F1, int x, int y, int N, int& i2, int& j2, int& F2) {
    auto m1 = [N](int v) { return ((v - 1) % N + N) % N + 1; };  // mod1
    i2 = i1; j2 = j1; F2 = F1;
    if (!(x != 0 && y != 0)) {
        if (x != 0) {
            const int s = i1 + x;
            if (s >= 1 && s <= N) { i2 = s; return; }
            const bool hi = s > N;
            switch (F1) {
            case 1: i2 = m1(s); F2 = hi ? 2 : 4; break;
            case 2: i2 = m1(s); F2 = hi ? 3 : 1; break;
            case 3: i2 = m1(s); F2 = hi ? 4 : 2; break;
            case 4: i2 = m1(s); F2 = hi ? 1 : 3; break;
            case 5:
                if (hi) { i2 = N - j1 + 1; j2 = m1(s); F2 = 3; }
                else { i2 = j1; j2 = 1 - i1 - x; F2 = 1; }
                break;
            case 6:
                if (hi) { i2 = j1; j2 = N - m1(s) + 1; F2 = 3; }
                else { i2 = N - j1 + 1; j2 = N - i1 - x; F2 = 1; }
                break;
            }
        } else {
            const int t = j1 + y;
            if (t >= 1 && t <= N) { j2 = t; return; }
            const bool hi = t > N;
            switch (F1) {
            case 1:
                if (hi) { i2 = m1(t); j2 = N + 1 - i1; F2 = 6; }
                else { i2 = 1 - j1 - y; j2 = i1; F2 = 5; }
                break;
            case 2: j2 = m1(t); F2 = hi ? 6 : 5; break;
            case 3:
                if (hi) { i2 = N - m1(t) + 1; j2 = i1; F2 = 6; }
                else { i2 = N + j1 + y; j2 = N - i1 + 1; F2 = 5; }
                break;
            case 4:
                if (hi) { i2 = N - i1 + 1; j2 = N - m1(t) + 1; F2 = 6; }
                else { i2 = N - i1 + 1; j2 = 1 - j1 - y; F2 = 5; }
                break;
            case 5:
                if (hi) { j2 = m1(t); F2 = 2; }
                else { i2 = N - i1 + 1; j2 = 1 - j1 - y; F2 = 4; }
                break;
            case 6:
                if (hi) { i2 = N - i1 + 1; j2 = N - m1(t) + 1; F2 = 4; }
                else { j2 = m1(t); F2 = 2; }
                break;
            }
        }
        return;
    }
    int ia, ja, Fa;
    cube_wrap(i1, j1, F1, x, 0, N, ia, ja, Fa);
    const bool lo = i1 + x < 1, hi = i1 + x > N;
    if (F1 == 6 && lo) cube_wrap(ia, ja, Fa, -y, 0, N, i2, j2, F2);
    else if (F1 == 6 && hi) cube_wrap(ia, ja, Fa, y, 0, N, i2, j2, F2);
    else if (F1 == 5 && hi) cube_wrap(ia, ja, Fa, -y, 0, N, i2, j2, F2);
    else if (F1 == 5 && lo) cube_wrap(ia, ja, Fa, y, 0, N, i2, j2, F2);
    else cube_wrap(ia, ja, Fa, 0, y, N, i2, j2, F2);
}

void cubemap_coord(int i, int j, int F, int N, int& ia, int& ja) {  // cubemap_coord_calc
    ia = i; ja = j;
    if (F == 1) ja += N;
    else if (F == 2) { ia += N; ja += N; }
    else if (F == 3) { ia += 2 * N; ja += N; }
    else if (F == 4) { ia += 3 * N; ja += N; }
    else if (F == 5) ia += N;
    else { ia += N; ja += 2 * N; }
}

// skybox_I_nu_calc (Wormhole.source/source_model.jl:150-172) at
// cross-layout texel (i, j) of map k
double skybox_I(int k, int i, int j, double f) {
    const int H = g_sky_h[k];
    const float* t = g_sky[k] + ((3LL * H - j) * 4LL * H + (i - 1)) * 3;
    const double Rc = 1.0 * t[0], Gc = 0.843 * t[1], Bc = 0.914 * t[2];
    return 1e-12 * (Rc * normal_gauss(f, 5e-5, 0.001587) + Gc * normal_gauss(f, 7e-5, 0.001879) +
                    Bc * normal_gauss(f, 9e-5, 0.002141));
}

// D2_Gauss and distort_gauss (my_special_functions.jl:28-52)
double d2_gauss(double x, double y, double sx, double sy, double t) {
    const double c = std::cos(t), s = std::sin(t);
    const double a = c * c / (2 * sx * sx) + s * s / (2 * sy * sy);
    const double b = -s * c / (2 * sx * sx) + s * c / (2 * sy * sy);
    const double cc = s * s / (2 * sx * sx) + c * c / (2 * sy * sy);
    return 1.0 / (2 * kPi * sx * sy) * std::exp(-(a * x * x + 2 * b * x * y + cc * y * y));
}

void distort_gauss(double sx, double sy, double t, double a, double b, double& sxo, double& syo, double& to) {
    const double c = std::cos(t), s = std::sin(t);
    const double xx = a * a * (sx * sx * c * c + sy * sy * s * s);
    const double yy = b * b * (sx * sx * s * s + sy * sy * c * c);
    const double xy = a * b * (sx * sx - sy * sy) * std::sin(2 * t) / 2;
    const double r = std::sqrt((xx - yy) * (xx - yy) + 4 * xy * xy);
    sxo = std::sqrt((xx + yy + r) / 2);
    syo = std::sqrt((xx + yy - r) / 2);
    to = std::atan2(2 * xy, xx - yy) / 2;
}

// skybox_handling! (Wormhole.source/source_model.jl:393-443):
// calc_skybox_coord (:175-263, R_sph_to_cart gen_geometry.jl:110-122),
// cubemap_coord_calc (gen_geometry.jl:347-370), skybox_I_nu_calc (:150-172);
// with a bundle b (camera_bundle's layout), calc_skybox_I_nu_beam! (:266-358).
// Texels that wrap off the map (faces under 10 texels; the reference stops
// with an index error) and a footprint with a NaN width add nothing.
// Minkowski_Sphere_Cartesian.source/source_model.jl:175-431: the same lookup
// at every ray's end, skybox 1, the velocity already Cartesian.
void wormhole_skybox(const OScene& sc, double* ray, int N, const double* freq, const double* bund) {
    int k = 0;
    double v[4] = {0, 0, 0, 0};
    if (sc.kind == RTW_SCENE_MINKOWSKI_CART_SPHERE) {
        for (int a = 0; a < 4; ++a) v[a] = ray[4 + a];
    } else {
        const double rl = sc.wh_r(ray[1]);
        if (!(rl > 50) || ray[1] == 0) return;
        k = ray[1] > 0 ? 0 : 1;
        const double th = ray[2], ph = ray[3];
        const double e[4] = {ray[4], ray[5], rl * ray[6], rl * std::sin(th) * ray[7]};
        double R[4][4] = {};
        R[0][0] = 1;
        R[1][1] = std::sin(th) * std::cos(ph); R[1][2] = std::cos(th) * std::cos(ph); R[1][3] = -std::sin(ph);
        R[2][1] = std::sin(th) * std::sin(ph); R[2][2] = std::cos(th) * std::sin(ph); R[2][3] = std::cos(ph);
        R[3][1] = std::cos(th); R[3][2] = -std::sin(th);
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) v[a] += R[a][b] * e[b];
    }
    if (!g_sky[k]) return;
    for (int a = 0; a < 4; ++a)
        if (!std::isfinite(v[a])) return;  // a NaN ray (the reference stops with an error)
    const int H = g_sky_h[k];
    const double nv = std::sqrt(v[1] * v[1] + v[2] * v[2] + v[3] * v[3]);
    const double x = v[1] / nv, y = v[2] / nv, z = v[3] / nv;
    int face;
    if (std::fabs(x) >= std::fabs(y) && std::fabs(x) >= std::fabs(z)) face = x > 0 ? 1 : 3;
    else if (std::fabs(y) >= std::fabs(x) && std::fabs(y) >= std::fabs(z)) face = y > 0 ? 4 : 2;
    else face = z > 0 ? 6 : 5;
    double u, w;
    switch (face) {
    case 1: u = -y / std::fabs(x); w = z / std::fabs(x); break;
    case 2: u = -x / std::fabs(y); w = z / std::fabs(y); break;
    case 3: u = y / std::fabs(x); w = z / std::fabs(x); break;
    case 4: u = x / std::fabs(y); w = z / std::fabs(y); break;
    case 5: u = -x / std::fabs(z); w = -y / std::fabs(z); break;
    default: u = -x / std::fabs(z); w = y / std::fabs(z); break;
    }
    long long i = std::min((long long)std::floor(H * (u + 1) / 2) + 1, (long long)H);
    long long j = std::min((long long)std::floor(H * (w + 1) / 2) + 1, (long long)H);
    switch (face) {
    case 1: j += H; break;
    case 2: i += H; j += H; break;
    case 3: i += 2 * H; j += H; break;
    case 4: i += 3 * H; j += H; break;
    case 5: i += H; break;
    default: i += H; j += 2 * H; break;
    }
    const double fs = ray[4];  // -g(u, k) with u = (1, 0, 0, 0), g_tt = -1
    if (bund) {
        // face-local (i, j): undo the cross offsets taken above
        int il = (int)i, jl = (int)j;
        switch (face) {
        case 1: jl -= H; break;
        case 2: il -= H; jl -= H; break;
        case 3: il -= 2 * H; jl -= H; break;
        case 4: il -= 3 * H; jl -= H; break;
        case 5: il -= H; break;
        default: il -= H; jl -= 2 * H; break;
        }
        const double dprime = bund[5] * fs;
        const double A = std::sqrt(bund[1] * bund[1] + bund[2] * bund[2]);
        const double B = std::sqrt(bund[3] * bund[3] + bund[4] * bund[4]);
        const double dmaj = dprime * (A + B), dmin = dprime * (A - B);
        const double mu = bund[0] + std::arg(std::complex<double>(bund[1], bund[2]) *
                                             std::complex<double>(bund[3], bund[4])) / 2;
        const double sky_beamscale = std::atan(2.0 / (H + 1)) / 2;
        double sx, sy, tn;
        distort_gauss(dmaj, dmin, mu, 1.0 / (sky_beamscale + kNoDivZero), 1.0 / (sky_beamscale + kNoDivZero), sx, sy,
                      tn);
        if (!(sx > 0 && sy > 0 && std::isfinite(sx) && std::isfinite(sy))) return;
        const int hw = (int)std::min(std::ceil(std::max(sx, sy)), 10.0);
        std::vector<double> In(N, 0.0);
        for (int kk = -hw; kk <= hw; ++kk)
            for (int ll = -hw; ll <= hw; ++ll) {
                int iw, jw, Fw, ia, ja;
                cube_wrap(il, jl, face, kk, ll, H, iw, jw, Fw);
                cubemap_coord(iw, jw, Fw, H, ia, ja);
                if (ia < 1 || ia > 4 * H || ja < 1 || ja > 3 * H) continue;
                for (int c = 0; c < N; ++c) {
                    const double f = freq[c] * fs;
                    In[c] += d2_gauss(kk, ll, sx, sy, tn) * skybox_I(k, ia, ja, f) * std::exp(-ray[9 + 2 * c]) /
                             (f * f * f);
                }
            }
        for (int c = 0; c < N; ++c) ray[8 + 2 * c] += In[c];
        return;
    }
    for (int c = 0; c < N; ++c) {
        const double f = freq[c] * fs;
        ray[8 + 2 * c] += skybox_I(k, (int)i, (int)j, f) * std::exp(-ray[9 + 2 * c]) / (f * f * f);
    }
}

extern "C" {

// the wormhole's skybox k (0: positive-l side, 1: negative), h pixels per
// face edge (tex NULL: none); kept until changed
int oracle_set_ray_bundles(int on) {  // gen_image's ray_bundles; kept until changed
    g_bundles = on ? 1 : 0;
    return RTW_OK;
}

int oracle_cube_wrap(int i, int j, int face, int x, int y, int n, int* out) {
    if (!out || n < 1 || face < 1 || face > 6) return RTW_ERR_INVALID_PARAM;
    cube_wrap(i, j, face, x, y, n, out[0], out[1], out[2]);
    return RTW_OK;
}

// per-pixel diagnostics of the next renders (NULL: off); kept until changed
int oracle_set_diagnostics(int* crossings, int* escape_substeps) {
    g_diag_cross = crossings;
    g_diag_escape = escape_substeps;
    return RTW_OK;
}

// the bremsstrahlung torus's Gaunt-factor table ([146][81] float32; NULL: none); kept until changed
int oracle_set_gaunt(const float* lut) {
    g_gaunt = lut;
    return RTW_OK;
}

// the oracle's own Gaunt factor at gam2 and u (the table set by oracle_set_gaunt)
float oracle_gaunt(double gam2, double u) { return gaunt_van_hoof_oracle(gam2, u); }

int oracle_set_skybox(int k, const float* tex, int h) {
    if (k < 0 || k > 1 || (tex && h < 1)) return RTW_ERR_INVALID_PARAM;
    g_sky[k] = tex;
    g_sky_h[k] = tex ? h : 0;
    return RTW_OK;
}


// Forward-mode tangents of the synchrotron torus's render (FSAL step): per
// pixel the spectrum (I per bin) and dI/d(spin, inclination, n_e0, b_0,
// theta_e0) [n][n_colors][5], inclination in radians (the camera's theta).
// mode 0: the discrete adjoint's convention for step sizes, 1: tangents
// through every step size (see TorusFwd). Optional class, step counts and
// polar Euler sub-steps per pixel.
int oracle_torus_forward(const rtw_scene* scene, rtw_camera* cam, const double* colors_nm, int n_colors,
                         double max_dt_scale, int mode, const long long* pixel_ids, long long n_ids,
                         double* spectrum, double* tangents, unsigned char* cls, unsigned int* steps, int* escapes,
                         int n_threads) {
    if (!scene || !cam || !colors_nm || n_colors <= 0 || n_colors > RTW_MAX_BINS) return RTW_ERR_INVALID_PARAM;
    if (scene->kind != RTW_SCENE_KERR_SYNCHRO_TORUS || (mode != 0 && mode != 1)) return RTW_ERR_UNSUPPORTED;
    if (cam->speed != 0) return RTW_ERR_UNSUPPORTED;  // a static camera: theta is the inclination
    OScene sc(*scene);
    if (sc.is_singularity(cam->position)) return RTW_ERR_INVALID_CAMERA;
    CameraGeom cg;
    camera_geom(sc, *cam, cg);
    cam->y_pix = cg.yp;
    const long long P = (long long)cg.xp * cg.yp;
    const long long n = pixel_ids ? n_ids : P;
    // e R2 L R as camera_geom forms it; only the inverse vierbein carries tangents
    Mat4 Rm, Lm, R2;
    intrinsic_rotation(cam->pointing, Rm);
    boost_z(-cam->speed, Lm);
    final_rotation(cam->direction, R2);
    D5 al(sc.a), thc(cam->position[2]), n0(sc.n0), b0(sc.b0), th0(sc.th0);
    al.d[0] = 1;
    thc.d[1] = 1;
    n0.d[2] = 1;
    b0.d[3] = 1;
    th0.d[4] = 1;
    D5 e[4][4];
    {
        using std::cos;
        using std::sin;
        using std::sqrt;
        const D5 r(cam->position[1]);
        const D5 Sig = r * r + sqT(al * cos(thc));
        const D5 Del = r * r - r * sc.rs + al * al;
        const D5 A = (r * r + al * al) * Sig + sc.rs * r * sqT(al * sin(thc));
        e[0][0] = sqrt(A / (Sig * Del));
        e[3][0] = (sc.rs * al * r / A) * e[0][0];
        e[1][1] = sqrt(Del / Sig);
        e[2][2] = 1.0 / sqrt(Sig);
        e[3][3] = sqrt(Sig / A) / sin(thc);
    }
    auto mul = [](const D5 a[4][4], const Mat4 b, D5 c[4][4]) {
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) {
                D5 acc = 0;
                for (int k = 0; k < 4; ++k) acc += a[i][k] * b[k][j];
                c[i][j] = acc;
            }
    };
    D5 t1[4][4], t2[4][4], M[4][4];
    mul(e, R2, t1);
    mul(t1, Lm, t2);
    mul(t2, Rm, M);
    std::vector<double> freq(n_colors);
    for (int c = 0; c < n_colors; ++c) freq[c] = 1.0 / colors_nm[c];
    const int N = n_colors, L = 8 + 2 * N;
    const double tol = cam->tolerance;
    const long long max_steps = cam->max_steps;
    const int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1)
    for (long long q = 0; q < n; ++q) {
        TorusFwd<D5> w(sc, N, freq.data(), tol, max_dt_scale, mode);
        w.al = al;
        w.n0 = n0;
        w.b0 = b0;
        w.th0 = th0;
        const long long p = pixel_ids ? pixel_ids[q] : q;
        const int i = (int)(p % cg.xp), j = (int)(p / cg.xp);
        const double wq = cg.rh * ((i + 1) - 0.5) - cg.W;
        const double hq = cg.rv * ((j + 1) - 0.5) - cg.H;
        const double th = std::atan(std::sqrt(wq * wq + hq * hq));
        double ph;
        if (wq > 0) ph = std::atan(hq / wq);
        else if (wq < 0 && hq >= 0) ph = std::atan(hq / wq) + kPi;
        else if (wq < 0 && hq < 0) ph = std::atan(hq / wq) - kPi;
        else if (wq == 0 && hq > 0) ph = kPi / 2;
        else if (wq == 0 && hq < 0) ph = -kPi / 2;
        else ph = 0;
        const double v[4] = {1, -std::sin(th) * std::cos(ph), -std::sin(th) * std::sin(ph), -std::cos(th)};
        std::vector<D5> ray(L, D5(0.0));
        ray[0] = cam->position[0];
        ray[1] = cam->position[1];
        ray[2] = thc;
        ray[3] = cam->position[3];
        for (int rr = 0; rr < 4; ++rr) {
            D5 acc = 0;
            for (int k = 0; k < 4; ++k) acc += M[rr][k] * v[k];
            ray[4 + rr] = acc;
        }
        D5 dt = -w.pad_max_dt(ray.data());
        w.rhs(ray.data(), w.k1.data());
        bool rejected = false;
        long long step_count = 0, esc = 0;
        int klass = 0;
        while (true) {
            bool rj = false;
            dt = w.step(ray.data(), dt, rejected, &rj, &esc);
            rejected = rj;
            ++step_count;
            klass = w.terminate(ray.data(), max_steps, step_count);
            if (klass) break;
        }
        for (int k = 0; k < 8; ++k)
            if (!std::isfinite(ray[k].v)) klass = RTW_CLASS_NAN;
        if (cls) cls[q] = (unsigned char)klass;
        if (steps) steps[q] = (unsigned int)step_count;
        if (escapes) escapes[q] = (int)esc;
        for (int c = 0; c < N; ++c) {
            if (spectrum) spectrum[(long long)N * q + c] = ray[8 + 2 * c].v;
            if (tangents)
                for (int t = 0; t < kTan; ++t) tangents[((long long)N * q + c) * kTan + t] = ray[8 + 2 * c].d[t];
        }
    }
    return RTW_OK;
}

int oracle_abi_version(void) { return RTW_ABI_VERSION; }

int oracle_cie(const double* colors, int n, double* wx, double* wy, double* wz, double* fac) {
    if (!colors || n <= 0) return RTW_ERR_INVALID_PARAM;
    cie_weights(colors, n, wx, wy, wz, fac);
    return RTW_OK;
}

double oracle_cie_eval(int which, double wl) {
    if (which == 0) return cie_lobes(wl, 0, 3);
    if (which == 1) return cie_lobes(wl, 3, 2);
    return cie_lobes(wl, 5, 2);
}

int oracle_constants(double* emission_scale, double* f_factor) {
    *emission_scale = kEmissionScale;
    *f_factor = kFFactor;
    return RTW_OK;
}

int oracle_camera_rays(const rtw_scene* scene, rtw_camera* cam, double* rays, long long n_pix) {
    OScene sc(*scene);
    CameraGeom cg;
    camera_geom(sc, *cam, cg);
    cam->y_pix = cg.yp;
    if ((long long)cg.xp * cg.yp != n_pix) return RTW_ERR_INVALID_PARAM;
    for (int j = 0; j < cg.yp; ++j)
        for (int i = 0; i < cg.xp; ++i) camera_ray(cg, *cam, i, j, rays + 8 * ((long long)i + (long long)cg.xp * j));
    return RTW_OK;
}

// Slope of a full state R[8 + 2N] (calc_ray_derivative!).
int oracle_rhs(const rtw_scene* scene, const double* colors_nm, int n_colors, const double* R, double* slope) {
    OScene sc(*scene);
    std::vector<double> freq(n_colors);
    for (int c = 0; c < n_colors; ++c) freq[c] = 1.0 / colors_nm[c];
    RayWork w;
    w.init(n_colors, freq.data(), 1e-4, 0.1, false);
    rhs(sc, w, R, slope);
    return RTW_OK;
}

int oracle_metric(const rtw_scene* scene, const double* x, double* g16) {
    OScene sc(*scene);
    double g[4][4];
    sc.lower_metric(x, g);
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) g16[4 * i + j] = g[i][j];
    return RTW_OK;
}

double oracle_pad_max_dt(const rtw_scene* scene, const double* x, double scale) {
    OScene sc(*scene);
    return sc.pad_max_dt(x, scale);
}

// Traces the pixels `pixel_ids` (or all pixels when pixel_ids == NULL) of one
// camera. Outputs are indexed by position in the pixel list:
//   xyz[n][3], cls[n], steps[n], spectrum[n][N] (Ray[9+2c]), tau[n][N]
//   (Ray[10+2c]), state[n][8]; NULL pointers are skipped. counters (may be
//   NULL): [0] step attempts, [1] rejected, [2] polar Euler sub-steps.
// n_threads <= 0: all OpenMP threads. Returns rtw_status.
int oracle_render(const rtw_scene* scene, rtw_camera* cam, const double* colors_nm, int n_colors,
                  double max_dt_scale, int integrator, const long long* pixel_ids, long long n_ids, double* xyz,
                  unsigned char* cls, unsigned int* steps, double* spectrum, double* tau, double* state,
                  long long* counters, int n_threads) {
    if (!scene || !cam || !colors_nm || n_colors <= 0 || n_colors > RTW_MAX_BINS) return RTW_ERR_INVALID_PARAM;
    OScene sc(*scene);
    sc.bundles = g_bundles != 0;
    if (sc.is_singularity(cam->position)) return RTW_ERR_INVALID_CAMERA;
    CameraGeom cg;
    camera_geom(sc, *cam, cg);
    cam->y_pix = cg.yp;
    const long long P = (long long)cg.xp * cg.yp;
    const long long n = pixel_ids ? n_ids : P;
    std::vector<double> freq(n_colors), wx(n_colors), wy(n_colors), wz(n_colors), fac(n_colors);
    for (int c = 0; c < n_colors; ++c) freq[c] = 1.0 / colors_nm[c];
    cie_weights(colors_nm, n_colors, wx.data(), wy.data(), wz.data(), fac.data());
    const int N = n_colors, L = 8 + 2 * N;
    const double tol = cam->tolerance;
    const long long max_steps = cam->max_steps;
    int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
    const long long chunk = std::max(1LL, (n + 100LL * nt - 1) / (100LL * nt));
    long long tot_steps = 0, tot_rej = 0, tot_esc = 0;
#pragma omp parallel num_threads(nt) reduction(+ : tot_steps, tot_rej, tot_esc)
    {
        RayWork w;
        w.init(N, freq.data(), tol, max_dt_scale, integrator == RTW_DP45_FSAL);
        std::vector<double> ray(L);
#pragma omp for schedule(dynamic, chunk)
        for (long long q = 0; q < n; ++q) {
            const long long p = pixel_ids ? pixel_ids[q] : q;
            const int i = (int)(p % cg.xp), j = (int)(p / cg.xp);
            std::fill(ray.begin(), ray.end(), 0.0);
            camera_ray(cg, *cam, i, j, ray.data());
            long long step_count = 0, esc = 0, rej = 0;
            int crossings = 0;
            int klass = integrate_ray(sc, w, ray.data(), max_dt_scale, tol, max_steps, &step_count, &rej, &esc,
                                      &crossings);
            tot_rej += rej;
            for (int k = 0; k < 8; ++k)
                if (!std::isfinite(ray[k])) klass = RTW_CLASS_NAN;
            if (sc.is_wh() || sc.kind == RTW_SCENE_MINKOWSKI_CART_SPHERE) {
                double bund[6];
                if (g_bundles) camera_bundle(cg, i, j, bund);
                wormhole_skybox(sc, ray.data(), N, freq.data(), g_bundles ? bund : nullptr);
            }
            tot_steps += step_count;
            tot_esc += esc;
            if (g_diag_cross) g_diag_cross[q] = crossings;
            if (g_diag_escape) g_diag_escape[q] = (int)esc;
            if (cls) cls[q] = (unsigned char)klass;
            if (steps) steps[q] = (unsigned int)step_count;
            if (xyz) {
                double X = 0, Y = 0, Z = 0;
                for (int c = 0; c < N; ++c) {
                    const double il = ray[8 + 2 * c] * freq[c] * freq[c] * freq[c] * kLightC / (colors_nm[c] * colors_nm[c]);
                    X += il * wx[c];
                    Y += il * wy[c];
                    Z += il * wz[c];
                }
                xyz[3 * q + 0] = X;
                xyz[3 * q + 1] = Y;
                xyz[3 * q + 2] = Z;
            }
            if (spectrum)
                for (int c = 0; c < N; ++c) spectrum[(long long)N * q + c] = ray[8 + 2 * c];
            if (tau)
                for (int c = 0; c < N; ++c) tau[(long long)N * q + c] = ray[9 + 2 * c];
            if (state)
                for (int k = 0; k < 8; ++k) state[8 * q + k] = ray[k];
        }
    }
    if (counters) {
        counters[0] = tot_steps;
        counters[1] = tot_rej;
        counters[2] = tot_esc;
    }
    return RTW_OK;
}

// Algorithmic work of the reference's form over the given pixels (all when
// pixel_ids is null): the oracle's own integration of those rays (the same
// arithmetic, hence the same path and step counts as oracle_render) run over
// the counting scalar Cnt. The scene's step-size cap, polar-escape and
// termination tests and the camera set-up are not counted. Thin-disk scenes
// (Minkowski sphere, Schwarzschild disk, Kerr thin and thick disk) only.
// out[0] flops, out[1] transcendentals (div/sqrt/exp/log/sin/cos 1, pow 2),
// out[2] step attempts, out[3] rays.
int oracle_work(const rtw_scene* scene, rtw_camera* cam, const double* colors_nm, int n_colors,
                double max_dt_scale, int integrator, const long long* pixel_ids, long long n_ids, long long* out,
                int n_threads) {
    if (!scene || !cam || !colors_nm || !out || n_colors <= 0 || n_colors > RTW_MAX_BINS) return RTW_ERR_INVALID_PARAM;
    if (scene->kind != RTW_SCENE_MINKOWSKI_SPHERE && scene->kind != RTW_SCENE_SCHWARZSCHILD_DISK &&
        scene->kind != RTW_SCENE_KERR_DISK && scene->kind != RTW_SCENE_KERR_THICK_DISK)
        return RTW_ERR_UNSUPPORTED;
    OScene sc(*scene);
    if (sc.is_singularity(cam->position)) return RTW_ERR_INVALID_CAMERA;
    CameraGeom cg;
    camera_geom(sc, *cam, cg);
    cam->y_pix = cg.yp;
    const long long P = (long long)cg.xp * cg.yp;
    const long long n = pixel_ids ? n_ids : P;
    std::vector<double> freq(n_colors);
    for (int c = 0; c < n_colors; ++c) freq[c] = 1.0 / colors_nm[c];
    const int N = n_colors, L = 8 + 2 * N;
    const double tol = cam->tolerance;
    const long long max_steps = cam->max_steps;
    int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
    const long long chunk = std::max(1LL, (n + 100LL * nt - 1) / (100LL * nt));
    long long flops = 0, special = 0, attempts = 0, rays = 0;
#pragma omp parallel num_threads(nt) reduction(+ : flops, special, attempts, rays)
    {
        RayWorkT<Cnt> w;
        w.init(N, freq.data(), tol, max_dt_scale, integrator == RTW_DP45_FSAL);
        std::vector<double> ray0(L);
        std::vector<Cnt> ray(L);
        tally() = OpTally{};
#pragma omp for schedule(dynamic, chunk)
        for (long long q = 0; q < n; ++q) {
            const long long p = pixel_ids ? pixel_ids[q] : q;
            const int i = (int)(p % cg.xp), j = (int)(p / cg.xp);
            std::fill(ray0.begin(), ray0.end(), 0.0);
            camera_ray(cg, *cam, i, j, ray0.data());
            for (int k = 0; k < L; ++k) ray[k] = Cnt(ray0[k]);
            long long step_count = 0, esc = 0, rej = 0;
            int crossings = 0;
            integrate_ray(sc, w, ray.data(), max_dt_scale, tol, max_steps, &step_count, &rej, &esc, &crossings);
            attempts += step_count;
            ++rays;
        }
        flops += tally().flops;
        special += tally().special;
    }
    out[0] = flops;
    out[1] = special;
    out[2] = attempts;
    out[3] = rays;
    return RTW_OK;
}

}  // extern "C"
