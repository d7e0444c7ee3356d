// rtw_opcount.cu - host evaluations of the trace kernel's own device functors:
// (1) rtw_scene_rhs: the scene right-hand side in FP64 (or FP32), for checking
// the kernel's formulas against the oracle without a GPU; (2) algorithmic
// operation counts of the kernel's arithmetic, obtained by running the same
// scene functors and Dormand-Prince attempt on the host with a counting scalar. Used for the roofline: the
// achieved FLOP/s of a render is these counts times the render's counters
// (step attempts, emitting attempts, spectral attempts) over its device time.
//
// Conventions: add, sub, mul = 1 flop each (an FMA = 2); div, sqrt, exp, pow
// = 1 flop + 1 MUFU op (pow and sincos: 2 + 2). Comparisons and sign flips
// are free.
#include <cmath>
#include <cstring>

#include "rtw_trace.cuh"

namespace rtw {

struct Tally {
    long long flops = 0, mufu = 0;
};
static Tally g_tally;

struct CS {
    double v;
    CS() : v(0) {}
    CS(double x) : v(x) {}
    explicit operator double() const { return v; }
};

inline CS operator+(CS a, CS b) { ++g_tally.flops; return CS(a.v + b.v); }
inline CS operator-(CS a, CS b) { ++g_tally.flops; return CS(a.v - b.v); }
inline CS operator*(CS a, CS b) { ++g_tally.flops; return CS(a.v * b.v); }
inline CS operator/(CS a, CS b) { ++g_tally.flops; ++g_tally.mufu; return CS(a.v / b.v); }
inline CS operator-(CS a) { return CS(-a.v); }
inline CS& operator+=(CS& a, CS b) { a = a + b; return a; }
inline bool operator<(CS a, CS b) { return a.v < b.v; }
inline bool operator>(CS a, CS b) { return a.v > b.v; }
inline bool operator<=(CS a, CS b) { return a.v <= b.v; }
inline bool operator>=(CS a, CS b) { return a.v >= b.v; }
inline bool operator==(CS a, CS b) { return a.v == b.v; }
inline bool operator!=(CS a, CS b) { return a.v != b.v; }
inline CS operator*(double a, CS b) { return CS(a) * b; }
inline CS operator*(CS a, double b) { return a * CS(b); }

inline void rsincos(CS x, CS* s, CS* c) {
    g_tally.flops += 2;
    g_tally.mufu += 2;
    *s = CS(std::sin(x.v));
    *c = CS(std::cos(x.v));
}
inline CS rsqrt_(CS x) { ++g_tally.flops; ++g_tally.mufu; return CS(std::sqrt(x.v)); }
inline CS rexp_(CS x) { ++g_tally.flops; ++g_tally.mufu; return CS(std::exp(x.v)); }
inline CS rpow_(CS x, CS y) { g_tally.flops += 2; g_tally.mufu += 2; return CS(std::pow(x.v, y.v)); }
inline CS rinv(CS x) { ++g_tally.flops; ++g_tally.mufu; return CS(1.0 / x.v); }
inline CS cdiv(CS a, CS b) { return a / b; }
inline CS cabs(CS a) { return CS(std::fabs(a.v)); }
inline CS cmax(CS a, CS b) { return CS(std::fmax(a.v, b.v)); }
inline CS cmin(CS a, CS b) { return CS(std::fmin(a.v, b.v)); }

template <int KIND>
static void count_kind(const DevScene& sc, const double* xv, const double* xe, rtw_op_counts* out) {
    typedef typename SceneOf<KIND>::type SCN;
    CS z[10], k[9];
    Emit<CS> em;
    // vacuum right-hand side
    for (int i = 0; i < 10; ++i) z[i] = CS(xv[i]);
    g_tally = Tally();
    SCN::template rhs<CS>(sc, z, k, em);
    out->rhs_vacuum = (double)g_tally.flops;
    out->rhs_vacuum_mufu = (double)g_tally.mufu;
    // emitting right-hand side
    for (int i = 0; i < 10; ++i) z[i] = CS(xe[i]);
    g_tally = Tally();
    SCN::template rhs<CS>(sc, z, k, em);
    out->rhs_emit = (double)g_tally.flops;
    out->rhs_emit_mufu = (double)g_tally.mufu;
    // one whole attempt at the vacuum point: 6 right-hand sides + the rest
    CS k1[9], ns[9], nk1[9], A[6], X[6], err2;
    for (int i = 0; i < 9; ++i) k1[i] = k[i];
    bool emit = false;
    g_tally = Tally();
    dp45_attempt<SCN, CS, CS, CS, CS>(sc, xv, k1, -1e-3, 1e-8, 64, false, ns, nk1, A, X, 1, err2, emit);
    // controller (decide: sqrt, log2/exp2, ~12 flops) and the FP64 update
    // x + h ns of an accepted attempt (9 FMA)
    const double controller_flops = 12 + 18, controller_mufu = 3;
    out->step_overhead = (double)g_tally.flops - 6 * out->rhs_vacuum + controller_flops;
    out->step_overhead_mufu = (double)g_tally.mufu - 6 * out->rhs_vacuum_mufu + controller_mufu;
    // spectral work per bin of one attempt (warp-cooperative phase): five new
    // stage slopes of 3 flops + ex2 + rcp each, the 5th-order and error
    // combinations (20), the compensated add (6), tolerance and squared
    // error (7)
    out->bin_step = 5 * 3 + 20 + 6 + 7;
    out->bin_step_mufu = 5 * 2 + 1;
}

}  // namespace rtw

extern "C" rtw_status rtw_get_op_counts(int32_t kind, rtw_op_counts* out) {
    using namespace rtw;
    if (!out) return RTW_ERR_INVALID_PARAM;
    std::memset(out, 0, sizeof(*out));
    rtw_scene s;
    if (rtw_scene_default(kind, &s) != RTW_OK) return RTW_ERR_INVALID_PARAM;
    DevScene sc;
    std::memset(&sc, 0, sizeof(sc));
    sc.kind = kind;
    sc.M = 1; sc.a = (kind == RTW_SCENE_KERR_DISK || kind == RTW_SCENE_KERR_THICK_DISK) ? 0.9 : 0.0;
    sc.rs = 2; sc.sqrtM = 1;
    sc.r_ev = kind == RTW_SCENE_MINKOWSKI_SPHERE ? 0.0 : (sc.a != 0 ? 1 + std::sqrt(1 - sc.a * sc.a) : 2.0);
    sc.r_pm = sc.a != 0 ? 2 * std::sqrt(1 - sc.a * sc.a) : 0.0;
    sc.r_in = kind == RTW_SCENE_MINKOWSKI_SPHERE ? 0.0 : 6.0;
    sc.r_out = kind == RTW_SCENE_MINKOWSKI_SPHERE ? 1.0 : 20.0;
    sc.th_lo = 1.4; sc.th_hi = 1.75;
    sc.T = 1e4; sc.anu = 1; sc.esc = 100; sc.wind = 8 * 3.141592653589793;
    sc.rho_r0 = 6; sc.rho_h = 0.1; sc.rho_idx = -2; sc.t_idx = -0.75;
    const double re = kind == RTW_SCENE_MINKOWSKI_SPHERE ? 0.5 : 10.0;
    const double xv[10] = {0, 40.0, 1.3, 0, 1.1, -0.9, 0.001, 0.002, 0, 40.0 - sc.r_ev};
    const double xe[10] = {0, re, 1.5707, 0, 1.1, -0.9, 0.001, 0.02, 0.3, re - sc.r_ev};
    switch (kind) {
    case 0: count_kind<0>(sc, xv, xe, out); break;
    case 1: count_kind<1>(sc, xv, xe, out); break;
    case 2: count_kind<2>(sc, xv, xe, out); break;
    default: count_kind<3>(sc, xv, xe, out); break;
    }
    return RTW_OK;
}

namespace rtw {
template <int KIND, class R>
static void host_rhs(const DevScene& sc, const double* state, double* slope, double* emit) {
    typedef typename SceneOf<KIND>::type SCN;
    R z[10], k[9];
    Emit<R> em;
    for (int i = 0; i < 9; ++i) z[i] = R(state[i]);
    z[9] = R(state[1] - sc.r_ev);
    SCN::template rhs<R>(sc, z, k, em);
    for (int i = 0; i < 9; ++i) slope[i] = double(k[i]);
    if (emit) {
        emit[0] = double(em.A);
        emit[1] = double(em.X);
        emit[2] = double(em.ktau);
    }
}
}  // namespace rtw

extern "C" rtw_status rtw_scene_rhs(const rtw_scene* scene, int32_t fp32, const double* state, double* slope,
                                    double* emit) {
    using namespace rtw;
    if (!scene || !state || !slope || scene->kind < 0 || scene->kind > RTW_SCENE_KERR_THICK_DISK)
        return RTW_ERR_INVALID_PARAM;
    DevScene sc;
    make_dev_scene(*scene, sc);
    switch (scene->kind * 2 + (fp32 ? 1 : 0)) {
    case 0: host_rhs<0, double>(sc, state, slope, emit); break;
    case 1: host_rhs<0, float>(sc, state, slope, emit); break;
    case 2: host_rhs<1, double>(sc, state, slope, emit); break;
    case 3: host_rhs<1, float>(sc, state, slope, emit); break;
    case 4: host_rhs<2, double>(sc, state, slope, emit); break;
    case 5: host_rhs<2, float>(sc, state, slope, emit); break;
    case 6: host_rhs<3, double>(sc, state, slope, emit); break;
    default: host_rhs<3, float>(sc, state, slope, emit); break;
    }
    return RTW_OK;
}
