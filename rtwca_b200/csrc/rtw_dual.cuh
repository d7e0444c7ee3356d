// rtw_dual.cuh - forward-mode dual numbers (a value and K tangents) and the
// scalar helpers that let one generic formula run as float, double or Dual.
// The adjoint kernel seeds the tangents with the inputs of a right-hand-side
// piece and contracts the resulting Jacobian columns with the cotangent.
#pragma once

#include <cmath>

#ifndef RTW_HD
#define RTW_HD __host__ __device__ __forceinline__
#endif

namespace rtw {

template <class T, int K>
struct Dual {
    T v;
    T d[K];
    RTW_HD Dual() : v(0) {
#pragma unroll
        for (int i = 0; i < K; ++i) d[i] = 0;
    }
    RTW_HD Dual(T x) : v(x) {  // a constant
#pragma unroll
        for (int i = 0; i < K; ++i) d[i] = 0;
    }
    // variable number `slot` of the K inputs
    RTW_HD static Dual var(T x, int slot) {
        Dual r(x);
        r.d[slot] = T(1);
        return r;
    }
};

// a function of one argument with value f and derivative df at u.v
template <class T, int K>
RTW_HD Dual<T, K> chain(const Dual<T, K>& u, T f, T df) {
    Dual<T, K> r;
    r.v = f;
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = df * u.d[i];
    return r;
}

template <class T, int K>
RTW_HD Dual<T, K> operator+(const Dual<T, K>& a, const Dual<T, K>& b) {
    Dual<T, K> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <class T, int K>
RTW_HD Dual<T, K> operator-(const Dual<T, K>& a, const Dual<T, K>& b) {
    Dual<T, K> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <class T, int K>
RTW_HD Dual<T, K> operator-(const Dual<T, K>& a) {
    Dual<T, K> r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = -a.d[i];
    return r;
}
template <class T, int K>
RTW_HD Dual<T, K> operator*(const Dual<T, K>& a, const Dual<T, K>& b) {
    Dual<T, K> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <class T, int K>
RTW_HD Dual<T, K> operator/(const Dual<T, K>& a, const Dual<T, K>& b) {
    const T ib = T(1) / b.v;
    Dual<T, K> r;
    r.v = a.v * ib;
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}
template <class T, int K>
RTW_HD Dual<T, K> operator+(const Dual<T, K>& a, T b) {
    Dual<T, K> r = a;
    r.v += b;
    return r;
}
template <class T, int K>
RTW_HD Dual<T, K> operator+(T b, const Dual<T, K>& a) { return a + b; }
template <class T, int K>
RTW_HD Dual<T, K> operator-(const Dual<T, K>& a, T b) {
    Dual<T, K> r = a;
    r.v -= b;
    return r;
}
template <class T, int K>
RTW_HD Dual<T, K> operator-(T b, const Dual<T, K>& a) { return -a + b; }
template <class T, int K>
RTW_HD Dual<T, K> operator*(const Dual<T, K>& a, T b) {
    Dual<T, K> r;
    r.v = a.v * b;
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = a.d[i] * b;
    return r;
}
template <class T, int K>
RTW_HD Dual<T, K> operator*(T b, const Dual<T, K>& a) { return a * b; }
template <class T, int K>
RTW_HD Dual<T, K> operator/(const Dual<T, K>& a, T b) { return a * (T(1) / b); }
template <class T, int K>
RTW_HD Dual<T, K> operator/(T a, const Dual<T, K>& b) {
    const T ib = T(1) / b.v;
    return chain(b, a * ib, -a * ib * ib);
}

// ---- generic scalar helpers ------------------------------------------------
RTW_HD float val(float x) { return x; }
RTW_HD double val(double x) { return x; }
template <class T, int K>
RTW_HD T val(const Dual<T, K>& x) { return x.v; }

RTW_HD float tsqrt(float x) { return sqrtf(x); }
RTW_HD double tsqrt(double x) { return sqrt(x); }
RTW_HD float texp(float x) { return expf(x); }
RTW_HD double texp(double x) { return exp(x); }
RTW_HD float tlog(float x) { return logf(x); }
RTW_HD double tlog(double x) { return log(x); }
RTW_HD float tsin(float x) { return sinf(x); }
RTW_HD double tsin(double x) { return sin(x); }
RTW_HD float tcos(float x) { return cosf(x); }
RTW_HD double tcos(double x) { return cos(x); }
RTW_HD float texpm1(float x) { return expm1f(x); }
RTW_HD double texpm1(double x) { return expm1(x); }
RTW_HD float tatan(float x) { return atanf(x); }
RTW_HD double tatan(double x) { return atan(x); }

template <class T, int K>
RTW_HD Dual<T, K> tsqrt(const Dual<T, K>& u) {
    const T s = tsqrt(u.v);
    return chain(u, s, T(0.5) / s);
}
template <class T, int K>
RTW_HD Dual<T, K> texp(const Dual<T, K>& u) {
    const T e = texp(u.v);
    return chain(u, e, e);
}
template <class T, int K>
RTW_HD Dual<T, K> texpm1(const Dual<T, K>& u) {
    return chain(u, texpm1(u.v), texp(u.v));
}
template <class T, int K>
RTW_HD Dual<T, K> tlog(const Dual<T, K>& u) { return chain(u, tlog(u.v), T(1) / u.v); }
template <class T, int K>
RTW_HD Dual<T, K> tsin(const Dual<T, K>& u) { return chain(u, tsin(u.v), tcos(u.v)); }
template <class T, int K>
RTW_HD Dual<T, K> tcos(const Dual<T, K>& u) { return chain(u, tcos(u.v), -tsin(u.v)); }
template <class T, int K>
RTW_HD Dual<T, K> tatan(const Dual<T, K>& u) { return chain(u, tatan(u.v), T(1) / (T(1) + u.v * u.v)); }

// u^p for u > 0 and a constant exponent
template <class S>
RTW_HD S tpow(const S& u, double p) {
    return texp(tlog(u) * decltype(val(u))(p));
}

}  // namespace rtw
