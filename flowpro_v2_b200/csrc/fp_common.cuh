// Common device/host definitions: error handling, element-type constants and the
// forward-mode number type used by the tangent (JVP) and block-Jacobian kernels.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "../../include/flowgpu.h"

#define FP_HD __host__ __device__ __forceinline__

// Status word written by kernels (never a trap): bit flags OR-ed atomically.
enum : unsigned {
    FP_DEV_NONFINITE = 1u,
    FP_DEV_SINGULAR = 2u,
    FP_DEV_TIMEOUT = 4u,
    FP_DEV_BOUNDS = 8u,
};

// ---------------------------------------------------------------------------
// Forward-mode number with N tangent directions.  The residual kernels are
// templated on the scalar type, so one code path gives R (double), R and
// (dR/dW) v (Dual<1>), or N columns of an element Jacobian (Dual<N>).
template <int N>
struct Dual {
    double v;
    double d[N];
    FP_HD Dual() : v(0) {
#pragma unroll
        for (int i = 0; i < N; i++) d[i] = 0;
    }
    FP_HD Dual(double x) : v(x) {
#pragma unroll
        for (int i = 0; i < N; i++) d[i] = 0;
    }
    FP_HD Dual& operator+=(const Dual& o) {
        v += o.v;
#pragma unroll
        for (int i = 0; i < N; i++) d[i] += o.d[i];
        return *this;
    }
    FP_HD Dual& operator-=(const Dual& o) {
        v -= o.v;
#pragma unroll
        for (int i = 0; i < N; i++) d[i] -= o.d[i];
        return *this;
    }
    FP_HD Dual& operator*=(const Dual& o) {
#pragma unroll
        for (int i = 0; i < N; i++) d[i] = d[i] * o.v + v * o.d[i];
        v *= o.v;
        return *this;
    }
    FP_HD Dual& operator/=(const Dual& o) {
        double inv = 1.0 / o.v;
        double q = v * inv;
#pragma unroll
        for (int i = 0; i < N; i++) d[i] = (d[i] - q * o.d[i]) * inv;
        v = q;
        return *this;
    }
};

template <int N>
FP_HD Dual<N> operator+(Dual<N> a, const Dual<N>& b) { return a += b; }
template <int N>
FP_HD Dual<N> operator-(Dual<N> a, const Dual<N>& b) { return a -= b; }
template <int N>
FP_HD Dual<N> operator*(Dual<N> a, const Dual<N>& b) { return a *= b; }
template <int N>
FP_HD Dual<N> operator/(Dual<N> a, const Dual<N>& b) { return a /= b; }
template <int N>
FP_HD Dual<N> operator-(Dual<N> a) {
    a.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; i++) a.d[i] = -a.d[i];
    return a;
}
template <int N>
FP_HD Dual<N> operator+(Dual<N> a, double b) { a.v += b; return a; }
template <int N>
FP_HD Dual<N> operator+(double b, Dual<N> a) { a.v += b; return a; }
template <int N>
FP_HD Dual<N> operator-(Dual<N> a, double b) { a.v -= b; return a; }
template <int N>
FP_HD Dual<N> operator-(double b, Dual<N> a) {
    a = -a;
    a.v += b;
    return a;
}
template <int N>
FP_HD Dual<N> operator*(Dual<N> a, double b) {
    a.v *= b;
#pragma unroll
    for (int i = 0; i < N; i++) a.d[i] *= b;
    return a;
}
template <int N>
FP_HD Dual<N> operator*(double b, Dual<N> a) { return a * b; }
template <int N>
FP_HD Dual<N> operator/(Dual<N> a, double b) {
    double inv = 1.0 / b;
    a.v = a.v / b;
#pragma unroll
    for (int i = 0; i < N; i++) a.d[i] *= inv;
    return a;
}
template <int N>
FP_HD Dual<N> operator/(double b, const Dual<N>& a) {
    Dual<N> r;
    r.v = b / a.v;
    double f = -r.v / a.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = f * a.d[i];
    return r;
}

// value access and comparisons (branches follow the primal value)
FP_HD double val(double x) { return x; }
template <int N>
FP_HD double val(const Dual<N>& x) { return x.v; }

FP_HD double dsqrt(double x) { return sqrt(x); }
FP_HD double dexp(double x) { return exp(x); }
FP_HD double dfabs(double x) { return fabs(x); }
FP_HD double dpow(double x, double y) { return pow(x, y); }
template <int N>
FP_HD Dual<N> dsqrt(const Dual<N>& a) {
    Dual<N> r;
    r.v = sqrt(a.v);
    double f = r.v > 0 ? 0.5 / r.v : 0.0;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = f * a.d[i];
    return r;
}
template <int N>
FP_HD Dual<N> dexp(const Dual<N>& a) {
    Dual<N> r;
    r.v = exp(a.v);
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = r.v * a.d[i];
    return r;
}
template <int N>
FP_HD Dual<N> dfabs(const Dual<N>& a) { return a.v < 0 ? -a : a; }
// x^y with a constant exponent
template <int N>
FP_HD Dual<N> dpow(const Dual<N>& a, double y) {
    Dual<N> r;
    r.v = pow(a.v, y);
    double f = (a.v != 0.0) ? y * pow(a.v, y - 1.0) : (y == 1.0 ? 1.0 : 0.0);
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = f * a.d[i];
    return r;
}

template <class T>
FP_HD T dmax(const T& a, const T& b) { return val(a) >= val(b) ? a : b; }  // Math.max(a, b)
template <class T>
FP_HD T dmin(const T& a, const T& b) { return val(a) <= val(b) ? a : b; }

// Reference element constants
template <int DIM>
struct Simplex {
    static constexpr int NV = DIM + 1;      // vertices
    static constexpr int NF = DIM + 1;      // faces
    static constexpr int NVF = DIM;         // vertices per face
};
