// dual.cuh - forward-mode dual numbers v + sum_k d[k] e_k (N tangents), used
// by the adjoint kernel to obtain exact Jacobians of the geodesic
// acceleration and of the colour lookups from the same templated code that
// renders.  Comparisons and branches use the value part only, so control
// flow is frozen at the primal (what a discrete adjoint differentiates).
#pragma once
#include <cuda_runtime.h>

namespace prr {

// The Dual overloads below are declared in this namespace; keep the plain
// float/double math functions visible to unqualified calls here as well.
using ::acos;
using ::atan2;
using ::cos;
using ::fabs;
using ::floor;
using ::fmax;
using ::fmin;
using ::sin;
using ::sqrt;

template <int N> struct Dual {
    double v;
    double d[N];
    __host__ __device__ Dual() : v(0.0) {
#pragma unroll
        for (int k = 0; k < N; k++) d[k] = 0.0;
    }
    __host__ __device__ Dual(double x) : v(x) {
#pragma unroll
        for (int k = 0; k < N; k++) d[k] = 0.0;
    }
    __host__ __device__ static Dual var(double x, int k)
    {
        Dual r(x);
        r.d[k] = 1.0;
        return r;
    }
    __host__ __device__ explicit operator double() const { return v; }
    __host__ __device__ explicit operator float() const { return (float)v; }
    __host__ __device__ explicit operator int() const { return (int)v; }
};

#define PRR_DUAL_BIN(OP, VAL, DER)                                                                                 \
    template <int N> __host__ __device__ inline Dual<N> operator OP(const Dual<N> &a, const Dual<N> &b)             \
    {                                                                                                              \
        Dual<N> r;                                                                                                 \
        r.v = VAL;                                                                                                 \
        _Pragma("unroll") for (int k = 0; k < N; k++) r.d[k] = DER;                                                \
        return r;                                                                                                  \
    }
PRR_DUAL_BIN(+, a.v + b.v, a.d[k] + b.d[k])
PRR_DUAL_BIN(-, a.v - b.v, a.d[k] - b.d[k])
PRR_DUAL_BIN(*, a.v * b.v, a.d[k] * b.v + a.v * b.d[k])
#undef PRR_DUAL_BIN

template <int N> __host__ __device__ inline Dual<N> operator/(const Dual<N> &a, const Dual<N> &b)
{
    Dual<N> r;
    double ib = 1.0 / b.v;
    r.v = a.v * ib;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
    return r;
}
template <int N> __host__ __device__ inline Dual<N> operator-(const Dual<N> &a)
{
    Dual<N> r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = -a.d[k];
    return r;
}
template <int N> __host__ __device__ inline Dual<N> operator+(const Dual<N> &a, double b) { return a + Dual<N>(b); }
template <int N> __host__ __device__ inline Dual<N> operator+(double a, const Dual<N> &b) { return Dual<N>(a) + b; }
template <int N> __host__ __device__ inline Dual<N> operator-(const Dual<N> &a, double b) { return a - Dual<N>(b); }
template <int N> __host__ __device__ inline Dual<N> operator-(double a, const Dual<N> &b) { return Dual<N>(a) - b; }
template <int N> __host__ __device__ inline Dual<N> operator*(const Dual<N> &a, double b)
{
    Dual<N> r;
    r.v = a.v * b;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = a.d[k] * b;
    return r;
}
template <int N> __host__ __device__ inline Dual<N> operator*(double a, const Dual<N> &b) { return b * a; }
template <int N> __host__ __device__ inline Dual<N> operator/(const Dual<N> &a, double b) { return a * (1.0 / b); }
template <int N> __host__ __device__ inline Dual<N> operator/(double a, const Dual<N> &b) { return Dual<N>(a) / b; }
template <int N> __host__ __device__ inline Dual<N> &operator+=(Dual<N> &a, const Dual<N> &b) { return a = a + b; }
template <int N> __host__ __device__ inline Dual<N> &operator-=(Dual<N> &a, const Dual<N> &b) { return a = a - b; }
template <int N> __host__ __device__ inline Dual<N> &operator*=(Dual<N> &a, const Dual<N> &b) { return a = a * b; }

#define PRR_DUAL_CMP(OP)                                                                                           \
    template <int N> __host__ __device__ inline bool operator OP(const Dual<N> &a, const Dual<N> &b) { return a.v OP b.v; } \
    template <int N> __host__ __device__ inline bool operator OP(const Dual<N> &a, double b) { return a.v OP b; }      \
    template <int N> __host__ __device__ inline bool operator OP(double a, const Dual<N> &b) { return a OP b.v; }
PRR_DUAL_CMP(<)
PRR_DUAL_CMP(>)
PRR_DUAL_CMP(<=)
PRR_DUAL_CMP(>=)
PRR_DUAL_CMP(==)
PRR_DUAL_CMP(!=)
#undef PRR_DUAL_CMP

template <int N> __host__ __device__ inline Dual<N> chain(const Dual<N> &a, double f, double df)
{
    Dual<N> r;
    r.v = f;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = df * a.d[k];
    return r;
}
template <int N> __host__ __device__ inline Dual<N> sqrt(const Dual<N> &a)
{
    double s = ::sqrt(a.v);
    return chain(a, s, s > 0.0 ? 0.5 / s : 0.0);
}
template <int N> __host__ __device__ inline Dual<N> fabs(const Dual<N> &a) { return a.v < 0.0 ? -a : a; }
template <int N> __host__ __device__ inline Dual<N> fmax(const Dual<N> &a, const Dual<N> &b) { return a.v >= b.v ? a : b; }
template <int N> __host__ __device__ inline Dual<N> fmin(const Dual<N> &a, const Dual<N> &b) { return a.v <= b.v ? a : b; }
template <int N> __host__ __device__ inline Dual<N> floor(const Dual<N> &a) { return Dual<N>(::floor(a.v)); }
template <int N> __host__ __device__ inline Dual<N> acos(const Dual<N> &a)
{
    double s = 1.0 - a.v * a.v;
    return chain(a, ::acos(a.v), s > 0.0 ? -1.0 / ::sqrt(s) : 0.0);
}
template <int N> __host__ __device__ inline Dual<N> atan2(const Dual<N> &y, const Dual<N> &x)
{
    Dual<N> r;
    r.v = ::atan2(y.v, x.v);
    double den = x.v * x.v + y.v * y.v;
    double a = den > 0.0 ? x.v / den : 0.0, b = den > 0.0 ? -y.v / den : 0.0;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = a * y.d[k] + b * x.d[k];
    return r;
}
template <int N> __host__ __device__ inline Dual<N> sin(const Dual<N> &a) { return chain(a, ::sin(a.v), ::cos(a.v)); }
template <int N> __host__ __device__ inline Dual<N> cos(const Dual<N> &a) { return chain(a, ::cos(a.v), -::sin(a.v)); }

}  // namespace prr
