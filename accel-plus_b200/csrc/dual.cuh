// dual.cuh — forward-mode dual numbers: value plus N directional derivatives.
//
// Instantiating the literal element maps (elem_literal.cuh) with Dual<6> propagates the six unit
// tangents through every element pass, which gives the exact one-turn Jacobian; Dual<7> adds one
// parameter direction for per-element vector-Jacobian products in the adjoint.
#pragma once
#include <cmath>

namespace accel {

template <int N>
struct Dual {
    double v;
    double d[N];
    __host__ __device__ Dual() {}
    __host__ __device__ Dual(double x) : v(x) {
#pragma unroll
        for (int i = 0; i < N; i++) d[i] = 0.0;
    }
};

#define DUAL_BIN(OP, VAL, DER)                                                                  \
    template <int N>                                                                            \
    __host__ __device__ __forceinline__ Dual<N> operator OP(const Dual<N>& a, const Dual<N>& b) { \
        Dual<N> r;                                                                              \
        r.v = VAL;                                                                              \
        _Pragma("unroll") for (int i = 0; i < N; i++) r.d[i] = DER;                             \
        return r;                                                                               \
    }
DUAL_BIN(+, a.v + b.v, a.d[i] + b.d[i])
DUAL_BIN(-, a.v - b.v, a.d[i] - b.d[i])
DUAL_BIN(*, a.v * b.v, a.d[i] * b.v + a.v * b.d[i])
#undef DUAL_BIN

template <int N>
__host__ __device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v / b.v;
    double ib = 1.0 / b.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
    Dual<N> r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = -a.d[i];
    return r;
}
// mixed with double
template <int N> __host__ __device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, double b) { Dual<N> r = a; r.v += b; return r; }
template <int N> __host__ __device__ __forceinline__ Dual<N> operator+(double a, const Dual<N>& b) { Dual<N> r = b; r.v += a; return r; }
template <int N> __host__ __device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, double b) { Dual<N> r = a; r.v -= b; return r; }
template <int N> __host__ __device__ __forceinline__ Dual<N> operator-(double a, const Dual<N>& b) { return Dual<N>(a) - b; }
template <int N> __host__ __device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, double b) {
    Dual<N> r; r.v = a.v * b;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * b;
    return r;
}
template <int N> __host__ __device__ __forceinline__ Dual<N> operator*(double a, const Dual<N>& b) { return b * a; }
template <int N> __host__ __device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, double b) {
    Dual<N> r; r.v = a.v / b;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] / b;
    return r;
}
template <int N> __host__ __device__ __forceinline__ Dual<N> operator/(double a, const Dual<N>& b) { return Dual<N>(a) / b; }
template <int N> __host__ __device__ __forceinline__ Dual<N>& operator+=(Dual<N>& a, const Dual<N>& b) { a = a + b; return a; }
template <int N> __host__ __device__ __forceinline__ Dual<N>& operator-=(Dual<N>& a, const Dual<N>& b) { a = a - b; return a; }
template <int N> __host__ __device__ __forceinline__ Dual<N>& operator*=(Dual<N>& a, const Dual<N>& b) { a = a * b; return a; }
template <int N> __host__ __device__ __forceinline__ Dual<N>& operator+=(Dual<N>& a, double b) { a.v += b; return a; }
template <int N> __host__ __device__ __forceinline__ Dual<N>& operator-=(Dual<N>& a, double b) { a.v -= b; return a; }
template <int N> __host__ __device__ __forceinline__ Dual<N>& operator*=(Dual<N>& a, double b) { a = a * b; return a; }

template <int N> __host__ __device__ __forceinline__ bool operator<=(const Dual<N>& a, double b) { return a.v <= b; }
template <int N> __host__ __device__ __forceinline__ bool operator>=(const Dual<N>& a, double b) { return a.v >= b; }
template <int N> __host__ __device__ __forceinline__ bool operator>(const Dual<N>& a, double b) { return a.v > b; }
template <int N> __host__ __device__ __forceinline__ bool operator<(const Dual<N>& a, double b) { return a.v < b; }

template <int N, class F, class G>
__device__ __forceinline__ Dual<N> dual_apply(const Dual<N>& a, F f, G df) {
    Dual<N> r;
    r.v = f(a.v);
    double g = df(a.v, r.v);
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = g * a.d[i];
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> sqrt(const Dual<N>& a) {
    return dual_apply(a, [](double x) { return ::sqrt(x); }, [](double, double s) { return 0.5 / s; });
}
template <int N> __device__ __forceinline__ Dual<N> sin(const Dual<N>& a) {
    return dual_apply(a, [](double x) { return ::sin(x); }, [](double x, double) { return ::cos(x); });
}
template <int N> __device__ __forceinline__ Dual<N> cos(const Dual<N>& a) {
    return dual_apply(a, [](double x) { return ::cos(x); }, [](double x, double) { return -::sin(x); });
}
template <int N> __device__ __forceinline__ Dual<N> sinh(const Dual<N>& a) {
    return dual_apply(a, [](double x) { return ::sinh(x); }, [](double x, double) { return ::cosh(x); });
}
template <int N> __device__ __forceinline__ Dual<N> cosh(const Dual<N>& a) {
    return dual_apply(a, [](double x) { return ::cosh(x); }, [](double x, double) { return ::sinh(x); });
}
template <int N> __device__ __forceinline__ Dual<N> fabs(const Dual<N>& a) {
    return a.v < 0 ? -a : a;
}

// the plain double overloads stay visible next to the Dual ones inside this namespace
// atan2(y, x): d = (x dy - y dx) / (x^2 + y^2)
template <int N> __device__ __forceinline__ Dual<N> atan2(const Dual<N>& y, const Dual<N>& x) {
    Dual<N> r;
    r.v = ::atan2(y.v, x.v);
    const double q = 1.0 / (x.v * x.v + y.v * y.v);
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = (x.v * y.d[i] - y.v * x.d[i]) * q;
    return r;
}
using ::atan2;
using ::sqrt;
using ::sin;
using ::cos;
using ::sinh;
using ::cosh;
using ::fabs;
using ::exp;
using ::log;

template <class T> __host__ __device__ __forceinline__ double val(const T& x) { return x; }
template <int N> __host__ __device__ __forceinline__ double val(const Dual<N>& x) { return x.v; }

}  // namespace accel
