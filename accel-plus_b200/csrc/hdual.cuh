// hdual.cuh — hyper-dual numbers for the derivative of a transfer matrix with respect to one knob.
//
// A value carries, besides itself, its first derivatives in the six initial coordinates (d[i]),
// its first derivative in a knob k (k), and the mixed second derivatives d^2/(dr0_i dk) (m[i]):
// a truncated Taylor expansion in (dr0, dk) with dr0_i dr0_j = dk^2 = 0.  Propagating the
// literal element maps with the state seeded as r_i + dr0_i and the knob's coefficients as
// c + dk gives, at the end of the line, the transfer matrix M_ij = r_i.d[j] and its exact knob
// derivative dM_ij/dk = r_i.m[j], with no difference in the knob.
//
// Products: (a b).m_i = a.m_i b + a b.m_i + a.d_i b.k + a.k b.d_i.  A smooth function f applied
// to a gives f(a), f'(a) a.d, f'(a) a.k, f'(a) a.m + f''(a) a.d a.k.
#pragma once
#include <cmath>

namespace accel {

struct HDual {
    double v, k;
    double d[6], m[6];
    __host__ __device__ HDual() {}
    __host__ __device__ HDual(double x) : v(x), k(0.0) {
#pragma unroll
        for (int i = 0; i < 6; i++) d[i] = m[i] = 0.0;
    }
};

__host__ __device__ __forceinline__ HDual operator+(const HDual& a, const HDual& b) {
    HDual r;
    r.v = a.v + b.v;
    r.k = a.k + b.k;
#pragma unroll
    for (int i = 0; i < 6; i++) { r.d[i] = a.d[i] + b.d[i]; r.m[i] = a.m[i] + b.m[i]; }
    return r;
}
__host__ __device__ __forceinline__ HDual operator-(const HDual& a, const HDual& b) {
    HDual r;
    r.v = a.v - b.v;
    r.k = a.k - b.k;
#pragma unroll
    for (int i = 0; i < 6; i++) { r.d[i] = a.d[i] - b.d[i]; r.m[i] = a.m[i] - b.m[i]; }
    return r;
}
__host__ __device__ __forceinline__ HDual operator-(const HDual& a) {
    HDual r;
    r.v = -a.v;
    r.k = -a.k;
#pragma unroll
    for (int i = 0; i < 6; i++) { r.d[i] = -a.d[i]; r.m[i] = -a.m[i]; }
    return r;
}
__host__ __device__ __forceinline__ HDual operator*(const HDual& a, const HDual& b) {
    HDual r;
    r.v = a.v * b.v;
    r.k = a.k * b.v + a.v * b.k;
#pragma unroll
    for (int i = 0; i < 6; i++) {
        r.d[i] = a.d[i] * b.v + a.v * b.d[i];
        r.m[i] = a.m[i] * b.v + a.v * b.m[i] + a.d[i] * b.k + a.k * b.d[i];
    }
    return r;
}
// f(a) from f = f(a.v), f1 = f'(a.v), f2 = f''(a.v)
__host__ __device__ __forceinline__ HDual hd_chain(const HDual& a, double f, double f1, double f2) {
    HDual r;
    r.v = f;
    r.k = f1 * a.k;
#pragma unroll
    for (int i = 0; i < 6; i++) {
        r.d[i] = f1 * a.d[i];
        r.m[i] = f1 * a.m[i] + f2 * a.d[i] * a.k;
    }
    return r;
}
__host__ __device__ __forceinline__ HDual hd_inv(const HDual& b) {
    const double q = 1.0 / b.v;
    return hd_chain(b, q, -q * q, 2.0 * q * q * q);
}
__host__ __device__ __forceinline__ HDual operator/(const HDual& a, const HDual& b) {
    HDual r = a * hd_inv(b);
    r.v = a.v / b.v;  // the value as the plain division rounds it
    return r;
}

// mixed with double
__host__ __device__ __forceinline__ HDual operator+(const HDual& a, double b) { HDual r = a; r.v += b; return r; }
__host__ __device__ __forceinline__ HDual operator+(double a, const HDual& b) { HDual r = b; r.v += a; return r; }
__host__ __device__ __forceinline__ HDual operator-(const HDual& a, double b) { HDual r = a; r.v -= b; return r; }
__host__ __device__ __forceinline__ HDual operator-(double a, const HDual& b) { HDual r = -b; r.v = a - b.v; return r; }
__host__ __device__ __forceinline__ HDual operator*(const HDual& a, double b) {
    HDual r;
    r.v = a.v * b;
    r.k = a.k * b;
#pragma unroll
    for (int i = 0; i < 6; i++) { r.d[i] = a.d[i] * b; r.m[i] = a.m[i] * b; }
    return r;
}
__host__ __device__ __forceinline__ HDual operator*(double a, const HDual& b) { return b * a; }
__host__ __device__ __forceinline__ HDual operator/(const HDual& a, double b) {
    HDual r;
    r.v = a.v / b;
    r.k = a.k / b;
#pragma unroll
    for (int i = 0; i < 6; i++) { r.d[i] = a.d[i] / b; r.m[i] = a.m[i] / b; }
    return r;
}
__host__ __device__ __forceinline__ HDual operator/(double a, const HDual& b) {
    HDual r = hd_inv(b) * a;
    r.v = a / b.v;
    return r;
}
__host__ __device__ __forceinline__ HDual& operator+=(HDual& a, const HDual& b) { a = a + b; return a; }
__host__ __device__ __forceinline__ HDual& operator-=(HDual& a, const HDual& b) { a = a - b; return a; }
__host__ __device__ __forceinline__ HDual& operator*=(HDual& a, const HDual& b) { a = a * b; return a; }
__host__ __device__ __forceinline__ HDual& operator+=(HDual& a, double b) { a.v += b; return a; }
__host__ __device__ __forceinline__ HDual& operator-=(HDual& a, double b) { a.v -= b; return a; }
__host__ __device__ __forceinline__ HDual& operator*=(HDual& a, double b) { a = a * b; return a; }

__host__ __device__ __forceinline__ bool operator<=(const HDual& a, double b) { return a.v <= b; }
__host__ __device__ __forceinline__ bool operator>=(const HDual& a, double b) { return a.v >= b; }
__host__ __device__ __forceinline__ bool operator>(const HDual& a, double b) { return a.v > b; }
__host__ __device__ __forceinline__ bool operator<(const HDual& a, double b) { return a.v < b; }

__device__ __forceinline__ HDual sqrt(const HDual& a) {
    const double s = ::sqrt(a.v);
    return hd_chain(a, s, 0.5 / s, -0.25 / (s * a.v));
}
__device__ __forceinline__ HDual sin(const HDual& a) {
    const double s = ::sin(a.v), c = ::cos(a.v);
    return hd_chain(a, s, c, -s);
}
__device__ __forceinline__ HDual cos(const HDual& a) {
    const double s = ::sin(a.v), c = ::cos(a.v);
    return hd_chain(a, c, -s, -c);
}
__device__ __forceinline__ HDual sinh(const HDual& a) {
    const double s = ::sinh(a.v), c = ::cosh(a.v);
    return hd_chain(a, s, c, s);
}
__device__ __forceinline__ HDual cosh(const HDual& a) {
    const double s = ::sinh(a.v), c = ::cosh(a.v);
    return hd_chain(a, c, s, c);
}
__device__ __forceinline__ HDual fabs(const HDual& a) { return a.v < 0 ? -a : a; }
// atan2(y, x): first partials (x, -y) / rho2; second partials from them
__device__ __forceinline__ HDual atan2(const HDual& y, const HDual& x) {
    const double q = 1.0 / (x.v * x.v + y.v * y.v);
    const double fy = x.v * q, fx = -y.v * q;                     // d/dy, d/dx
    const double fyy = -2.0 * x.v * y.v * q * q, fxx = -fyy;      // d2/dy2, d2/dx2
    const double fxy = (y.v * y.v - x.v * x.v) * q * q;           // d2/dxdy
    HDual r;
    r.v = ::atan2(y.v, x.v);
    r.k = fy * y.k + fx * x.k;
#pragma unroll
    for (int i = 0; i < 6; i++) {
        r.d[i] = fy * y.d[i] + fx * x.d[i];
        r.m[i] = fy * y.m[i] + fx * x.m[i] + fyy * y.d[i] * y.k + fxx * x.d[i] * x.k +
                 fxy * (x.d[i] * y.k + y.d[i] * x.k);
    }
    return r;
}

__host__ __device__ __forceinline__ double val(const HDual& x) { return x.v; }

}  // namespace accel
