// jacobian.cuh — element maps that carry their Jacobian explicitly (forward-mode, sparse).
//
// The block-Jacobian tape of the adjoint needs, per particle and per unit of elements, the state
// and d(state)/d(unit input).  Dual numbers give that for any map but pay a full 6-direction
// product for every operation; the primitives of the tracking maps touch only two to four
// coordinates each, so here every primitive updates the state and the rows of the Jacobian it
// changes, with hand-derived partials taken at the primitive's input:
//
//   fastdrift   x += N px, y += N py, z -= w q   (N = L/D, w = N/(2D), D = 1 + delta, q = px^2 + py^2)
//               dx/dpx = N, dx/dd = -N px / D;  dz/dpx = -2 w px, dz/dpy = -2 w py, dz/dd = 2 w q / D
//   thin kick   px -= K Re P(z), py += K Im P(z), P = sum (B_n + i A_n) z^n, z = x + i y
//               dpx/dx = -K Re P', dpx/dy = K Im P', dpy/dx = K Im P', dpy/dy = K Re P'
//   bend edge   px += psi x, py -= psi y
//   hx drift    (atpass.cpp:343-355, coefficients a = L/D, b = hL^2/(4D^2), c = hL/(2D),
//               dd = L/(2D^2), g = hL/2; their delta-derivatives -a/D, -2b/D, -c/D, -2dd/D)
//   curved kick (atpass.cpp:199-235 without radiation)
//   cavity      delta += V sin(k z + phi): ddelta/dz = V k cos(k z + phi)
//
// m[i * NC + k] = d s_i / d in_k for k < 6; with NC = 7, column 6 is the derivative with respect
// to one element parameter (a multipole coefficient), whose explicit partial is added at each
// kick.  Rows are updated from the unchanged rows of the inputs, so no copy of the matrix is
// needed.  The values follow the fused tracker's maps (elem_fast.cuh) in exact arithmetic; the
// tape only needs them as linearisation points.
//
// ZD = false is for a run of elements in which nothing reads z or changes delta (no cavity):
// there the z column stays the unit vector e_z and the delta row stays e_delta, so the row
// updates skip column z and a term "a * row(delta)" only adds a to column delta.  Adding a * 0
// changes nothing, so this is the same arithmetic with the zero terms left out.
// ZR = false (only with ZD = false) also leaves the z row at e_z.  In a line where no element
// reads z, the adjoint of z is the seed's z component at every unit, so with a seed whose z
// component is zero the z row is multiplied by zero in the reverse sweep and need not be formed.
#pragma once
#include "engine.h"
#include "adjoint_params.h"

namespace accel {
namespace jac {

enum { X = 0, PX = 1, Y = 2, PY = 3, Z = 4, D = 5 };

template <int NC, bool ZD = true, bool ZR = true>
struct JS {
    static_assert(ZR || !ZD, "the z row may be left out only where nothing reads z");
    double s[6];
    double m[6 * NC];
};

// columns the row updates touch
__host__ __device__ constexpr bool live_col(bool zd, int k) { return zd || k != Z; }

template <int NC, bool ZD, bool ZR>
__device__ __forceinline__ void set_identity(JS<NC, ZD, ZR>& j) {
#pragma unroll
    for (int i = 0; i < 6 * NC; i++) j.m[i] = 0.0;
#pragma unroll
    for (int i = 0; i < 6; i++) j.m[i * NC + i] = 1.0;
}

// row[dst] += a * row[src]
template <int NC, bool ZD, bool ZR>
__device__ __forceinline__ void axpy(JS<NC, ZD, ZR>& j, int dst, int src, double a) {
#pragma unroll
    for (int k = 0; k < NC; k++)
        if (live_col(ZD, k)) j.m[dst * NC + k] = fma(a, j.m[src * NC + k], j.m[dst * NC + k]);
}

// row[dst] += a * row[delta]
template <int NC, bool ZD, bool ZR>
__device__ __forceinline__ void dterm(JS<NC, ZD, ZR>& j, int dst, double a) {
    if (ZD) axpy(j, dst, D, a);
    else j.m[dst * NC + D] += a;
}

// row[dst] += a * row[s1] + b * row[s2]
template <int NC, bool ZD, bool ZR>
__device__ __forceinline__ void add2(JS<NC, ZD, ZR>& j, int dst, int s1, double a, int s2, double b) {
#pragma unroll
    for (int k = 0; k < NC; k++)
        if (live_col(ZD, k))
            j.m[dst * NC + k] = fma(b, j.m[s2 * NC + k], fma(a, j.m[s1 * NC + k], j.m[dst * NC + k]));
}

// row[dst] += a * row[s1] + b * row[s2] + e * row[s3]
template <int NC, bool ZD, bool ZR>
__device__ __forceinline__ void add3(JS<NC, ZD, ZR>& j, int dst, int s1, double a, int s2, double b, int s3, double e) {
#pragma unroll
    for (int k = 0; k < NC; k++)
        if (live_col(ZD, k))
            j.m[dst * NC + k] =
                fma(e, j.m[s3 * NC + k], fma(b, j.m[s2 * NC + k], fma(a, j.m[s1 * NC + k], j.m[dst * NC + k])));
}

// row[dst] = c * row[dst] + a * row[s1] (+ b * row[s2])
template <int NC, bool ZD, bool ZR>
__device__ __forceinline__ void scale_add1(JS<NC, ZD, ZR>& j, int dst, double c, int s1, double a) {
#pragma unroll
    for (int k = 0; k < NC; k++)
        if (live_col(ZD, k)) j.m[dst * NC + k] = fma(a, j.m[s1 * NC + k], c * j.m[dst * NC + k]);
}
template <int NC, bool ZD, bool ZR>
__device__ __forceinline__ void scale_add2(JS<NC, ZD, ZR>& j, int dst, double c, int s1, double a, int s2, double b) {
#pragma unroll
    for (int k = 0; k < NC; k++)
        if (live_col(ZD, k))
            j.m[dst * NC + k] = fma(b, j.m[s2 * NC + k], fma(a, j.m[s1 * NC + k], c * j.m[dst * NC + k]));
}

__device__ __forceinline__ bool lost(const double* s) { return s[X] != s[X]; }

// fastdrift with NormL = N = L * inv, inv = 1 / (1 + delta)
template <int NC, bool ZD, bool ZR>
__device__ __forceinline__ void drift(JS<NC, ZD, ZR>& j, double N, double inv) {
    double* s = j.s;
    const double px = s[PX], py = s[PY];
    const double q = fma(px, px, py * py);
    const double w = 0.5 * N * inv;
    // z first: it reads the px, py, delta rows only, like x and y
    if constexpr (ZR) {
        add2(j, Z, PX, -2.0 * w * px, PY, -2.0 * w * py);
        dterm(j, Z, 2.0 * w * q * inv);
    }
    axpy(j, X, PX, N);
    dterm(j, X, -N * inv * px);
    axpy(j, Y, PY, N);
    dterm(j, Y, -N * inv * py);
    s[X] = fma(N, px, s[X]);
    s[Y] = fma(N, py, s[Y]);
    s[Z] = fma(-w, q, s[Z]);
}

// P(z) = sum_{n<=M} (B_n + i A_n) z^n and P'(z), Horner from order M.  A and B point into the
// element record (read through the cache), so a run-time order indexes no local array; A may be
// null (no skew terms).
__device__ __forceinline__ void poly(const double* __restrict__ A, const double* __restrict__ B, int M,
                                     double x, double y, double& pr, double& pi, double& dr, double& di) {
    pr = B[M];
    pi = A ? A[M] : 0.0;
    dr = 0.0;
    di = 0.0;
    for (int n = M - 1; n >= 0; n--) {
        // P' <- P' z + P, then P <- P z + c_n
        const double ndr = fma(dr, x, fma(-di, y, pr));
        const double ndi = fma(di, x, fma(dr, y, pi));
        dr = ndr;
        di = ndi;
        const double npr = fma(pr, x, fma(-pi, y, B[n]));
        const double npi = fma(pi, x, fma(pr, y, A ? A[n] : 0.0));
        pr = npr;
        pi = npi;
    }
}

// thin kick of weight K; with NC = 7 and a parameter (kind PK_B / PK_A of order pn), its explicit
// partial is added to column 6: d px/d B_n = -K Re z^n, d py/d B_n = K Im z^n,
// d px/d A_n = K Im z^n, d py/d A_n = K Re z^n.
template <int NC, bool ZD, bool ZR>
__device__ __forceinline__ void kick(JS<NC, ZD, ZR>& j, const double* A, const double* B, int M, double K, int pkind,
                                     int pn) {
    double* s = j.s;
    const double x = s[X], y = s[Y];
    double pr, pi, dr, di;
    poly(A, B, M, x, y, pr, pi, dr, di);
    const double a = K * dr, b = K * di;
    add2(j, PX, X, -a, Y, b);
    add2(j, PY, X, b, Y, a);
    if (NC == 7) {
        double zr = 1.0, zi = 0.0;
        for (int n = 0; n < pn; n++) {
            const double t = fma(zr, x, -zi * y);
            zi = fma(zr, y, zi * x);
            zr = t;
        }
        if (pkind == adj::PK_B) {
            j.m[PX * NC + NC - 1] = fma(-K, zr, j.m[PX * NC + NC - 1]);
            j.m[PY * NC + NC - 1] = fma(K, zi, j.m[PY * NC + NC - 1]);
        } else if (pkind == adj::PK_A) {
            j.m[PX * NC + NC - 1] = fma(K, zi, j.m[PX * NC + NC - 1]);
            j.m[PY * NC + NC - 1] = fma(K, zr, j.m[PY * NC + NC - 1]);
        }
    }
    s[PX] = fma(-K, pr, s[PX]);
    s[PY] = fma(K, pi, s[PY]);
}

// StrMPole (accel.cpp:800-847), Yoshida slices; delta is constant inside the element
template <int NC, bool ZD, bool ZR>
__device__ __forceinline__ void strmpole(JS<NC, ZD, ZR>& j, const DevElem& e, int pkind, int pn) {
    const double* A = e.v + V_A;
    const double* B = e.v + V_B;
    const int M = e.order_eff;
    if (e.op == OP_STRKICK) { kick(j, A, B, M, 1.0, pkind, pn); return; }
    const double inv = 1.0 / (1.0 + j.s[D]);
    const double N1 = e.v[V_L1] * inv, N2 = e.v[V_L2] * inv, K1 = e.v[V_K1], K2 = e.v[V_K2];
    // one copy of the drift and of the kick in the code, stepped through the slice's sequence
    // D1 K1 D2 K2 D2 K1 D1 (the tape kernel is large enough for instruction fetch to stall it)
#pragma unroll 1
    for (int m = 0; m < e.nslice; m++) {
#pragma unroll 1
        for (int k = 0; k < 4; k++) {
            drift(j, (k == 0 || k == 3) ? N1 : N2, inv);
            if (k < 3) kick(j, A, B, M, k == 1 ? K2 : K1, pkind, pn);
        }
    }
}

// hx drift of length L with curvature h at fixed delta (inv = 1 / (1 + delta))
template <bool ZD, bool ZR>
__device__ __forceinline__ void hxdrift(JS<6, ZD, ZR>& j, double L, double h, double inv) {
    double* s = j.s;
    const double px = s[PX], py = s[PY];
    const double a = inv * L, b = 0.25 * h * L * L * inv * inv, c = 0.5 * h * L * inv;
    const double dd = 0.5 * L * inv * inv, g = 0.5 * h * L;
    const double pxx = px * px, pyy = py * py, q = pxx + pyy;
    const double hx1 = fma(h, s[X], 1.0);
    const double gp = fma(g, px, 1.0);
    // z and y read the old x, px, py, delta rows; x then reads old px, py; px last
    if constexpr (ZR) {
        add3(j, Z, X, -h * dd * q, PX, -2.0 * hx1 * dd * px, PY, -2.0 * hx1 * dd * py);
        dterm(j, Z, 2.0 * inv * hx1 * dd * q);
    }
    add3(j, Y, X, h * a * py * gp, PX, hx1 * a * py * g, PY, hx1 * a * gp);
    dterm(j, Y, -inv * hx1 * a * py * gp);
    scale_add2(j, X, fma(h * px, a, 1.0), PX, fma(2.0 * b, px, hx1 * a), PY, -2.0 * b * py);
    dterm(j, X, -inv * fma(hx1 * px, a, 2.0 * b * (pxx - pyy)));
    scale_add1(j, PX, fma(-2.0 * c, px, 1.0), PY, -2.0 * c * py);
    dterm(j, PX, c * inv * q);
    s[X] = fma(hx1 * px, a, fma(b, pxx - pyy, s[X]));
    s[PX] = fma(-c, q, px);
    s[Y] = fma(hx1 * a * py, gp, s[Y]);
    s[Z] = fma(-hx1 * dd, q, s[Z]);
}

// curved kick of weight L (atpass.cpp:199-235, no radiation), field B[0..M] (no skew terms)
template <bool ZD, bool ZR>
__device__ __forceinline__ void bend_kick(JS<6, ZD, ZR>& j, const double* B, int M, double h, double K1, double K2,
                                          double L) {
    double* s = j.s;
    const double x = s[X], y = s[Y], x2 = x * x, y2 = y * y;
    double re, im, dr, di;
    poly(nullptr, B, M, x, y, re, im, dr, di);
    const double c43K2 = 4.0 / 3.0 * K2, c3 = h / 6.0 * K1 - K2 / 3.0;
    const double t1 = fma(h, x, fma(K1, fma(-0.5, y2, x2), K2 * x * fma(-4.0 / 3.0, y2, x2)));
    const double t1x = h + 2.0 * K1 * x + K2 * fma(3.0, x2, -4.0 / 3.0 * y2);
    const double t1y = -K1 * y - 8.0 / 3.0 * K2 * x * y;
    const double av = fma(h, t1, fma(-h, s[D], re));
    const double ax = fma(h, t1x, dr), ay = fma(h, t1y, -di), ad = -h;
    const double t2 = fma(x * y, fma(c43K2, x, K1), c3 * y2 * y);
    const double t2x = y * fma(2.0 * c43K2, x, K1), t2y = fma(x, fma(c43K2, x, K1), 3.0 * c3 * y2);
    add2(j, PX, X, -L * ax, Y, -L * ay);
    dterm(j, PX, -L * ad);
    add2(j, PY, X, L * fma(h, t2x, di), Y, L * fma(h, t2y, dr));
    if constexpr (ZR) axpy(j, Z, X, -L * h);
    s[PX] = fma(-L, av, s[PX]);
    s[PY] = fma(L, fma(h, t2, im), s[PY]);
    s[Z] = fma(-L * h, x, s[Z]);
}

// BendMPole without radiation (accel.cpp:649-705): edge, Yoshida slices, edge
template <bool ZD, bool ZR>
__device__ __forceinline__ void bendmpole(JS<6, ZD, ZR>& j, const DevElem& e) {
    const double* B = e.v + V_B;
    const int M = e.order_eff;
    const double h = e.v[V_IRHO], K1b = e.v[V_BK1], K2b = e.v[V_BK2];
    const double L1 = e.v[V_L1], L2 = e.v[V_L2], K1 = e.v[V_K1], K2 = e.v[V_K2];
    const double psi1 = e.v[V_PSI1], psi2 = e.v[V_PSI2];
    axpy(j, PX, X, psi1);
    axpy(j, PY, Y, -psi1);
    j.s[PX] = fma(j.s[X], psi1, j.s[PX]);
    j.s[PY] = fma(-j.s[Y], psi1, j.s[PY]);
    const double inv = 1.0 / (1.0 + j.s[D]);
#pragma unroll 1
    for (int m = 0; m < e.nslice; m++) {
#pragma unroll 1
        for (int k = 0; k < 4; k++) {
            hxdrift(j, (k == 0 || k == 3) ? L1 : L2, h, inv);
            if (k < 3) bend_kick(j, B, M, h, K1b, K2b, k == 1 ? K2 : K1);
        }
    }
    axpy(j, PX, X, psi2);
    axpy(j, PY, Y, -psi2);
    j.s[PX] = fma(j.s[X], psi2, j.s[PX]);
    j.s[PY] = fma(-j.s[Y], psi2, j.s[PY]);
}

template <int NC, bool ZD, bool ZR>
__device__ __forceinline__ void drift_len(JS<NC, ZD, ZR>& j, double L) {
    const double inv = 1.0 / (1.0 + j.s[D]);
    drift(j, L * inv, inv);
}

// Cavity (accel.cpp:903-923): reads z and changes delta, so only with ZD = true
__device__ __forceinline__ void cavity(JS<6, true>& j, const DevElem& e) {
    const double len = e.v[V_LEN];
    if (len != 0) drift_len(j, 0.5 * len);
    if (e.flags) {
        const double k = e.v[V_KZ], ph = fma(k, j.s[Z], e.v[V_PHIS]);
        axpy(j, D, Z, e.v[V_NV] * k * cos(ph));
        j.s[D] = fma(e.v[V_NV], sin(ph), j.s[D]);
    }
    if (len != 0) drift_len(j, 0.5 * len);
}

// Aperture (accel.cpp:337-387): a lost particle's x becomes NaN, which ends its tape
__device__ __forceinline__ bool aperture_hit(double* s, const DevElem& e) {
    const double a = e.v[V_XMIN], b = e.v[V_XMAX], c = e.v[V_YMIN], d = e.v[V_YMAX];
    if (s[X] <= a || s[X] >= b || s[Y] <= c || s[Y] >= d) {
        s[X] = __longlong_as_double(0x7ff8000000000000ll);
        return true;
    }
    return false;
}

}  // namespace jac
}  // namespace accel
