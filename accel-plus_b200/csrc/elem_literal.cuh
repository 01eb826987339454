// elem_literal.cuh — the reference's per-particle maps, operation for operation.
//
// Used by the plain per-element kernel (kern_plain.cu, built with --fmad=false so every add and
// multiply rounds separately, as on the x86-64 host) and, instantiated with Dual<N>, by the exact
// tangent map.  Each function keeps the operand order of the reference line it cites, which is
// what makes the plain kernel's doubles identical to the reference library's for the elements
// without per-particle transcendentals (drifts, multipoles, apertures, correctors, matrices).
// Parameter-only subexpressions (slice lengths, irho*tan(e), CRAD, ...) arrive precomputed in the
// element record (compile.cpp), evaluated on the host with the same operand order.
#pragma once
#include <type_traits>
#include <cmath>
#include "engine.h"
#include "dual.cuh"
#include "philox.cuh"

namespace accel {
namespace lit {

template <class T> __device__ __forceinline__ bool is_lost(const T& x) { double v = val(x); return v != v; }

// atpass.cpp:6-13 (path-length term as written: SQR(px + SQR(y)) with the advanced y)
template <class T>
__device__ __forceinline__ void drift(T* r, double L) {
    T p_norm = 1.0 / (1 + r[5]);
    r[0] += r[1] * L;
    r[2] += r[3] * L;
    r[4] -= (p_norm * p_norm) * L * ((r[1] + r[2] * r[2]) * (r[1] + r[2] * r[2])) / 2.0;
}

// atpass.cpp:416-428
template <class T, class U>
__device__ __forceinline__ void fastdrift(T* r, const U& NormL) {
    T dx = NormL * r[1];
    T dy = NormL * r[3];
    r[0] += dx;
    r[2] += dy;
    r[4] -= NormL * (r[1] * r[1] + r[3] * r[3]) / (2 * (1 + r[5]));
}

// atpass.cpp:358-414, Horner from max_order down (A, B in registers)
template <class T, class C>
__device__ __forceinline__ void strthinkick(T* r, const C* A, const C* B, double L, int max_order) {
    T ReSum = T(B[max_order]);
    T ImSum = T(A[max_order]);
    for (int i = max_order - 1; i >= 0; i--) {
        T ReSumTemp = ReSum * r[0] - ImSum * r[2] + B[i];
        ImSum = ImSum * r[0] + ReSum * r[2] + A[i];
        ReSum = ReSumTemp;
    }
    r[1] -= L * ReSum;
    r[3] += L * ImSum;
}

// atpass.cpp:343-355
template <class T>
__device__ __forceinline__ void bendhxdrift(T* r, double L, double h) {
    double hs = h * L;
    T i1pd = 1.0 / (1 + r[5]);
    T x = r[0], px = r[1], py = r[3];
    r[0] += (1 + h * x) * px * i1pd * L + 1 / 4. * hs * L * (px * px - py * py) * i1pd * i1pd;
    r[1] -= hs * (px * px + py * py) * i1pd / 2.0;
    r[2] += (1.0 + h * x) * i1pd * py * L * (1. + px * hs / 2.0);
    r[4] -= (1.0 + h * x) * i1pd * i1pd * L / 2.0 * (px * px + py * py);
}

// atpass.cpp:199-235
template <class T>
__device__ __forceinline__ void bndthinkick(T* r, const double* B, double K1, double K2, double L,
                                            double h, int max_order) {
    T ReSum = T(B[max_order]);
    T ImSum = T(0.0);
    for (int i = max_order - 1; i >= 0; i--) {
        T ReSumTemp = ReSum * r[0] - ImSum * r[2] + B[i];
        ImSum = ImSum * r[0] + ReSum * r[2];
        ReSum = ReSumTemp;
    }
    r[1] -= L * (-h * r[5] + ReSum + h * (h * r[0] + K1 * (r[0] * r[0] - 0.5 * r[2] * r[2]) + K2 * (r[0] * r[0] * r[0] - 4.0 / 3.0 * r[0] * r[2] * r[2])));
    r[3] += L * (ImSum + h * (K1 * r[0] * r[2] + 4.0 / 3.0 * K2 * r[0] * r[0] * r[2] + (h / 6.0 * K1 - K2 / 3.0) * r[2] * r[2] * r[2]));
    r[4] -= L * h * r[0];
}

// atpass.cpp:237-253
template <class T>
__device__ __forceinline__ T B2perp(const T& bx, const T& by, double irho, const T& x, const T& xpr,
                                    const T& ypr) {
    T v_norm2 = 1 / ((1 + x * irho) * (1 + x * irho) + xpr * xpr + ypr * ypr);
    T a = by * (1 + x * irho), b = bx * (1 + x * irho), c = bx * ypr - by * xpr;
    return (a * a + b * b + c * c) * v_norm2;
}

// atpass.cpp:255-339; `gauss` supplies the QE deviate (flag 2 only).
template <class T>
__device__ __forceinline__ void bndthinkickrad(T* r, const double* B, double K1, double K2, double L,
                                               double irho, double CRAD, double qecoef,
                                               int max_order, int flag_rad, double gauss) {
    T ReSum = T(B[max_order]);
    T ImSum = T(0.0);
    double h = irho;
    for (int i = max_order - 1; i >= 0; i--) {
        T ReSumTemp = ReSum * r[0] - ImSum * r[2] + B[i];
        ImSum = ImSum * r[0] + ReSum * r[2];
        ReSum = ReSumTemp;
    }
    T p_norm = 1 / (1 + r[5]);
    T x = r[0];
    T xpr = r[1] * p_norm;
    T y = r[2];
    T ypr = r[3] * p_norm;
    ImSum += h * (K1 * h - K2) * y * y * y / 6.0;
    ReSum += -K1 * h * y * y / 2.0 + h * (K1 * h - K2) * x * y * y / 2.0;
    T B2P = B2perp(ImSum, ReSum + irho, irho, x, xpr, ypr);
    if (flag_rad == 1) {
        r[5] = r[5] - CRAD * ((1 + r[5]) * (1 + r[5])) * B2P * (1 + x * irho + (xpr * xpr + ypr * ypr) / 2) * L;
    } else if (flag_rad == 2) {
        T mean_dpp = CRAD * ((1 + r[5]) * (1 + r[5])) * B2P * (1 + x * irho + (xpr * xpr + ypr * ypr) / 2) * L;
        T sigma_dpp = (val(mean_dpp) >= 0) ? sqrt(qecoef * mean_dpp) : sqrt((-qecoef) * mean_dpp);
        r[5] = r[5] - (mean_dpp + gauss * sigma_dpp);
    }
    p_norm = 1 / (1 + r[5]);
    r[1] = xpr / p_norm;
    r[3] = ypr / p_norm;
    r[1] -= L * (-h * r[5] + ReSum + h * (h * r[0] + K1 * (r[0] * r[0] - 0.5 * r[2] * r[2]) + K2 * (r[0] * r[0] * r[0] - 4.0 / 3.0 * r[0] * r[2] * r[2])));
    r[3] += L * (ImSum + h * (K1 * r[0] * r[2] + 4.0 / 3.0 * K2 * r[0] * r[0] * r[2] + (h / 6.0 * K1 - K2 / 3.0) * r[2] * r[2] * r[2]));
    r[4] -= L * h * r[0];
}

// atpass.cpp:15-72 (K is the element's parameter; KT carries a derivative when needed)
template <class T, class KT>
__device__ __forceinline__ void quad6(T* r, double L, const KT& K) {
    if (val(K) == 0) { drift(r, L); return; }
    T p_norm = 1 / (1 + r[5]);
    T x = r[0];
    T xpr = r[1] * p_norm;
    T y = r[2];
    T ypr = r[3] * p_norm;
    T g = fabs(K) / (1 + r[5]);
    T t = sqrt(g);
    T lt = L * t;
    T MHD, M12, M21, MVD, M34, M43;
    if (val(K) > 0) {
        MHD = cos(lt); M12 = sin(lt) / t; M21 = -M12 * g;
        MVD = cosh(lt); M34 = sinh(lt) / t; M43 = M34 * g;
    } else {
        MHD = cosh(lt); M12 = sinh(lt) / t; M21 = M12 * g;
        MVD = cos(lt); M34 = sin(lt) / t; M43 = -M34 * g;
    }
    r[0] = MHD * x + M12 * xpr;
    r[1] = (M21 * x + MHD * xpr) / p_norm;
    r[2] = MVD * y + M34 * ypr;
    r[3] = (M43 * y + MVD * ypr) / p_norm;
    r[4] -= g * (x * x * (L - MHD * M12) - y * y * (L - MVD * M34)) / 4;
    r[4] -= (xpr * xpr * (L + MHD * M12) + ypr * ypr * (L + MVD * M34)) / 4;
    r[4] -= (x * xpr * M12 * M21 + y * ypr * M34 * M43) / 2;
}

// atpass.cpp:76-187 with ByError = 0 (ABend::pass, accel.cpp:541)
template <class T>
__device__ __forceinline__ void bend6(T* r, double L, double b_angle, double grd) {
    const double ByError = 0;
    double Kx = b_angle / L;
    T p_norm = 1 / (1 + r[5]);
    T G1 = (Kx * Kx + grd) * p_norm;
    T G2 = -grd * p_norm;
    T MHD, M12, M21, MVD, M34, M43, sqrtG1 = T(0.0), arg1 = T(0.0);
    if (val(G1) == 0) { MHD = T(1.0); M12 = T(L); M21 = T(0.0); }
    else if (val(G1) > 0) {
        sqrtG1 = sqrt(G1); arg1 = L * sqrtG1;
        MHD = cos(arg1); M12 = sin(arg1) / sqrtG1; M21 = -sin(arg1) * sqrtG1;
    } else {
        sqrtG1 = sqrt(-G1); arg1 = L * sqrtG1;
        MHD = cosh(arg1); M12 = sinh(arg1) / sqrtG1; M21 = sinh(arg1) * sqrtG1;
    }
    if (val(G2) == 0) { MVD = T(1.0); M34 = T(L); M43 = T(0.0); }
    else if (val(G2) > 0) {
        T sqrtG2 = sqrt(G2); T arg2 = L * sqrtG2;
        MVD = cos(arg2); M34 = sin(arg2) / sqrtG2; M43 = -sin(arg2) * sqrtG2;
    } else {
        T sqrtG2 = sqrt(-G2); T arg2 = L * sqrtG2;
        MVD = cosh(arg2); M34 = sinh(arg2) / sqrtG2; M43 = sinh(arg2) * sqrtG2;
    }
    T x = r[0], xpr = r[1] * p_norm, y = r[2], ypr = r[3] * p_norm, delta = r[5];
    r[0] = MHD * x + M12 * xpr;
    r[1] = (M21 * x + MHD * xpr) / p_norm;
    T dpb = delta * p_norm - ByError;
    if (val(G1) == 0) {
        r[0] += dpb * L * L * Kx / 2;
        r[1] += dpb * L * Kx / p_norm;
    } else if (val(G1) > 0) {
        r[0] += dpb * (1 - cos(arg1)) * Kx / G1;
        r[1] += dpb * sin(arg1) * Kx / (sqrtG1 * p_norm);
    } else {
        r[0] += dpb * (1 - cosh(arg1)) * Kx / G1;
        r[1] += dpb * sinh(arg1) * Kx / (sqrtG1 * p_norm);
    }
    r[2] = MVD * y + M34 * ypr;
    r[3] = (M43 * y + MVD * ypr) / p_norm;
    r[4] -= xpr * xpr * (L + MHD * M12) / 4;
    if (val(G1) != 0) {
        r[4] -= (L - MHD * M12) * (x * x * G1 + dpb * dpb * Kx * Kx / G1 - 2 * x * Kx * dpb) / 4;
        r[4] -= M12 * M21 * (x * xpr - xpr * dpb * Kx / G1) / 2;
        r[4] -= Kx * x * M12 + xpr * (1 - MHD) * Kx / G1 + dpb * (L - M12) * Kx * Kx / G1;
    }
    r[4] -= ((L - MVD * M34) * y * y * G2 + ypr * ypr * (L + MVD * M34)) / 4;
    r[4] -= M34 * M43 * y * ypr / 2;
}

// AAperture test (accel.cpp:350-354): code into z, NaN into x.
template <class T>
__device__ __forceinline__ bool aperture_test(T* r, double xmin, double xmax, double ymin, double ymax) {
    double x = val(r[0]), y = val(r[2]);
    if (x <= xmin || x >= xmax || y <= ymin || y >= ymax) {
        r[4] = T((double)((x <= xmin) * 1 + (x >= xmax) * 2 + (y <= ymin) * 3 + (y >= ymax) * 4));
        r[0] = T(nan(""));
        return true;
    }
    return false;
}

// Normal deviate source for QE: counter = (pid, turn, element, kick); kick counts up.
struct QeSource {
    uint64_t seed;
    uint32_t pid, turn, elem, kick;
    __device__ double next() { return qe_normal(seed, pid, turn, elem, kick++); }
};

// One element on one particle.  Returns without touching a lost particle (x NaN), which is what
// every reference pass method does first (e.g. accel.cpp:166-167).
// WigTable interpolation (interp2, utility.cpp:174-188): the bilinear interpolation of a table
// on a rectangular grid from Numerical Recipes 3rd ed. (Bilin_interp, interp_2d.h), restated.
// The cell is found by bisection on a monotonic grid of n >= 2 points (the book's locate,
// interp_1d.h), so a point outside the grid is extrapolated from the edge cell.
__device__ __forceinline__ int grid_cell(const double* g, int n, double x) {
    const bool ascending = g[n - 1] >= g[0];
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        int mid = (hi + lo) >> 1;
        if ((x >= g[mid]) == ascending) lo = mid;
        else hi = mid;
    }
    return lo;
}

// t, u: the point's fractions across cell (i, j); z: a table [my][mx], z[jj*mx + ii] at
// (xl[ii], yl[jj]).  Sum and product order as written in the book.
template <class T>
__device__ __forceinline__ T bilinear(const double* z, int mx, int i, int j, const T& t, const T& u) {
    const double z00 = z[j * mx + i], z10 = z[j * mx + i + 1];
    const double z01 = z[(j + 1) * mx + i], z11 = z[(j + 1) * mx + i + 1];
    return (1. - t) * (1. - u) * z00 + t * (1. - u) * z10 + (1. - t) * u * z01 + t * u * z11;
}

template <class T>
__device__ void pass(const DevElem& e, T* r, QeSource& q) {
    if (is_lost(r[0])) return;
    const double len = e.v[V_LEN];
    switch (e.op) {
    case OP_NOP:
        return;
    case OP_DRIFT:  // accel.cpp:158-177
        fastdrift(r, len / (1.0 + r[5]));
        return;
    case OP_STRKICK: {  // accel.cpp:824-827
        double A[ACCEL_MAX_MPOLE], B[ACCEL_MAX_MPOLE];
#pragma unroll
        for (int i = 0; i < ACCEL_MAX_MPOLE; i++) { A[i] = e.v[V_A + i]; B[i] = e.v[V_B + i]; }
        strthinkick(r, A, B, 1.0, ACCEL_MAX_MPOLE - 1);
        return;
    }
    case OP_STRMPOLE: {  // accel.cpp:800-847
        double A[ACCEL_MAX_MPOLE], B[ACCEL_MAX_MPOLE];
#pragma unroll
        for (int i = 0; i < ACCEL_MAX_MPOLE; i++) { A[i] = e.v[V_A + i]; B[i] = e.v[V_B + i]; }
        const double L1 = e.v[V_L1], L2 = e.v[V_L2], K1 = e.v[V_K1], K2 = e.v[V_K2];
        for (int m = 0; m < e.nslice; m++) {
            T norm = 1 / (1 + r[5]);
            T NormL1 = L1 * norm, NormL2 = L2 * norm;
            fastdrift(r, NormL1);
            strthinkick(r, A, B, K1, ACCEL_MAX_MPOLE - 1);
            fastdrift(r, NormL2);
            strthinkick(r, A, B, K2, ACCEL_MAX_MPOLE - 1);
            fastdrift(r, NormL2);
            strthinkick(r, A, B, K1, ACCEL_MAX_MPOLE - 1);
            fastdrift(r, NormL1);
        }
        return;
    }
    case OP_BENDMPOLE: {  // accel.cpp:649-705
        double B[ACCEL_MAX_MPOLE];
#pragma unroll
        for (int i = 0; i < ACCEL_MAX_MPOLE; i++) B[i] = e.v[V_B + i];
        const double L1 = e.v[V_L1], L2 = e.v[V_L2], K1 = e.v[V_K1], K2 = e.v[V_K2], SL = e.v[V_SL];
        const double h = e.v[V_IRHO], bk1 = e.v[V_BK1], bk2 = e.v[V_BK2];
        const double crad = e.v[V_CRAD], qec = e.v[V_QECOEF];
        const int mo = e.order_lit, rad = e.flags;
        // edge(e1): psi precomputed as irho*tan(e1) (atpass.cpp:190-196)
        r[1] += r[0] * e.v[V_PSI1];
        r[3] -= r[2] * e.v[V_PSI1];
        for (int m = 0; m < e.nslice; m++) {
            if (rad <= 1) {
                bendhxdrift(r, L1, h);
                if (rad) bndthinkickrad(r, B, bk1, bk2, K1, h, crad, qec, mo, rad, 0.0);
                else bndthinkick(r, B, bk1, bk2, K1, h, mo);
                bendhxdrift(r, L2, h);
                if (rad) bndthinkickrad(r, B, bk1, bk2, K2, h, crad, qec, mo, rad, 0.0);
                else bndthinkick(r, B, bk1, bk2, K2, h, mo);
                bendhxdrift(r, L2, h);
                if (rad) bndthinkickrad(r, B, bk1, bk2, K1, h, crad, qec, mo, rad, 0.0);
                else bndthinkick(r, B, bk1, bk2, K1, h, mo);
                bendhxdrift(r, L1, h);
            } else {
                bendhxdrift(r, 0.5 * SL, h);
                bndthinkickrad(r, B, bk1, bk2, SL, h, crad, qec, mo, rad, q.next());
                bendhxdrift(r, 0.5 * SL, h);
            }
        }
        r[1] += r[0] * e.v[V_PSI2];
        r[3] -= r[2] * e.v[V_PSI2];
        return;
    }
    case OP_QUAD:  // accel.cpp:193-209
        quad6(r, len, e.v[V_QK]);
        return;
    case OP_BEND:  // accel.cpp:523-550
        r[1] += r[0] * e.v[V_BPSI1];
        r[3] -= r[2] * e.v[V_BPSI1];
        bend6(r, len, e.v[V_THETA], e.v[V_GRD]);
        r[1] += r[0] * e.v[V_BPSI2];
        r[3] -= r[2] * e.v[V_BPSI2];
        return;
    case OP_CAVITY: {  // accel.cpp:903-923
        if (len != 0) fastdrift(r, 0.5 * len / (1 + r[5]));
        if (e.flags) r[5] += e.v[V_NV] * sin(e.v[V_TF] * r[4] / 2.99792458e8 + e.v[V_PHIS]);
        if (len != 0) fastdrift(r, 0.5 * len / (1 + r[5]));
        return;
    }
    case OP_APERTURE: {  // accel.cpp:337-387
        const double a = e.v[V_XMIN], b = e.v[V_XMAX], c = e.v[V_YMIN], d = e.v[V_YMAX];
        if (aperture_test(r, a, b, c, d)) return;
        if (len != 0) {
            fastdrift(r, len / (1 + r[5]));
            aperture_test(r, a, b, c, d);
        }
        return;
    }
    case OP_CRABCAV: {  // accel.cpp:991-1032
        const double k = e.v[V_CK];
        if (len != 0) fastdrift(r, 0.5 * len / (1 + r[5]));
        if (e.flags) {
            T omega_t = -k * r[4] + e.v[V_CPHIS];
            if (e.v[V_CSIGPHI] > 0) omega_t = omega_t + e.v[V_CSIGPHI] * q.next();
            double nvxa = e.v[V_CNVX], nvya = e.v[V_CNVY];
            if (e.v[V_CSIGDVV] > 0) {
                nvxa = nvxa * (1.0 + e.v[V_CSIGDVV] * q.next());
                nvya = nvya * (1.0 + e.v[V_CSIGDVV] * q.next());
            }
            r[1] += nvxa * sin(omega_t);
            r[3] += nvya * sin(omega_t);
            r[5] += -(nvya * r[2] + nvxa * r[0]) * k * cos(omega_t) / (1 + r[5]);
        }
        if (len != 0) fastdrift(r, 0.5 * len / (1 + r[5]));
        return;
    }
    case OP_RFMULT: {  // accel.cpp:1146-1197, cylindrical sums of the RF multipole
        const double k = e.v[V_RK];
        if (len != 0) fastdrift(r, 0.5 * len / (1 + r[5]));
        T omega_t = -k * r[4] + e.v[V_RPHIS];
        if (e.v[V_RSIGPHI] > 0) omega_t = omega_t + e.v[V_RSIGPHI] * q.next();
        const int M = (int)e.v[V_RM];
        if constexpr (std::is_same<T, double>::value) {
            T rho = sqrt(r[0] * r[0] + r[2] * r[2]);
            T phis = atan2(r[2], r[0]);
            T AsL = T(0.0), ArhoL = T(0.0), AphiL = T(0.0), nrho = T(1.0);
            for (int n = 0; n < M; n++) {
                T nphi = (double)(n + 1) * phis;
                T td = e.v[V_B + n] * cos(nphi) + e.v[V_A + n] * sin(nphi);
                ArhoL += nrho * td;
                AphiL += nrho * (-e.v[V_B + n] * sin(nphi) + e.v[V_A + n] * cos(nphi));
                nrho = nrho * rho;
                AsL += 1.0 / (n + 1) * nrho * td;
            }
            r[1] += (ArhoL * cos(phis) - AphiL * sin(phis)) * cos(omega_t);
            r[3] += (ArhoL * sin(phis) + AphiL * cos(phis)) * cos(omega_t);
            r[5] += k * AsL * sin(omega_t) / (1. + r[5]);
        } else {
            // the same kicks in Cartesian form, smooth at x = y = 0 for derivative types:
            // with c_n = B_n - i A_n and z = x + i y, P = sum c_n z^n, Q = sum c_n z^(n+1) / (n+1);
            // dpx = Re P cos(wt), dpy = -Im P cos(wt), d(delta) = k Re Q sin(wt) / (1 + delta)
            T zr = T(1.0), zi = T(0.0), Pr = T(0.0), Pi = T(0.0), Qr = T(0.0);
            for (int n = 0; n < M; n++) {
                const double cr = e.v[V_B + n], ci = -e.v[V_A + n];
                Pr += cr * zr - ci * zi;
                Pi += cr * zi + ci * zr;
                T nr = zr * r[0] - zi * r[2];
                zi = zr * r[2] + zi * r[0];
                zr = nr;
                Qr += (cr * zr - ci * zi) / (double)(n + 1);
            }
            r[1] += Pr * cos(omega_t);
            r[3] -= Pi * cos(omega_t);
            r[5] += k * Qr * sin(omega_t) / (1. + r[5]);
        }
        if (len != 0) fastdrift(r, 0.5 * len / (1 + r[5]));
        return;
    }
    case OP_IDEALWIG: {  // accel.cpp:1463-1533
        if (len == 0) return;
        const double k = e.v[V_WK], h = e.v[V_WH], crad = e.v[V_WCRAD];
        const int ns = e.nslice, wt = (int)e.v[V_WTYPE];
        const bool rad = e.flags != 0;
        auto rad_kick = [&]() {
            T dp = r[5];
            T yp = r[3] / (1 + dp);
            T xp = r[1] / (1 + dp);
            r[5] = r[5] - crad * ((1 + r[5]) * (1 + r[5])) * h * h * len / ns / 2.0;
            r[1] = xp * (1 + r[5]);
            r[3] = yp * (1 + r[5]);
        };
        for (int j = 0; j < ns; j++) {
            fastdrift(r, 0.5 * len / (1 + r[5]) / ns);
            T y = r[2];
            T x = r[0];
            if (rad) rad_kick();
            if (wt == 0) {
                T y3 = y * y * y;
                double k2 = k * k;
                r[3] -= h * h * (0.5 * y + 1.0 / 3.0 * y3 * k2 + 1.0 / 15.0 * y3 * y * y * k2 * k2) * len / ns;
            } else if (wt == 1) {
                T x3 = x * x * x;
                double k2 = k * k;
                r[1] -= h * h * (0.5 * x + 1.0 / 3.0 * x3 * k2 + 1.0 / 15.0 * x3 * x * x * k2 * k2) * len / ns;
            }
            if (rad) rad_kick();
            fastdrift(r, 0.5 * len / (1 + r[5]) / ns);
        }
        return;
    }
    case OP_WIGTABLE: {  // accel.cpp:1335-1377
        const int mx = (int)e.v[V_TMX], my = (int)e.v[V_TMY], ns = e.nslice;
        const double* tab;
        memcpy(&tab, &e.v[V_TPTR], sizeof(tab));
        const double* xl = tab;
        const double* yl = tab + mx;
        const double* xk = yl + my;
        const double* yk = xk + mx * my;
        // both kicks at the point (x, y); the reference interpolates each table separately, with
        // the same cell and fractions
        auto kicks = [&](T& kx, T& ky) {
            const T x = r[0], y = r[2];
            const int i = grid_cell(xl, mx, val(x)), j = grid_cell(yl, my, val(y));
            const T t = (x - xl[i]) / (xl[i + 1] - xl[i]);
            const T u = (y - yl[j]) / (yl[j + 1] - yl[j]);
            kx = bilinear(xk, mx, i, j, t, u);
            ky = bilinear(yk, mx, i, j, t, u);
        };
        if (len == 0) {
            T kx, ky;
            kicks(kx, ky);
            r[1] += kx;
            r[3] += ky;
            return;
        }
        const double hl = e.v[V_THL];
        for (int j = 0; j < ns; j++) {
            fastdrift(r, hl / (1 + r[5]) / ns);
            T kx, ky;
            kicks(kx, ky);
            r[1] += kx / ns;
            r[3] += ky / ns;
            fastdrift(r, hl / (1 + r[5]) / ns);
        }
        return;
    }
    case OP_CORRECTOR: {  // accel.cpp:270-292
        T pn = (1 + r[5]);
        if (len != 0) fastdrift(r, 0.5 * len / pn);
        r[1] += e.v[V_KX] / pn;
        r[3] += e.v[V_KY] / pn;
        if (len != 0) fastdrift(r, 0.5 * len / pn);
        return;
    }
    case OP_MATRIX: {  // accel.cpp:1699-1730
        if (len != 0) fastdrift(r, 0.5 * len / (1 + r[5]));
        T tr[6];
#pragma unroll
        for (int j = 0; j < 6; j++) {
            const double* m = e.v + V_MAT + 6 * j;
            tr[j] = m[0] * r[0] + m[1] * r[1] + m[2] * r[2] + m[3] * r[3] + m[4] * r[4] + m[5] * r[5];
        }
#pragma unroll
        for (int j = 0; j < 6; j++) r[j] = tr[j];
        if (len != 0) fastdrift(r, 0.5 * len / (1 + r[5]));
        return;
    }
    case OP_SYNCRAD: {  // accel.cpp:1806-1854
        if (len != 0) fastdrift(r, 0.5 * len / (1 + r[5]));
        if (e.flags & 1) {
            r[0] *= (1 - e.v[V_ALFX]);
            r[2] *= (1 - e.v[V_ALFY]);
            r[5] *= (1 - e.v[V_ALFZ]);
        }
        if (e.flags & 2) {
            r[0] += e.v[V_SIGX] * e.v[V_SX] * q.next();
            r[2] += e.v[V_SIGY] * e.v[V_SY] * q.next();
            r[5] += e.v[V_SIGD] * e.v[V_SZ] * q.next();
        }
        if (len != 0) fastdrift(r, 0.5 * len / (1 + r[5]));
        return;
    }
    default:
        return;  // collective elements are applied by their own kernels
    }
}

}  // namespace lit
}  // namespace accel
