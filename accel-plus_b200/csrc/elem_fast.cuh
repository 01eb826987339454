// elem_fast.cuh — register-resident element maps for the fused persistent kernel.
//
// Same integrators as the reference (atpass.cpp), rearranged for the FP64 pipe:
//  * the six coordinates live in registers for the whole turn (struct St);
//  * multipole Horner sums start at the element's highest non-zero coefficient (the reference
//    always starts at index 9 for StrMPole, accel.cpp:826,837-841, and at MaxNPole-1 for
//    BendMPole; the leading zero terms add exact zeros for finite coordinates);
//  * 1/(1+delta) is formed once per element where delta cannot change inside it (no radiation),
//    and the element's per-slice constants are folded with it;
//  * the adjacent full-length drifts that end one Yoshida slice and begin the next are merged;
//  * in radiating bends the hx-drift constants are formed once per element and 1/(1+delta)
//    enters through the angles, and the radiated power of a pure dipole field uses
//    |B x v|^2 = By^2 ((1+hx)^2 + x'^2);
//  * a*b+c contracts to FMA.
// None of these changes the map beyond rounding; the parity tests bound the difference.
#pragma once
#include <cmath>
#include "engine.h"
#include "philox.cuh"

namespace accel {
namespace fast {

struct St { double x, px, y, py, z, d; };

// Elements and multipole orders outside the specialised paths run the literal map through one
// out-of-line call that takes and returns the state by value (defined in kern_fused.cu), so the
// hot path's state never has its address taken and stays in registers.
__device__ __noinline__ St rare_elem(St s, const DevElem* __restrict__ e, uint64_t seed,
                                     uint32_t pid, uint32_t turn);

__device__ __forceinline__ double rcp(double a) { return __drcp_rn(a); }

// fastdrift with NormL = nl and nlh = nl / (2 (1 + delta)) (atpass.cpp:416-428)
__device__ __forceinline__ void drift(St& s, double nl, double nlh) {
    double q = fma(s.px, s.px, s.py * s.py);
    s.x = fma(nl, s.px, s.x);
    s.y = fma(nl, s.py, s.y);
    s.z = fma(-nlh, q, s.z);
}

// Straight multipole kick (atpass.cpp:358-414) at compile-time order M.  SK is the skew level:
// 0 no skew terms, 1 only A[0] (a skew dipole, e.g. the feed-down of a vertical offset),
// 2 skew terms up to A[M].
template <int M, int SK>
__device__ __forceinline__ void kick(St& s, const double* A, const double* B, double K) {
    if constexpr (M == 0) {
        s.px = fma(-K, B[0], s.px);
        if (SK) s.py = fma(K, A[0], s.py);
    } else {
        double re = B[M];
        double im = (SK == 2) ? A[M] : 0.0;
#pragma unroll
        for (int i = M - 1; i >= 0; i--) {
            const bool first = (i == M - 1) && SK != 2;  // im is still exactly zero
            const bool use_a = (SK == 2 || (SK == 1 && i == 0));
            double nre, nim;
            if (first) {
                nre = fma(re, s.x, B[i]);
                nim = use_a ? fma(re, s.y, A[i]) : re * s.y;
            } else {
                nre = fma(re, s.x, fma(-im, s.y, B[i]));
                nim = use_a ? fma(im, s.x, fma(re, s.y, A[i])) : fma(im, s.x, re * s.y);
            }
            re = nre;
            im = nim;
        }
        s.px = fma(-K, re, s.px);
        s.py = fma(K, im, s.py);
    }
}

// AStrMPole::pass (accel.cpp:800-847), len > 0, effective order M, skew level SK.
template <int M, int SK>
__device__ __forceinline__ void strmpole(St& s, const DevElem* __restrict__ e) {
    double A[M + 1], B[M + 1];
#pragma unroll
    for (int i = 0; i <= M; i++) {
        B[i] = e->h[H_B + i];
        A[i] = (SK == 2 || (SK == 1 && i == 0)) ? e->h[H_A + i] : 0.0;
    }
    const double L1 = e->h[H_L1], L2 = e->h[H_L2], K1 = e->h[H_K1], K2 = e->h[H_K2];
    const int ns = e->nslice;
    const double inv = rcp(1.0 + s.d);
    const double h = 0.5 * inv;
    const double nl1 = L1 * inv, nl2 = L2 * inv;
    const double nlh1 = nl1 * h, nlh2 = nl2 * h;
    drift(s, nl1, nlh1);
    for (int m = 0; m < ns; m++) {
        kick<M, SK>(s, A, B, K1);
        drift(s, nl2, nlh2);
        kick<M, SK>(s, A, B, K2);
        drift(s, nl2, nlh2);
        kick<M, SK>(s, A, B, K1);
        if (m + 1 < ns) drift(s, 2.0 * nl1, 2.0 * nlh1);
    }
    drift(s, nl1, nlh1);
}

// flags: STR_SKEW set when any A is non-zero; STR_SKEW0 when A[0] is the only one.
__device__ __forceinline__ void strmpole_dispatch(St& s, const DevElem* __restrict__ e) {
    const int sk = (e->flags & STR_SKEW) ? ((e->flags & STR_SKEW0) ? 1 : 2) : 0;
    switch (e->order_eff * 4 + sk) {
    case 0: strmpole<0, 0>(s, e); break;
    case 1: strmpole<0, 1>(s, e); break;
    case 2: strmpole<0, 2>(s, e); break;
    case 4: strmpole<1, 0>(s, e); break;
    case 5: strmpole<1, 1>(s, e); break;
    case 6: strmpole<1, 2>(s, e); break;
    case 8: strmpole<2, 0>(s, e); break;
    case 9: strmpole<2, 1>(s, e); break;
    case 10: strmpole<2, 2>(s, e); break;
    case 12: strmpole<3, 0>(s, e); break;
    case 13: strmpole<3, 1>(s, e); break;
    case 14: strmpole<3, 2>(s, e); break;
    default: s = rare_elem(s, e, 0, 0, 0); break;
    }
}

// ---- BendMPole ------------------------------------------------------------------------------
// hx drift (atpass.cpp:343-355) with delta fixed: a = L/(1+d), b = hL^2/(4(1+d)^2),
// c = hL/(2(1+d)), dd = L/(2(1+d)^2), g = hL/2
struct HxCoef { double a, b, c, dd, g; };

__device__ __forceinline__ HxCoef hx_coef(double L, double h, double inv) {
    HxCoef k;
    const double hs = h * L, inv2 = inv * inv;
    k.a = inv * L;
    k.b = (0.25 * hs * L) * inv2;
    k.c = (0.5 * hs) * inv;
    k.dd = (0.5 * L) * inv2;
    k.g = 0.5 * hs;
    return k;
}

__device__ __forceinline__ void hxdrift(St& s, double h, const HxCoef& k) {
    double px = s.px, py = s.py;
    double pxx = px * px, pyy = py * py;
    double q = pxx + pyy;
    double hx1 = fma(h, s.x, 1.0);
    s.x = fma(hx1 * px, k.a, fma(k.b, pxx - pyy, s.x));
    s.px = fma(-k.c, q, px);
    s.y = fma(hx1 * k.a * py, fma(px, k.g, 1.0), s.y);
    s.z = fma(-hx1 * k.dd, q, s.z);
}

// The same hx drift while delta changes between drifts (radiation): the element constants
// L, hL/2, L/2 and hL^2/4 are formed once, and 1/(1+delta) enters through the angles
// P = px/(1+d), Q = py/(1+d): x += (1+hx) L P + (hL^2/4)(P^2 - Q^2), px -= (hL/2)(P px + Q py),
// y += (1+hx) L Q (1 + (hL/2) px), z -= (1+hx)(L/2)(P^2 + Q^2).
struct HxConst { double L, c, dd, b; };  // L, hL/2, L/2, hL^2/4

__device__ __forceinline__ HxConst hx_const(double L, double h) {
    return HxConst{L, 0.5 * h * L, 0.5 * L, 0.25 * h * L * L};
}

__device__ __forceinline__ void hxdrift_inv(St& s, double h, const HxConst& k, double inv) {
    const double px = s.px, py = s.py;
    const double P = px * inv, Q = py * inv;
    const double QQ = Q * Q;
    const double s2 = fma(P, P, QQ), d2 = fma(P, P, -QQ);
    const double hx1 = fma(h, s.x, 1.0);
    const double hL = hx1 * k.L;
    s.x = fma(hL, P, fma(k.b, d2, s.x));
    s.px = fma(-k.c, fma(P, px, Q * py), px);
    s.y = fma(hL * Q, fma(px, k.c, 1.0), s.y);
    s.z = fma(-hx1 * k.dd, s2, s.z);
}

// Horner over B only (bendMPole kicks carry no skew terms), order M
template <int M>
__device__ __forceinline__ void horner_b(const St& s, const double* B, double& re, double& im) {
    re = B[M];
    im = 0.0;
#pragma unroll
    for (int i = M - 1; i >= 0; i--) {
        double nre, nim;
        if (i == M - 1) {
            nre = fma(re, s.x, B[i]);
            nim = re * s.y;
        } else {
            nre = fma(re, s.x, fma(-im, s.y, B[i]));
            nim = fma(im, s.x, re * s.y);
        }
        re = nre;
        im = nim;
    }
}

// Element constants of the curved kick (atpass.cpp:199-235)
struct BkCoef {
    double h, K1, K2, c43K2, c3;   // c3 = h/6 K1 - K2/3
    double cI, cR1, cR2;           // radiation: h(K1 h - K2)/6, -K1 h/2, h(K1 h - K2)/2
};

// With K1 = K2 = 0 (a pure dipole field plus B[0..M]) the curved kick reduces to
// px -= L (re + h (h x - delta)), py += L im, z -= L h x.
// NOIM: the field has no imaginary part at all (a dipole field B[0] alone, M = 0, and K1 = K2 =
// 0), so the vertical kick is zero and is skipped (fma(L, 0, py) = py for finite L).
template <bool PURE, bool NOIM = false>
__device__ __forceinline__ void bend_kick_core(St& s, const BkCoef& c, double re, double im,
                                               double L) {
    if (PURE) {
        s.px = fma(-L, fma(c.h, fma(c.h, s.x, -s.d), re), s.px);
        if (!NOIM) s.py = fma(L, im, s.py);
        s.z = fma(-L * c.h, s.x, s.z);
        return;
    }
    double x = s.x, y = s.y;
    double x2 = x * x, y2 = y * y;
    double t1 = fma(c.h, x, fma(c.K1, fma(-0.5, y2, x2), c.K2 * x * fma(-4.0 / 3.0, y2, x2)));
    double a = fma(c.h, t1, fma(-c.h, s.d, re));
    s.px = fma(-L, a, s.px);
    double t2 = fma(x * y, fma(c.c43K2, x, c.K1), c.c3 * y2 * y);
    s.py = fma(L, fma(c.h, t2, im), s.py);
    s.z = fma(-L * c.h, x, s.z);
}

// bndthinkickrad (atpass.cpp:255-339); returns the new 1/(1+delta) for the following drift.
// The energy loss per kick D is tiny (|D/(1+delta)| ~ 1e-7), so the new inverse is the old one
// times 1/(1-u), u = D/(1+delta), summed to u^3 (truncation below 1e-20 relative); a loss
// above |u| = 1e-4 takes the exact reciprocal.
// cradL = crad x L, the element's radiation constant times the kick's length.
template <int M, int RAD, bool PURE>
__device__ __forceinline__ double bend_kick_rad(St& s, const double* B, const BkCoef& c, double L,
                                                double cradL, double qec, double inv, double gauss) {
    double re, im;
    horner_b<M>(s, B, re, im);
    double x = s.x, y = s.y, y2 = y * y;
    double xpr = s.px * inv, ypr = s.py * inv;
    if (!PURE) {
        im = fma(c.cI, y2 * y, im);
        re = fma(y2, fma(c.cR2, x, c.cR1), re);
    }
    double hx1 = fma(x, c.h, 1.0);
    double by = re + c.h, bx = im;
    // with no imaginary field (M = 0, PURE) bx is exactly 0 and its terms are +0: left out, and
    // |B x v|^2 = by^2 ((1+hx)^2 + x'^2) since the cross term by x' has no partner
    constexpr bool NOIM = (M == 0) && PURE;
    double xx = xpr * xpr, yy = ypr * ypr;
    double vq = xx + yy;
    double b2p;
    if constexpr (NOIM) {
        double t = fma(hx1, hx1, xx);
        b2p = (by * by) * t * rcp(t + yy);
    } else {
        double vn2 = rcp(fma(hx1, hx1, vq));
        double cr = fma(bx, ypr, -by * xpr);
        b2p = fma(by * hx1, by * hx1, fma(bx * hx1, bx * hx1, cr * cr)) * vn2;
    }
    double opd = 1.0 + s.d;
    double mean = cradL * (opd * opd) * b2p * fma(0.5, vq, hx1);
    double loss;
    if (RAD == 1) {
        loss = mean;
    } else {
        double sig = sqrt(fabs(qec * mean));
        loss = fma(gauss, sig, mean);
    }
    s.d = s.d - loss;
    double opd2 = 1.0 + s.d;
    s.px = xpr * opd2;
    s.py = ypr * opd2;
    bend_kick_core<PURE, NOIM>(s, c, re, im, L);
    const double u = loss * inv;  // 1/(1+d-D) = inv (1 + u + u^2 + u^3 + ...)
    if (fabs(u) < 1e-4) return fma(inv * u, fma(u, u, u) + 1.0, inv);
    return rcp(opd2);
}

template <int M, bool PURE>
__device__ __forceinline__ void bendmpole(St& s, const DevElem* __restrict__ e,
                                          uint64_t seed, uint32_t pid, uint32_t turn) {
    double B[M + 1];
#pragma unroll
    for (int i = 0; i <= M; i++) B[i] = e->h[H_BB + i];
    const int rad = e->flags;
    const int ns = e->nslice;
    BkCoef c;
    c.h = e->h[H_IRHO];
    c.K1 = e->h[H_BK1];
    c.K2 = e->h[H_BK2];
    c.c43K2 = 4.0 / 3.0 * c.K2;
    c.c3 = c.h / 6.0 * c.K1 - c.K2 / 3.0;
    double kh = c.K1 * c.h - c.K2;
    c.cI = c.h * kh / 6.0;
    c.cR1 = -c.K1 * c.h / 2.0;
    c.cR2 = c.h * kh / 2.0;
    const double L1 = e->h[H_L1], L2 = e->h[H_L2], K1 = e->h[H_K1], K2 = e->h[H_K2];
    const double psi1 = e->h[H_PSI1], psi2 = e->h[H_PSI2];
    s.px = fma(s.x, psi1, s.px);
    s.py = fma(-s.y, psi1, s.py);
    if (rad == 0) {
        const double inv = rcp(1.0 + s.d);
        const HxCoef k1 = hx_coef(L1, c.h, inv), k2 = hx_coef(L2, c.h, inv);
        for (int m = 0; m < ns; m++) {
            double re, im;
            hxdrift(s, c.h, k1);
            horner_b<M>(s, B, re, im); bend_kick_core<PURE, (M == 0) && PURE>(s, c, re, im, K1);
            hxdrift(s, c.h, k2);
            horner_b<M>(s, B, re, im); bend_kick_core<PURE, (M == 0) && PURE>(s, c, re, im, K2);
            hxdrift(s, c.h, k2);
            horner_b<M>(s, B, re, im); bend_kick_core<PURE, (M == 0) && PURE>(s, c, re, im, K1);
            hxdrift(s, c.h, k1);
        }
    } else if (rad == 1) {
        const double crad = e->h[H_CRAD];
        const double cK1 = crad * K1, cK2 = crad * K2;
        const HxConst k1 = hx_const(L1, c.h), k2 = hx_const(L2, c.h);
        double inv = rcp(1.0 + s.d);
        for (int m = 0; m < ns; m++) {
            hxdrift_inv(s, c.h, k1, inv);
            inv = bend_kick_rad<M, 1, PURE>(s, B, c, K1, cK1, 0.0, inv, 0.0);
            hxdrift_inv(s, c.h, k2, inv);
            inv = bend_kick_rad<M, 1, PURE>(s, B, c, K2, cK2, 0.0, inv, 0.0);
            hxdrift_inv(s, c.h, k2, inv);
            inv = bend_kick_rad<M, 1, PURE>(s, B, c, K1, cK1, 0.0, inv, 0.0);
            hxdrift_inv(s, c.h, k1, inv);
        }
    } else {
        const double crad = e->h[H_CRAD], qec = e->v[V_QECOEF], SL = e->v[V_SL];
        const HxConst kh = hx_const(0.5 * SL, c.h);
        const double cSL = crad * SL;
        double inv = rcp(1.0 + s.d);
        for (int m = 0; m < ns; m++) {
            hxdrift_inv(s, c.h, kh, inv);
            double g = qe_normal(seed, pid, turn, (uint32_t)e->elem, (uint32_t)m);
            inv = bend_kick_rad<M, 2, PURE>(s, B, c, SL, cSL, qec, inv, g);
            hxdrift_inv(s, c.h, kh, inv);
        }
    }
    s.px = fma(s.x, psi2, s.px);
    s.py = fma(-s.y, psi2, s.py);
}

__device__ __forceinline__ void bendmpole_dispatch(St& s, const DevElem* __restrict__ e,
                                                   uint64_t seed, uint32_t pid, uint32_t turn) {
    // h carries B[0..3]: orders above kHotOrder go out of line
    const bool pure = e->h[H_BK1] == 0.0 && e->h[H_BK2] == 0.0;
    switch (e->order_eff * 2 + (pure ? 1 : 0)) {
    case 0: bendmpole<0, false>(s, e, seed, pid, turn); break;
    case 1: bendmpole<0, true>(s, e, seed, pid, turn); break;
    case 2: bendmpole<1, false>(s, e, seed, pid, turn); break;
    case 3: bendmpole<1, true>(s, e, seed, pid, turn); break;
    case 4: bendmpole<2, false>(s, e, seed, pid, turn); break;
    case 5: bendmpole<2, true>(s, e, seed, pid, turn); break;
    case 6: bendmpole<3, false>(s, e, seed, pid, turn); break;
    case 7: bendmpole<3, true>(s, e, seed, pid, turn); break;
    default: s = rare_elem(s, e, seed, pid, turn); break;
    }
}

// ---- other elements ------------------------------------------------------------------------
__device__ __forceinline__ void drift_elem(St& s, double len) {
    double inv = rcp(1.0 + s.d);
    double nl = len * inv;
    drift(s, nl, nl * 0.5 * inv);
}

__device__ __forceinline__ void cavity(St& s, const DevElem* __restrict__ e) {
    const double len = e->h[H_LEN];
    if (len != 0) drift_elem(s, 0.5 * len);
    if (e->flags) s.d = fma(e->h[H_NV], sin(fma(e->h[H_KZ], s.z, e->h[H_PHIS])), s.d);
    if (len != 0) drift_elem(s, 0.5 * len);
}

__device__ __forceinline__ bool aperture_hit(St& s, const DevElem* __restrict__ e) {
    const double a = e->h[H_XMIN], b = e->h[H_XMAX], c = e->h[H_YMIN], d = e->h[H_YMAX];
    if (s.x <= a || s.x >= b || s.y <= c || s.y >= d) {
        s.z = (double)((s.x <= a) * 1 + (s.x >= b) * 2 + (s.y <= c) * 3 + (s.y >= d) * 4);
        s.x = __longlong_as_double(0x7ff8000000000000ll);
        return true;
    }
    return false;
}

__device__ __forceinline__ void aperture(St& s, const DevElem* __restrict__ e) {
    if (aperture_hit(s, e)) return;
    if (e->h[H_LEN] != 0) {
        drift_elem(s, e->h[H_LEN]);
        aperture_hit(s, e);
    }
}

}  // namespace fast
}  // namespace accel
