// adjoint.cuh — reverse-mode (vector-Jacobian) passes of the element maps.
//
// Each function takes an element's INPUT state r (6 doubles, from the tape) and the adjoint of its
// OUTPUT, lam, and overwrites lam with the adjoint of the input, accumulating parameter
// gradients.  The primal arithmetic inside is the literal map's (elem_literal.cuh), with the
// multipole Horner sums started at the highest non-zero coefficient, which for finite inputs is
// bit-identical to starting at index 9.
//
// Hand-derived VJPs:
//   fastdrift  x1 = x + N px, y1 = y + N py, z1 = z - N (px^2 + py^2) / (2 D), D = 1 + delta,
//              N = L / D (the caller's NormL):
//              lam_px += lam_x1 N - lam_z1 N px / D,  lam_py += lam_y1 N - lam_z1 N py / D,
//              lam_d  += -(lam_x1 px + lam_y1 py) N / D + lam_z1 N (px^2 + py^2) / D^2
//   strthinkick  px1 = px - K Re P(z), py1 = py + K Im P(z), P = sum (B_n + i A_n) z^n:
//              lam_x += K (-lam_px1 Re P' + lam_py1 Im P'),  lam_y += K (lam_px1 Im P' + lam_py1 Re P')
//              dL/dB_n += K (-lam_px1 Re z^n + lam_py1 Im z^n),  dL/dA_n += K (lam_px1 Im z^n + lam_py1 Re z^n)
// Other elements: the element's 6x6 (or 6x7 with Quad K) Jacobian from the Dual literal map,
// then lam_in = J^T lam_out.
#pragma once
#include "dual.cuh"
#include "elem_literal.cuh"
#include "engine.h"
#include "adjoint_params.h"

namespace accel {
namespace adj {

constexpr int kMaxSlicesTaped = 32;

struct ElemParams {
    int n;                          // parameters of this element (<= kMaxParamsPerElem)
    int kind[kMaxParamsPerElem];
    int index[kMaxParamsPerElem];
    double acc[kMaxParamsPerElem];  // this particle's dL/dp for the current element pass
};

// ---- forward (literal, effective order) ---------------------------------------------------------
__device__ __forceinline__ void fwd_drift(double* r, double N) { lit::fastdrift(r, N); }

__device__ __forceinline__ void fwd_kick(double* r, const double* A, const double* B, double K, int M) {
    lit::strthinkick(r, A, B, K, M);
}

// One element forward with the literal maps at the effective Horner order (exactly the plain
// kernel's result for finite inputs).
__device__ __forceinline__ void forward(const DevElem& e, double* r) {
    if (lit::is_lost(r[0])) return;
    if (e.op == OP_STRMPOLE || e.op == OP_STRKICK) {
        double A[ACCEL_MAX_MPOLE], B[ACCEL_MAX_MPOLE];
#pragma unroll
        for (int i = 0; i < ACCEL_MAX_MPOLE; i++) { A[i] = e.v[V_A + i]; B[i] = e.v[V_B + i]; }
        const int M = e.order_eff;
        if (e.op == OP_STRKICK) { fwd_kick(r, A, B, 1.0, M); return; }
        const double L1 = e.v[V_L1], L2 = e.v[V_L2], K1 = e.v[V_K1], K2 = e.v[V_K2];
        for (int m = 0; m < e.nslice; m++) {
            double norm = 1 / (1 + r[5]);
            double N1 = L1 * norm, N2 = L2 * norm;
            fwd_drift(r, N1);
            fwd_kick(r, A, B, K1, M);
            fwd_drift(r, N2);
            fwd_kick(r, A, B, K2, M);
            fwd_drift(r, N2);
            fwd_kick(r, A, B, K1, M);
            fwd_drift(r, N1);
        }
        return;
    }
    lit::QeSource q{0, 0, 0, 0, 0};
    lit::pass<double>(e, r, q);
}

// The same forward map on any number type (Dual<6> for the block Jacobians of the tape).
template <class T>
__device__ __forceinline__ void forward_t(const DevElem& e, T* r) {
    if (lit::is_lost(r[0])) return;
    if (e.op == OP_STRMPOLE || e.op == OP_STRKICK) {
        double A[ACCEL_MAX_MPOLE], B[ACCEL_MAX_MPOLE];
#pragma unroll
        for (int i = 0; i < ACCEL_MAX_MPOLE; i++) { A[i] = e.v[V_A + i]; B[i] = e.v[V_B + i]; }
        const int M = e.order_eff;
        if (e.op == OP_STRKICK) { lit::strthinkick(r, A, B, 1.0, M); return; }
        const double L1 = e.v[V_L1], L2 = e.v[V_L2], K1 = e.v[V_K1], K2 = e.v[V_K2];
        // delta does not change inside the element: the slices' NormL are the same every time
        const T norm = 1 / (1 + r[5]);
        const T N1 = L1 * norm, N2 = L2 * norm;
        for (int m = 0; m < e.nslice; m++) {
            lit::fastdrift(r, N1);
            lit::strthinkick(r, A, B, K1, M);
            lit::fastdrift(r, N2);
            lit::strthinkick(r, A, B, K2, M);
            lit::fastdrift(r, N2);
            lit::strthinkick(r, A, B, K1, M);
            lit::fastdrift(r, N1);
        }
        return;
    }
    lit::QeSource q{0, 0, 0, 0, 0};
    lit::pass<T>(e, r, q);
}

// Parameter element on dual numbers with parameter directions: r carries d/d(block input) in
// d[0..5]; directions 6 + j stand for the element's parameters j = 0 .. n-1 (kind/index as in
// ElemParams).  Afterwards r[i].d[k] (k < 6) is the Jacobian of block and element together and
// r[i].d[6 + j] = d out_i / d p_j.  The coefficients stay plain doubles: each kick is taken on
// the dual state, then each parameter's explicit derivative is added to its direction; with
// P = sum (B_n + i A_n) z^n and the kick px -= K Re P, py += K Im P,
//   d px / d B_n = -K Re z^n,  d py / d B_n = K Im z^n,  d px / d A_n = K Im z^n,  d py / d A_n = K Re z^n.
constexpr int kPD = 6 + kMaxParamsPerElem;
__device__ __forceinline__ void forward_params(const DevElem& e, Dual<kPD>* r, int n, const int* kind,
                                               const int* index) {
    if (lit::is_lost(r[0])) return;
    if (e.op == OP_QUAD) {
        Dual<kPD> K(e.v[V_QK]);
        for (int j = 0; j < n; j++)
            if (kind[j] == PK_QUADK) K.d[6 + j] = 1.0;
        lit::quad6(r, e.v[V_LEN], K);
        return;
    }
    double A[ACCEL_MAX_MPOLE], B[ACCEL_MAX_MPOLE];
#pragma unroll
    for (int i = 0; i < ACCEL_MAX_MPOLE; i++) { A[i] = e.v[V_A + i]; B[i] = e.v[V_B + i]; }
    const int M = e.order_eff;
    auto kick = [&](double K) {
        const double x = r[0].v, y = r[2].v;
        lit::strthinkick(r, A, B, K, M);
        for (int j = 0; j < n; j++) {
            double zr = 1.0, zi = 0.0;
            for (int q = 0; q < index[j]; q++) {
                const double t = zr * x - zi * y;
                zi = zr * y + zi * x;
                zr = t;
            }
            if (kind[j] == PK_B) { r[1].d[6 + j] -= K * zr; r[3].d[6 + j] += K * zi; }
            else if (kind[j] == PK_A) { r[1].d[6 + j] += K * zi; r[3].d[6 + j] += K * zr; }
        }
    };
    if (e.op == OP_STRKICK) { kick(1.0); return; }
    const double L1 = e.v[V_L1], L2 = e.v[V_L2], K1 = e.v[V_K1], K2 = e.v[V_K2];
    const Dual<kPD> norm = 1 / (1 + r[5]);  // delta is constant inside the element
    const Dual<kPD> N1 = L1 * norm, N2 = L2 * norm;
    for (int m = 0; m < e.nslice; m++) {
        lit::fastdrift(r, N1);
        kick(K1);
        lit::fastdrift(r, N2);
        kick(K2);
        lit::fastdrift(r, N2);
        kick(K1);
        lit::fastdrift(r, N1);
    }
}

// ---- VJPs ---------------------------------------------------------------------------------------
// r: the drift's input (only px, py, delta are read); N = L/(1+delta) as the forward used it.
__device__ __forceinline__ void vjp_drift(double px, double py, double d, double N, double* lam) {
    const double D = 1 + d;
    const double iD = 1.0 / D;
    const double Q = px * px + py * py;
    const double lx = lam[0], ly = lam[2], lz = lam[4];
    lam[1] += lx * N - lz * N * px * iD;
    lam[3] += ly * N - lz * N * py * iD;
    lam[5] += -(lx * px + ly * py) * N * iD + lz * N * Q * iD * iD;
}

// r: the kick's input (x, y); accumulates parameter gradients of this element into P.
__device__ __forceinline__ void vjp_kick(double x, double y, const double* A, const double* B, double K,
                                         int M, double* lam, ElemParams& P) {
    // P(z) and P'(z) by Horner
    double pr = B[M], pi = A[M], dr = 0.0, di = 0.0;
    for (int i = M - 1; i >= 0; i--) {
        double ndr = dr * x - di * y + pr, ndi = dr * y + di * x + pi;
        double npr = pr * x - pi * y + B[i], npi = pr * y + pi * x + A[i];
        dr = ndr; di = ndi; pr = npr; pi = npi;
    }
    const double lpx = lam[1], lpy = lam[3];
    lam[0] += K * (-lpx * dr + lpy * di);
    lam[2] += K * (lpx * di + lpy * dr);
    for (int j = 0; j < P.n; j++) {
        if (P.kind[j] == PK_QUADK) continue;
        // z^n
        double zr = 1.0, zi = 0.0;
        for (int k = 0; k < P.index[j]; k++) {
            double t = zr * x - zi * y;
            zi = zr * y + zi * x;
            zr = t;
        }
        if (P.kind[j] == PK_B) P.acc[j] += K * (-lpx * zr + lpy * zi);
        else P.acc[j] += K * (lpx * zi + lpy * zr);
    }
}

// StrMPole: recompute slices, then reverse each slice sub-step by sub-step.
__device__ __forceinline__ void vjp_strmpole(const DevElem& e, const double* r_in, double* lam, ElemParams& P) {
    double A[ACCEL_MAX_MPOLE], B[ACCEL_MAX_MPOLE];
#pragma unroll
    for (int i = 0; i < ACCEL_MAX_MPOLE; i++) { A[i] = e.v[V_A + i]; B[i] = e.v[V_B + i]; }
    const int M = e.order_eff;
    if (e.op == OP_STRKICK) {
        vjp_kick(r_in[0], r_in[2], A, B, 1.0, M, lam, P);
        return;
    }
    const double L1 = e.v[V_L1], L2 = e.v[V_L2], K1 = e.v[V_K1], K2 = e.v[V_K2];
    const int ns = e.nslice;
    const double d = r_in[5];  // constant through the element
    const double norm = 1 / (1 + d);
    const double N1 = L1 * norm, N2 = L2 * norm;
    // slice inputs (x, px, y, py); past kMaxSlicesTaped the slice input is recomputed
    double tape[kMaxSlicesTaped][4];
    double r[6];
    for (int k = 0; k < 6; k++) r[k] = r_in[k];
    for (int m = 0; m < ns && m < kMaxSlicesTaped; m++) {
        tape[m][0] = r[0]; tape[m][1] = r[1]; tape[m][2] = r[2]; tape[m][3] = r[3];
        fwd_drift(r, N1); fwd_kick(r, A, B, K1, M); fwd_drift(r, N2); fwd_kick(r, A, B, K2, M);
        fwd_drift(r, N2); fwd_kick(r, A, B, K1, M); fwd_drift(r, N1);
    }
    for (int m = ns - 1; m >= 0; m--) {
        double s[6];
        if (m < kMaxSlicesTaped) {
            s[0] = tape[m][0]; s[1] = tape[m][1]; s[2] = tape[m][2]; s[3] = tape[m][3];
        } else {
            for (int k = 0; k < 6; k++) s[k] = r_in[k];
            for (int q = 0; q < m; q++) {
                fwd_drift(s, N1); fwd_kick(s, A, B, K1, M); fwd_drift(s, N2); fwd_kick(s, A, B, K2, M);
                fwd_drift(s, N2); fwd_kick(s, A, B, K1, M); fwd_drift(s, N1);
            }
        }
        s[4] = 0.0;
        s[5] = d;
        // sub-step inputs within the slice (z is not needed by any VJP)
        double st[7][4];
        st[0][0] = s[0]; st[0][1] = s[1]; st[0][2] = s[2]; st[0][3] = s[3];
        fwd_drift(s, N1);      st[1][0] = s[0]; st[1][1] = s[1]; st[1][2] = s[2]; st[1][3] = s[3];
        fwd_kick(s, A, B, K1, M); st[2][0] = s[0]; st[2][1] = s[1]; st[2][2] = s[2]; st[2][3] = s[3];
        fwd_drift(s, N2);      st[3][0] = s[0]; st[3][1] = s[1]; st[3][2] = s[2]; st[3][3] = s[3];
        fwd_kick(s, A, B, K2, M); st[4][0] = s[0]; st[4][1] = s[1]; st[4][2] = s[2]; st[4][3] = s[3];
        fwd_drift(s, N2);      st[5][0] = s[0]; st[5][1] = s[1]; st[5][2] = s[2]; st[5][3] = s[3];
        fwd_kick(s, A, B, K1, M); st[6][0] = s[0]; st[6][1] = s[1]; st[6][2] = s[2]; st[6][3] = s[3];
        vjp_drift(st[6][1], st[6][3], d, N1, lam);
        vjp_kick(st[5][0], st[5][2], A, B, K1, M, lam, P);
        vjp_drift(st[4][1], st[4][3], d, N2, lam);
        vjp_kick(st[3][0], st[3][2], A, B, K2, M, lam, P);
        vjp_drift(st[2][1], st[2][3], d, N2, lam);
        vjp_kick(st[1][0], st[1][2], A, B, K1, M, lam, P);
        vjp_drift(st[0][1], st[0][3], d, N1, lam);
    }
}

// Any element through its Dual Jacobian: lam <- J^T lam (Quad K as a seventh direction).
__device__ __forceinline__ void vjp_generic(const DevElem& e, const double* r_in, double* lam, ElemParams& P) {
    lit::QeSource q{0, 0, 0, 0, 0};
    int kq = -1;
    for (int j = 0; j < P.n; j++)
        if (P.kind[j] == PK_QUADK) kq = j;
    if (e.op == OP_QUAD && kq >= 0) {
        Dual<7> r[6];
        for (int i = 0; i < 6; i++) { r[i] = Dual<7>(r_in[i]); r[i].d[i] = 1.0; }
        Dual<7> K(e.v[V_QK]);
        K.d[6] = 1.0;
        lit::quad6(r, e.v[V_LEN], K);
        double out[6];
        for (int j = 0; j < 6; j++) {
            double s = 0;
            for (int i = 0; i < 6; i++) s += r[i].d[j] * lam[i];
            out[j] = s;
        }
        double gk = 0;
        for (int i = 0; i < 6; i++) gk += r[i].d[6] * lam[i];
        P.acc[kq] += gk;
        for (int j = 0; j < 6; j++) lam[j] = out[j];
        return;
    }
    Dual<6> r[6];
    for (int i = 0; i < 6; i++) { r[i] = Dual<6>(r_in[i]); r[i].d[i] = 1.0; }
    lit::pass<Dual<6>>(e, r, q);
    double out[6];
    for (int j = 0; j < 6; j++) {
        double s = 0;
        for (int i = 0; i < 6; i++) s += r[i].d[j] * lam[i];
        out[j] = s;
    }
    for (int j = 0; j < 6; j++) lam[j] = out[j];
}

__device__ __forceinline__ void vjp(const DevElem& e, const double* r_in, double* lam, ElemParams& P) {
    switch (e.op) {
    case OP_NOP: return;
    case OP_DRIFT: {
        const double N = e.v[V_LEN] / (1.0 + r_in[5]);
        vjp_drift(r_in[1], r_in[3], r_in[5], N, lam);
        return;
    }
    case OP_STRMPOLE:
    case OP_STRKICK: vjp_strmpole(e, r_in, lam, P); return;
    case OP_APERTURE: {
        // a surviving particle passes unchanged (len 0) or through the drift between the tests
        if (e.v[V_LEN] != 0) {
            const double N = e.v[V_LEN] / (1 + r_in[5]);
            vjp_drift(r_in[1], r_in[3], r_in[5], N, lam);
        }
        return;
    }
    default: vjp_generic(e, r_in, lam, P); return;
    }
}

}  // namespace adj
}  // namespace accel
