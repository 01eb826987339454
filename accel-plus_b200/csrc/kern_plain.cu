// kern_plain.cu — the plain per-element FP64 kernel and the transfer-matrix kernels.
//
// Built with --fmad=false: every product and sum rounds on its own, as on the x86-64 host, and
// the element maps keep the reference's operand order (elem_literal.cuh).  One launch per
// element per turn, one thread per particle, state in HBM (SoA): this is the straightforward GPU
// form of AccelElement::pass, the comparator the fused kernel is measured against.
#include <cuda_runtime.h>
#include <cstdint>
#include "kernels.h"
#include "hdual.cuh"
#include "elem_literal.cuh"

namespace accel {

__global__ void __launch_bounds__(256) k_plain_elem(const TrackParams P, int e,
                                                    const int32_t* __restrict__ turn_ctr) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n = P.ntot;
    if (p >= n) return;
    double* __restrict__ st = P.st;
    double r[6];
    r[0] = st[p];
    if (r[0] != r[0]) return;
    r[1] = st[n + p]; r[2] = st[2 * n + p]; r[3] = st[3 * n + p]; r[4] = st[4 * n + p]; r[5] = st[5 * n + p];
    const int inst = P.pinst ? P.pinst[p] : 0;
    const DevElem& el = P.tables[(P.tbl_off ? P.tbl_off[inst] : 0) + e];
    lit::QeSource q{P.seed, (uint32_t)p, (uint32_t)((P.rng_base ? *P.rng_base : 0) + P.rng_turn0 + *turn_ctr), (uint32_t)el.elem, 0u};
    lit::pass<double>(el, r, q);
    st[p] = r[0]; st[n + p] = r[1]; st[2 * n + p] = r[2];
    st[3 * n + p] = r[3]; st[4 * n + p] = r[4]; st[5 * n + p] = r[5];
}

void launch_plain_elem(const TrackParams& p, int e, const int32_t* turn_ctr, cudaStream_t s) {
    if (p.ntot <= 0) return;
    k_plain_elem<<<(unsigned)((p.ntot + 255) / 256), 256, 0, s>>>(p, e, turn_ctr);
}

// End of a turn: the per-turn NaN scan of trackDA (aline.cpp:646-659), then the turn counter.
__global__ void k_plain_turn_end(const TrackParams P, const int32_t* __restrict__ turn_ctr) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P.ntot) return;
    if (P.loss_turn[p] < 0 && P.st[p] != P.st[p]) P.loss_turn[p] = P.turn0 + *turn_ctr;
}
__global__ void k_inc(int32_t* c) { *c += 1; }

void launch_plain_turn_end(const TrackParams& p, int32_t* turn_ctr, cudaStream_t s) {
    if (p.ntot > 0) k_plain_turn_end<<<(unsigned)((p.ntot + 255) / 256), 256, 0, s>>>(p, turn_ctr);
    k_inc<<<1, 1, 0, s>>>(turn_ctr);
}

// Exact mode: the same literal maps and the same --fmad=false arithmetic as k_plain_elem, so the
// coordinates are bit-identical to the plain kernel's, but one thread carries its particle
// through the elements [e0, e1) of `nturn` turns with the state in registers (no HBM round trip
// and no launch per element).  The QE counters are the plain kernel's (turn = the line's base +
// rng_turn0 + device turn counter, element index).  With record, a particle found lost at the
// end of a turn gets that turn as its loss turn, as k_plain_turn_end records it; without it (a
// range of a turn that a collective element splits) the caller's turn-end kernel does that.
__global__ void __launch_bounds__(128) k_exact(const TrackParams P, int e0, int e1, int nturn,
                                               const int32_t* __restrict__ turn_ctr, int record) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n = P.ntot;
    if (p >= n) return;
    double* __restrict__ st = P.st;
    double r[6];
    r[0] = st[p];
    if (r[0] != r[0]) return;
    r[1] = st[n + p]; r[2] = st[2 * n + p]; r[3] = st[3 * n + p]; r[4] = st[4 * n + p]; r[5] = st[5 * n + p];
    const int inst = P.pinst ? P.pinst[p] : 0;
    const DevElem* __restrict__ T = P.tables + (P.tbl_off ? P.tbl_off[inst] : 0);
    const int t0 = *turn_ctr;
    const uint32_t rbase = (uint32_t)((P.rng_base ? *P.rng_base : 0) + P.rng_turn0);
    for (int t = 0; t < nturn; t++) {
        for (int e = e0; e < e1; e++) {
            lit::QeSource q{P.seed, (uint32_t)p, rbase + (uint32_t)(t0 + t), (uint32_t)T[e].elem, 0u};
            lit::pass<double>(T[e], r, q);
            if (r[0] != r[0]) break;
        }
        if (r[0] != r[0]) {
            if (record && P.loss_turn[p] < 0) P.loss_turn[p] = P.turn0 + t0 + t;
            break;
        }
    }
    st[p] = r[0]; st[n + p] = r[1]; st[2 * n + p] = r[2];
    st[3 * n + p] = r[3]; st[4 * n + p] = r[4]; st[5 * n + p] = r[5];
}
__global__ void k_add(int32_t* c, int v) { *c += v; }

void launch_exact(const TrackParams& p, int e0, int e1, int nturn, int32_t* turn_ctr, bool record,
                  cudaStream_t s) {
    if (p.ntot > 0)
        k_exact<<<(unsigned)((p.ntot + 127) / 128), 128, 0, s>>>(p, e0, e1, nturn, turn_ctr, record ? 1 : 0);
    if (record) k_add<<<1, 1, 0, s>>>(turn_ctr, nturn);
}

// One-turn matrix.  method 0: exact tangent map — the literal maps on Dual<6> seeded with the
// identity; method 1: twelve particles at +/-delta, m_ij = (r+_i - r-_i)/2/delta (aline.cpp:900-927).
__global__ void k_m66_exact(const DevElem* __restrict__ tbl, int e0, int e1, const double* r0, double* m) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Dual<6> r[6];
    for (int i = 0; i < 6; i++) {
        r[i] = Dual<6>(r0[i]);
        r[i].d[i] = 1.0;
    }
    lit::QeSource q{0, 0, 0, 0, 0};
    for (int e = e0; e < e1; e++) lit::pass<Dual<6>>(tbl[e], r, q);
    for (int i = 0; i < 6; i++)
        for (int j = 0; j < 6; j++) m[6 * i + j] = r[i].d[j];
}

__global__ void k_m66_fd(const DevElem* __restrict__ tbl, int e0, int e1, const double* r0,
                         double delta, double* m) {
    __shared__ double rr[12][6];
    const int j = threadIdx.x;
    if (j < 12) {
        double r[6];
        for (int k = 0; k < 6; k++) r[k] = r0[k];
        if (j < 6) r[j] = r0[j] + delta;
        else r[j - 6] = r0[j - 6] - delta;
        lit::QeSource q{0, 0, 0, 0, 0};
        for (int e = e0; e < e1; e++) lit::pass<double>(tbl[e], r, q);
        for (int k = 0; k < 6; k++) rr[j][k] = r[k];
    }
    __syncthreads();
    if (j < 36) {
        int row = j / 6, col = j % 6;
        m[j] = (rr[col][row] - rr[col + 6][row]) / 2.0 / delta;
    }
}

// A knob element on hyper-dual numbers: its coefficient `idx` (kind 1: StrMPole PolynomB, kind 2:
// StrMPole PolynomA, kind 3: Quad K) carries a unit knob derivative; otherwise the literal map of
// lit::pass, slice for slice (accel.cpp:800-847, 824-827, 193-209).
__device__ void pass_knob(const DevElem& e, HDual* r, int kind, int idx) {
    if (lit::is_lost(r[0])) return;
    if (e.op == OP_QUAD) {
        HDual K(e.v[V_QK]);
        K.k = 1.0;
        lit::quad6(r, e.v[V_LEN], K);
        return;
    }
    HDual A[ACCEL_MAX_MPOLE], B[ACCEL_MAX_MPOLE];
    for (int i = 0; i < ACCEL_MAX_MPOLE; i++) { A[i] = HDual(e.v[V_A + i]); B[i] = HDual(e.v[V_B + i]); }
    if (kind == 1) B[idx].k = 1.0;
    else A[idx].k = 1.0;
    if (e.op == OP_STRKICK) {
        lit::strthinkick(r, A, B, 1.0, ACCEL_MAX_MPOLE - 1);
        return;
    }
    const double L1 = e.v[V_L1], L2 = e.v[V_L2], K1 = e.v[V_K1], K2 = e.v[V_K2];
    for (int m = 0; m < e.nslice; m++) {
        HDual norm = 1 / (1 + r[5]);
        HDual NormL1 = L1 * norm, NormL2 = L2 * norm;
        lit::fastdrift(r, NormL1);
        lit::strthinkick(r, A, B, K1, ACCEL_MAX_MPOLE - 1);
        lit::fastdrift(r, NormL2);
        lit::strthinkick(r, A, B, K2, ACCEL_MAX_MPOLE - 1);
        lit::fastdrift(r, NormL2);
        lit::strthinkick(r, A, B, K1, ACCEL_MAX_MPOLE - 1);
        lit::fastdrift(r, NormL1);
    }
}

// Transfer matrix of [e0, e1) about r0 and its exact derivative with respect to one knob that
// moves every coefficient knob[] names by the same amount: the literal maps on hyper-dual numbers
// (hdual.cuh), m_ij = r_i.d[j], dm_ij = r_i.m[j].  knob[e] for element e: 0 when the knob does
// not move it, else kind * 16 + coefficient index.
__global__ void k_m66_knob(const DevElem* __restrict__ tbl, int e0, int e1, const double* r0,
                           const int32_t* __restrict__ knob, double* m, double* dm) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    HDual r[6];
    for (int i = 0; i < 6; i++) {
        r[i] = HDual(r0[i]);
        r[i].d[i] = 1.0;
    }
    lit::QeSource q{0, 0, 0, 0, 0};
    for (int e = e0; e < e1; e++) {
        const int kc = knob[e];
        if (kc == 0) lit::pass<HDual>(tbl[e], r, q);
        else pass_knob(tbl[e], r, kc >> 4, kc & 15);
    }
    for (int i = 0; i < 6; i++)
        for (int j = 0; j < 6; j++) {
            m[6 * i + j] = r[i].d[j];
            dm[6 * i + j] = r[i].m[j];
        }
}

void launch_m66_knob(const DevElem* tbl, int e0, int e1, const double* r0_dev, const int32_t* knob_dev,
                     double* m_dev, double* dm_dev, cudaStream_t s) {
    k_m66_knob<<<1, 32, 0, s>>>(tbl, e0, e1, r0_dev, knob_dev, m_dev, dm_dev);
}

void launch_m66(const DevElem* tbl, int e0, int e1, const double* r0_dev, double delta, int method,
                double* m_dev, cudaStream_t s) {
    if (method == 0) k_m66_exact<<<1, 32, 0, s>>>(tbl, e0, e1, r0_dev, m_dev);
    else k_m66_fd<<<1, 64, 0, s>>>(tbl, e0, e1, r0_dev, delta, m_dev);
}

}  // namespace accel
