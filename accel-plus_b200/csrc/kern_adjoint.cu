// kern_adjoint.cu — forward-with-checkpoints and reverse-turn kernels of the adjoint pair.
//
// The forward runs and the recomputation of turn-start states use the register-resident element
// maps of the fused tracker (elem_fast.cuh), with the literal map for everything they do not
// specialise; the tapes are taken with dual numbers on the literal maps.
//
// One thread per particle in the forward and sweep kernels (particles are independent; only
// parameter gradients are summed over them).  State, adjoint and tapes are SoA in HBM:
//   st[6][n]             state being advanced
//   lam[6][n]            adjoint dL/d(state)
//   ckpt[nseg][6][n]     state at the first turn of every checkpoint segment
//   turn_tape[K][6][n]   turn-start states of the segment being reversed (recomputed)
//   tape[ne][6][n]       element-input states of the turn being reversed (recomputed)
// Parameter gradients: each warp shuffles its lanes' contributions to lane 0, which adds them to
// its own row of a shared-memory table; each block then folds its rows in a fixed order into its
// own row of pacc[nblocks][nparam]; k_adj_reduce sums the rows in order.  No atomics, so the
// result is deterministic.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include "adjoint.cuh"
#include "elem_fast.cuh"
#include "jacobian.cuh"
#include "kernels.h"

namespace accel {

namespace {
// Elements the fast maps do not specialise take the literal map, out of line, state by value.
__device__ __noinline__ fast::St literal_elem(fast::St s, const DevElem* __restrict__ e) {
    double r[6] = {s.x, s.px, s.y, s.py, s.z, s.d};
    adj::forward(*e, r);
    return fast::St{r[0], r[1], r[2], r[3], r[4], r[5]};
}

// One element on the fast maps of the fused tracker (an adjoint's line has no radiation).
__device__ __forceinline__ void fast_elem(fast::St& s, const DevElem* __restrict__ e) {
    switch (e->op) {
    case OP_NOP: return;
    case OP_DRIFT: fast::drift_elem(s, e->h[H_LEN]); return;
    case OP_CAVITY: fast::cavity(s, e); return;
    case OP_APERTURE: fast::aperture(s, e); return;
    case OP_STRMPOLE: {
        const int sk = (e->flags & STR_SKEW) ? ((e->flags & STR_SKEW0) ? 1 : 2) : 0;
        switch (e->order_eff * 4 + sk) {
        case 0: fast::strmpole<0, 0>(s, e); return;
        case 1: fast::strmpole<0, 1>(s, e); return;
        case 2: fast::strmpole<0, 2>(s, e); return;
        case 4: fast::strmpole<1, 0>(s, e); return;
        case 5: fast::strmpole<1, 1>(s, e); return;
        case 6: fast::strmpole<1, 2>(s, e); return;
        case 8: fast::strmpole<2, 0>(s, e); return;
        case 9: fast::strmpole<2, 1>(s, e); return;
        case 10: fast::strmpole<2, 2>(s, e); return;
        case 12: fast::strmpole<3, 0>(s, e); return;
        case 13: fast::strmpole<3, 1>(s, e); return;
        case 14: fast::strmpole<3, 2>(s, e); return;
        default: break;
        }
        break;
    }
    case OP_BENDMPOLE: {
        if (e->flags != 0) break;
        const bool pure = e->h[H_BK1] == 0.0 && e->h[H_BK2] == 0.0;
        switch (e->order_eff * 2 + (pure ? 1 : 0)) {
        case 0: fast::bendmpole<0, false>(s, e, 0, 0, 0); return;
        case 1: fast::bendmpole<0, true>(s, e, 0, 0, 0); return;
        case 2: fast::bendmpole<1, false>(s, e, 0, 0, 0); return;
        case 3: fast::bendmpole<1, true>(s, e, 0, 0, 0); return;
        case 4: fast::bendmpole<2, false>(s, e, 0, 0, 0); return;
        case 5: fast::bendmpole<2, true>(s, e, 0, 0, 0); return;
        case 6: fast::bendmpole<3, false>(s, e, 0, 0, 0); return;
        case 7: fast::bendmpole<3, true>(s, e, 0, 0, 0); return;
        default: break;
        }
        break;
    }
    default: break;
    }
    s = literal_elem(s, e);
}

__device__ __forceinline__ void fast_turn(const AdjParams& a, double* r) {
    fast::St s{r[0], r[1], r[2], r[3], r[4], r[5]};
    for (int e = 0; e < a.ne; e++) {
        fast_elem(s, a.tbl + e);
        if (s.x != s.x) break;
    }
    r[0] = s.x; r[1] = s.px; r[2] = s.y; r[3] = s.py; r[4] = s.z; r[5] = s.d;
}
}  // namespace

namespace {
constexpr unsigned FULL = 0xffffffffu;
constexpr int kAdjThreads = 64;
constexpr int kTile = 32;  // particles per tile of the tape layouts (one warp of the sweep)
constexpr unsigned kSmSlots = kAdjSmSlots;
}  // namespace

int adj_blocks(int64_t n) { return (int)((n + kAdjThreads - 1) / kAdjThreads); }

__device__ __forceinline__ void load6(const double* s, int64_t n, int64_t p, double* r) {
#pragma unroll
    for (int k = 0; k < 6; k++) r[k] = s[k * n + p];
}
__device__ __forceinline__ void store6(double* s, int64_t n, int64_t p, const double* r) {
#pragma unroll
    for (int k = 0; k < 6; k++) s[k * n + p] = r[k];
}

// Forward: nturn turns from st, checkpoint every `every` turns; st ends at the final state.  With
// turn_tape (the run's turn starts fit the tape budget) every turn's starting state is kept too,
// so the reverse pass needs no recomputation; the states are the ones recomputing would give.
// Turns [t0, t0 + nturn) of the run: a long run may be issued as several launches in a row (st
// carries the state from one to the next), checkpoints and turn starts indexed by the run's turn.
// sm_fwd (may be null): per SM, the number of forward blocks running on it; each block counts
// itself in on entry and out when all its threads are done, so that the tape kernel running
// beside the forward can leave those SMs to it (k_adj_jtape's work loop).
__device__ __forceinline__ unsigned sm_id() {
    unsigned id;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(id));
    return id;
}

template <int BS>
__global__ void __launch_bounds__(BS) k_adj_fwd(const AdjParams a, double* ckpt, int t0, int nturn, int every,
                                                double* turn_tape, int* sm_fwd) {
    const unsigned sm = sm_id();
    if (sm_fwd && threadIdx.x == 0 && sm < kSmSlots) atomicAdd(sm_fwd + sm, 1);
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < a.n) {
        double r[6];
        load6(a.st, a.n, p, r);
        for (int t = t0; t < t0 + nturn; t++) {
            if (t % every == 0) store6(ckpt + (int64_t)(t / every) * 6 * a.n, a.n, p, r);
            if (turn_tape) store6(turn_tape + (int64_t)t * 6 * a.n, a.n, p, r);
            if (!(r[0] != r[0])) fast_turn(a, r);
        }
        store6(a.st, a.n, p, r);
    }
    if (sm_fwd) {
        __syncthreads();
        if (threadIdx.x == 0 && sm < kSmSlots) atomicSub(sm_fwd + sm, 1);
    }
}

// Recompute checkpoint segments seg0 .. seg0+nseg-1 at once, (segment, particle) per thread,
// storing the starting state of each of their turns at turn_tape[turn - tape_t0].  The segments
// are independent given their checkpoints, so recomputing all of them in one launch (when their
// turn starts fit in memory) is nseg times wider than one segment before its reversal.
__global__ void __launch_bounds__(kAdjThreads) k_adj_recompute(const AdjParams a, const double* ckpt,
                                                               double* turn_tape, int nturn, int every, int seg0,
                                                               int nseg, int tape_t0) {
    const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (int64_t)nseg * a.n) return;
    const int seg = seg0 + (int)(gid / a.n);
    const int64_t p = gid - (int64_t)(seg - seg0) * a.n;
    const int t0 = seg * every, nt = min(every, nturn - t0);
    double r[6];
    load6(ckpt + (int64_t)seg * 6 * a.n, a.n, p, r);
    for (int j = 0; j < nt; j++) {
        store6(turn_tape + (int64_t)(t0 + j - tape_t0) * 6 * a.n, a.n, p, r);
        if (j + 1 < nt && !(r[0] != r[0])) fast_turn(a, r);
    }
}

// Reverse one turn: re-track it from r_start writing each element's input to the tape, then
// apply the elements' VJPs last to first.  final_x: a particle lost by the end carries no
// gradient (its loss term is absent), so its adjoint stays zero and it is skipped.
__global__ void __launch_bounds__(kAdjThreads) k_adj_turn_reverse(const AdjParams a, const double* r_start,
                                                                  const double* final_x) {
    extern __shared__ double rows[];  // [warps][nparam]
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int j = threadIdx.x; j < nwarps * a.nparam; j += blockDim.x) rows[j] = 0.0;
    __syncthreads();
    const bool have = p < a.n;
    const bool alive = have && !(final_x[p] != final_x[p]);
    double lam[6] = {0, 0, 0, 0, 0, 0};
    if (alive) {
        double r[6];
        load6(r_start, a.n, p, r);
        for (int e = 0; e < a.ne; e++) {
            store6(a.tape + (int64_t)e * 6 * a.n, a.n, p, r);
            adj::forward(a.tbl[e], r);
        }
        load6(a.lam, a.n, p, lam);
    }
    for (int e = a.ne - 1; e >= 0; e--) {
        adj::ElemParams P;
        P.n = a.pcount[e];
        const int f = a.pfirst[e];
        for (int j = 0; j < P.n; j++) {
            P.kind[j] = a.pkind[f + j];
            P.index[j] = a.pindex[f + j];
            P.acc[j] = 0.0;
        }
        if (alive) {
            double r_in[6];
            load6(a.tape + (int64_t)e * 6 * a.n, a.n, p, r_in);
            adj::vjp(a.tbl[e], r_in, lam, P);
        }
        for (int j = 0; j < P.n; j++) {  // P.n is the same for every lane (one lattice)
            double v = P.acc[j];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
            if (lane == 0) rows[warp * a.nparam + f + j] += v;
        }
    }
    if (alive) store6(a.lam, a.n, p, lam);
    __syncthreads();
    for (int j = threadIdx.x; j < a.nparam; j += blockDim.x) {
        double s = 0;
        for (int w = 0; w < nwarps; w++) s += rows[w * a.nparam + j];
        a.pgrad_part[(int64_t)blockIdx.x * a.nparam + j] += s;
    }
}

// ---- block-Jacobian tape -------------------------------------------------------------------------
// Elements the explicit-Jacobian maps do not cover take the literal map on dual numbers whose
// directions are the current Jacobian's rows (J <- J_elem J), out of line, by value.
__device__ __noinline__ jac::JS<6> dual_elem(jac::JS<6> j, const DevElem* __restrict__ e) {
    Dual<6> r[6];
#pragma unroll
    for (int i = 0; i < 6; i++) {
        r[i] = Dual<6>(j.s[i]);
#pragma unroll
        for (int k = 0; k < 6; k++) r[i].d[k] = j.m[6 * i + k];
    }
    adj::forward_t(*e, r);
#pragma unroll
    for (int i = 0; i < 6; i++) {
        j.s[i] = r[i].v;
#pragma unroll
        for (int k = 0; k < 6; k++) j.m[6 * i + k] = r[i].d[k];
    }
    return j;
}

// GENERAL = false: the line holds only the element kinds below and every parameter element is a
// multipole with one B or A coefficient (the host checks, jtape_needs_general), so no call is
// made and the kernel keeps the small register budget of the explicit maps.  ZD = false: the
// unit has no element that reads z or changes delta (unit_zd, set by the host), so the cavity
// case cannot occur in it.
template <bool GENERAL, bool ZD, bool ZR>
__device__ __forceinline__ void jac_elem(jac::JS<6, ZD, ZR>& j, const DevElem* __restrict__ e) {
    if (jac::lost(j.s)) return;
    switch (e->op) {
    case OP_NOP: return;
    case OP_DRIFT: jac::drift_len(j, e->v[V_LEN]); return;
    case OP_STRMPOLE:
    case OP_STRKICK: jac::strmpole(j, *e, -1, 0); return;
    case OP_BENDMPOLE:
        if (e->flags) break;  // radiation (refused by the adjoint; kept general here)
        jac::bendmpole(j, *e);
        return;
    case OP_CAVITY:
        if constexpr (ZD) jac::cavity(j, *e);
        return;
    case OP_APERTURE:
        if (jac::aperture_hit(j.s, *e)) return;
        if (e->v[V_LEN] != 0) {
            jac::drift_len(j, e->v[V_LEN]);
            jac::aperture_hit(j.s, *e);
        }
        return;
    default: break;
    }
    if constexpr (GENERAL && ZD) j = dual_elem(j, e);
}

// A parameter element outside the explicit path (several parameters, Quad K, ...): dual numbers
// with parameter directions (adj::forward_params); writes the unit Jacobian and the parameter
// sensitivities and returns the state.
__device__ __noinline__ fast::St param_elem_dual(jac::JS<6> j, const DevElem* __restrict__ e, int np,
                                                 const int32_t* __restrict__ kinds,
                                                 const int32_t* __restrict__ indices, double* __restrict__ J,
                                                 double* __restrict__ S, int64_t estride, int64_t pstride) {
    int kind[adj::kMaxParamsPerElem], index[adj::kMaxParamsPerElem];
    for (int q = 0; q < np; q++) { kind[q] = kinds[q]; index[q] = indices[q]; }
    Dual<adj::kPD> q[6];
#pragma unroll
    for (int i = 0; i < 6; i++) {
        q[i] = Dual<adj::kPD>(j.s[i]);
#pragma unroll
        for (int k = 0; k < 6; k++) q[i].d[k] = j.m[6 * i + k];
    }
    adj::forward_params(*e, q, np, kind, index);
#pragma unroll
    for (int i = 0; i < 6; i++)
#pragma unroll
        for (int k = 0; k < 6; k++) J[(6 * i + k) * estride] = q[i].d[k];
    for (int p = 0; p < np; p++)
#pragma unroll
        for (int i = 0; i < 6; i++) S[p * pstride + i * estride] = q[i].d[6 + p];
    return fast::St{q[0].v, q[1].v, q[2].v, q[3].v, q[4].v, q[5].v};
}

// The elements of a turn are cut after each parameter element (one carrying parameters whose
// gradient is returned): unit c = the plain elements before parameter element c, then element c
// itself (c = 0 .. npe-1), and a last unit of the plain elements after the last one.  For a chunk
// of nt turns of the current segment (turn-start states in turn_tape, turns j0 .. j0+nt-1), one
// thread per (turn, particle) re-tracks its turn carrying the Jacobian explicitly
// (jacobian.cuh), restarted at every unit, and stores, with t = turn - j0, particle p in tile
// b = p / 32 at lane l = p % 32 and ntile = ceil(n / 32) (one unit of one tile is contiguous, so
// the sweep streams it into shared memory as a block):
//   jt[(((t * (npe + 1) + c) * ntile + b) * 36 + 6 * i + k) * 32 + l] = d out_i / d in_k of unit c,
//   st[(((t * nparam + q) * ntile + b) * 6 + i) * 32 + l]             = d out_i / d p_q at the
//                                                 output of the unit whose element carries q.
// Every turn of the chunk is independent, so this runs nt x n threads wide; the sequential part
// of the reverse sweep (k_adj_jsweep) is left with 6x6 products and dot products.  A particle lost
// by the end of the forward run carries no adjoint and is skipped.
// One unit: the plain elements [e0, e1), then parameter element pe (or none, pe < 0); stores the
// unit's Jacobian at J and the parameter sensitivities at S (tiled, stride kTile per entry and
// pstride per parameter) and advances the state s.
template <bool GENERAL, bool ZD, bool ZR>
__device__ __forceinline__ void jtape_unit(const AdjParams& a, double* s, int e0, int e1, int pe,
                                           double* __restrict__ J, double* __restrict__ S, int64_t pstride) {
    jac::JS<6, ZD, ZR> j;
#pragma unroll
    for (int i = 0; i < 6; i++) j.s[i] = s[i];
    jac::set_identity(j);
    for (int e = e0; e < e1; e++) jac_elem<GENERAL, ZD, ZR>(j, a.tbl + e);
    if (pe >= 0) {
        const DevElem* el = a.tbl + pe;
        const int np = a.pcount[pe], f = a.pfirst[pe], kind = a.pkind[f];
        if (np == 1 && (el->op == OP_STRMPOLE || el->op == OP_STRKICK) && (kind == adj::PK_B || kind == adj::PK_A) &&
            !jac::lost(j.s)) {
            jac::JS<7, ZD, ZR> q;
#pragma unroll
            for (int i = 0; i < 6; i++) {
                q.s[i] = j.s[i];
#pragma unroll
                for (int k = 0; k < 6; k++) q.m[7 * i + k] = j.m[6 * i + k];
                q.m[7 * i + 6] = 0.0;
            }
            jac::strmpole(q, *el, kind, a.pindex[f]);
#pragma unroll
            for (int i = 0; i < 6; i++) {
#pragma unroll
                for (int k = 0; k < 6; k++) J[(6 * i + k) * kTile] = q.m[7 * i + k];
                S[i * kTile] = q.m[7 * i + 6];
                s[i] = q.s[i];
            }
            return;
        }
        if constexpr (GENERAL && ZD) {
            const fast::St o = param_elem_dual(j, el, np, a.pkind + f, a.pindex + f, J, S, kTile, pstride);
            s[0] = o.x; s[1] = o.px; s[2] = o.y; s[3] = o.py; s[4] = o.z; s[5] = o.d;
            return;
        }
    }
#pragma unroll
    for (int i = 0; i < 6; i++) {
#pragma unroll
        for (int k = 0; k < 6; k++) J[(6 * i + k) * kTile] = j.m[6 * i + k];
        s[i] = j.s[i];
    }
}

// ZR = false: the z rows of the unit Jacobians are left at e_z (jacobian.cuh), for a line with no
// element that reads z and a reverse sweep whose seed has no z component.
template <bool GENERAL, bool ZR>
__device__ __forceinline__ void jtape_one(const AdjParams& a, const double* turn_tape, int j0, int64_t gid,
                                          const double* final_x, int npe, double* jt, double* sens) {
    const int64_t n = a.n;
    const int t = (int)(gid / n);
    const int64_t p = gid - (int64_t)t * n;
    // a particle lost by the end is skipped when that is known (final_x given); a tape written
    // while the forward still runs covers every particle, and the sweep ignores the lost ones
    if (final_x && final_x[p] != final_x[p]) return;
    const int64_t ntile = (n + kTile - 1) / kTile, b = p / kTile;
    const int l = (int)(p % kTile);
    const double* s0 = turn_tape + (int64_t)(j0 + t) * 6 * n;
    double s[6];
#pragma unroll
    for (int i = 0; i < 6; i++) s[i] = s0[i * n + p];
    const int64_t pstride = ntile * 6 * kTile;
    int e0 = 0;
    for (int c = 0; c <= npe; c++) {
        const int pe = c < npe ? a.pelem[c] : -1;
        const int e1 = c < npe ? pe : a.ne;
        double* J = jt + ((((int64_t)t * (npe + 1) + c) * ntile + b) * 36) * kTile + l;
        double* S = pe >= 0 ? sens + ((((int64_t)t * a.nparam + a.pfirst[pe]) * ntile + b) * 6) * kTile + l : nullptr;
        if constexpr (GENERAL) {
            jtape_unit<true, true, true>(a, s, e0, e1, pe, J, S, pstride);
        } else {
            if (a.unit_zd[c]) jtape_unit<false, true, true>(a, s, e0, e1, pe, J, S, pstride);
            else jtape_unit<false, false, ZR>(a, s, e0, e1, pe, J, S, pstride);
        }
        e0 = e1 + 1;
    }
}

// Two ways to cover the n x nt (turn, particle) units, one per thread:
//   work == null: one unit per thread of the grid;
//   work != null: a grid sized to the resident blocks takes groups of 128 units from the counter
//     *work (zeroed before the launch) until none is left.  While the forward runs beside it,
//     a block whose SM holds a forward block (sm_fwd, see k_adj_fwd) takes no more work and
//     leaves, so the latency-bound forward keeps its SMs to itself; block 0 never leaves, so
//     every unit is taped whatever the placement.  Each pass of the loop takes one group or
//     leaves, and the counter only grows, so the loop ends.
template <bool GENERAL, bool ZR>
__global__ void __launch_bounds__(128, GENERAL ? 1 : 3) k_adj_jtape(const AdjParams a, const double* turn_tape, int j0,
                                                                    int nt, const double* final_x, int npe, double* jt,
                                                                    double* sens, int* work, const int* sm_fwd) {
    const int64_t units = a.n * (int64_t)nt;
    if (!work) {
        const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (gid < units) jtape_one<GENERAL, ZR>(a, turn_tape, j0, gid, final_x, npe, jt, sens);
        return;
    }
    const int64_t groups = (units + 127) / 128;
    const unsigned sm = sm_id();
    __shared__ int64_t s_group;
    for (;;) {
        if (threadIdx.x == 0) {
            const bool yield = sm_fwd && blockIdx.x != 0 && sm < kSmSlots &&
                               *(volatile const int*)(sm_fwd + sm) > 0;
            s_group = yield ? -1 : (int64_t)atomicAdd(work, 1);
        }
        __syncthreads();
        const int64_t g = s_group;
        __syncthreads();
        if (g < 0 || g >= groups) return;
        const int64_t gid = g * 128 + threadIdx.x;
        if (gid < units) jtape_one<GENERAL, ZR>(a, turn_tape, j0, gid, final_x, npe, jt, sens);
    }
}

// Reverse sweep over the chunk's turns, last to first: at each unit's output the parameter
// gradients take sens^T lam, then lam <- J^T lam.  pelem lists the parameter elements in line
// order.  One warp per tile of 32 particles, one particle per lane.  The sweep is a dependent
// chain per particle and the tile count is small (n / 32), so the unit tiles are streamed into
// shared memory kSweepStages units ahead with asynchronous copies (cp.async, waited on with
// cp.async.wait_group: no spin loop) and each step reads its operands from shared memory.
// Gradients: each lane adds into its own slot rows[q * 32 + lane] (shared memory, or global
// memory past kSweepSmemParams parameters), summed over the lanes in order at the end.
constexpr int kSweepStages = 6;
constexpr int kSweepSmemParams = 384;
constexpr int kStageDoubles = (36 + 6 * adj::kMaxParamsPerElem) * kTile;

__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__global__ void __launch_bounds__(kTile) k_adj_jsweep(const AdjParams a, int nt, const double* final_x, int npe,
                                                      const int32_t* pelem, const double* jt, const double* sens,
                                                      double* grow) {
    extern __shared__ __align__(16) double smem[];
    double* stage = smem;                                    // [kSweepStages][kStageDoubles]
    const bool srows = a.nparam <= kSweepSmemParams;
    double* rows = srows ? smem + kSweepStages * kStageDoubles  // [nparam][32]
                         : grow + (int64_t)blockIdx.x * a.nparam * kTile;
    const int64_t n = a.n, ntile = (n + kTile - 1) / kTile, b = blockIdx.x;
    const int lane = threadIdx.x;
    const int64_t p = b * kTile + lane;
    for (int q = 0; q < a.nparam; q++) rows[q * kTile + lane] = 0.0;
    const bool alive = p < n && !(final_x[p] != final_x[p]);
    double lam[6] = {0, 0, 0, 0, 0, 0};
    if (alive) load6(a.lam, n, p, lam);
    const int U = nt * (npe + 1);  // units of the chunk; unit u = t * (npe + 1) + c, swept u = U-1 .. 0
    const int64_t jstride = ntile * 36 * kTile;           // doubles between consecutive units' tiles
    const int64_t sstride = ntile * 6 * kTile;            // between consecutive parameters' tiles
    // the copy cursor runs kSweepStages units ahead of the sweep; (t, c) counters, no division
    int it = nt - 1, ic = npe, ist = 0, iu = U - 1;
    auto issue = [&]() {
        if (iu >= 0) {
            double* dst = stage + ist * kStageDoubles;
            const double* src = jt + (int64_t)iu * jstride + b * 36 * kTile;
#pragma unroll
            for (int k = 0; k < 36 * kTile / 2 / kTile; k++) cp_async16(dst + 2 * (lane + k * kTile), src + 2 * (lane + k * kTile));
            if (ic < npe) {
                const int e = pelem[ic], np = a.pcount[e], f = a.pfirst[e];
                const double* ss = sens + ((int64_t)it * a.nparam + f) * sstride + b * 6 * kTile;
                for (int j = 0; j < np; j++) {
                    double* sd = dst + (36 + 6 * j) * kTile;
#pragma unroll
                    for (int k = 0; k < 6 * kTile / 2 / kTile; k++)
                        cp_async16(sd + 2 * (lane + k * kTile), ss + j * sstride + 2 * (lane + k * kTile));
                }
            }
            iu--;
            if (--ic < 0) { ic = npe; it--; }
        }
        cp_async_commit();
        if (++ist == kSweepStages) ist = 0;
    };
    for (int i = 0; i < kSweepStages; i++) issue();
    int c = npe, st = 0;
    for (int i = 0; i < U; i++) {
        cp_async_wait<kSweepStages - 1>();
        __syncwarp();
        const double* S = stage + st * kStageDoubles;
        if (c < npe && alive) {
            const int e = pelem[c], np = a.pcount[e], f = a.pfirst[e];
            for (int j = 0; j < np; j++) {
                double v = 0.0;
#pragma unroll
                for (int k = 0; k < 6; k++) v = fma(S[(36 + 6 * j + k) * kTile + lane], lam[k], v);
                rows[(f + j) * kTile + lane] += v;
            }
        }
        if (alive) {
            double out[6];
#pragma unroll
            for (int k = 0; k < 6; k++) {
                double acc = 0.0;
#pragma unroll
                for (int m = 0; m < 6; m++) acc = fma(S[(6 * m + k) * kTile + lane], lam[m], acc);
                out[k] = acc;
            }
#pragma unroll
            for (int k = 0; k < 6; k++) lam[k] = out[k];
        }
        __syncwarp();
        issue();  // into the slot just read (the cursor is kSweepStages units ahead)
        if (--c < 0) c = npe;
        if (++st == kSweepStages) st = 0;
    }
    cp_async_wait<0>();
    if (alive) store6(a.lam, n, p, lam);
    __syncwarp();
    for (int q = lane; q < a.nparam; q += kTile) {
        double sum = 0.0;
        for (int w = 0; w < kTile; w++) sum += rows[q * kTile + w];
        a.pgrad_part[b * a.nparam + q] += sum;
    }
}

// flag = 1 when any of v[0 .. n) is not zero (the flag is zeroed before the launch)
__global__ void k_any_nonzero(const double* __restrict__ v, int64_t n, int* flag) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (v[i] != 0.0) {
            *flag = 1;
            return;
        }
}

void launch_any_nonzero(const double* v, int64_t n, int* flag, cudaStream_t s) {
    cudaMemsetAsync(flag, 0, sizeof(int), s);
    k_any_nonzero<<<(unsigned)std::min<int64_t>(1024, (n + 255) / 256 + 1), 256, 0, s>>>(v, n, flag);
}

__global__ void k_adj_reduce(const double* part, int nblk, int nparam, double* out) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nparam; j += gridDim.x * blockDim.x) {
        double s = 0;
        for (int b = 0; b < nblk; b++) s += part[(int64_t)b * nparam + j];
        out[j] = s;
    }
}

void launch_adj_forward(const AdjParams& a, double* ckpt, int t0, int nturn, int every, double* turn_tape,
                        cudaStream_t s, int threads, int* sm_fwd) {
    const unsigned nb = (unsigned)((a.n + threads - 1) / threads);
    switch (threads) {
    case 128: k_adj_fwd<128><<<nb, 128, 0, s>>>(a, ckpt, t0, nturn, every, turn_tape, sm_fwd); break;
    case 256: k_adj_fwd<256><<<nb, 256, 0, s>>>(a, ckpt, t0, nturn, every, turn_tape, sm_fwd); break;
    default:
        k_adj_fwd<kAdjThreads><<<adj_blocks(a.n), kAdjThreads, 0, s>>>(a, ckpt, t0, nturn, every, turn_tape, sm_fwd);
        break;
    }
}
void launch_adj_recompute(const AdjParams& a, const double* ckpt, double* turn_tape, int nturn, int every,
                          int seg0, int nseg, cudaStream_t s) {
    const int64_t threads = (int64_t)nseg * a.n;
    k_adj_recompute<<<(unsigned)((threads + kAdjThreads - 1) / kAdjThreads), kAdjThreads, 0, s>>>(
        a, ckpt, turn_tape, nturn, every, seg0, nseg, seg0 * every);
}
int adj_part_rows(int64_t n) { return (int)std::max<int64_t>((n + kTile - 1) / kTile, adj_blocks(n)); }
void launch_adj_turn_reverse(const AdjParams& a, const double* r_start, const double* final_x, cudaStream_t s) {
    const size_t sh = sizeof(double) * (kAdjThreads / 32) * (size_t)a.nparam;
    k_adj_turn_reverse<<<adj_blocks(a.n), kAdjThreads, sh, s>>>(a, r_start, final_x);
}
void jtape_unit_zd(const DevElem* t, int ne, const int32_t* pelem, int npe, int32_t* unit_zd) {
    int e0 = 0;
    for (int c = 0; c <= npe; c++) {
        const int e1 = c < npe ? pelem[c] : ne - 1;  // inclusive: the parameter element too
        int zd = 0;
        for (int e = e0; e <= e1 && e < ne; e++) {
            const int op = t[e].op;
            const bool plain = op == OP_NOP || op == OP_DRIFT || op == OP_STRMPOLE || op == OP_STRKICK ||
                               op == OP_APERTURE || (op == OP_BENDMPOLE && t[e].flags == 0);
            if (!plain) zd = 1;
        }
        unit_zd[c] = zd;
        e0 = e1 + 1;
    }
}

bool jtape_needs_general(const DevElem* t, int ne, const int32_t* pcount, const int32_t* pfirst,
                         const int32_t* pkind) {
    for (int e = 0; e < ne; e++) {
        const int op = t[e].op;
        if (pcount[e] == 0) {
            switch (op) {
            case OP_NOP: case OP_DRIFT: case OP_STRMPOLE: case OP_STRKICK: case OP_CAVITY: case OP_APERTURE:
                break;
            case OP_BENDMPOLE:
                if (t[e].flags) return true;
                break;
            default:
                return true;
            }
        } else {
            const int k = pkind[pfirst[e]];
            if (pcount[e] != 1 || !(op == OP_STRMPOLE || op == OP_STRKICK) || !(k == adj::PK_B || k == adj::PK_A))
                return true;
        }
    }
    return false;
}

void launch_adj_jtape(const AdjParams& a, const double* turn_tape, int j0, int nt, const double* final_x,
                      int npe, double* jt, double* sens, bool general, cudaStream_t s, int* work,
                      const int* sm_fwd, int sm_count, bool zrow) {
    const int64_t threads = a.n * (int64_t)nt;
    unsigned grid = (unsigned)((threads + 127) / 128);
    // general lines always carry the z row
    auto kern = general ? k_adj_jtape<true, true> : zrow ? k_adj_jtape<false, true> : k_adj_jtape<false, false>;
    if (work) {
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, 0);
        grid = std::min<unsigned>(grid, (unsigned)std::max(1, per_sm * sm_count));
    }
    kern<<<grid, 128, 0, s>>>(a, turn_tape, j0, nt, final_x, npe, jt, sens, work, sm_fwd);
}
void launch_adj_jsweep(const AdjParams& a, int nt, const double* final_x, int npe, const int32_t* pelem,
                       const double* jt, const double* sens, double* grow, cudaStream_t s) {
    const int64_t ntile = (a.n + kTile - 1) / kTile;
    size_t sh = sizeof(double) * (size_t)kSweepStages * kStageDoubles;
    if (a.nparam <= kSweepSmemParams) sh += sizeof(double) * (size_t)a.nparam * kTile;
    cudaFuncSetAttribute(k_adj_jsweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
    k_adj_jsweep<<<(unsigned)ntile, kTile, sh, s>>>(a, nt, final_x, npe, pelem, jt, sens, grow);
}
void launch_adj_reduce(const double* part, int nblk, int nparam, double* out, cudaStream_t s) {
    if (nparam > 0) k_adj_reduce<<<(nparam + 127) / 128, 128, 0, s>>>(part, nblk, nparam, out);
}

}  // namespace accel
