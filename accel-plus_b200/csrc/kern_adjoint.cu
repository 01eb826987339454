// kern_adjoint.cu — forward-with-checkpoints and reverse-turn kernels of the adjoint pair.
//
// One thread per particle throughout (particles are independent; only parameter gradients are
// summed over them).  State, adjoint and tapes are SoA in HBM:
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
#include <cstdint>
#include "adjoint.cuh"
#include "kernels.h"

namespace accel {

namespace {
constexpr unsigned FULL = 0xffffffffu;
constexpr int kAdjThreads = 64;
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

// Forward: nturn turns from st, checkpoint every `every` turns; st ends at the final state.
__global__ void __launch_bounds__(kAdjThreads) k_adj_fwd(const AdjParams a, double* ckpt, int nturn, int every) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    double r[6];
    load6(a.st, a.n, p, r);
    for (int t = 0; t < nturn; t++) {
        if (t % every == 0) store6(ckpt + (int64_t)(t / every) * 6 * a.n, a.n, p, r);
        for (int e = 0; e < a.ne; e++) adj::forward(a.tbl[e], r);
    }
    store6(a.st, a.n, p, r);
}

// Recompute nt turns from a checkpoint, storing each turn's starting state.
__global__ void __launch_bounds__(kAdjThreads) k_adj_recompute(const AdjParams a, const double* ck,
                                                               double* turn_tape, int nt) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    double r[6];
    load6(ck, a.n, p, r);
    for (int j = 0; j < nt; j++) {
        store6(turn_tape + (int64_t)j * 6 * a.n, a.n, p, r);
        if (j + 1 < nt)
            for (int e = 0; e < a.ne; e++) adj::forward(a.tbl[e], r);
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

__global__ void k_adj_reduce(const double* part, int nblk, int nparam, double* out) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nparam; j += gridDim.x * blockDim.x) {
        double s = 0;
        for (int b = 0; b < nblk; b++) s += part[(int64_t)b * nparam + j];
        out[j] = s;
    }
}

void launch_adj_forward(const AdjParams& a, double* ckpt, int nturn, int every, cudaStream_t s) {
    k_adj_fwd<<<adj_blocks(a.n), kAdjThreads, 0, s>>>(a, ckpt, nturn, every);
}
void launch_adj_recompute(const AdjParams& a, const double* ck, double* turn_tape, int nt, cudaStream_t s) {
    k_adj_recompute<<<adj_blocks(a.n), kAdjThreads, 0, s>>>(a, ck, turn_tape, nt);
}
void launch_adj_turn_reverse(const AdjParams& a, const double* r_start, const double* final_x, cudaStream_t s) {
    const size_t sh = sizeof(double) * (kAdjThreads / 32) * (size_t)a.nparam;
    k_adj_turn_reverse<<<adj_blocks(a.n), kAdjThreads, sh, s>>>(a, r_start, final_x);
}
void launch_adj_reduce(const double* part, int nblk, int nparam, double* out, cudaStream_t s) {
    if (nparam > 0) k_adj_reduce<<<(nparam + 127) / 128, 128, 0, s>>>(part, nblk, nparam, out);
}

}  // namespace accel
