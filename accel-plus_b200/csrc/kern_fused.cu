// kern_fused.cu — the fused persistent FP64 tracker and its support kernels (sm_100a).
//
// Fused kernel design:
//  * one thread per macroparticle; its six coordinates stay in registers for every element of
//    every turn of a segment, so HBM sees 96 B per particle per segment (SoA, coalesced);
//  * persistent warps pull chunks of 32 live particles from an atomic counter, so the grid is
//    sized to the SM count and tail imbalance is one chunk;
//  * element records are read through L1 as warp-wide broadcasts (every lane of a chunk whose
//    particles belong to one lattice instance reads the same record);
//  * a particle is lost when x turns NaN (aperture hit or arithmetic); the warp stops early when
//    __any_sync finds no live lane, and between segments a stable stream compaction
//    (k_compact) drops lost particles from the live list, so later segments run dense warps;
//  * segments, compaction and collective elements are captured into one CUDA graph by the host.
#include <cuda_runtime.h>
#include <cstdint>
#include <cmath>
#include "kernels.h"
#include "elem_fast.cuh"
#include "elem_literal.cuh"

namespace accel {

namespace {
constexpr unsigned FULL = 0xffffffffu;
__device__ __forceinline__ bool nan_(double v) { return v != v; }
__device__ __forceinline__ double qnan() { return __longlong_as_double(0x7ff8000000000000ll); }
}  // namespace

// Rare elements (thin and high-order multipoles, Quad, Bend, Corrector, Matrix, SyncRad) run the
// literal map out of line; the state goes in and out by value.
__device__ __noinline__ fast::St fast::rare_elem(fast::St s, const DevElem* __restrict__ e,
                                                 uint64_t seed, uint32_t pid, uint32_t turn) {
    double r[6] = {s.x, s.px, s.y, s.py, s.z, s.d};
    lit::QeSource q{seed, pid, turn, (uint32_t)e->elem, 0u};
    lit::pass<double>(*e, r, q);
    return fast::St{r[0], r[1], r[2], r[3], r[4], r[5]};
}

__device__ __forceinline__ void fused_elem(fast::St& s, const DevElem* __restrict__ e, uint64_t seed,
                                           uint32_t pid, uint32_t turn) {
    switch (e->op) {
    case OP_NOP: break;
    case OP_DRIFT: fast::drift_elem(s, e->h[H_LEN]); break;
    case OP_STRMPOLE: fast::strmpole_dispatch(s, e); break;
    case OP_STRKICK: s = fast::rare_elem(s, e, seed, pid, turn); break;
    case OP_BENDMPOLE: fast::bendmpole_dispatch(s, e, seed, pid, turn); break;
    case OP_CAVITY: fast::cavity(s, e); break;
    case OP_APERTURE: fast::aperture(s, e); break;
    case OP_TRANSWAKE:
    case OP_LONGWAKE: break;  // collective: the host never puts one inside a fused range
    default: s = fast::rare_elem(s, e, seed, pid, turn); break;
    }
}

template <int BS, int MINB>
__global__ void __launch_bounds__(BS, MINB) k_fused(const TrackParams P) {
    const int lane = threadIdx.x & 31;
    const int nlive = *P.nlive;
    const int64_t n = P.ntot;
    const int tbase = P.turn_dev ? *P.turn_dev : 0;
    const int rbase = (P.rng_base ? *P.rng_base : 0) + tbase;
    double* __restrict__ st = P.st;
    // sched 1: this block owns chunks [c0, c1) of the live list, its warps stride through them
    const int nchunk = (nlive + 31) / 32;
    const int per_block = (nchunk + gridDim.x - 1) / gridDim.x;
    const int c0 = blockIdx.x * per_block, c1 = min(nchunk, c0 + per_block);
    int cnext = c0 + (threadIdx.x >> 5);
    for (;;) {
        int base = 0;
        if (P.sched == 0) {
            if (lane == 0) base = atomicAdd(P.chunk_ctr, 32);
            base = __shfl_sync(FULL, base, 0);
        } else {
            if (cnext >= c1) break;
            base = cnext * 32;
            cnext += BS / 32;
        }
        if (base >= nlive) break;
        const int idx = base + lane;
        const bool have = idx < nlive;
        const int p = have ? P.live[idx] : 0;
        fast::St s;
        if (have) {
            s.x = st[p]; s.px = st[n + p]; s.y = st[2 * n + p];
            s.py = st[3 * n + p]; s.z = st[4 * n + p]; s.d = st[5 * n + p];
        } else {
            s.x = qnan(); s.px = s.y = s.py = s.z = s.d = 0.0;
        }
        const int inst = (have && P.pinst) ? P.pinst[p] : 0;
        const DevElem* __restrict__ T = P.tables + (P.tbl_off ? P.tbl_off[inst] : 0);
        bool alive = have && !nan_(s.x);
        for (int t = 0; t < P.nturn; t++) {
            if (!__any_sync(FULL, alive)) break;
            if (alive) {
                const uint32_t rt = (uint32_t)(rbase + P.rng_turn0 + t);
                for (int e = P.e0; e < P.e1; e++) {
                    // pull the next element's parameter line into L1 while this one computes
                    const DevElem* nx = T + (e + 1 < P.e1 ? e + 1 : P.e0);
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(nx));
                    fused_elem(s, T + e, P.seed, (uint32_t)p, rt);
                    if (nan_(s.x)) break;
                }
                if (nan_(s.x)) {
                    alive = false;
                    P.loss_turn[p] = P.turn0 + tbase + t;
                    if (P.lost_flag) *P.lost_flag = 1;
                }
            }
        }
        if (have) {
            st[p] = s.x; st[n + p] = s.px; st[2 * n + p] = s.y;
            st[3 * n + p] = s.py; st[4 * n + p] = s.z; st[5 * n + p] = s.d;
        }
    }
}

// Variant table: (block, min blocks per SM) pairs the autotuner chooses from; the launch bound
// caps registers per thread at 65536 / (block * min_blocks).
#define FUSED_VARIANTS(X) X(0, 128, 4) X(1, 128, 3) X(2, 256, 2) X(3, 64, 8) X(4, 128, 5) X(5, 128, 2)

VariantInfo fused_variant_info(int v) {
    switch (v) {
#define X(i, b, m) case i: return VariantInfo{b, m};
        FUSED_VARIANTS(X)
#undef X
    default: return VariantInfo{128, 4};
    }
}

int fused_blocks_per_sm(int v) {
    int nb = 0;
    switch (v) {
#define X(i, b, m) case i: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_fused<b, m>, b, 0); break;
        FUSED_VARIANTS(X)
#undef X
    default: break;
    }
    return nb;
}

void launch_fused(const TrackParams& p, int v, int grid, cudaStream_t s) {
    switch (v) {
#define X(i, b, m) case i: k_fused<b, m><<<grid, b, 0, s>>>(p); break;
        FUSED_VARIANTS(X)
#undef X
    default: k_fused<128, 4><<<grid, 128, 0, s>>>(p); break;
    }
}

__global__ void k_rng_advance(int32_t* b, int nturn) { *b += nturn; }
void launch_rng_advance(int32_t* base, int nturn, cudaStream_t s) {
    if (base) k_rng_advance<<<1, 1, 0, s>>>(base, nturn);
}

// ---- stable stream compaction of the live list (one block, blocked tiles) --------------------
// In place is safe: each tile is read into registers before any thread writes, and an item is
// written at or before the index it was read from.  When nothing was lost since the last
// compaction (lost_flag clear) the list is already compact and is left as it is.
__global__ void __launch_bounds__(1024) k_compact(int32_t* live, int32_t* nlive, const double* __restrict__ x,
                                                  int32_t* chunk_ctr, int32_t* turn_ctr, int turns,
                                                  int32_t* lost_flag) {
    constexpr int ITEMS = 8;
    constexpr int TILE = 1024 * ITEMS;
    __shared__ int warp_tot[32];
    __shared__ int s_carry;
    const int32_t* live_in = live;
    int32_t* live_out = live;
    const bool scan = !lost_flag || *lost_flag != 0;
    const int n = scan ? *nlive : 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (int base = 0; base < n; base += TILE) {
        int idx[ITEMS];
        int cnt = 0;
        unsigned keep = 0;
#pragma unroll
        for (int k = 0; k < ITEMS; k++) {
            int i = base + threadIdx.x * ITEMS + k;
            idx[k] = 0;
            if (i < n) {
                idx[k] = live_in[i];
                if (!nan_(x[idx[k]])) { keep |= 1u << k; cnt++; }
            }
        }
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int v = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += v;
        }
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            int w = warp_tot[lane];
            int wi = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int v = __shfl_up_sync(FULL, wi, o);
                if (lane >= o) wi += v;
            }
            warp_tot[lane] = wi - w;  // exclusive prefix of warp totals
            if (lane == 31) warp_tot[lane] = wi - w;
        }
        __syncthreads();
        int off = s_carry + warp_tot[warp] + (incl - cnt);
#pragma unroll
        for (int k = 0; k < ITEMS; k++)
            if (keep & (1u << k)) live_out[off++] = idx[k];
        __syncthreads();
        if (threadIdx.x == 1023) s_carry = off;  // last thread ends at the tile's total
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (scan) {
            *nlive = s_carry;
            if (lost_flag) *lost_flag = 0;
        }
        *chunk_ctr = 0;
        if (turn_ctr) *turn_ctr += turns;
    }
}

void launch_compact(int32_t* live, int32_t* nlive, const double* x, int32_t* chunk_ctr, int32_t* turn_ctr,
                    int turns, int32_t* lost_flag, cudaStream_t s) {
    k_compact<<<1, 1024, 0, s>>>(live, nlive, x, chunk_ctr, turn_ctr, turns, lost_flag);
}

__global__ void k_init_live(const double* __restrict__ x, int64_t n, int32_t* loss_turn,
                            int32_t* live, int32_t* nlive, int32_t* chunk_ctr, int init_loss) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) { *nlive = (int32_t)n; *chunk_ctr = 0; }
    if (i < n) {
        live[i] = (int32_t)i;
        if (init_loss) loss_turn[i] = nan_(x[i]) ? 0 : -1;
    }
}

void launch_init_live(const double* x, int64_t n, int32_t* loss_turn, int32_t* live, int32_t* nlive,
                      int32_t* chunk_ctr, int init_loss, cudaStream_t s) {
    int64_t g = (n + 255) / 256;
    if (g < 1) g = 1;
    k_init_live<<<(unsigned)g, 256, 0, s>>>(x, n, loss_turn, live, nlive, chunk_ctr, init_loss);
}

__global__ void k_aos_to_soa(const double* __restrict__ a, double* __restrict__ s, int64_t n) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 6 * n) s[(i % 6) * n + i / 6] = a[i];
}
__global__ void k_soa_to_aos(const double* __restrict__ s, double* __restrict__ a, int64_t n) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 6 * n) a[i] = s[(i % 6) * n + i / 6];
}
void launch_aos_to_soa(const double* aos, double* soa, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    k_aos_to_soa<<<(unsigned)((6 * n + 255) / 256), 256, 0, s>>>(aos, soa, n);
}
void launch_soa_to_aos(const double* soa, double* aos, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    k_soa_to_aos<<<(unsigned)((6 * n + 255) / 256), 256, 0, s>>>(soa, aos, n);
}

__global__ void k_fill_i32(int32_t* p, int32_t v, int64_t n) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}
__global__ void k_copy_i32(const int32_t* a, int32_t* b, int64_t n) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i];
}
void launch_fill_i32(int32_t* p, int32_t v, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    k_fill_i32<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(p, v, n);
}
void launch_copy_i32(const int32_t* src, int32_t* dst, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    k_copy_i32<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src, dst, n);
}

// ---- longitudinal broadband-resonator wake (no reference counterpart) ------------------------
// Scratch layout (doubles): [0] zmin [1] zmax [2] dz [3] inv_dz [4] nlive [5] qper
//   [8 .. 8+2*G) per-block min/max partials, then V[nbins]; int scratch: counts[nbins].
constexpr int kLwBlocks = 296;  // 2 x 148 SMs
constexpr int kLwThreads = 256;
size_t longwake_scratch_doubles(int nbins) { return 8 + 2 * kLwBlocks + 2 * (size_t)kLwBlocks + nbins + 8; }

__global__ void __launch_bounds__(kLwThreads) k_lw_drift_minmax(TrackParams P, double half_len,
                                                                double* scr) {
    __shared__ double smin[kLwThreads / 32], smax[kLwThreads / 32];
    __shared__ double scnt[kLwThreads / 32];
    const int nlive = *P.nlive;
    const int64_t n = P.ntot;
    double mn = INFINITY, mx = -INFINITY, cnt = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nlive; i += gridDim.x * blockDim.x) {
        int p = P.live[i];
        double x = P.st[p];
        if (nan_(x)) continue;
        if (half_len != 0) {
            fast::St s{x, P.st[n + p], P.st[2 * n + p], P.st[3 * n + p], P.st[4 * n + p], P.st[5 * n + p]};
            fast::drift_elem(s, half_len);
            P.st[p] = s.x; P.st[2 * n + p] = s.y; P.st[4 * n + p] = s.z;
        }
        double z = P.st[4 * n + p];
        mn = fmin(mn, z);
        mx = fmax(mx, z);
        cnt += 1.0;
    }
    for (int o = 16; o > 0; o >>= 1) {
        mn = fmin(mn, __shfl_xor_sync(FULL, mn, o));
        mx = fmax(mx, __shfl_xor_sync(FULL, mx, o));
        cnt += __shfl_xor_sync(FULL, cnt, o);
    }
    int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { smin[w] = mn; smax[w] = mx; scnt[w] = cnt; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < kLwThreads / 32; k++) { mn = fmin(mn, smin[k]); mx = fmax(mx, smax[k]); }
        double c = 0;
        for (int k = 0; k < kLwThreads / 32; k++) c += scnt[k];
        scr[8 + blockIdx.x] = smin[0] < mn ? smin[0] : mn;
        scr[8 + kLwBlocks + blockIdx.x] = smax[0] > mx ? smax[0] : mx;
        scr[8 + 2 * kLwBlocks + blockIdx.x] = c;
    }
}

__global__ void k_lw_setup(double* scr, int32_t* counts, int nbins, double charge_nc) {
    // one block: reduce the partials (fixed order), bin geometry, zero the histogram
    if (threadIdx.x == 0) {
        double mn = INFINITY, mx = -INFINITY, c = 0;
        for (int b = 0; b < kLwBlocks; b++) {
            mn = fmin(mn, scr[8 + b]);
            mx = fmax(mx, scr[8 + kLwBlocks + b]);
            c += scr[8 + 2 * kLwBlocks + b];
        }
        double dz = (mx - mn) / nbins;
        if (!(dz > 0)) dz = 1e-12;
        scr[0] = mn; scr[1] = mx; scr[2] = dz; scr[3] = 1.0 / dz; scr[4] = c;
        scr[5] = (c > 0) ? charge_nc * 1e-9 / c : 0.0;
    }
    for (int b = threadIdx.x; b < nbins; b += blockDim.x) counts[b] = 0;
}

__device__ __forceinline__ int lw_bin(double z, double zmin, double inv_dz, int nbins) {
    int b = (int)((z - zmin) * inv_dz);
    return b < 0 ? 0 : (b > nbins - 1 ? nbins - 1 : b);
}

// Histogram: shared-memory counts; lanes hitting the same bin are merged first (match + popc).
__global__ void __launch_bounds__(kLwThreads) k_lw_hist(TrackParams P, const double* scr,
                                                        int32_t* counts, int nbins) {
    extern __shared__ int sh[];
    for (int b = threadIdx.x; b < nbins; b += blockDim.x) sh[b] = 0;
    __syncthreads();
    const int nlive = *P.nlive;
    const int64_t n = P.ntot;
    const double zmin = scr[0], inv_dz = scr[3];
    const int lane = threadIdx.x & 31;
    for (int i0 = blockIdx.x * blockDim.x; i0 < nlive; i0 += gridDim.x * blockDim.x) {
        int i = i0 + threadIdx.x;
        int b = -1;
        if (i < nlive) {
            int p = P.live[i];
            if (!nan_(P.st[p])) b = lw_bin(P.st[4 * n + p], zmin, inv_dz, nbins);
        }
        unsigned peers = __match_any_sync(FULL, b);
        int leader = __ffs(peers) - 1;
        if (b >= 0 && lane == leader) atomicAdd(&sh[b], __popc(peers));
    }
    __syncthreads();
    for (int b = threadIdx.x; b < nbins; b += blockDim.x)
        if (sh[b]) atomicAdd(&counts[b], sh[b]);
}

// Wake potential per bin: V_j = qper [ W(0)/2 c_j + sum_{k>j} W((k-j) dz) c_k ].
__global__ void k_lw_voltage(double* scr, const int32_t* counts, int nbins, double Rs, double fr,
                             double Q) {
    extern __shared__ double w[];
    const double dz = scr[2], qper = scr[5];
    const double wr = 2 * 3.1415926535897932384626 * fr;
    const double a = wr / (2 * Q);
    const double wb = sqrt(wr * wr - a * a);
    const double amp = wr * Rs / Q;
    for (int k = threadIdx.x; k < nbins; k += blockDim.x) {
        double tau = k * dz / 2.99792458e8;
        w[k] = amp * exp(-a * tau) * (cos(wb * tau) - (a / wb) * sin(wb * tau));
    }
    __syncthreads();
    double* V = scr + 8 + 3 * kLwBlocks;
    for (int j = threadIdx.x; j < nbins; j += blockDim.x) {
        double v = 0.5 * amp * counts[j] * qper;
        for (int k = j + 1; k < nbins; k++) v += w[k - j] * counts[k] * qper;
        V[j] = v;
    }
}

__global__ void __launch_bounds__(kLwThreads) k_lw_kick(TrackParams P, const double* scr, int nbins,
                                                        double inv_e, double half_len) {
    const int nlive = *P.nlive;
    const int64_t n = P.ntot;
    const double zmin = scr[0], inv_dz = scr[3];
    const double* V = scr + 8 + 3 * kLwBlocks;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nlive; i += gridDim.x * blockDim.x) {
        int p = P.live[i];
        if (nan_(P.st[p])) continue;
        int b = lw_bin(P.st[4 * n + p], zmin, inv_dz, nbins);
        double d = P.st[5 * n + p] - V[b] * inv_e;
        P.st[5 * n + p] = d;
        if (half_len != 0) {
            fast::St s{P.st[p], P.st[n + p], P.st[2 * n + p], P.st[3 * n + p], P.st[4 * n + p], d};
            fast::drift_elem(s, half_len);
            P.st[p] = s.x; P.st[2 * n + p] = s.y; P.st[4 * n + p] = s.z;
        }
    }
}

// The wake in three stages, so that a multi-GPU run can exchange the bunch's z range and count
// after stage 1 and its bin counts after stage 2 (capi.cpp).  Stage 1: first half drift, z range
// and live count, local bin geometry, zeroed counts (with the wake off, also the second half
// drift: the element is then done).  Stage 2: histogram.  Stage 3: wake potential and kick, then
// the second half drift.
LwParams longwake_params(const DevElem& e) {
    LwParams w;
    w.half = 0.5 * e.v[V_LEN];
    w.energy = e.v[V_W + 0];
    w.charge = e.v[V_W + 1];
    w.Rs = e.v[V_W + 2];
    w.fr = e.v[V_W + 3];
    w.Q = e.v[V_W + 4];
    w.nbins = (int)e.v[V_W + 5];
    if (w.nbins < 1) w.nbins = 1;
    if (w.nbins > 4096) w.nbins = 4096;
    w.on = e.flags != 0;
    return w;
}

void launch_longwake_stage(int stage, const TrackParams& p, const LwParams& w, double* scr, int32_t* counts,
                           cudaStream_t s) {
    if (stage == 1) {
        k_lw_drift_minmax<<<kLwBlocks, kLwThreads, 0, s>>>(p, w.half, scr);
        if (!w.on) {
            // wake off: the second half drift still applies
            k_lw_kick<<<kLwBlocks, kLwThreads, 0, s>>>(p, scr, 0, 0.0, w.half);
            return;
        }
        k_lw_setup<<<1, 256, 0, s>>>(scr, counts, w.nbins, w.charge);
    } else if (stage == 2) {
        k_lw_hist<<<kLwBlocks, kLwThreads, w.nbins * sizeof(int), s>>>(p, scr, counts, w.nbins);
    } else {
        k_lw_voltage<<<1, 256, w.nbins * sizeof(double), s>>>(scr, counts, w.nbins, w.Rs, w.fr, w.Q);
        k_lw_kick<<<kLwBlocks, kLwThreads, 0, s>>>(p, scr, w.nbins, 1.0 / (w.energy * 1e6), w.half);
    }
}

void launch_longwake(const TrackParams& p, const DevElem* e_dev, const DevElem& e, double* scr,
                     int32_t* counts, cudaStream_t s) {
    (void)e_dev;
    const LwParams w = longwake_params(e);
    launch_longwake_stage(1, p, w, scr, counts, s);
    if (!w.on) return;
    launch_longwake_stage(2, p, w, scr, counts, s);
    launch_longwake_stage(3, p, w, scr, counts, s);
}

// ---- transverse resonator wake, O(N^2) pairwise as ATransWake::pass (accel.cpp:1603-1657) ----
// Semantics for len != 0: all particles take the first half drift before any kick (the reference
// interleaves drift and kick per particle, so its result depends on particle order there).
__global__ void k_tw_drift(TrackParams P, double half_len) {
    const int nlive = *P.nlive;
    const int64_t n = P.ntot;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nlive; i += gridDim.x * blockDim.x) {
        int p = P.live[i];
        if (nan_(P.st[p]) || half_len == 0) continue;
        fast::St s{P.st[p], P.st[n + p], P.st[2 * n + p], P.st[3 * n + p], P.st[4 * n + p], P.st[5 * n + p]};
        fast::drift_elem(s, half_len);
        P.st[p] = s.x; P.st[2 * n + p] = s.y; P.st[4 * n + p] = s.z;
    }
}

__global__ void k_tw_kick(TrackParams P, DevElem e) {
    const int nlive = *P.nlive;
    const int64_t n = P.ntot;
    const double PI = 3.1415926535897932384626, C0 = 2.99792458e8;
    const double energy = e.v[V_W + 0], Ne = e.v[V_W + 1], Wx = e.v[V_W + 2], fRx = e.v[V_W + 3],
                 Qx = e.v[V_W + 4], Wy = e.v[V_W + 5], fRy = e.v[V_W + 6], Qy = e.v[V_W + 7];
    const double q = Ne / n * 1000;
    const double kRx = 2 * PI * fRx * 1.0e9 / C0, kRy = 2 * PI * fRy * 1.0e9 / C0;
    const double ax = kRx / 2 / Qx, ay = kRy / 2 / Qy;
    const double kbx = kRx * sqrt(1.0 - 0.25 / (Qx * Qx)), kby = kRy * sqrt(1.0 - 0.25 / (Qy * Qy));
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nlive; i += gridDim.x * blockDim.x) {
        int p = P.live[i];
        if (nan_(P.st[p])) continue;
        const double zi = P.st[4 * n + p];
        double dxp = 0, dyp = 0;
        for (int j = 0; j < nlive; j++) {
            int pj = P.live[j];
            if (pj == p) continue;
            double xj = P.st[pj];
            if (nan_(xj)) continue;
            double zij = zi - P.st[4 * n + pj];
            if (zij > 0) continue;
            dxp = dxp - q * Wx * exp(ax * zij) * sin(kbx * zij) * xj / energy / 1.0e6;
            dyp = dyp - q * Wy * exp(ay * zij) * sin(kby * zij) * P.st[2 * n + pj] / energy / 1.0e6;
        }
        P.st[n + p] += dxp * (1 + P.st[5 * n + p]);
        P.st[3 * n + p] += dyp * (1 + P.st[5 * n + p]);
    }
}

void launch_tw_drift(const TrackParams& p, double half_len, cudaStream_t s) {
    k_tw_drift<<<296, 256, 0, s>>>(p, half_len);
}

void launch_transwake(const TrackParams& p, const DevElem* e_dev, const DevElem& e, double* xsnap,
                      cudaStream_t s) {
    (void)e_dev; (void)xsnap;
    const double half = 0.5 * e.v[V_LEN];
    if (half != 0) k_tw_drift<<<296, 256, 0, s>>>(p, half);
    if (e.flags) k_tw_kick<<<296, 256, 0, s>>>(p, e);
    if (half != 0) k_tw_drift<<<296, 256, 0, s>>>(p, half);
}

// ---- beam moments (calc_beam_stat, utility.cpp:387-438), deterministic two-pass --------------
constexpr int kStatThreads = 256;
int beam_stat_blocks(int64_t n) {
    int64_t b = (n + kStatThreads * 4 - 1) / (kStatThreads * 4);
    if (b < 1) b = 1;
    if (b > 1024) b = 1024;
    return (int)b;
}

template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* out) {
    __shared__ double sh[kStatThreads / 32][K];
#pragma unroll
    for (int k = 0; k < K; k++)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(FULL, v[k], o);
    int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < K; k++) sh[w][k] = v[k];
    __syncthreads();
    if (threadIdx.x < K) {
        double s = 0;
        for (int j = 0; j < kStatThreads / 32; j++) s += sh[j][threadIdx.x];
        out[threadIdx.x] = s;
    }
}

__global__ void k_stat1(const double* st, int64_t n, double* part) {
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (nan_(st[i])) continue;
        for (int k = 0; k < 6; k++) v[k] += st[k * n + i];
        v[6] += 1.0;
    }
    block_sum<7>(v, part + 7 * blockIdx.x);
}
__global__ void k_stat_fin(const double* part, int nblk, int K, double* out) {
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        double s = 0;
        for (int b = 0; b < nblk; b++) s += part[K * b + k];
        out[k] = s;
    }
}
__global__ void k_stat2(const double* st, int64_t n, const double* sums, double* part) {
    double v[12] = {0};
    const double cnt = sums[6];
    double m[6];
    for (int k = 0; k < 6; k++) m[k] = sums[k] / cnt;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (nan_(st[i])) continue;
        double d[6];
        for (int k = 0; k < 6; k++) { d[k] = st[k * n + i] - m[k]; v[k] += d[k] * d[k]; }
        v[6] += d[0] * d[1]; v[7] += d[2] * d[3]; v[8] += d[0] * d[5];
        v[9] += d[1] * d[5]; v[10] += d[2] * d[4]; v[11] += d[3] * d[4];
    }
    block_sum<12>(v, part + 12 * blockIdx.x);
}
__global__ void k_stat_out(const double* s1, const double* s2, double* out) {
    if (threadIdx.x == 0) {
        double c = s1[6];
        for (int k = 0; k < 6; k++) {
            out[k] = s1[k] / c;
            out[6 + k] = sqrt(s2[k] / c);
            out[12 + k] = s2[6 + k] / c;
        }
        out[18] = c;
    }
}

int launch_beam_stat(const double* st, int64_t n, double* part, int nblk, double* out, cudaStream_t s,
                     StatReduce reduce, void* rctx) {
    double* s1 = part + 12 * (size_t)nblk;
    double* s2 = s1 + 8;
    k_stat1<<<nblk, kStatThreads, 0, s>>>(st, n, part);
    k_stat_fin<<<1, 32, 0, s>>>(part, nblk, 7, s1);
    int r = reduce ? reduce(rctx, s1, 7, s) : 0;  // the sums and live count of every rank
    if (r) return r;
    k_stat2<<<nblk, kStatThreads, 0, s>>>(st, n, s1, part);
    k_stat_fin<<<1, 32, 0, s>>>(part, nblk, 12, s2);
    r = reduce ? reduce(rctx, s2, 12, s) : 0;  // the centred second moments of every rank
    if (r) return r;
    k_stat_out<<<1, 32, 0, s>>>(s1, s2, out);
    return 0;
}

// ---- FP64 FMA throughput probe --------------------------------------------------------------
// FP64 roofline probe: 8 independent FMA chains per thread, 2,048 threads per SM (full
// occupancy), a loop long enough (about 10 ms) that launch and tail effects vanish.  One DFMA
// warp instruction occupies the SM sub-partition's FP64 unit for two cycles, so the issue slots
// left over cover the loop's own instructions and the probe can reach the pipe's rate.
constexpr int kPeakChains = 8;

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// clk (4 words): block 0's thread 0 records its SM clock counter and the global nanosecond timer
// at the start and at the end of its loop, which gives the SM clock while the probe runs.
__global__ void __launch_bounds__(512, 4) k_fp64_peak(double* out, unsigned long long* clk, int iters,
                                                       double b, double c) {
    const bool rec = blockIdx.x == 0 && threadIdx.x == 0;
    if (rec) {
        clk[0] = clock64();
        clk[1] = global_ns();
    }
    double a[kPeakChains];
#pragma unroll
    for (int j = 0; j < kPeakChains; j++) a[j] = threadIdx.x * 1e-9 + j;
#pragma unroll 4
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int j = 0; j < kPeakChains; j++) a[j] = fma(a[j], b, c);
    }
    double r = 0;
#pragma unroll
    for (int j = 0; j < kPeakChains; j++) r += a[j];
    if (r == 1234.5) out[0] = r;  // keeps the chains live
    if (rec) {
        clk[2] = clock64();
        clk[3] = global_ns();
    }
}

double fp64_peak_run(int sm_count, cudaStream_t s, float* ms_out, double* sm_mhz_out) {
    const int iters = 1 << 16, threads = 512, blocks = sm_count * 4;  // about 9 ms
    double* dummy = nullptr;
    cudaMallocAsync(&dummy, sizeof(double) + 4 * sizeof(unsigned long long), s);
    unsigned long long* clk = (unsigned long long*)(dummy + 1);
    k_fp64_peak<<<blocks, threads, 0, s>>>(dummy, clk, iters / 8, 0.999999, 1e-7);  // warm-up
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    double mhz = 0;
    for (int rep = 0; rep < 3; rep++) {  // the best of three
        cudaEventRecord(e0, s);
        k_fp64_peak<<<blocks, threads, 0, s>>>(dummy, clk, iters, 0.999999, 1e-7);
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) {
            best = ms;
            unsigned long long h[4] = {0, 0, 0, 0};
            cudaMemcpy(h, clk, sizeof(h), cudaMemcpyDeviceToHost);
            mhz = h[3] > h[1] ? (double)(h[2] - h[0]) / (double)(h[3] - h[1]) * 1e3 : 0.0;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFreeAsync(dummy, s);
    if (ms_out) *ms_out = best;
    if (sm_mhz_out) *sm_mhz_out = mhz;
    double flops = 2.0 * kPeakChains * (double)iters * threads * (double)blocks;
    return flops / (best * 1e-3) / 1e12;
}

}  // namespace accel
