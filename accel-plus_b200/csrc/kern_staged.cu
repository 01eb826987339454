// kern_staged.cu — the instance-staged variant of the fused FP64 tracker (sm_100a).
//
// The same persistent tracker as k_fused (kern_fused.cu): one thread per particle, coordinates in
// registers across the turns of a segment, losses checked inline.  What differs is where the
// element records come from.  It is a separate module from the production fused kernel, so a
// fault in either cannot reach the other.
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

// Elements outside the specialised paths run the literal map out of line, the state in and out
// by value (the same arrangement as the fused kernel's rare-element call).
__device__ __noinline__ fast::St staged_literal(fast::St s, const DevElem* __restrict__ e, uint64_t seed,
                                                uint32_t pid, uint32_t turn) {
    double r[6] = {s.x, s.px, s.y, s.py, s.z, s.d};
    lit::QeSource q{seed, pid, turn, (uint32_t)e->elem, 0u};
    lit::pass<double>(*e, r, q);
    return fast::St{r[0], r[1], r[2], r[3], r[4], r[5]};
}

// the specialised multipole paths by effective order (0..3) and skew level, as the fused kernel
// dispatches them; h is a hot line
__device__ __forceinline__ void staged_strmpole(fast::St& s, const DevElem* __restrict__ h) {
    const int sk = (h->flags & STR_SKEW) ? ((h->flags & STR_SKEW0) ? 1 : 2) : 0;
    switch (h->order_eff * 4 + sk) {
    case 0: fast::strmpole<0, 0>(s, h); break;
    case 1: fast::strmpole<0, 1>(s, h); break;
    case 2: fast::strmpole<0, 2>(s, h); break;
    case 4: fast::strmpole<1, 0>(s, h); break;
    case 5: fast::strmpole<1, 1>(s, h); break;
    case 6: fast::strmpole<1, 2>(s, h); break;
    case 8: fast::strmpole<2, 0>(s, h); break;
    case 9: fast::strmpole<2, 1>(s, h); break;
    case 10: fast::strmpole<2, 2>(s, h); break;
    case 12: fast::strmpole<3, 0>(s, h); break;
    case 13: fast::strmpole<3, 1>(s, h); break;
    default: fast::strmpole<3, 2>(s, h); break;
    }
}

__device__ __forceinline__ void staged_bendmpole(fast::St& s, const DevElem* __restrict__ h, uint64_t seed,
                                                 uint32_t pid, uint32_t turn) {
    const bool pure = h->h[H_BK1] == 0.0 && h->h[H_BK2] == 0.0;
    switch (h->order_eff * 2 + (pure ? 1 : 0)) {
    case 0: fast::bendmpole<0, false>(s, h, seed, pid, turn); break;
    case 1: fast::bendmpole<0, true>(s, h, seed, pid, turn); break;
    case 2: fast::bendmpole<1, false>(s, h, seed, pid, turn); break;
    case 3: fast::bendmpole<1, true>(s, h, seed, pid, turn); break;
    case 4: fast::bendmpole<2, false>(s, h, seed, pid, turn); break;
    case 5: fast::bendmpole<2, true>(s, h, seed, pid, turn); break;
    case 6: fast::bendmpole<3, false>(s, h, seed, pid, turn); break;
    default: fast::bendmpole<3, true>(s, h, seed, pid, turn); break;
    }
}

// ---- instance-staged variant: element hot lines in shared memory --------------------------------
// The element records of the instance a block works on are read from shared memory instead of
// through L1.  Each record's first 128-byte line holds everything the fast maps read (engine.h),
// so the library keeps a contiguous copy of those lines (k_extract_hot, hot[record]) and a block
// stages the ne lines of one instance (60 KB for the 470-element DBA) with one bulk asynchronous
// copy (cp.async.bulk, the TMA engine's one-dimensional form; CTA-local, no multicast) whose
// completion an mbarrier signals.  Work is handed out per block: a task is the next BS entries of
// the live list, which is grouped by instance (stable compaction keeps it so), and the block
// restages only when a task's first particle belongs to another instance than the staged one.
// Lanes whose particle belongs to another instance (a task straddling two) read their records
// from global memory as the plain fused kernel does; so do the rare elements and the
// quantum-excitation bends, whose parameters lie beyond the hot line.
struct alignas(128) HotLine {
    uint4 q[8];
};
static_assert(sizeof(HotLine) == 128, "a hot line is one 128-byte line");

__global__ void k_extract_hot(const DevElem* __restrict__ tbl, int64_t nrec, HotLine* __restrict__ hot) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;  // (record, 16-byte word)
    if (i >= nrec * 8) return;
    const int64_t r = i >> 3;
    const int w = (int)(i & 7);
    hot[r].q[w] = reinterpret_cast<const HotLine*>(tbl + r)->q[w];
}

void launch_extract_hot(const DevElem* tbl, int64_t nrec, void* hot, cudaStream_t s) {
    const int64_t threads = nrec * 8;
    if (threads > 0)
        k_extract_hot<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(tbl, nrec, (HotLine*)hot);
}

// one element with its hot line `h` (shared or global memory) and its full record `e` (global),
// with the fused kernel's arithmetic: the multipoles up to order 3, the bends, cavities,
// apertures and drifts by their fast maps (quantum-excitation bends on the full record, whose
// parameters lie beyond the hot line); higher orders and the other element kinds by the literal
// map on the full record
__device__ __forceinline__ void fused_elem_staged(fast::St& s, const DevElem* __restrict__ h,
                                                  const DevElem* __restrict__ e, uint64_t seed,
                                                  uint32_t pid, uint32_t turn) {
    switch (h->op) {
    case OP_NOP: break;
    case OP_DRIFT: fast::drift_elem(s, h->h[H_LEN]); break;
    case OP_STRMPOLE:
        if (h->order_eff <= kHotOrder) staged_strmpole(s, h);
        else s = staged_literal(s, e, seed, pid, turn);
        break;
    case OP_BENDMPOLE:  // quantum-excitation bends read past the hot line: their full record
        if (h->order_eff <= kHotOrder) staged_bendmpole(s, h->flags != 2 ? h : e, seed, pid, turn);
        else s = staged_literal(s, e, seed, pid, turn);
        break;
    case OP_CAVITY: fast::cavity(s, h); break;
    case OP_APERTURE: fast::aperture(s, h); break;
    case OP_TRANSWAKE:
    case OP_LONGWAKE: break;
    default: s = staged_literal(s, e, seed, pid, turn); break;
    }
}

// mbarrier helpers (shared::cta addresses); the wait is bounded
__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t a, uint32_t bytes) {
    asm volatile("{ .reg .b64 st; mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1; }" ::"r"(a), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_wait(uint32_t a, uint32_t phase, int limit) {
    for (int i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                     : "=r"(done) : "r"(a), "r"(phase) : "memory");
        if (done) return true;
    }
    return false;
}
constexpr int kStageWaitLimit = 1 << 22;  // try_wait rounds before a stage counts as failed

template <int BS, int MINB>
__global__ void __launch_bounds__(BS, MINB) k_fused_staged(const TrackParams P, const HotLine* __restrict__ hot,
                                                           int ne) {
    extern __shared__ __align__(128) unsigned char sm_hot[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ int s_base, s_inst, s_fail;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nlive = *P.nlive;
    const int64_t n = P.ntot;
    const int tbase = P.turn_dev ? *P.turn_dev : 0;
    const int rbase = (P.rng_base ? *P.rng_base : 0) + tbase;
    double* __restrict__ st = P.st;
    const uint32_t bytes = (uint32_t)ne * 128u;
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(sm_hot);
    const uint32_t ma = (uint32_t)__cvta_generic_to_shared(&mbar);
    if (threadIdx.x == 0) {
        mbar_init(ma, 1);
        s_fail = 0;
    }
    __syncthreads();
    int staged = -1;
    uint32_t phase = 0;
    for (;;) {
        if (threadIdx.x == 0) {
            const int b = atomicAdd(P.chunk_ctr, BS);
            s_base = b;
            s_inst = b < nlive ? (P.pinst ? P.pinst[P.live[b]] : 0) : -1;
        }
        __syncthreads();
        const int base = s_base, inst0 = s_inst;
        if (base >= nlive) break;
        if (inst0 != staged) {
            // every thread is past its reads of the previous table (the barrier above)
            if (threadIdx.x == 0) {
                const HotLine* src = hot + (P.tbl_off ? P.tbl_off[inst0] : 0);
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                mbar_expect_tx(ma, bytes);
                asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                             ::"r"(sa), "l"(src), "r"(bytes), "r"(ma) : "memory");
                const int first = P.stage_wait < 0 ? 0 : P.stage_wait == 0 ? kStageWaitLimit : P.stage_wait;
                if (!mbar_wait(ma, phase, first)) {
                    s_fail = 1;
                    atomicExch(P.err, 1);
                    mbar_wait(ma, phase, kStageWaitLimit);  // the copy in flight, before leaving
                }
            }
            __syncthreads();
            if (s_fail) return;
            phase ^= 1u;
            staged = inst0;
        }
        const int idx = base + warp * 32 + lane;
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
        const bool shared_lines = inst == staged;
        bool alive = have && !nan_(s.x);
        for (int t = 0; t < P.nturn; t++) {
            if (!__any_sync(FULL, alive)) break;
            if (alive) {
                const uint32_t rt = (uint32_t)(rbase + P.rng_turn0 + t);
                for (int e = P.e0; e < P.e1; e++) {
                    const DevElem* h = shared_lines ? reinterpret_cast<const DevElem*>(sm_hot + 128 * e) : T + e;
                    fused_elem_staged(s, h, T + e, P.seed, (uint32_t)p, rt);
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
        __syncthreads();  // the table may be restaged for the next task
    }
}

// (block, min blocks per SM): 60 KB of lines per block leaves room for three blocks per SM
#define STAGED_VARIANTS(X) X(0, 128, 3) X(1, 256, 2) X(2, 192, 3)

VariantInfo staged_variant_info(int v) {
    switch (v) {
#define X(i, b, m) case i: return VariantInfo{b, m};
        STAGED_VARIANTS(X)
#undef X
    default: return VariantInfo{128, 3};
    }
}

template <int BS, int MINB>
static int staged_bps(int bytes) {
    if (cudaFuncSetAttribute(k_fused_staged<BS, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) !=
        cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_fused_staged<BS, MINB>, BS, bytes) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return nb;
}

int staged_blocks_per_sm(int v, int ne) {
    const int bytes = ne * 128;
    switch (v) {
#define X(i, b, m) case i: return staged_bps<b, m>(bytes);
        STAGED_VARIANTS(X)
#undef X
    default: return 0;
    }
}

void launch_fused_staged(const TrackParams& p, int v, const void* hot, int ne, int grid, cudaStream_t s) {
    const size_t bytes = (size_t)ne * 128;
    switch (v) {
#define X(i, b, m) case i: k_fused_staged<b, m><<<grid, b, bytes, s>>>(p, (const HotLine*)hot, ne); break;
        STAGED_VARIANTS(X)
#undef X
    default: break;
    }
}

}  // namespace accel
