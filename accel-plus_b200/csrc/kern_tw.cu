// kern_tw.cu — the transverse resonator wake in O(N log N) (fused mode).
//
// ATransWake::pass (accel.cpp:1603-1657) kicks particle i by
//   dx'_i = -q/(E 1e6) sum_{j != i, z_j >= z_i} Wx exp(ax z_ij) sin(kbx z_ij) x_j,  z_ij = z_i - z_j,
// (and the same in y), an O(N^2) pair sum.  With a reference zr = max z, exp(ax z_ij) =
// exp(ax (z_i - zr)) exp(ax (zr - z_j)) and sin(kb z_ij) = sin(kb z_i) cos(kb z_j) - cos(kb z_i)
// sin(kb z_j), so
//   sum_j ... = exp(ax (z_i - zr)) [ sin(kb z_i) C_i - cos(kb z_i) S_i ],
//   C_i = sum_{j} E_j cos(kb z_j) x_j,  S_i = sum_{j} E_j sin(kb z_j) x_j,  E_j = exp(ax (zr - z_j)),
// over the j with z_j >= z_i other than i.  Sorted by z, highest first, those j are a prefix (up to
// the end of i's group of equal z), so every C_i and S_i is a prefix sum less i's own term: one
// sort, one scan, one binary search per particle.  The result is the same sum in another order
// of operations; where ax (z_max - z_min) would make E_j overflow (above 600), each particle takes
// the pair sum instead.  The plain and exact modes keep the reference's pair sum
// (kern_fused.cu), whose order of operations they reproduce.
//
// A bunch spread over several GPUs: every rank offers the same number of entries (slots, at least
// its particle count; z = -inf marks an empty one), the entries of all ranks are all-gathered
// between the two stages, every rank sorts and scans the whole list and kicks its own particles;
// the charge per particle is Ne over the particles of all ranks.
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/block/block_scan.cuh>
#include <cstdint>
#include <cmath>
#include <algorithm>
#include "kernels.h"

namespace accel {

namespace {
constexpr double kPi = 3.1415926535897932384626, kC0 = 2.99792458e8;

struct Quad4 {
    double cx, sx, cy, sy;
};
struct Quad4Sum {
    __host__ __device__ __forceinline__ Quad4 operator()(const Quad4& a, const Quad4& b) const {
        return Quad4{a.cx + b.cx, a.sx + b.sx, a.cy + b.cy, a.sy + b.sy};
    }
};

// The prefix sums in a fixed order of additions, so that a run is reproducible bit for bit (a
// decoupled look-back scan adds its partial sums in an order that depends on timing): within a
// tile of 1024 entries each thread sums its 4 in order and a block scan combines the threads;
// one block scans the tile totals (each thread a contiguous run of them, in order); the kick adds
// its tile's offset to the entry's in-tile prefix.
constexpr int kScanThreads = 256, kScanItems = 4, kScanTile = kScanThreads * kScanItems;
constexpr int kTileScanThreads = 1024;

__global__ void __launch_bounds__(kScanThreads) k_tw_scan_tiles(const Quad4* in, Quad4* out, Quad4* tile_sum,
                                                                int64_t total) {
    using BS = cub::BlockScan<Quad4, kScanThreads>;
    __shared__ typename BS::TempStorage ts;
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    Quad4 v[kScanItems];
    Quad4 acc{0, 0, 0, 0};
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        const int64_t i = base + j;
        const Quad4 x = i < total ? in[i] : Quad4{0, 0, 0, 0};
        acc = j == 0 ? x : Quad4Sum()(acc, x);
        v[j] = acc;
    }
    Quad4 excl, agg;
    BS(ts).ExclusiveScan(acc, excl, Quad4{0, 0, 0, 0}, Quad4Sum(), agg);
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        const int64_t i = base + j;
        if (i < total) out[i] = threadIdx.x == 0 ? v[j] : Quad4Sum()(excl, v[j]);
    }
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = agg;
}

// in place: tile totals -> exclusive tile offsets
__global__ void __launch_bounds__(kTileScanThreads) k_tw_scan_tile_sums(Quad4* tile_sum, int64_t ntiles) {
    using BS = cub::BlockScan<Quad4, kTileScanThreads>;
    __shared__ typename BS::TempStorage ts;
    const int64_t per = (ntiles + kTileScanThreads - 1) / kTileScanThreads;
    const int64_t b0 = (int64_t)threadIdx.x * per, b1 = b0 + per < ntiles ? b0 + per : ntiles;
    Quad4 acc{0, 0, 0, 0};
    for (int64_t b = b0; b < b1; b++) acc = b == b0 ? tile_sum[b] : Quad4Sum()(acc, tile_sum[b]);
    Quad4 run, agg;
    BS(ts).ExclusiveScan(acc, run, Quad4{0, 0, 0, 0}, Quad4Sum(), agg);
    for (int64_t b = b0; b < b1; b++) {
        const Quad4 t = tile_sum[b];
        tile_sum[b] = run;
        run = b == 0 ? t : Quad4Sum()(run, t);
    }
}

struct TwConst {
    double q, energy, Wx, Wy, ax, ay, kbx, kby;
};

__host__ __device__ TwConst tw_const(const DevElem& e, int64_t n) {
    TwConst c;
    c.energy = e.v[V_W + 0];
    const double Ne = e.v[V_W + 1], fRx = e.v[V_W + 3], Qx = e.v[V_W + 4], fRy = e.v[V_W + 6], Qy = e.v[V_W + 7];
    c.Wx = e.v[V_W + 2];
    c.Wy = e.v[V_W + 5];
    c.q = Ne / n * 1000;
    const double kRx = 2 * kPi * fRx * 1.0e9 / kC0, kRy = 2 * kPi * fRy * 1.0e9 / kC0;
    c.ax = kRx / 2 / Qx;
    c.ay = kRy / 2 / Qy;
    c.kbx = kRx * sqrt(1.0 - 0.25 / (Qx * Qx));
    c.kby = kRy * sqrt(1.0 - 0.25 / (Qy * Qy));
    return c;
}

// this rank's entries: slot i < nlive holds live particle live[i] (z, x, y), z = -inf when it was
// lost before the wake; slots past nlive hold -inf.  Also the entry indices of all ranks' entries.
__global__ void k_tw_entries(const TrackParams P, double* key, double* xs, double* ys, int64_t slots,
                             int32_t* val, int64_t total, int32_t* nvalid_local) {
    const int nlive = *P.nlive;
    const int64_t n = P.ntot;
    const int64_t m = slots > total ? slots : total;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        if (i < total) val[i] = (int32_t)i;
        if (i >= slots) continue;
        bool ok = false;
        double z = -INFINITY, x = 0, y = 0;
        if (i < nlive) {
            const int p = P.live[i];
            x = P.st[p];
            ok = !(x != x);
            if (ok) {
                z = P.st[4 * n + p];
                y = P.st[2 * n + p];
            } else {
                x = 0;
            }
        }
        key[i] = z;
        xs[i] = x;
        ys[i] = y;
        const unsigned act = __activemask();
        const unsigned b = __ballot_sync(act, ok);
        if ((threadIdx.x & 31) == __ffs(act) - 1 && b) atomicAdd(nvalid_local, __popc(b));
    }
}

// per sorted position: the entry's four terms E cos x, E sin x (and in y), zero past the valid ones
__global__ void k_tw_terms(const double* key, const int32_t* val, const double* xg, const double* yg,
                           const int32_t* nvalid, int64_t total, TwConst c, Quad4* terms) {
    const int nv = *nvalid;
    const double zr = nv > 0 ? key[0] : 0.0;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        Quad4 t{0, 0, 0, 0};
        if (k < nv) {
            const int g = val[k];
            const double z = key[k], x = xg[g], y = yg[g];
            const double ex = exp(c.ax * (zr - z)), ey = exp(c.ay * (zr - z));
            double sx, cx, sy, cy;
            sincos(c.kbx * z, &sx, &cx);
            sincos(c.kby * z, &sy, &cy);
            t = Quad4{ex * cx * x, ex * sx * x, ey * cy * y, ey * sy * y};
        }
        terms[k] = t;
    }
}

// kick of the sorted entries that are this rank's particles, from the prefix sums (or, when the z
// range is too long for the factorisation, from the pair sum over the sorted entries)
__global__ void k_tw_kick_sorted(const TrackParams P, const double* key, const int32_t* val, const double* xg,
                                 const double* yg, const int32_t* nvalid, int64_t slots, int rank, TwConst c,
                                 const Quad4* terms, const Quad4* prefix, const Quad4* tile_off) {
    const int nv = *nvalid;
    const int nlive = *P.nlive;
    const int64_t n = P.ntot;
    if (nv == 0) return;
    const double zr = key[0], zmin = key[nv - 1];
    const bool factor = c.ax * (zr - zmin) <= 600.0 && c.ay * (zr - zmin) <= 600.0;
    const double scale = c.q / c.energy / 1.0e6;
    // the pair sum over all entries, O(N^2), where the bunch is too long for the factorisation:
    // counted, so that a caller can see the slow path was taken
    if (!factor && P.tw_pair_passes && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(P.tw_pair_passes, 1);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nv; k += gridDim.x * blockDim.x) {
        const int64_t g = val[k];
        // this rank's live slots only (a slot past nlive can sort among the first nv only when a
        // live particle carries a non-finite z)
        if (g / slots != rank || g - (int64_t)rank * slots >= nlive) continue;
        const int p = P.live[g - (int64_t)rank * slots];
        const double zi = key[k];
        double dxp, dyp;
        if (factor) {
            // last position whose z >= zi: the end of zi's group in the descending order
            int lo = k, hi = nv - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (key[mid] >= zi) lo = mid;
                else hi = mid - 1;
            }
            const int tile = lo / kScanTile;
            const Quad4 a = tile == 0 ? prefix[lo] : Quad4Sum()(tile_off[tile], prefix[lo]), own = terms[k];
            const double Cx = a.cx - own.cx, Sx = a.sx - own.sx, Cy = a.cy - own.cy, Sy = a.sy - own.sy;
            double sx, cx, sy, cy;
            sincos(c.kbx * zi, &sx, &cx);
            sincos(c.kby * zi, &sy, &cy);
            dxp = -scale * c.Wx * exp(c.ax * (zi - zr)) * (sx * Cx - cx * Sx);
            dyp = -scale * c.Wy * exp(c.ay * (zi - zr)) * (sy * Cy - cy * Sy);
        } else {
            dxp = 0;
            dyp = 0;
            for (int j = 0; j < nv && key[j] >= zi; j++) {
                if (j == k) continue;
                const int gj = val[j];
                const double zij = zi - key[j];
                dxp -= c.q * c.Wx * exp(c.ax * zij) * sin(c.kbx * zij) * xg[gj] / c.energy / 1.0e6;
                dyp -= c.q * c.Wy * exp(c.ay * zij) * sin(c.kby * zij) * yg[gj] / c.energy / 1.0e6;
            }
        }
        P.st[n + p] += dxp * (1 + P.st[5 * n + p]);
        P.st[3 * n + p] += dyp * (1 + P.st[5 * n + p]);
    }
}

__global__ void k_tw_zero(int32_t* c) { c[0] = 0; c[1] = 0; }

// carves the scratch (base may be null: offsets only); returns the bytes used
size_t carve(char* base, int64_t slots, int nranks, bool gather, TwLayout& t) {
    const int64_t total = slots * nranks;
    size_t off = 0;
    auto take = [&](size_t b) {
        char* p = base ? base + off : nullptr;
        off += (b + 255) / 256 * 256;
        return p;
    };
    t.slots = slots;
    t.total = total;
    t.key_g = (double*)take(sizeof(double) * total);
    t.x_g = (double*)take(sizeof(double) * total);
    t.y_g = (double*)take(sizeof(double) * total);
    if (gather) {
        t.key_s = (double*)take(sizeof(double) * slots);
        t.x_s = (double*)take(sizeof(double) * slots);
        t.y_s = (double*)take(sizeof(double) * slots);
    } else {
        t.key_s = t.key_g;
        t.x_s = t.x_g;
        t.y_s = t.y_g;
    }
    t.key_sorted = (double*)take(sizeof(double) * total);
    t.val_in = (int32_t*)take(sizeof(int32_t) * total);
    t.val_sorted = (int32_t*)take(sizeof(int32_t) * total);
    t.terms = take(sizeof(Quad4) * total);
    t.prefix = take(sizeof(Quad4) * total);
    t.tile_off = take(sizeof(Quad4) * ((total + kScanTile - 1) / kScanTile));
    t.nvalid = (int32_t*)take(16);
    t.tmp = base ? base + off : nullptr;
    size_t sort_tmp = 0;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, sort_tmp, (const double*)nullptr, (double*)nullptr,
                                              (const int32_t*)nullptr, (int32_t*)nullptr, (int)total);
    t.tmp_bytes = sort_tmp;
    return off + t.tmp_bytes;
}
}  // namespace

size_t tw_sorted_scratch_bytes(int64_t slots, int nranks, bool gather) {
    TwLayout t;
    return carve(nullptr, std::max<int64_t>(1, slots), nranks, gather, t);
}

TwLayout tw_layout(void* scratch, int64_t slots, int nranks, bool gather) {
    TwLayout t;
    carve((char*)scratch, std::max<int64_t>(1, slots), nranks, gather, t);
    return t;
}

void launch_transwake_sorted_stage(int stage, const TrackParams& p, const DevElem& e, const TwLayout& t,
                                   int rank, int64_t ntot_all, cudaStream_t s) {
    const double half = 0.5 * e.v[V_LEN];
    const TwConst c = tw_const(e, ntot_all);
    // with gathered entries the total count is nvalid[1], else this rank's nvalid[0]
    const int32_t* nv = t.key_s != t.key_g ? t.nvalid + 1 : t.nvalid;
    if (stage == 1) {
        // with length: the half drifts around the kick, as the pair-sum path
        if (half != 0) launch_tw_drift(p, half, s);
        if (!e.flags) return;
        k_tw_zero<<<1, 1, 0, s>>>(t.nvalid);
        k_tw_entries<<<296, 256, 0, s>>>(p, t.key_s, t.x_s, t.y_s, t.slots, t.val_in, t.total, t.nvalid);
        return;
    }
    if (e.flags) {
        size_t tmp_bytes = t.tmp_bytes;
        cub::DeviceRadixSort::SortPairsDescending(t.tmp, tmp_bytes, t.key_g, t.key_sorted, t.val_in, t.val_sorted,
                                                  (int)t.total, 0, 64, s);
        k_tw_terms<<<296, 256, 0, s>>>(t.key_sorted, t.val_sorted, t.x_g, t.y_g, nv, t.total, c, (Quad4*)t.terms);
        const int64_t ntiles = (t.total + kScanTile - 1) / kScanTile;
        k_tw_scan_tiles<<<(unsigned)ntiles, kScanThreads, 0, s>>>((const Quad4*)t.terms, (Quad4*)t.prefix,
                                                                 (Quad4*)t.tile_off, t.total);
        k_tw_scan_tile_sums<<<1, kTileScanThreads, 0, s>>>((Quad4*)t.tile_off, ntiles);
        k_tw_kick_sorted<<<296, 256, 0, s>>>(p, t.key_sorted, t.val_sorted, t.x_g, t.y_g, nv, t.slots, rank, c,
                                             (const Quad4*)t.terms, (const Quad4*)t.prefix,
                                             (const Quad4*)t.tile_off);
    }
    if (half != 0) launch_tw_drift(p, half, s);
}

}  // namespace accel
