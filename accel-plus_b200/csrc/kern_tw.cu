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
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
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

// sort keys: z of each live particle (-inf for one lost before the wake, sorted last)
__global__ void k_tw_keys(const TrackParams P, double* keys, int32_t* vals, int32_t* nvalid) {
    const int nlive = *P.nlive;
    const int64_t n = P.ntot;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nlive; i += gridDim.x * blockDim.x) {
        const int p = P.live[i];
        const double x = P.st[p];
        const bool ok = !(x != x);
        keys[i] = ok ? P.st[4 * n + p] : -INFINITY;
        vals[i] = p;
        if (ok) atomicAdd(nvalid, 1);
    }
}

// per sorted position: the particle's four terms E cos x, E sin x (and in y), zero when lost
__global__ void k_tw_terms(const TrackParams P, const double* keys, const int32_t* vals, const int32_t* nvalid,
                           TwConst c, Quad4* terms) {
    const int nv = *nvalid;
    const int64_t n = P.ntot;
    const double zr = nv > 0 ? keys[0] : 0.0;
    // every one of the ntot entries the scan reads: zero past the valid ones
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        Quad4 t{0, 0, 0, 0};
        if (k < nv) {
            const int p = vals[k];
            const double z = keys[k], x = P.st[p], y = P.st[2 * n + p];
            const double ex = exp(c.ax * (zr - z)), ey = exp(c.ay * (zr - z));
            double sx, cx, sy, cy;
            sincos(c.kbx * z, &sx, &cx);
            sincos(c.kby * z, &sy, &cy);
            t = Quad4{ex * cx * x, ex * sx * x, ey * cy * y, ey * sy * y};
        }
        terms[k] = t;
    }
}

// kick of sorted position k from the prefix sums (or, when the z range is too long for the
// factorisation, from the pair sum over the sorted list)
__global__ void k_tw_kick_sorted(const TrackParams P, const double* keys, const int32_t* vals,
                                 const int32_t* nvalid, TwConst c, const Quad4* terms, const Quad4* prefix) {
    const int nv = *nvalid;
    const int64_t n = P.ntot;
    if (nv == 0) return;
    const double zr = keys[0], zmin = keys[nv - 1];
    const bool factor = c.ax * (zr - zmin) <= 600.0 && c.ay * (zr - zmin) <= 600.0;
    const double scale = c.q / c.energy / 1.0e6;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nv; k += gridDim.x * blockDim.x) {
        const int p = vals[k];
        const double zi = keys[k];
        double dxp, dyp;
        if (factor) {
            // last position whose z >= zi: the end of zi's group in the descending order
            int lo = k, hi = nv - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (keys[mid] >= zi) lo = mid;
                else hi = mid - 1;
            }
            const Quad4 a = prefix[lo], own = terms[k];
            const double Cx = a.cx - own.cx, Sx = a.sx - own.sx, Cy = a.cy - own.cy, Sy = a.sy - own.sy;
            double sx, cx, sy, cy;
            sincos(c.kbx * zi, &sx, &cx);
            sincos(c.kby * zi, &sy, &cy);
            dxp = -scale * c.Wx * exp(c.ax * (zi - zr)) * (sx * Cx - cx * Sx);
            dyp = -scale * c.Wy * exp(c.ay * (zi - zr)) * (sy * Cy - cy * Sy);
        } else {
            dxp = 0;
            dyp = 0;
            for (int j = 0; j < nv && keys[j] >= zi; j++) {
                if (j == k) continue;
                const int pj = vals[j];
                const double zij = zi - keys[j];
                dxp -= c.q * c.Wx * exp(c.ax * zij) * sin(c.kbx * zij) * P.st[pj] / c.energy / 1.0e6;
                dyp -= c.q * c.Wy * exp(c.ay * zij) * sin(c.kby * zij) * P.st[2 * n + pj] / c.energy / 1.0e6;
            }
        }
        P.st[n + p] += dxp * (1 + P.st[5 * n + p]);
        P.st[3 * n + p] += dyp * (1 + P.st[5 * n + p]);
    }
}

__global__ void k_tw_zero(int32_t* c) { *c = 0; }
__global__ void k_tw_fill(double* a, double v, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        a[i] = v;
}
}  // namespace

size_t tw_sorted_scratch_bytes(int64_t n) {
    size_t sort_tmp = 0, scan_tmp = 0;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, sort_tmp, (const double*)nullptr, (double*)nullptr,
                                              (const int32_t*)nullptr, (int32_t*)nullptr, (int)n);
    cub::DeviceScan::InclusiveScan(nullptr, scan_tmp, (const Quad4*)nullptr, (Quad4*)nullptr, Quad4Sum(), (int)n);
    const size_t a = 256;
    auto up = [&](size_t b) { return (b + a - 1) / a * a; };
    return up(2 * n * sizeof(double)) + up(2 * n * sizeof(int32_t)) + up(2 * n * sizeof(Quad4)) + up(16) +
           up(std::max(sort_tmp, scan_tmp));
}

void launch_transwake_sorted(const TrackParams& p, const DevElem& e, void* scratch, size_t scratch_bytes,
                             cudaStream_t s) {
    const int64_t n = p.ntot;
    const size_t a = 256;
    auto up = [&](size_t b) { return (b + a - 1) / a * a; };
    char* base = (char*)scratch;
    double* keys_in = (double*)base;
    double* keys_out = keys_in + n;
    base += up(2 * n * sizeof(double));
    int32_t* vals_in = (int32_t*)base;
    int32_t* vals_out = vals_in + n;
    base += up(2 * n * sizeof(int32_t));
    Quad4* terms = (Quad4*)base;
    Quad4* prefix = terms + n;
    base += up(2 * n * sizeof(Quad4));
    int32_t* nvalid = (int32_t*)base;
    base += up(16);
    void* tmp = base;
    size_t tmp_bytes = scratch_bytes - (size_t)(base - (char*)scratch);
    const TwConst c = tw_const(e, n);
    const double half = 0.5 * e.v[V_LEN];
    // with length: the half drifts around the kick, as the pair-sum path
    if (half != 0) launch_tw_drift(p, half, s);
    if (e.flags) {
        k_tw_zero<<<1, 1, 0, s>>>(nvalid);
        // the live count is on the device: size every pass for all ntot entries (entries past
        // nlive are not read; the sort and scan run over ntot, with keys -inf past nlive)
        k_tw_fill<<<296, 256, 0, s>>>(keys_in, -INFINITY, n);
        k_tw_keys<<<296, 256, 0, s>>>(p, keys_in, vals_in, nvalid);
        cub::DeviceRadixSort::SortPairsDescending(tmp, tmp_bytes, keys_in, keys_out, vals_in, vals_out, (int)n, 0,
                                                  64, s);
        k_tw_terms<<<296, 256, 0, s>>>(p, keys_out, vals_out, nvalid, c, terms);
        cub::DeviceScan::InclusiveScan(tmp, tmp_bytes, terms, prefix, Quad4Sum(), (int)n, s);
        k_tw_kick_sorted<<<296, 256, 0, s>>>(p, keys_out, vals_out, nvalid, c, terms, prefix);
    }
    if (half != 0) launch_tw_drift(p, half, s);
}

}  // namespace accel
