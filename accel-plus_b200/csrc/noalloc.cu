// noalloc.cu — beam moments of a device-resident particle array without any device allocation.
//
// accel_beam_stat (capi.cpp) stages its input and its block partials in buffers that the context
// grows on demand with cudaMalloc.  Some callers cannot let a library allocate: code whose device
// memory is fully reserved up front by a memory pool or another framework's caching allocator
// (a cudaMalloc there fails, or takes memory the pool counted on), and loops that sample the beam
// every few turns, where a cudaMalloc/cudaFree pair can synchronise the device and stall the
// tracking pipeline.
// accel_beam_stat_noalloc serves them: it reads the caller's array in place (either layout), keeps
// its partial sums in the fixed device array below, and writes the result to a caller-provided
// device buffer.  The cost is a hard capacity and one shared scratch per device.
//
// Scratch contents.  Every cell a call reads is written earlier in the same call, so nothing in
// the scratch has to start at zero and nothing is left for the next call.
//
// Moments follow calc_beam_stat (utility.cpp:387-438): particles whose x is NaN are lost and left
// out; the means, the rms sizes sqrt(<d_k^2>) and the six cross moments <xx'>, <yy'>, <x dp>,
// <x' dp>, <y z>, <y' z> about the means, and the live count.  Like calc_beam_stat and
// accel_beam_stat, the moments are divided by the live count, so with every particle lost they
// are NaN (0/0) and the count is 0.  The sums run in two passes (means,
// then centred second moments) over fixed blocks of 1024 particles, so a given N always adds in
// the same order and the result is reproducible bit for bit from call to call.
#include <cuda_runtime.h>
#include <cstdint>
#include <mutex>
#include <string>
#include "accel_gpu.h"
#include "engine.h"

namespace {

constexpr int kThreads = 256;
constexpr int kPerBlock = kThreads * 4;  // particles one block sums
constexpr int kMaxBlocks = ACCEL_NOALLOC_STAT_MAX_N / kPerBlock;
static_assert(kMaxBlocks * kPerBlock == ACCEL_NOALLOC_STAT_MAX_N, "capacity is whole blocks");
// per block: 7 first-pass sums (6 coordinates + count), then 12 second-pass sums; 32 totals
constexpr int kScratchDoubles = 12 * kMaxBlocks + 32;

// 12 * 4096 + 32 doubles = 393,472 bytes on each device that loads this library
static __device__ __align__(256) double g_stat_scratch[kScratchDoubles];

constexpr unsigned kFull = 0xffffffffu;

template <int LAYOUT>
__device__ __forceinline__ double coord(const double* r, int64_t n, int64_t i, int k) {
    return LAYOUT == ACCEL_LAYOUT_AOS ? r[6 * i + k] : r[k * n + i];
}

template <int K>
__device__ __forceinline__ void block_reduce(double (&v)[K], double* out) {
    __shared__ double sh[kThreads / 32][K];
#pragma unroll
    for (int k = 0; k < K; k++)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(kFull, v[k], o);
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < K; k++) sh[w][k] = v[k];
    __syncthreads();
    if (threadIdx.x < K) {
        double s = 0;
        for (int j = 0; j < kThreads / 32; j++) s += sh[j][threadIdx.x];
        out[threadIdx.x] = s;
    }
}

// pass 1: block b sums particles [b * 1024, (b + 1) * 1024)
template <int LAYOUT>
__global__ void __launch_bounds__(kThreads) k_na_sum1(const double* r, int64_t n, double* part) {
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    const int64_t base = (int64_t)blockIdx.x * kPerBlock;
    for (int j = threadIdx.x; j < kPerBlock; j += kThreads) {
        const int64_t i = base + j;
        if (i >= n) break;
        const double x = coord<LAYOUT>(r, n, i, 0);
        if (x != x) continue;
        v[0] += x;
        for (int k = 1; k < 6; k++) v[k] += coord<LAYOUT>(r, n, i, k);
        v[6] += 1.0;
    }
    block_reduce<7>(v, part + 7 * blockIdx.x);
}

// totals over blocks, in block order (one warp, one lane per quantity)
__global__ void k_na_total(const double* part, int nblk, int K, double* out) {
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        double s = 0;
        for (int b = 0; b < nblk; b++) s += part[K * b + k];
        out[k] = s;
    }
}

// pass 2: centred second moments about the pass-1 means
template <int LAYOUT>
__global__ void __launch_bounds__(kThreads) k_na_sum2(const double* r, int64_t n, const double* s1, double* part) {
    double v[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    const double cnt = s1[6];
    double m[6];
    for (int k = 0; k < 6; k++) m[k] = cnt > 0 ? s1[k] / cnt : 0.0;
    const int64_t base = (int64_t)blockIdx.x * kPerBlock;
    for (int j = threadIdx.x; j < kPerBlock; j += kThreads) {
        const int64_t i = base + j;
        if (i >= n) break;
        const double x = coord<LAYOUT>(r, n, i, 0);
        if (x != x) continue;
        double d[6];
        d[0] = x - m[0];
        for (int k = 1; k < 6; k++) d[k] = coord<LAYOUT>(r, n, i, k) - m[k];
        for (int k = 0; k < 6; k++) v[k] += d[k] * d[k];
        v[6] += d[0] * d[1]; v[7] += d[2] * d[3]; v[8] += d[0] * d[5];
        v[9] += d[1] * d[5]; v[10] += d[2] * d[4]; v[11] += d[3] * d[4];
    }
    block_reduce<12>(v, part + 12 * blockIdx.x);
}

__global__ void k_na_out(const double* s1, const double* s2, double* out) {
    if (threadIdx.x != 0) return;
    const double c = s1[6];  // 0 when every particle is lost: the moments come out NaN
    for (int k = 0; k < 6; k++) {
        out[k] = s1[k] / c;
        out[6 + k] = sqrt(s2[k] / c);
        out[12 + k] = s2[6 + k] / c;
    }
    out[18] = c;
}

// Set-up per device: the scratch's device address, and every kernel of this file loaded, so
// that later calls only launch.  Done on a device's first call and kept once it succeeds; a
// failed set-up is retried by the next call on that device.
constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
double* g_scratch[kMaxDevices];  // non-null once the device's set-up succeeded

cudaError_t setup_device(int dev) {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (g_scratch[dev]) return cudaSuccess;
    double* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&p, g_stat_scratch);
    cudaFuncAttributes fa;
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_na_sum1<ACCEL_LAYOUT_AOS>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_na_sum1<ACCEL_LAYOUT_SOA>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_na_sum2<ACCEL_LAYOUT_AOS>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_na_sum2<ACCEL_LAYOUT_SOA>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_na_total);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_na_out);
    if (e != cudaSuccess) {
        cudaGetLastError();  // this set-up's own error; the next call tries again
        return e;
    }
    g_scratch[dev] = p;
    return cudaSuccess;
}

bool on_device(const void* p, int* dev) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) return false;
    *dev = a.device;
    return true;
}

template <int LAYOUT>
void launch(const double* r, int64_t n, int nblk, double* scratch, double* out, cudaStream_t s) {
    double* part = scratch;                  // 12 * nblk (pass 1 uses the first 7 * nblk)
    double* s1 = scratch + 12 * kMaxBlocks;  // 8 totals of pass 1
    double* s2 = s1 + 8;                     // 12 totals of pass 2
    k_na_sum1<LAYOUT><<<nblk, kThreads, 0, s>>>(r, n, part);
    k_na_total<<<1, 32, 0, s>>>(part, nblk, 7, s1);
    k_na_sum2<LAYOUT><<<nblk, kThreads, 0, s>>>(r, n, s1, part);
    k_na_total<<<1, 32, 0, s>>>(part, nblk, 12, s2);
    k_na_out<<<1, 32, 0, s>>>(s1, s2, out);
}

}  // namespace

extern "C" int accel_beam_stat_noalloc(const double* r, int layout, int64_t N, double* out, void* stream) {
    using accel::fail;
    if (!r || !out) return fail(ACCEL_E_INVALID, "accel_beam_stat_noalloc: r and out must be device pointers");
    if (layout != ACCEL_LAYOUT_AOS && layout != ACCEL_LAYOUT_SOA)
        return fail(ACCEL_E_INVALID, "accel_beam_stat_noalloc: layout must be ACCEL_LAYOUT_AOS or ACCEL_LAYOUT_SOA");
    if (N <= 0) return fail(ACCEL_E_INVALID, "accel_beam_stat_noalloc: N must be positive");
    if (N > ACCEL_NOALLOC_STAT_MAX_N)
        return fail(ACCEL_E_TOO_LARGE, "accel_beam_stat_noalloc: N = " + std::to_string(N) + " exceeds the " +
                                           std::to_string(ACCEL_NOALLOC_STAT_MAX_N) +
                                           " particles its fixed scratch holds; use accel_beam_stat");
    int dev = -1, dev_out = -1;
    if (!on_device(r, &dev)) return fail(ACCEL_E_INVALID, "accel_beam_stat_noalloc: r is not device memory");
    if (!on_device(out, &dev_out) || dev_out != dev)
        return fail(ACCEL_E_INVALID, "accel_beam_stat_noalloc: out is not device memory on the device of r");
    if (dev < 0 || dev >= kMaxDevices) return fail(ACCEL_E_INVALID, "accel_beam_stat_noalloc: device index out of range");
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) {
        cudaGetLastError();
        return fail(ACCEL_E_CUDA, "accel_beam_stat_noalloc: cudaGetDevice failed");
    }
    if (prev != dev && cudaSetDevice(dev) != cudaSuccess) {
        cudaGetLastError();
        return fail(ACCEL_E_CUDA, "accel_beam_stat_noalloc: cudaSetDevice failed");
    }
    int status = ACCEL_OK;
    const cudaError_t pending = cudaPeekAtLastError();  // left by earlier work; not consumed here
    const cudaError_t se = pending == cudaSuccess ? setup_device(dev) : cudaSuccess;
    if (pending != cudaSuccess) {
        status = fail(ACCEL_E_CUDA, std::string("accel_beam_stat_noalloc: a CUDA error of earlier work is pending (") +
                                        cudaGetErrorString(pending) + "); nothing launched");
    } else if (se != cudaSuccess) {
        status = fail(ACCEL_E_CUDA, std::string("accel_beam_stat_noalloc: set-up (cudaGetSymbolAddress) failed: ") +
                                        cudaGetErrorString(se));
    } else {
        const int nblk = (int)((N + kPerBlock - 1) / kPerBlock);
        cudaStream_t s = (cudaStream_t)stream;
        if (layout == ACCEL_LAYOUT_AOS) launch<ACCEL_LAYOUT_AOS>(r, N, nblk, g_scratch[dev], out, s);
        else launch<ACCEL_LAYOUT_SOA>(r, N, nblk, g_scratch[dev], out, s);
        cudaError_t e = cudaGetLastError();  // no error was pending before these launches
        if (e != cudaSuccess)
            status = fail(ACCEL_E_CUDA, std::string("accel_beam_stat_noalloc: launch failed: ") + cudaGetErrorString(e));
    }
    if (prev != dev) cudaSetDevice(prev);
    return status;
}
