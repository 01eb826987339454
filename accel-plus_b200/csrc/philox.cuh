// philox.cuh — counter-based normal deviates for quantum excitation.
//
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC'11): ten rounds of two 32x32->64 multiplies with the published multipliers and Weyl key
// increments.  The counter is (particle id, turn, element, kick) and the key is the 64-bit seed,
// so every kick's deviate is a pure function of where it happens: no state, no ordering
// dependence, identical under any launch shape or compaction order.  Two 53-bit uniforms from the
// four outputs give one Box-Muller pair.  The reference draws its deviates from rand() through a
// shared static Box-Muller (utility.cpp:194-217); parity for these runs is statistical.
#pragma once
#include <cstdint>

namespace accel {

struct Philox4 { uint32_t x[4]; };

__host__ __device__ __forceinline__ void philox_round(uint32_t c[4], const uint32_t k[2]) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    uint64_t p0 = (uint64_t)M0 * c[0];
    uint64_t p1 = (uint64_t)M1 * c[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c[1] ^ k[0];
    uint32_t n1 = lo1;
    uint32_t n2 = hi0 ^ c[3] ^ k[1];
    uint32_t n3 = lo0;
    c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
}

__host__ __device__ __forceinline__ Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2,
                                                          uint32_t c3, uint64_t key) {
    uint32_t c[4] = {c0, c1, c2, c3};
    uint32_t k[2] = {(uint32_t)key, (uint32_t)(key >> 32)};
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; r++) {
        philox_round(c, k);
        k[0] += W0;
        k[1] += W1;
    }
    Philox4 o;
    o.x[0] = c[0]; o.x[1] = c[1]; o.x[2] = c[2]; o.x[3] = c[3];
    return o;
}

// Uniform in (0, 1): 53 random bits, offset by half an ulp so log() never sees zero.
__host__ __device__ __forceinline__ double u53(uint32_t hi, uint32_t lo) {
    uint64_t v = ((uint64_t)hi << 21) ^ (uint64_t)lo;
    v &= ((1ull << 53) - 1);
    return ((double)v + 0.5) * (1.0 / 9007199254740992.0);
}

// One standard normal for (particle, turn, element, kick).
__device__ __forceinline__ double qe_normal(uint64_t seed, uint32_t pid, uint32_t turn,
                                            uint32_t elem, uint32_t kick) {
    Philox4 o = philox4x32_10(pid, turn, elem, kick, seed);
    double u1 = u53(o.x[0], o.x[1]);
    double u2 = u53(o.x[2], o.x[3]);
    double rad = sqrt(-2.0 * log(u1));
    return rad * cospi(2.0 * u2);
}

}  // namespace accel
