// common.cuh -- shared definitions of the sm_100a Monte Carlo engine.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pc {

// Per-sublattice bond table. A site of sublattice `sl` in cell (cx,cy,cz) has
// neighbours nb[e] = (cell + (dx,dy,dz) wrapped, sublattice nb[e].sl), grouped
// into shells [shell_end[k-1], shell_end[k]) that share one 3x3 matrix J[k]
// (row-major): h = sum_k J[k] * sum_{e in shell k} S_nb(e). This is the
// structured form of the reference's per-spin BondShell lists
// (include/MC.hpp:38-41, src/MC.cpp:15-52): same shells, same matrices, with
// index arithmetic in place of pointers.
constexpr int kMaxShell = 16;
constexpr int kMaxNb = 64;

struct NbEntry {
    int8_t dx, dy, dz;
    uint8_t sl;
};

struct SlTable {
    int32_t n_shell;
    int32_t n_nb;
    int32_t shell_end[kMaxShell];
    int32_t shell_spec[kMaxShell];  // coupling spec index; +1000 if the shell applies J^T
    float J[kMaxShell][9];
    NbEntry nb[kMaxNb];
};

// A tile is a run of up to `count` consecutive cells of one sublattice of one
// replica: x = replica, y = (slot of the sublattice in the colour's table list
// << 8) | sublattice, z = first cell, w = count.
using Tile = int4;

struct ReplicaDev {
    int32_t L;
    int32_t Nc;
    int64_t off;    // offset of the replica's spins in the global float4 array
    uint64_t divL;  // fast-division magic for L (pyro_struct.cuh)
};

// ---------------------------------------------------------------- Philox
// Philox4x32-10 (Salmon et al., SC'11): 10 rounds of the two multiply/xor
// S-boxes with a Weyl-sequence key schedule.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k.x += 0x9E3779B9u;
            k.y += 0xBB67AE85u;
        }
        const uint32_t lo0 = 0xD2511F53u * c.x;
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    }
    return c;
}

// Counter layout shared with the host documentation (include/pyrocmc.h).
__device__ __forceinline__ uint4 site_draw(uint64_t seed, uint32_t replica, uint64_t sweep, uint32_t draw,
                                           uint32_t site) {
    return philox4x32_10(make_uint4(site, uint32_t(sweep), draw | (uint32_t(sweep >> 32) << 8), replica),
                         make_uint2(uint32_t(seed), uint32_t(seed >> 32)));
}

// The ten round keys of the Weyl schedule for a 64-bit seed (round r:
// seed + r x (0x9E3779B9, 0xBB67AE85) per 32-bit half), formed once on the
// host: kernels that take them as parameters read each round's key as an
// operand instead of adding the schedule constants per site.
struct PhiloxKeys {
    uint2 k[10];
};
inline PhiloxKeys philox_round_keys(uint64_t seed) {
    PhiloxKeys rk;
    uint32_t kx = uint32_t(seed), ky = uint32_t(seed >> 32);
    for (int r = 0; r < 10; ++r) {
        rk.k[r] = make_uint2(kx, ky);
        kx += 0x9E3779B9u;
        ky += 0xBB67AE85u;
    }
    return rk;
}
// philox4x32_10 with the round keys given (same output)
__device__ __forceinline__ uint4 philox4x32_10_rk(uint4 c, const PhiloxKeys& rk) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c.x;
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ rk.k[r].x, lo1, hi0 ^ c.w ^ rk.k[r].y, lo0);
    }
    return c;
}
__device__ __forceinline__ uint4 site_draw_rk(const PhiloxKeys& rk, uint32_t replica, uint64_t sweep, uint32_t draw,
                                              uint32_t site) {
    return philox4x32_10_rk(make_uint4(site, uint32_t(sweep), draw | (uint32_t(sweep >> 32) << 8), replica), rk);
}

__device__ __forceinline__ float u24_open0(uint32_t x) { return float((x >> 8) + 1u) * (1.0f / 16777216.0f); }
__device__ __forceinline__ float u24(uint32_t x) { return float(x >> 8) * (1.0f / 16777216.0f); }
__device__ __forceinline__ float u24_lowbytes(uint4 w) {
    return float((w.x & 0xffu) | ((w.y & 0xffu) << 8) | ((w.z & 0xffu) << 16)) * (1.0f / 16777216.0f);
}

constexpr uint32_t kDrawMetropolis = 0;
constexpr uint32_t kDrawLifted = 1;  // lifted Metropolis: Exp(1) from word 0, acceptance uniform from word 1
constexpr uint32_t kDrawOverrelax0 = 2;
constexpr uint32_t kDrawInit = 250;
constexpr uint32_t kDrawExchange = 251;

// Wrap a cell coordinate that is at most one period outside [0, L).
__device__ __forceinline__ int wrap1(int x, int L) {
    x += (x < 0) ? L : 0;
    x -= (x >= L) ? L : 0;
    return x;
}

}  // namespace pc
