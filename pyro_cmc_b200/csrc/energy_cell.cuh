// energy_cell.cuh -- the energy of one cubic cell with each bond counted once
// (total_energy_per_unit_cell, src/MC.cpp:305-312): the device code shared by
// energy_cell_kernel (energy_cell.cu) and the energy phase of the persistent
// tempering kernel (pt_persistent.cu).
//
// The reference sums 0.5 S_i.h_i - S_i.B over sites, i.e. every bond twice
// from its two ends. Here every bond is counted once, by one of its ends: a
// thread owns the 16 sites of one cubic cell and the bonds from them whose cell
// offset to the other end is "forward" (dz > 0; else dy > 0; else dx > 0; a
// bond inside the cell belongs to its lower sublattice). The matrix seen from
// the other end is the transpose, so the bond energy S_i.J S_j is the same
// from either end and the sum equals the reference's.
//
// Why per cell: of the 240 bonds a cell owns, 78 join two of its own sites
// (read once, kept in registers) and the other 162 reach only 48 distinct
// sites of neighbouring cells (pyro_struct.cuh's offsets: 9 forward cell
// offsets with 4 or 8 target sublattices each). A cell therefore issues 16 + 48
// coalesced float4 loads instead of the 16 x 16 of a per-site thread that
// gathers its neighbours on higher sublattices. Consecutive threads take
// consecutive cells along x, so every load of a warp is a 512-byte row segment.
//
// Bond energies accumulate in FP32 (as the per-site local field of the other
// kernels is FP32): four sums per cell, each bond's S_i.S_j times its j; or,
// when every group's j is the same on all 16 sublattices (`uniform`: the
// pyrochlore J1-J2-J3 model with isotropic couplings), one sum of bare
// S_i.S_j per group (three multiply-adds a bond), multiplied by the group's j
// once per cell. The Zeeman and magnetisation terms use the cell's summed
// spin; everything above the cell is FP64.
#pragma once
#include <cuda_runtime.h>

#include <utility>

#include "common.cuh"
#include "kernels.h"
#include "struct_field.cuh"

namespace pc {


__host__ __device__ constexpr bool bond_owned(int sl, int e) {
    const int dx = nb_dx(sl, e), dy = nb_dy(sl, e), dz = nb_dz(sl, e);
    if (dz != 0) return dz > 0;
    if (dy != 0) return dy > 0;
    if (dx != 0) return dx > 0;
    return sl < nb_sl(sl, e);
}

constexpr int kMaxIntra = 128;
constexpr int kMaxTargets = 64;
constexpr int kMaxRemote = 256;

struct CellBonds {
    int n_intra;
    int isl[kMaxIntra], is2[kMaxIntra], ig[kMaxIntra];  // own site, other own site, group (of isl)
    int n_tgt;
    int ts2[kMaxTargets], tdx[kMaxTargets], tdy[kMaxTargets], tdz[kMaxTargets];
    int tb[kMaxTargets + 1];  // bonds of target t: [tb[t], tb[t+1]) of the remote list
    int n_rem;
    int rsl[kMaxRemote], rg[kMaxRemote];  // own site and group of each remote bond
};

__host__ __device__ constexpr int target_key(int s2, int dx, int dy, int dz) {
    return (((dz + 1) * 3 + (dy + 1)) * 3 + (dx + 1)) * 16 + s2;
}

__host__ __device__ constexpr CellBonds make_cell_bonds() {
    CellBonds b{};
    int key[kMaxRemote] = {};
    // intra-cell bonds in (sl, e) order; remote bonds collected with their key
    for (int sl = 0; sl < 16; ++sl)
        for (int e = 0; e < kStructNb; ++e) {
            if (!bond_owned(sl, e)) continue;
            const int dx = nb_dx(sl, e), dy = nb_dy(sl, e), dz = nb_dz(sl, e);
            const int g = group_of(sl, e);
            if (dx == 0 && dy == 0 && dz == 0) {
                b.isl[b.n_intra] = sl;
                b.is2[b.n_intra] = nb_sl(sl, e);
                b.ig[b.n_intra] = g;
                ++b.n_intra;
            } else {
                key[b.n_rem] = target_key(nb_sl(sl, e), dx, dy, dz);
                b.rsl[b.n_rem] = sl;
                b.rg[b.n_rem] = g;
                ++b.n_rem;
            }
        }
    // stable insertion sort of the remote bonds by target: increasing
    // (dz, dy, dx, s2), and (sl, e) order inside one target
    for (int i = 1; i < b.n_rem; ++i) {
        const int k = key[i], sl = b.rsl[i], g = b.rg[i];
        int j = i - 1;
        while (j >= 0 && key[j] > k) {
            key[j + 1] = key[j];
            b.rsl[j + 1] = b.rsl[j];
            b.rg[j + 1] = b.rg[j];
            --j;
        }
        key[j + 1] = k;
        b.rsl[j + 1] = sl;
        b.rg[j + 1] = g;
    }
    for (int i = 0; i < b.n_rem; ++i)
        if (i == 0 || key[i] != key[i - 1]) {
            const int k = key[i];
            b.ts2[b.n_tgt] = k % 16;
            b.tdx[b.n_tgt] = (k / 16) % 3 - 1;
            b.tdy[b.n_tgt] = (k / 48) % 3 - 1;
            b.tdz[b.n_tgt] = k / 144 - 1;
            b.tb[b.n_tgt] = i;
            ++b.n_tgt;
        }
    b.tb[b.n_tgt] = b.n_rem;
    return b;
}

constexpr CellBonds kCB = make_cell_bonds();
static_assert(kCB.n_intra <= kMaxIntra && kCB.n_tgt <= kMaxTargets && kCB.n_rem <= kMaxRemote, "cell bond tables");
static_assert(2 * (kCB.n_intra + kCB.n_rem) == 16 * kStructNb, "every bond owned by exactly one end");

__host__ __device__ constexpr int cb_n_intra() { return kCB.n_intra; }
__host__ __device__ constexpr int cb_n_tgt() { return kCB.n_tgt; }
__host__ __device__ constexpr int cb_isl(int k) { return kCB.isl[k]; }
__host__ __device__ constexpr int cb_is2(int k) { return kCB.is2[k]; }
__host__ __device__ constexpr int cb_ig(int k) { return kCB.ig[k]; }
__host__ __device__ constexpr int cb_ts2(int t) { return kCB.ts2[t]; }
__host__ __device__ constexpr int cb_tdx(int t) { return kCB.tdx[t]; }
__host__ __device__ constexpr int cb_tdy(int t) { return kCB.tdy[t]; }
__host__ __device__ constexpr int cb_tdz(int t) { return kCB.tdz[t]; }
__host__ __device__ constexpr int cb_tb(int t) { return kCB.tb[t]; }
__host__ __device__ constexpr int cb_rsl(int k) { return kCB.rsl[k]; }
__host__ __device__ constexpr int cb_rg(int k) { return kCB.rg[k]; }

// Bond energies accumulate in kAcc FP32 sums per cell: site sl into sum
// sl % 4 (fewer live registers than one sum per site), or group G into sum G
// (UNI).
constexpr int kAcc = kGroups;
static_assert(kAcc >= 4, "per-site sums use four accumulators");

// acc += S_SL . M[SL][G] n  (ISO: M = j I; ISO 2: the J2 group is zero and
// skipped); UNI: acc[G] += S_SL . n, the group's j applied per cell
template <int SL, int G, int ISO, bool UNI>
__device__ __forceinline__ void bond_term(float (&acc)[kAcc], const float3 (&own)[16], const float3& n,
                                          const PyroMats& mats) {
    if constexpr (ISO == 2 && G == 3) {
        return;
    } else if constexpr (UNI) {
        acc[G] = fmaf(own[SL].z, n.z, fmaf(own[SL].y, n.y, fmaf(own[SL].x, n.x, acc[G])));
    } else if constexpr (ISO != 0) {
        const float d = own[SL].x * n.x + own[SL].y * n.y + own[SL].z * n.z;
        acc[SL % 4] = fmaf(mats.M[SL][G][0], d, acc[SL % 4]);
    } else {
        const float* J = mats.M[SL][G];
        const float tx = J[0] * n.x + J[1] * n.y + J[2] * n.z;
        const float ty = J[3] * n.x + J[4] * n.y + J[5] * n.z;
        const float tz = J[6] * n.x + J[7] * n.y + J[8] * n.z;
        acc[SL % 4] += own[SL].x * tx + own[SL].y * ty + own[SL].z * tz;
    }
}

template <int ISO, bool UNI, int... K>
__device__ __forceinline__ void intra_bonds(float (&acc)[kAcc], const float3 (&own)[16], const PyroMats& mats,
                                            std::integer_sequence<int, K...>) {
    (bond_term<cb_isl(K), cb_ig(K), ISO, UNI>(acc, own, own[cb_is2(K)], mats), ...);
}

template <int T, int ISO, bool UNI, int... K>
__device__ __forceinline__ void target_bonds(float (&acc)[kAcc], const float3 (&own)[16], const float3& n,
                                             const PyroMats& mats, std::integer_sequence<int, K...>) {
    (bond_term<cb_rsl(cb_tb(T) + K), cb_rg(cb_tb(T) + K), ISO, UNI>(acc, own, n, mats), ...);
}

template <int T, bool NC>
__device__ __forceinline__ float3 load_target(const char* base, uint32_t sl_bytes, const Coords& c) {
    const uint32_t off = uint32_t(cb_ts2(T)) * sl_bytes + uint32_t(pick<cb_tdx(T)>(c.x)) +
                         uint32_t(pick<cb_tdy(T)>(c.y)) + uint32_t(pick<cb_tdz(T)>(c.z));
    const float4 v = load_spin<NC>(reinterpret_cast<const float4*>(base + off));
    return make_float3(v.x, v.y, v.z);
}

// Targets [T0, T0 + sizeof...(K)) loaded together (one round trip), then their bonds.
template <int T0, int ISO, bool UNI, bool NC, int... K>
__device__ __forceinline__ void target_batch(float (&acc)[kAcc], const float3 (&own)[16], const char* base,
                                             uint32_t sl_bytes, const Coords& c, const PyroMats& mats,
                                             std::integer_sequence<int, K...>) {
    const float3 n[sizeof...(K)] = {load_target<T0 + K, NC>(base, sl_bytes, c)...};
    (target_bonds<T0 + K, ISO, UNI>(acc, own, n[K], mats,
                               std::make_integer_sequence<int, cb_tb(T0 + K + 1) - cb_tb(T0 + K)>{}),
     ...);
}

// Targets loaded together per batch. With 4 (and 5 resident blocks of 128:
// 96 registers, a few spilled to L1) the L = 64 energy takes 28 us against 33
// with 8 targets and 3 blocks (168 registers, no spills): more warps in flight
// hide more of the gather latency than the spills cost (same sums either way).
constexpr int kTargetBatch = 4;

template <int T0, int ISO, bool UNI, bool NC>
__device__ __forceinline__ void remote_bonds(float (&acc)[kAcc], const float3 (&own)[16], const char* base,
                                             uint32_t sl_bytes, const Coords& c, const PyroMats& mats) {
    if constexpr (T0 < cb_n_tgt()) {
        constexpr int n = (cb_n_tgt() - T0) < kTargetBatch ? (cb_n_tgt() - T0) : kTargetBatch;
        target_batch<T0, ISO, UNI, NC>(acc, own, base, sl_bytes, c, mats, std::make_integer_sequence<int, n>{});
        remote_bonds<T0 + n, ISO, UNI, NC>(acc, own, base, sl_bytes, c, mats);
    }
}

template <bool NC, int... SL>
__device__ __forceinline__ void load_own(float3 (&own)[16], const char* base, uint32_t sl_bytes, const Coords& c,
                                         std::integer_sequence<int, SL...>) {
    const float4 v[16] = {load_spin<NC>(reinterpret_cast<const float4*>(base + uint32_t(SL) * sl_bytes +
                                                                        uint32_t(c.x[1]) + uint32_t(c.y[1]) +
                                                                        uint32_t(c.z[1])))...};
    ((own[SL] = make_float3(v[SL].x, v[SL].y, v[SL].z)), ...);
}

// The cubic cell at coordinates c of the lattice whose spins start at base
// (sublattice stride sl_bytes): v[0] = its owned bond energies - S.B, v[1..3]
// = its summed spin; GROUPS (with UNI): gs[G] = its bare sum of S_i.S_j over
// the owned bonds of group G. NC: loads through the read-only path (the
// stand-alone kernel); false: coherent weak loads (the persistent kernel,
// whose earlier phases wrote the spins).
template <int ISO, bool UNI, bool NC, bool GROUPS = false>
__device__ __forceinline__ void cell_energy(double (&v)[4], const char* base, uint32_t sl_bytes, const Coords& c,
                                            const PyroMats& mats, const float* B, double* gs = nullptr) {
    static_assert(!GROUPS || UNI, "group sums come from the per-group accumulators");
    float3 own[16];
    load_own<NC>(own, base, sl_bytes, c, std::make_integer_sequence<int, 16>{});
    float acc[kAcc];
#pragma unroll
    for (int k = 0; k < kAcc; ++k) acc[k] = 0.f;
    intra_bonds<ISO, UNI>(acc, own, mats, std::make_integer_sequence<int, cb_n_intra()>{});
    remote_bonds<0, ISO, UNI, NC>(acc, own, base, sl_bytes, c, mats);
#pragma unroll
    for (int k = 0; k < (UNI ? kAcc : 4); ++k) v[0] += UNI ? double(mats.M[0][k][0]) * double(acc[k]) : double(acc[k]);
    if constexpr (GROUPS) {
#pragma unroll
        for (int k = 0; k < kAcc; ++k) gs[k] = double(acc[k]);
    }
    float3 m = own[0];
#pragma unroll
    for (int sl = 1; sl < 16; ++sl) {
        m.x += own[sl].x;
        m.y += own[sl].y;
        m.z += own[sl].z;
    }
    v[0] -= double(fmaf(m.z, B[2], fmaf(m.y, B[1], m.x * B[0])));
    v[1] = double(m.x);
    v[2] = double(m.y);
    v[3] = double(m.z);
}

}  // namespace pc
