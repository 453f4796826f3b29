// struct_field.cuh -- the local field of a site through the compile-time
// pyrochlore neighbour structure (pyro_struct.cuh), shared by the kernels that
// use the structured path.
#pragma once

#include <cuda_runtime.h>

#include <utility>

#include "common.cuh"
#include "pyro_struct.cuh"

namespace pc {

// Structured local field (compile-time neighbour offsets of sublattice SL,
// pyro_struct.cuh): the wrapped neighbour coordinates are formed once, each
// of the 30 neighbours is one add-and-load with offsets fixed at compile time,
// groups with a zero matrix are skipped. Same sum as local_field() with the
// shells grouped per target.
// Byte offsets of the wrapped cx-1, cx, cx+1 (times 16), of the rows
// L(cy-1), L cy, L(cy+1) and of the planes L^2(cz-1), L^2 cz, L^2(cz+1): a
// neighbour's address is the replica's base plus one unsigned 32-bit sum
// (spins of one replica span far less than 4 GB), which costs fewer integer
// instructions than 64-bit element indexing (measured 5 % per colour pass).
struct Coords {
    int x[3], y[3], z[3];
};

template <int D>
__device__ __forceinline__ int pick(const int (&v)[3]) {
    if constexpr (D < 0)
        return v[0];
    else if constexpr (D > 0)
        return v[2];
    else
        return v[1];
}

// NC: the spins are read-only for the whole kernel (a colour pass reads other
// sublattices than it writes), so loads may use the non-coherent read-only
// path (__ldg). A kernel that also writes the spins it gathers in a later
// phase (the persistent tempering kernel: colour passes separated by grid
// barriers) loads with NC = false: ordinary weak loads (ld.global.ca), which
// keep the L1 hits of neighbouring threads inside a phase; the grid barrier's
// gpu-scope fences order them after the other blocks' writes of the earlier
// phases (PTX memory model: fence, flag, fence message passing).
template <bool NC>
__device__ __forceinline__ float4 load_spin(const float4* p) {
    if constexpr (NC)
        return __ldg(p);
    else
        return __ldca(p);
}

// h += J t for a general 3x3 group matrix J (row-major), with every rounding
// fixed: h_a = fma(J[3a+2], t.z, fma(J[3a+1], t.y, fma(J[3a], t.x, h_a))).
// Left to the compiler, the contraction of the plain expression into FMAs may
// differ between the kernels that inline it, and the chains of the per-pass,
// persistent, staged and cluster-resident sweeps would part at the first
// decision the last bit changes. For J = j I the two outer terms add exact
// zeros, so the result is fma(j, t_a, h_a): the bits of add_group_iso.
__device__ __forceinline__ void add_matvec(float3& h, const float* J, const float3& t) {
    h.x = fmaf(J[2], t.z, fmaf(J[1], t.y, fmaf(J[0], t.x, h.x)));
    h.y = fmaf(J[5], t.z, fmaf(J[4], t.y, fmaf(J[3], t.x, h.y)));
    h.z = fmaf(J[8], t.z, fmaf(J[7], t.y, fmaf(J[6], t.x, h.z)));
}

// UB: the neighbour's address as the base of its sublattice (the same for
// every thread of a tile, so the compiler keeps the bases in uniform
// registers) plus its cell's byte offset, one vector add per load instead of a
// full offset sum. The same address either way; which form is faster depends
// on the kernel (the fused isotropic colour pass at L = 64: 10.03 -> 9.83 us
// with it, 72 registers and still 7 blocks; the Metropolis-only pass goes to
// 74 registers and 6 blocks, the register-capped persistent kernel spills).
template <int SL, int E, bool NC = true, bool UB = false>
__device__ __forceinline__ float4 load_nb(const float4* __restrict__ S, int Nc, const Coords& c) {
    constexpr int s2 = nb_sl(SL, E), dx = nb_dx(SL, E), dy = nb_dy(SL, E), dz = nb_dz(SL, E);
    if constexpr (UB) {
        const uint32_t xyz = uint32_t(pick<dx>(c.x)) + uint32_t(pick<dy>(c.y)) + uint32_t(pick<dz>(c.z));
        const char* base = reinterpret_cast<const char*>(S) + uint32_t(s2) * (uint32_t(Nc) << 4);
        return load_spin<NC>(reinterpret_cast<const float4*>(base + xyz));
    } else {
        const uint32_t off = uint32_t(s2) * (uint32_t(Nc) << 4) + uint32_t(pick<dx>(c.x)) + uint32_t(pick<dy>(c.y)) +
                             uint32_t(pick<dz>(c.z));
        return load_spin<NC>(reinterpret_cast<const float4*>(reinterpret_cast<const char*>(S) + off));
    }
}

template <int SL, int G, bool NC, bool UB, int... K>
__device__ __forceinline__ float3 group_sum(const float4* __restrict__ S, int Nc, const Coords& c,
                                            std::integer_sequence<int, K...>) {
    constexpr int B = grp_begin(SL, G);
    const float4 v[sizeof...(K)] = {load_nb<SL, B + K, NC, UB>(S, Nc, c)...};
    float3 t = make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int k = 0; k < int(sizeof...(K)); ++k) {
        t.x += v[k].x;
        t.y += v[k].y;
        t.z += v[k].z;
    }
    return t;
}

template <int SL, int G, bool NC = true>
__device__ __forceinline__ void add_group(float3& h, const float4* __restrict__ S, int Nc, const Coords& c,
                                          const PyroMats& mats) {
    if (mats.active[SL] & (1u << G)) {
        const float3 t = group_sum<SL, G, NC, false>(S, Nc, c, std::make_integer_sequence<int, grp_size(SL, G)>{});
        const float* J = mats.M[SL][G];
        add_matvec(h, J, t);
    }
}

// add_group for a group whose matrix is j I, j != 0 (every group of a system
// with nonzero isotropic couplings: J2, J3, and J1 with Delta = 1): three
// multiply-adds instead of nine, and no test of the group's activity.
// add_group gives the same bits on such a matrix (add_matvec: its two zero
// terms add exact zeros to fma(j, t, h)).
template <int SL, int G, bool NC = true, bool UB = false>
__device__ __forceinline__ void add_group_iso(float3& h, const float4* __restrict__ S, int Nc, const Coords& c,
                                              const PyroMats& mats) {
    const float3 t = group_sum<SL, G, NC, UB>(S, Nc, c, std::make_integer_sequence<int, grp_size(SL, G)>{});
    const float j = mats.M[SL][G][0];
    h.x = fmaf(j, t.x, h.x);
    h.y = fmaf(j, t.y, h.y);
    h.z = fmaf(j, t.z, h.z);
}

__device__ __forceinline__ Coords cell_coords(int cell, int L, uint64_t divL) {
    const int q = fdiv(cell, divL);  // cy + L*cz
    const int cx = cell - q * L;
    const int cz = fdiv(q, divL);
    const int cy = q - cz * L;
    const int L16 = L << 4, LL16 = L * L16;
    Coords c;
    c.x[0] = (cx == 0 ? L - 1 : cx - 1) << 4;
    c.x[1] = cx << 4;
    c.x[2] = (cx == L - 1 ? 0 : cx + 1) << 4;
    c.y[0] = L16 * (cy == 0 ? L - 1 : cy - 1);
    c.y[1] = L16 * cy;
    c.y[2] = L16 * (cy == L - 1 ? 0 : cy + 1);
    c.z[0] = LL16 * (cz == 0 ? L - 1 : cz - 1);
    c.z[1] = LL16 * cz;
    c.z[2] = LL16 * (cz == L - 1 ? 0 : cz + 1);
    return c;
}

// All 30 neighbour loads issued at once (a group with a zero matrix loads
// nothing: the loads are predicated, not branched around), so one memory round
// trip covers the whole site instead of one per group.
template <int SL, int OFF, int... E>
__device__ __forceinline__ void load_range(float4 (&v)[kStructNb], const float4* __restrict__ S, int Nc,
                                           const Coords& c, uint32_t act, std::integer_sequence<int, E...>) {
    ((v[OFF + E] = (act & (1u << group_of(SL, OFF + E))) ? load_nb<SL, OFF + E>(S, Nc, c)
                                                          : make_float4(0.f, 0.f, 0.f, 0.f)),
     ...);
}
// neighbours [B, E) of sublattice SL into v[B..E)
template <int SL, int B, int E>
__device__ __forceinline__ void load_nbs(float4 (&v)[kStructNb], const float4* __restrict__ S, int Nc, const Coords& c,
                                         uint32_t act) {
    load_range<SL, B>(v, S, Nc, c, act, std::make_integer_sequence<int, E - B>{});
}

template <int SL, int G>
__device__ __forceinline__ void add_group_v(float3& h, const float4 (&v)[kStructNb], const PyroMats& mats) {
    constexpr int B = grp_begin(SL, G), E = grp_begin(SL, G + 1);
    float3 t = make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int k = B; k < E; ++k) {
        t.x += v[k].x;
        t.y += v[k].y;
        t.z += v[k].z;
    }
    const float* J = mats.M[SL][G];
    add_matvec(h, J, t);
}

// h += sum of the group matrices times the group sums, groups [G0, G1)
template <int SL, int G0, int G1>
__device__ __forceinline__ void field_groups(float3& h, const float4 (&v)[kStructNb], const PyroMats& mats) {
    if constexpr (G0 < G1) {
        add_group_v<SL, G0>(h, v, mats);
        field_groups<SL, G0 + 1, G1>(h, v, mats);
    }
}

// Each bond once: the field of site i of sublattice SL restricted to the
// neighbours on higher sublattices, h+_i = sum_G M_G sum_{e in G, s2 > SL} S_e.
// Since the matrix seen from the other end is the transpose, the energy
// 0.5 sum_i S_i.h_i equals sum_i S_i.h+_i: half the neighbour loads.
template <int SL, int E, bool NC = true>
__device__ __forceinline__ void add_upper(float3& t, const float4* __restrict__ S, int Nc, const Coords& c) {
    if constexpr (nb_sl(SL, E) > SL) {
        const float4 v = load_nb<SL, E, NC>(S, Nc, c);
        t.x += v.x;
        t.y += v.y;
        t.z += v.z;
    }
}
__host__ __device__ constexpr bool group_has_upper(int sl, int g) {
    for (int e = grp_begin(sl, g); e < grp_begin(sl, g + 1); ++e)
        if (nb_sl(sl, e) > sl) return true;
    return false;
}
// ISO 1: every group matrix is j I with j != 0; ISO 2: so but the J2 group
// (group 3), which is 0 and skipped (as add_group_iso: no activity test,
// three multiply-adds per group, the same bits).
template <int SL, int G, int ISO, bool NC, int... K>
__device__ __forceinline__ void add_group_upper(float3& h, const float4* __restrict__ S, int Nc, const Coords& c,
                                                const PyroMats& mats, std::integer_sequence<int, K...>) {
    if constexpr (group_has_upper(SL, G) && !(ISO == 2 && G == 3)) {
        if (ISO || (mats.active[SL] & (1u << G))) {
            constexpr int B = grp_begin(SL, G);
            float3 t = make_float3(0.f, 0.f, 0.f);
            (add_upper<SL, B + K, NC>(t, S, Nc, c), ...);
            const float* J = mats.M[SL][G];
            if constexpr (ISO) {
                h.x = fmaf(J[0], t.x, h.x);
                h.y = fmaf(J[0], t.y, h.y);
                h.z = fmaf(J[0], t.z, h.z);
            } else {
                add_matvec(h, J, t);
            }
        }
    }
}
template <int SL, int G, int ISO, bool NC>
__device__ __forceinline__ void add_group_upper(float3& h, const float4* __restrict__ S, int Nc, const Coords& c,
                                                const PyroMats& mats) {
    add_group_upper<SL, G, ISO, NC>(h, S, Nc, c, mats, std::make_integer_sequence<int, grp_size(SL, G)>{});
}
template <int SL, int ISO = 0, bool NC = true>
__device__ __forceinline__ float3 struct_field_upper(const float4* __restrict__ S, const PyroMats& mats, int cell,
                                                     int L, int Nc, uint64_t divL) {
    const Coords c = cell_coords(cell, L, divL);
    float3 h = make_float3(0.f, 0.f, 0.f);
    add_group_upper<SL, 0, ISO, NC>(h, S, Nc, c, mats);
    add_group_upper<SL, 1, ISO, NC>(h, S, Nc, c, mats);
    add_group_upper<SL, 2, ISO, NC>(h, S, Nc, c, mats);
    add_group_upper<SL, 3, ISO, NC>(h, S, Nc, c, mats);
    add_group_upper<SL, 4, ISO, NC>(h, S, Nc, c, mats);
    add_group_upper<SL, 5, ISO, NC>(h, S, Nc, c, mats);
    return h;
}

template <int SL>
__device__ __forceinline__ float3 struct_field(const float4* __restrict__ S, const PyroMats& mats, int cell,
                                               int L, int Nc, uint64_t divL) {
    const Coords c = cell_coords(cell, L, divL);
    float3 h = make_float3(0.f, 0.f, 0.f);
    add_group<SL, 0>(h, S, Nc, c, mats);
    add_group<SL, 1>(h, S, Nc, c, mats);
    add_group<SL, 2>(h, S, Nc, c, mats);
    add_group<SL, 3>(h, S, Nc, c, mats);
    add_group<SL, 4>(h, S, Nc, c, mats);
    add_group<SL, 5>(h, S, Nc, c, mats);
    return h;
}

}  // namespace pc
