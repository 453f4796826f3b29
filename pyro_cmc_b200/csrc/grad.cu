// grad.cu -- energy gradient through the compile-time pyrochlore neighbour
// structure (sm_100a).
//
// Per site i of sublattice SL: the local field h_i (the group sums of its 30
// structural neighbours times the group matrices), the energy
// 0.5 S_i.h_i - S_i.B, and dE/dS_i = g_r/Nc (h_i - B). With coupling
// gradients requested, each group's neighbour sum is split by bond side
// (this site's pyro_sl <= the neighbour's: the bond applies J, S_i (x) t;
// otherwise J^T, t (x) S_i, as setup_lattice splits the shells,
// src/MC.cpp:28-50) and 0.5 x the outer product is added to dE/dJ of every
// spec that owns those displacements: summed over all sites this counts each
// bond of the spec once on each end, sum over bonds S_src (x) S_tgt.
//
// A work item is up to kGradK consecutive tiles of one (replica, sublattice):
// each thread takes one site per tile, so the per-warp reductions of the
// coupling products (FP32 shuffles, FP64 from the warp sum on) and of the
// energy (FP64) are paid once per kGradK sites. Every warp adds into its own
// shared-memory row and the rows are summed in warp order, so the result does
// not depend on scheduling.
#include <cuda_runtime.h>

#include <utility>

#include "common.cuh"
#include "kernels.h"
#include "moves.cuh"
#include "struct_field.cuh"

namespace pc {

// bond side of structural neighbour e of sublattice sl: 0 applies J, 1 J^T
__host__ __device__ constexpr int nb_side(int sl, int e) { return (sl % 4 <= nb_sl(sl, e) % 4) ? 0 : 1; }
__host__ __device__ constexpr bool group_has_side(int sl, int g, int side) {
    for (int e = grp_begin(sl, g); e < grp_begin(sl, g + 1); ++e)
        if (nb_side(sl, e) == side) return true;
    return false;
}

template <int SIDE>
__device__ __forceinline__ void add_side(float3& t0, float3& t1, const float4& v) {
    if constexpr (SIDE == 0) {
        t0.x += v.x;
        t0.y += v.y;
        t0.z += v.z;
    } else {
        t1.x += v.x;
        t1.y += v.y;
        t1.z += v.z;
    }
}

// group G's neighbour sums on side 0 and side 1, each in neighbour order; the
// group's loads are issued together
template <int SL, int G, int... K>
__device__ __forceinline__ void group_sides(float3& t0, float3& t1, const float4* __restrict__ S, int Nc,
                                            const Coords& c, std::integer_sequence<int, K...>) {
    constexpr int B = grp_begin(SL, G);
    const float4 v[sizeof...(K)] = {load_nb<SL, B + K>(S, Nc, c)...};
    (add_side<nb_side(SL, B + K)>(t0, t1, v[K]), ...);
}

template <typename T>
__device__ __forceinline__ T warp_total(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// 0.5 x the warp's sum of p into dE/dJ of every spec in mask (lane 0 writes
// the warp's own row). Not inlined: one copy serves every (sublattice, group,
// side), which keeps the kernel's code within the instruction cache.
__device__ __noinline__ void add_products(float p0, float p1, float p2, float p3, float p4, float p5, float p6,
                                          float p7, float p8, uint32_t mask, double* wrow, int lane) {
    const float p[9] = {p0, p1, p2, p3, p4, p5, p6, p7, p8};
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const float v = warp_total(p[i]);
        if (lane == 0)
            for (uint32_t m = mask; m; m &= m - 1) wrow[4 + 9 * (__ffs(int(m)) - 1) + i] += 0.5 * double(v);
    }
}
__device__ __forceinline__ void add_products(const float (&p)[9], uint32_t mask, double* wrow, int lane) {
    add_products(p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], p[8], mask, wrow, lane);
}

template <int KS>
struct GradSites {
    Coords c[KS];
    float3 s[KS];
    float3 h[KS];
    int cell[KS];
    bool live[KS];
};

template <int SL, int G, bool WJ, int KS>
__device__ __forceinline__ void grad_group(const GradStructArgs& a, const float4* S, int Nc, GradSites<KS>& q,
                                           double* wrow, int lane) {
    if (!WJ && !(a.mats.active[SL] & (1u << G))) return;
    constexpr bool kSide0 = group_has_side(SL, G, 0), kSide1 = group_has_side(SL, G, 1);
    const float* M = a.mats.M[SL][G];
    float p0[9] = {}, p1[9] = {};
#pragma unroll
    for (int k = 0; k < KS; ++k) {
        if (!q.live[k]) continue;
        float3 t0 = make_float3(0.f, 0.f, 0.f), t1 = make_float3(0.f, 0.f, 0.f);
        group_sides<SL, G>(t0, t1, S, Nc, q.c[k], std::make_integer_sequence<int, grp_size(SL, G)>{});
        const float tx = t0.x + t1.x, ty = t0.y + t1.y, tz = t0.z + t1.z;
        q.h[k].x += M[0] * tx + M[1] * ty + M[2] * tz;
        q.h[k].y += M[3] * tx + M[4] * ty + M[5] * tz;
        q.h[k].z += M[6] * tx + M[7] * ty + M[8] * tz;
        if constexpr (WJ) {
            const float sv[3] = {q.s[k].x, q.s[k].y, q.s[k].z};
            const float a0[3] = {t0.x, t0.y, t0.z}, a1[3] = {t1.x, t1.y, t1.z};
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    p0[3 * i + j] += sv[i] * a0[j];
                    p1[3 * i + j] += a1[i] * sv[j];
                }
        }
    }
    if constexpr (WJ) {
        if constexpr (kSide0) add_products(p0, a.spec_mask[SL][G][0], wrow, lane);
        if constexpr (kSide1) add_products(p1, a.spec_mask[SL][G][1], wrow, lane);
    }
}

// KS sites of the item at once (tiles tl[0..n), n <= KS): their field, energy
// and spin gradient, and with WJ the coupling products of all KS sites reduced
// once per (group, side). Energy and sum S accumulate into v.
template <int SL, bool WJ, int KS>
__device__ __forceinline__ void grad_sites(const GradStructArgs& a, const Tile* tl, int n, const ReplicaDev& rep,
                                           int r, double* wrow, double (&v)[4]) {
    const int lane = threadIdx.x & 31;
    const int Nc = rep.Nc;
    const float4* S = a.spins + rep.off;
    GradSites<KS> q;
#pragma unroll
    for (int k = 0; k < KS; ++k) {
        q.live[k] = k < n && int(threadIdx.x) < tl[k].w;
        q.cell[k] = q.live[k] ? tl[k].z + int(threadIdx.x) : 0;
        q.c[k] = cell_coords(q.cell[k], rep.L, rep.divL);
        const float4 s0 = q.live[k] ? S[size_t(SL) * Nc + q.cell[k]] : make_float4(0.f, 0.f, 0.f, 0.f);
        q.s[k] = make_float3(s0.x, s0.y, s0.z);
        q.h[k] = make_float3(0.f, 0.f, 0.f);
    }
    grad_group<SL, 0, WJ>(a, S, Nc, q, wrow, lane);
    grad_group<SL, 1, WJ>(a, S, Nc, q, wrow, lane);
    grad_group<SL, 2, WJ>(a, S, Nc, q, wrow, lane);
    grad_group<SL, 3, WJ>(a, S, Nc, q, wrow, lane);
    grad_group<SL, 4, WJ>(a, S, Nc, q, wrow, lane);
    grad_group<SL, 5, WJ>(a, S, Nc, q, wrow, lane);
    const float gs = float(a.g[r] / double(Nc));
#pragma unroll
    for (int k = 0; k < KS; ++k) {
        if (!q.live[k]) continue;
        const float3 s = q.s[k], h = q.h[k];
        v[0] += 0.5 * double(s.x * h.x + s.y * h.y + s.z * h.z) - double(s.x * a.B[0] + s.y * a.B[1] + s.z * a.B[2]);
        v[1] += s.x;
        v[2] += s.y;
        v[3] += s.z;
        if (a.grad_S)
            a.grad_S[rep.off + size_t(SL) * Nc + q.cell[k]] =
                make_float4(gs * (h.x - a.B[0]), gs * (h.y - a.B[1]), gs * (h.z - a.B[2]), 0.f);
    }
}

// One work item: with WJ all its sites at once (the coupling products are
// reduced once per item); without, one site after another (fewest registers).
template <int SL, bool WJ>
__device__ __forceinline__ void grad_item(const GradStructArgs& a, const Tile* tl, int nt, const ReplicaDev& rep,
                                          int r, double* wrow) {
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    if constexpr (WJ) {
        grad_sites<SL, true, kGradK>(a, tl, nt, rep, r, wrow, v);
    } else {
        for (int k = 0; k < nt; ++k) grad_sites<SL, false, 1>(a, tl + k, 1, rep, r, wrow, v);
    }
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const double t = warp_total(v[j]);
        if (lane == 0) wrow[j] += t;
    }
}

template <bool WJ>
__global__ void __launch_bounds__(256) energy_grad_struct_kernel(const __grid_constant__ GradStructArgs a) {
    extern __shared__ double wacc[];  // [warps][width]
    const int nw = int(blockDim.x >> 5), warp = int(threadIdx.x >> 5);
    for (int i = blockIdx.x; i < a.n_items; i += gridDim.x) {
        for (int j = threadIdx.x; j < nw * a.width; j += blockDim.x) wacc[j] = 0.0;
        __syncthreads();
        const int4 it = a.items[i];
        const Tile* tl = a.tiles + it.x;
        const Tile t0 = tl[0];
        const int r = t0.x, sl = t0.y & 0xff;
        const ReplicaDev rep = a.reps[r];
        double* wrow = wacc + size_t(warp) * a.width;
#define PC_CALL(K) grad_item<K, WJ>(a, tl, it.y, rep, r, wrow)
        PC_SL_SWITCH(sl, PC_CALL)
#undef PC_CALL
        __syncthreads();
        for (int j = threadIdx.x; j < a.width; j += blockDim.x) {
            double s = 0.0;
            for (int w = 0; w < nw; ++w) s += wacc[w * a.width + j];
            a.partial[size_t(it.z) * a.width + j] = s;
        }
        __syncthreads();
    }
}

void launch_energy_grad_struct(const GradStructArgs& a, bool want_J, int threads, cudaStream_t st) {
    const size_t smem = sizeof(double) * size_t(threads / 32) * size_t(a.width);
    if (want_J) {
        // per-warp rows of 4 + 9 n_spec doubles: the default shared-memory
        // carveout (the smallest one would hold two CTAs per SM)
        energy_grad_struct_kernel<true><<<a.n_items, threads, smem, st>>>(a);
    } else {
        prefer_l1(reinterpret_cast<const void*>(energy_grad_struct_kernel<false>));
        energy_grad_struct_kernel<false><<<a.n_items, threads, smem, st>>>(a);
    }
}

}  // namespace pc
