// moves.cuh -- the per-site moves and the colour-pass kernel templates
// (generic bond-table pass, structured pyrochlore pass), shared by the
// translation units that instantiate them: sweep.cu (Metropolis,
// overrelaxation and fused passes), sweep_lifted.cu (lifted Metropolis) and
// sweep_staged.cu (row-staged passes), each family in its own module.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <set>
#include <utility>

#include "common.cuh"
#include "kernels.h"
#include "struct_field.cuh"

namespace pc {

__device__ __forceinline__ void stage_tables(SlTable* dst, const SlTable* src, int n_tab, const int* sls) {
    const int words = int(sizeof(SlTable) / 4);
    for (int t = 0; t < n_tab; ++t) {
        const int* s = reinterpret_cast<const int*>(src + sls[t]);
        int* d = reinterpret_cast<int*>(dst + t);
        for (int i = threadIdx.x; i < words; i += blockDim.x) d[i] = s[i];
    }
}

// The random numbers of a proposal from Philox words. The radius of a
// Box-Muller pair, sqrt(-2 ln u) for u = u24_open0(w) in (0, 1], uses the
// hardware logarithm (__logf: absolute error below 2^-21.4 on [0.5, 2], 3 ulp
// elsewhere), clamped at 0 so that a logarithm rounded above 0 for u next to
// 1 gives radius 0. A uniform angle is 2 pi (u24(w) - 1/2) in [-pi, pi), the
// range where the hardware sine and cosine (__sincosf) are accurate to 2^-21.4
// absolute; its distribution on the circle is that of 2 pi u. These errors
// are far below anything a Monte Carlo proposal resolves; the pass runs 6 %
// faster than with the correctly rounded logf and sincospif.
__device__ __forceinline__ float bm_radius(uint32_t w) { return sqrtf(fmaxf(-2.f * __logf(u24_open0(w)), 0.f)); }
__device__ __forceinline__ void uniform_angle(uint32_t w, float* s, float* c) {
    __sincosf(6.2831853f * (u24(w) - 0.5f), s, c);
}

// Dot product and the products of the moves with every rounding fixed: an FMA
// chain in a fixed order. Left to the compiler, the contraction of the plain
// expressions into FMAs may differ between the kernels that inline a move
// (per-pass, persistent, staged, cluster-resident), and their chains would
// part at the first decision that the last bit changes.
__device__ __forceinline__ float dot3_rn(float ax, float ay, float az, float bx, float by, float bz) {
    return fmaf(az, bz, fmaf(ay, by, __fmul_rn(ax, bx)));
}

// h = sum over shells J_k * sum of neighbour spins (MC_runner::local_field,
// src/MC.cpp:87-96).
__device__ __forceinline__ float3 local_field(const float4* __restrict__ S, const SlTable& tb, int cx, int cy, int cz,
                                              int L, int Nc) {
    float hx = 0.f, hy = 0.f, hz = 0.f;
    int e = 0;
    const int ns = tb.n_shell;
    for (int k = 0; k < ns; ++k) {
        float tx = 0.f, ty = 0.f, tz = 0.f;
        const int end = tb.shell_end[k];
        for (; e < end; ++e) {
            const NbEntry nb = tb.nb[e];
            const int x = wrap1(cx + nb.dx, L), y = wrap1(cy + nb.dy, L), z = wrap1(cz + nb.dz, L);
            const float4 o = __ldg(&S[size_t(nb.sl) * Nc + x + L * (y + L * z)]);
            tx += o.x;
            ty += o.y;
            tz += o.z;
        }
        const float* J = tb.J[k];
        hx += J[0] * tx + J[1] * ty + J[2] * tz;
        hy += J[3] * tx + J[4] * ty + J[5] * tz;
        hz += J[6] * tx + J[7] * ty + J[8] * tz;
    }
    return make_float3(hx, hy, hz);
}

// The move at site i with local field h (global field not yet subtracted):
// Metropolis (local_Metropolis, src/MC.cpp:111-130) or one overrelaxation
// (overrelax_all, src/MC.cpp:145-153; mirror_about_vector :98-100). Returns
// whether a Metropolis proposal was accepted.
// The overrelaxation of spin s0 about the effective field h (global field
// already subtracted): rotate_about_vector by the given angle (src/MC.cpp:102-109)
// or mirror_about_vector (:98-100), renormalised against FP32 drift. Returns
// false (spin unchanged) for a zero field or a zero spin.
template <bool REFLECT>
__device__ __forceinline__ bool overrelax_spin(float4 s0, float3 h, float sn, float cs, float4& out) {
    const float n2 = dot3_rn(h.x, h.y, h.z, h.x, h.y, h.z);
    // a zero local field leaves the spin as it is; so does a zero spin (the
    // reference's default-constructed state, which rotation keeps at zero)
    if (!(n2 > 1e-30f) || !(dot3_rn(s0.x, s0.y, s0.z, s0.x, s0.y, s0.z) > 0.f)) return false;
    const float av = dot3_rn(h.x, h.y, h.z, s0.x, s0.y, s0.z);
    float nx, ny, nz;
    if (REFLECT) {
        const float f = __fdividef(2.f * av, n2 + 1e-10f);
        nx = fmaf(f, h.x, -s0.x);
        ny = fmaf(f, h.y, -s0.y);
        nz = fmaf(f, h.z, -s0.z);
    } else {
        // cs s + f h + g (h x s)
        const float f = __fdividef((1.f - cs) * av, n2);
        const float g = sn * rsqrtf(n2);
        const float cx = fmaf(h.y, s0.z, -__fmul_rn(h.z, s0.y));
        const float cy = fmaf(h.z, s0.x, -__fmul_rn(h.x, s0.z));
        const float cz = fmaf(h.x, s0.y, -__fmul_rn(h.y, s0.x));
        nx = fmaf(g, cx, fmaf(f, h.x, __fmul_rn(cs, s0.x)));
        ny = fmaf(g, cy, fmaf(f, h.y, __fmul_rn(cs, s0.y)));
        nz = fmaf(g, cz, fmaf(f, h.z, __fmul_rn(cs, s0.z)));
    }
    const float inv = rsqrtf(dot3_rn(nx, ny, nz, nx, ny, nz));
    out = make_float4(nx * inv, ny * inv, nz * inv, s0.w);  // w: the lifting direction, kept
    return true;
}

// Metropolis proposal of local_Metropolis (src/MC.cpp:111-130) at site i with
// effective field h: returns whether it is accepted; `out` holds the new spin.
__device__ __forceinline__ bool metropolis_spin(const PassArgs& a, float4 s0, float3 h, int r, uint64_t sweep, size_t i,
                                                float4& out) {
    const double T = a.T_rep[r];
    const float sigma = sqrtf(float(T) * a.inv_T_ref);
    const float invT = float(1.0 / T);
    const uint4 w = site_draw(a.seed, uint32_t(r), sweep, kDrawMetropolis, uint32_t(i));
    // Box-Muller on the top 24 bits of words (0,1) and (2,3)
    const float r0 = bm_radius(w.x);
    const float r1 = bm_radius(w.z);
    float s_a, c_a, s_b, c_b;
    uniform_angle(w.y, &s_a, &c_a);
    uniform_angle(w.w, &s_b, &c_b);
    float nx = fmaf(sigma, __fmul_rn(r0, c_a), s0.x);
    float ny = fmaf(sigma, __fmul_rn(r0, s_a), s0.y);
    float nz = fmaf(sigma, __fmul_rn(r1, c_b), s0.z);
    const float inv = rsqrtf(dot3_rn(nx, ny, nz, nx, ny, nz));
    nx *= inv;
    ny *= inv;
    nz *= inv;
    const float dE = dot3_rn(nx - s0.x, ny - s0.y, nz - s0.z, h.x, h.y, h.z);
    if (dE < 0.f || u24_lowbytes(w) < __expf(-dE * invT)) {
        out = make_float4(nx, ny, nz, s0.w);
        return true;
    }
    out = s0;
    return false;
}

// Lifted Metropolis at site i with effective field h (global field already
// subtracted). The lifting direction is the sign of w (w >= 0: +1, the
// reference's initial lifted_dir); a rejected or bounced move flips it.
//   u-form (src/MC.cpp:249-281): u = S.h_hat slides by dir*sqrt(T/T_ref)*E,
//     E ~ Exp(1), at fixed azimuth; off the sphere or at a pole: bounce.
//   rotation form (src/MC.cpp:194-244): rotate by dir*sqrt(T/T_ref) about
//     S x h; a pole or a pole crossing bounces; acceptance
//     min(1, |S' x h| / |S x h| e^{-dE/T}).
// Draws: Philox draw kDrawLifted, Exp(1) = -ln(open uniform of word 0), the
// acceptance uniform from word 1. Returns whether the move was accepted; `out`
// always holds the new state (spin and direction).
template <bool ROT>
__device__ __forceinline__ bool lifted_spin(const PassArgs& a, float4 s0, float3 h, int r, uint64_t sweep, size_t i,
                                            float4& out) {
    const double T = a.T_rep[r];
    const float step = sqrtf(float(T) * a.inv_T_ref);
    const float invT = float(1.0 / T);
    const uint4 w = site_draw(a.seed, uint32_t(r), sweep, kDrawLifted, uint32_t(i));
    const float u01 = u24(w.y);
    const float dir = s0.w < 0.f ? -1.f : 1.f;
    out = make_float4(s0.x, s0.y, s0.z, -dir);  // the bounce / rejection state
    const float curr = s0.x * h.x + s0.y * h.y + s0.z * h.z;
    float nx, ny, nz, ratio;
    if (!ROT) {
        const float n2 = h.x * h.x + h.y * h.y + h.z * h.z;
        if (!(n2 > 0.f)) return false;  // no field: the direction is undefined
        const float ih = rsqrtf(n2);
        const float hx = h.x * ih, hy = h.y * ih, hz = h.z * ih;
        const float u = hx * s0.x + hy * s0.y + hz * s0.z;
        const float nu = u + dir * step * (-logf(u24_open0(w.x)));
        const float one_u2 = 1.f - u * u;
        if (nu > 1.f || nu < -1.f || !(fabsf(one_u2) >= 1e-12f)) return false;
        const float f = sqrtf((1.f - nu * nu) / one_u2);
        nx = nu * hx + f * (s0.x - u * hx);
        ny = nu * hy + f * (s0.y - u * hy);
        nz = nu * hz + f * (s0.z - u * hz);
        const float inv = rsqrtf(nx * nx + ny * ny + nz * nz);
        nx *= inv;
        ny *= inv;
        nz *= inv;
        ratio = __expf(-(nx * h.x + ny * h.y + nz * h.z - curr) * invT);
    } else {
        const float ax = s0.y * h.z - s0.z * h.y, ay = s0.z * h.x - s0.x * h.z, az = s0.x * h.y - s0.y * h.x;
        const float n2_old = ax * ax + ay * ay + az * az;
        if (!(n2_old > 1e-20f)) return false;  // pole: the meridian is undefined
        float sn, cs;
        sincosf(dir * step, &sn, &cs);
        // Rodrigues about the unnormalised axis (axis . S = 0 up to rounding)
        const float av = ax * s0.x + ay * s0.y + az * s0.z;
        const float g = sn * rsqrtf(n2_old), f = (1.f - cs) * av / n2_old;
        nx = cs * s0.x + f * ax + g * (ay * s0.z - az * s0.y);
        ny = cs * s0.y + f * ay + g * (az * s0.x - ax * s0.z);
        nz = cs * s0.z + f * az + g * (ax * s0.y - ay * s0.x);
        const float inv = rsqrtf(nx * nx + ny * ny + nz * nz);
        nx *= inv;
        ny *= inv;
        nz *= inv;
        const float bx = ny * h.z - nz * h.y, by = nz * h.x - nx * h.z, bz = nx * h.y - ny * h.x;
        if (ax * bx + ay * by + az * bz < 0.f) return false;  // crossed a pole
        const float n2_new = bx * bx + by * by + bz * bz;
        ratio = sqrtf(n2_new / n2_old) * __expf(-(nx * h.x + ny * h.y + nz * h.z - curr) * invT);
    }
    if (u01 < ratio) {
        out = make_float4(nx, ny, nz, dir);
        return true;
    }
    return false;
}

// The w component a pass writes: the lifting direction survives overrelaxation
// and lifted passes (the passes of a lifted sweep); a standard Metropolis or
// fused pass writes 0, resetting it to +1.
template <int MODE>
__device__ __forceinline__ float w_after(float w) {
    return (MODE == kMetropolis || MODE == kFusedRotate || MODE == kFusedReflect) ? 0.f : w;
}

// The move at site i with local field h (global field not yet subtracted).
// Returns whether a Metropolis proposal was accepted.
template <int MODE>
__device__ __forceinline__ bool apply_move(const PassArgs& a, float4* S, size_t i, float3 h, int r, uint64_t sweep) {
    const float4 s0 = S[i];
    h.x -= a.B[0];
    h.y -= a.B[1];
    h.z -= a.B[2];
    if constexpr (MODE == kLifted || MODE == kLiftedRot) {
        float4 s1;
        const bool acc = lifted_spin<MODE == kLiftedRot>(a, s0, h, r, sweep, i, s1);
        S[i] = s1;  // the direction changes on rejection too
        return acc;
    }
    bool acc = false;
    float4 s1 = s0;
    s1.w = w_after<MODE>(s0.w);
    if (MODE == kMetropolis || MODE == kFusedRotate || MODE == kFusedReflect)
        acc = metropolis_spin(a, s1, h, r, sweep, i, s1);
    if (MODE == kMetropolis) {
        if (acc) S[i] = s1;
        return acc;
    }
    float sn = 0.f, cs = 1.f;
    if (MODE == kOverrelaxRotate || MODE == kFusedRotate) {
        const uint4 w = site_draw(a.seed, uint32_t(r), sweep, kDrawOverrelax0 + uint32_t(a.or_pass), uint32_t(i));
        uniform_angle(w.x, &sn, &cs);
    } else if (MODE == kOverrelaxTheta) {
        sincosf(float(a.theta[i]), &sn, &cs);
    }
    float4 s2;
    const bool moved = overrelax_spin<MODE == kOverrelaxReflect || MODE == kFusedReflect>(s1, h, sn, cs, s2);
    if (moved)
        S[i] = s2;
    else if (acc)
        S[i] = s1;
    return acc;
}

// Accepted-move counting: each thread keeps a running count while its block
// works through tiles of one replica and the block flushes it (one atomic)
// when the replica changes and at the end. Tiles are replica-contiguous, so
// a single-replica pass costs one atomic per block.
__device__ __forceinline__ void flush_accepted(const PassArgs& a, unsigned int& mine, int r, unsigned int* warp_acc) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned int c = mine;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if (lane == 0) warp_acc[warp] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int tot = 0;
        for (int wi = 0; wi < int(blockDim.x >> 5); ++wi) tot += warp_acc[wi];
        if (tot) atomicAdd(a.acc + r, (unsigned long long)tot);
    }
    __syncthreads();
    mine = 0;
}

// Programmatic dependent launch. pdl_wait at entry: wait until the previous
// kernel on the stream has finished and its writes are visible. pdl_trigger
// once a CTA's updates are done: the next pass may start launching when every
// CTA has triggered, overlapping its launch with this pass's last CTAs.
// Triggering at entry instead made the next pass's CTAs resident early, where
// they held warp slots the running pass needed (measured 6 % slower at L=64).
// Both are no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Generic colour pass: bond tables (any coupling set) staged in shared memory.
template <int MODE>
__global__ void __launch_bounds__(512) colour_pass_kernel(const __grid_constant__ PassArgs a) {
    __shared__ SlTable tab[4];
    __shared__ unsigned int warp_acc[16];
    stage_tables(tab, a.tables, a.n_tab, a.tab_sl);  // tables are never written by kernels
    pdl_wait();
    __syncthreads();
    const uint64_t sweep = *a.sweep_base + a.sweep_offset;
    unsigned int mine = 0;
    int r_cur = -1;
    for (int t = blockIdx.x; t < a.n_tiles; t += gridDim.x) {
        const Tile tile = a.tiles[t];
        const int r = tile.x;
        if ((MODE == kMetropolis || MODE >= kFusedRotate) && r != r_cur) {
            if (r_cur >= 0) flush_accepted(a, mine, r_cur, warp_acc);
            r_cur = r;
        }
        const int k = tile.y >> 8, sl = tile.y & 0xff;
        const ReplicaDev rep = a.reps[r];
        const int L = rep.L, Nc = rep.Nc;
        float4* S = a.spins + rep.off;
        if (int(threadIdx.x) < tile.w) {
            const int cell = tile.z + int(threadIdx.x);
            const int cx = cell % L, cy = (cell / L) % L, cz = cell / (L * L);
            const float3 h = local_field(S, tab[k], cx, cy, cz, L, Nc);
            mine += apply_move<MODE>(a, S, size_t(sl) * Nc + cell, h, r, sweep) ? 1u : 0u;
        }
    }
    pdl_trigger();
    if ((MODE == kMetropolis || MODE >= kFusedRotate) && r_cur >= 0) flush_accepted(a, mine, r_cur, warp_acc);
}

// One site of the structured pass. How the 30 neighbour loads are issued is
// chosen by the autotuner (more loads in flight per thread costs registers,
// hence resident warps):
//   VAR 0: group by group (six short load batches, fewest registers);
//   VAR 1: all 30 at once, before the Philox draw and the proposal (which do
//          not depend on the local field) are computed;
//   VAR 2: J1 + J2 neighbours (18) before the draw, J3 (12) after it;
//   kVarIso, kVarIsoNoJ2: VAR 0 for systems whose group matrices are all j I
//          (or all but a zero J2 group), chosen by the host in place of VAR 0:
//          the same bits, fewer instructions, no per-group branches.
template <int SL, int VAR_>
__device__ __forceinline__ float3 site_field(const float4* __restrict__ S, const PassArgs& a, const ReplicaDev& rep,
                                             const Coords& c, float4 (&v)[kStructNb], int phase) {
    constexpr int VAR = VAR_ & ~(kVarCoherent | kVarUniformBase);
    constexpr bool NC = (VAR_ & kVarCoherent) == 0;
    constexpr bool UB = (VAR_ & kVarUniformBase) != 0;
    static_assert(NC || VAR == 0 || VAR == kVarIso || VAR == kVarIsoNoJ2, "coherent loads: variants 0 and iso");
    constexpr int kJ3 = grp_begin(SL, 4);
    float3 h = make_float3(0.f, 0.f, 0.f);
    if constexpr (VAR == 0) {
        if (phase == 1) {
            add_group<SL, 0, NC>(h, S, rep.Nc, c, a.mats);
            add_group<SL, 1, NC>(h, S, rep.Nc, c, a.mats);
            add_group<SL, 2, NC>(h, S, rep.Nc, c, a.mats);
            add_group<SL, 3, NC>(h, S, rep.Nc, c, a.mats);
            add_group<SL, 4, NC>(h, S, rep.Nc, c, a.mats);
            add_group<SL, 5, NC>(h, S, rep.Nc, c, a.mats);
        }
    } else if constexpr (VAR == kVarIso || VAR == kVarIsoNoJ2) {
        if (phase == 1) {
            add_group_iso<SL, 0, NC, UB>(h, S, rep.Nc, c, a.mats);
            add_group_iso<SL, 1, NC, UB>(h, S, rep.Nc, c, a.mats);
            add_group_iso<SL, 2, NC, UB>(h, S, rep.Nc, c, a.mats);
            if constexpr (VAR == kVarIso) add_group_iso<SL, 3, NC, UB>(h, S, rep.Nc, c, a.mats);
            add_group_iso<SL, 4, NC, UB>(h, S, rep.Nc, c, a.mats);
            add_group_iso<SL, 5, NC, UB>(h, S, rep.Nc, c, a.mats);
        }
    } else if constexpr (VAR == 1) {
        if (phase == 0)
            load_nbs<SL, 0, kStructNb>(v, S, rep.Nc, c, a.mats.active[SL]);
        else
            field_groups<SL, 0, kGroups>(h, v, a.mats);
    } else {
        if (phase == 0) {
            load_nbs<SL, 0, kJ3>(v, S, rep.Nc, c, a.mats.active[SL]);
        } else {
            field_groups<SL, 0, 4>(h, v, a.mats);
            load_nbs<SL, kJ3, kStructNb>(v, S, rep.Nc, c, a.mats.active[SL]);
            field_groups<SL, 4, kGroups>(h, v, a.mats);
        }
    }
    return h;
}

template <int MODE, int SL, int VAR>
__device__ __forceinline__ bool struct_site(const PassArgs& a, float4* S, const ReplicaDev& rep, int r, int cell,
                                            uint64_t sweep) {
    const Coords c = cell_coords(cell, rep.L, rep.divL);
    float4 v[kStructNb];
    site_field<SL, VAR>(S, a, rep, c, v, 0);  // issue loads (VAR 1, 2)
    const size_t i = size_t(SL) * rep.Nc + cell;
    constexpr bool kCoherent = (VAR & kVarCoherent) != 0;
    const float4 s0 = kCoherent ? __ldca(S + i) : S[i];
    constexpr bool kMet = MODE == kMetropolis || MODE == kFusedRotate || MODE == kFusedReflect;
    constexpr bool kRot = MODE == kOverrelaxRotate || MODE == kFusedRotate;
    // draws first: they do not depend on the local field, so they overlap the loads
    uint4 w = make_uint4(0, 0, 0, 0);
    float sigma = 0.f, invT = 0.f;
    if (kMet) {
        const float2 q = kCoherent ? __ldca(a.Tq + r) : a.Tq[r];
        sigma = q.x;
        invT = q.y;
        w = site_draw_rk(a.rkeys, uint32_t(r), sweep, kDrawMetropolis, uint32_t(i));
    }
    float sn = 0.f, cs = 1.f;
    if (kRot) {
        const uint4 wo = site_draw_rk(a.rkeys, uint32_t(r), sweep, kDrawOverrelax0 + uint32_t(a.or_pass), uint32_t(i));
        uniform_angle(wo.x, &sn, &cs);
    } else if (MODE == kOverrelaxTheta) {
        sincosf(float(a.theta[i]), &sn, &cs);
    }
    float4 s1 = s0;
    s1.w = w_after<MODE>(s0.w);
    float nx = 0.f, ny = 0.f, nz = 0.f, u = 0.f;
    if (kMet) {
        const float r0 = bm_radius(w.x);
        const float r1 = bm_radius(w.z);
        float s_a, c_a, s_b, c_b;
        uniform_angle(w.y, &s_a, &c_a);
        uniform_angle(w.w, &s_b, &c_b);
        nx = fmaf(sigma, __fmul_rn(r0, c_a), s0.x);
        ny = fmaf(sigma, __fmul_rn(r0, s_a), s0.y);
        nz = fmaf(sigma, __fmul_rn(r1, c_b), s0.z);
        const float inv = rsqrtf(dot3_rn(nx, ny, nz, nx, ny, nz));
        nx *= inv;
        ny *= inv;
        nz *= inv;
        u = u24_lowbytes(w);
    }
    float3 h = site_field<SL, VAR>(S, a, rep, c, v, 1);
    h.x -= a.B[0];
    h.y -= a.B[1];
    h.z -= a.B[2];
    if constexpr (MODE == kLifted || MODE == kLiftedRot) {
        float4 s1;
        const bool lacc = lifted_spin<MODE == kLiftedRot>(a, s0, h, r, sweep, i, s1);
        S[i] = s1;
        return lacc;
    }
    bool acc = false;
    if (kMet) {
        const float dE = dot3_rn(nx - s0.x, ny - s0.y, nz - s0.z, h.x, h.y, h.z);
        if (dE < 0.f || u < __expf(-dE * invT)) {
            s1 = make_float4(nx, ny, nz, w_after<MODE>(s0.w));
            acc = true;
        }
        if (MODE == kMetropolis) {
            if (acc) S[i] = s1;
            return acc;
        }
    }
    float4 s2;
    const bool moved = overrelax_spin<MODE == kOverrelaxReflect || MODE == kFusedReflect>(s1, h, sn, cs, s2);
    if (moved)
        S[i] = s2;
    else if (acc)
        S[i] = s1;
    return acc;
}

#define PC_SL_SWITCH(sl, CALL) \
    switch (sl) {              \
        case 0: CALL(0); break;   \
        case 1: CALL(1); break;   \
        case 2: CALL(2); break;   \
        case 3: CALL(3); break;   \
        case 4: CALL(4); break;   \
        case 5: CALL(5); break;   \
        case 6: CALL(6); break;   \
        case 7: CALL(7); break;   \
        case 8: CALL(8); break;   \
        case 9: CALL(9); break;   \
        case 10: CALL(10); break; \
        case 11: CALL(11); break; \
        case 12: CALL(12); break; \
        case 13: CALL(13); break; \
        case 14: CALL(14); break; \
        case 15: CALL(15); break; \
        default: break;           \
    }

// Structured colour pass: pyrochlore neighbour offsets fixed at compile time,
// coupling matrices per (sublattice, group) in the kernel parameters.
template <int MODE, int VAR>
__global__ void __launch_bounds__(256) struct_pass_kernel(const __grid_constant__ PassArgs a) {
    // fused isotropic rotation passes with every group active: neighbour
    // addresses from per-sublattice bases (measured faster there; other passes
    // keep the full offset sums -- with J2 = 0 the faster tile moved, and the
    // persistent kernel, which inherits the tile, lost more than the pass gained)
    constexpr int VARX = (MODE == kFusedRotate && VAR == kVarIso) ? (VAR | kVarUniformBase) : VAR;
    __shared__ unsigned int warp_acc[8];
    pdl_wait();
    const uint64_t sweep = *a.sweep_base + a.sweep_offset;
    unsigned int mine = 0;
    int r_cur = -1;
    for (int t = blockIdx.x; t < a.n_tiles; t += gridDim.x) {
        const Tile tile = a.tiles[t];
        const int r = tile.x, sl = tile.y & 0xff;
        if ((MODE == kMetropolis || MODE >= kFusedRotate) && r != r_cur) {
            if (r_cur >= 0) flush_accepted(a, mine, r_cur, warp_acc);
            r_cur = r;
        }
        const ReplicaDev rep = a.reps[r];
        float4* S = a.spins + rep.off;
        if (int(threadIdx.x) < tile.w) {
            const int cell = tile.z + int(threadIdx.x);
            bool accepted = false;
#define PC_CALL(K) accepted = struct_site<MODE, K, VARX>(a, S, rep, r, cell, sweep)
            PC_SL_SWITCH(sl, PC_CALL)
#undef PC_CALL
            mine += accepted ? 1u : 0u;
        }
    }
    pdl_trigger();
    if ((MODE == kMetropolis || MODE >= kFusedRotate) && r_cur >= 0) flush_accepted(a, mine, r_cur, warp_acc);
}

// The colour passes gather 30 neighbours per site through L1 and use almost no
// shared memory: ask for the largest L1 (smallest shared-memory carveout), once
// per kernel and device, whatever kernels with large shared memory (the S(q)
// stages) ran before. With the 8 KB configuration this leaves 7 resident
// blocks of 128 threads (every block holds 1 KB of shared memory for the
// system) where 64 registers would allow 8; a larger carveout that admits the
// 8th block (the driver chose 164 KB for a 7 % request) measured slower at
// L = 64 (10.73 against 10.50 us per pass): the L1 it takes costs more than
// the extra warps give.
inline void prefer_l1(const void* fn) {
    static std::mutex mu;
    static std::set<std::pair<int, const void*>> done;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    if (done.insert({dev, fn}).second)
        cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, int(cudaSharedmemCarveoutMaxL1));
}

template <typename Kern>
inline void launch_pass(Kern k, const PassArgs& a, int grid, int threads, cudaStream_t st, bool pdl,
                        size_t smem = 0) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(grid));
    cfg.blockDim = dim3(unsigned(threads));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    if (smem == 0) prefer_l1(reinterpret_cast<const void*>(k));
    cudaLaunchKernelEx(&cfg, k, a);
}

}  // namespace pc
