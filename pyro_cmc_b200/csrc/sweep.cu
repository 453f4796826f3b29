// sweep.cu -- colour-sliced Metropolis / overrelaxation passes, energy and
// local-field reductions, energy gradient (sm_100a).
//
// One launch updates one colour class: sublattices that share no bond, so all
// their sites are updated in parallel with the result of a sequential pass in
// storage order (src/MC.cpp:155-163 visits spins[sl*Nc + cell] in order; inside
// one sublattice the order is immaterial because no two of its sites are
// bonded). Spins are float4 (x, y, z, unused) in sublattice-major SoA order,
// so a warp reads 32 consecutive cells of one sublattice: its own spins and
// each neighbour slot are coalesced 512-byte loads. The colour's bond tables
// are staged once per CTA in shared memory; CTAs loop over tiles.
#include <cuda_runtime.h>

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
    const float n2 = h.x * h.x + h.y * h.y + h.z * h.z;
    // a zero local field leaves the spin as it is; so does a zero spin (the
    // reference's default-constructed state, which rotation keeps at zero)
    if (!(n2 > 1e-30f) || !(s0.x * s0.x + s0.y * s0.y + s0.z * s0.z > 0.f)) return false;
    const float av = h.x * s0.x + h.y * s0.y + h.z * s0.z;
    float nx, ny, nz;
    if (REFLECT) {
        const float f = 2.f * av / (n2 + 1e-10f);
        nx = -s0.x + f * h.x;
        ny = -s0.y + f * h.y;
        nz = -s0.z + f * h.z;
    } else {
        const float f = (1.f - cs) * av / n2;
        const float g = sn * rsqrtf(n2);
        nx = cs * s0.x + f * h.x + g * (h.y * s0.z - h.z * s0.y);
        ny = cs * s0.y + f * h.y + g * (h.z * s0.x - h.x * s0.z);
        nz = cs * s0.z + f * h.z + g * (h.x * s0.y - h.y * s0.x);
    }
    const float inv = rsqrtf(nx * nx + ny * ny + nz * nz);
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
    const float r0 = sqrtf(-2.f * logf(u24_open0(w.x)));
    const float r1 = sqrtf(-2.f * logf(u24_open0(w.z)));
    float s_a, c_a, s_b, c_b;
    sincospif(2.f * u24(w.y), &s_a, &c_a);
    sincospif(2.f * u24(w.w), &s_b, &c_b);
    float nx = s0.x + sigma * (r0 * c_a);
    float ny = s0.y + sigma * (r0 * s_a);
    float nz = s0.z + sigma * (r1 * c_b);
    const float inv = rsqrtf(nx * nx + ny * ny + nz * nz);
    nx *= inv;
    ny *= inv;
    nz *= inv;
    const float dE = (nx - s0.x) * h.x + (ny - s0.y) * h.y + (nz - s0.z) * h.z;
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
        sincospif(2.f * u24(w.x), &sn, &cs);
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

// Programmatic dependent launch: let the next kernel on the stream start its
// launch now, then wait until the previous kernel has finished and its writes
// are visible (both are no-ops for a kernel launched without the attribute).
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Generic colour pass: bond tables (any coupling set) staged in shared memory.
template <int MODE>
__global__ void __launch_bounds__(512) colour_pass_kernel(const __grid_constant__ PassArgs a) {
    __shared__ SlTable tab[4];
    __shared__ unsigned int warp_acc[16];
    stage_tables(tab, a.tables, a.n_tab, a.tab_sl);  // tables are never written by kernels
    pdl_enter();
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
    if ((MODE == kMetropolis || MODE >= kFusedRotate) && r_cur >= 0) flush_accepted(a, mine, r_cur, warp_acc);
}

// One site of the structured pass. How the 30 neighbour loads are issued is
// chosen by the autotuner (more loads in flight per thread costs registers,
// hence resident warps):
//   VAR 0: group by group (six short load batches, fewest registers);
//   VAR 1: all 30 at once, before the Philox draw and the proposal (which do
//          not depend on the local field) are computed;
//   VAR 2: J1 + J2 neighbours (18) before the draw, J3 (12) after it.
template <int SL, int VAR>
__device__ __forceinline__ float3 site_field(const float4* __restrict__ S, const PassArgs& a, const ReplicaDev& rep,
                                             const Coords& c, float4 (&v)[kStructNb], int phase) {
    constexpr int kJ3 = grp_begin(SL, 4);
    float3 h = make_float3(0.f, 0.f, 0.f);
    if constexpr (VAR == 0) {
        if (phase == 1) {
            add_group<SL, 0>(h, S, rep.Nc, c, a.mats);
            add_group<SL, 1>(h, S, rep.Nc, c, a.mats);
            add_group<SL, 2>(h, S, rep.Nc, c, a.mats);
            add_group<SL, 3>(h, S, rep.Nc, c, a.mats);
            add_group<SL, 4>(h, S, rep.Nc, c, a.mats);
            add_group<SL, 5>(h, S, rep.Nc, c, a.mats);
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
    const float4 s0 = S[i];
    constexpr bool kMet = MODE == kMetropolis || MODE == kFusedRotate || MODE == kFusedReflect;
    constexpr bool kRot = MODE == kOverrelaxRotate || MODE == kFusedRotate;
    // draws first: they do not depend on the local field, so they overlap the loads
    uint4 w = make_uint4(0, 0, 0, 0);
    float sigma = 0.f, invT = 0.f;
    if (kMet) {
        const double T = a.T_rep[r];
        sigma = sqrtf(float(T) * a.inv_T_ref);
        invT = float(1.0 / T);
        w = site_draw(a.seed, uint32_t(r), sweep, kDrawMetropolis, uint32_t(i));
    }
    float sn = 0.f, cs = 1.f;
    if (kRot) {
        const uint4 wo = site_draw(a.seed, uint32_t(r), sweep, kDrawOverrelax0 + uint32_t(a.or_pass), uint32_t(i));
        sincospif(2.f * u24(wo.x), &sn, &cs);
    } else if (MODE == kOverrelaxTheta) {
        sincosf(float(a.theta[i]), &sn, &cs);
    }
    float4 s1 = s0;
    s1.w = w_after<MODE>(s0.w);
    float nx = 0.f, ny = 0.f, nz = 0.f, u = 0.f;
    if (kMet) {
        const float r0 = sqrtf(-2.f * logf(u24_open0(w.x)));
        const float r1 = sqrtf(-2.f * logf(u24_open0(w.z)));
        float s_a, c_a, s_b, c_b;
        sincospif(2.f * u24(w.y), &s_a, &c_a);
        sincospif(2.f * u24(w.w), &s_b, &c_b);
        nx = s0.x + sigma * (r0 * c_a);
        ny = s0.y + sigma * (r0 * s_a);
        nz = s0.z + sigma * (r1 * c_b);
        const float inv = rsqrtf(nx * nx + ny * ny + nz * nz);
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
        const float dE = (nx - s0.x) * h.x + (ny - s0.y) * h.y + (nz - s0.z) * h.z;
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
    __shared__ unsigned int warp_acc[8];
    pdl_enter();
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
#define PC_CALL(K) accepted = struct_site<MODE, K, VAR>(a, S, rep, r, cell, sweep)
            PC_SL_SWITCH(sl, PC_CALL)
#undef PC_CALL
            mine += accepted ? 1u : 0u;
        }
    }
    if ((MODE == kMetropolis || MODE >= kFusedRotate) && r_cur >= 0) flush_accepted(a, mine, r_cur, warp_acc);
}

// ---------------------------------------------------- staged colour pass
// Load variant 3: a CTA updates one tile of R x-rows of one sublattice
// (cells cx in [0, L), cy in [cy0, cy0 + R), fixed cz). Every neighbour of
// those sites lies in one of the sublattice's 24 neighbour rows (kRows) over
// the same R rows shifted by (dy, dz), at x offset -1, 0 or +1. Thread 0 stages
// the 24 row blocks (R*L float4 each, two pieces where the block wraps in y)
// into shared memory with bulk asynchronous copies that complete on one
// mbarrier; meanwhile every thread loads its own spin and draws its random
// numbers. After the barrier the 30 neighbour reads come from shared memory.
// All copies of a tile are in flight at once, with no registers held for them.

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for phase `parity`: false if it did not complete within
// kMaxPolls polls (each poll is a hardware-timed try_wait).
constexpr int kMaxPolls = 1 << 22;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (int i = 0; i < kMaxPolls; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// Global -> shared bulk copy (16-byte aligned addresses, size a multiple of 16)
// completing `bytes` transactions on the mbarrier.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Row block U of sublattice SL for the tile: rows cy0 + dy .. cy0 + dy + R - 1
// (mod L) of plane cz + dz of sublattice s2 -> rows[U][0..R)[0..L).
template <int SL, int U>
__device__ __forceinline__ void issue_row(float4* rows, const float4* S, int Nc, int L, int cy0, int cz, int R,
                                          uint64_t* bar) {
    constexpr int s2 = row_s2(SL, U), dy = row_dy(SL, U), dz = row_dz(SL, U);
    const int z = wrap1(cz + dz, L);
    const int ys = wrap1(cy0 + dy, L);
    const float4* base = S + size_t(s2) * Nc + size_t(z) * L * L;
    float4* dst = rows + size_t(U) * R * L;
    const int n1 = min(R, L - ys);
    bulk_copy_g2s(dst, base + size_t(ys) * L, uint32_t(n1 * L * 16), bar);
    if (R > n1) bulk_copy_g2s(dst + size_t(n1) * L, base, uint32_t((R - n1) * L * 16), bar);
}
template <int SL, int... U>
__device__ __forceinline__ void issue_rows(float4* rows, const float4* S, int Nc, int L, int cy0, int cz, int R,
                                           uint64_t* bar, std::integer_sequence<int, U...>) {
    (issue_row<SL, U>(rows, S, Nc, L, cy0, cz, R, bar), ...);
}

__device__ __forceinline__ void add_xyz(float3& t, float4 v) {
    t.x += v.x;
    t.y += v.y;
    t.z += v.z;
}

struct RowPos {
    int base;        // (rho) * L: offset of the site's row inside one row block
    int RL;          // R * L: size of one row block
    int xm, x0, xp;  // wrapped cx - 1, cx, cx + 1
};
template <int SL, int E>
__device__ __forceinline__ float4 row_nb(const float4* rows, const RowPos& q) {
    constexpr int u = row_of(SL, E), dx = nb_dx(SL, E);
    const int x = dx < 0 ? q.xm : (dx > 0 ? q.xp : q.x0);
    return rows[u * q.RL + q.base + x];
}
template <int SL, int G, int... K>
__device__ __forceinline__ float3 row_group_sum(const float4* rows, const RowPos& q, std::integer_sequence<int, K...>) {
    constexpr int B = grp_begin(SL, G);
    float3 t = make_float3(0.f, 0.f, 0.f);
    (add_xyz(t, row_nb<SL, B + K>(rows, q)), ...);
    return t;
}
template <int SL, int G>
__device__ __forceinline__ void row_add_group(float3& h, const float4* rows, const RowPos& q, const PyroMats& mats) {
    if (mats.active[SL] & (1u << G)) {
        const float3 t = row_group_sum<SL, G>(rows, q, std::make_integer_sequence<int, grp_size(SL, G)>{});
        const float* J = mats.M[SL][G];
        h.x += J[0] * t.x + J[1] * t.y + J[2] * t.z;
        h.y += J[3] * t.x + J[4] * t.y + J[5] * t.z;
        h.z += J[6] * t.x + J[7] * t.y + J[8] * t.z;
    }
}
template <int SL>
__device__ __forceinline__ float3 row_field(const float4* rows, const RowPos& q, const PyroMats& mats) {
    float3 h = make_float3(0.f, 0.f, 0.f);
    row_add_group<SL, 0>(h, rows, q, mats);
    row_add_group<SL, 1>(h, rows, q, mats);
    row_add_group<SL, 2>(h, rows, q, mats);
    row_add_group<SL, 3>(h, rows, q, mats);
    row_add_group<SL, 4>(h, rows, q, mats);
    row_add_group<SL, 5>(h, rows, q, mats);
    return h;
}

// One tile of sublattice SL; returns 1 if this thread's Metropolis proposal
// was accepted. Every thread of the CTA calls it (barrier inside).
template <int MODE, int SL>
__device__ __forceinline__ unsigned staged_tile(const PassArgs& a, const Tile tile, const ReplicaDev& rep, int r,
                                                float4* rows, uint64_t* bar, uint64_t sweep) {
    const int L = rep.L, Nc = rep.Nc, R = tile.w, row0 = tile.z;
    const int cz = fdiv(row0, rep.divL), cy0 = row0 - cz * L;
    const int RL = R * L;
    float4* S = a.spins + rep.off;
    constexpr int U = rows_n(SL);
    if (threadIdx.x == 0) {
        mbar_expect_tx(bar, uint32_t(U * RL * 16));
        issue_rows<SL>(rows, S, Nc, L, cy0, cz, R, bar, std::make_integer_sequence<int, U>{});
    }
    const int t = threadIdx.x;
    const bool live = t < RL;
    const size_t i = size_t(SL) * Nc + size_t(row0) * L + (live ? t : 0);
    const float4 s0 = live ? S[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    constexpr bool kMet = MODE == kMetropolis || MODE == kFusedRotate || MODE == kFusedReflect;
    constexpr bool kRot = MODE == kOverrelaxRotate || MODE == kFusedRotate;
    // draws and the proposal before the barrier: they overlap the copies
    float nx = 0.f, ny = 0.f, nz = 0.f, u = 0.f, invT = 0.f;
    if (kMet && live) {
        const double T = a.T_rep[r];
        const float sigma = sqrtf(float(T) * a.inv_T_ref);
        invT = float(1.0 / T);
        const uint4 w = site_draw(a.seed, uint32_t(r), sweep, kDrawMetropolis, uint32_t(i));
        const float r0 = sqrtf(-2.f * logf(u24_open0(w.x)));
        const float r1 = sqrtf(-2.f * logf(u24_open0(w.z)));
        float s_a, c_a, s_b, c_b;
        sincospif(2.f * u24(w.y), &s_a, &c_a);
        sincospif(2.f * u24(w.w), &s_b, &c_b);
        nx = s0.x + sigma * (r0 * c_a);
        ny = s0.y + sigma * (r0 * s_a);
        nz = s0.z + sigma * (r1 * c_b);
        const float inv = rsqrtf(nx * nx + ny * ny + nz * nz);
        nx *= inv;
        ny *= inv;
        nz *= inv;
        u = u24_lowbytes(w);
    }
    float sn = 0.f, cs = 1.f;
    if (live) {
        if (kRot) {
            const uint4 wo = site_draw(a.seed, uint32_t(r), sweep, kDrawOverrelax0 + uint32_t(a.or_pass), uint32_t(i));
            sincospif(2.f * u24(wo.x), &sn, &cs);
        } else if (MODE == kOverrelaxTheta) {
            sincosf(float(a.theta[i]), &sn, &cs);
        }
    }
    if (!mbar_wait_bounded(bar, 0)) {
        // the copies did not land: report, give them one more bounded wait, skip the update
        if (threadIdx.x == 0) atomicExch(a.err, 1);
        mbar_wait_bounded(bar, 0);
        return 0u;
    }
    if (!live) return 0u;
    const int rho = fdiv(t, rep.divL), cx = t - rho * L;
    RowPos q;
    q.base = rho * L;
    q.RL = RL;
    q.x0 = cx;
    q.xm = cx == 0 ? L - 1 : cx - 1;
    q.xp = cx == L - 1 ? 0 : cx + 1;
    float3 h = row_field<SL>(rows, q, a.mats);
    h.x -= a.B[0];
    h.y -= a.B[1];
    h.z -= a.B[2];
    if constexpr (MODE == kLifted || MODE == kLiftedRot) {
        float4 s1;
        const bool lacc = lifted_spin<MODE == kLiftedRot>(a, s0, h, r, sweep, i, s1);
        S[i] = s1;
        return lacc ? 1u : 0u;
    }
    bool acc = false;
    float4 s1 = s0;
    s1.w = w_after<MODE>(s0.w);
    if (kMet) {
        const float dE = (nx - s0.x) * h.x + (ny - s0.y) * h.y + (nz - s0.z) * h.z;
        if (dE < 0.f || u < __expf(-dE * invT)) {
            s1 = make_float4(nx, ny, nz, w_after<MODE>(s0.w));
            acc = true;
        }
        if (MODE == kMetropolis) {
            if (acc) S[i] = s1;
            return acc ? 1u : 0u;
        }
    }
    float4 s2;
    const bool moved = overrelax_spin<MODE == kOverrelaxReflect || MODE == kFusedReflect>(s1, h, sn, cs, s2);
    if (moved)
        S[i] = s2;
    else if (acc)
        S[i] = s1;
    return acc ? 1u : 0u;
}

// One CTA per row tile; dynamic shared memory = 24 row blocks of the largest tile.
template <int MODE>
__global__ void __launch_bounds__(256) staged_pass_kernel(const __grid_constant__ PassArgs a) {
    extern __shared__ __align__(128) float4 rows[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ unsigned int warp_acc[8];
    const Tile tile = a.tiles[blockIdx.x];
    const int r = tile.x, sl = tile.y & 0xff;
    const ReplicaDev rep = a.reps[r];
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    pdl_enter();  // spins are read only after the previous kernel finished
    const uint64_t sweep = *a.sweep_base + a.sweep_offset;
    unsigned mine = 0;
#define PC_CALL(K) mine = staged_tile<MODE, K>(a, tile, rep, r, rows, &bar, sweep)
    PC_SL_SWITCH(sl, PC_CALL)
#undef PC_CALL
    if (MODE == kMetropolis || MODE >= kFusedRotate) flush_accepted(a, mine, r, warp_acc);
}

size_t staged_smem_bytes(int max_rl) { return size_t(max_rows()) * size_t(max_rl) * sizeof(float4); }

template <int MODE>
static void prepare_staged() {
    cudaFuncSetAttribute(staged_pass_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         int(staged_smem_bytes(256)));
}
void staged_prepare() {
    prepare_staged<kMetropolis>();
    prepare_staged<kOverrelaxRotate>();
    prepare_staged<kOverrelaxReflect>();
    prepare_staged<kOverrelaxTheta>();
    prepare_staged<kFusedRotate>();
    prepare_staged<kFusedReflect>();
    prepare_staged<kLifted>();
    prepare_staged<kLiftedRot>();
}

template <typename Kern>
static void launch_pass(Kern k, const PassArgs& a, int grid, int threads, cudaStream_t st, bool pdl,
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
    cudaLaunchKernelEx(&cfg, k, a);
}

template <int VAR>
static void launch_struct(PassMode mode, const PassArgs& a, int grid, int threads, cudaStream_t st, bool pdl) {
    switch (mode) {
        case kMetropolis: launch_pass(struct_pass_kernel<kMetropolis, VAR>, a, grid, threads, st, pdl); break;
        case kOverrelaxRotate: launch_pass(struct_pass_kernel<kOverrelaxRotate, VAR>, a, grid, threads, st, pdl); break;
        case kOverrelaxReflect: launch_pass(struct_pass_kernel<kOverrelaxReflect, VAR>, a, grid, threads, st, pdl); break;
        case kOverrelaxTheta: launch_pass(struct_pass_kernel<kOverrelaxTheta, VAR>, a, grid, threads, st, pdl); break;
        case kFusedRotate: launch_pass(struct_pass_kernel<kFusedRotate, VAR>, a, grid, threads, st, pdl); break;
        case kFusedReflect: launch_pass(struct_pass_kernel<kFusedReflect, VAR>, a, grid, threads, st, pdl); break;
        case kLifted: launch_pass(struct_pass_kernel<kLifted, VAR>, a, grid, threads, st, pdl); break;
        case kLiftedRot: launch_pass(struct_pass_kernel<kLiftedRot, VAR>, a, grid, threads, st, pdl); break;
    }
}

static void launch_staged(PassMode mode, const PassArgs& a, int threads, cudaStream_t st, bool pdl) {
    const size_t smem = staged_smem_bytes(a.staged_rl);
    const int grid = a.n_tiles;  // one CTA per row tile
    switch (mode) {
        case kMetropolis: launch_pass(staged_pass_kernel<kMetropolis>, a, grid, threads, st, pdl, smem); break;
        case kOverrelaxRotate: launch_pass(staged_pass_kernel<kOverrelaxRotate>, a, grid, threads, st, pdl, smem); break;
        case kOverrelaxReflect: launch_pass(staged_pass_kernel<kOverrelaxReflect>, a, grid, threads, st, pdl, smem); break;
        case kOverrelaxTheta: launch_pass(staged_pass_kernel<kOverrelaxTheta>, a, grid, threads, st, pdl, smem); break;
        case kFusedRotate: launch_pass(staged_pass_kernel<kFusedRotate>, a, grid, threads, st, pdl, smem); break;
        case kFusedReflect: launch_pass(staged_pass_kernel<kFusedReflect>, a, grid, threads, st, pdl, smem); break;
        case kLifted: launch_pass(staged_pass_kernel<kLifted>, a, grid, threads, st, pdl, smem); break;
        case kLiftedRot: launch_pass(staged_pass_kernel<kLiftedRot>, a, grid, threads, st, pdl, smem); break;
    }
}

void launch_colour_pass(PassMode mode, const PassArgs& a, int grid, int threads, cudaStream_t st, bool pdl) {
    if (a.structured && a.load_variant == 3) {
        launch_staged(mode, a, threads, st, pdl);
        return;
    }
    if (a.structured && threads <= 256) {
        if (a.load_variant == 1)
            launch_struct<1>(mode, a, grid, threads, st, pdl);
        else if (a.load_variant == 2)
            launch_struct<2>(mode, a, grid, threads, st, pdl);
        else
            launch_struct<0>(mode, a, grid, threads, st, pdl);
        return;
    }
    switch (mode) {
        case kMetropolis: launch_pass(colour_pass_kernel<kMetropolis>, a, grid, threads, st, pdl); break;
        case kOverrelaxRotate: launch_pass(colour_pass_kernel<kOverrelaxRotate>, a, grid, threads, st, pdl); break;
        case kOverrelaxReflect: launch_pass(colour_pass_kernel<kOverrelaxReflect>, a, grid, threads, st, pdl); break;
        case kOverrelaxTheta: launch_pass(colour_pass_kernel<kOverrelaxTheta>, a, grid, threads, st, pdl); break;
        case kFusedRotate: launch_pass(colour_pass_kernel<kFusedRotate>, a, grid, threads, st, pdl); break;
        case kFusedReflect: launch_pass(colour_pass_kernel<kFusedReflect>, a, grid, threads, st, pdl); break;
        case kLifted: launch_pass(colour_pass_kernel<kLifted>, a, grid, threads, st, pdl); break;
        case kLiftedRot: launch_pass(colour_pass_kernel<kLiftedRot>, a, grid, threads, st, pdl); break;
    }
}

// ------------------------------------------------------------- reductions
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of NV doubles; result valid in thread 0. `red` holds
// NV * 32 doubles.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; ++j) v[j] = warp_sum(v[j]);
    if (lane == 0)
#pragma unroll
        for (int j = 0; j < NV; ++j) red[j * 32 + warp] = v[j];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            double x = lane < nw ? red[j * 32 + lane] : 0.0;
            v[j] = warp_sum(x);
        }
    }
    __syncthreads();
}

// Energy terms per tile (total_energy_per_unit_cell, src/MC.cpp:305-312):
// sum_i 0.5 S_i.h_i - S_i.B, plus sum_i S_i. Every sublattice of every
// replica; tables staged per tile (one sublattice per tile).
__global__ void __launch_bounds__(512) energy_partials_kernel(const __grid_constant__ EnergyArgs a) {
    __shared__ SlTable tab;
    __shared__ double red[4 * 32];
    for (int t = blockIdx.x; t < a.n_tiles; t += gridDim.x) {
        const Tile tile = a.tiles[t];
        const int r = tile.x, sl = tile.y & 0xff;
        __syncthreads();
        stage_tables(&tab, a.tables, 1, &sl);
        __syncthreads();
        const ReplicaDev rep = a.reps[r];
        const int L = rep.L, Nc = rep.Nc;
        const float4* S = a.spins + rep.off;
        double v[4] = {0, 0, 0, 0};
        if (int(threadIdx.x) < tile.w) {
            const int cell = tile.z + int(threadIdx.x);
            const int cx = cell % L, cy = (cell / L) % L, cz = cell / (L * L);
            const float4 s0 = S[size_t(sl) * Nc + cell];
            const float3 h = local_field(S, tab, cx, cy, cz, L, Nc);
            v[0] = 0.5 * double(s0.x * h.x + s0.y * h.y + s0.z * h.z) -
                   double(s0.x * a.B[0] + s0.y * a.B[1] + s0.z * a.B[2]);
            v[1] = s0.x;
            v[2] = s0.y;
            v[3] = s0.z;
        }
        block_sum<4>(v, red);
        if (threadIdx.x == 0)
            for (int j = 0; j < 4; ++j) a.partial[size_t(t) * 4 + j] = v[j];
    }
}

template <int SL>
__device__ __forceinline__ float3 struct_field_e(const EnergyArgs& a, const float4* S, const ReplicaDev& rep, int cell) {
    return struct_field<SL>(S, a.mats, cell, rep.L, rep.Nc, rep.divL);
}

__global__ void __launch_bounds__(256) energy_struct_kernel(const __grid_constant__ EnergyArgs a) {
    __shared__ double red[4 * 32];
    for (int t = blockIdx.x; t < a.n_tiles; t += gridDim.x) {
        const Tile tile = a.tiles[t];
        const int r = tile.x, sl = tile.y & 0xff;
        const ReplicaDev rep = a.reps[r];
        const float4* S = a.spins + rep.off;
        double v[4] = {0, 0, 0, 0};
        if (int(threadIdx.x) < tile.w) {
            const int cell = tile.z + int(threadIdx.x);
            const float4 s0 = S[size_t(sl) * rep.Nc + cell];
            float3 h = make_float3(0.f, 0.f, 0.f);
#define PC_CALL(K) h = struct_field_e<K>(a, S, rep, cell)
            PC_SL_SWITCH(sl, PC_CALL)
#undef PC_CALL
            v[0] = 0.5 * double(s0.x * h.x + s0.y * h.y + s0.z * h.z) -
                   double(s0.x * a.B[0] + s0.y * a.B[1] + s0.z * a.B[2]);
            v[1] = s0.x;
            v[2] = s0.y;
            v[3] = s0.z;
        }
        block_sum<4>(v, red);
        if (threadIdx.x == 0)
            for (int j = 0; j < 4; ++j) a.partial[size_t(t) * 4 + j] = v[j];
    }
}

void launch_energy_partials(const EnergyArgs& a, int threads, cudaStream_t st) {
    // one CTA per tile: many resident CTAs per SM hide the neighbour-gather latency
    const int grid = a.n_tiles;
    if (a.structured && threads <= 256)
        energy_struct_kernel<<<grid, threads, 0, st>>>(a);
    else
        energy_partials_kernel<<<grid, threads, 0, st>>>(a);
}

// One block per replica: each thread sums a fixed strided subset of the
// replica's tile partials, then a fixed-shape tree combines them, so the
// result does not depend on scheduling (deterministic).
__global__ void __launch_bounds__(1024) energy_finalize_kernel(const double* partial, const int32_t* tb,
                                                              const int32_t* te, const ReplicaDev* reps, int R,
                                                              double* e, double* mag) {
    __shared__ double red[4 * 32];
    const int r = blockIdx.x;
    if (r >= R) return;
    double v[4] = {0, 0, 0, 0};
    const double4* p4 = reinterpret_cast<const double4*>(partial);
#pragma unroll 8
    for (int t = tb[r] + int(threadIdx.x); t < te[r]; t += blockDim.x) {
        const double4 q = p4[t];
        v[0] += q.x;
        v[1] += q.y;
        v[2] += q.z;
        v[3] += q.w;
    }
    block_sum<4>(v, red);
    if (threadIdx.x == 0) {
        e[r] = v[0] / double(reps[r].Nc);
        if (mag)
            for (int j = 0; j < 3; ++j) mag[3 * r + j] = v[1 + j];
    }
}

void launch_energy_finalize(const double* partial, const int32_t* tile_begin, const int32_t* tile_end,
                            const ReplicaDev* reps, int R, double* e, double* mag, cudaStream_t st) {
    energy_finalize_kernel<<<R, 1024, 0, st>>>(partial, tile_begin, tile_end, reps, R, e, mag);
}

__global__ void __launch_bounds__(512) local_field_kernel(const FieldArgs a) {
    __shared__ SlTable tab;
    for (int t = blockIdx.x; t < a.n_tiles; t += gridDim.x) {
        const Tile tile = a.tiles[t];
        const int r = tile.x, sl = tile.y & 0xff;
        __syncthreads();
        stage_tables(&tab, a.tables, 1, &sl);
        __syncthreads();
        const ReplicaDev rep = a.reps[r];
        if (int(threadIdx.x) < tile.w) {
            const int L = rep.L, Nc = rep.Nc;
            const int cell = tile.z + int(threadIdx.x);
            const int cx = cell % L, cy = (cell / L) % L, cz = cell / (L * L);
            const float3 h = local_field(a.spins + rep.off, tab, cx, cy, cz, L, Nc);
            a.h_out[rep.off + size_t(sl) * Nc + cell] = make_float4(h.x, h.y, h.z, 0.f);
        }
    }
}

void launch_local_field(const FieldArgs& a, int threads, cudaStream_t st) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = a.n_tiles < sms * 4 ? a.n_tiles : sms * 4;
    local_field_kernel<<<grid, threads, 0, st>>>(a);
}

// Energy gradient. Per site: grad_S = g/Nc (h - B). Per shell (spec c, J or
// J^T side): 0.5 S_i (x) t (source side) or 0.5 t (x) S_i (target side), with
// t the shell's neighbour sum; over all sites this is sum over the spec's bonds
// of S_src (x) S_tgt = dE/dJ_spec. Partial layout per tile:
// [0] energy sum, [1..3] sum S, [4 + 9c + 3a + b] dE/dJ_c[a][b].
__global__ void __launch_bounds__(256) energy_grad_kernel(const GradArgs a) {
    __shared__ SlTable tab;
    extern __shared__ double acc[];  // [4 + 9*n_spec]
    const int width = 4 + 9 * a.n_spec;
    const int lane = threadIdx.x & 31;
    for (int t = blockIdx.x; t < a.n_tiles; t += gridDim.x) {
        const Tile tile = a.tiles[t];
        const int r = tile.x, sl = tile.y & 0xff;
        __syncthreads();
        stage_tables(&tab, a.tables, 1, &sl);
        for (int j = threadIdx.x; j < width; j += blockDim.x) acc[j] = 0.0;
        __syncthreads();
        const ReplicaDev rep = a.reps[r];
        const int L = rep.L, Nc = rep.Nc;
        const float4* S = a.spins + rep.off;
        const bool live = int(threadIdx.x) < tile.w;
        const int cell = tile.z + int(threadIdx.x);
        const int cx = cell % L, cy = (cell / L) % L, cz = cell / (L * L);
        float4 s0 = make_float4(0, 0, 0, 0);
        if (live) s0 = S[size_t(sl) * Nc + cell];
        float hx = 0.f, hy = 0.f, hz = 0.f;
        int e = 0;
        for (int k = 0; k < tab.n_shell; ++k) {
            float tx = 0.f, ty = 0.f, tz = 0.f;
            const int end = tab.shell_end[k];
            for (; e < end; ++e) {
                if (!live) continue;
                const NbEntry nb = tab.nb[e];
                const int x = wrap1(cx + nb.dx, L), y = wrap1(cy + nb.dy, L), z = wrap1(cz + nb.dz, L);
                const float4 o = __ldg(&S[size_t(nb.sl) * Nc + x + L * (y + L * z)]);
                tx += o.x;
                ty += o.y;
                tz += o.z;
            }
            const float* J = tab.J[k];
            hx += J[0] * tx + J[1] * ty + J[2] * tz;
            hy += J[3] * tx + J[4] * ty + J[5] * tz;
            hz += J[6] * tx + J[7] * ty + J[8] * tz;
            const int spec = tab.shell_spec[k] % 1000;
            const bool tr = tab.shell_spec[k] >= 1000;
            const float sv[3] = {s0.x, s0.y, s0.z};
            const float tv[3] = {tx, ty, tz};
#pragma unroll
            for (int p = 0; p < 3; ++p)
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    double v = 0.5 * double(tr ? tv[p] * sv[q] : sv[p] * tv[q]);
                    v = warp_sum(v);
                    if (lane == 0) atomicAdd(&acc[4 + 9 * spec + 3 * p + q], v);
                }
        }
        double ev = 0.0;
        if (live) {
            ev = 0.5 * double(s0.x * hx + s0.y * hy + s0.z * hz) -
                 double(s0.x * a.B[0] + s0.y * a.B[1] + s0.z * a.B[2]);
            if (a.grad_S) {
                const float gs = float(a.g[r] / double(Nc));
                a.grad_S[rep.off + size_t(sl) * Nc + cell] =
                    make_float4(gs * (hx - a.B[0]), gs * (hy - a.B[1]), gs * (hz - a.B[2]), 0.f);
            }
        }
        const double v4[4] = {ev, s0.x, s0.y, s0.z};
        for (int j = 0; j < 4; ++j) {
            const double v = warp_sum(v4[j]);
            if (lane == 0) atomicAdd(&acc[j], v);
        }
        __syncthreads();
        for (int j = threadIdx.x; j < width; j += blockDim.x) a.partial[size_t(t) * width + j] = acc[j];
    }
}

void launch_energy_grad_partials(const GradArgs& a, int threads, cudaStream_t st) {
    const int grid = a.n_tiles;  // one CTA per tile
    const size_t smem = sizeof(double) * size_t(4 + 9 * a.n_spec);
    energy_grad_kernel<<<grid, threads, smem, st>>>(a);
}

__global__ void grad_finalize_kernel(const double* partial, int width, const int32_t* tb, const int32_t* te, int R,
                                     double* out) {
    const int r = blockIdx.x;
    for (int j = threadIdx.x; j < width; j += blockDim.x) {
        double v = 0.0;
        for (int t = tb[r]; t < te[r]; ++t) v += partial[size_t(t) * width + j];
        out[size_t(r) * width + j] = v;
    }
}

void launch_grad_finalize(const double* partial, int width, const int32_t* tile_begin, const int32_t* tile_end, int R,
                          double* out, cudaStream_t st) {
    grad_finalize_kernel<<<R, 128, 0, st>>>(partial, width, tile_begin, tile_end, R, out);
}

// Uniform on S^2: z = 1 - 2u, phi = 2 pi u'.
__global__ void random_spins_kernel(float4* spins, const ReplicaDev* reps, const Tile* tiles, int n_tiles,
                                    uint64_t seed) {
    for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const Tile tile = tiles[t];
        if (int(threadIdx.x) >= tile.w) continue;
        const int r = tile.x, sl = tile.y & 0xff;
        const ReplicaDev rep = reps[r];
        const size_t i = size_t(sl) * rep.Nc + tile.z + threadIdx.x;
        const uint4 w = site_draw(seed, uint32_t(r), 0, kDrawInit, uint32_t(i));
        const float z = 1.f - 2.f * u24(w.x);
        float sn, cs;
        sincospif(2.f * u24(w.y), &sn, &cs);
        const float rho = sqrtf(fmaxf(0.f, 1.f - z * z));
        spins[rep.off + i] = make_float4(rho * cs, rho * sn, z, 0.f);
    }
}

void launch_random_spins(float4* spins, const ReplicaDev* reps, const Tile* tiles, int n_tiles, uint64_t seed,
                         int threads, cudaStream_t st) {
    const int grid = n_tiles < 4096 ? n_tiles : 4096;
    random_spins_kernel<<<grid, threads, 0, st>>>(spins, reps, tiles, n_tiles, seed);
}

__global__ void advance_counter_kernel(uint64_t* c, uint64_t n) { *c += n; }
void launch_advance_counter(uint64_t* counter, uint64_t n, cudaStream_t st) {
    advance_counter_kernel<<<1, 1, 0, st>>>(counter, n);
}

}  // namespace pc
