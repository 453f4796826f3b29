// sweep_staged.cu -- load variant 3 of the structured colour pass: neighbour
// rows staged into shared memory by bulk asynchronous copies (sm_100a).
#include <cuda_runtime.h>

#include <mutex>
#include <set>
#include <utility>

#include "moves.cuh"

namespace pc {

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
// `polls` polls (each poll is a hardware-timed try_wait).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int polls) {
    for (int i = 0; i < polls; ++i)
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
        add_matvec(h, J, t);
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
    float sn = 0.f, cs = 1.f;
    if (live) {
        if (kRot) {
            const uint4 wo = site_draw(a.seed, uint32_t(r), sweep, kDrawOverrelax0 + uint32_t(a.or_pass), uint32_t(i));
            uniform_angle(wo.x, &sn, &cs);
        } else if (MODE == kOverrelaxTheta) {
            sincosf(float(a.theta[i]), &sn, &cs);
        }
    }
    if (!mbar_wait_bounded(bar, 0, a.wait_polls)) {
        // the copies did not land: report, give them one more wait (at the
        // full bound, so none is left writing into this CTA's shared memory
        // after it exits), skip the update
        if (threadIdx.x == 0) atomicExch(a.err, 1);
        mbar_wait_bounded(bar, 0, kStagedMaxPolls);
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
        const float dE = dot3_rn(nx - s0.x, ny - s0.y, nz - s0.z, h.x, h.y, h.z);
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
    pdl_wait();  // spins are read only after the previous kernel finished
    const uint64_t sweep = *a.sweep_base + a.sweep_offset;
    unsigned mine = 0;
#define PC_CALL(K) mine = staged_tile<MODE, K>(a, tile, rep, r, rows, &bar, sweep)
    PC_SL_SWITCH(sl, PC_CALL)
#undef PC_CALL
    pdl_trigger();
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

// The shared-memory limit of the staged kernels is raised on their first use on
// a device, not at setup: systems that never use load variant 3 never load
// this module.
void launch_staged(PassMode mode, const PassArgs& a, int threads, cudaStream_t st, bool pdl) {
    {
        static std::mutex mu;
        static std::set<int> ready;
        int dev = 0;
        cudaGetDevice(&dev);
        std::lock_guard<std::mutex> lock(mu);
        if (ready.insert(dev).second) staged_prepare();
    }
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

}  // namespace pc
