// sweep_cluster.cu -- cluster-resident sweeps for small lattices (sm_100a).
//
// A lattice of L <= 16 (16 L^3 float4, 64 KB at L = 16) fits in the
// distributed shared memory of one thread-block cluster: CTA z of the
// cluster holds z plane z of all 16 sublattices ([16][L*L] float4) and one
// thread per cell of its plane. The spins are read from HBM once, every
// colour pass of n_sweeps sweeps runs in the same launch with the neighbour
// gathers served from shared memory (the planes z-1 and z+1 of the cluster
// peers through their shared::cluster windows), a cluster barrier
// (release/acquire) between passes, and the spins are written back once.
// Small single lattices are otherwise bound by one kernel launch per colour
// pass (4096 sites per pass at L = 16).
//
// The chain is the colour-pass chain of sweep.cu: the same passes in the same
// order, the same Philox draws keyed by (seed, replica, sweep, draw, site), the
// same move arithmetic and the same group-by-group local field. The two
// compilations may contract multiply-adds differently, so the chains agree up
// to rounding (measured: identical for the first sublattices of a sweep, then
// last-bit differences of 1e-7..1e-6).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <utility>

#include "common.cuh"
#include "kernels.h"
#include "moves.cuh"
#include "struct_field.cuh"

namespace cg = cooperative_groups;

namespace pc {

// Neighbour E of sublattice SL from the cluster planes: P[dz + 1] is plane
// z + dz (own plane for dz = 0), x and y wrapped as in Coords.
template <int SL, int E>
__device__ __forceinline__ float4 cl_load_nb(const float4* const (&P)[3], int LL, const Coords& c) {
    constexpr int s2 = nb_sl(SL, E), dx = nb_dx(SL, E), dy = nb_dy(SL, E), dz = nb_dz(SL, E);
    return P[dz + 1][s2 * LL + pick<dx>(c.x) + pick<dy>(c.y)];
}
template <int SL, int... E>
__device__ __forceinline__ void cl_load_all(float4 (&v)[kStructNb], const float4* const (&P)[3], int LL,
                                            const Coords& c, std::integer_sequence<int, E...>) {
    ((v[E] = cl_load_nb<SL, E>(P, LL, c)), ...);
}
// add_group (struct_field.cuh) on loaded neighbours: the group's sum in
// neighbour order, then the group matrix
template <int SL, int G>
__device__ __forceinline__ void cl_add_group(float3& h, const float4 (&v)[kStructNb], const PyroMats& mats) {
    if (mats.active[SL] & (1u << G)) {
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
}

// What a site's move needs besides its local field, formed before the field
// (struct_site, sweep.cu): the spin, the Metropolis proposal and acceptance
// uniform, the overrelaxation angle.
struct Proposal {
    float4 s0;
    float nx, ny, nz, u, invT, sn, cs;
};

template <int MODE>
__device__ __forceinline__ Proposal cl_prepare(const ClusterArgs& a, const float4* own, int own_idx, int r,
                                               uint64_t sweep, int or_pass, size_t i) {
    constexpr bool kMet = MODE == kMetropolis || MODE == kFusedRotate || MODE == kFusedReflect;
    constexpr bool kRot = MODE == kOverrelaxRotate || MODE == kFusedRotate;
    Proposal p;
    p.s0 = own[own_idx];
    const float4 s0 = p.s0;
    uint4 w = make_uint4(0, 0, 0, 0);
    float sigma = 0.f;
    p.invT = 0.f;
    if (kMet) {
        const double T = a.T_rep[r];
        sigma = sqrtf(float(T) * a.inv_T_ref);
        p.invT = float(1.0 / T);
        w = site_draw(a.seed, uint32_t(r), sweep, kDrawMetropolis, uint32_t(i));
    }
    p.sn = 0.f;
    p.cs = 1.f;
    if (kRot) {
        const uint4 wo = site_draw(a.seed, uint32_t(r), sweep, kDrawOverrelax0 + uint32_t(or_pass), uint32_t(i));
        uniform_angle(wo.x, &p.sn, &p.cs);
    }
    p.nx = p.ny = p.nz = p.u = 0.f;
    if (kMet) {
        const float r0 = bm_radius(w.x);
        const float r1 = bm_radius(w.z);
        float s_a, c_a, s_b, c_b;
        uniform_angle(w.y, &s_a, &c_a);
        uniform_angle(w.w, &s_b, &c_b);
        float nx = fmaf(sigma, __fmul_rn(r0, c_a), s0.x);
        float ny = fmaf(sigma, __fmul_rn(r0, s_a), s0.y);
        float nz = fmaf(sigma, __fmul_rn(r1, c_b), s0.z);
        const float inv = rsqrtf(dot3_rn(nx, ny, nz, nx, ny, nz));
        p.nx = nx * inv;
        p.ny = ny * inv;
        p.nz = nz * inv;
        p.u = u24_lowbytes(w);
    }
    return p;
}

// The site's local field from the cluster planes (all 30 neighbour loads in
// flight at once) and its move; returns whether a Metropolis proposal was
// accepted.
template <int MODE, int SL>
__device__ __forceinline__ bool cl_finish(const ClusterArgs& a, float4* own, int own_idx, const float4* const (&P)[3],
                                          int LL, const Coords& c, const Proposal& p) {
    constexpr bool kMet = MODE == kMetropolis || MODE == kFusedRotate || MODE == kFusedReflect;
    float4 v[kStructNb];
    cl_load_all<SL>(v, P, LL, c, std::make_integer_sequence<int, kStructNb>{});
    float3 h = make_float3(0.f, 0.f, 0.f);
    cl_add_group<SL, 0>(h, v, a.mats);
    cl_add_group<SL, 1>(h, v, a.mats);
    cl_add_group<SL, 2>(h, v, a.mats);
    cl_add_group<SL, 3>(h, v, a.mats);
    cl_add_group<SL, 4>(h, v, a.mats);
    cl_add_group<SL, 5>(h, v, a.mats);
    h.x -= a.B[0];
    h.y -= a.B[1];
    h.z -= a.B[2];
    const float4 s0 = p.s0;
    float4 s1 = s0;
    s1.w = w_after<MODE>(s0.w);
    bool acc = false;
    if (kMet) {
        const float dE = dot3_rn(p.nx - s0.x, p.ny - s0.y, p.nz - s0.z, h.x, h.y, h.z);
        if (dE < 0.f || p.u < __expf(-dE * p.invT)) {
            s1 = make_float4(p.nx, p.ny, p.nz, w_after<MODE>(s0.w));
            acc = true;
        }
        if (MODE == kMetropolis) {
            if (acc) own[own_idx] = s1;
            return acc;
        }
    }
    float4 s2;
    const bool moved = overrelax_spin<MODE == kOverrelaxReflect || MODE == kFusedReflect>(s1, h, p.sn, p.cs, s2);
    if (moved)
        own[own_idx] = s2;
    else if (acc)
        own[own_idx] = s1;
    return acc;
}

// Per sublattice: one out-of-line function per move mode (the 16 inlined
// neighbour structures of one mode in one function keep the kernel's own
// register allocation small).
template <int MODE>
__device__ __noinline__ bool cl_finish_sl(int sl, const ClusterArgs& a, float4* own, int own_idx,
                                          const float4* const (&P)[3], int LL, const Coords& c, const Proposal& p) {
    bool acc = false;
#define PC_CALL(K) acc = cl_finish<MODE, K>(a, own, own_idx, P, LL, c, p)
    PC_SL_SWITCH(sl, PC_CALL)
#undef PC_CALL
    return acc;
}

// Cluster barrier in two halves: arrive (release: this CTA's spin writes are
// ordered before) and wait (acquire: the peers' writes are visible after).
__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release;" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire;" ::: "memory"); }

// The steps of one launch, in order: for each sweep, each round (round 0 the
// FIRST mode, the others overrelaxation, as enqueue_sweep in system.cu), each
// colour class, each sublattice of the class. A cluster barrier follows the
// last sublattice of each class.
struct StepIter {
    int s = 0, round = 0, k = 0, j = 0;
    __device__ bool next(const ClusterArgs& a, int rounds) {
        if (++j < a.class_n[k]) return true;
        j = 0;
        if (++k < a.n_classes) return true;
        k = 0;
        if (++round < rounds) return true;
        round = 0;
        return ++s < a.n_sweeps;
    }
};

// FIRST: the mode of a sweep's first round of colour passes (a fused mode, or
// kMetropolis); OR: the overrelaxation mode of the remaining rounds.
// Pipelined per thread: the next step's proposal (draws, Box-Muller, angle;
// independent of the neighbours, and its own spin is written by no one else)
// is formed between this CTA's barrier arrival and its wait, so it overlaps
// the barrier; after the wait only the neighbour loads, the local field and
// the accept/overrelax decision remain on the critical path of a pass.
template <int FIRST, int OR>
__global__ void __launch_bounds__(256) cluster_sweep_kernel(const __grid_constant__ ClusterArgs a) {
    extern __shared__ __align__(16) float4 plane[];  // [16][L*L]: this CTA's z plane of every sublattice
    __shared__ unsigned int warp_acc[8];
    cg::cluster_group cl = cg::this_cluster();
    const int L = a.L, LL = L * L, Nc = LL * L;
    const int z = int(cl.block_rank());
    const int r = int(blockIdx.x) / L;  // one cluster per replica
    const ReplicaDev rep = a.reps[r];
    float4* S = a.spins + rep.off;
    const int t = int(threadIdx.x);
    const bool live = t < LL;
    if (live)
        for (int sl = 0; sl < 16; ++sl) plane[sl * LL + t] = S[size_t(sl) * Nc + size_t(z) * LL + t];
    const float4* P[3] = {cl.map_shared_rank(plane, unsigned((z + L - 1) % L)), plane,
                          cl.map_shared_rank(plane, unsigned((z + 1) % L))};
    Coords c;
    {
        const int cx = live ? t % L : 0, cy = live ? t / L : 0;
        c.x[0] = cx == 0 ? L - 1 : cx - 1;
        c.x[1] = cx;
        c.x[2] = cx == L - 1 ? 0 : cx + 1;
        c.y[0] = L * (cy == 0 ? L - 1 : cy - 1);
        c.y[1] = L * cy;
        c.y[2] = L * (cy == L - 1 ? 0 : cy + 1);
        c.z[0] = c.z[1] = c.z[2] = 0;
    }
    const size_t cell = size_t(z) * LL + size_t(t);
    const uint64_t sweep0 = *a.sweep_base;
    constexpr bool kFusedFirst = FIRST != kMetropolis;
    const int rounds = kFusedFirst ? a.n_or : 1 + a.n_or;
    // the proposal of a step; live threads only
    auto prepare = [&](const StepIter& q) {
        const int sl = a.class_sl[q.k][q.j];
        const size_t i = size_t(sl) * Nc + cell;
        const uint64_t sweep = sweep0 + uint64_t(q.s);
        return q.round == 0 ? cl_prepare<FIRST>(a, plane, sl * LL + t, r, sweep, 0, i)
                            : cl_prepare<OR>(a, plane, sl * LL + t, r, sweep, kFusedFirst ? q.round : q.round - 1, i);
    };
    unsigned int mine = 0;
    StepIter q;
    const bool any = a.n_sweeps > 0 && rounds > 0;
    Proposal p;
    cluster_arrive();  // every plane loaded ...
    if (any && live) p = prepare(q);
    cluster_wait();  // ... before any neighbour is read
    bool more = any;
    while (more) {
        if (live) {
            const int sl = a.class_sl[q.k][q.j];
            if (q.round == 0)
                mine += cl_finish_sl<FIRST>(sl, a, plane, sl * LL + t, P, LL, c, p) ? 1u : 0u;
            else
                cl_finish_sl<OR>(sl, a, plane, sl * LL + t, P, LL, c, p);
        }
        const bool barrier = q.j + 1 == a.class_n[q.k];
        more = q.next(a, rounds);
        if (barrier) cluster_arrive();
        if (more && live) p = prepare(q);
        if (barrier) cluster_wait();
    }
    if (live)
        for (int sl = 0; sl < 16; ++sl) S[size_t(sl) * Nc + size_t(z) * LL + t] = plane[sl * LL + t];
    const int lane = t & 31, warp = t >> 5;
    unsigned int v = mine;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) warp_acc[warp] = v;
    __syncthreads();
    if (t == 0) {
        unsigned int tot = 0;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) tot += warp_acc[w];
        if (tot) atomicAdd(a.acc + r, (unsigned long long)tot);
    }
}

size_t cluster_smem_bytes(int L) { return size_t(16) * size_t(L) * size_t(L) * sizeof(float4); }

static int cluster_threads(int L) { return ((L * L + 31) / 32) * 32; }

template <typename K>
static int capacity_of(K kernel, int L) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    // the limit for the largest lattice, whatever size is asked about first
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(cluster_smem_bytes(16)));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(L));
    cfg.blockDim = dim3(unsigned(cluster_threads(L)));
    cfg.dynamicSmemBytes = cluster_smem_bytes(L);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = unsigned(L);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, kernel, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

template <int FIRST, int OR>
static void launch_one(const ClusterArgs& a, int R, cudaStream_t st) {
    auto kernel = cluster_sweep_kernel<FIRST, OR>;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(R * a.L));
    cfg.blockDim = dim3(unsigned(cluster_threads(a.L)));
    cfg.dynamicSmemBytes = cluster_smem_bytes(a.L);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = unsigned(a.L);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, a);
}

int cluster_capacity(int L, int fused, int reflect) {
    if (L < 2 || L > 16) return 0;
    if (fused)
        return reflect ? capacity_of(cluster_sweep_kernel<kFusedReflect, kOverrelaxReflect>, L)
                       : capacity_of(cluster_sweep_kernel<kFusedRotate, kOverrelaxRotate>, L);
    return reflect ? capacity_of(cluster_sweep_kernel<kMetropolis, kOverrelaxReflect>, L)
                   : capacity_of(cluster_sweep_kernel<kMetropolis, kOverrelaxRotate>, L);
}

void launch_cluster_sweeps(const ClusterArgs& a, int R, cudaStream_t st) {
    if (a.fused)
        a.reflect ? launch_one<kFusedReflect, kOverrelaxReflect>(a, R, st)
                  : launch_one<kFusedRotate, kOverrelaxRotate>(a, R, st);
    else
        a.reflect ? launch_one<kMetropolis, kOverrelaxReflect>(a, R, st)
                  : launch_one<kMetropolis, kOverrelaxRotate>(a, R, st);
}

}  // namespace pc
