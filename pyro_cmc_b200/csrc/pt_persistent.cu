// pt_persistent.cu -- tempering rounds of a batch of replicas (any mix of
// lattice sizes) in one persistent cooperative launch: the sweeps, energies
// and exchanges of src/temper.cpp:418-474 for every replica of every ladder,
// without a kernel boundary between colour passes.
//
// Work distribution: the tiles of a colour class (every replica's sites of
// the class's sublattices, replica-contiguous) are dealt to the resident
// blocks in a grid-stride loop, exactly as the per-pass kernel deals them, and
// the same site code runs (struct_site, moves.cuh), so a chain is the same
// sequence of updates as with one launch per colour pass. Phases are separated
// by a grid barrier (arrive on a counter, wait on a generation word). Spins,
// temperatures and energies written in an earlier phase of the launch are read
// with ordinary loads ordered by the barrier's fences (kVarCoherent), never
// through the read-only path.
//
// The energy phase runs the per-cell energy of the stand-alone kernel
// (cell_energy, energy_cell.cuh: one thread per cubic cell, every bond once)
// with coherent loads into per-tile FP64 partials, the next phase sums each
// replica's partials in a fixed order (deterministic), and block 0 runs the
// exchange round (pt_exchange_block, as the stand-alone exchange kernel does).
//
// Every barrier wait is bounded (max_polls polls of ~64 ns): when one runs out
// the block sets *err = kErrGridBarrier, every block leaves at its next
// barrier, and the host reports PC_ERR_TIMEOUT. A cooperative launch only
// starts when all blocks fit on the device at once, so the waits end unless a
// block faults.
#include <cuda_runtime.h>

#include "common.cuh"
#include "energy_cell.cuh"
#include "kernels.h"
#include "moves.cuh"
#include "pt.cuh"
#include "struct_field.cuh"

namespace pc {

namespace {

// Two-level arrival: block b arrives on sub-counter b % kBarrierGroups (each
// on its own 128-byte line), the last arrival of a group arrives on the top
// counter, and the last of those bumps the generation that every block waits
// on. Arrivals on one address are serialised at its L2 slice; spread over the
// groups, a barrier of ~1000 blocks costs about two atomic round trips instead
// of ~1000 serialised atomics.
__device__ __forceinline__ bool grid_barrier(const PersistArgs& p) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int* gen = p.bar + 1;
        volatile int* err = p.pass.err;
        const unsigned int g = *gen;  // before arriving: the generation cannot move until this block arrives
        __threadfence();              // this block's writes before the arrival
        const unsigned int grp = blockIdx.x % kBarrierGroups;
        const unsigned int n_grp = (gridDim.x - grp + kBarrierGroups - 1) / kBarrierGroups;
        const unsigned int n_top = gridDim.x < kBarrierGroups ? gridDim.x : kBarrierGroups;
        unsigned int* sub = p.bar + kBarrierStride * (1 + grp);
        int ok = 1;
        bool waiter = true;
        if (atomicAdd(sub, 1u) == n_grp - 1) {
            atomicExch(sub, 0u);
            __threadfence();
            if (atomicAdd(p.bar, 1u) == n_top - 1) {
                atomicExch(p.bar, 0u);
                __threadfence();
                atomicAdd(p.bar + 1, 1u);
                waiter = false;
            }
        }
        if (waiter) {
            int polls = 0;
            while (*gen == g) {
                if (*err != 0) {
                    ok = 0;
                    break;
                }
                if (++polls > p.max_polls) {
                    atomicExch(p.pass.err, kErrGridBarrier);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();  // the other blocks' writes after the wait
        if (*err != 0) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Block-wide sum of four doubles; result valid in thread 0.
__device__ __forceinline__ void block_sum4(double (&v)[4], double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[j] += __shfl_down_sync(0xffffffffu, v[j], o);
        if (lane == 0) red[j * 32 + warp] = v[j];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            double x = lane < nw ? red[j * 32 + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            v[j] = x;
        }
    }
    __syncthreads();
}

template <int MODE, int VAR>
__device__ __forceinline__ void persist_pass(const PersistArgs& p, int colour, uint64_t sweep, unsigned int& mine,
                                             int& r_cur, unsigned int* warp_acc) {
    const PassArgs& a = p.pass;
    const Tile* tiles = p.colour_tiles[colour];
    const int n = p.n_colour_tiles[colour];
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const Tile tile = tiles[t];
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
}

// One thread per cubic cell (cell_energy with coherent loads) over the cell
// tiles of the stand-alone energy kernel (kEnergyCellThreads cells each); a
// block narrower than a tile takes its cells in turns.
template <int ISO, bool UNI>
__device__ __forceinline__ void persist_energy(const PersistArgs& p, double* red) {
    for (int t = blockIdx.x; t < p.n_c_tiles; t += gridDim.x) {
        const int4 tile = p.c_tiles[t];  // (replica, first cell, cells, -)
        const ReplicaDev rep = p.pass.reps[tile.x];
        double v[4] = {0.0, 0.0, 0.0, 0.0};
        for (int k = int(threadIdx.x); k < tile.z; k += int(blockDim.x)) {
            double w[4] = {0.0, 0.0, 0.0, 0.0};
            const Coords c = cell_coords(tile.y + k, rep.L, rep.divL);
            cell_energy<ISO, UNI, false>(w, reinterpret_cast<const char*>(p.pass.spins + rep.off),
                                         uint32_t(rep.Nc) << 4, c, p.pass.mats, p.pass.B);
            for (int j = 0; j < 4; ++j) v[j] += w[j];
        }
        block_sum4(v, red);
        if (threadIdx.x == 0)
            for (int j = 0; j < 4; ++j) p.partial[size_t(t) * 4 + j] = v[j];
    }
}

// e[r] = (sum of replica r's tile partials) / Nc in a fixed order: thread k sums
// tiles begin + k, begin + k + blockDim, ..., then a fixed-shape tree.
__device__ __forceinline__ void persist_finalize(const PersistArgs& p, double* red) {
    const double2* p2 = reinterpret_cast<const double2*>(p.partial);
    for (int r = blockIdx.x; r < p.R; r += gridDim.x) {
        double v[4] = {0.0, 0.0, 0.0, 0.0};
        for (int t = p.c_begin[r] + int(threadIdx.x); t < p.c_end[r]; t += blockDim.x) {
            const double2 q0 = __ldcg(p2 + 2 * size_t(t)), q1 = __ldcg(p2 + 2 * size_t(t) + 1);
            v[0] += q0.x;
            v[1] += q0.y;
            v[2] += q1.x;
            v[3] += q1.y;
        }
        block_sum4(v, red);
        if (threadIdx.x == 0) {
            p.e[r] = v[0] / double(p.pass.reps[r].Nc);
            if (p.mag)
                for (int j = 0; j < 3; ++j) p.mag[3 * r + j] = v[1 + j];
        }
    }
}

template <int ISO>
__host__ __device__ constexpr int persist_var() {
    return (ISO == 1 ? kVarIso : ISO == 2 ? kVarIsoNoJ2 : 0) | kVarCoherent;
}

// Registers per thread: what the colour passes alone compile to. The per-cell
// energy phase would take up to 255 and with them fewer resident blocks for
// every pass; capped, it spills to L1 instead (it runs once per round).
template <int FUSED, int ISO>
__host__ __device__ constexpr int persist_max_regs() {
    return FUSED ? (ISO == 2 ? 80 : ISO == 1 ? 64 : 56) : (ISO == 0 ? 64 : 80);
}

template <int FUSED, int ISO>
__global__ void __maxnreg__((persist_max_regs<FUSED, ISO>())) pt_persistent_kernel(const __grid_constant__ PersistArgs p) {
    __shared__ unsigned int warp_acc[8];
    __shared__ double red[4 * 32];
    constexpr int VAR = persist_var<ISO>();
    const uint64_t base = __ldcg(p.sweep);
    unsigned int mine = 0;
    int r_cur = -1;
    bool ok = true;
    for (int round = 0; ok && round < p.n_rounds; ++round) {
        for (int i = 0; ok && i < p.n_sweep; ++i) {
            const uint64_t sweep = base + uint64_t(round) * uint64_t(p.n_sweep) + uint64_t(i);
            if constexpr (FUSED) {
                for (int c = 0; ok && c < p.n_colours; ++c) {
                    persist_pass<kFusedRotate, VAR>(p, c, sweep, mine, r_cur, warp_acc);
                    ok = grid_barrier(p);
                }
            } else {
                for (int c = 0; ok && c < p.n_colours; ++c) {
                    persist_pass<kMetropolis, VAR>(p, c, sweep, mine, r_cur, warp_acc);
                    ok = grid_barrier(p);
                }
                for (int c = 0; ok && c < p.n_colours; ++c) {
                    persist_pass<kOverrelaxRotate, VAR>(p, c, sweep, mine, r_cur, warp_acc);
                    ok = grid_barrier(p);
                }
            }
        }
        if (ok && p.exchange) {
            if constexpr (ISO != 0) {
                if (p.uniform)
                    persist_energy<ISO, true>(p, red);
                else
                    persist_energy<ISO, false>(p, red);
            } else {
                persist_energy<0, false>(p, red);
            }
            ok = grid_barrier(p);
            if (ok) {
                persist_finalize(p, red);
                ok = grid_barrier(p);
            }
            if (ok) {
                if (blockIdx.x == 0) pt_exchange_block(p.pt);
                ok = grid_barrier(p);
            }
        }
    }
    if (r_cur >= 0) flush_accepted(p.pass, mine, r_cur, warp_acc);
    // every block read the counter before the first barrier, which all passed
    if (ok && blockIdx.x == 0 && threadIdx.x == 0 && p.n_rounds > 0 && p.n_sweep > 0)
        *p.sweep = base + uint64_t(p.n_rounds) * uint64_t(p.n_sweep);
}

const void* persistent_fn(int iso, int fused) {
    if (fused) {
        if (iso == 1) return reinterpret_cast<const void*>(pt_persistent_kernel<1, 1>);
        if (iso == 2) return reinterpret_cast<const void*>(pt_persistent_kernel<1, 2>);
        return reinterpret_cast<const void*>(pt_persistent_kernel<1, 0>);
    }
    if (iso == 1) return reinterpret_cast<const void*>(pt_persistent_kernel<0, 1>);
    if (iso == 2) return reinterpret_cast<const void*>(pt_persistent_kernel<0, 2>);
    return reinterpret_cast<const void*>(pt_persistent_kernel<0, 0>);
}

}  // namespace

static_assert(sizeof(PersistArgs) <= 32764, "kernel parameter space");

int pt_persistent_capacity(int iso, int fused, int threads) {
    const void* fn = persistent_fn(iso, fused);
    prefer_l1(fn);
    int dev = 0, sms = 0, per_sm = 0, coop = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, 0) != cudaSuccess) return 0;
    return per_sm * sms;
}

int launch_pt_persistent(const PersistArgs& a, int iso, int grid, int threads, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(grid));
    cfg.blockDim = dim3(unsigned(threads));
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e;
    if (a.fused) {
        if (iso == 1)
            e = cudaLaunchKernelEx(&cfg, pt_persistent_kernel<1, 1>, a);
        else if (iso == 2)
            e = cudaLaunchKernelEx(&cfg, pt_persistent_kernel<1, 2>, a);
        else
            e = cudaLaunchKernelEx(&cfg, pt_persistent_kernel<1, 0>, a);
    } else {
        if (iso == 1)
            e = cudaLaunchKernelEx(&cfg, pt_persistent_kernel<0, 1>, a);
        else if (iso == 2)
            e = cudaLaunchKernelEx(&cfg, pt_persistent_kernel<0, 2>, a);
        else
            e = cudaLaunchKernelEx(&cfg, pt_persistent_kernel<0, 0>, a);
    }
    return int(e);
}

}  // namespace pc
