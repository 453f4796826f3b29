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
#include "moves.cuh"
#include "struct_field.cuh"

namespace pc {

template <int VAR>
static void launch_struct(PassMode mode, const PassArgs& a, int grid, int threads, cudaStream_t st, bool pdl) {
    switch (mode) {
        case kMetropolis: launch_pass(struct_pass_kernel<kMetropolis, VAR>, a, grid, threads, st, pdl); break;
        case kOverrelaxRotate: launch_pass(struct_pass_kernel<kOverrelaxRotate, VAR>, a, grid, threads, st, pdl); break;
        case kOverrelaxReflect: launch_pass(struct_pass_kernel<kOverrelaxReflect, VAR>, a, grid, threads, st, pdl); break;
        case kOverrelaxTheta: launch_pass(struct_pass_kernel<kOverrelaxTheta, VAR>, a, grid, threads, st, pdl); break;
        case kFusedRotate: launch_pass(struct_pass_kernel<kFusedRotate, VAR>, a, grid, threads, st, pdl); break;
        case kFusedReflect: launch_pass(struct_pass_kernel<kFusedReflect, VAR>, a, grid, threads, st, pdl); break;
        default: break;
    }
}

void launch_colour_pass(PassMode mode, const PassArgs& a, int grid, int threads, cudaStream_t st, bool pdl) {
    if (a.structured && a.load_variant == 3) {  // row tiles, every mode: own module (sweep_staged.cu)
        launch_staged(mode, a, threads, st, pdl);
        return;
    }
    if (mode == kLifted || mode == kLiftedRot) {  // own module (sweep_lifted.cu)
        launch_lifted_pass(mode, a, grid, threads, st, pdl);
        return;
    }
    if (a.structured && threads <= 256) {
        if (a.load_variant == 1)
            launch_struct<1>(mode, a, grid, threads, st, pdl);
        else if (a.load_variant == 2)
            launch_struct<2>(mode, a, grid, threads, st, pdl);
        else if (a.load_variant == kVarIso)
            launch_struct<kVarIso>(mode, a, grid, threads, st, pdl);
        else if (a.load_variant == kVarIsoNoJ2)
            launch_struct<kVarIsoNoJ2>(mode, a, grid, threads, st, pdl);
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
        default: break;
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
    for (int u = blockIdx.x; u < a.n_tiles; u += gridDim.x) {
        const int t = a.order[u];
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

template <int SL, int ISO>
__device__ __forceinline__ float3 struct_field_e(const EnergyArgs& a, const float4* S, const ReplicaDev& rep, int cell) {
    return struct_field_upper<SL, ISO>(S, a.mats, cell, rep.L, rep.Nc, rep.divL);
}

// ISO: EnergyArgs::iso (0 general, 1 all groups j I, 2 all but a zero J2 group)
template <int ISO>
__global__ void __launch_bounds__(256) energy_struct_kernel(const __grid_constant__ EnergyArgs a) {
    __shared__ double red[4 * 32];
    for (int u = blockIdx.x; u < a.n_tiles; u += gridDim.x) {
        const int t = a.order[u];  // sublattice by sublattice: CTAs resident together run the same code
        const Tile tile = a.tiles[t];
        const int r = tile.x, sl = tile.y & 0xff;
        const ReplicaDev rep = a.reps[r];
        const float4* S = a.spins + rep.off;
        double v[4] = {0, 0, 0, 0};
        if (int(threadIdx.x) < tile.w) {
            const int cell = tile.z + int(threadIdx.x);
            const float4 s0 = S[size_t(sl) * rep.Nc + cell];
            float3 h = make_float3(0.f, 0.f, 0.f);
#define PC_CALL(K) h = struct_field_e<K, ISO>(a, S, rep, cell)
            PC_SL_SWITCH(sl, PC_CALL)
#undef PC_CALL
            // h: the bonds to higher sublattices only, each bond counted once
            v[0] = double(s0.x * h.x + s0.y * h.y + s0.z * h.z) -
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
    if (a.structured && threads <= 256) {
        if (a.iso == 1) {
            prefer_l1(reinterpret_cast<const void*>(energy_struct_kernel<1>));
            energy_struct_kernel<1><<<grid, threads, 0, st>>>(a);
        } else if (a.iso == 2) {
            prefer_l1(reinterpret_cast<const void*>(energy_struct_kernel<2>));
            energy_struct_kernel<2><<<grid, threads, 0, st>>>(a);
        } else {
            prefer_l1(reinterpret_cast<const void*>(energy_struct_kernel<0>));
            energy_struct_kernel<0><<<grid, threads, 0, st>>>(a);
        }
    } else {
        prefer_l1(reinterpret_cast<const void*>(energy_partials_kernel));
        energy_partials_kernel<<<grid, threads, 0, st>>>(a);
    }
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

__global__ void refresh_tq_kernel(const double* T, float2* q, int R, float inv_T_ref) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) q[r] = proposal_consts(T[r], inv_T_ref);
}
void launch_refresh_tq(const double* T, float2* q, int R, float inv_T_ref, cudaStream_t st) {
    refresh_tq_kernel<<<(R + 255) / 256, 256, 0, st>>>(T, q, R, inv_T_ref);
}
void launch_advance_counter(uint64_t* counter, uint64_t n, cudaStream_t st) {
    advance_counter_kernel<<<1, 1, 0, st>>>(counter, n);
}

}  // namespace pc
