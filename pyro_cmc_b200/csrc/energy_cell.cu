// energy_cell.cu -- energy per cubic cell and magnetisation with one thread
// per cubic cell (total_energy_per_unit_cell, src/MC.cpp:305-312); the per-cell
// sums are cell_energy (energy_cell.cuh), per-CTA FP64 partials are summed per
// replica in fixed order by energy_finalize_kernel (deterministic).
#include <cuda_runtime.h>

#include "energy_cell.cuh"
#include "kernels.h"

namespace pc {

template <int ISO, bool UNI, bool GROUPS>
__global__ void __launch_bounds__(kEnergyCellThreads, 5) energy_cell_kernel(const __grid_constant__ EnergyCellArgs a) {
    constexpr int NV = GROUPS ? 4 + kGroups : 4;
    __shared__ double red[NV * 32];
    const int4 tile = a.tiles[blockIdx.x];  // (replica, first cell, cells, -)
    const ReplicaDev rep = a.reps[tile.x];
    double v[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) v[j] = 0.0;
    if (int(threadIdx.x) < tile.z) {
        const int cell = tile.y + int(threadIdx.x);
        const Coords c = cell_coords(cell, rep.L, rep.divL);
        double (&v4)[4] = *reinterpret_cast<double(*)[4]>(v);
        cell_energy<ISO, UNI, true, GROUPS>(v4, reinterpret_cast<const char*>(a.spins + rep.off),
                                            uint32_t(rep.Nc) << 4, c, a.mats, a.B, GROUPS ? v + 4 : nullptr);
    }
    // block-wide FP64 sum: warp shuffles, then one warp over the warp sums
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[j] += __shfl_down_sync(0xffffffffu, v[j], o);
        if (lane == 0) red[j * 32 + warp] = v[j];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            double x = lane < nw ? red[j * 32 + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if (lane == 0) {
                if (j < 4)
                    a.partial[size_t(blockIdx.x) * 4 + j] = x;
                else
                    a.group_partial[size_t(blockIdx.x) * kGroups + (j - 4)] = x;
            }
        }
    }
}

void launch_energy_cells(const EnergyCellArgs& a, cudaStream_t st) {
    if (a.n_tiles <= 0) return;
    const bool uni = a.uniform != 0;
    if (a.iso == 1 && uni && a.group_partial)
        energy_cell_kernel<1, true, true><<<a.n_tiles, kEnergyCellThreads, 0, st>>>(a);
    else if (a.iso == 1 && uni)
        energy_cell_kernel<1, true, false><<<a.n_tiles, kEnergyCellThreads, 0, st>>>(a);
    else if (a.iso == 2 && uni)
        energy_cell_kernel<2, true, false><<<a.n_tiles, kEnergyCellThreads, 0, st>>>(a);
    else if (a.iso == 1)
        energy_cell_kernel<1, false, false><<<a.n_tiles, kEnergyCellThreads, 0, st>>>(a);
    else if (a.iso == 2)
        energy_cell_kernel<2, false, false><<<a.n_tiles, kEnergyCellThreads, 0, st>>>(a);
    else
        energy_cell_kernel<0, false, false><<<a.n_tiles, kEnergyCellThreads, 0, st>>>(a);
}

}  // namespace pc
