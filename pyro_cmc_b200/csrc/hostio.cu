// hostio.cu -- the device side of the host-buffer step with three floats per
// spin (pc_step_host3): host spins cross the bus as packed (x, y, z), 12 bytes
// a site instead of the 16 of the device's float4. The fourth component (the
// lifting direction of lifted Metropolis) never leaves the device: unpacking
// keeps it, packing drops it.
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"

namespace pc {

__global__ void spins_from_xyz_kernel(float4* __restrict__ spins, const float* __restrict__ xyz, int64_t n) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        float4 s = spins[i];
        s.x = xyz[3 * i];
        s.y = xyz[3 * i + 1];
        s.z = xyz[3 * i + 2];
        spins[i] = s;
    }
}

__global__ void spins_to_xyz_kernel(float* __restrict__ xyz, const float4* __restrict__ spins, int64_t n) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const float4 s = spins[i];
        xyz[3 * i] = s.x;
        xyz[3 * i + 1] = s.y;
        xyz[3 * i + 2] = s.z;
    }
}

static int io_grid(int64_t n) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t blocks = (n + 255) / 256;
    return int(blocks < int64_t(sms) * 8 ? blocks : int64_t(sms) * 8);
}

void launch_spins_from_xyz(float4* spins, const float* xyz, int64_t n, cudaStream_t st) {
    if (n > 0) spins_from_xyz_kernel<<<io_grid(n), 256, 0, st>>>(spins, xyz, n);
}

void launch_spins_to_xyz(float* xyz, const float4* spins, int64_t n, cudaStream_t st) {
    if (n > 0) spins_to_xyz_kernel<<<io_grid(n), 256, 0, st>>>(xyz, spins, n);
}

}  // namespace pc
