// pt.cu -- replica exchange decided on the device (replaces the MPI exchange of
// src/temper.cpp:437-473); the round itself is pt_exchange_block (pt.cuh).
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"
#include "pt.cuh"

namespace pc {

__global__ void pt_exchange_kernel(const PtArgs a) { pt_exchange_block(a); }

void launch_pt_exchange(const PtArgs& a, cudaStream_t st) { pt_exchange_kernel<<<1, 128, 0, st>>>(a); }

}  // namespace pc
