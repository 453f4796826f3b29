// sweep_lifted.cu -- lifted Metropolis passes (src/MC.cpp:194-302): the
// structured and generic colour-pass kernels instantiated for the two lifted
// moves, in their own module (sm_100a).
#include <cuda_runtime.h>

#include "moves.cuh"

namespace pc {

template <int MODE>
static void launch_lifted_mode(const PassArgs& a, int grid, int threads, cudaStream_t st, bool pdl) {
    if (a.structured && threads <= 256) {
        if (a.load_variant == 1)
            launch_pass(struct_pass_kernel<MODE, 1>, a, grid, threads, st, pdl);
        else if (a.load_variant == 2)
            launch_pass(struct_pass_kernel<MODE, 2>, a, grid, threads, st, pdl);
        else
            launch_pass(struct_pass_kernel<MODE, 0>, a, grid, threads, st, pdl);
        return;
    }
    launch_pass(colour_pass_kernel<MODE>, a, grid, threads, st, pdl);
}

void launch_lifted_pass(PassMode mode, const PassArgs& a, int grid, int threads, cudaStream_t st, bool pdl) {
    if (mode == kLiftedRot)
        launch_lifted_mode<kLiftedRot>(a, grid, threads, st, pdl);
    else
        launch_lifted_mode<kLifted>(a, grid, threads, st, pdl);
}

}  // namespace pc
