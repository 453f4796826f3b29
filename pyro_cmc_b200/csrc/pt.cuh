// pt.cuh -- one tempering exchange round by one thread block, shared by the
// stand-alone exchange kernel (pt.cu) and the persistent tempering kernel
// (pt_persistent.cu) so both take the same decisions from the same energies.
//
// Replicas never move: an accepted swap exchanges the temperature labels of two
// replicas (a permutation), so no spin bytes cross memory. Per round: every
// slot (temperature) takes one energy sample from the replica currently at it
// (src/temper.cpp:432-435), then each ladder attempts the checkerboard pairs of
// the round's parity: pairs (0,1),(2,3),... on even rounds, (1,2),(3,4),... on
// odd ones, slot 0 hottest. The hotter slot's rule is the reference's
// (src/temper.cpp:437-473): arg = (1/T - 1/T')(E - E') on total energies,
// accept if arg >= 0 or U < e^arg.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"

namespace pc {

// Every thread of the block calls this. The replica energies are read with
// L2-coherent loads: in the persistent kernel other blocks wrote them.
__device__ __forceinline__ void pt_exchange_block(const PtArgs& a) {
    const uint64_t round = *a.round;
    for (int s = threadIdx.x; s < a.n_slots; s += blockDim.x) {
        const int r = a.rep_of_slot[s];
        const double e = __ldcg(a.e_rep + r);
        a.E_sum[s] += e;
        a.E2_sum[s] += e * e;
        a.n_e[s] += 1ull;
    }
    __syncthreads();
    for (int l = threadIdx.x; l < a.n_ladders; l += blockDim.x) {
        const int b = a.ladder_begin[l], end = a.ladder_begin[l + 1];
        for (int s = b + int(round & 1ull); s + 1 < end; s += 2) {
            const int ra = a.rep_of_slot[s], rb = a.rep_of_slot[s + 1];
            const double Ta = a.T_slot[s], Tb = a.T_slot[s + 1];
            const double Ea = __ldcg(a.e_rep + ra) * double(a.reps[ra].Nc);
            const double Eb = __ldcg(a.e_rep + rb) * double(a.reps[rb].Nc);
            const double arg = (1.0 / Ta - 1.0 / Tb) * (Ea - Eb);
            const uint4 w = philox4x32_10(
                make_uint4(uint32_t(s), uint32_t(round), kDrawExchange | (uint32_t(round >> 32) << 8), 0xffffffffu),
                make_uint2(uint32_t(a.seed), uint32_t(a.seed >> 32)));
            const double u = double(w.x >> 8) * (1.0 / 16777216.0);
            const bool acc = arg >= 0.0 || u < exp(arg);
            a.attempts[s] += 1ull;
            if (acc) {
                a.accepts[s] += 1ull;
                a.rep_of_slot[s] = rb;
                a.rep_of_slot[s + 1] = ra;
                a.slot_of_rep[ra] = s + 1;
                a.slot_of_rep[rb] = s;
                a.T_rep[ra] = Tb;
                a.T_rep[rb] = Ta;
                a.Tq[ra] = proposal_consts(Tb, a.inv_T_ref);
                a.Tq[rb] = proposal_consts(Ta, a.inv_T_ref);
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) *a.round = round + 1ull;
}

}  // namespace pc
