// noalloc.cu -- energy and magnetisation of a caller-owned spin array without
// any device allocation (pc_energy_noalloc in include/pyrocmc.h).
//
// Who needs it: callers that must not call cudaMalloc or cudaFree. Examples:
// a program whose device memory is owned by a framework's caching allocator
// (a cudaMalloc behind its back fragments the pool and can fail once the pool
// has taken the free memory), or a tight loop that cannot afford the implicit
// device-wide synchronisation of cudaFree. The regular entry points keep their
// scratch in buffers allocated with the system; this one keeps its scratch --
// the per-tile partial sums of the reduction -- in a fixed array compiled into
// the library.
//
// Limits and sharing:
//  * L <= 64 (4,194,304 spins): 16 sublattices x L^3/256 tiles x 4 doubles
//    must fit in the 512 KiB array; larger L is rejected before any GPU work.
//  * The array lives on every GPU that loads the library until the process
//    exits. Every call on a device uses the same array and leaves its last
//    contents there; each call overwrites every partial it reads, so nothing
//    needs to start at zero. Two calls whose kernels overlap on the GPU (for
//    example on two streams) race on the array and give wrong results.
//  * The array's device address is looked up with cudaGetSymbolAddress by the
//    first call in each CUDA context (the first call on a device, and the
//    first call after that device's context was destroyed and re-created,
//    e.g. by cudaDeviceReset, which reloads the module at a new address).
//    Make that first call before any stream capture.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/pyrocmc.h"
#include "common.cuh"
#include "pyro_struct.cuh"
#include "struct_field.cuh"

namespace pc {
void set_last_error(const std::string& msg);  // system.cu
}

namespace {

constexpr int kNoallocMaxL = 64;
constexpr int kTileCells = 256;
constexpr int kMaxTiles = 16 * (kNoallocMaxL * kNoallocMaxL * kNoallocMaxL / kTileCells);
constexpr int kMaxDevices = 64;

// The scratch: 4 doubles (energy term, S_x, S_y, S_z) per tile of 256 cells.
static __device__ __align__(256) double g_noalloc_partials[kMaxTiles * 4];

struct NoallocArgs {
    const float4* spins;
    int L;
    int Nc;
    uint64_t divL;
    int tiles_per_sl;
    float B[3];
    pc::PyroMats mats;
    double* partial;
    double* out;
};

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

template <int SL>
__device__ __forceinline__ float3 field_at(const NoallocArgs& a, int cell) {
    return pc::struct_field<SL>(a.spins, a.mats, cell, a.L, a.Nc, a.divL);
}

// One block per tile: 256 consecutive cells of one sublattice.
__global__ void __launch_bounds__(kTileCells) noalloc_energy_tiles(const __grid_constant__ NoallocArgs a) {
    __shared__ double red[4][kTileCells / 32];
    const int sl = blockIdx.x / a.tiles_per_sl;
    const int cell = (blockIdx.x % a.tiles_per_sl) * kTileCells + int(threadIdx.x);
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    if (cell < a.Nc) {
        const float4 s0 = a.spins[size_t(sl) * a.Nc + cell];
        float3 h = make_float3(0.f, 0.f, 0.f);
        switch (sl) {
            case 0: h = field_at<0>(a, cell); break;
            case 1: h = field_at<1>(a, cell); break;
            case 2: h = field_at<2>(a, cell); break;
            case 3: h = field_at<3>(a, cell); break;
            case 4: h = field_at<4>(a, cell); break;
            case 5: h = field_at<5>(a, cell); break;
            case 6: h = field_at<6>(a, cell); break;
            case 7: h = field_at<7>(a, cell); break;
            case 8: h = field_at<8>(a, cell); break;
            case 9: h = field_at<9>(a, cell); break;
            case 10: h = field_at<10>(a, cell); break;
            case 11: h = field_at<11>(a, cell); break;
            case 12: h = field_at<12>(a, cell); break;
            case 13: h = field_at<13>(a, cell); break;
            case 14: h = field_at<14>(a, cell); break;
            default: h = field_at<15>(a, cell); break;
        }
        // total_energy_per_unit_cell's terms (0.5 S.h - S.B) and the spin sum
        v[0] = 0.5 * double(s0.x * h.x + s0.y * h.y + s0.z * h.z) -
               double(s0.x * a.B[0] + s0.y * a.B[1] + s0.z * a.B[2]);
        v[1] = s0.x;
        v[2] = s0.y;
        v[3] = s0.z;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int j = 0; j < 4; ++j) {
        const double w = warp_sum_d(v[j]);
        if (lane == 0) red[j][warp] = w;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double t = 0.0;
        for (int w = 0; w < kTileCells / 32; ++w) t += red[threadIdx.x][w];
        a.partial[size_t(blockIdx.x) * 4 + threadIdx.x] = t;
    }
}

// One block: fixed-order sum of the tile partials (deterministic).
__global__ void __launch_bounds__(kTileCells) noalloc_energy_sum(const __grid_constant__ NoallocArgs a, int n_tiles) {
    __shared__ double red[4][kTileCells / 32];
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int t = threadIdx.x; t < n_tiles; t += blockDim.x)
        for (int j = 0; j < 4; ++j) v[j] += a.partial[size_t(t) * 4 + j];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int j = 0; j < 4; ++j) {
        const double w = warp_sum_d(v[j]);
        if (lane == 0) red[j][warp] = w;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double t = 0.0;
        for (int w = 0; w < kTileCells / 32; ++w) t += red[threadIdx.x][w];
        a.out[threadIdx.x] = threadIdx.x == 0 ? t / double(a.Nc) : t;
    }
}

std::mutex g_mu;
// Per device: the context the address was looked up in, and the address.
struct ScratchAddr {
    unsigned long long ctx_id = 0;
    bool valid = false;
    double* ptr = nullptr;
};
ScratchAddr g_scratch[kMaxDevices];

int noalloc_fail(int code, const std::string& msg) {
    pc::set_last_error(msg);
    return code;
}

// Identity of the calling thread's current context on `dev`. The driver
// entry points are fetched through the runtime, so the library does not
// link against libcuda. A thread that has not yet made a runtime call has no
// current context: cudaSetDevice binds (and if needed creates) the primary
// context of `dev`, which the following runtime calls would use anyway.
int current_context_id(int dev, unsigned long long* id) {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    if (!get_current || !get_id) {
        void* f1 = nullptr;
        void* f2 = nullptr;
        cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = q1;
        cudaError_t e1 = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1);
        cudaError_t e2 = cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2);
        if (e1 != cudaSuccess || e2 != cudaSuccess || q1 != cudaDriverEntryPointSuccess ||
            q2 != cudaDriverEntryPointSuccess || !f1 || !f2)
            return noalloc_fail(PC_ERR_CUDA, "pc_energy_noalloc: driver entry points cuCtxGetCurrent/cuCtxGetId "
                                             "not available");
        get_current = reinterpret_cast<GetCurrent>(f1);
        get_id = reinterpret_cast<GetId>(f2);
    }
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS) return noalloc_fail(PC_ERR_CUDA, "pc_energy_noalloc: cuCtxGetCurrent failed");
    if (!ctx) {
        const cudaError_t e = cudaSetDevice(dev);
        if (e != cudaSuccess)
            return noalloc_fail(PC_ERR_CUDA, std::string("pc_energy_noalloc: cudaSetDevice: ") + cudaGetErrorString(e));
        if (get_current(&ctx) != CUDA_SUCCESS || !ctx)
            return noalloc_fail(PC_ERR_CUDA, "pc_energy_noalloc: no current CUDA context");
    }
    if (get_id(ctx, id) != CUDA_SUCCESS) return noalloc_fail(PC_ERR_CUDA, "pc_energy_noalloc: cuCtxGetId failed");
    return PC_OK;
}

}  // namespace

extern "C" int pc_energy_noalloc(const void* spins_dev, int L, const double* params, void* out_dev, void* stream) {
    if (!spins_dev || !params || !out_dev) return noalloc_fail(PC_ERR_INVALID, "pc_energy_noalloc: null argument");
    // the kernels read float4 spins and write doubles: misaligned pointers
    // (e.g. an offset view into a larger buffer) are rejected, not faulted on
    if (reinterpret_cast<uintptr_t>(spins_dev) % 16 != 0)
        return noalloc_fail(PC_ERR_INVALID, "pc_energy_noalloc: spins_dev is not 16-byte aligned (float4 spins)");
    if (reinterpret_cast<uintptr_t>(out_dev) % 8 != 0)
        return noalloc_fail(PC_ERR_INVALID, "pc_energy_noalloc: out_dev is not 8-byte aligned (doubles)");
    if (L < 1 || L > kNoallocMaxL)
        return noalloc_fail(PC_ERR_INVALID, "pc_energy_noalloc: L = " + std::to_string(L) +
                                                " is outside 1..64, the size its fixed scratch array holds");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_fail(PC_ERR_CUDA, std::string("pc_energy_noalloc: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(PC_ERR_UNSUPPORTED, "pc_energy_noalloc: device index too large");
    double* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        unsigned long long ctx_id = 0;
        const int rc = current_context_id(dev, &ctx_id);
        if (rc) return rc;
        ScratchAddr& slot = g_scratch[dev];
        if (!slot.valid || slot.ctx_id != ctx_id) {
            // once per context: the host-side symbol is only a stand-in, the
            // kernels need the array's device address in this context
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_partials);
            if (e != cudaSuccess)
                return noalloc_fail(PC_ERR_CUDA, std::string("pc_energy_noalloc: cudaGetSymbolAddress: ") +
                                                     cudaGetErrorString(e));
            slot.ptr = static_cast<double*>(p);
            slot.ctx_id = ctx_id;
            slot.valid = true;
        }
        scratch = slot.ptr;
    }
    NoallocArgs a;
    std::memset(&a, 0, sizeof(a));
    a.spins = static_cast<const float4*>(spins_dev);
    a.L = L;
    a.Nc = L * L * L;
    a.divL = pc::fastdiv_magic(L);
    a.tiles_per_sl = (a.Nc + kTileCells - 1) / kTileCells;
    for (int i = 0; i < 3; ++i) a.B[i] = float(params[4 + i]);
    // build_J1J2J3_h's couplings (include/cli_bits.hpp:175-200) per
    // (sublattice, neighbour group): J1 [I + (Delta-1) z_p z_nu^T] towards
    // pyro sublattice nu, J2 I, J3 I, J3 I; z_p = link[p]/sqrt(3)
    const int link[4][3] = {{1, 1, 1}, {1, -1, -1}, {-1, 1, -1}, {-1, -1, 1}};
    const double J1 = params[0], J2 = params[1], J3 = params[2], Delta = params[3];
    for (int sl = 0; sl < 16; ++sl) {
        const int p = sl % 4;
        for (int g = 0; g < pc::kGroups; ++g) {
            double M[9];
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) {
                    const double I = r == c ? 1.0 : 0.0;
                    if (g < 3) {
                        const int nu = pc::kStruct.t[sl].gnu[g];
                        M[3 * r + c] = J1 * (I + (Delta - 1.0) * double(link[p][r] * link[nu][c]) / 3.0);
                    } else {
                        M[3 * r + c] = (g == 3 ? J2 : J3) * I;
                    }
                }
            bool nonzero = false;
            for (int i = 0; i < 9; ++i) {
                a.mats.M[sl][g][i] = float(M[i]);
                nonzero = nonzero || M[i] != 0.0;
            }
            if (nonzero) a.mats.active[sl] |= 1u << g;
        }
    }
    a.partial = scratch;
    a.out = static_cast<double*>(out_dev);
    const int n_tiles = 16 * a.tiles_per_sl;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    noalloc_energy_tiles<<<n_tiles, kTileCells, 0, st>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(PC_ERR_CUDA, std::string("pc_energy_noalloc: ") + cudaGetErrorString(e));
    noalloc_energy_sum<<<1, kTileCells, 0, st>>>(a, n_tiles);
    e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(PC_ERR_CUDA, std::string("pc_energy_noalloc: ") + cudaGetErrorString(e));
    return PC_OK;
}
