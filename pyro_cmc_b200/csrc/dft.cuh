// dft.cuh -- in-place 1-D DFTs of shared-memory lines for the S(q) kernels.
//
// A line of length L = P*Q is transformed by the two-level Cooley-Tukey split:
//   pass A (in place): for each n2 < Q, the P-point DFT of x[Q n1 + n2] over
//     n1, times w^(n2 k1), back into positions k1*Q + n2 (the same positions);
//   pass B: for each k1 < P, the Q-point DFT of positions k1*Q + n2 over n2,
//     written to k1 + P k2 (other positions: read to registers, barrier, write).
// with w = exp(-2 pi i / L) (forward) or its conjugate (INV, the unnormalised
// inverse). The small DFTs run in registers with compile-time twiddles for
// sizes up to kMaxRadix; larger factors use a table-driven loop.
#pragma once

#include <cuda_runtime.h>

#include <utility>

namespace pc {

constexpr int kMaxRadix = 8;

// cos / sin of 2 pi m / P for compile-time m, P: Taylor series after reduction
// of the angle to [-pi/4, pi/4] by octant (compile-time only).
constexpr double kPiD = 3.14159265358979323846264338327950288;
constexpr double ct_sin_series(double x) {
    double t = x, s = x;
    for (int k = 1; k < 20; ++k) {
        t *= -x * x / double((2 * k) * (2 * k + 1));
        s += t;
    }
    return s;
}
constexpr double ct_cos_series(double x) {
    double t = 1.0, s = 1.0;
    for (int k = 1; k < 20; ++k) {
        t *= -x * x / double((2 * k - 1) * (2 * k));
        s += t;
    }
    return s;
}
// angle 2 pi m / P with m reduced into [0, P)
constexpr double ct_cos2pi(int m, int P) {
    m = ((m % P) + P) % P;
    // work with 8P-ths of a turn: octant o, remainder in [0, P)
    const int e = 8 * m;             // angle in units of 2 pi / (8P)
    const int o = e / P;             // octant 0..7
    const double r = double(e - o * P) / double(P) * (kPiD / 4.0);  // in [0, pi/4)
    switch (o) {
        case 0: return ct_cos_series(r);
        case 1: return ct_sin_series(kPiD / 4.0 - r);
        case 2: return -ct_sin_series(r);
        case 3: return -ct_cos_series(kPiD / 4.0 - r);
        case 4: return -ct_cos_series(r);
        case 5: return -ct_sin_series(kPiD / 4.0 - r);
        case 6: return ct_sin_series(r);
        default: return ct_cos_series(kPiD / 4.0 - r);
    }
}
constexpr double ct_sin2pi(int m, int P) { return ct_cos2pi(m * 4 - P, 4 * P); }  // sin a = cos(a - pi/2)

__device__ __forceinline__ float2 c_mul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 c_mulc(float2 a, float2 b) {  // a * conj(b)
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// y[K] += x[N] * w^(N K) for one (K, N), w = exp(-+2 pi i / P)
template <int P, bool INV, int K, int N>
__device__ __forceinline__ void dft_term(float2& acc, const float2 (&x)[kMaxRadix]) {
    constexpr float c = float(ct_cos2pi(N * K, P));
    constexpr float s = float((INV ? 1.0 : -1.0) * ct_sin2pi(N * K, P));
    if constexpr (((N * K) % P) == 0) {
        acc.x += x[N].x;
        acc.y += x[N].y;
    } else {
        acc.x += x[N].x * c - x[N].y * s;
        acc.y += x[N].x * s + x[N].y * c;
    }
}
template <int P, bool INV, int K, int... N>
__device__ __forceinline__ float2 dft_out(const float2 (&x)[kMaxRadix], std::integer_sequence<int, N...>) {
    float2 acc = make_float2(0.f, 0.f);
    (dft_term<P, INV, K, N>(acc, x), ...);
    return acc;
}
template <int P, bool INV, int... K>
__device__ __forceinline__ void dft_all(float2 (&x)[kMaxRadix], std::integer_sequence<int, K...>) {
    const float2 y[sizeof...(K)] = {dft_out<P, INV, K>(x, std::make_integer_sequence<int, P>{})...};
#pragma unroll
    for (int k = 0; k < P; ++k) x[k] = y[k];
}
// P-point DFT of x[0..P) in registers
template <int P, bool INV>
__device__ __forceinline__ void small_dft(float2 (&x)[kMaxRadix]) {
    if constexpr (P > 1) dft_all<P, INV>(x, std::make_integer_sequence<int, P>{});
}

// Runtime-P dispatch (P uniform across the block)
template <bool INV>
__device__ __forceinline__ void small_dft_rt(float2 (&x)[kMaxRadix], int P) {
    switch (P) {
        case 2: small_dft<2, INV>(x); break;
        case 3: small_dft<3, INV>(x); break;
        case 4: small_dft<4, INV>(x); break;
        case 5: small_dft<5, INV>(x); break;
        case 6: small_dft<6, INV>(x); break;
        case 7: small_dft<7, INV>(x); break;
        case 8: small_dft<8, INV>(x); break;
        default: break;
    }
}

// Transforms n_lines lines in place; element e of line l at data[l*ls + e*es].
// tw[j] = exp(-2 pi i j / L). Requires P, Q <= kMaxRadix. Ends with a barrier.
template <bool INV>
__device__ void dft_lines_inplace(float2* data, int L, int P, int Q, int n_lines, int ls, int es, const float2* tw) {
    // pass A: items (line, n2)
    const int itemsA = n_lines * Q;
    for (int it = threadIdx.x; it < itemsA; it += blockDim.x) {
        const int l = it % n_lines, n2 = it / n_lines;
        float2* base = data + l * ls;
        float2 x[kMaxRadix];
#pragma unroll
        for (int n1 = 0; n1 < kMaxRadix; ++n1)
            if (n1 < P) x[n1] = base[(Q * n1 + n2) * es];
        small_dft_rt<INV>(x, P);
        int wi = 0;
#pragma unroll
        for (int k1 = 0; k1 < kMaxRadix; ++k1)
            if (k1 < P) {
                const float2 w = tw[wi];
                base[(k1 * Q + n2) * es] = INV ? c_mulc(x[k1], w) : c_mul(x[k1], w);
                wi += n2;
                wi -= (wi >= L) ? L : 0;
            }
    }
    __syncthreads();
    // pass B: items (line, k1); registers across the barrier
    const int itemsB = n_lines * P;
    constexpr int kMaxItems = 4;  // items per thread held across the barrier
    float2 keep[kMaxItems][kMaxRadix];
    int n_mine = 0;
    for (int it = threadIdx.x; it < itemsB && n_mine < kMaxItems; it += blockDim.x, ++n_mine) {
        const int l = it % n_lines, k1 = it / n_lines;
        const float2* base = data + l * ls;
#pragma unroll
        for (int n2 = 0; n2 < kMaxRadix; ++n2)
            if (n2 < Q) keep[n_mine][n2] = base[(k1 * Q + n2) * es];
        small_dft_rt<INV>(keep[n_mine], Q);
    }
    __syncthreads();
    int m = 0;
    for (int it = threadIdx.x; it < itemsB && m < kMaxItems; it += blockDim.x, ++m) {
        const int l = it % n_lines, k1 = it / n_lines;
        float2* base = data + l * ls;
#pragma unroll
        for (int k2 = 0; k2 < kMaxRadix; ++k2)
            if (k2 < Q) base[(k1 + P * k2) * es] = keep[m][k2];
    }
    __syncthreads();
}

}  // namespace pc
