// dft.cuh -- in-place 1-D DFTs of shared-memory lines for the S(q) kernels.
//
// A line of length L = P*Q (P, Q <= kMaxRadix) is transformed by the
// two-level Cooley-Tukey split, in place:
//   pass A: for each n2 < Q, the P-point DFT of x[Q n1 + n2] over n1, times
//     w^(n2 k1), written back to positions k1*Q + n2 (the positions it read);
//   pass B: for each k1 < P, the Q-point DFT of positions k1*Q + n2 over n2,
//     written to k1 + P k2 (all reads of a round of lines happen before any
//     write: registers across a barrier);
// with w = exp(-2 pi i / L), or its conjugate for INV (the unnormalised
// inverse). The P- and Q-point DFTs run in registers as direct sums whose
// coefficients are compile-time constants; terms whose coefficient is 0 or
// +-1 cost no multiply.
//
// Lines live in shared memory at addr(line, element), a functor chosen by the
// caller (swizzled layouts avoid bank conflicts). The item-to-thread map is
// line-fast (consecutive threads take consecutive lines) or element-fast.
#pragma once

#include <cuda_runtime.h>

#include <utility>

namespace pc {

constexpr int kMaxRadix = 8;

// cos / sin of 2 pi m / P at compile time: the angle is reduced to one octant
// and evaluated by its Taylor series (20 terms: below 1e-17 on [0, pi/4]).
constexpr double kPiD = 3.14159265358979323846264338327950288;
__host__ __device__ constexpr double ct_sin_series(double x) {
    double t = x, s = x;
    for (int k = 1; k < 20; ++k) {
        t *= -x * x / double((2 * k) * (2 * k + 1));
        s += t;
    }
    return s;
}
__host__ __device__ constexpr double ct_cos_series(double x) {
    double t = 1.0, s = 1.0;
    for (int k = 1; k < 20; ++k) {
        t *= -x * x / double((2 * k - 1) * (2 * k));
        s += t;
    }
    return s;
}
__host__ __device__ constexpr double ct_cos2pi(int m, int P) {
    m = ((m % P) + P) % P;
    const int e = 8 * m;  // angle in units of 2 pi / (8P)
    const int o = e / P;  // octant
    const double r = double(e - o * P) / double(P) * (kPiD / 4.0);
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
// sin a = cos(a - pi/2)
__host__ __device__ constexpr double ct_sin2pi(int m, int P) { return ct_cos2pi(4 * m - P, 4 * P); }

__device__ __forceinline__ float2 c_mul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 c_mulc(float2 a, float2 b) {  // a * conj(b)
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// acc += x * coef for a compile-time coefficient class:
// 0 -> nothing, 1 -> +x, -1 -> -x, 2 -> general multiply-add
template <int CN>
__device__ __forceinline__ void mac_part(float& acc, float x, float coef) {
    if constexpr (CN == 1)
        acc += x;
    else if constexpr (CN == -1)
        acc -= x;
    else if constexpr (CN == 2)
        acc = fmaf(x, coef, acc);
}
__host__ __device__ constexpr int coef_class(double v) {
    return (v == 0.0) ? 0 : (v == 1.0) ? 1 : (v == -1.0) ? -1 : 2;
}

// acc += x[N] * (c + i s), (c, s) = (cos, -+sin)(2 pi N K / P)
template <int P, bool INV, int K, int N>
__device__ __forceinline__ void dft_term(float2& acc, const float2 (&x)[kMaxRadix]) {
    constexpr double cd = ct_cos2pi(N * K, P);
    constexpr double sd = (INV ? 1.0 : -1.0) * ct_sin2pi(N * K, P);
    constexpr int cc = coef_class(cd), sc = coef_class(sd);
    constexpr float c = float(cd), s = float(sd);
    mac_part<cc>(acc.x, x[N].x, c);                  // re += x.re c
    mac_part<(sc == 2 ? 2 : -sc)>(acc.x, x[N].y, -s);  // re -= x.im s
    mac_part<sc>(acc.y, x[N].x, s);                  // im += x.re s
    mac_part<cc>(acc.y, x[N].y, c);                  // im += x.im c
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
    for (int k = 0; k < int(sizeof...(K)); ++k) x[k] = y[k];
}
// P-point DFT of x[0..P) in registers
template <int P, bool INV>
__device__ __forceinline__ void small_dft(float2 (&x)[kMaxRadix]) {
    if constexpr (P > 1) dft_all<P, INV>(x, std::make_integer_sequence<int, P>{});
}
// runtime P (uniform across the block); P = 1 is the identity
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

// Pass A over n_lines lines (no barrier inside; the caller syncs after).
// tw[j] = exp(-2 pi i j / L), j < L.
template <bool INV, bool LINE_FAST, class Addr>
__device__ __forceinline__ void dft_pass_a(float2* d, int P, int Q, int n_lines, Addr addr, const float2* tw) {
    const int items = n_lines * Q;
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
        const int l = LINE_FAST ? it % n_lines : it / Q;
        const int n2 = LINE_FAST ? it / n_lines : it % Q;
        float2 x[kMaxRadix];
#pragma unroll
        for (int n1 = 0; n1 < kMaxRadix; ++n1)
            if (n1 < P) x[n1] = d[addr(l, Q * n1 + n2)];
        small_dft_rt<INV>(x, P);
        d[addr(l, n2)] = x[0];
#pragma unroll
        for (int k1 = 1; k1 < kMaxRadix; ++k1)
            if (k1 < P) {
                const float2 w = tw[n2 * k1];  // n2 k1 < L
                d[addr(l, k1 * Q + n2)] = INV ? c_mulc(x[k1], w) : c_mul(x[k1], w);
            }
    }
}

// Pass B over n_lines lines in rounds of lines_per_round whole lines, so that a
// thread holds at most kPassBItems items across the barrier. Requires
// lines_per_round * P <= kPassBItems * blockDim.x. Ends with a barrier.
constexpr int kPassBItems = 2;
template <bool INV, bool LINE_FAST, class Addr>
__device__ __forceinline__ void dft_pass_b(float2* d, int P, int Q, int n_lines, int lines_per_round, Addr addr) {
    for (int l0 = 0; l0 < n_lines; l0 += lines_per_round) {
        const int nl = min(lines_per_round, n_lines - l0);
        const int items = nl * P;
        float2 keep[kPassBItems][kMaxRadix];
#pragma unroll
        for (int m = 0; m < kPassBItems; ++m) {
            const int it = threadIdx.x + m * blockDim.x;
            if (it < items) {
                const int l = l0 + (LINE_FAST ? it % nl : it / P);
                const int k1 = LINE_FAST ? it / nl : it % P;
#pragma unroll
                for (int n2 = 0; n2 < kMaxRadix; ++n2)
                    if (n2 < Q) keep[m][n2] = d[addr(l, k1 * Q + n2)];
                small_dft_rt<INV>(keep[m], Q);
            }
        }
        __syncthreads();
#pragma unroll
        for (int m = 0; m < kPassBItems; ++m) {
            const int it = threadIdx.x + m * blockDim.x;
            if (it < items) {
                const int l = l0 + (LINE_FAST ? it % nl : it / P);
                const int k1 = LINE_FAST ? it / nl : it % P;
#pragma unroll
                for (int k2 = 0; k2 < kMaxRadix; ++k2)
                    if (k2 < Q) d[addr(l, k1 + P * k2)] = keep[m][k2];
            }
        }
        __syncthreads();
    }
}

// Full transform: pass A, barrier, pass B (ends with a barrier).
template <bool INV, bool LINE_FAST, class Addr>
__device__ __forceinline__ void dft_lines(float2* d, int P, int Q, int n_lines, int lines_per_round, Addr addr,
                                          const float2* tw) {
    dft_pass_a<INV, LINE_FAST>(d, P, Q, n_lines, addr, tw);
    __syncthreads();
    dft_pass_b<INV, LINE_FAST>(d, P, Q, n_lines, lines_per_round, addr);
}

}  // namespace pc
