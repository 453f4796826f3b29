// ssf.cu -- static structure factor (ssf_manager::sample,
// include/ssf_manager.hpp:260-293) as a batched shared-memory DFT (sm_100a).
//
// The reference forms, per correlator (a,b), S(q) = sum_{mu,nu}
// exp(+i q.(r_mu - r_nu)) conj(A^a_mu(q)) A^b_nu(q) from 16 per-sublattice DFTs
// A_mu. That double sum factorises: S(q) = conj(B^a(q)) B^b(q) with
// B^a(q) = sum_mu exp(-i q.r_mu) A^a_mu(q) = sum_i exp(-i q.x_i) S^a_i, which is
// what is computed here: O(16 n_k) per component instead of O(256 n_k) per
// correlator, and no [n_k,16,16] buffer.
//
// The phase exp(-i q.r_mu) factorises per axis, and the 16 sublattices have 4
// distinct z offsets r_z in {-1, 1, 3, 5} with 4 sublattices each. So:
//   stage 1 (per replica, z plane, z group): 2-D DFT over (x, y) of each of the
//     group's 4 sublattices, times exp(-i(qx rx + qy ry)), summed -> G;
//   stage 2 (per replica, Ky, Kx chunk): DFT over z of the 4 group planes,
//     times exp(-i qz rz), summed -> B^a(K); then the correlators and the FP64
//     accumulation of S and (Re S)^2, (Im S)^2.
// Each 1-D DFT of length L = P*Q is a two-level Cooley-Tukey split (P-point
// DFTs, twiddle, Q-point DFTs) on shared-memory lines. FP32 transforms, FP64
// accumulators.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "dft.cuh"
#include "kernels.h"

namespace pc {

// Unwrapped sublattice offsets r_sl = link[p] + R_fcc[f], sl = 4f + p
// (include/pyrochlore_geometry.hpp:16-29).
__constant__ int c_rsl[16][3] = {
    {1, 1, 1},  {1, -1, -1}, {-1, 1, -1}, {-1, -1, 1},  // f = 0
    {1, 5, 5},  {1, 3, 3},   {-1, 5, 3},  {-1, 3, 5},   // f = 1 (0,4,4)
    {5, 1, 5},  {5, -1, 3},  {3, 1, 3},   {3, -1, 5},   // f = 2 (4,0,4)
    {5, 5, 1},  {5, 3, -1},  {3, 5, -1},  {3, 3, 1},    // f = 3 (4,4,0)
};
// Sublattices by z offset: group g has r_z = 2g - 1.
__constant__ int c_zgroup[4][4] = {{1, 2, 13, 14}, {0, 3, 12, 15}, {5, 6, 9, 10}, {4, 7, 8, 11}};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// Twiddles tw[j] = exp(-2 pi i j / L), phases ph[j] = exp(-2 pi i j / (8L)).
__device__ void fill_tables(float2* tw, float2* ph, int L) {
    for (int j = threadIdx.x; j < L; j += blockDim.x) {
        float s, c;
        sincospif(-2.f * float(j) / float(L), &s, &c);
        tw[j] = make_float2(c, s);
    }
    for (int j = threadIdx.x; j < 8 * L; j += blockDim.x) {
        float s, c;
        sincospif(-2.f * float(j) / float(8 * L), &s, &c);
        ph[j] = make_float2(c, s);
    }
}

__device__ __forceinline__ float2 phase(const float2* ph, int L, int Kr) {
    int j = Kr % (8 * L);
    j += (j < 0) ? 8 * L : 0;
    return ph[j];
}

// One Cooley-Tukey half pass over n_lines lines of length L = P*Q; element e of
// line l lives at l*lstride + e*estride. INV selects conj twiddles (the
// unnormalised inverse transform).
//   stage A: out[k1*Q + n2] = w^(n2 k1) sum_{n1<P} in[Q n1 + n2] w^(Q n1 k1)
//   stage B: out[k1 + P k2] = sum_{n2<Q} in[k1*Q + n2] w^(P n2 k2)
// line_fast: consecutive threads take consecutive lines (for lines whose
// elements are strided), otherwise consecutive elements of one line.
template <bool STAGE_B, bool INV>
__device__ void ct_half(const float2* __restrict__ in, float2* __restrict__ out, int L, int P, int Q, int n_lines,
                        int lstride, int estride, const float2* tw, bool line_fast) {
    const int total = n_lines * L;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        int l, j;
        if (line_fast) {
            l = idx % n_lines;
            j = idx / n_lines;
        } else {
            l = idx / L;
            j = idx % L;
        }
        const float2* src = in + l * lstride;
        float2 acc = make_float2(0.f, 0.f);
        if (!STAGE_B) {
            const int k1 = j / Q, n2 = j % Q;
            const int step = (Q * k1) % L;
            int wi = 0;
            for (int n1 = 0; n1 < P; ++n1) {
                const float2 x = src[(Q * n1 + n2) * estride];
                const float2 w = tw[wi];
                acc = INV ? make_float2(acc.x + x.x * w.x + x.y * w.y, acc.y + x.y * w.x - x.x * w.y)
                          : make_float2(acc.x + x.x * w.x - x.y * w.y, acc.y + x.x * w.y + x.y * w.x);
                wi += step;
                wi -= (wi >= L) ? L : 0;
            }
            const float2 w = tw[(n2 * k1) % L];
            acc = INV ? cmulc(acc, w) : cmul(acc, w);
        } else {
            const int k1 = j % P, k2 = j / P;
            const int step = (P * k2) % L;
            int wi = 0;
            for (int n2 = 0; n2 < Q; ++n2) {
                const float2 x = src[(k1 * Q + n2) * estride];
                const float2 w = tw[wi];
                acc = INV ? make_float2(acc.x + x.x * w.x + x.y * w.y, acc.y + x.y * w.x - x.x * w.y)
                          : make_float2(acc.x + x.x * w.x - x.y * w.y, acc.y + x.x * w.y + x.y * w.x);
                wi += step;
                wi -= (wi >= L) ? L : 0;
            }
        }
        out[l * lstride + j * estride] = acc;
    }
}

// Full 1-D transform of all lines, result back in `a` (b is scratch).
template <bool INV>
__device__ __forceinline__ void dft_lines_generic(float2* a, float2* b, int L, int P, int Q, int n_lines, int lstride,
                                          int estride, const float2* tw, bool line_fast) {
    ct_half<false, INV>(a, b, L, P, Q, n_lines, lstride, estride, tw, line_fast);
    __syncthreads();
    ct_half<true, INV>(b, a, L, P, Q, n_lines, lstride, estride, tw, line_fast);
    __syncthreads();
}

// ------------------------------------------------------- fast path, P, Q <= 8
// Stage 1, one CTA per (replica, z plane, z group, pair of the group's
// sublattices s0, s1). The six real planes of the pair become three complex
// planes, A0 = Sx0 + i Sy0, A1 = Sx1 + i Sy1, Az = Sz0 + i Sz1, whose 2-D DFTs
// are split again by Hermitian symmetry (F real => F(-K) = conj F(K)):
//   X0 = (A0(K) + conj A0(-K)) / 2,  Y0 = (A0(K) - conj A0(-K)) / 2i, ...
// Each component's X0 e^{-i q.r_s0} + X1 e^{-i q.r_s1} (x, y parts of the
// phase) goes to its own half-group plane of G; stage 2 adds the two halves of
// a group. G layout: [replica][component][2 gz + pair][nz][Ky][Kx].
//
// Plane layout in shared memory: element (x, y) at y L + sw(x, y). With L a
// multiple of 16, sw swaps 8-element blocks by the parity of y and permutes
// inside a block by the block index, so the row passes (one thread per 8-element
// stretch) and the column passes (consecutive x) are free of bank conflicts at
// L = 64.
template <bool SWZ>
__device__ __forceinline__ int plane_pos(int x, int y, int L) {
    if constexpr (SWZ)
        return y * L + ((((x >> 3) ^ (y & 1)) << 3) | ((x & 7) ^ ((x >> 3) & 7)));
    else
        return y * L + x;
}

__host__ __device__ __forceinline__ bool ssf_fast_path(int P, int Q) { return P <= kMaxRadix && Q <= kMaxRadix; }

// The split L = P*Q of the host's split_PQ (largest divisor P <= sqrt L), at
// compile time for the instantiated sizes. LT = 0: sizes from the geometry at
// run time.
__host__ __device__ constexpr int ct_split_P(int L) {
    int best = 1;
    for (int p = 1; p * p <= L; ++p)
        if (L % p == 0) best = p;
    return best;
}
template <int LT>
struct SsfDims {
    int L, P, Q;
    __device__ __forceinline__ explicit SsfDims(const SsfGeom& g)
        : L(LT ? LT : g.L), P(LT ? ct_split_P(LT) : g.P), Q(LT ? LT / ct_split_P(LT) : g.Q) {}
};

template <int LT, bool SWZ, bool RES>
__global__ void __launch_bounds__(512) ssf_plane_kernel(const SsfGeom g, const float4* __restrict__ spins,
                                                        const ReplicaDev* __restrict__ reps, float2* __restrict__ G) {
    extern __shared__ float2 sm[];
    const SsfDims<LT> dm(g);
    const int L = dm.L, LL = L * L, P = dm.P, Q = dm.Q;
    float2* tw = sm;
    float2* ph = tw + L;
    float2* buf = ph + 8 * L;  // planes A0, A1, Az
    const int h = blockIdx.x & 7, gz = h >> 1, pr = h & 1;
    const int nz = (blockIdx.x >> 3) % L;
    const int rp = (blockIdx.x >> 3) / L;
    const ReplicaDev rep = reps[g.rep_index[rp]];
    const int s0 = c_zgroup[gz][2 * pr], s1 = c_zgroup[gz][2 * pr + 1];
    const float4* p0 = spins + rep.off + size_t(s0) * rep.Nc + size_t(nz) * LL;
    const float4* p1 = spins + rep.off + size_t(s1) * rep.Nc + size_t(nz) * LL;
    fill_tables(tw, ph, L);
    for (int i = threadIdx.x; i < LL; i += blockDim.x) {
        const int y = i / L, x = i - y * L;
        const float4 a = p0[i], b = p1[i];
        const int q = plane_pos<SWZ>(x, y, L);
        buf[q] = make_float2(a.x, a.y);
        buf[LL + q] = make_float2(b.x, b.y);
        buf[2 * LL + q] = make_float2(a.z, b.z);
    }
    __syncthreads();
    const int lpr = max(1, int(kPassBItems * blockDim.x) / P);
    auto row = [=](int l, int e) {  // line (plane b, row y), element x
        const int b = l / L;
        return b * LL + plane_pos<SWZ>(e, l - b * L, L);
    };
    dft_lines<false, false>(buf, P, Q, 3 * L, lpr, row, tw);
    auto col = [=](int l, int e) {  // line (plane b, column x), element y
        const int b = l / L;
        return b * LL + plane_pos<SWZ>(l - b * L, e, L);
    };
    dft_lines<false, true>(buf, P, Q, 3 * L, lpr, col, tw);
    const int rx0 = c_rsl[s0][0], ry0 = c_rsl[s0][1], rx1 = c_rsl[s1][0], ry1 = c_rsl[s1][1];
    const size_t L3 = size_t(L) * LL;
    if constexpr (RES) {
        // per-sublattice planes, no phases: G[replica][a][sl][nz][Ky][Kx]
        float2* Gr = G + size_t(rp) * 48 * L3 + size_t(nz) * LL;
        for (int i = threadIdx.x; i < LL; i += blockDim.x) {
            const int Ky = i / L, Kx = i - Ky * L;
            const int q = plane_pos<SWZ>(Kx, Ky, L);
            const int qm = plane_pos<SWZ>(Kx ? L - Kx : 0, Ky ? L - Ky : 0, L);
            const float2 a = buf[q], am = buf[qm];
            const float2 b = buf[LL + q], bm = buf[LL + qm];
            const float2 z = buf[2 * LL + q], zm = buf[2 * LL + qm];
            Gr[size_t(0 * 16 + s0) * L3 + i] = make_float2(0.5f * (a.x + am.x), 0.5f * (a.y - am.y));
            Gr[size_t(1 * 16 + s0) * L3 + i] = make_float2(0.5f * (a.y + am.y), -0.5f * (a.x - am.x));
            Gr[size_t(2 * 16 + s0) * L3 + i] = make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
            Gr[size_t(0 * 16 + s1) * L3 + i] = make_float2(0.5f * (b.x + bm.x), 0.5f * (b.y - bm.y));
            Gr[size_t(1 * 16 + s1) * L3 + i] = make_float2(0.5f * (b.y + bm.y), -0.5f * (b.x - bm.x));
            Gr[size_t(2 * 16 + s1) * L3 + i] = make_float2(0.5f * (z.y + zm.y), -0.5f * (z.x - zm.x));
        }
        return;
    }
    float2* Gx = G + ((size_t(rp) * 3) * 8 + h) * L3 + size_t(nz) * LL;
    float2* Gy = Gx + 8 * L3;
    float2* Gz = Gy + 8 * L3;
    for (int i = threadIdx.x; i < LL; i += blockDim.x) {
        const int Ky = i / L, Kx = i - Ky * L;
        const int q = plane_pos<SWZ>(Kx, Ky, L);
        const int qm = plane_pos<SWZ>(Kx ? L - Kx : 0, Ky ? L - Ky : 0, L);
        const float2 a = buf[q], am = buf[qm];
        const float2 b = buf[LL + q], bm = buf[LL + qm];
        const float2 z = buf[2 * LL + q], zm = buf[2 * LL + qm];
        const float2 e0 = cmul(phase(ph, L, Kx * rx0), phase(ph, L, Ky * ry0));
        const float2 e1 = cmul(phase(ph, L, Kx * rx1), phase(ph, L, Ky * ry1));
        // (F + conj F-)/2 and (F - conj F-)/2i
        const float2 X0 = make_float2(0.5f * (a.x + am.x), 0.5f * (a.y - am.y));
        const float2 Y0 = make_float2(0.5f * (a.y + am.y), -0.5f * (a.x - am.x));
        const float2 X1 = make_float2(0.5f * (b.x + bm.x), 0.5f * (b.y - bm.y));
        const float2 Y1 = make_float2(0.5f * (b.y + bm.y), -0.5f * (b.x - bm.x));
        const float2 Z0 = make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
        const float2 Z1 = make_float2(0.5f * (z.y + zm.y), -0.5f * (z.x - zm.x));
        const float2 u0 = cmul(X0, e0), u1 = cmul(X1, e1);
        const float2 v0 = cmul(Y0, e0), v1 = cmul(Y1, e1);
        const float2 w0 = cmul(Z0, e0), w1 = cmul(Z1, e1);
        Gx[i] = make_float2(u0.x + u1.x, u0.y + u1.y);
        Gy[i] = make_float2(v0.x + v1.x, v0.y + v1.y);
        Gz[i] = make_float2(w0.x + w1.x, w0.y + w1.y);
    }
}

__host__ __device__ __forceinline__ int ssf_chunk(int L) { return L < 16 ? L : 16; }

// Stage 2, one CTA per (replica, Ky, chunk of C Kx values): the z-DFT of the
// 12 (component, z group) line sets, the z part of the phase, the sum over
// groups -> B^a(K), then the correlators and the FP64 accumulators. Shared
// layout T[(a*4 + gz)][z][CP], CP = C + 1 (odd row stride: the per-K reads
// with consecutive Kz hit distinct banks).
template <int LT>
__global__ void __launch_bounds__(512) ssf_line_kernel(const SsfGeom g, const float2* __restrict__ G, const SsfOut o) {
    extern __shared__ float2 sm[];
    const SsfDims<LT> dm(g);
    const int L = dm.L, LL = L * L, P = dm.P, Q = dm.Q;
    const int C = ssf_chunk(L), CP = C + 1;
    const int n_chunk = (L + C - 1) / C;
    float2* tw = sm;
    float2* ph = tw + L;
    float2* T = ph + 8 * L;
    const int chunk = blockIdx.x % n_chunk;
    const int Ky = (blockIdx.x / n_chunk) % L;
    const int rp = (blockIdx.x / n_chunk) / L;
    const int Kx0 = chunk * C;
    const int nc = min(C, L - Kx0);
    const size_t L3 = size_t(L) * LL;
    fill_tables(tw, ph, L);
    for (int i = threadIdx.x; i < 12 * L * C; i += blockDim.x) {
        const int c = i % C, zr = i / C;  // zr = (a*4 + gz) * L + z
        const int ag = zr / L, z = zr - ag * L;
        float2 v = make_float2(0.f, 0.f);
        if (c < nc) {
            const int a = ag >> 2, gz = ag & 3;
            const float2* src = G + ((size_t(rp) * 3 + a) * 8 + 2 * gz) * L3 + size_t(z) * LL + size_t(Ky) * L + Kx0 + c;
            const float2 u = src[0], w = src[L3];  // the group's two sublattice pairs
            v = make_float2(u.x + w.x, u.y + w.y);
        }
        T[zr * CP + c] = v;
    }
    __syncthreads();
    const int lpr = max(1, int(kPassBItems * blockDim.x) / P);
    auto zl = [=](int l, int e) {  // line (a*4 + gz, c), element z
        const int ag = l / C;
        return (ag * L + e) * CP + (l - ag * C);
    };
    dft_lines<false, true>(T, P, Q, 12 * C, lpr, zl, tw);
    const int rep_glob = g.rep_index[rp];
    const int n_k = L * LL;
    const int slot = o.acc_sum ? o.slot_of_rep[rep_glob] : -1;
    for (int i = threadIdx.x; i < L * nc; i += blockDim.x) {
        const int c = i / L, Kz = i - c * L;
        float2 B[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            float2 acc = make_float2(0.f, 0.f);
#pragma unroll
            for (int gz = 0; gz < 4; ++gz) {
                const float2 v = cmul(T[((a * 4 + gz) * L + Kz) * CP + c], phase(ph, L, Kz * (2 * gz - 1)));
                acc.x += v.x;
                acc.y += v.y;
            }
            B[a] = acc;
        }
        const size_t k = (size_t(Kx0 + c) * L + Ky) * L + Kz;
        if (o.amp)
            for (int a = 0; a < 3; ++a) o.amp[(size_t(rp) * 3 + a) * n_k + k] = B[a];
        if (o.val || slot >= 0) {
            double* __restrict__ acc_s = slot >= 0 ? o.acc_sum + size_t(slot) * o.slot_stride : nullptr;
            double* __restrict__ acc_q = slot >= 0 ? o.acc_sq + size_t(slot) * o.slot_stride : nullptr;
            // correlators in groups of three: the group's accumulator loads are
            // issued together, then the updates, then the stores
#pragma unroll
            for (int c0 = 0; c0 < 9; c0 += 3) {
                double re[3], im[3];
                double2 sv[3], qv[3];
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const int cc = c0 + j;
                    if (cc < o.n_corr) {
                        const int ca = o.corr_a[cc], cb = o.corr_b[cc];
                        const float2 ba = ca == 0 ? B[0] : (ca == 1 ? B[1] : B[2]);
                        const float2 bb = cb == 0 ? B[0] : (cb == 1 ? B[1] : B[2]);
                        // conj(B^a) B^b
                        re[j] = double(ba.x) * bb.x + double(ba.y) * bb.y;
                        im[j] = double(ba.x) * bb.y - double(ba.y) * bb.x;
                        if (acc_s) {
                            sv[j] = *reinterpret_cast<const double2*>(acc_s + (size_t(cc) * n_k + k) * 2);
                            qv[j] = *reinterpret_cast<const double2*>(acc_q + (size_t(cc) * n_k + k) * 2);
                        }
                    }
                }
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const int cc = c0 + j;
                    if (cc < o.n_corr) {
                        if (o.val)
                            *reinterpret_cast<double2*>(o.val + ((size_t(rp) * o.n_corr + cc) * n_k + k) * 2) =
                                make_double2(re[j], im[j]);
                        if (acc_s) {
                            *reinterpret_cast<double2*>(acc_s + (size_t(cc) * n_k + k) * 2) =
                                make_double2(sv[j].x + re[j], sv[j].y + im[j]);
                            *reinterpret_cast<double2*>(acc_q + (size_t(cc) * n_k + k) * 2) =
                                make_double2(qv[j].x + re[j] * re[j], qv[j].y + im[j] * im[j]);
                        }
                    }
                }
            }
        }
    }
}

// ------------------------------------------------ sublattice-resolved S(q)
// The reference's correlate() output before contract(): for each correlator
// (a, b), C_{mu nu}(K) = conj(A^a_mu(K)) A^b_nu(K) with A^a_mu the 3-D DFT over
// cells of S^a on sublattice mu (include/ssf_manager.hpp:260-293; the layout
// [n_corr, n_k, n_sl, n_sl, 2] that src/temper.cpp:121-159 writes). Stage 1 is
// ssf_plane_kernel<.., RES = true> (per-sublattice planes, no phases);
// then the z-DFT in place, then one CTA per (replica, K) for the 256 (mu, nu).
__host__ __device__ __forceinline__ int ssf_chunk_res(int L) { return L <= 16 ? L : (L <= 32 ? 8 : 4); }

template <int LT>
__global__ void __launch_bounds__(256) ssf_zdft_res_kernel(const SsfGeom g, float2* __restrict__ G) {
    extern __shared__ float2 sm[];
    const SsfDims<LT> dm(g);
    const int L = dm.L, LL = L * L, P = dm.P, Q = dm.Q;
    const int C = ssf_chunk_res(L), CP = C + 1, PS = L * CP + 1;  // odd plane stride
    const int n_chunk = (L + C - 1) / C;
    float2* tw = sm;
    float2* ph = tw + L;
    float2* T = ph + 8 * L;  // [48][L][CP], planes PS apart
    const int chunk = blockIdx.x % n_chunk;
    const int Ky = (blockIdx.x / n_chunk) % L;
    const int rp = (blockIdx.x / n_chunk) / L;
    const int Kx0 = chunk * C;
    const int nc = min(C, L - Kx0);
    const size_t L3 = size_t(L) * LL;
    float2* base = G + size_t(rp) * 48 * L3 + size_t(Ky) * L + Kx0;
    fill_tables(tw, ph, L);
    for (int i = threadIdx.x; i < 48 * L * C; i += blockDim.x) {
        const int c = i % C, zr = i / C;  // zr = plane * L + z
        const int pl = zr / L, z = zr - pl * L;
        T[pl * PS + z * CP + c] = c < nc ? base[size_t(pl) * L3 + size_t(z) * LL + c] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    const int lpr = max(1, int(kPassBItems * blockDim.x) / P);
    auto zl = [=](int l, int e) {
        const int pl = l / C;
        return pl * PS + e * CP + (l - pl * C);
    };
    dft_lines<false, true>(T, P, Q, 48 * C, lpr, zl, tw);
    for (int i = threadIdx.x; i < 48 * L * C; i += blockDim.x) {
        const int c = i % C, zr = i / C;
        const int pl = zr / L, z = zr - pl * L;
        if (c < nc) base[size_t(pl) * L3 + size_t(z) * LL + c] = T[pl * PS + z * CP + c];
    }
}

// One CTA of 256 threads per (replica, K); thread t = 16 mu + nu.
__global__ void __launch_bounds__(256) ssf_accum_res_kernel(const SsfGeom g, const float2* __restrict__ A, const SsfOut o) {
    __shared__ float2 amp[48];
    const int L = g.L, LL = L * L;
    const int n_k = L * LL;
    const int k = blockIdx.x % n_k, rp = blockIdx.x / n_k;
    const int Kx = k / LL, Ky = (k / L) % L, Kz = k % L;
    const size_t L3 = size_t(L) * LL;
    const int t = threadIdx.x;
    if (t < 48) amp[t] = A[(size_t(rp) * 48 + t) * L3 + size_t(Kz) * LL + size_t(Ky) * L + Kx];
    __syncthreads();
    const int mu = t >> 4, nu = t & 15;
    const int rep_glob = g.rep_index[rp];
    const int slot = o.acc_sum ? o.slot_of_rep[rep_glob] : -1;
#pragma unroll
    for (int cc = 0; cc < 9; ++cc) {
        if (cc >= o.n_corr) break;
        const float2 a = amp[o.corr_a[cc] * 16 + mu], b = amp[o.corr_b[cc] * 16 + nu];
        const double re = double(a.x) * b.x + double(a.y) * b.y;  // conj(A^a_mu) A^b_nu
        const double im = double(a.x) * b.y - double(a.y) * b.x;
        const size_t off = (size_t(cc) * n_k + k) * 256 + t;
        if (o.val) reinterpret_cast<double2*>(o.val + (size_t(rp) * o.n_corr * n_k * 256) * 2)[off] = make_double2(re, im);
        if (slot >= 0) {
            double2* s = reinterpret_cast<double2*>(o.acc_sum + size_t(slot) * o.slot_stride) + off;
            double2* q = reinterpret_cast<double2*>(o.acc_sq + size_t(slot) * o.slot_stride) + off;
            const double2 sv = *s, qv = *q;
            *s = make_double2(sv.x + re, sv.y + im);
            *q = make_double2(qv.x + re * re, qv.y + im * im);
        }
    }
}

// ------------------------------------------------ fast-path backward (P, Q <= 8)
// dLoss/dS_i^c = Re sum_K exp(+i q.x_i) Y^c(K), with
// Y^c(K) = sum_corr [c == a] conj(D) B^b + [c == b] D B^a, D = dL/dReS + i dL/dImS.
// Adjoint stage z, one CTA per (replica, Ky, chunk of C Kx values): Y^a times
// the conjugate z phase of each z group, inverse z-DFT of the 12 line sets ->
// H[replica][a][gz][nz][Ky][Kx].
template <int LT>
__global__ void __launch_bounds__(512) ssf_line_adj_kernel(const SsfGeom g, const SsfOut o, const double* __restrict__ dval,
                                                           const float2* __restrict__ amp, float2* __restrict__ H) {
    extern __shared__ float2 sm[];
    const SsfDims<LT> dm(g);
    const int L = dm.L, LL = L * L, P = dm.P, Q = dm.Q;
    const int C = ssf_chunk(L), CP = C + 1;
    const int n_chunk = (L + C - 1) / C;
    float2* tw = sm;
    float2* ph = tw + L;
    float2* T = ph + 8 * L;
    const int chunk = blockIdx.x % n_chunk;
    const int Ky = (blockIdx.x / n_chunk) % L;
    const int rp = (blockIdx.x / n_chunk) / L;
    const int Kx0 = chunk * C;
    const int nc = min(C, L - Kx0);
    const int n_k = L * LL;
    fill_tables(tw, ph, L);
    __syncthreads();
    for (int i = threadIdx.x; i < L * C; i += blockDim.x) {
        const int c = i / L, Kz = i - c * L;
        float2 y[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
        if (c < nc) {
            const size_t k = (size_t(Kx0 + c) * L + Ky) * L + Kz;
            float2 b[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) b[a] = amp[(size_t(rp) * 3 + a) * n_k + k];
#pragma unroll
            for (int cc = 0; cc < 9; ++cc) {
                if (cc >= o.n_corr) break;
                const double2 d2 = *reinterpret_cast<const double2*>(dval + ((size_t(rp) * o.n_corr + cc) * n_k + k) * 2);
                const float2 D = make_float2(float(d2.x), float(d2.y));
                const int ca = o.corr_a[cc], cb = o.corr_b[cc];
                const float2 ba = ca == 0 ? b[0] : (ca == 1 ? b[1] : b[2]);
                const float2 bb = cb == 0 ? b[0] : (cb == 1 ? b[1] : b[2]);
                const float2 t1 = cmulc(bb, D);  // conj(D) B^b -> Y^a
                const float2 t2 = cmul(D, ba);   // D B^a      -> Y^b
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    if (q == ca) {
                        y[q].x += t1.x;
                        y[q].y += t1.y;
                    }
                    if (q == cb) {
                        y[q].x += t2.x;
                        y[q].y += t2.y;
                    }
                }
            }
        }
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int gz = 0; gz < 4; ++gz)  // times exp(+i qz rz)
                T[((a * 4 + gz) * L + Kz) * CP + c] = cmulc(y[a], phase(ph, L, Kz * (2 * gz - 1)));
    }
    __syncthreads();
    const int lpr = max(1, int(kPassBItems * blockDim.x) / P);
    auto zl = [=](int l, int e) {
        const int ag = l / C;
        return (ag * L + e) * CP + (l - ag * C);
    };
    dft_lines<true, true>(T, P, Q, 12 * C, lpr, zl, tw);
    const size_t L3 = size_t(L) * LL;
    for (int i = threadIdx.x; i < 12 * L * C; i += blockDim.x) {
        const int c = i % C, zr = i / C;  // zr = (a*4 + gz) * L + nz
        if (c >= nc) continue;
        const int ag = zr / L, nz = zr - ag * L;
        H[(size_t(rp) * 12 + ag) * L3 + size_t(nz) * LL + size_t(Ky) * L + Kx0 + c] = T[zr * CP + c];
    }
}

// Adjoint stage xy, one CTA per (replica, z plane, z group, sublattice pair):
// X_a(K) = H_a(K) exp(+i q.r_s0) (x, y parts), Y_a likewise for s1; the real
// part of the inverse 2-D DFT of X_a is the inverse DFT of its Hermitian part
// (X_a(K) + conj X_a(-K)) / 2, so Z_a = herm(X_a) + i herm(Y_a) gives both
// sublattices' gradients in one transform: Re -> s0, Im -> s1.
template <int LT, bool SWZ>
__global__ void __launch_bounds__(512) ssf_plane_adj_kernel(const SsfGeom g, const float2* __restrict__ H,
                                                            const ReplicaDev* __restrict__ reps,
                                                            float4* __restrict__ grad) {
    extern __shared__ float2 sm[];
    const SsfDims<LT> dm(g);
    const int L = dm.L, LL = L * L, P = dm.P, Q = dm.Q;
    float2* tw = sm;
    float2* ph = tw + L;
    float2* buf = ph + 8 * L;  // planes Z_0, Z_1, Z_2
    const int h = blockIdx.x & 7, gz = h >> 1, pr = h & 1;
    const int nz = (blockIdx.x >> 3) % L;
    const int rp = (blockIdx.x >> 3) / L;
    const ReplicaDev rep = reps[g.rep_index[rp]];
    const int s0 = c_zgroup[gz][2 * pr], s1 = c_zgroup[gz][2 * pr + 1];
    const int rx0 = c_rsl[s0][0], ry0 = c_rsl[s0][1], rx1 = c_rsl[s1][0], ry1 = c_rsl[s1][1];
    const size_t L3 = size_t(L) * LL;
    fill_tables(tw, ph, L);
    __syncthreads();
    for (int i = threadIdx.x; i < LL; i += blockDim.x) {
        const int Ky = i / L, Kx = i - Ky * L;
        const int mx = Kx ? L - Kx : 0, my = Ky ? L - Ky : 0;
        const int im = my * L + mx;
        // conj of the forward phases at K and at -K
        const float2 e0 = cmul(phase(ph, L, Kx * rx0), phase(ph, L, Ky * ry0));
        const float2 e1 = cmul(phase(ph, L, Kx * rx1), phase(ph, L, Ky * ry1));
        const float2 f0 = cmul(phase(ph, L, mx * rx0), phase(ph, L, my * ry0));
        const float2 f1 = cmul(phase(ph, L, mx * rx1), phase(ph, L, my * ry1));
        const int q = plane_pos<SWZ>(Kx, Ky, L);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float2* Ha = H + ((size_t(rp) * 3 + a) * 4 + gz) * L3 + size_t(nz) * LL;
            const float2 hk = Ha[i], hm = Ha[im];
            const float2 X = cmulc(hk, e0), Xm = cmulc(hm, f0);  // X(K), X(-K)
            const float2 Y = cmulc(hk, e1), Ym = cmulc(hm, f1);
            // herm(X) = (X + conj Xm)/2, herm(Y) likewise; Z = herm(X) + i herm(Y)
            const float2 hx = make_float2(0.5f * (X.x + Xm.x), 0.5f * (X.y - Xm.y));
            const float2 hy = make_float2(0.5f * (Y.x + Ym.x), 0.5f * (Y.y - Ym.y));
            buf[a * LL + q] = make_float2(hx.x - hy.y, hx.y + hy.x);
        }
    }
    __syncthreads();
    const int lpr = max(1, int(kPassBItems * blockDim.x) / P);
    auto col = [=](int l, int e) {
        const int b = l / L;
        return b * LL + plane_pos<SWZ>(l - b * L, e, L);
    };
    dft_lines<true, true>(buf, P, Q, 3 * L, lpr, col, tw);
    auto row = [=](int l, int e) {
        const int b = l / L;
        return b * LL + plane_pos<SWZ>(e, l - b * L, L);
    };
    dft_lines<true, false>(buf, P, Q, 3 * L, lpr, row, tw);
    float4* g0 = grad + rep.off + size_t(s0) * rep.Nc + size_t(nz) * LL;
    float4* g1 = grad + rep.off + size_t(s1) * rep.Nc + size_t(nz) * LL;
    for (int i = threadIdx.x; i < LL; i += blockDim.x) {
        const int y = i / L, x = i - y * L;
        const int q = plane_pos<SWZ>(x, y, L);
        const float2 z0 = buf[q], z1 = buf[LL + q], z2 = buf[2 * LL + q];
        g0[i] = make_float4(z0.x, z1.x, z2.x, 0.f);
        g1[i] = make_float4(z0.y, z1.y, z2.y, 0.f);
    }
}

// ------------------------------------------------ generic path, P or Q > 8
// stage 1: per (replica, z plane, z group), runtime-length DFT loops
__global__ void __launch_bounds__(256) ssf_xy_kernel(const SsfGeom g, const float4* __restrict__ spins,
                                                     const ReplicaDev* reps, float2* __restrict__ G) {
    extern __shared__ float2 sm[];
    const int L = g.L, LL = L * L;
    float2* tw = sm;
    float2* ph = tw + L;
    float2* acc = ph + 8 * L;
    float2* w0 = acc + LL;
    float2* w1 = w0 + LL;
    const int gz = blockIdx.x & 3;
    const int nz = (blockIdx.x >> 2) % L;
    const int rp = (blockIdx.x >> 2) / L;
    const ReplicaDev rep = reps[g.rep_index[rp]];
    const float4* S = spins + rep.off;
    fill_tables(tw, ph, L);
    for (int a = 0; a < 3; ++a) {
        for (int i = threadIdx.x; i < LL; i += blockDim.x) acc[i] = make_float2(0.f, 0.f);
        for (int m = 0; m < 4; ++m) {
            const int sl = c_zgroup[gz][m];
            const float4* plane = S + size_t(sl) * rep.Nc + size_t(nz) * LL;
            __syncthreads();
            for (int i = threadIdx.x; i < LL; i += blockDim.x) {
                const float4 v = plane[i];
                w0[i] = make_float2(a == 0 ? v.x : (a == 1 ? v.y : v.z), 0.f);
            }
            __syncthreads();
            dft_lines_generic<false>(w0, w1, L, g.P, g.Q, L, L, 1, tw, false);  // along x (rows)
            dft_lines_generic<false>(w0, w1, L, g.P, g.Q, L, 1, L, tw, true);   // along y (columns)
            const int rx = c_rsl[sl][0], ry = c_rsl[sl][1];
            for (int i = threadIdx.x; i < LL; i += blockDim.x) {
                const int Kx = i % L, Ky = i / L;
                const float2 p = cmul(phase(ph, L, Kx * rx), phase(ph, L, Ky * ry));
                const float2 v = cmul(w0[i], p);
                acc[i].x += v.x;
                acc[i].y += v.y;
            }
        }
        __syncthreads();
        float2* dst = G + ((size_t(rp) * 3 + a) * 4 + gz) * size_t(L) * LL + size_t(nz) * LL;
        for (int i = threadIdx.x; i < LL; i += blockDim.x) dst[i] = acc[i];
        __syncthreads();
    }
}

template <bool RES>
void launch_plane(const SsfGeom& g, const float4* spins, const ReplicaDev* reps, float2* G, int grid, int threads,
                  size_t smem, cudaStream_t st) {
    switch (g.L) {
        case 64: ssf_plane_kernel<64, true, RES><<<grid, threads, smem, st>>>(g, spins, reps, G); break;
        case 32: ssf_plane_kernel<32, true, RES><<<grid, threads, smem, st>>>(g, spins, reps, G); break;
        case 24: ssf_plane_kernel<24, false, RES><<<grid, threads, smem, st>>>(g, spins, reps, G); break;
        case 16: ssf_plane_kernel<16, true, RES><<<grid, threads, smem, st>>>(g, spins, reps, G); break;
        case 12: ssf_plane_kernel<12, false, RES><<<grid, threads, smem, st>>>(g, spins, reps, G); break;
        case 8: ssf_plane_kernel<8, false, RES><<<grid, threads, smem, st>>>(g, spins, reps, G); break;
        default:
            if (g.L % 16 == 0)
                ssf_plane_kernel<0, true, RES><<<grid, threads, smem, st>>>(g, spins, reps, G);
            else
                ssf_plane_kernel<0, false, RES><<<grid, threads, smem, st>>>(g, spins, reps, G);
    }
}

int ssf_plane_threads(int L) { return std::min(512, std::max(64, (L * L / 8 + 31) / 32 * 32)); }
int ssf_line_threads(int L, int P, int Q) {
    const int items = 12 * ssf_chunk(L) * std::max(P, Q) / 4;
    return std::min(512, std::max(64, (items + 31) / 32 * 32));
}

void launch_ssf_xy(const SsfGeom& g, const float4* spins, const ReplicaDev* reps, float2* G, cudaStream_t st) {
    const int L = g.L;
    const size_t smem = sizeof(float2) * (size_t(9) * L + 3 * size_t(L) * L);
    if (ssf_fast_path(g.P, g.Q)) {
        const int threads = ssf_plane_threads(L);
        const int grid = g.n_rep * L * 8;
        if (g.resolved)
            launch_plane<true>(g, spins, reps, G, grid, threads, smem, st);
        else
            launch_plane<false>(g, spins, reps, G, grid, threads, smem, st);
        return;
    }
    ssf_xy_kernel<<<g.n_rep * L * 4, 256, smem, st>>>(g, spins, reps, G);
}

// ------------------------------------------------------------------ stage 2
__global__ void __launch_bounds__(256) ssf_z_kernel(const SsfGeom g, const float2* __restrict__ G, const SsfOut o) {
    extern __shared__ float2 sm[];
    const int L = g.L, LL = L * L;
    const int C = ssf_chunk(L);
    const int n_chunk = (L + C - 1) / C;
    float2* tw = sm;
    float2* ph = tw + L;
    float2* Bq = ph + 8 * L;    // [3][L(Kz)][C]
    float2* w0 = Bq + 3 * L * C;  // [L][C]
    float2* w1 = w0 + L * C;
    const int chunk = blockIdx.x % n_chunk;
    const int Ky = (blockIdx.x / n_chunk) % L;
    const int rp = (blockIdx.x / n_chunk) / L;
    const int Kx0 = chunk * C;
    const int nc = min(C, L - Kx0);
    fill_tables(tw, ph, L);
    for (int a = 0; a < 3; ++a) {
        float2* B = Bq + a * L * C;
        for (int i = threadIdx.x; i < L * C; i += blockDim.x) B[i] = make_float2(0.f, 0.f);
        for (int gz = 0; gz < 4; ++gz) {
            const float2* src = G + ((size_t(rp) * 3 + a) * 4 + gz) * size_t(L) * LL + size_t(Ky) * L + Kx0;
            __syncthreads();
            for (int i = threadIdx.x; i < L * C; i += blockDim.x) {
                const int c = i % C, nz = i / C;
                w0[i] = c < nc ? src[size_t(nz) * LL + c] : make_float2(0.f, 0.f);
            }
            __syncthreads();
            dft_lines_generic<false>(w0, w1, L, g.P, g.Q, C, 1, C, tw, true);  // along z
            const int rz = 2 * gz - 1;
            for (int i = threadIdx.x; i < L * C; i += blockDim.x) {
                const int Kz = i / C;
                const float2 v = cmul(w0[i], phase(ph, L, Kz * rz));
                B[i].x += v.x;
                B[i].y += v.y;
            }
        }
    }
    __syncthreads();
    const int rep_glob = g.rep_index[rp];
    const int n_k = L * LL;
    if (o.amp) {
        for (int a = 0; a < 3; ++a)
            for (int i = threadIdx.x; i < L * nc; i += blockDim.x) {
                const int Kz = i % L, c = i / L;
                const size_t k = (size_t(Kx0 + c) * L + Ky) * L + Kz;
                o.amp[(size_t(rp) * 3 + a) * n_k + k] = Bq[(a * L + Kz) * C + c];
            }
    }
    if (o.val || o.acc_sum) {
        const int slot = o.acc_sum ? o.slot_of_rep[rep_glob] : -1;
        for (int cc = 0; cc < o.n_corr; ++cc) {
            const int ca = o.corr_a[cc], cb = o.corr_b[cc];
            for (int i = threadIdx.x; i < L * nc; i += blockDim.x) {
                const int Kz = i % L, c = i / L;
                const float2 ba = Bq[(ca * L + Kz) * C + c];
                const float2 bb = Bq[(cb * L + Kz) * C + c];
                // conj(B^a) B^b
                const double re = double(ba.x) * bb.x + double(ba.y) * bb.y;
                const double im = double(ba.x) * bb.y - double(ba.y) * bb.x;
                const size_t k = (size_t(Kx0 + c) * L + Ky) * L + Kz;
                if (o.val) {
                    double* v = o.val + ((size_t(rp) * o.n_corr + cc) * n_k + k) * 2;
                    v[0] = re;
                    v[1] = im;
                }
                if (slot >= 0) {
                    double* s = o.acc_sum + size_t(slot) * o.slot_stride + (size_t(cc) * n_k + k) * 2;
                    double* q = o.acc_sq + size_t(slot) * o.slot_stride + (size_t(cc) * n_k + k) * 2;
                    s[0] += re;
                    s[1] += im;
                    q[0] += re * re;
                    q[1] += im * im;
                }
            }
        }
    }
}

bool ssf_resolved_supported(int P, int Q) { return ssf_fast_path(P, Q); }

void launch_ssf_zdft_res(const SsfGeom& g, float2* A, cudaStream_t st) {
    const int L = g.L;
    const int Cr = ssf_chunk_res(L);
    const size_t smem = sizeof(float2) * (size_t(9) * L + 48 * (size_t(L) * (Cr + 1) + 1));
    const int grid = g.n_rep * L * ((L + Cr - 1) / Cr);
    switch (L) {
        case 64: ssf_zdft_res_kernel<64><<<grid, 256, smem, st>>>(g, A); break;
        case 32: ssf_zdft_res_kernel<32><<<grid, 256, smem, st>>>(g, A); break;
        case 16: ssf_zdft_res_kernel<16><<<grid, 256, smem, st>>>(g, A); break;
        case 8: ssf_zdft_res_kernel<8><<<grid, 256, smem, st>>>(g, A); break;
        default: ssf_zdft_res_kernel<0><<<grid, 256, smem, st>>>(g, A);
    }
}

void launch_ssf_z(const SsfGeom& g, const float2* G, const SsfOut& o, cudaStream_t st) {
    const int L = g.L, C = ssf_chunk(L);
    const int n_chunk = (L + C - 1) / C;
    if (ssf_fast_path(g.P, g.Q) && g.resolved) {
        float2* A = const_cast<float2*>(G);
        launch_ssf_zdft_res(g, A, st);
        ssf_accum_res_kernel<<<g.n_rep * L * L * L, 256, 0, st>>>(g, A, o);
        return;
    }
    if (ssf_fast_path(g.P, g.Q)) {
        const size_t smem = sizeof(float2) * (size_t(9) * L + 12 * size_t(L) * (C + 1));
        const int grid = g.n_rep * L * n_chunk, threads = ssf_line_threads(L, g.P, g.Q);
        switch (L) {
            case 64: ssf_line_kernel<64><<<grid, threads, smem, st>>>(g, G, o); break;
            case 32: ssf_line_kernel<32><<<grid, threads, smem, st>>>(g, G, o); break;
            case 24: ssf_line_kernel<24><<<grid, threads, smem, st>>>(g, G, o); break;
            case 16: ssf_line_kernel<16><<<grid, threads, smem, st>>>(g, G, o); break;
            case 12: ssf_line_kernel<12><<<grid, threads, smem, st>>>(g, G, o); break;
            case 8: ssf_line_kernel<8><<<grid, threads, smem, st>>>(g, G, o); break;
            default: ssf_line_kernel<0><<<grid, threads, smem, st>>>(g, G, o);
        }
        return;
    }
    const size_t smem = sizeof(float2) * (size_t(9) * L + 5 * size_t(L) * C);
    ssf_z_kernel<<<g.n_rep * L * n_chunk, 256, smem, st>>>(g, G, o);
}

// --------------------------------------------------------------- backward
// dLoss/dS_i^c = Re sum_K exp(+i q.x_i) Y^c(K), with
// Y^c(K) = sum_corr [c == a] conj(D) B^b + [c == b] D B^a, D = dL/dReS + i dL/dImS.
// Adjoint stage z: per (replica, Ky, Kx chunk) build Y, then for each z group
// H_g(Kx,Ky,nz) = sum_Kz exp(+2pi i Kz nz/L) exp(+i qz rz) Y(Kx,Ky,Kz).
__global__ void __launch_bounds__(256) ssf_adj_z_kernel(const SsfGeom g, const SsfOut o, const double* __restrict__ dval,
                                                        const float2* __restrict__ amp, float2* __restrict__ H) {
    extern __shared__ float2 sm[];
    const int L = g.L, LL = L * L;
    const int C = ssf_chunk(L);
    const int n_chunk = (L + C - 1) / C;
    float2* tw = sm;
    float2* ph = tw + L;
    float2* Y = ph + 8 * L;      // [3][L][C]
    float2* w0 = Y + 3 * L * C;  // [L][C]
    float2* w1 = w0 + L * C;
    const int chunk = blockIdx.x % n_chunk;
    const int Ky = (blockIdx.x / n_chunk) % L;
    const int rp = (blockIdx.x / n_chunk) / L;
    const int Kx0 = chunk * C;
    const int nc = min(C, L - Kx0);
    const int n_k = L * LL;
    fill_tables(tw, ph, L);
    for (int i = threadIdx.x; i < 3 * L * C; i += blockDim.x) Y[i] = make_float2(0.f, 0.f);
    __syncthreads();
    for (int i = threadIdx.x; i < L * nc; i += blockDim.x) {
        const int Kz = i % L, c = i / L;
        const size_t k = (size_t(Kx0 + c) * L + Ky) * L + Kz;
        float2 b[3];
        for (int a = 0; a < 3; ++a) b[a] = amp[(size_t(rp) * 3 + a) * n_k + k];
        float2 y[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
        for (int cc = 0; cc < o.n_corr; ++cc) {
            const double* d = dval + ((size_t(rp) * o.n_corr + cc) * n_k + k) * 2;
            const float2 D = make_float2(float(d[0]), float(d[1]));
            const int ca = o.corr_a[cc], cb = o.corr_b[cc];
            const float2 t1 = cmulc(b[cb], D);  // conj(D) B^b
            y[ca].x += t1.x;
            y[ca].y += t1.y;
            const float2 t2 = cmul(D, b[ca]);  // D B^a
            y[cb].x += t2.x;
            y[cb].y += t2.y;
        }
        for (int a = 0; a < 3; ++a) Y[(a * L + Kz) * C + c] = y[a];
    }
    for (int a = 0; a < 3; ++a)
        for (int gz = 0; gz < 4; ++gz) {
            const int rz = 2 * gz - 1;
            __syncthreads();
            for (int i = threadIdx.x; i < L * C; i += blockDim.x) {
                const int Kz = i / C;
                w0[i] = cmulc(Y[a * L * C + i], phase(ph, L, Kz * rz));  // times exp(+i qz rz)
            }
            __syncthreads();
            dft_lines_generic<true>(w0, w1, L, g.P, g.Q, C, 1, C, tw, true);
            float2* dst = H + ((size_t(rp) * 3 + a) * 4 + gz) * size_t(L) * LL + size_t(Ky) * L + Kx0;
            for (int i = threadIdx.x; i < L * nc; i += blockDim.x) {
                const int c = i % nc, nz = i / nc;
                dst[size_t(nz) * LL + c] = w0[nz * C + c];
            }
        }
}

// Adjoint stage xy: per (replica, z plane, z group): for each sublattice of the
// group, grad^a(x,y) = Re sum_{Kx,Ky} exp(+2 pi i (Kx x + Ky y)/L)
// exp(+i(qx rx + qy ry)) H_g(Kx,Ky).
__global__ void __launch_bounds__(256) ssf_adj_xy_kernel(const SsfGeom g, const float2* __restrict__ H,
                                                         const ReplicaDev* reps, float* __restrict__ grad) {
    extern __shared__ float2 sm[];
    const int L = g.L, LL = L * L;
    float2* tw = sm;
    float2* ph = tw + L;
    float2* hp = ph + 8 * L;
    float2* w0 = hp + LL;
    float2* w1 = w0 + LL;
    const int gz = blockIdx.x & 3;
    const int nz = (blockIdx.x >> 2) % L;
    const int rp = (blockIdx.x >> 2) / L;
    const ReplicaDev rep = reps[g.rep_index[rp]];
    fill_tables(tw, ph, L);
    for (int a = 0; a < 3; ++a) {
        const float2* src = H + ((size_t(rp) * 3 + a) * 4 + gz) * size_t(L) * LL + size_t(nz) * LL;
        __syncthreads();
        for (int i = threadIdx.x; i < LL; i += blockDim.x) hp[i] = src[i];
        for (int m = 0; m < 4; ++m) {
            const int sl = c_zgroup[gz][m];
            const int rx = c_rsl[sl][0], ry = c_rsl[sl][1];
            __syncthreads();
            for (int i = threadIdx.x; i < LL; i += blockDim.x) {
                const int Kx = i % L, Ky = i / L;
                const float2 p = cmul(phase(ph, L, Kx * rx), phase(ph, L, Ky * ry));
                w0[i] = cmulc(hp[i], p);
            }
            __syncthreads();
            dft_lines_generic<true>(w0, w1, L, g.P, g.Q, L, 1, L, tw, true);   // along y
            dft_lines_generic<true>(w0, w1, L, g.P, g.Q, L, L, 1, tw, false);  // along x
            float* dst = grad + 4 * (size_t(rep.off) + size_t(sl) * rep.Nc + size_t(nz) * LL) + a;
            for (int i = threadIdx.x; i < LL; i += blockDim.x) dst[4 * size_t(i)] = w0[i].x;
        }
    }
}

template <bool RES>
void prepare_plane(int smem_max) {
    cudaFuncSetAttribute(ssf_plane_kernel<64, true, RES>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_plane_kernel<32, true, RES>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_plane_kernel<16, true, RES>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_plane_kernel<8, false, RES>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_plane_kernel<12, false, RES>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_plane_kernel<24, false, RES>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_plane_kernel<0, true, RES>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_plane_kernel<0, false, RES>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
}

void ssf_prepare() {
    const int smem_max = 200 * 1024;
    prepare_plane<false>(smem_max);
    prepare_plane<true>(smem_max);
    cudaFuncSetAttribute(ssf_zdft_res_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_zdft_res_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_zdft_res_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_zdft_res_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_zdft_res_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_line_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_line_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_line_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_line_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_line_kernel<12>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_line_kernel<24>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_line_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_line_adj_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_line_adj_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_line_adj_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_line_adj_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_line_adj_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_plane_adj_kernel<64, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_plane_adj_kernel<32, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_plane_adj_kernel<16, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_plane_adj_kernel<8, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_plane_adj_kernel<0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_plane_adj_kernel<0, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ssf_xy_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(ssf_z_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(ssf_adj_z_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(ssf_adj_xy_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

void launch_ssf_adjoint(const SsfGeom& g, const SsfOut& o, const double* dval, const float2* amp, float2* H,
                        float4* grad_S, const ReplicaDev* reps, cudaStream_t st) {
    const int L = g.L, C = ssf_chunk(L);
    const int n_chunk = (L + C - 1) / C;
    if (ssf_fast_path(g.P, g.Q)) {
        const size_t smem_z = sizeof(float2) * (size_t(9) * L + 12 * size_t(L) * (C + 1));
        const int grid_z = g.n_rep * L * n_chunk, thr_z = ssf_line_threads(L, g.P, g.Q);
        const size_t smem_xy = sizeof(float2) * (size_t(9) * L + 3 * size_t(L) * L);
        const int grid_xy = g.n_rep * L * 8, thr_xy = ssf_plane_threads(L);
        switch (L) {
            case 64:
                ssf_line_adj_kernel<64><<<grid_z, thr_z, smem_z, st>>>(g, o, dval, amp, H);
                ssf_plane_adj_kernel<64, true><<<grid_xy, thr_xy, smem_xy, st>>>(g, H, reps, grad_S);
                break;
            case 32:
                ssf_line_adj_kernel<32><<<grid_z, thr_z, smem_z, st>>>(g, o, dval, amp, H);
                ssf_plane_adj_kernel<32, true><<<grid_xy, thr_xy, smem_xy, st>>>(g, H, reps, grad_S);
                break;
            case 16:
                ssf_line_adj_kernel<16><<<grid_z, thr_z, smem_z, st>>>(g, o, dval, amp, H);
                ssf_plane_adj_kernel<16, true><<<grid_xy, thr_xy, smem_xy, st>>>(g, H, reps, grad_S);
                break;
            case 8:
                ssf_line_adj_kernel<8><<<grid_z, thr_z, smem_z, st>>>(g, o, dval, amp, H);
                ssf_plane_adj_kernel<8, false><<<grid_xy, thr_xy, smem_xy, st>>>(g, H, reps, grad_S);
                break;
            default:
                ssf_line_adj_kernel<0><<<grid_z, thr_z, smem_z, st>>>(g, o, dval, amp, H);
                if (L % 16 == 0)
                    ssf_plane_adj_kernel<0, true><<<grid_xy, thr_xy, smem_xy, st>>>(g, H, reps, grad_S);
                else
                    ssf_plane_adj_kernel<0, false><<<grid_xy, thr_xy, smem_xy, st>>>(g, H, reps, grad_S);
        }
        return;
    }
    const size_t smem_z = sizeof(float2) * (size_t(9) * L + 5 * size_t(L) * C);
    ssf_adj_z_kernel<<<g.n_rep * L * n_chunk, 256, smem_z, st>>>(g, o, dval, amp, H);
    const size_t smem_xy = sizeof(float2) * (size_t(9) * L + 3 * size_t(L) * L);
    ssf_adj_xy_kernel<<<g.n_rep * L * 4, 256, smem_xy, st>>>(g, H, reps, reinterpret_cast<float*>(grad_S));
}

}  // namespace pc
