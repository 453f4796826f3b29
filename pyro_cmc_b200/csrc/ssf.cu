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

#include "common.cuh"
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
__device__ __forceinline__ void dft_lines(float2* a, float2* b, int L, int P, int Q, int n_lines, int lstride,
                                          int estride, const float2* tw, bool line_fast) {
    ct_half<false, INV>(a, b, L, P, Q, n_lines, lstride, estride, tw, line_fast);
    __syncthreads();
    ct_half<true, INV>(b, a, L, P, Q, n_lines, lstride, estride, tw, line_fast);
    __syncthreads();
}

// ------------------------------------------------------------------ stage 1
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
            dft_lines<false>(w0, w1, L, g.P, g.Q, L, L, 1, tw, false);  // along x (rows)
            dft_lines<false>(w0, w1, L, g.P, g.Q, L, 1, L, tw, true);   // along y (columns)
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

__host__ __device__ __forceinline__ int ssf_chunk(int L) { return L < 16 ? L : 16; }

void launch_ssf_xy(const SsfGeom& g, const float4* spins, const ReplicaDev* reps, float2* G, cudaStream_t st) {
    const int L = g.L;
    const size_t smem = sizeof(float2) * (size_t(9) * L + 3 * size_t(L) * L);
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
            dft_lines<false>(w0, w1, L, g.P, g.Q, C, 1, C, tw, true);  // along z
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

void launch_ssf_z(const SsfGeom& g, const float2* G, const SsfOut& o, cudaStream_t st) {
    const int L = g.L, C = ssf_chunk(L);
    const int n_chunk = (L + C - 1) / C;
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
            dft_lines<true>(w0, w1, L, g.P, g.Q, C, 1, C, tw, true);
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
            dft_lines<true>(w0, w1, L, g.P, g.Q, L, 1, L, tw, true);   // along y
            dft_lines<true>(w0, w1, L, g.P, g.Q, L, L, 1, tw, false);  // along x
            float* dst = grad + 4 * (size_t(rep.off) + size_t(sl) * rep.Nc + size_t(nz) * LL) + a;
            for (int i = threadIdx.x; i < LL; i += blockDim.x) dst[4 * size_t(i)] = w0[i].x;
        }
    }
}

void ssf_prepare() {
    cudaFuncSetAttribute(ssf_xy_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(ssf_z_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(ssf_adj_z_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(ssf_adj_xy_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

void launch_ssf_adjoint(const SsfGeom& g, const SsfOut& o, const double* dval, const float2* amp, float2* H,
                        float4* grad_S, const ReplicaDev* reps, cudaStream_t st) {
    const int L = g.L, C = ssf_chunk(L);
    const int n_chunk = (L + C - 1) / C;
    const size_t smem_z = sizeof(float2) * (size_t(9) * L + 5 * size_t(L) * C);
    ssf_adj_z_kernel<<<g.n_rep * L * n_chunk, 256, smem_z, st>>>(g, o, dval, amp, H);
    const size_t smem_xy = sizeof(float2) * (size_t(9) * L + 3 * size_t(L) * L);
    ssf_adj_xy_kernel<<<g.n_rep * L * 4, 256, smem_xy, st>>>(g, H, reps, reinterpret_cast<float*>(grad_S));
}

}  // namespace pc
