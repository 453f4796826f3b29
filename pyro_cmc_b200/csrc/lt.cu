// lt.cu -- the Luttinger-Tisza bound of src/luttinger_tisza.cpp on the GPU.
//
// For every k of the L^3 grid the 48 x 48 Hermitian matrix
//   M(k)[3a+i][3b+j] = sum over directed bonds a -> b (displacement d) of
//                      J_bond[i][j] exp(i k.d)                 (:153-166)
// (bonds of build_bonds, :31-81: J1 (XXZ: J1[I + (Delta-1) z_mu z_nu^T]), J2,
// J3a, J3b from every one of the 16 sublattices, zero couplings skipped) is
// reduced to a real symmetric tridiagonal matrix by Householder reflections
// in FP64 shared memory (one CTA per k), and its smallest eigenvalue is found
// by Sturm-sequence bisection. The eigenvector at the minimising k* comes from
// inverse iteration (LU with partial pivoting of M - sigma I). E/spin =
// lambda_min / 2 (:181). k = 2 pi K / (8 L), the S(q) grid.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <limits>
#include <string>
#include <vector>

#include "../../include/pyrocmc.h"

namespace pc {
void set_last_error(const std::string& msg);
}

namespace {

constexpr int kN = 48;     // 3 spin components x 16 sublattices
constexpr int kMaxD = 8;   // |d| components of the bond displacements are <= 4 (cell side 8)
constexpr int kPh = 2 * kMaxD + 1;

struct LtBond {
    int a, b;     // source / target sublattice
    int d[3];     // displacement (coordinate units)
    double J[9];  // row-major 3x3
};

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// M(k) into A (row-major, both triangles): thread per (pair of sublattices),
// bonds grouped by (a, b) through pair_begin[a*16 + b] .. pair_begin[+1].
__device__ void build_M(double2* A, const LtBond* bonds, const int* pair_begin, const double2 (*ph)[kPh]) {
    for (int e = threadIdx.x; e < kN * kN; e += blockDim.x) A[e] = make_double2(0.0, 0.0);
    __syncthreads();
    for (int pr = threadIdx.x; pr < 256; pr += blockDim.x) {
        const int a = pr >> 4, b = pr & 15;
        double2 acc[9];
        for (int q = 0; q < 9; ++q) acc[q] = make_double2(0.0, 0.0);
        for (int t = pair_begin[pr]; t < pair_begin[pr + 1]; ++t) {
            const LtBond& bd = bonds[t];
            const double2 e = cmul(cmul(ph[0][bd.d[0] + kMaxD], ph[1][bd.d[1] + kMaxD]), ph[2][bd.d[2] + kMaxD]);
            for (int q = 0; q < 9; ++q) acc[q] = cadd(acc[q], make_double2(bd.J[q] * e.x, bd.J[q] * e.y));
        }
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) A[(3 * a + i) * kN + 3 * b + j] = cadd(A[(3 * a + i) * kN + 3 * b + j], acc[3 * i + j]);
    }
    __syncthreads();
}

__device__ void fill_phases(double2 (*ph)[kPh], const int K[3], int L) {
    for (int t = threadIdx.x; t < 3 * kPh; t += blockDim.x) {
        const int ax = t / kPh, dd = t % kPh - kMaxD;
        double s, c;
        sincospi(2.0 * double(K[ax]) * double(dd) / (8.0 * double(L)), &s, &c);
        ph[ax][t % kPh] = make_double2(c, s);
    }
    __syncthreads();
}

// Number of eigenvalues of the tridiagonal (d, b) below x (Sturm count).
__device__ int sturm_count(const double* d, const double* b2, double x) {
    int cnt = 0;
    double q = d[0] - x;
    if (q < 0) ++cnt;
    for (int i = 1; i < kN; ++i) {
        if (q == 0.0) q = -1e-300;
        q = (d[i] - x) - b2[i - 1] / q;
        if (q < 0) ++cnt;
    }
    return cnt;
}

__global__ void __launch_bounds__(128) lt_min_kernel(const LtBond* __restrict__ bonds, const int* __restrict__ pair_begin,
                                                     int L, double* __restrict__ lambda_min) {
    extern __shared__ double2 A[];  // kN*kN
    __shared__ double2 v[kN], p[kN];
    __shared__ double2 ph[3][kPh];
    __shared__ double dg[kN], b2[kN];
    __shared__ double red[4];
    const int n_k = L * L * L;
    for (int kf = blockIdx.x; kf < n_k; kf += gridDim.x) {
        const int K[3] = {kf / (L * L), (kf / L) % L, kf % L};
        fill_phases(ph, K, L);
        build_M(A, bonds, pair_begin, ph);
        // Householder: column k below the diagonal -> alpha e1
        for (int k = 0; k < kN - 2; ++k) {
            const int m = kN - k - 1;  // length of x = A[k+1.., k]
            if (threadIdx.x == 0) {
                double sig = 0.0;
                for (int i = 1; i < m; ++i) {
                    const double2 x = A[(k + 1 + i) * kN + k];
                    sig += x.x * x.x + x.y * x.y;
                }
                const double2 x0 = A[(k + 1) * kN + k];
                const double ax0 = sqrt(x0.x * x0.x + x0.y * x0.y);
                const double xn = sqrt(ax0 * ax0 + sig);
                dg[k] = A[k * kN + k].x;
                b2[k] = xn * xn;
                red[0] = xn;
                if (xn > 0.0 && sig > 0.0) {
                    const double2 phs = ax0 > 0.0 ? make_double2(x0.x / ax0, x0.y / ax0) : make_double2(1.0, 0.0);
                    const double2 alpha = make_double2(-phs.x * xn, -phs.y * xn);
                    const double2 v0 = make_double2(x0.x - alpha.x, x0.y - alpha.y);
                    red[1] = 2.0 / (v0.x * v0.x + v0.y * v0.y + sig);  // beta
                    v[0] = v0;
                } else {
                    red[1] = 0.0;  // already reduced
                }
            }
            __syncthreads();
            const double beta = red[1];
            if (beta == 0.0) {
                __syncthreads();
                continue;
            }
            for (int i = 1 + threadIdx.x; i < m; i += blockDim.x) v[i] = A[(k + 1 + i) * kN + k];
            __syncthreads();
            // p = beta * A_sub v
            for (int i = threadIdx.x; i < m; i += blockDim.x) {
                double2 s = make_double2(0.0, 0.0);
                const double2* row = A + (k + 1 + i) * kN + (k + 1);
                for (int j = 0; j < m; ++j) s = cadd(s, cmul(row[j], v[j]));
                p[i] = make_double2(beta * s.x, beta * s.y);
            }
            __syncthreads();
            if (threadIdx.x == 0) {  // K = beta/2 v^H p (real)
                double s = 0.0;
                for (int i = 0; i < m; ++i) s += v[i].x * p[i].x + v[i].y * p[i].y;
                red[2] = 0.5 * beta * s;
            }
            __syncthreads();
            const double Kc = red[2];
            for (int i = threadIdx.x; i < m; i += blockDim.x) p[i] = make_double2(p[i].x - Kc * v[i].x, p[i].y - Kc * v[i].y);
            __syncthreads();
            // A_sub -= v w^H + w v^H   (w = p)
            for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
                const int i = e / m, j = e % m;
                double2& a = A[(k + 1 + i) * kN + (k + 1 + j)];
                const double2 t1 = cmul(v[i], cconj(p[j])), t2 = cmul(p[i], cconj(v[j]));
                a = make_double2(a.x - t1.x - t2.x, a.y - t1.y - t2.y);
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            dg[kN - 2] = A[(kN - 2) * kN + kN - 2].x;
            dg[kN - 1] = A[(kN - 1) * kN + kN - 1].x;
            const double2 e = A[(kN - 1) * kN + kN - 2];
            b2[kN - 2] = e.x * e.x + e.y * e.y;
            // Gershgorin bounds, then bisection for the smallest eigenvalue
            double lo = 1e300, hi = -1e300;
            for (int i = 0; i < kN; ++i) {
                const double r = (i > 0 ? sqrt(b2[i - 1]) : 0.0) + (i < kN - 1 ? sqrt(b2[i]) : 0.0);
                lo = fmin(lo, dg[i] - r);
                hi = fmax(hi, dg[i] + r);
            }
            for (int it = 0; it < 200 && hi - lo > 1e-15 * fmax(1.0, fmax(fabs(lo), fabs(hi))); ++it) {
                const double mid = 0.5 * (lo + hi);
                if (sturm_count(dg, b2, mid) >= 1)
                    hi = mid;
                else
                    lo = mid;
            }
            lambda_min[kf] = 0.5 * (lo + hi);
        }
        __syncthreads();
    }
}

// Inverse iteration at one k: (M - sigma I) x = b by LU with partial pivoting
// (one thread; 48 x 48), three iterations from b = (1, ..., 1).
__global__ void lt_vector_kernel(const LtBond* __restrict__ bonds, const int* __restrict__ pair_begin, int L, int kf,
                                 double sigma, double2* __restrict__ out) {
    extern __shared__ double2 A[];
    __shared__ double2 ph[3][kPh];
    __shared__ double2 x[kN];
    __shared__ int piv[kN];
    const int K[3] = {kf / (L * L), (kf / L) % L, kf % L};
    fill_phases(ph, K, L);
    build_M(A, bonds, pair_begin, ph);
    if (threadIdx.x != 0) return;
    for (int i = 0; i < kN; ++i) A[i * kN + i].x -= sigma;
    for (int c = 0; c < kN; ++c) {  // LU, row pivoting
        int best = c;
        double bm = -1.0;
        for (int r = c; r < kN; ++r) {
            const double2 a = A[r * kN + c];
            const double m2 = a.x * a.x + a.y * a.y;
            if (m2 > bm) {
                bm = m2;
                best = r;
            }
        }
        piv[c] = best;
        if (best != c)
            for (int j = 0; j < kN; ++j) {
                const double2 t = A[c * kN + j];
                A[c * kN + j] = A[best * kN + j];
                A[best * kN + j] = t;
            }
        double2 d = A[c * kN + c];
        if (d.x == 0.0 && d.y == 0.0) d = make_double2(1e-300, 0.0);
        const double dn = d.x * d.x + d.y * d.y;
        const double2 inv = make_double2(d.x / dn, -d.y / dn);
        for (int r = c + 1; r < kN; ++r) {
            const double2 f = cmul(A[r * kN + c], inv);
            A[r * kN + c] = f;
            for (int j = c + 1; j < kN; ++j) {
                const double2 t = cmul(f, A[c * kN + j]);
                A[r * kN + j] = make_double2(A[r * kN + j].x - t.x, A[r * kN + j].y - t.y);
            }
        }
    }
    for (int i = 0; i < kN; ++i) x[i] = make_double2(1.0, 0.0);
    for (int iter = 0; iter < 3; ++iter) {
        for (int c = 0; c < kN; ++c)
            if (piv[c] != c) {
                const double2 t = x[c];
                x[c] = x[piv[c]];
                x[piv[c]] = t;
            }
        for (int r = 1; r < kN; ++r)  // L y = b (unit lower)
            for (int j = 0; j < r; ++j) {
                const double2 t = cmul(A[r * kN + j], x[j]);
                x[r] = make_double2(x[r].x - t.x, x[r].y - t.y);
            }
        for (int r = kN - 1; r >= 0; --r) {  // U x = y
            for (int j = r + 1; j < kN; ++j) {
                const double2 t = cmul(A[r * kN + j], x[j]);
                x[r] = make_double2(x[r].x - t.x, x[r].y - t.y);
            }
            double2 d = A[r * kN + r];
            if (d.x == 0.0 && d.y == 0.0) d = make_double2(1e-300, 0.0);
            const double dn = d.x * d.x + d.y * d.y;
            x[r] = cmul(x[r], make_double2(d.x / dn, -d.y / dn));
        }
        double nrm = 0.0;
        for (int i = 0; i < kN; ++i) nrm += x[i].x * x[i].x + x[i].y * x[i].y;
        nrm = 1.0 / sqrt(nrm);
        for (int i = 0; i < kN; ++i) x[i] = make_double2(x[i].x * nrm, x[i].y * nrm);
    }
    for (int i = 0; i < kN; ++i) out[i] = x[i];
}

// The unwrapped sublattice offsets r_sl = link[p] + R_fcc[f], sl = 4f + p
// (include/pyrochlore_geometry.hpp:16-29), and the sublattice at a position.
const int kLinkLt[4][3] = {{1, 1, 1}, {1, -1, -1}, {-1, 1, -1}, {-1, -1, 1}};
const int kFccLt[4][3] = {{0, 0, 0}, {0, 4, 4}, {4, 0, 4}, {4, 4, 0}};
int lt_sl_of(const int x[3]) {
    for (int sl = 0; sl < 16; ++sl) {
        bool ok = true;
        for (int a = 0; a < 3; ++a)
            ok = ok && ((x[a] - kLinkLt[sl % 4][a] - kFccLt[sl / 4][a]) % 8 + 8) % 8 == 0;
        if (ok) return sl;
    }
    return -1;
}

int lt_fail(int code, const std::string& m) {
    pc::set_last_error(m);
    return code;
}

}  // namespace

extern "C" int pc_lt_minimum(int L, double J1, double J2, double J3, double Delta, double* lambda_map,
                             double* e_per_spin, int64_t* k_star, double* eigvec) {
    if (L < 1 || L > 256) return lt_fail(PC_ERR_INVALID, "LT: L must be in [1, 256]");
    // build_bonds (src/luttinger_tisza.cpp:31-81)
    const double s3 = std::sqrt(3.0);
    std::vector<LtBond> bonds;
    const double js[4] = {J1, J2, J3, J3};
    for (int kind = 1; kind <= 4; ++kind) {
        const double j = js[kind - 1];
        if (j == 0.0) continue;
        for (int a = 0; a < 16; ++a) {
            int64_t dd[3 * 64];
            int n = 0;
            const int rc = pc_pyrochlore_displacements(kind, a % 4, dd, 64, &n);
            if (rc) return rc;
            for (int t = 0; t < n; ++t) {
                LtBond b;
                b.a = a;
                int x[3];
                for (int q = 0; q < 3; ++q) {
                    b.d[q] = int(dd[3 * t + q]);
                    x[q] = kLinkLt[a % 4][q] + kFccLt[a / 4][q] + b.d[q];
                }
                b.b = lt_sl_of(x);
                if (b.b < 0) return lt_fail(PC_ERR_UNSUPPORTED, "LT: bond target is not a site");
                for (int p = 0; p < 3; ++p)
                    for (int q = 0; q < 3; ++q) {
                        double v = (p == q) ? 1.0 : 0.0;
                        if (kind == 1 && Delta != 1.0)
                            v += (Delta - 1.0) * (kLinkLt[a % 4][p] / s3) * (kLinkLt[b.b % 4][q] / s3);
                        b.J[3 * p + q] = j * v;
                    }
                bonds.push_back(b);
            }
        }
    }
    std::stable_sort(bonds.begin(), bonds.end(),
                     [](const LtBond& x, const LtBond& y) { return x.a * 16 + x.b < y.a * 16 + y.b; });
    std::vector<int> pair_begin(257, 0);
    for (const auto& b : bonds) pair_begin[size_t(b.a * 16 + b.b) + 1]++;
    for (int i = 0; i < 256; ++i) pair_begin[size_t(i) + 1] += pair_begin[size_t(i)];
    const int n_k = L * L * L;
    LtBond* d_bonds = nullptr;
    int* d_pb = nullptr;
    double* d_lam = nullptr;
    double2* d_vec = nullptr;
    cudaStream_t st = nullptr;
    auto cleanup = [&]() {
        if (st) cudaStreamSynchronize(st);
        cudaFree(d_bonds);
        cudaFree(d_pb);
        cudaFree(d_lam);
        cudaFree(d_vec);
        if (st) cudaStreamDestroy(st);
    };
    auto ck = [&](cudaError_t e) -> int {
        if (e == cudaSuccess) return PC_OK;
        cleanup();
        return lt_fail(PC_ERR_CUDA, std::string("LT: ") + cudaGetErrorString(e));
    };
    int rc = ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    if (rc) return rc;
    if ((rc = ck(cudaMalloc(&d_bonds, sizeof(LtBond) * std::max<size_t>(1, bonds.size()))))) return rc;
    if ((rc = ck(cudaMalloc(&d_pb, sizeof(int) * 257)))) return rc;
    if ((rc = ck(cudaMalloc(&d_lam, sizeof(double) * size_t(n_k))))) return rc;
    if ((rc = ck(cudaMalloc(&d_vec, sizeof(double2) * kN)))) return rc;
    if (!bonds.empty() &&
        (rc = ck(cudaMemcpyAsync(d_bonds, bonds.data(), sizeof(LtBond) * bonds.size(), cudaMemcpyHostToDevice, st))))
        return rc;
    if ((rc = ck(cudaMemcpyAsync(d_pb, pair_begin.data(), sizeof(int) * 257, cudaMemcpyHostToDevice, st)))) return rc;
    const size_t smem = sizeof(double2) * kN * kN;
    if ((rc = ck(cudaFuncSetAttribute(lt_min_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)))))
        return rc;
    if ((rc = ck(cudaFuncSetAttribute(lt_vector_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)))))
        return rc;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    lt_min_kernel<<<std::min(n_k, sms * 8), 128, smem, st>>>(d_bonds, d_pb, L, d_lam);
    if ((rc = ck(cudaGetLastError()))) return rc;
    std::vector<double> lam(static_cast<size_t>(n_k));
    if ((rc = ck(cudaMemcpyAsync(lam.data(), d_lam, sizeof(double) * size_t(n_k), cudaMemcpyDeviceToHost, st)))) return rc;
    if ((rc = ck(cudaStreamSynchronize(st)))) return rc;
    // the first k in flat order attaining the minimum (the reference keeps the first strict minimum)
    int kbest = 0;
    for (int k = 1; k < n_k; ++k)
        if (lam[size_t(k)] < lam[size_t(kbest)]) kbest = k;
    const double lmin = lam[size_t(kbest)];
    if (lambda_map) std::copy(lam.begin(), lam.end(), lambda_map);
    if (e_per_spin) *e_per_spin = 0.5 * lmin;
    if (k_star) {
        k_star[0] = kbest / (L * L);
        k_star[1] = (kbest / L) % L;
        k_star[2] = kbest % L;
    }
    if (eigvec) {
        const double sigma = lmin - 1e-9 * std::max(1.0, std::fabs(lmin));
        lt_vector_kernel<<<1, 64, smem, st>>>(d_bonds, d_pb, L, kbest, sigma, d_vec);
        if ((rc = ck(cudaGetLastError()))) return rc;
        std::vector<double2> vec(static_cast<size_t>(kN));
        if ((rc = ck(cudaMemcpyAsync(vec.data(), d_vec, sizeof(double2) * kN, cudaMemcpyDeviceToHost, st)))) return rc;
        if ((rc = ck(cudaStreamSynchronize(st)))) return rc;
        for (int i = 0; i < kN; ++i) {
            eigvec[2 * i] = vec[size_t(i)].x;
            eigvec[2 * i + 1] = vec[size_t(i)].y;
        }
    }
    cleanup();
    return PC_OK;
}
