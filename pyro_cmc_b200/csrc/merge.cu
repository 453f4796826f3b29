// merge.cu -- merging seed-repeated S(q) accumulators on the device
// (scripts/acc_runs.py:228-370, merge_group, and :103-167, plane_invariants).
//
// K accumulator slots (one per seed, the same temperature, the same sample
// count n per seed) are merged per (correlator, k, re/im):
//   static_corr   = sum_s C_s               (C_s: a seed's raw sum of S(q))
//   static_corr_2 = sum_s C_s^2             (inter-seed second moment)
//   var_inter     = static_corr_2/(K n^2) - (static_corr/(K n))^2
//   var_intra     = sum_s Q_s / n - static_corr_2 / n^2
//                   (Q_s: a seed's sum of squared samples, the slot's sq sums)
// and per seed and k the O(3)-invariant spiral-plane observables of the
// seed's thermal average M = C_s / n (needs xx, yy, zz, xy, xz, yz):
//   T = Re M_sym - tr/3,  w = 3 sqrt(6) det T / max(Tr(T^2)^{3/2}, floor),
//   chi_frac = |kappa| / max(tr, tr_floor), kappa^2 = 4 (Im M_yz^2 + Im M_xz^2 + Im M_xy^2),
// with the per-seed floors 1e-6 max_k Tr(T^2)^{3/2} and 1e-6 max_k tr + 1e-30.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "kernels.h"

namespace pc {

__global__ void merge_sums_kernel(const MergeArgs a) {
    const int64_t total = int64_t(a.n_corr) * a.n_k * 2;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
        double c = 0.0, c2 = 0.0, q = 0.0;
        for (int s = 0; s < a.K; ++s) {  // seeds in slot order: a fixed summation order
            const size_t off = size_t(a.slots[s]) * a.slot_stride + size_t(e);
            const double v = a.sum[off];
            c += v;
            c2 += v * v;
            q += a.sq[off];
        }
        a.out_corr[e] = c;
        a.out_corr2[e] = c2;
        const double n = a.n, K = double(a.K);
        a.out_var_inter[e] = c2 / (K * n * n) - (c / (K * n)) * (c / (K * n));
        if (a.out_var_intra) a.out_var_intra[e] = q / n - c2 / (n * n);
    }
}

// Per seed s and k: the seed's thermal average M = C_s / n of the six correlators.
struct Plane {
    double Txx, Tyy, Tzz, Txy, Txz, Tyz, tr, I2, det, kappa2;
};
__device__ Plane plane_at(const MergeArgs& a, int s, int k) {
    const double* base = a.sum + size_t(a.slots[s]) * a.slot_stride;
    auto re = [&](int c) { return base[(size_t(a.ix[c]) * a.n_k + k) * 2] / a.n; };
    auto im = [&](int c) { return base[(size_t(a.ix[c]) * a.n_k + k) * 2 + 1] / a.n; };
    Plane p;
    const double Mxx = re(0), Myy = re(1), Mzz = re(2);
    p.tr = Mxx + Myy + Mzz;
    const double t = p.tr / 3.0;
    p.Txx = Mxx - t;
    p.Tyy = Myy - t;
    p.Tzz = Mzz - t;
    p.Txy = re(3);
    p.Txz = re(4);
    p.Tyz = re(5);
    p.I2 = p.Txx * p.Txx + p.Tyy * p.Tyy + p.Tzz * p.Tzz + 2.0 * (p.Txy * p.Txy + p.Txz * p.Txz + p.Tyz * p.Tyz);
    p.det = p.Txx * (p.Tyy * p.Tzz - p.Tyz * p.Tyz) - p.Txy * (p.Txy * p.Tzz - p.Tyz * p.Txz) +
            p.Txz * (p.Txy * p.Tyz - p.Tyy * p.Txz);
    const double iyz = im(5), ixz = im(4), ixy = im(3);
    p.kappa2 = 4.0 * (iyz * iyz + ixz * ixz + ixy * ixy);
    return p;
}

__global__ void plane_max_kernel(const MergeArgs a) {
    const int s = blockIdx.y;
    double m1 = 0.0, m2 = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.n_k; k += gridDim.x * blockDim.x) {
        const Plane p = plane_at(a, s, k);
        m1 = fmax(m1, pow(p.I2, 1.5));
        m2 = fmax(m2, p.tr);
    }
    for (int o = 16; o > 0; o >>= 1) {
        m1 = fmax(m1, __shfl_down_sync(0xffffffffu, m1, o));
        m2 = fmax(m2, __shfl_down_sync(0xffffffffu, m2, o));
    }
    if ((threadIdx.x & 31) == 0) {  // non-negative doubles order like their bit patterns
        atomicMax(a.max_bits + 2 * s, (unsigned long long)__double_as_longlong(m1));
        atomicMax(a.max_bits + 2 * s + 1, (unsigned long long)__double_as_longlong(fmax(m2, 0.0)));
    }
}

__global__ void plane_kernel(const MergeArgs a) {
    const int s = blockIdx.y;
    const double floor_w = 1e-6 * __longlong_as_double(a.max_bits[2 * s]);
    const double floor_t = 1e-6 * __longlong_as_double(a.max_bits[2 * s + 1]) + 1e-30;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.n_k; k += gridDim.x * blockDim.x) {
        const Plane p = plane_at(a, s, k);
        const double w = 3.0 * sqrt(6.0) * p.det / fmax(pow(p.I2, 1.5), floor_w);
        a.w[size_t(s) * a.n_k + k] = fmin(1.0, fmax(-1.0, w));
        a.chi[size_t(s) * a.n_k + k] = fmin(1.0, fmax(0.0, sqrt(p.kappa2) / fmax(p.tr, floor_t)));
        a.tr[size_t(s) * a.n_k + k] = p.tr;
    }
}

void launch_ssf_merge(const MergeArgs& a, cudaStream_t st) {
    const int64_t total = int64_t(a.n_corr) * a.n_k * 2;
    const int grid = int(std::min<int64_t>((total + 255) / 256, 148 * 16));
    merge_sums_kernel<<<grid, 256, 0, st>>>(a);
    if (a.w) {
        const dim3 g2(unsigned(std::min(64, (a.n_k + 255) / 256)), unsigned(a.K));
        plane_max_kernel<<<g2, 256, 0, st>>>(a);
        plane_kernel<<<g2, 256, 0, st>>>(a);
    }
}

}  // namespace pc
