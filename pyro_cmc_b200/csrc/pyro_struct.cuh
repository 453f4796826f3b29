// pyro_struct.cuh -- the pyrochlore bond structure as compile-time constants.
//
// Every site of sublattice sl = 4f + p has 30 structural neighbours: 6 at
// |d|^2 = 8 (J1; two on each other pyro sublattice nu), 12 at |d|^2 = 24 (J2)
// and 12 at |d|^2 = 32 (J3), split into J3a (the midpoint is a site) and J3b
// (include/pyrochlore_geometry.hpp:110-149). They are derived here from the
// cell geometry by constexpr evaluation, so the sweep kernels address
// neighbours with compile-time offsets. Groups: 0..2 = J1 to the other pyro
// sublattices in increasing order, 3 = J2, 4 = J3a, 5 = J3b.
#pragma once

#include <stdint.h>

namespace pc {

constexpr int kStructNb = 30;
constexpr int kGroups = 6;

struct SNb {
    int sl, dx, dy, dz;
};
struct SStruct {
    SNb nb[kStructNb];
    int gbegin[kGroups + 1];
    int gnu[3];  // target pyro sublattice of the J1 groups
};

__host__ __device__ constexpr int cs_link(int p, int a) {
    return (p == 0) ? 1 : (p == 1) ? (a == 0 ? 1 : -1) : (p == 2) ? (a == 1 ? 1 : -1) : (a == 2 ? 1 : -1);
}
__host__ __device__ constexpr int cs_fcc(int f, int a) {
    return (f == 0) ? 0 : (f == 1) ? (a == 0 ? 0 : 4) : (f == 2) ? (a == 1 ? 0 : 4) : (a == 2 ? 0 : 4);
}
__host__ __device__ constexpr int cs_r(int sl, int a) { return cs_link(sl % 4, a) + cs_fcc(sl / 4, a); }
__host__ __device__ constexpr int cs_mod8(int a) { return ((a % 8) + 8) % 8; }
__host__ __device__ constexpr int cs_sl_at(int x, int y, int z) {
    for (int sl = 0; sl < 16; ++sl)
        if (cs_mod8(x - cs_r(sl, 0)) == 0 && cs_mod8(y - cs_r(sl, 1)) == 0 && cs_mod8(z - cs_r(sl, 2)) == 0) return sl;
    return -1;
}
// floor((x - r) / 8) for x - r a multiple of 8
__host__ __device__ constexpr int cs_cell_off(int x, int r) { return (x - r) >= 0 ? (x - r) / 8 : -((r - x) / 8); }

// Group of displacement (dx,dy,dz) from sublattice sl, or -1 if not structural.
__host__ __device__ constexpr int cs_group(int sl, int dx, int dy, int dz) {
    const int r2 = dx * dx + dy * dy + dz * dz;
    const int x = cs_r(sl, 0) + dx, y = cs_r(sl, 1) + dy, z = cs_r(sl, 2) + dz;
    const int s2 = cs_sl_at(x, y, z);
    if (s2 < 0) return -1;
    const int p = sl % 4, nu = s2 % 4;
    if (r2 == 8) {
        int k = 0;
        for (int q = 0; q < 4; ++q) {
            if (q == p) continue;
            if (q == nu) return k;
            ++k;
        }
        return -1;
    }
    if (r2 == 24) return 3;
    if (r2 == 32) return cs_sl_at(cs_r(sl, 0) + dx / 2, cs_r(sl, 1) + dy / 2, cs_r(sl, 2) + dz / 2) >= 0 ? 4 : 5;
    return -1;
}

// The 48 candidate displacements: the permutations and sign choices of
// (0,2,2) (|d|^2 = 8), (2,2,4) (24) and (4,4,0) (32).
__host__ __device__ constexpr int cs_candidate(int i, int a) {
    // i in [0,48): pattern block, then permutation, then signs
    const int pat = i < 12 ? 0 : (i < 36 ? 1 : 2);
    const int j = pat == 0 ? i : (pat == 1 ? i - 12 : i - 36);
    int v[3] = {0, 0, 0};
    if (pat == 0) {  // (0, +-2, +-2): zero position (3) x signs (4)
        const int zpos = j / 4, sg = j % 4;
        int k = 0;
        for (int c = 0; c < 3; ++c) {
            if (c == zpos) continue;
            v[c] = ((sg >> k) & 1) ? -2 : 2;
            ++k;
        }
    } else if (pat == 1) {  // (+-2, +-2, +-4): position of the 4 (3) x signs (8)
        const int fpos = j / 8, sg = j % 8;
        for (int c = 0; c < 3; ++c) v[c] = (c == fpos ? 4 : 2) * (((sg >> c) & 1) ? -1 : 1);
    } else {  // (+-4, +-4, 0): zero position (3) x signs (4)
        const int zpos = j / 4, sg = j % 4;
        int k = 0;
        for (int c = 0; c < 3; ++c) {
            if (c == zpos) continue;
            v[c] = ((sg >> k) & 1) ? -4 : 4;
            ++k;
        }
    }
    return v[a];
}

__host__ __device__ constexpr SStruct make_struct(int sl) {
    SStruct t{};
    int k = 0;
    for (int q = 0; q < 4; ++q)
        if (q != sl % 4) t.gnu[k++] = q;
    int grp[48] = {};
    int cnt[kGroups] = {};
    for (int i = 0; i < 48; ++i) {
        grp[i] = cs_group(sl, cs_candidate(i, 0), cs_candidate(i, 1), cs_candidate(i, 2));
        if (grp[i] >= 0) ++cnt[grp[i]];
    }
    int n = 0;
    for (int g = 0; g < kGroups; ++g) {
        t.gbegin[g] = n;
        n += cnt[g];
    }
    t.gbegin[kGroups] = n;
    int fill[kGroups] = {};
    for (int i = 0; i < 48; ++i) {
        const int g = grp[i];
        if (g < 0) continue;
        const int e = t.gbegin[g] + fill[g]++;
        const int x = cs_r(sl, 0) + cs_candidate(i, 0), y = cs_r(sl, 1) + cs_candidate(i, 1),
                  z = cs_r(sl, 2) + cs_candidate(i, 2);
        const int s2 = cs_sl_at(x, y, z);
        t.nb[e].sl = s2;
        t.nb[e].dx = cs_cell_off(x, cs_r(s2, 0));
        t.nb[e].dy = cs_cell_off(y, cs_r(s2, 1));
        t.nb[e].dz = cs_cell_off(z, cs_r(s2, 2));
    }
    return t;
}

struct SStructAll {
    SStruct t[16];
};
__host__ __device__ constexpr SStructAll make_all_struct() {
    SStructAll a{};
    for (int sl = 0; sl < 16; ++sl) a.t[sl] = make_struct(sl);
    return a;
}
// Evaluated once at compile time; device code reads it only through the
// constexpr accessors below (constant expressions), so no copy lives in memory.
constexpr SStructAll kStruct = make_all_struct();
__host__ __device__ constexpr int nb_sl(int sl, int e) { return kStruct.t[sl].nb[e].sl; }
__host__ __device__ constexpr int nb_dx(int sl, int e) { return kStruct.t[sl].nb[e].dx; }
__host__ __device__ constexpr int nb_dy(int sl, int e) { return kStruct.t[sl].nb[e].dy; }
__host__ __device__ constexpr int nb_dz(int sl, int e) { return kStruct.t[sl].nb[e].dz; }
__host__ __device__ constexpr int grp_begin(int sl, int g) { return kStruct.t[sl].gbegin[g]; }
__host__ __device__ constexpr int group_of(int sl, int e) {
    int g = 0;
    while (g + 1 < kGroups && kStruct.t[sl].gbegin[g + 1] <= e) ++g;
    return g;
}
__host__ __device__ constexpr int grp_size(int sl, int g) { return kStruct.t[sl].gbegin[g + 1] - kStruct.t[sl].gbegin[g]; }

// Neighbour rows: the distinct (sublattice, dy, dz) of the 30 neighbours of a
// sublattice, in first-use order. A row of cells (fixed cy, cz) of sublattice
// sl finds all its neighbours in these rows of the other sublattices, shifted
// by dx in {-1, 0, +1} along x. 24 rows for every sublattice of the pyrochlore
// structure; kMaxRows bounds the table.
constexpr int kMaxRows = 32;
struct SRows {
    int n;
    int s2[kMaxRows], dy[kMaxRows], dz[kMaxRows];
    int row_of[kStructNb];
};
__host__ __device__ constexpr SRows make_rows(int sl) {
    SRows r{};
    r.n = 0;
    for (int e = 0; e < kStructNb; ++e) {
        const SNb& b = kStruct.t[sl].nb[e];
        int u = 0;
        while (u < r.n && !(r.s2[u] == b.sl && r.dy[u] == b.dy && r.dz[u] == b.dz)) ++u;
        if (u == r.n) {
            r.s2[u] = b.sl;
            r.dy[u] = b.dy;
            r.dz[u] = b.dz;
            ++r.n;
        }
        r.row_of[e] = u;
    }
    return r;
}
struct SRowsAll {
    SRows t[16];
};
__host__ __device__ constexpr SRowsAll make_all_rows() {
    SRowsAll a{};
    for (int sl = 0; sl < 16; ++sl) a.t[sl] = make_rows(sl);
    return a;
}
constexpr SRowsAll kRows = make_all_rows();
__host__ __device__ constexpr int rows_n(int sl) { return kRows.t[sl].n; }
__host__ __device__ constexpr int row_s2(int sl, int u) { return kRows.t[sl].s2[u]; }
__host__ __device__ constexpr int row_dy(int sl, int u) { return kRows.t[sl].dy[u]; }
__host__ __device__ constexpr int row_dz(int sl, int u) { return kRows.t[sl].dz[u]; }
__host__ __device__ constexpr int row_of(int sl, int e) { return kRows.t[sl].row_of[e]; }
__host__ __device__ constexpr int max_rows() {
    int m = 0;
    for (int sl = 0; sl < 16; ++sl) m = kRows.t[sl].n > m ? kRows.t[sl].n : m;
    return m;
}
static_assert(max_rows() <= kMaxRows, "neighbour row table too small");

// Group matrices per sublattice (row-major 3x3) and the groups with a nonzero
// matrix; passed to the kernels by value (constant bank).
struct PyroMats {
    float M[16][kGroups][9];
    uint32_t active[16];  // bit g set: group g has a nonzero matrix
};

// Exact n / d for 0 <= n < 2^30, 1 <= d <= 1024 by multiplication:
// q = (n * m) >> 40 with m = floor(2^40/d) + 1 (the excess n*(m - 2^40/d)/2^40
// stays below 1/d). The 70-bit product is formed as the high word of
// (n << 24) * m.
__host__ __device__ inline uint64_t fastdiv_magic(int d) { return (uint64_t(1) << 40) / uint64_t(d) + 1; }
__device__ __forceinline__ int fdiv(int n, uint64_t m) { return int(__umul64hi(uint64_t(uint32_t(n)) << 24, m)); }

}  // namespace pc
