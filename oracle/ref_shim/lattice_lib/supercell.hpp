// supercell.hpp -- TEST INFRASTRUCTURE ONLY: a minimal stand-in for the parts
// of lattice_lib (Spuriosity1/latticelab >= 2.3.0, absent from this image)
// that the reference's src/MC.cpp and include/pyrochlore_geometry.hpp use, so
// that those files compile unchanged into oracle/_ref/ (see make_ref.sh).
//
// What it provides, and the conventions it fixes (lattice_lib's own are not
// available; these are the ones the rest of this repository documents):
//  * vector3::vec3<T> / vector3::mat33<T>: small value types with the
//    arithmetic MC.cpp uses. A matrix-vector product sums the three products
//    of a row left to right; nothing else is reassociated.
//  * ipos_t (vec3<int64_t>), imat33_t, ivec3_t.
//  * UnitCellSpecifier<T>: a cubic cell (lattice vectors as columns) plus its
//    objects in the order they are added.
//  * Supercell<T> built by build_supercell(cell, L*I): objects stored
//    sublattice-major, objects[sl * Nc + cell] with cell = cx + L*(cy + L*cz)
//    and ipos = cell_object.ipos + a*(cx, cy, cz) (a = cell side, 8);
//    get_object_at wraps positions periodically (mod a*L): the residues mod a
//    identify the sublattice, the exact quotient the cell.
// Only diagonal supercells (L*I) are supported.
//
// Which `abs` the unqualified call in MC.cpp's local_lifted_Metropolis
// (|1 - u*u| < 1e-16) resolves to depends on the headers included before it:
// with only <cmath>/<cstdlib> it is C's int abs(int), the argument truncates
// to 0 and the lifted u-form move rejects every proposal. The reference's own
// lifted acceptance test (test/bench_lifted.cpp:240-272) needs a working
// move, so its real include chain brings the floating-point overloads into
// the global namespace; <stdlib.h> (libstdc++'s wrapper, which declares
// `using std::abs;`) does that here.
#pragma once

#include <stdlib.h>
#include <math.h>

#include <array>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <tuple>
#include <utility>
#include <vector>

namespace vector3 {

template <typename T>
struct vec3 {
    T v[3] = {T(0), T(0), T(0)};
    constexpr vec3() = default;
    constexpr vec3(T a, T b, T c) : v{a, b, c} {}
    constexpr T& operator[](size_t i) { return v[i]; }
    constexpr const T& operator[](size_t i) const { return v[i]; }
    vec3& operator+=(const vec3& o) {
        for (int i = 0; i < 3; ++i) v[i] += o.v[i];
        return *this;
    }
    vec3& operator-=(const vec3& o) {
        for (int i = 0; i < 3; ++i) v[i] -= o.v[i];
        return *this;
    }
    vec3& operator*=(T s) {
        for (int i = 0; i < 3; ++i) v[i] *= s;
        return *this;
    }
    vec3& operator/=(T s) {
        for (int i = 0; i < 3; ++i) v[i] /= s;
        return *this;
    }
};

template <typename T>
vec3<T> operator+(const vec3<T>& a, const vec3<T>& b) {
    return {a[0] + b[0], a[1] + b[1], a[2] + b[2]};
}
template <typename T>
vec3<T> operator-(const vec3<T>& a, const vec3<T>& b) {
    return {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
}
template <typename T>
vec3<T> operator-(const vec3<T>& a) {
    return {-a[0], -a[1], -a[2]};
}
template <typename T>
vec3<T> operator*(T s, const vec3<T>& a) {
    return {s * a[0], s * a[1], s * a[2]};
}
template <typename T>
vec3<T> operator*(const vec3<T>& a, T s) {
    return {a[0] * s, a[1] * s, a[2] * s};
}
template <typename T>
vec3<T> operator/(const vec3<T>& a, T s) {
    return {a[0] / s, a[1] / s, a[2] / s};
}
template <typename T>
T dot(const vec3<T>& a, const vec3<T>& b) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
template <typename T>
bool operator==(const vec3<T>& a, const vec3<T>& b) {
    return a[0] == b[0] && a[1] == b[1] && a[2] == b[2];
}

using vec3d = vec3<double>;

// 3x3 matrix, row-major storage; m(r, c).
template <typename T>
struct mat33 {
    T m[9] = {T(0), T(0), T(0), T(0), T(0), T(0), T(0), T(0), T(0)};
    static mat33 from_cols(const std::array<T, 3>& c0, const std::array<T, 3>& c1, const std::array<T, 3>& c2) {
        mat33 r;
        for (int i = 0; i < 3; ++i) {
            r.m[3 * i + 0] = c0[size_t(i)];
            r.m[3 * i + 1] = c1[size_t(i)];
            r.m[3 * i + 2] = c2[size_t(i)];
        }
        return r;
    }
    T operator()(int r, int c) const { return m[3 * r + c]; }
    mat33 tr() const {
        mat33 r;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) r.m[3 * i + j] = m[3 * j + i];
        return r;
    }
};

template <typename T>
vec3<T> operator*(const mat33<T>& a, const vec3<T>& x) {
    return {a.m[0] * x[0] + a.m[1] * x[1] + a.m[2] * x[2], a.m[3] * x[0] + a.m[4] * x[1] + a.m[5] * x[2],
            a.m[6] * x[0] + a.m[7] * x[1] + a.m[8] * x[2]};
}
template <typename T>
mat33<T> operator*(T s, const mat33<T>& a) {
    mat33<T> r;
    for (int i = 0; i < 9; ++i) r.m[i] = s * a.m[i];
    return r;
}
template <typename T>
mat33<T> operator+(const mat33<T>& a, const mat33<T>& b) {
    mat33<T> r;
    for (int i = 0; i < 9; ++i) r.m[i] = a.m[i] + b.m[i];
    return r;
}

}  // namespace vector3

using ipos_t = vector3::vec3<int64_t>;
using ivec3_t = vector3::vec3<int>;
using imat33_t = vector3::mat33<int64_t>;

template <typename T>
using SlPos = std::vector<ipos_t>;

template <typename T>
struct UnitCellSpecifier {
    imat33_t cell;
    std::vector<T> objects;
    explicit UnitCellSpecifier(const imat33_t& c) : cell(c) {}
    void add(T&& o) { objects.push_back(std::move(o)); }
};

struct SupercellLattice {
    int64_t L = 1;
    int64_t a = 8;
    int64_t num_primitive_cells() const { return L * L * L; }
    imat33_t get_lattice_vectors() const {
        return imat33_t::from_cols({a * L, 0, 0}, {0, a * L, 0}, {0, 0, a * L});
    }
    vector3::mat33<double> get_reciprocal_lattice_vectors() const {
        const double k = 2 * M_PI / double(a * L);
        return vector3::mat33<double>::from_cols({k, 0, 0}, {0, k, 0}, {0, 0, k});
    }
};

template <typename T>
struct Supercell {
    SupercellLattice lattice;
    std::tuple<std::vector<T>> objects;
    std::tuple<SlPos<T>> sl_positions;
    std::vector<int> sl_of_mod;  // [a^3]: sublattice of a position by its residues mod a, -1 if none

    template <typename U>
    std::vector<U>& get_objects() {
        return std::get<std::vector<U>>(objects);
    }
    template <typename U>
    const std::vector<U>& get_objects() const {
        return std::get<std::vector<U>>(objects);
    }
    size_t size() const { return std::get<0>(objects).size(); }

    static int64_t pmod(int64_t v, int64_t m) { return ((v % m) + m) % m; }
    int64_t index_of(const ipos_t& x) const {
        const int64_t a = lattice.a, L = lattice.L;
        const int sl = sl_of_mod[size_t((pmod(x[0], a) * a + pmod(x[1], a)) * a + pmod(x[2], a))];
        if (sl < 0) throw std::out_of_range("get_object_at: no object at this position");
        const ipos_t& r = std::get<0>(sl_positions)[size_t(sl)];
        int64_t c[3];
        for (int i = 0; i < 3; ++i) c[i] = pmod((x[size_t(i)] - r[size_t(i)]) / a, L);  // exact division
        return int64_t(sl) * L * L * L + c[0] + L * (c[1] + L * c[2]);
    }
    template <typename U>
    U* get_object_at(const ipos_t& x) {
        return &std::get<std::vector<U>>(objects)[size_t(index_of(x))];
    }
};

template <typename T>
Supercell<T> build_supercell(const UnitCellSpecifier<T>& cell, const imat33_t& spec) {
    const int64_t L = spec(0, 0);
    if (spec(1, 1) != L || spec(2, 2) != L || spec(0, 1) || spec(0, 2) || spec(1, 0) || spec(1, 2) || spec(2, 0) ||
        spec(2, 1) || cell.cell(0, 0) != cell.cell(1, 1) || cell.cell(0, 0) != cell.cell(2, 2))
        throw std::invalid_argument("build_supercell stand-in: only cubic cells and L*I supercells");
    Supercell<T> sc;
    sc.lattice.L = L;
    sc.lattice.a = cell.cell(0, 0);
    auto& objs = std::get<0>(sc.objects);
    auto& slp = std::get<0>(sc.sl_positions);
    const int64_t a = sc.lattice.a, Nc = L * L * L;
    sc.sl_of_mod.assign(size_t(a * a * a), -1);
    objs.reserve(size_t(Nc) * cell.objects.size());
    for (const T& proto : cell.objects) {
        const ipos_t& r = proto.ipos;
        sc.sl_of_mod[size_t((Supercell<T>::pmod(r[0], a) * a + Supercell<T>::pmod(r[1], a)) * a +
                            Supercell<T>::pmod(r[2], a))] = int(slp.size());
        slp.push_back(r);
        for (int64_t c = 0; c < Nc; ++c) {
            const int64_t cx = c % L, cy = (c / L) % L, cz = c / (L * L);
            T o = proto;
            o.ipos = r + ipos_t{a * cx, a * cy, a * cz};
            objs.push_back(std::move(o));
        }
    }
    return sc;
}
