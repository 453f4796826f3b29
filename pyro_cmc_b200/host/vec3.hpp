// vec3.hpp -- the small vector/matrix types the reference's interfaces use
// (lattice_lib's vector3::vec3 / mat33, used by include/MC.hpp and
// include/cli_bits.hpp), restated for the host shims.
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <ostream>

namespace vector3 {

template <typename T>
struct vec3 {
    std::array<T, 3> v{};
    constexpr vec3() = default;
    constexpr vec3(T x, T y, T z) : v{x, y, z} {}
    template <typename U>
    constexpr explicit vec3(const vec3<U>& o) : v{T(o[0]), T(o[1]), T(o[2])} {}
    constexpr T& operator[](int i) { return v[size_t(i)]; }
    constexpr const T& operator[](int i) const { return v[size_t(i)]; }
    vec3& operator+=(const vec3& o) {
        for (int i = 0; i < 3; ++i) v[size_t(i)] += o[i];
        return *this;
    }
    vec3& operator-=(const vec3& o) {
        for (int i = 0; i < 3; ++i) v[size_t(i)] -= o[i];
        return *this;
    }
    vec3& operator/=(T s) {
        for (int i = 0; i < 3; ++i) v[size_t(i)] /= s;
        return *this;
    }
    friend vec3 operator+(vec3 a, const vec3& b) { return a += b; }
    friend vec3 operator-(vec3 a, const vec3& b) { return a -= b; }
    friend vec3 operator-(const vec3& a) { return vec3(-a[0], -a[1], -a[2]); }
    friend vec3 operator*(T s, const vec3& a) { return vec3(s * a[0], s * a[1], s * a[2]); }
    friend bool operator==(const vec3& a, const vec3& b) { return a.v == b.v; }
    friend std::ostream& operator<<(std::ostream& os, const vec3& a) {
        return os << "[" << a[0] << ", " << a[1] << ", " << a[2] << "]";
    }
};

template <typename T>
T dot(const vec3<T>& a, const vec3<T>& b) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

using vec3d = vec3<double>;

// 3x3 matrix, m(i, j) = row i, column j.
template <typename T>
struct mat33 {
    std::array<T, 9> m{};
    static mat33 from_cols(const std::array<T, 3>& c0, const std::array<T, 3>& c1, const std::array<T, 3>& c2) {
        mat33 r;
        for (int i = 0; i < 3; ++i) {
            r(i, 0) = c0[size_t(i)];
            r(i, 1) = c1[size_t(i)];
            r(i, 2) = c2[size_t(i)];
        }
        return r;
    }
    T& operator()(int i, int j) { return m[size_t(3 * i + j)]; }
    const T& operator()(int i, int j) const { return m[size_t(3 * i + j)]; }
    mat33 tr() const {
        mat33 r;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) r(i, j) = (*this)(j, i);
        return r;
    }
    friend mat33 operator+(mat33 a, const mat33& b) {
        for (int i = 0; i < 9; ++i) a.m[size_t(i)] += b.m[size_t(i)];
        return a;
    }
    friend mat33 operator*(T s, mat33 a) {
        for (auto& x : a.m) x *= s;
        return a;
    }
    friend vec3<T> operator*(const mat33& a, const vec3<T>& x) {
        vec3<T> r;
        for (int i = 0; i < 3; ++i) r[i] = a(i, 0) * x[0] + a(i, 1) * x[1] + a(i, 2) * x[2];
        return r;
    }
};

}  // namespace vector3

using ipos_t = vector3::vec3<int64_t>;
using ivec3_t = vector3::vec3<int64_t>;
using imat33_t = vector3::mat33<int64_t>;
