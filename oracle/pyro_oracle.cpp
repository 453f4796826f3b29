// pyro_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// An FP64 CPU restatement of the reference pyro_cmc Monte Carlo path, used by
// tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm as
// the checker and the CPU baseline. Nothing in the product links, loads or calls
// this file.
//
// Parity status: pinned on the reference's own code. oracle/make_ref.sh
// compiles the reference's src/MC.cpp unchanged (against the lattice_lib /
// HDF5 stand-ins in oracle/ref_shim/) into oracle/_ref/libref_mc.so, and
// tests/test_oracle_ref.py checks this restatement against it: positions and
// bond shells exactly, energy and local field to FP64 rounding, and whole
// sequential Metropolis + overrelaxation and lifted chains from the same
// Xoroshiro seed with identical accepted counts (committed as
// tests/golden/ref_mc_chains.npz). Further pins:
// (1) the reference's own geometry tables, parsed from
//     include/pyrochlore_geometry.hpp into tests/golden/geometry_tables.json,
// (2) Xoroshiro128++/SplitMix64 streams and libstdc++ distribution draws
//     produced by compiling the reference's include/XoshiroCpp.hpp
//     (oracle/make_ref.sh -> oracle/_ref/), committed as
//     tests/golden/xoshiro_streams.json,
// (3) analytic known answers derived from the reference code (ferromagnet
//     energy, zero-tetrahedron-sum states, energy-preserving overrelaxation).
// What the reference delegates to lattice_lib (DFT sign, flat-k order, the
// in-sublattice cell order) is NOT pinned by any reference artefact: those
// conventions are assumptions, stated where they are used below.
//
// Layout follows the reference data model (include/MC.hpp:38-63): an AoS
// vector of spins stored sublattice-major, spins[sl*Nc + cell]
// (src/MC.cpp:32), each with pointer bond shells.
//
// Build: oracle/Makefile (g++ -O3 -shared -fPIC).

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <random>
#include <set>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>
#include <chrono>

namespace orc {

using vec3 = std::array<double, 3>;
using mat33 = std::array<double, 9>;  // row-major, m[3*a+b]
using ipos = std::array<int64_t, 3>;

static inline vec3 add(const vec3& a, const vec3& b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
static inline vec3 sub(const vec3& a, const vec3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
static inline vec3 scale(double s, const vec3& a) { return {s * a[0], s * a[1], s * a[2]}; }
// v /= s of the reference's vec3 (a division per component, not a multiply by 1/s)
static inline vec3 vdiv(const vec3& a, double s) { return {a[0] / s, a[1] / s, a[2] / s}; }
static inline double dot(const vec3& a, const vec3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline vec3 cross(const vec3& a, const vec3& b) {
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
static inline vec3 matvec(const mat33& m, const vec3& v) {
    return {m[0] * v[0] + m[1] * v[1] + m[2] * v[2], m[3] * v[0] + m[4] * v[1] + m[5] * v[2],
            m[6] * v[0] + m[7] * v[1] + m[8] * v[2]};
}
static inline mat33 transpose(const mat33& m) { return {m[0], m[3], m[6], m[1], m[4], m[7], m[2], m[5], m[8]}; }

// ---------------------------------------------------------------------------
// RNG: Xoroshiro128++ seeded through SplitMix64, restated from the published
// algorithm (Blackman & Vigna); the reference uses the third-party header
// include/XoshiroCpp.hpp:351-362 (class) and :681-700 (SplitMix64 seeding).
// Pinned against that header by tests/golden/xoshiro_streams.json.
// ---------------------------------------------------------------------------
struct SplitMix64 {
    uint64_t s;
    explicit SplitMix64(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        return z ^ (z >> 31);
    }
};

struct Xoroshiro128pp {
    using result_type = uint64_t;
    uint64_t s0, s1;
    explicit Xoroshiro128pp(uint64_t seed = 1234567) {
        SplitMix64 sm(seed);
        s0 = sm.next();
        s1 = sm.next();
    }
    static constexpr uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    static constexpr result_type min() { return 0; }
    static constexpr result_type max() { return ~uint64_t(0); }
    result_type operator()() {
        const uint64_t a = s0;
        uint64_t b = s1;
        const uint64_t r = rotl(a + b, 17) + a;
        b ^= a;
        s0 = rotl(a, 49) ^ b ^ (b << 21);
        s1 = rotl(b, 28);
        return r;
    }
};

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), restated from the paper.
// This is the counter-based stream of the GPU path; the oracle uses it only in
// its "GPU-schedule mirror" sweep so one GPU sweep can be checked site by site.
// ---------------------------------------------------------------------------
static inline void philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint64_t p0 = uint64_t(0xD2511F53u) * c0;
        const uint64_t p1 = uint64_t(0xCD9E8D57u) * c2;
        const uint32_t hi0 = uint32_t(p0 >> 32), lo0 = uint32_t(p0);
        const uint32_t hi1 = uint32_t(p1 >> 32), lo1 = uint32_t(p1);
        const uint32_t n0 = hi1 ^ c1 ^ k0;
        const uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

// Draw layout shared with the GPU sweep kernels (documented in the C ABI header):
//   key  = (seed lo32, seed hi32)
//   ctr  = (site index within replica, sweep lo32, draw | (sweep hi32 << 8), replica)
//   draw 0: Metropolis -- words 0..3 give two Box-Muller pairs (top 24 bits each:
//           radius sqrt(-2 ln u) from words 0, 2, angle 2 pi (u - 1/2) from words 1, 3),
//           the acceptance uniform is the low bytes of words 0,1,2 (24 bits);
//   draw 2+k: overrelaxation pass k -- word 0's top 24 bits give the angle 2 pi (u - 1/2).
static inline void philox_site(uint64_t seed, uint32_t replica, uint64_t sweep, uint32_t draw, uint32_t site,
                               uint32_t out[4]) {
    const uint32_t key[2] = {uint32_t(seed), uint32_t(seed >> 32)};
    const uint32_t ctr[4] = {site, uint32_t(sweep), draw | (uint32_t(sweep >> 32) << 8), replica};
    philox4x32_10(ctr, key, out);
}
static inline double u24_open0(uint32_t x) { return (double((x >> 8)) + 1.0) * (1.0 / 16777216.0); }  // (0,1]
static inline double u24(uint32_t x) { return double(x >> 8) * (1.0 / 16777216.0); }                  // [0,1)
static inline double u24_lowbytes(const uint32_t w[4]) {
    const uint32_t v = (w[0] & 0xffu) | ((w[1] & 0xffu) << 8) | ((w[2] & 0xffu) << 16);
    return double(v) * (1.0 / 16777216.0);
}

// ---------------------------------------------------------------------------
// Geometry: the pyrochlore cubic cell of side 8 with 16 sites
// (include/pyrochlore_geometry.hpp:12-32): site sl = 4*f + p at
// link[p] + R_fcc[f], pyro_sl = p.
// ---------------------------------------------------------------------------
static const int64_t LINK[4][3] = {{1, 1, 1}, {1, -1, -1}, {-1, 1, -1}, {-1, -1, 1}};
static const int64_t RFCC[4][3] = {{0, 0, 0}, {0, 4, 4}, {4, 0, 4}, {4, 4, 0}};

static inline int64_t pmod(int64_t a, int64_t m) {
    int64_t r = a % m;
    return r < 0 ? r + m : r;
}

// Neighbour displacement tables, derived from geometry rather than transcribed:
// for a site of pyrochlore sublattice p, the displacements d with |d|^2 = 8 (J1),
// 24 (J2) or 32 (J3) that land on a lattice site; J3 is split into J3a (the
// midpoint is a site: "3rd neighbours WITH spin in the middle",
// pyrochlore_geometry.hpp:136-142) and J3b (:144-149). The sets are checked
// against the reference's own tables (tests/golden/geometry_tables.json).
static bool is_site(const ipos& x, int* sl_out = nullptr) {
    for (int f = 0; f < 4; ++f)
        for (int p = 0; p < 4; ++p) {
            bool ok = true;
            for (int a = 0; a < 3; ++a)
                if (pmod(x[a] - LINK[p][a] - RFCC[f][a], 8) != 0) ok = false;
            if (ok) {
                if (sl_out) *sl_out = 4 * f + p;
                return true;
            }
        }
    return false;
}

// kind: 1 = J1, 2 = J2, 3 = J3a, 4 = J3b
static std::vector<ipos> displacements(int p, int kind) {
    const int64_t r2 = kind == 1 ? 8 : kind == 2 ? 24 : 32;
    std::vector<ipos> out;
    const ipos x0 = {LINK[p][0], LINK[p][1], LINK[p][2]};
    for (int64_t dx = -4; dx <= 4; ++dx)
        for (int64_t dy = -4; dy <= 4; ++dy)
            for (int64_t dz = -4; dz <= 4; ++dz) {
                if (dx * dx + dy * dy + dz * dz != r2) continue;
                ipos x = {x0[0] + dx, x0[1] + dy, x0[2] + dz};
                if (!is_site(x)) continue;
                if (kind >= 3) {
                    ipos mid = {x0[0] + dx / 2, x0[1] + dy / 2, x0[2] + dz / 2};
                    const bool mid_site = is_site(mid);
                    if ((kind == 3) != mid_site) continue;
                }
                out.push_back({dx, dy, dz});
            }
    return out;
}

// J1 displacements from pyro_sl mu that land on pyro_sl nu
// (the nn1_pair_MN tables, pyrochlore_geometry.hpp:151-190).
static std::vector<ipos> pair_displacements(int mu, int nu) {
    std::vector<ipos> out;
    for (const auto& d : displacements(mu, 1)) {
        ipos x = {LINK[mu][0] + d[0], LINK[mu][1] + d[1], LINK[mu][2] + d[2]};
        int sl = -1;
        is_site(x, &sl);
        if (sl % 4 == nu) out.push_back(d);
    }
    return out;
}

struct Spin;
struct Shell {
    const mat33* J;
    std::vector<Spin*> bonds;
};
struct Spin {
    ipos pos;  // unwrapped: 8*cell + r_sl
    int pyro_sl = 0;
    int sl = 0;
    vec3 S{0, 0, 0};
    std::vector<Shell> shells;
    int8_t lifted_dir = 1;
};
struct Coupling {
    std::string name;
    std::vector<std::vector<ipos>> rel;  // rel[pyro_sl]
    mat33 J, Jt;
};

// Supercell L*I of the cubic cell. Cell order is the build's documented choice
// (cell = cx + L*(cy + L*cz)); lattice_lib's own order is not available.
struct Lattice {
    int L = 1;
    int Nc = 1;
    std::vector<Spin> spins;  // spins[sl*Nc + cell]  (src/MC.cpp:32)
    std::vector<ipos> r_sl;   // unwrapped sublattice positions
    int sl_of_mod8[512];

    explicit Lattice(int L_) : L(L_), Nc(L_ * L_ * L_) {
        for (int i = 0; i < 512; ++i) sl_of_mod8[i] = -1;
        for (int f = 0; f < 4; ++f)
            for (int p = 0; p < 4; ++p) {
                ipos r = {LINK[p][0] + RFCC[f][0], LINK[p][1] + RFCC[f][1], LINK[p][2] + RFCC[f][2]};
                r_sl.push_back(r);
                const int key = int(pmod(r[0], 8) * 64 + pmod(r[1], 8) * 8 + pmod(r[2], 8));
                sl_of_mod8[key] = 4 * f + p;
            }
        spins.resize(size_t(16) * Nc);
        for (int sl = 0; sl < 16; ++sl)
            for (int cz = 0; cz < L; ++cz)
                for (int cy = 0; cy < L; ++cy)
                    for (int cx = 0; cx < L; ++cx) {
                        const int cell = cx + L * (cy + L * cz);
                        Spin& s = spins[size_t(sl) * Nc + cell];
                        s.sl = sl;
                        s.pyro_sl = sl % 4;
                        s.pos = {8 * cx + r_sl[sl][0], 8 * cy + r_sl[sl][1], 8 * cz + r_sl[sl][2]};
                    }
    }
    size_t index_at(const ipos& x) const {
        const int key = int(pmod(x[0], 8) * 64 + pmod(x[1], 8) * 8 + pmod(x[2], 8));
        const int sl = sl_of_mod8[key];
        if (sl < 0) throw std::runtime_error("get_object_at: no site at this position");
        int64_t c[3];
        // (x - r) is a multiple of 8, so the division is exact
        for (int a = 0; a < 3; ++a) c[a] = pmod((x[a] - r_sl[sl][a]) / 8, L);
        return size_t(sl) * Nc + size_t(c[0] + L * (c[1] + L * c[2]));
    }
    Spin* get_object_at(const ipos& x) { return &spins[index_at(x)]; }
};

// ---------------------------------------------------------------------------
// MC runner: restates src/MC.cpp.
// ---------------------------------------------------------------------------
struct Runner {
    Lattice* lat;
    std::vector<Coupling> specs;
    std::map<std::string, size_t> index;
    vec3 B{0, 0, 0};
    double T_ref = 1.0;
    Xoroshiro128pp rng;
    std::normal_distribution<double> normal_dist;
    std::uniform_real_distribution<double> rand01{0.0, 1.0};
    std::exponential_distribution<double> exp_dist;  // rate 1 (include/MC.hpp:97)

    Runner(Lattice& l, uint64_t seed) : lat(&l), rng(seed) {}

    // src/MC.cpp:56-66
    void define_coupling(const std::string& name, const std::vector<std::vector<ipos>>& rel, const mat33& J) {
        if (index.count(name)) throw std::logic_error("Coupling names must be unique");
        index[name] = specs.size();
        specs.push_back({name, rel, J, transpose(J)});
    }

    // src/MC.cpp:15-52: per coupling, split each spin's neighbours into a
    // source shell (own pyro_sl <= other's -> J) and a target shell (-> Jt).
    void setup_lattice() {
        auto& spins = lat->spins;
        const int Np = lat->Nc;
        for (const auto& c : specs) {
            for (int sl = 0; sl < 16; ++sl) {
                const int pyro_sl = sl % 4;
                for (int cell = 0; cell < Np; ++cell) {
                    Spin* origin = &spins[size_t(sl) * Np + cell];
                    std::vector<Spin*> src, tgt;
                    for (const auto& v : c.rel.at(pyro_sl)) {
                        ipos x = {origin->pos[0] + v[0], origin->pos[1] + v[1], origin->pos[2] + v[2]};
                        Spin* other = lat->get_object_at(x);
                        if (origin->pyro_sl <= other->pyro_sl)
                            src.push_back(other);
                        else
                            tgt.push_back(other);
                    }
                    if (!src.empty()) origin->shells.push_back({&c.J, std::move(src)});
                    if (!tgt.empty()) origin->shells.push_back({&c.Jt, std::move(tgt)});
                }
            }
        }
    }

    // src/MC.cpp:87-96
    vec3 local_field(const Spin* s) const {
        vec3 h{0, 0, 0};
        for (const auto& shell : s->shells) {
            vec3 t{0, 0, 0};
            for (const Spin* o : shell.bonds) t = add(t, o->S);
            h = add(h, matvec(*shell.J, t));
        }
        return h;
    }

    // src/MC.cpp:102-109 (Rodrigues rotation about an unnormalised axis)
    static void rotate_about_vector(vec3& v, const vec3& axis, double theta) {
        const double c = std::cos(theta), s = std::sin(theta);
        const double n2 = dot(axis, axis);
        const vec3 ax = cross(axis, v);
        const double av = dot(axis, v);
        v = add(add(scale(c, v), scale(((1 - c) / n2) * av, axis)), scale(s / std::sqrt(n2), ax));
    }
    // src/MC.cpp:98-100
    static void mirror_about_vector(vec3& v, const vec3& axis) {
        const double f = 2 * (dot(axis, v) / (dot(axis, axis) + 1e-10));
        v = add(scale(-1.0, v), scale(f, axis));
    }

    // src/MC.cpp:111-130
    size_t local_Metropolis(double T, Spin* spin) {
        const vec3 h = sub(local_field(spin), B);
        const double curr_E = dot(spin->S, h);
        // vector3::vec3d(normal_dist(rng), normal_dist(rng), normal_dist(rng)):
        // the order in which a constructor's arguments are evaluated is
        // unspecified in C++; GCC on x86-64 evaluates them right to left, so the
        // reference as built draws the z component first. Pinned against the
        // reference's own MC.cpp compiled here (oracle/_ref/libref_mc.so).
        const double g2 = normal_dist(rng), g1 = normal_dist(rng), g0 = normal_dist(rng);
        vec3 nS = scale(std::sqrt(T / T_ref), vec3{g0, g1, g2});
        nS = add(nS, spin->S);
        const double n = std::sqrt(dot(nS, nS));
        nS = vdiv(nS, n);
        const double dE = dot(nS, h) - curr_E;
        if (dE < 0 || rand01(rng) < std::exp(-dE / T)) {
            spin->S = nS;
            return 1;
        }
        return 0;
    }

    // src/MC.cpp:145-153
    void overrelax_all() {
        for (auto& s : lat->spins) {
            const vec3 h = sub(local_field(&s), B);
            rotate_about_vector(s.S, h, 2 * M_PI * rand01(rng));
        }
    }

    // src/MC.cpp:155-163
    size_t sweep_local_Metropolis(double T, size_t n_overrelax) {
        size_t acc = 0;
        for (auto& s : lat->spins) acc += local_Metropolis(T, &s);
        for (size_t i = 0; i < n_overrelax; ++i) overrelax_all();
        return acc;
    }

    // --- lifted moves (the move formulas; the draws are passed in) -----
    // src/MC.cpp:249-281, u-form: slide u = S.h_hat by du = dir*sqrt(T/T_ref)*E,
    // E ~ Exp(1), keep the azimuth; out of [-1, 1] or at a pole: flip dir.
    bool lifted_u_move(double T, Spin* spin, const vec3& h, double e1, double u01) const {
        const double curr_E = dot(spin->S, h);
        const vec3 hh = vdiv(h, std::sqrt(dot(h, h)));
        const double u = dot(hh, spin->S);
        const double du = spin->lifted_dir * std::sqrt(T / T_ref) * e1;
        const double nu = u + du;
        if (nu > 1 || nu < -1 || std::abs(1 - u * u) < 1e-16) {
            spin->lifted_dir = int8_t(-spin->lifted_dir);
            return false;
        }
        vec3 nS = add(scale(nu, hh), scale(std::sqrt((1 - nu * nu) / (1 - u * u)), sub(spin->S, scale(u, hh))));
        nS = vdiv(nS, std::sqrt(dot(nS, nS)));
        const double dE = dot(nS, h) - curr_E;
        if (u01 < std::exp(-dE / T)) {
            spin->S = nS;
            return true;
        }
        spin->lifted_dir = int8_t(-spin->lifted_dir);
        return false;
    }
    // src/MC.cpp:194-244, rotation form: rotate by dir*sqrt(T/T_ref) about
    // S x h; poles and pole crossings bounce; acceptance carries the Jacobian
    // |S' x h| / |S x h|.
    bool lifted_rot_move(double T, Spin* spin, const vec3& h, double u01) const {
        const double curr_E = dot(spin->S, h);
        const double delta = std::sqrt(T / T_ref);
        const vec3 axis = cross(spin->S, h);
        const double n2_old = dot(axis, axis);
        if (n2_old <= 1e-20) {
            spin->lifted_dir = int8_t(-spin->lifted_dir);
            return false;
        }
        vec3 nS = spin->S;
        rotate_about_vector(nS, axis, spin->lifted_dir * delta);
        nS = vdiv(nS, std::sqrt(dot(nS, nS)));
        const vec3 axis_new = cross(nS, h);
        const double n2_new = dot(axis_new, axis_new);
        if (dot(axis, axis_new) < 0) {
            spin->lifted_dir = int8_t(-spin->lifted_dir);
            return false;
        }
        const double dE = dot(nS, h) - curr_E;
        if (u01 < std::sqrt(n2_new / n2_old) * std::exp(-dE / T)) {
            spin->S = nS;
            return true;
        }
        spin->lifted_dir = int8_t(-spin->lifted_dir);
        return false;
    }
    // src/MC.cpp:249-281 with the reference's draws (exp_dist, then rand01
    // only when the proposal stays on the sphere)
    size_t local_lifted_Metropolis(double T, Spin* spin) {
        const vec3 h = sub(local_field(spin), B);
        const double e1 = exp_dist(rng);
        const vec3 hh = vdiv(h, std::sqrt(dot(h, h)));
        const double u = dot(hh, spin->S);
        const double nu = u + spin->lifted_dir * std::sqrt(T / T_ref) * e1;
        if (nu > 1 || nu < -1 || std::abs(1 - u * u) < 1e-16) {
            spin->lifted_dir = int8_t(-spin->lifted_dir);
            return 0;
        }
        return lifted_u_move(T, spin, h, e1, rand01(rng)) ? 1 : 0;
    }
    // src/MC.cpp:194-244 (rand01 drawn only when the move reaches the test)
    size_t local_lifted_Metropolis_rot(double T, Spin* spin) {
        const vec3 h = sub(local_field(spin), B);
        const vec3 axis = cross(spin->S, h);
        if (dot(axis, axis) <= 1e-20) {
            spin->lifted_dir = int8_t(-spin->lifted_dir);
            return 0;
        }
        vec3 nS = spin->S;
        rotate_about_vector(nS, axis, spin->lifted_dir * std::sqrt(T / T_ref));
        nS = vdiv(nS, std::sqrt(dot(nS, nS)));
        if (dot(axis, cross(nS, h)) < 0) {
            spin->lifted_dir = int8_t(-spin->lifted_dir);
            return 0;
        }
        return lifted_rot_move(T, spin, h, rand01(rng)) ? 1 : 0;
    }
    // src/MC.cpp:284-302
    size_t sweep_lifted_Metropolis(double T, size_t n_overrelax, bool rot) {
        size_t acc = 0;
        for (auto& s : lat->spins) acc += rot ? local_lifted_Metropolis_rot(T, &s) : local_lifted_Metropolis(T, &s);
        for (size_t i = 0; i < n_overrelax; ++i) overrelax_all();
        return acc;
    }

    // src/MC.cpp:305-312
    double total_energy_per_unit_cell() const {
        double E = 0;
        for (const auto& s : lat->spins) {
            E += 0.5 * dot(s.S, local_field(&s));
            E -= dot(s.S, B);
        }
        return E / lat->Nc;
    }

    // --- GPU-schedule mirror --------------------------------------------
    // One sweep exactly as the GPU kernels schedule it: Metropolis over the
    // colour classes in the given order (sites inside one class are not bonded,
    // so the order inside a class is immaterial), then n_or overrelaxation
    // passes over the same classes, with Philox draws per site. The update
    // formulas are those of local_Metropolis / overrelax_all above.
    // fused: the first overrelaxation move of each site follows its Metropolis
    // move inside the same colour class, with the same local field.
    // update 1 / 2: the lifted move (u-form / rotation form) in place of the
    // Metropolis move, draws from Philox draw 1 (Exp(1) = -ln of the open
    // 24-bit uniform of word 0, the acceptance uniform from word 1); lifted
    // sweeps are never fused.
    size_t sweep_philox(double T, uint64_t seed, uint32_t replica, uint64_t sweep, int n_or,
                        const std::vector<std::vector<int>>& colour_sls, int or_mode, bool fused = false,
                        int update = 0) {
        size_t acc = 0;
        const double sigma = std::sqrt(T / T_ref);
        const bool fuse = fused && n_or >= 1 && update == 0;
        for (const auto& cls : colour_sls)
            for (int sl : cls)
                for (int cell = 0; cell < lat->Nc; ++cell) {
                    const uint32_t site = uint32_t(sl * lat->Nc + cell);
                    Spin* spin = &lat->spins[site];
                    if (update != 0) {
                        uint32_t wl[4];
                        philox_site(seed, replica, sweep, 1, site, wl);
                        const vec3 h = sub(local_field(spin), B);
                        const bool a = update == 1 ? lifted_u_move(T, spin, h, -std::log(u24_open0(wl[0])), u24(wl[1]))
                                                   : lifted_rot_move(T, spin, h, u24(wl[1]));
                        acc += a ? 1 : 0;
                        continue;
                    }
                    uint32_t w[4];
                    philox_site(seed, replica, sweep, 0, site, w);
                    const double r0 = std::sqrt(-2.0 * std::log(u24_open0(w[0])));
                    const double r1 = std::sqrt(-2.0 * std::log(u24_open0(w[2])));
                    const double t0 = 2 * M_PI * (u24(w[1]) - 0.5), t1 = 2 * M_PI * (u24(w[3]) - 0.5);
                    const vec3 g = {r0 * std::cos(t0), r0 * std::sin(t0), r1 * std::cos(t1)};
                    const double u = u24_lowbytes(w);
                    const vec3 h = sub(local_field(spin), B);
                    vec3 nS = add(spin->S, scale(sigma, g));
                    nS = scale(1.0 / std::sqrt(dot(nS, nS)), nS);
                    const double dE = dot(sub(nS, spin->S), h);
                    if (dE < 0 || u < std::exp(-dE / T)) {
                        spin->S = nS;
                        ++acc;
                    }
                    if (fuse && dot(h, h) >= 1e-30) {
                        if (or_mode == 1) {
                            mirror_about_vector(spin->S, h);
                        } else {
                            uint32_t wo[4];
                            philox_site(seed, replica, sweep, 2, site, wo);
                            rotate_about_vector(spin->S, h, 2 * M_PI * (u24(wo[0]) - 0.5));
                        }
                    }
                }
        for (int k = fuse ? 1 : 0; k < n_or; ++k)
            for (const auto& cls : colour_sls)
                for (int sl : cls)
                    for (int cell = 0; cell < lat->Nc; ++cell) {
                        const uint32_t site = uint32_t(sl * lat->Nc + cell);
                        Spin* spin = &lat->spins[site];
                        const vec3 h = sub(local_field(spin), B);
                        if (dot(h, h) < 1e-30) continue;
                        if (or_mode == 1) {
                            mirror_about_vector(spin->S, h);
                        } else {
                            uint32_t w[4];
                            philox_site(seed, replica, sweep, uint32_t(2 + k), site, w);
                            rotate_about_vector(spin->S, h, 2 * M_PI * (u24(w[0]) - 0.5));
                        }
                    }
        return acc;
    }
};

// The coupling set of include/cli_bits.hpp:144-207 (build_J1J2J3_h): J1 as six
// sublattice-pair XXZ specs J1[I + (Delta-1) z_mu (x) z_nu], then J2, J3a, J3b
// (always defined, even when zero). z_p = link[p]/sqrt(3) is the local [111]
// axis (pyrochlore::axis[p][2], pyrochlore_geometry.hpp:199-208).
static void define_pyro_couplings(Runner& mc, double J1, double J2, double J3, double Delta, int j1_mode) {
    const mat33 I = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    auto scaled = [](double s, const mat33& m) {
        mat33 r;
        for (int i = 0; i < 9; ++i) r[i] = s * m[i];
        return r;
    };
    if (j1_mode == 0) {
        static const int pairs[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
        const double s3 = std::sqrt(3.0);
        for (auto& pr : pairs) {
            const int mu = pr[0], nu = pr[1];
            std::vector<std::vector<ipos>> rel(4);
            rel[mu] = pair_displacements(mu, nu);
            rel[nu] = pair_displacements(nu, mu);
            mat33 M;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b)
                    M[3 * a + b] = J1 * ((a == b ? 1.0 : 0.0) + (Delta - 1) * (LINK[mu][a] / s3) * (LINK[nu][b] / s3));
            mc.define_coupling("J1_" + std::to_string(mu) + std::to_string(nu), rel, M);
        }
    } else {
        // test/spiral_byhand.cpp:81-83: one isotropic J1 spec on the full nn1 table
        std::vector<std::vector<ipos>> rel(4);
        for (int p = 0; p < 4; ++p) rel[p] = displacements(p, 1);
        mc.define_coupling("J1", rel, scaled(J1, I));
    }
    const char* names[3] = {"J2", "J3a", "J3b"};
    const double Js[3] = {J2, J3, J3};
    for (int k = 0; k < 3; ++k) {
        std::vector<std::vector<ipos>> rel(4);
        for (int p = 0; p < 4; ++p) rel[p] = displacements(p, 2 + k);
        mc.define_coupling(names[k], rel, scaled(Js[k], I));
    }
}

// ---------------------------------------------------------------------------
// Static structure factor of one configuration.
//
// ssf_manager::sample (include/ssf_manager.hpp:260-293):
//   A^a_mu(K) = DFT over cells of S^a on sublattice mu        (lattice_lib)
//   C_{mu nu}(K) = conj(A^a_mu(K)) A^b_nu(K)                   (correlate)
//   S^{ab}(K) = sum_{mu nu} exp(+i q.(r_mu - r_nu)) C_{mu nu}  (contract)
// Assumptions for what lattice_lib holds: forward DFT sign exp(-i K.n 2pi/L),
// unnormalised, q = 2*pi*K/(8L) per component, flat k in C order
// k = (K0*L + K1)*L + K2 (scripts/plot_ssf.py:56 reshapes it that way).
// ---------------------------------------------------------------------------
using cplx = std::complex<double>;

// Direct form: B^a(K) = sum_i exp(-i q_K . x_i) S^a_i, S^{ab} = conj(B^a) B^b.
static void ssf_direct(const Lattice& lat, const std::vector<std::pair<int, int>>& corr, double* out /*[nc][nk][2]*/) {
    const int L = lat.L, nk = lat.Nc;
    std::vector<cplx> Bk(size_t(3) * nk, cplx(0, 0));
    const double q0 = 2 * M_PI / (8.0 * L);
    for (int k = 0; k < nk; ++k) {
        const int K0 = k / (L * L), K1 = (k / L) % L, K2 = k % L;
        cplx b[3] = {0, 0, 0};
        for (const auto& s : lat.spins) {
            // positions taken mod 8L so the phase argument stays small
            const double ph = -q0 * (double(K0) * double(pmod(s.pos[0], 8 * L)) + double(K1) * double(pmod(s.pos[1], 8 * L)) +
                                     double(K2) * double(pmod(s.pos[2], 8 * L)));
            const cplx e(std::cos(ph), std::sin(ph));
            for (int a = 0; a < 3; ++a) b[a] += e * s.S[a];
        }
        for (int a = 0; a < 3; ++a) Bk[size_t(a) * nk + k] = b[a];
    }
    for (size_t c = 0; c < corr.size(); ++c)
        for (int k = 0; k < nk; ++k) {
            const cplx v = std::conj(Bk[size_t(corr[c].first) * nk + k]) * Bk[size_t(corr[c].second) * nk + k];
            out[(c * nk + k) * 2] = v.real();
            out[(c * nk + k) * 2 + 1] = v.imag();
        }
}

// Sublattice form, following ssf_manager::sample step by step (per-sublattice
// DFT over cells, 16x16 correlator, phase contraction). O(Nc^2) per sublattice:
// small L only. Also returns the sublattice-resolved correlator if asked.
static void ssf_sublattice(const Lattice& lat, const std::vector<std::pair<int, int>>& corr, double* out,
                           double* resolved /* [nc][nk][16][16][2] or null */) {
    const int L = lat.L, nk = lat.Nc;
    std::vector<cplx> A(size_t(3) * 16 * nk);
    for (int a = 0; a < 3; ++a)
        for (int sl = 0; sl < 16; ++sl)
            for (int k = 0; k < nk; ++k) {
                const int K0 = k / (L * L), K1 = (k / L) % L, K2 = k % L;
                cplx acc = 0;
                for (int cell = 0; cell < nk; ++cell) {
                    const int cx = cell % L, cy = (cell / L) % L, cz = cell / (L * L);
                    const double ph = -2 * M_PI * double(K0 * cx + K1 * cy + K2 * cz) / L;
                    acc += cplx(std::cos(ph), std::sin(ph)) * lat.spins[size_t(sl) * nk + cell].S[a];
                }
                A[(size_t(a) * 16 + sl) * nk + k] = acc;
            }
    const double q0 = 2 * M_PI / (8.0 * L);
    for (size_t c = 0; c < corr.size(); ++c)
        for (int k = 0; k < nk; ++k) {
            const int K0 = k / (L * L), K1 = (k / L) % L, K2 = k % L;
            cplx Sk = 0;
            for (int mu = 0; mu < 16; ++mu)
                for (int nu = 0; nu < 16; ++nu) {
                    const cplx Cmn = std::conj(A[(size_t(corr[c].first) * 16 + mu) * nk + k]) *
                                     A[(size_t(corr[c].second) * 16 + nu) * nk + k];
                    if (resolved) {
                        const size_t o = ((((c * nk) + k) * 16 + mu) * 16 + nu) * 2;
                        resolved[o] = Cmn.real();
                        resolved[o + 1] = Cmn.imag();
                    }
                    double dr[3];
                    for (int a = 0; a < 3; ++a) dr[a] = double(lat.r_sl[mu][a] - lat.r_sl[nu][a]);
                    const double ph = q0 * (K0 * dr[0] + K1 * dr[1] + K2 * dr[2]);
                    Sk += cplx(std::cos(ph), std::sin(ph)) * Cmn;
                }
            out[(c * nk + k) * 2] = Sk.real();
            out[(c * nk + k) * 2 + 1] = Sk.imag();
        }
}

// Separable form: the same per-sublattice DFT over cells as ssf_sublattice,
// done as three passes of 1-D DFTs along x, y and z (O(Nc L) per sublattice
// and component instead of O(Nc^2)), then the phase contraction written as
// S^{ab}(K) = conj(B^a(K)) B^b(K) with B^a(K) = sum_mu exp(-i q.r_mu) A^a_mu(K)
// (the mu-nu double sum of ssf_sublattice factorises). Used by the anneal
// protocol at larger L; equal to ssf_direct to FP64 rounding (tested).
static void ssf_separable(const Lattice& lat, const std::vector<std::pair<int, int>>& corr, double* out) {
    const int L = lat.L, nk = lat.Nc;
    std::vector<cplx> w(static_cast<size_t>(L));
    for (int m = 0; m < L; ++m) w[size_t(m)] = cplx(std::cos(-2 * M_PI * m / L), std::sin(-2 * M_PI * m / L));
    const double q0 = 2 * M_PI / (8.0 * L);
    std::vector<cplx> Bk(size_t(3) * nk, cplx(0, 0));
    std::vector<cplx> A(static_cast<size_t>(nk)), tmp(static_cast<size_t>(nk));
    for (int a = 0; a < 3; ++a)
        for (int sl = 0; sl < 16; ++sl) {
            for (int cell = 0; cell < nk; ++cell) A[size_t(cell)] = lat.spins[size_t(sl) * nk + cell].S[a];
            // axis d: stride 1 (x), L (y), L*L (z)
            for (int d = 0; d < 3; ++d) {
                const int stride = d == 0 ? 1 : (d == 1 ? L : L * L);
                for (int base = 0; base < nk; ++base) {
                    if ((base / stride) % L != 0) continue;  // base = start of a line along d
                    for (int K = 0; K < L; ++K) {
                        cplx acc = 0;
                        for (int n = 0; n < L; ++n) acc += w[size_t((K * n) % L)] * A[size_t(base + n * stride)];
                        tmp[size_t(base + K * stride)] = acc;
                    }
                }
                std::swap(A, tmp);
            }
            for (int Kz = 0; Kz < L; ++Kz)
                for (int Ky = 0; Ky < L; ++Ky)
                    for (int Kx = 0; Kx < L; ++Kx) {
                        const double ph = -q0 * (Kx * double(lat.r_sl[size_t(sl)][0]) + Ky * double(lat.r_sl[size_t(sl)][1]) +
                                                 Kz * double(lat.r_sl[size_t(sl)][2]));
                        const int k = (Kx * L + Ky) * L + Kz;
                        Bk[size_t(a) * nk + k] += cplx(std::cos(ph), std::sin(ph)) * A[size_t(Kx + L * (Ky + L * Kz))];
                    }
        }
    for (size_t c = 0; c < corr.size(); ++c)
        for (int k = 0; k < nk; ++k) {
            const cplx v = std::conj(Bk[size_t(corr[c].first) * nk + k]) * Bk[size_t(corr[c].second) * nk + k];
            out[(c * nk + k) * 2] = v.real();
            out[(c * nk + k) * 2 + 1] = v.imag();
        }
}

// generate_T_profile (include/cli_bits.hpp:250-289)
static std::pair<std::vector<double>, std::set<size_t>> generate_T_profile(double T_hot, double T_cold,
                                                                          std::vector<double> T_sample,
                                                                          size_t total_steps) {
    std::vector<double> T_sweep, T;
    const double factor = std::pow(T_cold / T_hot, 1.0 / double(total_steps));
    double t = T_hot / factor;
    for (size_t i = 0; i < total_steps; ++i) {
        t *= factor;
        T_sweep.push_back(t);
    }
    std::sort(T_sweep.begin(), T_sweep.end(), [](double a, double b) { return a > b; });
    std::sort(T_sample.begin(), T_sample.end(), [](double a, double b) { return a > b; });
    size_t i_samp = 0, i_sw = 0;
    std::set<size_t> idx;
    while (i_sw < T_sweep.size() && i_samp < T_sample.size()) {
        if (T_sweep[i_sw] > T_sample[i_samp]) {
            T.push_back(T_sweep[i_sw]);
            ++i_sw;
        } else {
            idx.insert(T.size());
            T.push_back(T_sample[i_samp]);
            ++i_samp;
        }
    }
    for (; i_samp < T_sample.size(); ++i_samp) {
        idx.insert(T.size());
        T.push_back(T_sample[i_samp]);
    }
    for (; i_sw < T_sweep.size(); ++i_sw) T.push_back(T_sweep[i_sw]);
    return {T, idx};
}

static void random_unit_spins(Lattice& lat, uint64_t seed) {
    std::mt19937_64 g(seed);
    std::normal_distribution<double> nd;
    for (auto& s : lat.spins) {
        vec3 v = {nd(g), nd(g), nd(g)};
        s.S = scale(1.0 / std::sqrt(dot(v, v)), v);
    }
}

struct System {
    Lattice lat;
    Runner mc;
    System(int L, uint64_t seed) : lat(L), mc(lat, seed) {}
};

static thread_local std::string g_err;

}  // namespace orc

using namespace orc;

// ---------------------------------------------------------------------------
// C entry points for the Python test harness (ctypes). All return 0 on success.
// ---------------------------------------------------------------------------
extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

// j1_mode 0: six XXZ pair specs (cli_bits.hpp:175-197); 1: one isotropic J1 spec
// (spiral_byhand.cpp:81-83).
void* orc_create(int L, double J1, double J2, double J3, double Delta, const double* B, double T_ref, uint64_t seed,
                 int j1_mode) {
    try {
        auto* s = new System(L, seed);
        define_pyro_couplings(s->mc, J1, J2, J3, Delta, j1_mode);
        s->mc.B = {B[0], B[1], B[2]};
        s->mc.T_ref = T_ref;
        s->mc.setup_lattice();
        return s;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}
void orc_destroy(void* h) { delete static_cast<System*>(h); }

int orc_num_spins(void* h) { return int(static_cast<System*>(h)->lat.spins.size()); }

void orc_set_spins(void* h, const double* S) {
    auto& sp = static_cast<System*>(h)->lat.spins;
    for (size_t i = 0; i < sp.size(); ++i) sp[i].S = {S[3 * i], S[3 * i + 1], S[3 * i + 2]};
}
void orc_get_spins(void* h, double* S) {
    auto& sp = static_cast<System*>(h)->lat.spins;
    for (size_t i = 0; i < sp.size(); ++i)
        for (int a = 0; a < 3; ++a) S[3 * i + a] = sp[i].S[a];
}
void orc_random_spins(void* h, uint64_t seed) { random_unit_spins(static_cast<System*>(h)->lat, seed); }
// A fresh MC_runner stream on the same lattice: Xoroshiro128++ re-seeded and
// the distributions' cached state cleared (normal_distribution keeps the
// second value of each polar pair), as if the runner were constructed anew.
void orc_reseed(void* h, uint64_t seed) {
    auto& mc = static_cast<System*>(h)->mc;
    mc.rng = Xoroshiro128pp(seed);
    mc.normal_dist.reset();
    mc.rand01.reset();
    mc.exp_dist.reset();
}
void orc_set_field(void* h, const double* B) { static_cast<System*>(h)->mc.B = {B[0], B[1], B[2]}; }

void orc_positions(void* h, int64_t* pos, int32_t* sl) {
    auto& sp = static_cast<System*>(h)->lat.spins;
    for (size_t i = 0; i < sp.size(); ++i) {
        for (int a = 0; a < 3; ++a) pos[3 * i + a] = sp[i].pos[a];
        sl[i] = sp[i].sl;
    }
}

// Neighbour indices of every site for each coupling spec, in the displacement
// order of that spec: out[(spec*N + i)*max_nb + j], -1 padded. Returns max_nb
// used, or -1 if max_nb is too small.
int orc_neighbours(void* h, int spec, int max_nb, int32_t* out) {
    auto* s = static_cast<System*>(h);
    const auto& c = s->mc.specs.at(size_t(spec));
    const size_t N = s->lat.spins.size();
    int used = 0;
    for (size_t i = 0; i < N; ++i) {
        const Spin& o = s->lat.spins[i];
        const auto& rel = c.rel.at(size_t(o.pyro_sl));
        if (int(rel.size()) > max_nb) return -1;
        used = std::max(used, int(rel.size()));
        for (int j = 0; j < max_nb; ++j) out[i * max_nb + j] = -1;
        for (size_t j = 0; j < rel.size(); ++j) {
            ipos x = {o.pos[0] + rel[j][0], o.pos[1] + rel[j][1], o.pos[2] + rel[j][2]};
            out[i * max_nb + j] = int32_t(s->lat.index_at(x));
        }
    }
    return used;
}
int orc_num_specs(void* h) { return int(static_cast<System*>(h)->mc.specs.size()); }
void orc_spec_matrix(void* h, int spec, double* J9) {
    const auto& c = static_cast<System*>(h)->mc.specs.at(size_t(spec));
    for (int i = 0; i < 9; ++i) J9[i] = c.J[i];
}
// Displacement table of one spec for one pyro sublattice: writes n*3 int64.
int orc_spec_displacements(void* h, int spec, int pyro_sl, int64_t* out, int max_n) {
    const auto& c = static_cast<System*>(h)->mc.specs.at(size_t(spec));
    const auto& r = c.rel.at(size_t(pyro_sl));
    if (int(r.size()) > max_n) return -1;
    for (size_t j = 0; j < r.size(); ++j)
        for (int a = 0; a < 3; ++a) out[3 * j + a] = r[j][a];
    return int(r.size());
}

double orc_energy(void* h) { return static_cast<System*>(h)->mc.total_energy_per_unit_cell(); }
void orc_magnetisation(void* h, double* m) {
    vec3 t{0, 0, 0};
    for (const auto& s : static_cast<System*>(h)->lat.spins) t = add(t, s.S);
    m[0] = t[0];
    m[1] = t[1];
    m[2] = t[2];
}

void orc_local_fields(void* h, double* out) {
    auto* s = static_cast<System*>(h);
    for (size_t i = 0; i < s->lat.spins.size(); ++i) {
        const vec3 v = s->mc.local_field(&s->lat.spins[i]);
        for (int a = 0; a < 3; ++a) out[3 * i + a] = v[a];
    }
}

// Coupling-matrix gradient dE_total/dJ_spec[a][b] = sum over bonds of the spec
// S_src[a] S_tgt[b] (each bond counted once), from the half sum over sites.
void orc_coupling_grads(void* h, double* out /* [n_specs][9] */) {
    auto* s = static_cast<System*>(h);
    const size_t ns = s->mc.specs.size();
    for (size_t i = 0; i < ns * 9; ++i) out[i] = 0;
    for (const auto& sp : s->lat.spins)
        for (const auto& sh : sp.shells) {
            size_t spec = 0;
            bool is_T = false;
            for (size_t c = 0; c < ns; ++c) {
                if (sh.J == &s->mc.specs[c].J) { spec = c; is_T = false; break; }
                if (sh.J == &s->mc.specs[c].Jt) { spec = c; is_T = true; break; }
            }
            vec3 t{0, 0, 0};
            for (const Spin* o : sh.bonds) t = add(t, o->S);
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b)
                    out[spec * 9 + 3 * a + b] += 0.5 * (is_T ? t[a] * sp.S[b] : sp.S[a] * t[b]);
        }
}

uint64_t orc_sweep(void* h, double T, int n_sweeps, int n_overrelax) {
    auto* s = static_cast<System*>(h);
    uint64_t acc = 0;
    for (int i = 0; i < n_sweeps; ++i) acc += s->mc.sweep_local_Metropolis(T, size_t(n_overrelax));
    return acc;
}

// colour_of_sl[16]: colour index per sublattice; colours visited 0..n_colours-1,
// sublattices inside a colour in increasing order.
uint64_t orc_sweep_lifted(void* h, double T, int n_sweeps, int n_overrelax, int rot) {
    auto* s = static_cast<System*>(h);
    uint64_t acc = 0;
    for (int i = 0; i < n_sweeps; ++i) acc += s->mc.sweep_lifted_Metropolis(T, size_t(n_overrelax), rot != 0);
    return acc;
}

// lifting directions (+1 / -1) per site in storage order
void orc_get_lifted(void* h, int8_t* out) {
    auto* s = static_cast<System*>(h);
    for (size_t i = 0; i < s->lat.spins.size(); ++i) out[i] = s->lat.spins[i].lifted_dir;
}
void orc_set_lifted(void* h, const int8_t* in) {
    auto* s = static_cast<System*>(h);
    for (size_t i = 0; i < s->lat.spins.size(); ++i) s->lat.spins[i].lifted_dir = in[i] < 0 ? int8_t(-1) : int8_t(1);
}

uint64_t orc_sweep_philox(void* h, double T, uint64_t seed, uint32_t replica, uint64_t sweep, int n_overrelax,
                          const int32_t* colour_of_sl, int or_mode, int fused, int update) {
    auto* s = static_cast<System*>(h);
    int nc = 0;
    for (int i = 0; i < 16; ++i) nc = std::max(nc, colour_of_sl[i] + 1);
    std::vector<std::vector<int>> cls(static_cast<size_t>(nc));
    for (int i = 0; i < 16; ++i) cls[size_t(colour_of_sl[i])].push_back(i);
    return s->mc.sweep_philox(T, seed, replica, sweep, n_overrelax, cls, or_mode, fused != 0, update);
}

// One overrelaxation pass with caller-supplied angles (theta[i] per site) or
// reflection (theta == nullptr): overrelax_all with the rand01 draw replaced by
// the given angle. Visits sites in storage order, or colour class by colour
// class when colour_of_sl[16] is given.
void orc_overrelax(void* h, const double* theta, const int32_t* colour_of_sl) {
    auto* s = static_cast<System*>(h);
    std::vector<size_t> order;
    const size_t Nc = size_t(s->lat.Nc);
    if (colour_of_sl) {
        int nc = 0;
        for (int i = 0; i < 16; ++i) nc = std::max(nc, colour_of_sl[i] + 1);
        for (int c = 0; c < nc; ++c)
            for (int sl = 0; sl < 16; ++sl)
                if (colour_of_sl[sl] == c)
                    for (size_t cell = 0; cell < Nc; ++cell) order.push_back(size_t(sl) * Nc + cell);
    } else {
        for (size_t i = 0; i < s->lat.spins.size(); ++i) order.push_back(i);
    }
    for (size_t i : order) {
        Spin& sp = s->lat.spins[i];
        const vec3 hh = sub(s->mc.local_field(&sp), s->mc.B);
        if (theta)
            Runner::rotate_about_vector(sp.S, hh, theta[i]);
        else
            Runner::mirror_about_vector(sp.S, hh);
    }
}

// corr: n_corr pairs (alpha,beta); out [n_corr][n_k][2]. mode 0 direct, 1 sublattice.
void orc_ssf(void* h, const int32_t* corr, int n_corr, int mode, double* out, double* resolved) {
    auto* s = static_cast<System*>(h);
    std::vector<std::pair<int, int>> c;
    for (int i = 0; i < n_corr; ++i) c.push_back({corr[2 * i], corr[2 * i + 1]});
    if (mode == 0)
        ssf_direct(s->lat, c, out);
    else if (mode == 2)
        ssf_separable(s->lat, c, out);
    else
        ssf_sublattice(s->lat, c, out, resolved);
}

// generate_T_profile; returns the number of temperatures written (<= max_n),
// marks sample indices in is_sample.
int orc_T_profile(double T_hot, double T_cold, const double* T_sample, int n_sample, int total_steps, double* T_out,
                  int32_t* is_sample, int max_n) {
    std::vector<double> ts(T_sample, T_sample + n_sample);
    auto [T, idx] = generate_T_profile(T_hot, T_cold, ts, size_t(total_steps));
    if (int(T.size()) > max_n) return -1;
    for (size_t i = 0; i < T.size(); ++i) {
        T_out[i] = T[i];
        is_sample[i] = idx.count(i) ? 1 : 0;
    }
    return int(T.size());
}

// The anneal protocol of src/anneal.cpp:193-227 on an existing system:
// burn-in at T_hot, then for each T of the profile n_sweep sweeps and one energy
// sample; at the sample temperatures n_sample x (n_sweep sweeps + SSF sample).
// e_out[n_T] receives the energy per cubic cell per temperature; ssf_sum/ssf_sq
// [n_T_sample][n_corr][n_k][2] the SSF accumulators in descending-T visit order.
int orc_anneal(void* h, double T_hot, double T_cold, const double* T_sample, int n_T_sample, int n_steps,
               int n_sweep, int n_burn_in, int n_samp, const int32_t* corr, int n_corr, double* T_out, double* e_out,
               double* ssf_sum, double* ssf_sq, int max_T) {
    auto* s = static_cast<System*>(h);
    std::vector<double> ts(T_sample, T_sample + n_T_sample);
    auto [T_grid, S_idx] = generate_T_profile(T_hot, T_cold, ts, size_t(n_steps));
    if (int(T_grid.size()) > max_T) return -1;
    std::vector<std::pair<int, int>> c;
    for (int i = 0; i < n_corr; ++i) c.push_back({corr[2 * i], corr[2 * i + 1]});
    const size_t nk = size_t(s->lat.Nc);
    std::vector<double> tmp(size_t(std::max(n_corr, 1)) * nk * 2);
    for (int i = 0; i < n_burn_in; ++i) s->mc.sweep_local_Metropolis(T_hot, 1);
    int slot = 0;
    for (size_t i = 0; i < T_grid.size(); ++i) {
        const double T = T_grid[i];
        T_out[i] = T;
        for (int n = 0; n < n_sweep; ++n) s->mc.sweep_local_Metropolis(T, 1);
        e_out[i] = s->mc.total_energy_per_unit_cell();
        if (S_idx.count(i)) {
            double* sum = ssf_sum + size_t(slot) * n_corr * nk * 2;
            double* sq = ssf_sq + size_t(slot) * n_corr * nk * 2;
            for (size_t j = 0; j < size_t(n_corr) * nk * 2; ++j) sum[j] = sq[j] = 0;
            for (int smp = 0; smp < n_samp; ++smp) {
                for (int n = 0; n < n_sweep; ++n) s->mc.sweep_local_Metropolis(T, 1);
                if (n_corr > 0) {
                    ssf_separable(s->lat, c, tmp.data());
                    for (size_t j = 0; j < size_t(n_corr) * nk * 2; ++j) {
                        sum[j] += tmp[j];
                        sq[j] += tmp[j] * tmp[j];
                    }
                }
            }
            ++slot;
        }
    }
    return int(T_grid.size());
}

// Parallel tempering as src/temper.cpp:386-474 runs it, with the MPI ranks
// emulated in one process: replica r holds temperature T[r] (T descending),
// its own runner seeded seed+r and swap rng seeded seed+R+r; checkerboard pairs
// by round parity; the lower (hotter) rank decides with
// arg = (1/T - 1/T')(E - E') on total energies; accepted pairs swap spins.
// A round is n_sweep sweeps (temper.cpp's non-sampled ranks add one extra
// sweep per round, :426-429: pass n_sweep+1 for that), then one energy sample
// per slot, then the exchange. e_sum/e2_sum per temperature slot;
// attempts/accepts per lower slot of each pair.
// n_burn_in sweeps per replica without exchanges, then n_burn_rounds full
// rounds (sweeps, energy, exchange) whose statistics are discarded, then the
// n_rounds measured rounds; the pair parity counts every round.
int orc_temper(int L, double J1, double J2, double J3, double Delta, const double* B, double T_ref, uint64_t seed,
               const double* T, int R, int n_burn_in, int n_burn_rounds, int n_rounds, int n_sweep, int init_random,
               double* e_sum, double* e2_sum, uint64_t* attempts, uint64_t* accepts) {
    try {
        std::vector<std::unique_ptr<System>> sys;
        std::vector<Xoroshiro128pp> swap_rng;
        for (int r = 0; r < R; ++r) {
            sys.emplace_back(new System(L, seed + uint64_t(r)));
            define_pyro_couplings(sys.back()->mc, J1, J2, J3, Delta, 0);
            sys.back()->mc.B = {B[0], B[1], B[2]};
            sys.back()->mc.T_ref = T_ref;
            sys.back()->mc.setup_lattice();
            if (init_random) random_unit_spins(sys.back()->lat, seed * 7919 + uint64_t(r));
            swap_rng.emplace_back(seed + uint64_t(R) + uint64_t(r));
        }
        std::uniform_real_distribution<double> rand01(0.0, 1.0);
        for (int r = 0; r < R; ++r) {
            e_sum[r] = e2_sum[r] = 0;
            attempts[r] = accepts[r] = 0;
        }
        for (int r = 0; r < R; ++r)
            for (int i = 0; i < n_burn_in; ++i) sys[r]->mc.sweep_local_Metropolis(T[r], 1);
        const double Np = double(sys[0]->lat.Nc);
        std::vector<double> e(static_cast<size_t>(R));
        for (int round = 0; round < n_burn_rounds + n_rounds; ++round) {
            const bool measured = round >= n_burn_rounds;
            for (int r = 0; r < R; ++r) {
                for (int sw = 0; sw < n_sweep; ++sw) sys[r]->mc.sweep_local_Metropolis(T[r], 1);
                e[r] = sys[r]->mc.total_energy_per_unit_cell();
                if (measured) {
                    e_sum[r] += e[r];
                    e2_sum[r] += e[r] * e[r];
                }
            }
            const int start = round % 2;
            for (int r = start; r + 1 < R; r += 2) {
                const double arg = (1.0 / T[r] - 1.0 / T[r + 1]) * (e[r] * Np - e[r + 1] * Np);
                const bool acc = arg >= 0.0 || rand01(swap_rng[r]) < std::exp(arg);
                if (measured) attempts[r]++;
                if (acc) {
                    if (measured) accepts[r]++;
                    for (size_t i = 0; i < sys[r]->lat.spins.size(); ++i)
                        std::swap(sys[r]->lat.spins[i].S, sys[r + 1]->lat.spins[i].S);
                }
            }
        }
        return 0;
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return 1;
    }
}

// CPU baseline: reference-faithful sweeps (sequential storage order, pointer
// shells, Xoroshiro128++ and libstdc++ distributions, src/MC.cpp:111-163) of
// n_threads independent L-lattices with J1..J3 and B, one per thread with its
// own seed (how acc_runs.py ensembles are produced), built in parallel.
struct Bench {
    std::vector<std::unique_ptr<System>> sys;
};

void* orc_bench_create(int L, double J1, double J2, double J3, const double* B, int n_threads, uint64_t seed) {
    auto* b = new Bench();
    b->sys.resize(size_t(n_threads));
    std::vector<std::thread> th;
    for (int t = 0; t < n_threads; ++t)
        th.emplace_back([&, t]() {
            auto s = std::make_unique<System>(L, seed + uint64_t(t));
            define_pyro_couplings(s->mc, J1, J2, J3, 1.0, 0);
            s->mc.B = {B[0], B[1], B[2]};
            s->mc.setup_lattice();
            random_unit_spins(s->lat, seed + 1000 + uint64_t(t));
            b->sys[size_t(t)] = std::move(s);
        });
    for (auto& x : th) x.join();
    return b;
}

// Runs n_sweeps sweeps at T on every lattice concurrently; returns the
// aggregate spin-updates per second (N * sweeps summed over lattices, over the
// slowest thread's time).
double orc_bench_run(void* h, double T, int n_sweeps) {
    auto* b = static_cast<Bench*>(h);
    const size_t n = b->sys.size();
    std::vector<double> secs(n, 0.0);
    std::vector<std::thread> th;
    for (size_t t = 0; t < n; ++t)
        th.emplace_back([&, t]() {
            const auto t0 = std::chrono::steady_clock::now();
            for (int i = 0; i < n_sweeps; ++i) b->sys[t]->mc.sweep_local_Metropolis(T, 1);
            secs[t] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        });
    for (auto& x : th) x.join();
    const double worst = *std::max_element(secs.begin(), secs.end());
    return double(b->sys[0]->lat.spins.size()) * double(n_sweeps) * double(n) / worst;
}

void orc_bench_destroy(void* h) { delete static_cast<Bench*>(h); }

double orc_bench_sweeps(int L, double J1, double J2, double J3, const double* B, double T, int n_sweeps,
                        int n_threads, uint64_t seed) {
    void* h = orc_bench_create(L, J1, J2, J3, B, n_threads, seed);
    const double r = orc_bench_run(h, T, n_sweeps);
    orc_bench_destroy(h);
    return r;
}

// Philox block for tests (known-answer vectors and the GPU draw layout).
void orc_philox(const uint32_t* ctr, const uint32_t* key, uint32_t* out) { philox4x32_10(ctr, key, out); }

// Xoroshiro128++ / libstdc++ distribution draws for pinning against the
// reference's XoshiroCpp.hpp: kind 0 raw u64, 1 normal, 2 uniform [0,1).
void orc_xoshiro_draws(uint64_t seed, int kind, int n, double* out_d, uint64_t* out_u) {
    Xoroshiro128pp g(seed);
    std::normal_distribution<double> nd;
    std::uniform_real_distribution<double> ud(0.0, 1.0);
    for (int i = 0; i < n; ++i) {
        if (kind == 0)
            out_u[i] = g();
        else if (kind == 1)
            out_d[i] = nd(g);
        else
            out_d[i] = ud(g);
    }
}

}  // extern "C"
