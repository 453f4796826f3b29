// ref_mc_main.cpp -- TEST INFRASTRUCTURE ONLY.
//
// C entry points over the reference's OWN Monte Carlo code: make_ref.sh
// compiles the reference's src/MC.cpp unchanged, where it lies, together with
// this file and the stand-ins under oracle/ref_shim/ (lattice_lib's Supercell,
// empty HDF5 and json declarations), into oracle/_ref/libref_mc.so. The tests
// use it to pin the oracle (oracle/pyro_oracle.cpp) on the reference itself:
// bond shells, local field, energy and whole sequential Metropolis /
// overrelaxation chains from the same Xoroshiro128++ seed. bench.py may time
// its sweep as the reference's CPU baseline. Nothing in the product loads it.
//
// The lattice is the reference's PyroCubicCell (include/pyrochlore_geometry.hpp
// :12-32) in an L*I supercell; the couplings are those of build_J1J2J3_h
// (include/cli_bits.hpp:144-207): six J1 sublattice-pair specs
// J1*(Delta-1)*Ising + J1*Heis from the reference's nn1_pair_MN tables and
// local axes, then J2, J3a, J3b (always defined), the global field and T_ref,
// then setup_lattice(). The runner is constructed with the raw seed (the
// reference passes hash_true_random(seed); the oracle takes the same raw seed).
//
// MC_runner::local_field is private in include/MC.hpp (the class's default
// access); it is reached here by reading that header, in this one file, with
// `class` spelled `struct` after every other header it includes has been
// included. MC.cpp itself is compiled unchanged; the class key changes
// neither the layout nor the (Itanium-mangled) symbol names.
#include <cassert>
#include <cstdint>
#include <cstring>
#include <exception>
#include <filesystem>
#include <map>
#include <random>
#include <string>
#include <vector>

#include <XoshiroCpp.hpp>
#include <lattice_lib/supercell.hpp>
#include <nlohmann/json.hpp>

#include "H5Ipublic.h"
#include "H5Ppublic.h"
#include "H5Tpublic.h"

#define class struct
#include "MC.hpp"
#undef class
#include "pyrochlore_geometry.hpp"

namespace {

struct RefSystem {
    CMC::Lattice lat;
    CMC::MC_runner mc;
    RefSystem(int L, uint64_t seed)
        : lat(build_supercell(PyroCubicCell(), imat33_t::from_cols({L, 0, 0}, {0, L, 0}, {0, 0, L}))),
          mc(lat, seed) {}
};

thread_local std::string g_err;

using mat33d = vector3::mat33<double>;
using vec3d = vector3::vec3<double>;

// build_J1J2J3_h's coupling definitions (include/cli_bits.hpp:166-202),
// with the parsed arguments passed in directly.
void define_couplings(CMC::MC_runner& mc, double J1, double J2, double J3, double Delta) {
    const mat33d Heis = mat33d::from_cols({1, 0, 0}, {0, 1, 0}, {0, 0, 1});
    static const std::pair<int, int> pairs[6] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
    static const std::vector<std::vector<ipos_t>>* nn1_pairs[6] = {
        &pyrochlore::nn1_pair_01, &pyrochlore::nn1_pair_02, &pyrochlore::nn1_pair_03,
        &pyrochlore::nn1_pair_12, &pyrochlore::nn1_pair_13, &pyrochlore::nn1_pair_23};
    for (int k = 0; k < 6; k++) {
        auto [mu, nu] = pairs[k];
        const vec3d& z_mu = pyrochlore::axis[mu][2];
        const vec3d& z_nu = pyrochlore::axis[nu][2];
        auto v2a = [](vec3d v) -> std::array<double, 3> { return {v[0], v[1], v[2]}; };
        mat33d Ising = mat33d::from_cols(v2a(z_nu[0] * z_mu), v2a(z_nu[1] * z_mu), v2a(z_nu[2] * z_mu));
        std::string pname = "J1_" + std::to_string(mu) + std::to_string(nu);
        mc.define_coupling(pname, *nn1_pairs[k], J1 * (Delta - 1) * Ising + J1 * Heis);
    }
    mc.define_coupling("J2", pyrochlore::nn2_dist, J2 * Heis);
    mc.define_coupling("J3a", pyrochlore::nn3a_dist, J3 * Heis);
    mc.define_coupling("J3b", pyrochlore::nn3b_dist, J3 * Heis);
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

void* ref_create(int L, double J1, double J2, double J3, double Delta, const double* B, double T_ref, uint64_t seed) {
    try {
        auto* s = new RefSystem(L, seed);
        define_couplings(s->mc, J1, J2, J3, Delta);
        s->mc.set_global_field(vec3d(B[0], B[1], B[2]));
        s->mc.settings.T_ref = T_ref;
        s->mc.setup_lattice();
        return s;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void ref_destroy(void* h) { delete static_cast<RefSystem*>(h); }

int64_t ref_num_spins(void* h) { return int64_t(static_cast<RefSystem*>(h)->lat.get_objects<CMC::HeisenbergSpin>().size()); }

void ref_set_spins(void* h, const double* S) {
    auto& sp = static_cast<RefSystem*>(h)->lat.get_objects<CMC::HeisenbergSpin>();
    for (size_t i = 0; i < sp.size(); ++i) sp[i].S = vec3d(S[3 * i], S[3 * i + 1], S[3 * i + 2]);
}

void ref_get_spins(void* h, double* S) {
    const auto& sp = static_cast<RefSystem*>(h)->lat.get_objects<CMC::HeisenbergSpin>();
    for (size_t i = 0; i < sp.size(); ++i)
        for (int a = 0; a < 3; ++a) S[3 * i + a] = sp[i].S[size_t(a)];
}

void ref_positions(void* h, int64_t* pos) {
    const auto& sp = static_cast<RefSystem*>(h)->lat.get_objects<CMC::HeisenbergSpin>();
    for (size_t i = 0; i < sp.size(); ++i)
        for (int a = 0; a < 3; ++a) pos[3 * i + a] = sp[i].ipos[size_t(a)];
}

// The bond shells setup_lattice built (src/MC.cpp:15-52), flattened: for each
// site in storage order, its shells in order, each as (matrix 9 doubles, count,
// neighbour site indices). Returns the number of int32 written into idx (the
// layout: per shell [n, i_1..i_n]) or -1 if max_idx is too small; mats gets 9
// doubles per shell and n_shells[site] the shell count.
int64_t ref_shells(void* h, int32_t* n_shells, double* mats, int64_t max_mats, int32_t* idx, int64_t max_idx) {
    auto* s = static_cast<RefSystem*>(h);
    const auto& sp = s->lat.get_objects<CMC::HeisenbergSpin>();
    const CMC::HeisenbergSpin* base = sp.data();
    int64_t w = 0, m = 0;
    for (size_t i = 0; i < sp.size(); ++i) {
        n_shells[i] = int32_t(sp[i].bond_shells.size());
        for (const auto& sh : sp[i].bond_shells) {
            if (m >= max_mats || w + 1 + int64_t(sh.bonds.size()) > max_idx) return -1;
            for (int a = 0; a < 9; ++a) mats[9 * m + a] = (*sh.J)(a / 3, a % 3);
            ++m;
            idx[w++] = int32_t(sh.bonds.size());
            for (const auto* o : sh.bonds) idx[w++] = int32_t(o - base);
        }
    }
    return w;
}

double ref_energy(void* h) { return static_cast<RefSystem*>(h)->mc.total_energy_per_unit_cell(); }

// MC_runner::local_field (src/MC.cpp:87-96) of every site, without the field.
void ref_local_fields(void* h, double* out) {
    auto* s = static_cast<RefSystem*>(h);
    const auto& sp = s->lat.get_objects<CMC::HeisenbergSpin>();
    for (size_t i = 0; i < sp.size(); ++i) {
        const vec3d f = s->mc.local_field(&sp[i]);
        for (int a = 0; a < 3; ++a) out[3 * i + a] = f[size_t(a)];
    }
}

uint64_t ref_sweep(void* h, double T, int n_sweeps, int n_overrelax) {
    auto* s = static_cast<RefSystem*>(h);
    uint64_t acc = 0;
    for (int i = 0; i < n_sweeps; ++i) acc += s->mc.sweep_local_Metropolis(T, size_t(n_overrelax));
    return acc;
}

uint64_t ref_sweep_lifted(void* h, double T, int n_sweeps, int n_overrelax, int rot) {
    auto* s = static_cast<RefSystem*>(h);
    uint64_t acc = 0;
    for (int i = 0; i < n_sweeps; ++i)
        acc += rot ? s->mc.sweep_lifted_Metropolis_rot(T, size_t(n_overrelax))
                   : s->mc.sweep_lifted_Metropolis(T, size_t(n_overrelax));
    return acc;
}

void ref_overrelax_all(void* h) { static_cast<RefSystem*>(h)->mc.overrelax_all(); }

void ref_get_lifted(void* h, int8_t* out) {
    const auto& sp = static_cast<RefSystem*>(h)->lat.get_objects<CMC::HeisenbergSpin>();
    for (size_t i = 0; i < sp.size(); ++i) out[i] = sp[i].lifted_dir;
}

}  // extern "C"
