// MC.hpp -- drop-in for the reference's include/MC.hpp on the B200 engine.
//
// CMC::MC_runner keeps the reference's interface (include/MC.hpp:87-140):
// define_coupling, set/get_global_field, setup_lattice,
// sweep_local_Metropolis(T, n_overrelax) -> accepted, overrelax_all,
// total_energy_per_unit_cell, rebind, settings.T_ref. The work runs on the GPU
// through the C ABI (include/pyrocmc.h); nothing is computed on the host.
//
// CMC::Lattice stands in for lattice_lib's Supercell<HeisenbergSpin>
// (include/MC.hpp:63) for the pyrochlore L*I supercell of the 16-site cubic
// cell: it exposes the members the drivers use (get_objects<HeisenbergSpin>(),
// lattice.num_primitive_cells(), lattice.size(), sl_positions, get_object_at)
// and owns the device copy of the spins. The device copy is authoritative
// while MC runs; get_objects() brings the host mirror up to date and hands it
// to the caller, whose edits are uploaded before the next device operation.
#pragma once

#include <cstdint>
#include <filesystem>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/pyrocmc.h"
#include "vec3.hpp"

namespace CMC {

using dmat33_t = vector3::mat33<double>;

// Throws the exception type the reference uses for the failing condition.
void check(int rc);

struct HeisenbergSpin {
    ipos_t ipos;  // wrapped into [0, 8L)
    int pyro_sl = 0;
    vector3::vec3d S;
    int8_t lifted_dir = 1;
};

// The index arithmetic of the cubic supercell (lattice_lib LatticeIndexing).
struct LatticeIndexing {
    int L = 1;
    int num_primitive_cells() const { return L * L * L; }
    ivec3_t size() const { return ivec3_t(L, L, L); }
    // lattice vectors of the supercell as columns (8L * I) and the reciprocal
    // vectors b_i with a_i . b_j = 2 pi delta_ij (rows)
    imat33_t get_lattice_vectors() const {
        return imat33_t::from_cols({8 * L, 0, 0}, {0, 8 * L, 0}, {0, 0, 8 * L});
    }
    vector3::mat33<double> get_reciprocal_lattice_vectors() const {
        const double b = 2 * M_PI / (8.0 * L);
        return vector3::mat33<double>::from_cols({b, 0, 0}, {0, b, 0}, {0, 0, b});
    }
    // q for integer k indices K: q = 2 pi K / (8L) (the k grid of the SSF)
    vector3::vec3d wavevector_from_idx3(const ivec3_t& K) const {
        const double b = 2 * M_PI / (8.0 * L);
        return vector3::vec3d(b * double(K[0]), b * double(K[1]), b * double(K[2]));
    }
};

class Lattice {
public:
    explicit Lattice(int L);
    ~Lattice();
    Lattice(const Lattice&) = delete;
    Lattice& operator=(const Lattice&) = delete;
    Lattice(Lattice&& o) noexcept;

    template <typename T>
    std::vector<HeisenbergSpin>& get_objects() {
        to_host();
        return spins_;
    }
    size_t num_spins() const { return spins_.size(); }
    HeisenbergSpin* get_object_at(const ipos_t& x);

    LatticeIndexing lattice;
    std::vector<ipos_t> sl_positions;  // r_sl = link[p] + R_fcc[f] (unwrapped)

    // device side
    pc_system* device() const { return sys_; }
    void to_device();  // upload the host mirror if the host holds the newer state
    void to_host();    // download if the device holds the newer state; host owns it after
    void mark_device_newer() { host_newer_ = false; device_newer_ = true; }

private:
    pc_system* sys_ = nullptr;
    std::vector<HeisenbergSpin> spins_;
    bool host_newer_ = true;
    bool device_newer_ = false;
};

// Specification of one coupling term (include/MC.hpp:72-77).
struct CouplingSpec {
    std::string name;
    std::vector<std::vector<ipos_t>> relative_vectors;
    dmat33_t J;
    dmat33_t Jt;
};

struct MC_parameters {
    double T_ref = 1.0;
    size_t verbosity = 2;
};

class MC_runner {
public:
    MC_parameters settings;

    MC_runner(Lattice& lat_, size_t seed);

    // Repoints the runner at a congruent Lattice (include/MC.hpp:117); the
    // couplings are replayed onto its device state if it has none yet.
    void rebind(Lattice& new_lat);

    double total_energy_per_unit_cell() const;

    void define_coupling(const std::string& name, const std::vector<std::vector<ipos_t>>& rel_vecs,
                         const vector3::mat33<double>& J);

    void set_global_field(const vector3::vec3<double>& h);
    vector3::vec3d get_global_field() const;

    void setup_lattice();

    void overrelax_all();
    size_t sweep_local_Metropolis(double T, size_t n_overrelax = 1);
    // n sweeps in one call (one host round trip)
    size_t sweep_local_Metropolis_n(double T, size_t n_sweeps, size_t n_overrelax = 1);
    // src/MC.cpp:284-302: lifted Metropolis sweeps (u-form / rotation form)
    size_t sweep_lifted_Metropolis(double T, size_t n_overrelax = 1);
    size_t sweep_lifted_Metropolis_rot(double T, size_t n_overrelax = 1);
    // n sweeps of the given single-site move (0 Metropolis, 1 lifted, 2 lifted rotation form)
    size_t sweep_n(int update, double T, size_t n_sweeps, size_t n_overrelax = 1);

    const std::vector<CouplingSpec>& couplings() const { return coupling_specs; }

private:
    std::vector<CouplingSpec> coupling_specs;
    std::map<std::string, size_t> index;
    vector3::vec3d global_field{0, 0, 0};
    Lattice* lat;
    size_t seed_;
    bool ready_ = false;

    void push_to(Lattice& l);
};

// /geometry group (src/MC.cpp:416-454): index_cell (int64 3x3), recip_vectors
// (f64 3x3); written into an output file (h5out.hpp).
class OutFile;
void write_geometry_group(OutFile& f, Lattice& sc, const char* group_name = "geometry");
// .spins file (src/MC.cpp:371-406): spin_pos int32 [N,3], spin_orientation f64 [N,3]
void save_spin_state(Lattice& lat, const std::filesystem::path& file_path);
// .spins_ft file (src/MC.cpp:320-368): spin_ft f64 [3, 16, n_k, 2], the raw
// per-sublattice DFT of each spin component (no sublattice phase)
void save_ft_spin_state(Lattice& lat, const std::filesystem::path& file_path);

}  // namespace CMC
