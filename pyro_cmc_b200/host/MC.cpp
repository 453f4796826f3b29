// MC.cpp -- CMC::Lattice and CMC::MC_runner over the C ABI (see MC.hpp).
#include "MC.hpp"

#include <cmath>
#include <stdexcept>

#include "h5out.hpp"

namespace CMC {

void check(int rc) {
    if (rc == PC_OK) return;
    const std::string msg = pc_last_error();
    if (rc == PC_ERR_INVALID) {
        if (msg.find("unique") != std::string::npos) throw std::logic_error(msg);
        throw std::invalid_argument(msg);
    }
    throw std::runtime_error(msg);
}

namespace {
const int64_t kLink[4][3] = {{1, 1, 1}, {1, -1, -1}, {-1, 1, -1}, {-1, -1, 1}};
const int64_t kFcc[4][3] = {{0, 0, 0}, {0, 4, 4}, {4, 0, 4}, {4, 4, 0}};
int64_t pmod(int64_t a, int64_t m) {
    const int64_t r = a % m;
    return r < 0 ? r + m : r;
}
}  // namespace

// Sites in the device order: sl = 4f + p at link[p] + R_fcc[f]
// (include/pyrochlore_geometry.hpp:12-32), spins[sl*Nc + cell],
// cell = cx + L*(cy + L*cz).
Lattice::Lattice(int L) {
    lattice.L = L;
    const int32_t Lv = L;
    check(pc_create(1, &Lv, 0, &sys_));
    for (int sl = 0; sl < 16; ++sl)
        sl_positions.push_back(ipos_t(kLink[sl % 4][0] + kFcc[sl / 4][0], kLink[sl % 4][1] + kFcc[sl / 4][1],
                                      kLink[sl % 4][2] + kFcc[sl / 4][2]));
    const int64_t Nc = int64_t(L) * L * L;
    spins_.resize(size_t(16 * Nc));
    for (int sl = 0; sl < 16; ++sl)
        for (int64_t cell = 0; cell < Nc; ++cell) {
            HeisenbergSpin& s = spins_[size_t(sl * Nc + cell)];
            const int64_t c[3] = {cell % L, (cell / L) % L, cell / (int64_t(L) * L)};
            for (int a = 0; a < 3; ++a) s.ipos[a] = pmod(8 * c[a] + sl_positions[size_t(sl)][a], 8 * int64_t(L));
            s.pyro_sl = sl % 4;
        }
}

Lattice::~Lattice() {
    if (sys_) pc_destroy(sys_);
}

Lattice::Lattice(Lattice&& o) noexcept
    : lattice(o.lattice),
      sl_positions(std::move(o.sl_positions)),
      sys_(o.sys_),
      spins_(std::move(o.spins_)),
      host_newer_(o.host_newer_),
      device_newer_(o.device_newer_) {
    o.sys_ = nullptr;
}

HeisenbergSpin* Lattice::get_object_at(const ipos_t& x) {
    const int L = lattice.L;
    const int64_t Nc = int64_t(L) * L * L;
    for (int sl = 0; sl < 16; ++sl) {
        const auto& r = sl_positions[size_t(sl)];
        if (pmod(x[0] - r[0], 8) || pmod(x[1] - r[1], 8) || pmod(x[2] - r[2], 8)) continue;
        const int64_t c[3] = {pmod((x[0] - r[0]) / 8, L), pmod((x[1] - r[1]) / 8, L), pmod((x[2] - r[2]) / 8, L)};
        to_host();
        return &spins_[size_t(sl * Nc + c[0] + L * (c[1] + int64_t(L) * c[2]))];
    }
    throw std::out_of_range("get_object_at: no site at this position");
}

// The device keeps each spin as a float4 whose fourth component carries the
// lifting direction (include/MC.hpp:57): its sign, >= 0 meaning +1.
void Lattice::to_device() {
    if (!host_newer_) return;
    std::vector<float> S(4 * spins_.size());
    for (size_t i = 0; i < spins_.size(); ++i) {
        for (int a = 0; a < 3; ++a) S[4 * i + size_t(a)] = float(spins_[i].S[a]);
        S[4 * i + 3] = spins_[i].lifted_dir < 0 ? -1.f : 1.f;
    }
    check(pc_set_spins_f4(sys_, 0, S.data()));
    host_newer_ = false;
}

void Lattice::to_host() {
    if (device_newer_) {
        std::vector<float> S(4 * spins_.size());
        check(pc_get_spins_f4(sys_, 0, S.data()));
        for (size_t i = 0; i < spins_.size(); ++i) {
            for (int a = 0; a < 3; ++a) spins_[i].S[a] = double(S[4 * i + size_t(a)]);
            spins_[i].lifted_dir = S[4 * i + 3] < 0.f ? int8_t(-1) : int8_t(1);
        }
        device_newer_ = false;
    }
    host_newer_ = true;  // the caller holds a mutable reference from here on
}

MC_runner::MC_runner(Lattice& lat_, size_t seed) : lat(&lat_), seed_(seed) {
    check(pc_set_seed(lat->device(), seed));
}

void MC_runner::define_coupling(const std::string& name, const std::vector<std::vector<ipos_t>>& rel_vecs,
                                const vector3::mat33<double>& J) {
    if (index.count(name)) throw std::logic_error("Coupling names must be unique");
    index[name] = coupling_specs.size();
    coupling_specs.push_back({name, rel_vecs, J, J.tr()});
}

void MC_runner::set_global_field(const vector3::vec3<double>& h) {
    global_field = h;
    const double B[3] = {h[0], h[1], h[2]};
    check(pc_set_global_field(lat->device(), B));
}

vector3::vec3d MC_runner::get_global_field() const { return global_field; }

void MC_runner::push_to(Lattice& l) {
    pc_system* s = l.device();
    check(pc_set_seed(s, seed_));
    for (const auto& c : coupling_specs) {
        std::vector<int64_t> rv;
        int32_t n[4] = {0, 0, 0, 0};
        for (int p = 0; p < 4; ++p) {
            if (size_t(p) < c.relative_vectors.size()) {
                n[p] = int32_t(c.relative_vectors[size_t(p)].size());
                for (const auto& v : c.relative_vectors[size_t(p)])
                    for (int a = 0; a < 3; ++a) rv.push_back(v[a]);
            }
        }
        check(pc_define_coupling(s, c.name.c_str(), rv.data(), n, c.J.m.data()));
    }
    const double B[3] = {global_field[0], global_field[1], global_field[2]};
    check(pc_set_global_field(s, B));
    check(pc_set_T_ref(s, settings.T_ref));
    check(pc_setup_lattice(s));
}

// src/MC.cpp:15-52, on the device: per-sublattice shells and colour classes.
void MC_runner::setup_lattice() {
    if (ready_) throw std::logic_error("setup_lattice() already called");
    push_to(*lat);
    ready_ = true;
}

void MC_runner::rebind(Lattice& new_lat) {
    if (new_lat.num_spins() != lat->num_spins()) throw std::logic_error("rebind: lattices differ in size");
    lat = &new_lat;
    int n_col = 0;
    if (ready_ && pc_colours(lat->device(), &n_col, nullptr) != PC_OK) push_to(*lat);
}

size_t MC_runner::sweep_n(int update, double T, size_t n_sweeps, size_t n_overrelax) {
    if (!ready_) throw std::logic_error("setup_lattice() has not been called");
    check(pc_set_T_ref(lat->device(), settings.T_ref));
    check(pc_set_update(lat->device(), update));
    lat->to_device();
    uint64_t acc = 0;
    check(pc_sweep(lat->device(), &T, int(n_sweeps), int(n_overrelax), &acc));
    lat->mark_device_newer();
    return size_t(acc);
}

size_t MC_runner::sweep_local_Metropolis_n(double T, size_t n_sweeps, size_t n_overrelax) {
    return sweep_n(0, T, n_sweeps, n_overrelax);
}

// src/MC.cpp:284-291
size_t MC_runner::sweep_lifted_Metropolis(double T, size_t n_overrelax) { return sweep_n(1, T, 1, n_overrelax); }

// src/MC.cpp:293-302
size_t MC_runner::sweep_lifted_Metropolis_rot(double T, size_t n_overrelax) { return sweep_n(2, T, 1, n_overrelax); }

// src/MC.cpp:155-163
size_t MC_runner::sweep_local_Metropolis(double T, size_t n_overrelax) {
    return sweep_local_Metropolis_n(T, 1, n_overrelax);
}

// src/MC.cpp:145-153: one random-angle overrelaxation pass
void MC_runner::overrelax_all() {
    if (!ready_) throw std::logic_error("setup_lattice() has not been called");
    lat->to_device();
    check(pc_overrelax_all(lat->device()));
    lat->mark_device_newer();
}

// src/MC.cpp:305-312
double MC_runner::total_energy_per_unit_cell() const {
    if (!ready_) throw std::logic_error("setup_lattice() has not been called");
    lat->to_device();
    double e = 0;
    check(pc_energy(lat->device(), &e, nullptr));
    return e;
}

void write_geometry_group(OutFile& f, Lattice& sc, const char* group_name) {
    const std::string g = std::string("/") + group_name;
    const auto A = sc.lattice.get_lattice_vectors();
    const auto B = sc.lattice.get_reciprocal_lattice_vectors();
    int64_t a[9];
    double b[9];
    for (int i = 0; i < 9; ++i) {
        a[i] = A(i / 3, i % 3);
        b[i] = B(i / 3, i % 3);
    }
    f.dataset_i64(g + "/index_cell", {3, 3}, a);
    f.dataset_f64(g + "/recip_vectors", {3, 3}, b);
}

void save_spin_state(Lattice& lat, const std::filesystem::path& file_path) {
    const auto& spins = lat.get_objects<HeisenbergSpin>();
    const size_t N = spins.size();
    std::vector<int32_t> pos(3 * N);
    std::vector<double> ori(3 * N);
    for (size_t i = 0; i < N; ++i)
        for (int a = 0; a < 3; ++a) {
            pos[3 * i + size_t(a)] = int32_t(spins[i].ipos[a]);
            ori[3 * i + size_t(a)] = spins[i].S[a];
        }
    OutFile f(file_path.string());
    f.dataset_i32("spin_pos", {N, 3}, pos.data());
    f.dataset_f64("spin_orientation", {N, 3}, ori.data());
    f.close();
}

// save_ft_spin_state (src/MC.cpp:320-368): dataset "spin_ft" [3, n_sl, n_k, 2],
// the per-sublattice DFT over cells of each spin component without the
// sublattice phase, computed on the device (pc_spin_ft).
void save_ft_spin_state(Lattice& lat, const std::filesystem::path& file_path) {
    const uint64_t nk = uint64_t(lat.num_spins() / 16);
    std::vector<double> ft(size_t(3 * 16 * nk * 2));
    lat.to_device();
    check(pc_spin_ft(lat.device(), 0, ft.data()));
    OutFile f(file_path.string());
    f.dataset_f64("spin_ft", {3, 16, nk, 2}, ft.data());
    f.close();
}

}  // namespace CMC
