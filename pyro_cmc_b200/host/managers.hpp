// managers.hpp -- drop-ins for include/abstract_manager.hpp,
// include/energy_manager.hpp and include/ssf_manager.hpp on the B200 engine.
//
// abstract_manager and energy_manager are host bookkeeping, as in the
// reference. ssf_manager keeps the reference's interface (both constructors,
// new_T/set_T, sample, flush, write_group, point_at, get_flat_buffer and the
// getters, include/ssf_manager.hpp:161-309) while the transform and the FP64
// accumulation run on the device (pc_ssf_* in include/pyrocmc.h): one device
// slot holds the current temperature's sums, as the reference holds one
// temperature's accumulators at a time.
#pragma once

#include <cmath>
#include <cstddef>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "MC.hpp"
#include "h5out.hpp"

// include/abstract_manager.hpp:12-51
class abstract_manager {
protected:
    std::vector<double> T_list;
    std::vector<size_t> n_samples;
    size_t curr_idx = 0;
    virtual void on_new_temp() {}

public:
    virtual ~abstract_manager() = default;
    void new_T(double T) {
        curr_idx = T_list.size();
        T_list.push_back(T);
        n_samples.push_back(0);
        on_new_temp();
    }
    void set_T(double T, double tol = 1e-8) {
        for (size_t i = 0; i < T_list.size(); i++)
            if (std::abs(T_list[i] - T) < tol) {
                curr_idx = i;
                return;
            }
        new_T(T);
    }
    double curr_T() const { return T_list[curr_idx]; }
    virtual void write_group(CMC::OutFile& f, const char* group_name) = 0;
};

// include/energy_manager.hpp:19-115
class energy_manager : public abstract_manager {
    std::vector<double> E, E2;
    void on_new_temp() override {
        E.push_back(0);
        E2.push_back(0);
    }

public:
    explicit energy_manager(size_t n_temperatures_reserve = 0) {
        E.reserve(n_temperatures_reserve);
        E2.reserve(n_temperatures_reserve);
    }
    double curr_E() const { return E[curr_idx] / double(n_samples[curr_idx]); }
    void sample(double e) {
        if (T_list.empty()) throw std::logic_error("energy_manager::sample before new_T");
        E[curr_idx] += e;
        E2[curr_idx] += e * e;
        n_samples[curr_idx]++;
    }
    void write_group(CMC::OutFile& f, const char* group_name = "/energy") override {
        const std::string g = group_name;
        const uint64_t n = E.size();
        f.dataset_f64(g + "/E", {n}, E.data());
        f.dataset_f64(g + "/E2", {n}, E2.data());
        f.dataset_f64(g + "/T_list", {n}, T_list.data());
        std::vector<uint64_t> ns(n_samples.begin(), n_samples.end());
        f.dataset_u64(g + "/n_samples", {n}, ns.data());
    }
};

struct CorrSpec {
    int alpha, beta;
    std::string label;
};

class ssf_manager : public abstract_manager {
public:
    // Non-streaming (temper.cpp, fieldcool.cpp): write_group writes the
    // current temperature's data into its slot of [n_corr, n_T, n_k, 2].
    ssf_manager(CMC::Lattice& sc, const std::vector<std::string>& correlator_names,
                size_t n_temperatures_reserve = 0, bool store_error_term = true);
    // Streaming (anneal.cpp): one slot per T_sample value, sorted ascending;
    // flush() writes the current temperature into its slot of static_corr
    // (and static_corr_2) in `file`, reserved at the first flush in the
    // layout of the first call (include/ssf_manager.hpp:375-465), and keeps
    // no copy; write_group(file) then adds the remaining datasets.
    ssf_manager(CMC::Lattice& sc, const std::vector<std::string>& correlator_names, CMC::OutFile& file,
                const char* group_name, const std::vector<double>& T_sample, bool store_error_term = true);

    void point_at(CMC::Lattice& sc2);

    int get_n_sl() const { return 16; }
    int get_n_kpoints() const { return n_kpoints_; }
    ivec3_t get_k_dims() const { return k_dims_; }
    int get_n_spins() const { return n_spins_; }
    size_t get_n_corr() const { return corr_specs_.size(); }
    size_t get_n_samples_at(size_t t) const { return n_samples.at(t); }
    double get_T_at(size_t t) const { return T_list.at(t); }
    std::vector<std::string> get_corr_labels() const;
    const std::vector<ipos_t>& get_sl_positions() const { return sl_positions_; }

    // [n_corr, n_k, 2] of the current temperature (t_idx must be curr_idx)
    void get_flat_buffer(size_t t_idx, std::vector<double>& corr_buf, std::vector<double>& corr_sq_buf) const;

    void sample();
    void flush();
    void write_group(CMC::OutFile& f, const char* group_name = "/ssf") override;

    // Keep the sublattice-resolved correlator C_{mu nu}(k) (the layout
    // [n_corr, n_T, n_k, 16, 16, 2] of the reference's temper output) instead
    // of the contracted S(q). Call before the first new_T().
    void set_sublattice_resolved(bool on);
    bool sublattice_resolved() const { return ew_ == 512; }

private:
    CMC::Lattice* sc_;
    std::vector<CorrSpec> corr_specs_;
    int n_kpoints_, n_spins_;
    ivec3_t k_dims_;
    std::vector<ipos_t> sl_positions_;
    bool store_error_term_;
    bool streaming_ = false;
    CMC::OutFile* file_ = nullptr;
    bool reserved_ = false;
    size_t h_sum_ = 0, h_sq_ = 0;
    std::string group_;
    std::vector<double> T_sorted_;
    // slot size_t(-1): sums carried over by point_at for the current
    // temperature
    std::map<size_t, std::pair<std::vector<double>, std::vector<double>>> flushed_;
    bool have_current_ = false;
    size_t ew_ = 2;  // doubles per (correlator, k): 2, or 16*16*2 resolved

    void configure(const std::vector<std::string>& names);
    void reserve_streamed();
    void on_new_temp() override;
};
