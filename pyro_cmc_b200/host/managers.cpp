// managers.cpp -- ssf_manager over the device S(q) accumulators.
#include "managers.hpp"

#include <algorithm>
#include <numeric>

namespace {
int axis_idx(char c) {
    if (c == 'x') return 0;
    if (c == 'y') return 1;
    if (c == 'z') return 2;
    throw std::invalid_argument(std::string("ssf_manager: unknown spin component '") + c + "'");
}
}  // namespace

void ssf_manager::configure(const std::vector<std::string>& names) {
    std::vector<const char*> ptrs;
    for (const auto& n : names) ptrs.push_back(n.c_str());
    const int32_t L = int32_t(sc_->lattice.L);
    CMC::check(pc_ssf_configure(sc_->device(), ptrs.data(), int(ptrs.size()), 1, &L));
    have_current_ = false;
}

ssf_manager::ssf_manager(CMC::Lattice& sc, const std::vector<std::string>& correlator_names, size_t,
                         bool store_error_term)
    : sc_(&sc),
      n_kpoints_(sc.lattice.num_primitive_cells()),
      n_spins_(int(sc.num_spins())),
      k_dims_(sc.lattice.size()),
      sl_positions_(sc.sl_positions),
      store_error_term_(store_error_term) {
    for (const auto& name : correlator_names) {  // include/ssf_manager.hpp:184-193
        if (name.size() != 2) throw std::invalid_argument("ssf_manager: correlator name must be 2 chars: " + name);
        corr_specs_.push_back({axis_idx(name[0]), axis_idx(name[1]), name});
    }
    configure(correlator_names);
}

ssf_manager::ssf_manager(CMC::Lattice& sc, const std::vector<std::string>& correlator_names, CMC::OutFile& file,
                         const char* group_name, const std::vector<double>& T_sample, bool store_error_term)
    : ssf_manager(sc, correlator_names, 0, store_error_term) {
    streaming_ = true;
    file_ = &file;
    group_ = group_name;
    T_sorted_ = T_sample;
    std::sort(T_sorted_.begin(), T_sorted_.end());
}

void ssf_manager::set_sublattice_resolved(bool on) {
    if (!T_list.empty()) throw std::logic_error("set_sublattice_resolved: call before the first new_T()");
    CMC::check(pc_ssf_set_resolved(sc_->device(), on ? 1 : 0));
    ew_ = on ? 512 : 2;
    configure(get_corr_labels());
}

std::vector<std::string> ssf_manager::get_corr_labels() const {
    std::vector<std::string> l;
    for (const auto& c : corr_specs_) l.push_back(c.label);
    return l;
}

void ssf_manager::on_new_temp() {
    CMC::check(pc_ssf_clear(sc_->device(), 0));
    have_current_ = true;
}

void ssf_manager::point_at(CMC::Lattice& sc2) {
    if (&sc2 == sc_) return;
    if (sc2.num_spins() != sc_->num_spins()) throw std::logic_error("point_at: lattices differ in size");
    // carry the current accumulators over to the new lattice's device
    std::vector<double> s, q;
    uint64_t n = 0;
    const bool carry = have_current_;
    if (carry) {
        s.resize(get_n_corr() * size_t(n_kpoints_) * ew_);
        q.resize(s.size());
        CMC::check(pc_ssf_read(sc_->device(), 0, s.data(), q.data(), &n));
    }
    sc_ = &sc2;
    CMC::check(pc_ssf_set_resolved(sc_->device(), ew_ == 512 ? 1 : 0));
    configure(get_corr_labels());
    if (carry) {
        // the accumulators restart on the new device; keep the old sums on the host
        auto& f = flushed_[size_t(-1)];
        if (f.first.empty()) {
            f.first.assign(s.size(), 0.0);
            f.second.assign(s.size(), 0.0);
        }
        for (size_t i = 0; i < s.size(); ++i) {
            f.first[i] += s[i];
            f.second[i] += q[i];
        }
        have_current_ = true;
    }
}

void ssf_manager::sample() {
    if (T_list.empty()) throw std::logic_error("ssf_manager::sample before new_T");
    if (!have_current_) throw std::logic_error("sample() called after flush() without new_T()");
    sc_->to_device();
    const int32_t slot = 0;
    CMC::check(pc_ssf_sample(sc_->device(), &slot));
    n_samples[curr_idx]++;
}

void ssf_manager::get_flat_buffer(size_t t_idx, std::vector<double>& corr_buf, std::vector<double>& corr_sq_buf) const {
    if (t_idx != curr_idx) throw std::logic_error("get_flat_buffer: t_idx must be the current temperature");
    const size_t n = get_n_corr() * size_t(n_kpoints_) * ew_;
    corr_buf.assign(n, 0.0);
    corr_sq_buf.assign(n, 0.0);
    uint64_t ns = 0;
    CMC::check(pc_ssf_read(sc_->device(), 0, corr_buf.data(), corr_sq_buf.data(), &ns));
    auto it = flushed_.find(size_t(-1));
    if (it != flushed_.end())
        for (size_t i = 0; i < n; ++i) {
            corr_buf[i] += it->second.first[i];
            corr_sq_buf[i] += it->second.second[i];
        }
    if (!store_error_term_) corr_sq_buf.clear();
}

// include/ssf_manager.hpp:375-405: static_corr[n_corr, n_T, n_k, 2] (or the
// sublattice-resolved [n_corr, n_T, n_k, 16, 16, 2]) reserved in full, zeros
// until a temperature is flushed into its slot.
void ssf_manager::reserve_streamed() {
    if (reserved_) return;
    const uint64_t nc = get_n_corr(), nT = T_sorted_.size(), nk = uint64_t(n_kpoints_);
    const std::vector<uint64_t> shape = ew_ == 512 ? std::vector<uint64_t>{nc, nT, nk, 16, 16, 2}
                                                   : std::vector<uint64_t>{nc, nT, nk, 2};
    h_sum_ = file_->reserve(group_ + "/static_corr", "<f8", shape, 8);
    if (store_error_term_) h_sq_ = file_->reserve(group_ + "/static_corr_2", "<f8", shape, 8);
    file_->commit();
    reserved_ = true;
}

// include/ssf_manager.hpp:413-465: write the current temperature into its slot
void ssf_manager::flush() {
    if (!streaming_) throw std::logic_error("flush() called on non-streaming ssf_manager");
    if (!have_current_) throw std::logic_error("flush() called with no accumulated data");
    const double T = T_list[curr_idx];
    auto it = std::find(T_sorted_.begin(), T_sorted_.end(), T);
    if (it == T_sorted_.end()) throw std::runtime_error("ssf_manager::flush: current temperature not found in T_sample");
    std::vector<double> s, q;
    get_flat_buffer(curr_idx, s, q);
    flushed_.erase(size_t(-1));
    reserve_streamed();
    const size_t slot = size_t(it - T_sorted_.begin()), nT = T_sorted_.size();
    const size_t row = size_t(n_kpoints_) * ew_;  // doubles per (correlator, temperature)
    for (size_t c = 0; c < get_n_corr(); ++c) {
        const uint64_t off = uint64_t((c * nT + slot) * row) * 8;
        file_->write_slice(h_sum_, off, s.data() + c * row, row * 8);
        if (store_error_term_) file_->write_slice(h_sq_, off, q.data() + c * row, row * 8);
    }
    have_current_ = false;
}

// include/ssf_manager.hpp:471-641: static_corr / static_corr_2
// [n_corr, n_T, n_k, 2], corr_lookup, T_list and n_samples sorted ascending,
// sl_positions [n_sl, 3] int64, attributes n_spins and k_dims.
void ssf_manager::write_group(CMC::OutFile& f, const char* group_name) {
    const std::string g = streaming_ ? group_ : std::string(group_name);
    if (streaming_ && have_current_ && !T_list.empty()) flush();
    const size_t n_T = T_list.size(), nc = get_n_corr(), nk = size_t(n_kpoints_);
    std::vector<size_t> ord(n_T);
    std::iota(ord.begin(), ord.end(), 0);
    std::sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return T_list[a] < T_list[b]; });
    const size_t n_T_out = streaming_ ? T_sorted_.size() : n_T;
    const size_t ew = ew_;
    if (streaming_) {
        // static_corr and static_corr_2 are already in the stream's file
        if (&f != file_) throw std::invalid_argument("ssf_manager::write_group: streaming writes into its own file");
        reserve_streamed();
    }
    std::vector<double> sum(streaming_ ? 0 : nc * n_T_out * nk * ew, 0.0), sq(sum.size(), 0.0);
    auto place = [&](size_t slot, const std::vector<double>& s, const std::vector<double>& q) {
        for (size_t c = 0; c < nc; ++c)
            for (size_t j = 0; j < nk * ew; ++j) {
                sum[(c * n_T_out + slot) * nk * ew + j] = s[c * nk * ew + j];
                if (!q.empty()) sq[(c * n_T_out + slot) * nk * ew + j] = q[c * nk * ew + j];
            }
    };
    if (!streaming_) {
        if (!T_list.empty()) {
            std::vector<double> s, q;
            get_flat_buffer(curr_idx, s, q);
            place(curr_idx, s, q);
        }
        const std::vector<uint64_t> shape = ew == 512 ? std::vector<uint64_t>{nc, n_T_out, nk, 16, 16, 2}
                                                      : std::vector<uint64_t>{nc, n_T_out, nk, 2};
        f.dataset_f64(g + "/static_corr", shape, sum.data());
        if (store_error_term_) f.dataset_f64(g + "/static_corr_2", shape, sq.data());
    }
    std::vector<double> sT;
    std::vector<uint64_t> sN;
    for (size_t i : ord) {
        sT.push_back(T_list[i]);
        sN.push_back(n_samples[i]);
    }
    f.dataset_f64(g + "/T_list", {uint64_t(sT.size())}, sT.data());
    f.dataset_u64(g + "/n_samples", {uint64_t(sN.size())}, sN.data());
    f.dataset_strings(g + "/corr_lookup", get_corr_labels());
    std::vector<int64_t> slp;
    for (const auto& p : sl_positions_)
        for (int a = 0; a < 3; ++a) slp.push_back(p[a]);
    f.dataset_i64(g + "/sl_positions", {uint64_t(sl_positions_.size()), 3}, slp.data());
    const int32_t ns = n_spins_;
    f.attribute(g, "n_spins", "<i4", {}, &ns, 4);
    const int32_t kd[3] = {int32_t(k_dims_[0]), int32_t(k_dims_[1]), int32_t(k_dims_[2])};
    f.attribute(g, "k_dims", "<i4", {3}, kd, 4);
}
