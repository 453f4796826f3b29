// temper -- parallel tempering with every replica resident on one GPU: the
// flags, temperature ladder and output tree of the reference's
// src/temper.cpp, with the MPI ranks replaced by batched replicas and the
// exchange decided on the device (pc_pt_*, include/pyrocmc.h).
//
//  * --n_replicas N replaces the MPI world size (one replica per rung);
//  * a round is n_sweep sweeps, an S(q) sample (xx, yy, zz) at every rung,
//    one energy sample per rung, then the checkerboard exchange
//    (temper.cpp:418-474); the reference's extra sweep on non-sampled ranks
//    (:426-429), a load-balancing device, is not reproduced;
//  * /ssf holds the rungs of --T_sample in the contracted layout
//    [n_corr, n_T, n_k, 2] that ssf_manager produces, or with --ssf_resolved
//    the sublattice-resolved layout [n_corr, n_T, n_k, 16, 16, 2] that the
//    reference's write_ssf_group (temper.cpp:121-159) is written for;
//  * output is <name>.out.h5 (<name>.out.npz with --npz); --seed is the Philox key.
#include <algorithm>
#include <cstdio>
#include <filesystem>
#include <iostream>
#include <numeric>

#include "cli_bits.hpp"
#include "h5out.hpp"
#include "managers.hpp"

using namespace CMC;

int main(int argc, char* argv[]) {
    ArgParser prog("temper");
    prog.flag({"--npz"}, "Write the output as NumPy .npz archives instead of HDF5 (.h5)");
    prog.option({"--output_dir", "-o"}, "Path to output", "", true);
    prog.option({"--seed", "-s"}, "Seed of the RNG (Philox key)", "", true);
    prog.option({"--n_replicas"}, "Number of replicas (rungs), one per temperature", "", true);
    prog.flag({"--save_state"}, "Save the spin state of the coldest replica");
    prog.flag({"--init_uniform"}, "Start from spins uniform on the sphere (device Philox) instead of zero");
    prog.flag({"--ssf_resolved"}, "Write /ssf sublattice-resolved, [n_corr, n_T, n_k, n_sl, n_sl, 2]");
    prog.option({"--T_hot"}, "Temperature of the hottest replica");
    prog.option({"--T_cold"}, "Temperature of the coldest replica (defaults to min(T_sample))");
    prog.option({"--T_ref"}, "Reference temperature for proposal distribution", "1.0");
    prog.option({"--T_sample"}, "Temperatures at which to accumulate the SSF", "", true, "+");
    prog.option({"--n_sweep", "-w"}, "Local-update sweeps per replica between exchange attempts", "16");
    prog.option({"--n_burn_in"}, "Sweeps at fixed T before exchange attempts begin", "16");
    prog.option({"--n_sample"}, "Number of exchange rounds while collecting statistics", "64");
    prog.option({"--prefix"}, "", "run");
    provide_physical_args(prog);
    try {
        prog.parse(argc, argv);
    } catch (const std::exception& err) {
        std::cerr << err.what() << std::endl << prog.usage();
        std::exit(1);
    }
    try {
        const std::string ext = prog.boolean("--npz") ? ".npz" : ".h5";
        const std::filesystem::path outdir(prog.str("--output_dir"));
        if (!std::filesystem::exists(outdir)) throw std::runtime_error("output_dir does not exist");
        const uint64_t seed = uint64_t(prog.integer("--seed"));
        const int R = int(prog.integer("--n_replicas"));
        const double T_hot = prog.is_used("--T_hot") ? prog.dbl("--T_hot") : 10.0;
        const std::vector<double> T_sample = prog.dbls("--T_sample");
        const double T_cold =
            prog.is_used("--T_cold") ? prog.dbl("--T_cold") : *std::min_element(T_sample.begin(), T_sample.end());
        const int n_sweep = int(prog.integer("--n_sweep"));
        const int n_burn_in = int(prog.integer("--n_burn_in"));
        const int n_sample = int(prog.integer("--n_sample"));
        if (R <= int(T_sample.size())) throw std::runtime_error("n_replicas must exceed T_sample count");
        if (R < 2) throw std::runtime_error("need at least 2 replicas");
        auto [T_grid, S_idx] = generate_T_profile(T_hot, T_cold, T_sample, size_t(R) - T_sample.size());
        const int L = int(prog.integer("L"));
        const auto B = prog.dbls("-B");
        std::stringstream name;
        name << prog.str("--prefix") << DELIM << name_LJ123(prog) << "B=" << B[0] << "," << B[1] << "," << B[2]
             << DELIM << "seed=" << seed << DELIM << "Tc=" << T_cold << DELIM << "sw=" << n_sweep << DELIM;

        // one MC_runner's couplings, replayed onto an R-replica system
        Lattice proto(L);
        auto mc = build_J1J2J3_h(prog, proto, seed);
        std::vector<int32_t> Ls(size_t(R), L);
        pc_system* sys = nullptr;
        check(pc_create(R, Ls.data(), seed, &sys));
        for (const auto& c : mc.couplings()) {
            std::vector<int64_t> rv;
            int32_t n[4] = {0, 0, 0, 0};
            for (int p = 0; p < 4; ++p) {
                n[p] = int32_t(c.relative_vectors[size_t(p)].size());
                for (const auto& v : c.relative_vectors[size_t(p)])
                    for (int a = 0; a < 3; ++a) rv.push_back(v[a]);
            }
            check(pc_define_coupling(sys, c.name.c_str(), rv.data(), n, c.J.m.data()));
        }
        check(pc_set_global_field(sys, B.data()));
        check(pc_set_T_ref(sys, prog.dbl("--T_ref")));
        check(pc_setup_lattice(sys));
        if (prog.boolean("--init_uniform")) check(pc_random_spins(sys, seed ^ 0x5eedULL));
        const char* corr[3] = {"xx", "yy", "zz"};
        std::vector<int32_t> L_of_slot(size_t(R), L);
        const bool resolved = prog.boolean("--ssf_resolved");
        const size_t ew = resolved ? 512 : 2;  // doubles per (correlator, k)
        check(pc_ssf_set_resolved(sys, resolved ? 1 : 0));
        check(pc_ssf_configure(sys, corr, 3, R, L_of_slot.data()));

        std::printf("[temper] Burning in %d replicas (%d sweeps each)...\n", R, n_burn_in);
        check(pc_sweep(sys, T_grid.data(), n_burn_in, 1, nullptr));
        check(pc_pt_configure(sys, T_grid.data()));
        std::printf("[temper] Begin sampling (%d rungs, %zu sampled, %d rounds)...\n", R, S_idx.size(), n_sample);
        check(pc_pt_run(sys, n_sample, n_sweep, n_sweep));

        std::vector<uint64_t> att(static_cast<size_t>(R)), acc(static_cast<size_t>(R));
        check(pc_pt_read_exchange(sys, att.data(), acc.data()));
        std::printf("\n[temper] per-pair swap acceptance:\n");
        for (int a = 0; a + 1 < R; a++)
            std::printf("  pair %3d<->%3d  T=%.4e <-> %.4e  accept=%5.1f%%  (%llu/%llu)\n", a, a + 1, T_grid[size_t(a)],
                        T_grid[size_t(a) + 1], att[size_t(a)] ? 100.0 * double(acc[size_t(a)]) / double(att[size_t(a)]) : 0.0,
                        (unsigned long long)acc[size_t(a)], (unsigned long long)att[size_t(a)]);

        // /energy, ascending in T (temper.cpp:571-580)
        std::vector<double> Ts(static_cast<size_t>(R)), E(static_cast<size_t>(R)), E2(static_cast<size_t>(R));
        std::vector<uint64_t> ne(static_cast<size_t>(R));
        check(pc_pt_read_energy(sys, Ts.data(), E.data(), E2.data(), ne.data()));
        std::vector<double> eT, eE, eE2;
        std::vector<uint64_t> en;
        for (int k = R - 1; k >= 0; --k) {
            eT.push_back(Ts[size_t(k)]);
            eE.push_back(E[size_t(k)]);
            eE2.push_back(E2[size_t(k)]);
            en.push_back(ne[size_t(k)]);
        }
        const auto file_path = outdir / (name.str() + ".out" + ext);
        OutFile file(file_path.string());
        const uint64_t nR = uint64_t(R);
        file.dataset_f64("/energy/T_list", {nR}, eT.data());
        file.dataset_f64("/energy/E", {nR}, eE.data());
        file.dataset_f64("/energy/E2", {nR}, eE2.data());
        file.dataset_u64("/energy/n_samples", {nR}, en.data());

        // /ssf: the sampled rungs, ascending in T
        std::vector<size_t> rungs(S_idx.begin(), S_idx.end());
        std::sort(rungs.begin(), rungs.end(), [&](size_t a, size_t b) { return T_grid[a] < T_grid[b]; });
        const size_t nk = size_t(L) * L * L, nT = rungs.size();
        std::vector<double> sum(3 * nT * nk * ew), sq(sum.size()), st;
        std::vector<uint64_t> sn;
        for (size_t t = 0; t < nT; ++t) {
            std::vector<double> s(3 * nk * ew), q(3 * nk * ew);
            uint64_t n = 0;
            check(pc_ssf_read(sys, int(rungs[t]), s.data(), q.data(), &n));
            for (size_t c = 0; c < 3; ++c)
                for (size_t j = 0; j < nk * ew; ++j) {
                    sum[(c * nT + t) * nk * ew + j] = s[c * nk * ew + j];
                    sq[(c * nT + t) * nk * ew + j] = q[c * nk * ew + j];
                }
            st.push_back(T_grid[rungs[t]]);
            sn.push_back(n);
        }
        const std::vector<uint64_t> shape =
            resolved ? std::vector<uint64_t>{3, nT, nk, 16, 16, 2} : std::vector<uint64_t>{3, nT, nk, 2};
        file.dataset_f64("/ssf/static_corr", shape, sum.data());
        file.dataset_f64("/ssf/static_corr_2", shape, sq.data());
        file.dataset_f64("/ssf/T_list", {nT}, st.data());
        file.dataset_u64("/ssf/n_samples", {nT}, sn.data());
        file.dataset_strings("/ssf/corr_lookup", {"xx", "yy", "zz"});
        std::vector<int64_t> slp;
        for (const auto& p : proto.sl_positions)
            for (int a = 0; a < 3; ++a) slp.push_back(p[a]);
        file.dataset_i64("/ssf/sl_positions", {16, 3}, slp.data());
        const int32_t n_spins = 16 * L * L * L;
        file.attribute("/ssf", "n_spins", "<i4", {}, &n_spins, 4);
        const int32_t kd[3] = {L, L, L};
        file.attribute("/ssf", "k_dims", "<i4", {3}, kd, 4);
        write_geometry_group(file, proto);
        file.close();
        std::printf("[temper] Saved to %s\n", file_path.string().c_str());

        if (prog.boolean("--save_state")) {
            // the replica currently at the coldest rung
            std::vector<int32_t> slot(static_cast<size_t>(R));
            check(pc_pt_slots(sys, slot.data()));
            const int cold = int(std::find(slot.begin(), slot.end(), R - 1) - slot.begin());
            std::vector<double> S(size_t(n_spins) * 3);
            check(pc_get_spins(sys, cold, S.data()));
            auto& spins = proto.get_objects<HeisenbergSpin>();
            for (size_t i = 0; i < spins.size(); ++i)
                for (int a = 0; a < 3; ++a) spins[i].S[a] = S[3 * i + size_t(a)];
            const auto f = outdir / (name.str() + ".spins" + ext);
            std::printf("[temper] Saving spin state of coldest replica (T=%.3e) to %s\n", T_grid.back(),
                        f.string().c_str());
            save_spin_state(proto, f);
        }
        pc_destroy(sys);
    } catch (const std::exception& e) {
        std::cerr << "temper: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
