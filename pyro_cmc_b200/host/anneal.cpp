// anneal -- simulated annealing on the B200 engine; the flags, schedule,
// console lines and output tree of the reference's src/anneal.cpp.
//
// Differences from the reference, all deliberate:
//  * the output <name>.out.h5 (/ssf, /energy, /geometry) is written by this
//    package's own HDF5 writer (h5file.hpp); --npz writes the same tree as
//    <name>.out.npz;
//  * --seed is the Philox key itself, not an index into a seed table;
//  * --save_state writes the spins (.spins.h5) and --save_state_ft the
//    per-sublattice spin DFT (.spindft.h5) as the README documents (the
//    reference swaps the two flags);
//  * additions: --init_uniform (start uniform on S^2 instead of the
//    default-constructed zero spins), --correlators (default: the reference's
//    six), --dry_run (print the run name and temperature grid and exit).
#include <algorithm>
#include <cstdio>
#include <filesystem>
#include <iostream>

#include "cli_bits.hpp"
#include "h5out.hpp"
#include "managers.hpp"

using namespace CMC;

int main(int argc, char* argv[]) {
    ArgParser prog("anneal");
    prog.flag({"--npz"}, "Write the output as NumPy .npz archives instead of HDF5 (.h5)");
    prog.option({"--output_dir", "-o"}, "Path to output", "", true);
    prog.option({"--seed", "-s"}, "Seed of the RNG (Philox key)", "", true);
    prog.flag({"--save_state"}, "Also write the final spin configuration to .spins.h5 (.spins.npz with --npz)");
    prog.flag({"--save_state_ft"}, "Also write the sublattice-resolved spin DFT to .spindft.h5 (.spindft.npz with --npz)");
    prog.flag({"--init_spiral"}, "Pre-initialise spins to a spiral with the wavevector given by --Q (requires --Q)");
    prog.flag({"--init_uniform"}, "Start from spins uniform on the sphere (device Philox) instead of zero");
    prog.option({"--T_hot"}, "Temperature  to begin annealing from");
    prog.option({"--T_cold"}, "Minimum temperature (defaults ti smallest T_sample)");
    prog.option({"--T_ref"}, "Reference temperature for proposal distribution", "1.0");
    prog.option({"--T_sample"}, "Final temperature", "", true, "+");
    prog.option({"--n_steps"}, "Number of annealing steps", "100");
    prog.option({"--n_sweep", "-w"}, "Number of sweeps to run per temperatur step", "16");
    prog.option({"--n_burn_in"}, "Number of sweeps to run at T_hot before we start annealing", "16");
    prog.option({"--n_sample"}, "Number of sweeps to run at T_cold while collecting statistics", "64");
    prog.option({"--prefix"}, "", "run");
    prog.flag({"--lifted"}, "Use lifted Metropolis (flip direction on rejection) instead of standard Metropolis");
    prog.option({"--correlators"}, "S(q) correlators", "xx yy zz xy xz yz", false, "+");
    prog.flag({"--dry_run"}, "Print the run name and temperature grid and exit");
    prog.flag({"--ssf_resolved"}, "Write /ssf sublattice-resolved, [n_corr, n_T, n_k, n_sl, n_sl, 2]");
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
        if (!std::filesystem::exists(outdir)) throw std::runtime_error("Cannot open outdir");
        const uint64_t seed = uint64_t(prog.integer("--seed"));
        const double T_hot = prog.is_used("--T_hot") ? prog.dbl("--T_hot") : 10;
        const std::vector<double> T_sample = prog.dbls("--T_sample");
        const double T_cold = prog.is_used("--T_cold") ? prog.dbl("--T_cold")
                                                       : *std::min_element(T_sample.begin(), T_sample.end());
        const size_t n_steps = size_t(prog.integer("--n_steps"));
        const size_t n_sweep = size_t(prog.integer("--n_sweep"));
        const size_t n_burn_in = size_t(prog.integer("--n_burn_in"));
        const size_t n_sample = size_t(prog.integer("--n_sample"));
        const auto B = prog.dbls("-B");
        if (B.size() < 3) throw std::runtime_error("--B requires 3 arguments");
        std::stringstream name;
        name << prog.str("--prefix") << DELIM << name_LJ123(prog) << "B=" << B[0] << "," << B[1] << "," << B[2]
             << DELIM << "seed=" << seed << DELIM << "Tc=" << T_cold << DELIM << "sw=" << n_sweep << DELIM;
        auto [T_grid, S_idx] = generate_T_profile(T_hot, T_cold, T_sample, n_steps);
        if (prog.boolean("--dry_run")) {
            std::cout << name.str() << "\n";
            for (size_t i = 0; i < T_grid.size(); ++i)
                std::printf("%zu %.17g %d\n", i, T_grid[i], S_idx.count(i) ? 1 : 0);
            return 0;
        }

        auto lat = build_pyro_lat(prog);
        auto mc = build_J1J2J3_h(prog, lat, seed);
        if (prog.boolean("--init_uniform")) {
            check(pc_random_spins(lat.device(), seed ^ 0x5eedULL));
            lat.mark_device_newer();
        }
        if (prog.boolean("--init_spiral")) {
            if (!prog.is_used("--Q")) throw std::runtime_error("--init_spiral requires --Q");
            const double Q_rounded = round_Qz_to_supercell(prog.dbl("--Q"), int(prog.integer("L")));
            const int spiral_axis = int(prog.integer("--spiral_axis"));
            std::printf("Pre-initialising to spiral order (Q=%.10g, axis=%d)...\n", Q_rounded, spiral_axis);
            init_spiral_state(lat, Q_rounded, spiral_axis);
        }
        energy_manager e_manager;
        const auto file_path = outdir / (name.str() + ".out" + ext);
        OutFile file(file_path.string());
        ssf_manager ssfm(lat, prog.strs("--correlators"), file, "/ssf", T_sample, true);
        if (prog.boolean("--ssf_resolved")) ssfm.set_sublattice_resolved(true);
        const double N = double(lat.num_spins());

        // src/anneal.cpp:184-188: --lifted swaps the single-site move
        const int update = prog.boolean("--lifted") ? 1 : 0;
        std::printf("Done. Begin anneal%s...\n", update ? " (lifted Metropolis)" : "");
        std::printf("Burning in (%zu sweeps)...\n", n_burn_in);
        mc.sweep_n(update, T_hot, n_burn_in);
        for (size_t i = 0; i < T_grid.size(); ++i) {
            const double T = T_grid[i];
            e_manager.new_T(T);
            const size_t accepted = mc.sweep_n(update, T, n_sweep);
            e_manager.sample(mc.total_energy_per_unit_cell());
            if (S_idx.count(i)) {
                std::printf("Sampling at T=%lf (%zu sweeps)...\n", T, n_sample);
                ssfm.new_T(T);
                for (size_t k = 0; k < n_sample; k++) {
                    const size_t accepted_ssf = mc.sweep_n(update, T, n_sweep);
                    std::printf("[ssf] Iter %4zu T=%.3e Acceptance rate: %.2f%%\n", k, T,
                                accepted_ssf * 100.0 / N / double(n_sweep));
                    ssfm.sample();
                }
                ssfm.flush();
            }
            std::printf("[anneal] Iter %4zu T=%.3e E=%3e Acceptance rate: %.2f%%\n", i, T, e_manager.curr_E(),
                        accepted * 100.0 / N / double(n_sweep));
        }
        ssfm.write_group(file, "/ssf");
        e_manager.write_group(file, "/energy");
        write_geometry_group(file, lat);
        file.close();
        std::cout << "Saved to \n" << file_path << std::endl;
        if (prog.boolean("--save_state")) {
            const auto f = outdir / (name.str() + ".spins" + ext);
            std::printf("Saving spin state to %s\n", f.string().c_str());
            save_spin_state(lat, f);
        }
        if (prog.boolean("--save_state_ft")) {
            const auto f = outdir / (name.str() + ".spindft" + ext);
            std::printf("Saving spin state FT to %s\n", f.string().c_str());
            save_ft_spin_state(lat, f);
        }
    } catch (const std::exception& e) {
        std::cerr << "anneal: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
