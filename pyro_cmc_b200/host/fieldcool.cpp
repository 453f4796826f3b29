// fieldcool -- anneal in a field, release the field at the final temperature,
// re-burn and sample S(q): the flow of the reference's src/fieldcool.cpp on
// the B200 engine. Output and seed differences as in anneal.cpp.
#include <cmath>
#include <cstdio>
#include <filesystem>
#include <iostream>

#include "cli_bits.hpp"
#include "h5out.hpp"
#include "managers.hpp"

using namespace CMC;

int main(int argc, char* argv[]) {
    ArgParser prog("fieldcool");
    prog.flag({"--npz"}, "Write the output as NumPy .npz archives instead of HDF5 (.h5)");
    prog.option({"--output_dir", "-o"}, "Path to output", "", true);
    prog.option({"--seed", "-s"}, "Seed of the RNG (Philox key)", "", true);
    prog.flag({"--save_state"}, "Also write the final spin configuration to .spins.h5 (.spins.npz with --npz)");
    prog.flag({"--init_spiral"}, "Pre-initialise spins to a spiral with the wavevector given by --Q (requires --Q)");
    prog.flag({"--init_uniform"}, "Start from spins uniform on the sphere (device Philox) instead of zero");
    prog.option({"--T_hot"}, "Temperature  to begin annealing from");
    prog.option({"--T_cold"}, "Final temperature", "", true);
    prog.option({"--T_ref"}, "Reference temperature for proposal distribution", "1.0");
    prog.option({"--n_steps"}, "Number of annealing steps", "100");
    prog.option({"--n_sweep", "-w"}, "Number of sweeps to run per temperature step", "16");
    prog.option({"--n_burn_in"}, "Number of sweeps to run at T_hot before we start annealing", "16");
    prog.option({"--n_sample"}, "Number of samples at T_cold", "64");
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
        if (!std::filesystem::exists(outdir)) throw std::runtime_error("Cannot open outdir");
        const uint64_t seed = uint64_t(prog.integer("--seed"));
        const double T_hot = prog.is_used("--T_hot") ? prog.dbl("--T_hot") : 10;
        const double T_cold = prog.dbl("--T_cold");
        const size_t n_steps = size_t(prog.integer("--n_steps"));
        const size_t n_sweep = size_t(prog.integer("--n_sweep"));
        const size_t n_burn_in = size_t(prog.integer("--n_burn_in"));
        const size_t n_sample = size_t(prog.integer("--n_sample"));
        double T = T_hot;
        auto lat = build_pyro_lat(prog);
        auto mc = build_J1J2J3_h(prog, lat, seed);
        if (prog.boolean("--init_uniform")) {
            check(pc_random_spins(lat.device(), seed ^ 0x5eedULL));
            lat.mark_device_newer();
        }
        if (prog.boolean("--init_spiral")) {
            if (!prog.is_used("--Q")) throw std::runtime_error("--init_spiral requires --Q");
            const double Q_rounded = round_Qz_to_supercell(prog.dbl("--Q"), int(prog.integer("L")));
            init_spiral_state(lat, Q_rounded, int(prog.integer("--spiral_axis")));
        }
        const auto B = prog.dbls("-B");
        std::stringstream name;
        name << prog.str("--prefix") << DELIM << name_LJ123(prog) << "B=" << B[0] << "," << B[1] << "," << B[2]
             << DELIM << "seed=" << seed << DELIM << "Tc=" << T_cold << DELIM;
        const double N = double(lat.num_spins());
        std::printf("Burning in (%zu sweeps)...\n", n_burn_in);
        mc.sweep_local_Metropolis_n(T_hot, n_burn_in);
        std::printf("Done. Begin anneal...\n");
        const double factor = std::pow(T_cold / T_hot, 1. / double(n_steps));  // src/fieldcool.cpp:154
        energy_manager e_manager;
        for (size_t i = 0; i < n_steps; i++) {
            e_manager.new_T(T);
            const size_t accepted = mc.sweep_local_Metropolis_n(T, n_sweep);
            e_manager.sample(mc.total_energy_per_unit_cell());
            std::printf("Iter %4zu T=%.3e E=%3e Acceptance rate: %.2f%%\n", i, T, e_manager.curr_E(),
                        accepted * 100.0 / N / double(n_sweep));
            T *= factor;
        }
        ssf_manager ssfm(lat, {"xx", "yy", "zz"}, 1);
        ssfm.new_T(T);
        std::printf("Releasing field and re-burning (%zu sweeps)...\n", n_burn_in);
        mc.set_global_field({0, 0, 0});
        mc.sweep_local_Metropolis_n(T, n_burn_in);
        std::printf("Sampling at T=%lf (%zu sweeps)...\n", T, n_sample);
        for (size_t i = 0; i < n_sample; i++) {
            const size_t accepted = mc.sweep_local_Metropolis_n(T, n_sweep);
            std::printf("[cold] Iter %4zu T=%.3e Acceptance rate: %.2f%%\n", i, T, accepted * 100.0 / N / double(n_sweep));
            ssfm.sample();
        }
        const auto file_path = outdir / (name.str() + ".out" + ext);
        OutFile file(file_path.string());
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
    } catch (const std::exception& e) {
        std::cerr << "fieldcool: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
