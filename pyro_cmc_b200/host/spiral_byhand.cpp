// spiral_byhand -- the deterministic spiral fixture of the reference's
// test/spiral_byhand.cpp on the B200 engine: J1 as one isotropic spec on the
// full nn1 table (default J1 = -1), S = (0, cos q.r, sin q.r) with
// q = wavevector_from_idx3(Q), one energy and one S(q) sample; writes the
// output tree and the spins.
#include <cmath>
#include <cstdio>
#include <filesystem>
#include <iostream>

#include "cli_bits.hpp"
#include "h5out.hpp"
#include "managers.hpp"

using namespace CMC;

int main(int argc, char* argv[]) {
    ArgParser prog("spiral_byhand");
    prog.flag({"--npz"}, "Write the output as NumPy .npz archives instead of HDF5 (.h5)");
    prog.option({"--output_dir", "-o"}, "Path to output", "", true);
    prog.positional("L", "Linear dimension of cubic supercell");
    prog.positional("Q", "Spiral wavevector index (3 integers)", 3);
    prog.option({"--J1"}, "Nearest-neighbour Heisenberg coupling strength", "-1.");
    prog.option({"--J2"}, "Second-nearest-neighbour Heisenberg coupling strength", "0.");
    prog.option({"--J3"}, "Third-nearest-neighbour Heisenberg coupling strength", "0.");
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
        const int L = int(prog.integer("L"));
        Lattice lat(L);
        MC_runner mc(lat, 0);
        using mat33d = vector3::mat33<double>;
        const mat33d I = mat33d::from_cols({1, 0, 0}, {0, 1, 0}, {0, 0, 1});
        mc.define_coupling("J1", pyro_table(1), prog.dbl("--J1") * I);
        mc.define_coupling("J2", pyro_table(2), prog.dbl("--J2") * I);
        mc.define_coupling("J3a", pyro_table(3), prog.dbl("--J3") * I);
        mc.define_coupling("J3b", pyro_table(4), prog.dbl("--J3") * I);
        mc.setup_lattice();
        const auto Qv = prog.ints("Q");
        const ivec3_t Q(Qv[0], Qv[1], Qv[2]);
        std::stringstream name;
        name << "L=" << L << DELIM << "Q=" << Q << DELIM;
        ssf_manager ssfm(lat, {"xx", "yy", "zz"}, 1);
        energy_manager e_manager;
        const auto q = lat.lattice.wavevector_from_idx3(Q);
        std::cout << "q = " << q << std::endl;
        for (auto& s : lat.get_objects<HeisenbergSpin>()) {
            const vector3::vec3d r(double(s.ipos[0]), double(s.ipos[1]), double(s.ipos[2]));
            const double phase = dot(q, r);
            s.S = vector3::vec3d(0, std::cos(phase), std::sin(phase));
        }
        ssfm.new_T(0);
        e_manager.new_T(0);
        const double total_E = mc.total_energy_per_unit_cell();
        ssfm.sample();
        e_manager.sample(total_E);
        std::cout << "Total E = " << total_E << std::endl;
        const auto file_path = outdir / (name.str() + ".out" + ext);
        OutFile file(file_path.string());
        ssfm.write_group(file, "/ssf");
        e_manager.write_group(file, "/energy");
        write_geometry_group(file, lat);
        file.close();
        std::cout << "Saved to \n" << file_path << std::endl;
        const auto f = outdir / (name.str() + ".spins" + ext);
        std::printf("Saving spin state to %s\n", f.string().c_str());
        save_spin_state(lat, f);
    } catch (const std::exception& e) {
        std::cerr << "spiral_byhand: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
