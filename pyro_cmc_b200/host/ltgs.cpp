// ltgs -- the Luttinger-Tisza ground-state bound of the reference's
// src/luttinger_tisza.cpp with the k sweep on the GPU (pc_lt_minimum): the
// same flags (provide_physical_args, --output_dir optional), the same printed
// lines, and the output tree eigenvalue_map, k_star_idx, k_star_vec, E_min,
// eigenvector [48, 2], /geometry/index_cell, /geometry/recip_vectors and the
// root attribute k_dims, in <name>ltgs.out.h5 (<name>ltgs.out.npz with --npz).
#include <cstdio>
#include <filesystem>
#include <iostream>
#include <vector>

#include "cli_bits.hpp"
#include "h5out.hpp"

using namespace CMC;

int main(int argc, char* argv[]) {
    ArgParser prog("ltgs");
    prog.flag({"--npz"}, "Write the output as NumPy .npz archives instead of HDF5 (.h5)");
    prog.option({"--output_dir", "-o"}, "Path to output directory");
    provide_physical_args(prog);
    try {
        prog.parse(argc, argv);
    } catch (const std::exception& err) {
        std::cerr << err.what() << "\n" << prog.usage();
        return 1;
    }
    try {
        const std::string ext = prog.boolean("--npz") ? ".npz" : ".h5";
        std::filesystem::path outdir;
        if (prog.is_used("--output_dir")) {
            outdir = prog.str("--output_dir");
            if (!std::filesystem::exists(outdir))
                throw std::runtime_error("output_dir does not exist: " + prog.str("--output_dir"));
        }
        const double J1 = prog.dbl("--J1"), J2 = prog.dbl("--J2"), J3 = resolve_J3(prog), Delta = prog.dbl("--Delta");
        const int L = int(prog.integer("L"));
        LatticeIndexing lat;
        lat.L = L;
        const int Nk = lat.num_primitive_cells();
        std::vector<double> lam(static_cast<size_t>(Nk)), vec(96);
        double E_per_spin = 0.0;
        int64_t ks[3] = {0, 0, 0};
        check(pc_lt_minimum(L, J1, J2, J3, Delta, lam.data(), &E_per_spin, ks, vec.data()));
        const double E_min = 2.0 * E_per_spin;
        const auto kv = lat.wavevector_from_idx3(ivec3_t(ks[0], ks[1], ks[2]));
        std::printf("LT minimum: \xce\xbb_min = %.6f  E/spin = %.6f\n", E_min, E_per_spin);
        std::printf("Eigvec sublattice |s_\xce\xb1|\xc2\xb2 :");
        for (int s = 0; s < 16; ++s) {
            double w = 0.0;
            for (int a = 0; a < 3; ++a) w += vec[size_t(2 * (3 * s + a))] * vec[size_t(2 * (3 * s + a))] +
                                             vec[size_t(2 * (3 * s + a) + 1)] * vec[size_t(2 * (3 * s + a) + 1)];
            std::printf(" %.4f", w);
        }
        std::printf("\n");
        std::printf("k*  idx = [%lld, %lld, %lld]\n", (long long)ks[0], (long long)ks[1], (long long)ks[2]);
        std::printf("k*  vec = [%.4f, %.4f, %.4f]  (rad / coord-unit)\n", kv[0], kv[1], kv[2]);
        if (!prog.is_used("--output_dir")) return 0;
        const auto file_path = outdir / (name_LJ123(prog) + "ltgs.out" + ext);
        OutFile f(file_path.string());
        f.dataset_f64("/eigenvalue_map", {uint64_t(Nk)}, lam.data());
        f.dataset_i64("/k_star_idx", {3}, ks);
        const double ksv[3] = {kv[0], kv[1], kv[2]};
        f.dataset_f64("/k_star_vec", {3}, ksv);
        f.dataset_f64("/E_min", {}, &E_per_spin);
        f.dataset_f64("/eigenvector", {48, 2}, vec.data());
        const auto A = lat.get_lattice_vectors();
        const auto Bm = lat.get_reciprocal_lattice_vectors();
        int64_t a9[9];
        double b9[9];
        for (int i = 0; i < 9; ++i) {
            a9[i] = A(i / 3, i % 3);
            b9[i] = Bm(i / 3, i % 3);
        }
        f.dataset_i64("/geometry/index_cell", {3, 3}, a9);
        f.dataset_f64("/geometry/recip_vectors", {3, 3}, b9);
        const int32_t kd[3] = {L, L, L};
        f.attribute("/", "k_dims", "<i4", {3}, kd, 4);
        f.close();
        std::cout << "Saved to " << file_path << "\n";
    } catch (const std::exception& e) {
        std::cerr << "ltgs: " << e.what() << "\n";
        return 1;
    }
    return 0;
}
