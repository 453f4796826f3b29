// cli_bits.hpp -- drop-in for the reference's include/cli_bits.hpp and
// include/format_bits.hpp: the same flags, defaults and helpers, over a small
// argument parser of this project (p-ranav argparse is not available).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <iostream>
#include <map>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "MC.hpp"

[[maybe_unused]] static const char* DELIM = "_";

// ---------------------------------------------------------------- parser
// Positional arguments and flags with one value, n values, at least one value
// ("+") or none (implicit booleans), with defaults and required flags.
class ArgParser {
public:
    explicit ArgParser(std::string prog) : prog_(std::move(prog)) {}

    struct Arg {
        std::vector<std::string> names;
        std::string help;
        std::string nargs = "1";  // "0" (flag), "1", "N", "+"
        int n = 1;
        bool required = false;
        bool positional = false;
        std::vector<std::string> defaults;
        std::vector<std::string> values;
        bool used = false;
    };

    ArgParser& positional(const std::string& name, const std::string& help, int n = 1) {
        Arg a;
        a.names = {name};
        a.help = help;
        a.positional = true;
        a.required = true;
        a.nargs = n == 1 ? "1" : "N";
        a.n = n;
        args_.push_back(a);
        return *this;
    }
    ArgParser& option(std::vector<std::string> names, const std::string& help, const std::string& def = "",
                      bool required = false, const std::string& nargs = "1", int n = 1) {
        Arg a;
        a.names = std::move(names);
        a.help = help;
        a.required = required;
        a.nargs = nargs;
        a.n = n;
        if (!def.empty()) {
            std::istringstream is(def);
            std::string t;
            while (is >> t) a.defaults.push_back(t);
        }
        args_.push_back(a);
        return *this;
    }
    ArgParser& flag(std::vector<std::string> names, const std::string& help) {
        Arg a;
        a.names = std::move(names);
        a.help = help;
        a.nargs = "0";
        a.n = 0;
        args_.push_back(a);
        return *this;
    }

    void parse(int argc, char** argv) {
        std::vector<std::string> tok(argv + 1, argv + argc);
        size_t i = 0;
        while (i < tok.size()) {
            const std::string& t = tok[i];
            if (t == "-h" || t == "--help") {
                std::cout << usage();
                std::exit(0);
            }
            Arg* a = is_option(t) ? find(t) : next_positional();
            if (!a) throw std::runtime_error("Unknown argument: " + t);
            if (!a->positional) ++i;
            a->used = true;
            a->values.clear();
            if (a->nargs == "0") continue;
            const size_t want = a->nargs == "+" ? size_t(-1) : size_t(a->n);
            while (i < tok.size() && a->values.size() < want && !(is_option(tok[i]) && !is_number(tok[i])))
                a->values.push_back(tok[i++]);
            if ((a->nargs == "+" && a->values.empty()) || (a->nargs != "+" && a->values.size() != want))
                throw std::runtime_error(a->names[0] + ": wrong number of values");
        }
        for (auto& a : args_)
            if (a.required && !a.used) throw std::runtime_error(a.names[0] + ": required argument missing");
    }

    bool is_used(const std::string& name) const { return get(name).used; }
    bool present(const std::string& name) const { return get(name).used || !get(name).defaults.empty(); }
    std::string str(const std::string& name) const { return vals(name).at(0); }
    double dbl(const std::string& name) const { return std::stod(str(name)); }
    long long integer(const std::string& name) const { return parse_int(str(name)); }
    bool boolean(const std::string& name) const { return get(name).used; }
    std::vector<double> dbls(const std::string& name) const {
        std::vector<double> r;
        for (const auto& v : vals(name)) r.push_back(std::stod(v));
        return r;
    }
    std::vector<long long> ints(const std::string& name) const {
        std::vector<long long> r;
        for (const auto& v : vals(name)) r.push_back(parse_int(v));
        return r;
    }
    std::vector<std::string> strs(const std::string& name) const { return vals(name); }

    std::string usage() const {
        std::ostringstream os;
        os << "usage: " << prog_ << "\n";
        for (const auto& a : args_) {
            os << "  ";
            for (size_t k = 0; k < a.names.size(); ++k) os << (k ? ", " : "") << a.names[k];
            os << "\t" << a.help;
            if (!a.defaults.empty()) {
                os << " [default:";
                for (const auto& d : a.defaults) os << " " << d;
                os << "]";
            }
            if (a.required) os << " [required]";
            os << "\n";
        }
        return os.str();
    }

private:
    std::string prog_;
    std::vector<Arg> args_;

    static bool is_number(const std::string& s) {
        if (s.empty()) return false;
        char* end = nullptr;
        std::strtod(s.c_str(), &end);
        return end && *end == '\0';
    }
    static bool is_option(const std::string& s) { return s.size() > 1 && s[0] == '-'; }
    static long long parse_int(const std::string& s) {
        // decimal, or hex with 0x (the README passes -s 0xdeadbeef)
        return std::stoll(s, nullptr, (s.size() > 2 && s[0] == '0' && (s[1] == 'x' || s[1] == 'X')) ? 16 : 10);
    }
    Arg* find(const std::string& t) {
        for (auto& a : args_)
            for (const auto& n : a.names)
                if (n == t) return &a;
        return nullptr;
    }
    Arg* next_positional() {
        for (auto& a : args_)
            if (a.positional && !a.used) return &a;
        return nullptr;
    }
    const Arg& get(const std::string& name) const {
        for (const auto& a : args_)
            for (const auto& n : a.names)
                if (n == name) return a;
        throw std::logic_error("no such argument: " + name);
    }
    std::vector<std::string> vals(const std::string& name) const {
        const Arg& a = get(name);
        if (a.used) return a.values;
        if (!a.defaults.empty()) return a.defaults;
        throw std::logic_error("No value provided for " + name);
    }
};

// ------------------------------------------------- include/cli_bits.hpp:28-74
inline void provide_physical_args(ArgParser& prog) {
    prog.positional("L", "Linear dimension of cubic supercell (e.g. L=2 has 2^3 *4 = 32 primitive cells)");
    prog.option({"--J1"}, "Nearest-neighbour Heisenberg coupling strength", "", true);
    prog.option({"--J2"}, "Second-nearest-neighbour Heisenberg coupling strength", "0");
    prog.option({"--J3"}, "Third-nearest-neighbour Heisenberg coupling strength (mutually exclusive with --Q)", "0");
    prog.option({"--K"}, "Biquadratic interaction strength", "0");
    prog.option({"--Q"}, "Nonzero spiral wavevector component in units of 2pi/a_cubic; J3 is set to minimise spiral "
                         "energy (mutually exclusive with --J3). Rounded to nearest supercell-commensurate value.");
    prog.option({"--spiral_axis", "-x"}, "Axis [0,1,2] (x,y,z) that the spiral wavevector --Q points along", "2");
    prog.option({"--Delta"}, "Nearest-neighbour XXZ anisotropy (local [111] frame): Jz = Delta*J1, Jperp = J1. "
                             "Delta=1 is isotropic Heisenberg.", "1.0");
    prog.option({"--external_field", "-B"}, "Global magnetic field", "0. 0. 0.", false, "N", 3);
}

// include/cli_bits.hpp:78-82
inline double J3_from_Qz(double J2, double Qz) {
    Qz *= 2 * M_PI / 8;
    return (-4 * J2 + 1. / std::cos(2 * Qz) - 2. * J2 / std::cos(2 * Qz)) / 8.;
}
// include/cli_bits.hpp:86-89
inline double round_Qz_to_supercell(double Qz, int L) {
    const double step = 1. / L;
    return std::round(Qz / step) * step;
}
// include/cli_bits.hpp:92-100
inline void warn_Qz_rounding(double Qz, double Qz_rounded) {
    const double diff = std::abs(Qz - Qz_rounded);
    const double tol = std::min(1e-10, 1e-3 * std::abs(Qz));
    if (diff > tol)
        std::fprintf(stderr, "WARNING: Qz=%.10g rounded to %.10g (diff=%.3e > tol=%.3e)\n", Qz, Qz_rounded, diff, tol);
}
// include/cli_bits.hpp:103-118
inline double resolve_J3(const ArgParser& prog) {
    const bool has_J3 = prog.is_used("--J3"), has_Q = prog.is_used("--Q");
    if (has_J3 && has_Q) throw std::runtime_error("--J3 and --Q are mutually exclusive");
    if (has_Q) {
        const int L = int(prog.integer("L"));
        const double Qz = round_Qz_to_supercell(prog.dbl("--Q"), L);
        const double J1 = prog.dbl("--J1");
        const double J2_eff = prog.dbl("--J2") / std::abs(J1);
        const double J3 = J3_from_Qz(J2_eff, Qz) * std::abs(J1);
        std::cout << "Calculated J3=" << J3 << std::endl;
        return J3;
    }
    return prog.dbl("--J3");
}

// include/cli_bits.hpp:129-134
inline CMC::Lattice build_pyro_lat(const ArgParser& prog) { return CMC::Lattice(int(prog.integer("L"))); }

// The pyrochlore displacement tables (include/pyrochlore_geometry.hpp:110-190),
// derived by the engine from the cell geometry.
inline std::vector<std::vector<ipos_t>> pyro_table(int kind) {
    std::vector<std::vector<ipos_t>> t(4);
    for (int p = 0; p < 4; ++p) {
        int64_t buf[3 * 64];
        int n = 0;
        CMC::check(pc_pyrochlore_displacements(kind, p, buf, 64, &n));
        for (int k = 0; k < n; ++k) t[size_t(p)].push_back(ipos_t(buf[3 * k], buf[3 * k + 1], buf[3 * k + 2]));
    }
    return t;
}
// nn1_pair_MN: J1 vectors of pair (mu, nu) from both ends
inline std::vector<std::vector<ipos_t>> nn1_pair(int mu, int nu) {
    std::vector<std::vector<ipos_t>> t(4);
    t[size_t(mu)] = pyro_table(10 + nu)[size_t(mu)];
    t[size_t(nu)] = pyro_table(10 + mu)[size_t(nu)];
    return t;
}

// include/cli_bits.hpp:144-207
inline CMC::MC_runner build_J1J2J3_h(const ArgParser& prog, CMC::Lattice& lat, uint64_t seed) {
    vector3::vec3d global_field;
    {
        const auto B = prog.dbls("-B");
        for (int i = 0; i < 3; i++) global_field[i] = B[size_t(i)];
    }
    const double J1 = prog.dbl("--J1"), J2 = prog.dbl("--J2");
    const double J3 = resolve_J3(prog);
    if (prog.is_used("--Q")) {
        const int L = int(prog.integer("L"));
        const double Qz = prog.dbl("--Q");
        const double Qz_rounded = round_Qz_to_supercell(Qz, L);
        warn_Qz_rounding(Qz, Qz_rounded);
        std::printf("Using Q=%.10g along axis %lld -> J3=%.10g\n", Qz_rounded, prog.integer("--spiral_axis"), J3);
    }
    const double Delta = prog.dbl("--Delta");
    // the seed is used as the Philox key directly (no seed-table lookup)
    CMC::MC_runner mc(lat, seed);
    using mat33d = vector3::mat33<double>;
    const mat33d I = mat33d::from_cols({1, 0, 0}, {0, 1, 0}, {0, 0, 1});
    static const int pairs[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
    for (auto& pr : pairs) {
        const int mu = pr[0], nu = pr[1];
        // J_spec = J1 [I + (Delta - 1) z_mu (x) z_nu], z_p = link[p]/sqrt(3)
        mat33d M = I;
        const int64_t link[4][3] = {{1, 1, 1}, {1, -1, -1}, {-1, 1, -1}, {-1, -1, 1}};
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) M(a, b) += (Delta - 1) * double(link[mu][a] * link[nu][b]) / 3.0;
        mc.define_coupling("J1_" + std::to_string(mu) + std::to_string(nu), nn1_pair(mu, nu), J1 * M);
    }
    mc.define_coupling("J2", pyro_table(2), J2 * I);
    mc.define_coupling("J3a", pyro_table(3), J3 * I);
    mc.define_coupling("J3b", pyro_table(4), J3 * I);
    mc.set_global_field(global_field);
    mc.settings.T_ref = prog.dbl("--T_ref");
    mc.setup_lattice();
    return mc;
}

// include/cli_bits.hpp:211-222
inline void init_spiral_state(CMC::Lattice& lat, double Q_rounded, int axis) {
    constexpr double a_cubic = 8.;
    const int idx_sin = (axis + 1) % 3, idx_cos = (axis + 2) % 3;
    for (auto& s : lat.get_objects<CMC::HeisenbergSpin>()) {
        const double phase = Q_rounded * 2 * M_PI * static_cast<double>(s.ipos[axis]) / a_cubic;
        vector3::vec3d S(0., 0., 0.);
        S[idx_cos] = std::cos(phase);
        S[idx_sin] = std::sin(phase);
        s.S = S;
    }
}

// include/cli_bits.hpp:224-245
inline std::string name_LJ123(const ArgParser& prog) {
    const double J1 = prog.dbl("--J1"), J2 = prog.dbl("--J2");
    const double J3 = resolve_J3(prog);
    const double Delta = prog.dbl("--Delta");
    const long long L = prog.integer("L");
    std::stringstream name;
    name << "L=" << L << DELIM << "J1=" << J1 << DELIM << "J2=" << J2 << DELIM << "J3=" << J3 << DELIM
         << "Delta=" << Delta << DELIM;
    if (prog.is_used("--Q")) {
        const double Qz_rounded = round_Qz_to_supercell(prog.dbl("--Q"), int(L));
        name << "Q=" << Qz_rounded << DELIM;
        const long long axis = prog.integer("--spiral_axis");
        if (axis != 2) name << "spiral_axis=" << axis << DELIM;
    }
    return name.str();
}

// include/cli_bits.hpp:250-289
inline std::pair<std::vector<double>, std::set<size_t>> generate_T_profile(double T_hot, double T_cold,
                                                                          std::vector<double> T_sample,
                                                                          size_t total_steps) {
    std::vector<double> T_sweep, T;
    const double factor = std::pow(T_cold / T_hot, 1. / double(total_steps));
    double t = T_hot / factor;
    for (size_t i = 0; i < total_steps; i++) {
        t *= factor;
        T_sweep.push_back(t);
    }
    std::sort(T_sweep.begin(), T_sweep.end(), [](double a, double b) { return a > b; });
    std::sort(T_sample.begin(), T_sample.end(), [](double a, double b) { return a > b; });
    size_t i_samp = 0, i_sw = 0;
    std::set<size_t> idx;
    while (i_sw < T_sweep.size() && i_samp < T_sample.size()) {
        if (T_sweep[i_sw] > T_sample[i_samp]) {
            T.push_back(T_sweep[i_sw]);
            i_sw++;
        } else {
            idx.insert(T.size());
            T.push_back(T_sample[i_samp]);
            i_samp++;
        }
    }
    for (; i_samp < T_sample.size(); i_samp++) {
        idx.insert(T.size());
        T.push_back(T_sample[i_samp]);
    }
    for (; i_sw < T_sweep.size(); i_sw++) T.push_back(T_sweep[i_sw]);
    return {T, idx};
}
