// Streams slices into a reserved dataset with OutFile for tests/test_host.py:
// /ssf/static_corr [2, 3, 4] reserved and committed, then the slices (c, t)
// for t = 0 and 2 written with values 100 c + 10 t + k. With argv[2] == "close"
// /ssf/T_list is added and the file closed; otherwise the process ends at once
// (std::_Exit, no destructors), as a run killed after its second flush would.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../pyro_cmc_b200/host/h5out.hpp"

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    CMC::OutFile f(argv[1]);
    const size_t h = f.reserve("/ssf/static_corr", "<f8", {2, 3, 4}, 8);
    f.commit();
    for (int t : {0, 2})
        for (int c = 0; c < 2; ++c) {
            double row[4];
            for (int k = 0; k < 4; ++k) row[k] = 100.0 * c + 10.0 * t + k;
            f.write_slice(h, uint64_t((c * 3 + t) * 4) * 8, row, sizeof row);
        }
    if (std::strcmp(argv[2], "close") == 0) {
        const double T[3] = {0.1, 0.2, 0.3};
        f.dataset_f64("/ssf/T_list", {3}, T);
        f.close();
        return 0;
    }
    std::_Exit(0);
}
