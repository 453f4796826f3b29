// Writes a small output tree with OutFile for tests/test_host.py.
#include <cstdint>
#include <vector>

#include "../../pyro_cmc_b200/host/h5out.hpp"

int main(int argc, char** argv) {
    CMC::OutFile f(argv[1]);
    std::vector<double> a(2 * 3 * 4);
    for (size_t i = 0; i < a.size(); ++i) a[i] = 0.5 * double(i) - 3.0;
    f.dataset_f64("/ssf/static_corr", {2, 3, 4}, a.data());
    const int64_t m[9] = {8, 0, 0, 0, 8, 0, 0, 0, 8};
    f.dataset_i64("/geometry/index_cell", {3, 3}, m);
    const uint64_t n[2] = {7, 9};
    f.dataset_u64("/energy/n_samples", {2}, n);
    f.dataset_strings("/ssf/corr_lookup", {"xx", "yz", "z"});
    const int32_t ns = 1024;
    f.attribute("/ssf", "n_spins", "<i4", {}, &ns, 4);
    const int32_t kd[3] = {4, 4, 4};
    f.attribute("/ssf", "k_dims", "<i4", {3}, kd, 4);
    f.close();
    (void)argc;
    return 0;
}
