// Edge cases of the HDF5 writer for tests/test_host.py: an empty string
// dataset, an attribute on a dataset, nested groups created implicitly, a
// scalar dataset, a 0-length dataset, and a dataset written after a commit.
#include <cstdint>
#include <vector>

#include "../../pyro_cmc_b200/host/h5out.hpp"

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    CMC::OutFile f(argv[1]);
    f.dataset_strings("/a/b/c/empty", {});
    const double v[4] = {1.5, -2.0, 3.25, 0.0};
    f.dataset_f64("/a/b/vec", {4}, v);
    const int32_t k = 7;
    f.attribute("/a/b/vec", "k", "<i4", {}, &k, 4);
    const double s = 42.0;
    f.dataset_f64("/scalar", {}, &s);
    f.dataset_f64("/a/none", {0}, nullptr);
    f.commit();
    const int64_t late[2] = {-1, 1};
    f.dataset_i64("/a/b/c/late", {2}, late);
    f.close();
    return 0;
}
