// Driver for oracle/make_ref.sh: prints draws of the reference's own
// XoshiroCpp::Xoroshiro128PlusPlus (include/XoshiroCpp.hpp:351-362), seeded the
// way MC_runner seeds it (include/MC.hpp:107-112, rng(seed)), through the same
// libstdc++ distributions MC_runner uses (include/MC.hpp:95-98).
// Output (one line per draw): "<seed> <kind> <index> <value>", kind 0 = raw
// uint64 (decimal), 1 = normal_distribution<double>, 2 = uniform [0,1).
#include <XoshiroCpp.hpp>
#include <cstdint>
#include <cstdio>
#include <random>

int main() {
    const std::uint64_t seeds[] = {0ull, 1ull, 42ull, 0xdeadbeefull, 0x72b123beull, 18446744073709551615ull};
    for (std::uint64_t seed : seeds) {
        {
            XoshiroCpp::Xoroshiro128PlusPlus g(seed);
            for (int i = 0; i < 16; ++i) std::printf("%llu 0 %d %llu\n", (unsigned long long)seed, i, (unsigned long long)g());
        }
        {
            XoshiroCpp::Xoroshiro128PlusPlus g(seed);
            std::normal_distribution<double> nd;
            for (int i = 0; i < 16; ++i) std::printf("%llu 1 %d %.17g\n", (unsigned long long)seed, i, nd(g));
        }
        {
            XoshiroCpp::Xoroshiro128PlusPlus g(seed);
            std::uniform_real_distribution<double> ud(0.0, 1.0);
            for (int i = 0; i < 16; ++i) std::printf("%llu 2 %d %.17g\n", (unsigned long long)seed, i, ud(g));
        }
    }
    return 0;
}
