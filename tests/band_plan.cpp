// Prints the band plan of md_b200/csrc/bands.hpp as JSON for tests/test_bands.py:
//   band_plan P K0 ncx Lx skin
// {"first": [...], "win_lo": [...], "win_n": [...], "W": [[...], ...],
//  "halo": [{"send": [...], "recv": [...], "local": [...], "send_n": [...], "recv_n": [...], "rng": [[a, n], [b, m]]}, ...]}
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "bands.hpp"

template <typename T>
static void list(const std::vector<T>& v)
{
    std::printf("[");
    for (size_t i = 0; i < v.size(); ++i) std::printf(i ? ", %lld" : "%lld", (long long)v[i]);
    std::printf("]");
}

int main(int argc, char** argv)
{
    if (argc != 6) {
        std::fprintf(stderr, "usage: band_plan P K0 ncx Lx skin\n");
        return 2;
    }
    const int P = std::atoi(argv[1]), K0 = std::atoi(argv[2]), ncx = std::atoi(argv[3]);
    const double Lx = std::atof(argv[4]), skin = std::atof(argv[5]);
    const mdf::BandPlan B = mdf::plan_bands(P, K0, ncx, Lx, skin);
    std::printf("{\"first\": ");
    list(B.first);
    std::printf(", \"win_lo\": ");
    list(B.win_lo);
    std::printf(", \"win_n\": ");
    list(B.win_n);
    std::printf(", \"W\": [");
    for (int t = 0; t < P; ++t) {
        if (t) std::printf(", ");
        list(B.W[t]);
    }
    std::printf("], \"halo\": [");
    for (int me = 0; me < P; ++me) {
        const mdf::HaloLists H = mdf::halo_lists(B, P, me, K0);
        std::printf(me ? ", {\"send\": " : "{\"send\": ");
        list(H.send);
        std::printf(", \"recv\": ");
        list(H.recv);
        std::printf(", \"local\": ");
        list(H.local);
        std::printf(", \"send_n\": ");
        list(H.send_n);
        std::printf(", \"recv_n\": ");
        list(H.recv_n);
        std::printf(", \"rng\": [[%d, %d], [%d, %d]]}", H.rng[0][0], H.rng[0][1], H.rng[1][0], H.rng[1][1]);
    }
    std::printf("]}\n");
    return 0;
}
