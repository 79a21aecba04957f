// Band decomposition of a split evaluation: the host arithmetic only (no
// CUDA), shared by the pair-list build (pairlist.cu build_bands) and its CPU
// test (tests/band_plan.cpp).
//
// Rank t of P takes the x-columns whose centres lie in its x-slab of the PME
// grid (planes [t K0p, (t+1) K0p), K0p = ceil(K0 / P)); the columns are
// numbered x-major, so those are contiguous column rows [first[t],
// first[t+1]) and contiguous clusters.  Its atoms were binned at x in
// [ca, cb) column widths, so with at most half the skin of drift their
// stencil bases lie in grid planes floor(ca K0/ncx - m) - 1 .. floor(cb K0/ncx
// + m) + 1 (m = half the skin in planes; one plane each side for rounding),
// and an order-4 stencil touches one plane below its base and two above: the
// rank's window.  Every rank computes every window (all hold all positions
// and the same list), so the planes a rank sends to each owner and receives
// from each rank follow without communication.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace mdf {

struct BandPlan {
    std::vector<int> first;              // [P + 1] first column row (x) of each rank
    std::vector<int> win_lo, win_n;      // [P] stencil-base window: start (unwrapped) and count
    std::vector<std::vector<int>> W;     // [P] real planes of each window, in unwrapped order
};

// P ranks, K0 planes along x, ncx column rows along x, box edge Lx, skin.
inline BandPlan plan_bands(int P, int K0, int ncx, double Lx, double skin)
{
    BandPlan B;
    const int K0p = (K0 + P - 1) / P;
    B.first.assign(P + 1, ncx);
    for (int cx = ncx - 1; cx >= 0; --cx) {
        const int t = std::min(P - 1, (int)std::floor((cx + 0.5) * K0 / ncx / K0p));
        for (int u = 0; u <= t; ++u) B.first[u] = std::min(B.first[u], cx);
    }
    B.first[0] = 0;
    B.first[P] = ncx;
    for (int t = 1; t < P; ++t) B.first[t] = std::max(B.first[t], B.first[t - 1]);
    const double m = 0.5 * skin * K0 / Lx;
    B.win_lo.assign(P, 0);
    B.win_n.assign(P, 0);
    B.W.assign(P, std::vector<int>());
    for (int t = 0; t < P; ++t) {
        const int ca = B.first[t], cb = B.first[t + 1];
        if (cb <= ca) continue;
        const int blo = (int)std::floor((double)ca * K0 / ncx - m) - 1;
        const int bhi = (int)std::floor((double)cb * K0 / ncx + m) + 1;
        B.win_lo[t] = blo;
        B.win_n[t] = std::min(bhi - blo + 1, K0);
        const int plo = blo - 1, phi = bhi + 2;   // stencil planes base - 1 .. base + 2
        if (phi - plo + 1 >= K0) {
            for (int p = 0; p < K0; ++p) B.W[t].push_back(p);
        } else {
            for (int p = plo; p <= phi; ++p) B.W[t].push_back(((p % K0) + K0) % K0);
        }
    }
    return B;
}

// Rank `me`'s halo lists: the planes of its window owned by each other rank
// (sent to them, in rank order), the planes of each other rank's window it
// owns (received from them, in rank order), the planes of its window it owns
// itself, and its window as at most two ranges of real planes (first, count).
struct HaloLists {
    std::vector<int> send, recv, local;
    std::vector<int64_t> send_n, recv_n;   // [P] planes per rank
    int rng[2][2] = {{0, 0}, {0, 0}};
};

inline HaloLists halo_lists(const BandPlan& B, int P, int me, int K0)
{
    HaloLists H;
    const int K0p = (K0 + P - 1) / P;
    auto owner = [&](int p) { return p / K0p; };
    H.send_n.assign(P, 0);
    H.recv_n.assign(P, 0);
    for (int t = 0; t < P; ++t) {
        if (t == me) {
            for (int p : B.W[me])
                if (owner(p) == me) H.local.push_back(p);
            continue;
        }
        for (int p : B.W[me])
            if (owner(p) == t) {
                H.send.push_back(p);
                ++H.send_n[t];
            }
        for (int p : B.W[t])
            if (owner(p) == me) {
                H.recv.push_back(p);
                ++H.recv_n[t];
            }
    }
    const std::vector<int>& w = B.W[me];
    if (!w.empty()) {
        if ((int)w.size() >= K0) {
            H.rng[0][0] = 0;
            H.rng[0][1] = K0;
        } else {
            const int p0 = w.front(), n = (int)w.size();
            const int n0 = std::min(n, K0 - p0);
            H.rng[0][0] = p0;
            H.rng[0][1] = n0;
            H.rng[1][0] = 0;
            H.rng[1][1] = n - n0;
        }
    }
    return H;
}

}  // namespace mdf
