"""The band decomposition of a split evaluation (md_b200/csrc/bands.hpp), on
the CPU: the same header the pair-list build includes, compiled into a small
harness (tests/band_plan.cpp) that prints the plan.

Checked for the c0, c4 and small geometries and edge cases (more ranks than
column rows, planes that do not divide evenly, one plane per rank, a large
skin): the bands tile the column rows in order, each column goes to the rank
whose x-slab holds its centre, every atom binned in a band keeps its whole
order-4 stencil inside the band's window while it drifts less than half the
skin (the spread kernel's own base-plane arithmetic), and the halo lists are
consistent between ranks (what r sends to t is what t receives from r, in the
same order; a window is its own planes plus the planes it sends).
"""
import json
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "md_b200", "csrc")

# (ranks, planes along x, column rows along x, box edge, skin)
CASES = [(2, 72, 15, 66.0, 2.0), (3, 72, 15, 66.0, 2.0), (4, 72, 15, 66.0, 2.0), (5, 72, 15, 66.0, 2.0),
         (8, 216, 49, 215.0, 2.0), (16, 216, 49, 215.0, 2.0), (2, 32, 6, 30.0, 2.0), (3, 32, 6, 30.0, 2.0),
         (8, 32, 6, 30.0, 2.0), (32, 32, 6, 30.0, 2.0), (2, 72, 15, 66.0, 8.0), (7, 100, 23, 100.0, 2.0)]


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("bands") / "band_plan")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I" + CSRC, os.path.join(HERE, "band_plan.cpp"), "-o", exe],
                   check=True)
    return exe


def plan(exe, P, K0, ncx, Lx, skin):
    out = subprocess.run([exe, str(P), str(K0), str(ncx), repr(Lx), repr(skin)], check=True, capture_output=True,
                         text=True).stdout
    return json.loads(out)


def split(lst, counts):
    out, k = [], 0
    for n in counts:
        out.append(lst[k:k + n])
        k += n
    assert k == len(lst)
    return out


@pytest.mark.parametrize("P,K0,ncx,Lx,skin", CASES)
def test_bands_tile_the_columns_by_slab(harness, P, K0, ncx, Lx, skin):
    B = plan(harness, P, K0, ncx, Lx, skin)
    first = B["first"]
    assert first[0] == 0 and first[P] == ncx
    assert all(a <= b for a, b in zip(first, first[1:]))
    K0p = (K0 + P - 1) // P
    for cx in range(ncx):
        t = max(r for r in range(P) if first[r] <= cx)
        assert first[t] <= cx < first[t + 1]
        assert t == min(P - 1, int(np.floor((cx + 0.5) * K0 / ncx / K0p)))


@pytest.mark.parametrize("P,K0,ncx,Lx,skin", CASES)
def test_every_stencil_stays_in_its_window_within_half_the_skin(harness, P, K0, ncx, Lx, skin):
    B = plan(harness, P, K0, ncx, Lx, skin)
    rng = np.random.default_rng(P * 1000 + K0)
    w = Lx / ncx
    for t in range(P):
        ca, cb = B["first"][t], B["first"][t + 1]
        if cb <= ca:
            assert B["win_n"][t] == 0 and B["W"][t] == []
            continue
        # atoms binned in the band: its edges and random points
        x = np.concatenate([[ca * w, cb * w - 1e-9, (ca + cb) * 0.5 * w], rng.uniform(ca * w, cb * w, 400)])
        x = x[(x >= 0) & (x < Lx)]
        W = set(B["W"][t])
        for d in (-0.4999 * skin, -0.25 * skin, 0.0, 0.25 * skin, 0.4999 * skin):
            u = np.mod(x + d, Lx) * K0 / Lx
            u = np.where(u >= K0, u - K0, u)
            base = np.minimum(np.floor(u).astype(int), K0 - 1)
            assert (np.mod(base - B["win_lo"][t], K0) < B["win_n"][t]).all()
            planes = set(np.mod(np.concatenate([base - 1, base, base + 1, base + 2]), K0).tolist())
            assert planes <= W, sorted(planes - W)[:4]


@pytest.mark.parametrize("P,K0,ncx,Lx,skin", CASES)
def test_halo_lists_agree_between_ranks(harness, P, K0, ncx, Lx, skin):
    B = plan(harness, P, K0, ncx, Lx, skin)
    K0p = (K0 + P - 1) // P
    H = B["halo"]
    sends = [split(h["send"], h["send_n"]) for h in H]
    recvs = [split(h["recv"], h["recv_n"]) for h in H]
    for r in range(P):
        assert H[r]["send_n"][r] == 0 and H[r]["recv_n"][r] == 0
        W = B["W"][r]
        assert all(0 <= p < K0 for p in W) and len(set(W)) == len(W)
        local = H[r]["local"]
        assert all(p // K0p == r for p in local)
        for t in range(P):
            assert all(p // K0p == t for p in sends[r][t])
            assert sends[r][t] == recvs[t][r]       # same planes, same order
        sent = [p for t in range(P) for p in sends[r][t]]
        assert sorted(local + sent) == sorted(W)
        (a, n), (b, m) = H[r]["rng"]
        cover = [(a + k) % K0 for k in range(n)] + [(b + k) % K0 for k in range(m)]
        assert sorted(cover) == sorted(W)


def test_c4_halo_is_a_few_planes(harness):
    """At 960k atoms (216^3, 49 column rows) and 8 or 16 ranks a window
    reaches at most 12 planes past its 27- or 14-plane slab."""
    for P in (8, 16):
        B = plan(harness, P, 216, 49, 215.0, 2.0)
        for h in B["halo"]:
            assert len(h["send"]) <= 12
