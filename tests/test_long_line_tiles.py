# SPDX-License-Identifier: Apache-2.0
"""The index arithmetic of the long-line cube pass's tiles (cube_long in cube.cu), restated on the
CPU: a CTA folds the tile [X0, X1) of a line of n samples with the window's segment ranges
G = the line's segments holding x + r and H = the reversed line's segments holding n - 1 - (x - r)
for x in the tile; it stages the samples they read, [vlo, vhi], and the output slots they write,
[xlo, xhi]. Checked here against a brute-force enumeration of every segment's samples and slots:
the staged ranges cover everything the folds touch, every output of the tile gets both its H and
its G, and the extents stay within the bounds the kernel uses to decide, alike for every tile of a
line, whether the tiles fit their shared memory."""

from __future__ import annotations

import random

import pytest

L = 4096  # kLongTile


def reflect(e: int, n: int) -> int:
    return -e - 1 if e < 0 else (2 * n - 1 - e if e >= n else e)


def span(u: int, v: int, n: int) -> tuple[int, int]:
    """reflect_span: the bounding interval of the samples that positions [u, v] read."""
    lo, hi = max(u, 0), min(v, n - 1)
    if u < 0:
        lo, hi = 0, max(hi, min(-u - 1, n - 1))
    if v > n - 1:
        hi, lo = n - 1, min(lo, max(2 * n - 1 - v, 0))
    return lo, hi


def tile(n: int, w: int, t: int):
    r = min((w - 1) // 2, n - 1)
    wa = 2 * r + 1
    o = (n * ((wa + 1) // 2)) % wa
    k_lo, k_hi = (r - o) // wa, (n - 1 + r - o) // wa
    e_max = n - 1 + r
    X0 = t * L
    X1 = min(X0 + L, n)
    gk0 = (X0 + r - o) // wa - k_lo
    gn = (X1 - 1 + r - o) // wa - k_lo - gk0 + 1
    hk0 = (n - X1 + r - o) // wa - k_lo
    hn = (n - 1 - X0 + r - o) // wa - k_lo - hk0 + 1
    gs = o + (k_lo + gk0) * wa
    ge = min(gs + gn * wa - 1, e_max)
    hs = o + (k_lo + hk0) * wa
    he = min(hs + hn * wa - 1, e_max)
    glo, ghi = span(gs, ge, n)
    hlo, hhi = span(hs, he, n)
    vlo, vhi = min(glo, n - 1 - hhi), max(ghi, n - 1 - hlo)
    xlo = min(max(gs, r) - r, n - 1 + r - he)
    xhi = max(ge - r, n - 1 + r - max(hs, r))
    return dict(r=r, wa=wa, o=o, k_lo=k_lo, nseg=k_hi - k_lo + 1, X0=X0, X1=X1, gk0=gk0, gn=gn, hk0=hk0, hn=hn,
                gs=gs, ge=ge, hs=hs, he=he, vlo=vlo, vhi=vhi, xlo=xlo, xhi=xhi, cps=(wa + 31) >> 5)


def cases(count: int, seed: int, max_w: int):
    rng = random.Random(seed)
    for _ in range(count):
        n = rng.randint(2, 65536)
        w = 2 * rng.randint(0, max_w) + 1
        t = rng.randrange((n + L - 1) // L)
        yield n, w, t


@pytest.mark.parametrize("max_w", [40, 1500])
def test_tiles_cover_what_their_folds_touch(max_w):
    for n, w, t in cases(1500, max_w, max_w):
        q = tile(n, w, t)
        r, wa = q["r"], q["wa"]
        assert 0 <= q["gk0"] and q["gk0"] + q["gn"] <= q["nseg"] and q["gn"] >= 1
        assert 0 <= q["hk0"] and q["hk0"] + q["hn"] <= q["nseg"] and q["hn"] >= 1
        read, g_slots, h_slots = set(), set(), set()
        for e in range(q["gs"], q["ge"] + 1):  # G: the line, slot e - r
            read.add(reflect(e, n))
            if e >= r:
                g_slots.add(e - r)
        for e in range(q["hs"], q["he"] + 1):  # H: the reversed line, slot n - 1 + r - e
            read.add(n - 1 - reflect(e, n))
            if e >= r:
                h_slots.add(n - 1 + r - e)
        assert q["vlo"] >= 0 and q["vhi"] <= n - 1
        assert min(read) >= q["vlo"] and max(read) <= q["vhi"], (n, w, t)
        slots = g_slots | h_slots
        assert min(slots) >= q["xlo"] and max(slots) <= q["xhi"], (n, w, t)
        for x in range(q["X0"], q["X1"]):
            assert x in g_slots and x in h_slots, (n, w, t, x)
        if wa == 1:  # one-sample windows fold exactly the tile's outputs
            assert (q["o"] + q["k_lo"] + q["gk0"], q["gn"]) == (q["X0"], q["X1"] - q["X0"])


def test_every_tile_within_the_shared_bounds():
    for n, w, t in cases(20000, 7, 70000):
        q = tile(n, w, t)
        nv, nx = q["vhi"] - q["vlo"] + 1, q["xhi"] - q["xlo"] + 1
        ts = max(q["gn"], q["hn"]) * q["cps"]
        bound = L + 2 * q["r"] + 2 * q["wa"] + 4
        assert nv <= bound and nx <= bound, (n, w, t)
        if q["cps"] > 1:  # one-chunk segments use no totals
            assert ts <= ((L + 2 * q["wa"]) // q["wa"] + 2) * q["cps"], (n, w, t)


def test_wide_windows_fit_the_chunk_table():
    """Windows too wide for the tiles fold in separate launches whose chunk tasks (segment k, chunk
    c) index a table of 2 x tot_slots(n) = 2 (n / 8 + 24) totals per line and rung, and whose carry
    launch stages that table in shared memory: nseg cps must fit it for every length and window."""
    rng = random.Random(11)
    for _ in range(200000):
        n = rng.randint(2, 65536)
        w = 2 * rng.randint(0, rng.choice([20, 200, 5000, 70000])) + 1
        r = min((w - 1) // 2, n - 1)
        wa = 2 * r + 1
        o = (n * ((wa + 1) // 2)) % wa
        nseg = (n - 1 + r - o) // wa - (r - o) // wa + 1
        cps = (wa + 31) >> 5
        if cps == 1:  # one-chunk segments always fold in the tiles (even in the smallest budget, the
            # 14 080 float64 samples of half an SM), so they never reach the chunk table
            span16 = (L + 2 * r + 2 * wa + 4 + 3) & ~3
            assert 2 * span16 <= 14080
            continue
        assert nseg * cps <= n // 8 + 24, (n, w, nseg, cps)
