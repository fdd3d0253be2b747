# SPDX-License-Identifier: Apache-2.0
"""The oracle (CPU restatement of the method) pinned to the reference's own corpora: the decisions
of the parity manifest (tests/data/parity_v2.json of eda-cuda) on every committed case, the golden
corpus (tests/data/golden) within its rows bound, and the ladder's tabulated values
(cpp/tests/rungs_table.inc of eda-cuda)."""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

import oracle
from conftest import batched, corpus, parity_cases, parity_input, restore_order

CASES = parity_cases()
IDS = sorted(CASES)


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run_oracle(cid: str):
    c = CASES[cid]
    x = parity_input(cid)
    xb, bax, ax, bshape = batched(x, c["axes"])
    rows, info = oracle.decompose(xb, max_imf=c["max_imf"], tie_tolerance=c["tie_tolerance"],
                                  check_finite=c["check_finite"], threads=4)
    P = rows.shape[1]
    y = rows.reshape(bshape + (P,) + xb.shape[1:]).transpose(restore_order(x.ndim, bax, ax))
    return x, y, info


@pytest.mark.parametrize("cid", IDS)
def test_oracle_reproduces_the_manifest_decisions(cid):
    c = CASES[cid]
    x, y, info = run_oracle(cid)
    assert list(y.shape) == c["y_shape"]
    assert [int(v) for v in info["n_imfs"]] == c["n_imfs"]
    assert [int(v) for v in info["error"]] == c["error"]
    for name in ("windows", "sifts"):
        a = np.ascontiguousarray(info[name].astype(np.int32))
        if name in c:
            assert [int(v) for v in a.reshape(-1)] == c[name]
        else:
            assert sha(a) == c[name + "_sha256"]


def test_oracle_is_bitwise_on_the_cases_without_a_scale_field():
    """Cases that stop before their first mode (no log / exp involved) are the reference's output
    bit for bit."""
    n = 0
    for cid in IDS:
        c = CASES[cid]
        if max(c["n_imfs"], default=0) == 0 and c["error"] == [0] * len(c["error"]) and len(c["info_axes"]) == 1:
            _, y, _ = run_oracle(cid)
            assert sha(y) == c["y_sha256"], cid
            n += 1
    assert n >= 5


META, ARR = corpus()


@pytest.mark.parametrize("name", sorted(META))
def test_oracle_reproduces_the_golden_corpus(name):
    m = META[name]
    x, modes = ARR[f"{name}.x"], ARR[f"{name}.modes"]
    rows, info = oracle.decompose(x[None], threads=4)
    y = rows[0]
    assert y.shape == modes.shape
    assert [int(v) for v in info["windows"][0]] == m["windows"]
    assert [int(v) for v in info["sifts"][0]] == m["sifts"]
    bound = (m["sensitivity"] / 1e-12) * 1000 * 2.0**-53 * np.abs(x).max()
    assert np.abs(y - modes).max() <= bound


# (d_min, d_max, w, n_max) -> rungs: rows of the reference's tabulated ladder (rungs_table.inc)
LADDER = [
    ((3.0, 9.0, 5, 64), [3, 5, 7, 11]),
    ((5.0, 5.0, 5, 64), [5]),
    ((0.75, 6.0, 3, 64), [1, 3, 5, 7]),
    ((0.2, 0.9, 3, 64), [1]),
    ((1.0, 1.0, 3, 10), [1]),
    ((0.75, 3.0, 3, 10), [1, 3]),
    ((2.25, 9.0, 9, 32), [3, 5, 7, 9]),
    ((13.0, 26.0, 13, 512), [13, 19, 27]),
    ((100.0, 400.0, 201, 100), [71, 101, 143, 201]),
    ((30.0, 900.0, 255, 128), [23, 31, 45, 63, 91, 127, 181, 255, 257]),
    ((4.0, 6.0, 7, 3), [3, 5, 7]),
    ((1.5, 2.5, 3, 2), [1, 3]),
]


@pytest.mark.parametrize("args,want", LADDER)
def test_ladder_matches_the_reference_table(args, want):
    assert oracle.rung_ladder(*args) == want


def test_cube_box_is_a_box_mean():
    rng = np.random.default_rng(0)
    f = rng.standard_normal((7, 9))
    out = oracle.cube(f, "box", 3)
    ref = np.zeros_like(f)
    pad = np.pad(f, 1, mode="symmetric")
    for i in range(7):
        for j in range(9):
            ref[i, j] = pad[i:i + 3, j:j + 3].mean()
    assert np.allclose(out, ref, rtol=1e-13, atol=1e-14)
    mx = oracle.cube(f, "max", 5)
    padm = np.pad(f, 2, mode="symmetric")
    refm = np.array([[padm[i:i + 5, j:j + 5].max() for j in range(9)] for i in range(7)])
    assert np.array_equal(mx, refm)
