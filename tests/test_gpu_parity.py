# SPDX-License-Identifier: Apache-2.0
"""The CUDA engine against the reference's recorded results and the oracle, through the public
call eda.decompose:

- decisions (IMF counts, error codes, windows, sifts) equal the parity manifest on every committed
  case (tests/data/parity_v2.json of eda-cuda);
- 1-D outputs equal the manifest's output hashes bit for bit (1-D involves no transform library:
  every operation is a canonical rounding, as in the reference);
- 2-D / 3-D rows agree with the oracle within the reference's parity rule between two transform
  libraries: |y - y_oracle| <= 10 sensitivity max|x| on the stable cases (the sensitivity is the
  manifest's one-ulp input probe);
- the golden corpus (tests/data/golden of eda-cuda): decisions exact, rows within its bound.
"""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

import oracle
from conftest import batched, corpus, parity_cases, parity_input, restore_order

pytestmark = pytest.mark.gpu

CASES = parity_cases()
IDS = sorted(CASES)
IDS_1D = [c for c in IDS if len(CASES[c]["info_axes"]) == 1]
IDS_ND = [c for c in IDS if len(CASES[c]["info_axes"]) > 1]


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def kwargs(c: dict) -> dict:
    return {"axes": c["axes"], "max_imf": c["max_imf"], "dtype": c["dtype"], "tie_tolerance": c["tie_tolerance"],
            "check_finite": c["check_finite"], "errors": c["errors"]}


_runs: dict = {}


def run(engine, cid: str):
    if cid not in _runs:
        x = parity_input(cid)
        y, info = engine.decompose(x, **kwargs(CASES[cid]), return_info=True)
        _runs[cid] = (x, y, info)
    return _runs[cid]


@pytest.mark.parametrize("cid", IDS)
def test_decisions_match_the_manifest(engine, cid):
    c = CASES[cid]
    x, y, info = run(engine, cid)
    assert list(y.shape) == c["y_shape"]
    assert [int(v) for v in info.n_imfs.reshape(-1)] == c["n_imfs"]
    assert [int(v) for v in info.error.reshape(-1)] == c["error"]
    for name in ("windows", "sifts"):
        a = np.ascontiguousarray(getattr(info, name))
        if name in c:
            assert [int(v) for v in a.reshape(-1)] == c[name]
        else:
            assert sha(a) == c[name + "_sha256"]


@pytest.mark.parametrize("cid", IDS_1D)
def test_1d_rows_are_the_references_bit_for_bit(engine, cid):
    c = CASES[cid]
    x, y, info = run(engine, cid)
    assert sha(y) == c["y_sha256"]
    assert sha(np.ascontiguousarray(info.spacing)) == c["spacing_sha256"]
    assert sha(np.ascontiguousarray(info.energy)) == c["energy_sha256"]


@pytest.mark.parametrize("cid", IDS_ND)
def test_nd_rows_agree_with_the_oracle(engine, cid):
    c = CASES[cid]
    if c["conditioning_class"] != "stable":
        pytest.skip("sensitive case: a one-ulp probe changes its decisions")
    x, y, info = run(engine, cid)
    xb, bax, ax, bshape = batched(x.astype(c["dtype"]), c["axes"])
    rows, _ = oracle.decompose(xb, max_imf=c["max_imf"], tie_tolerance=c["tie_tolerance"],
                               check_finite=c["check_finite"], threads=8)
    P = rows.shape[1]
    yo = rows.reshape(bshape + (P,) + xb.shape[1:]).transpose(restore_order(x.ndim, bax, ax))
    assert yo.shape == y.shape
    fin = np.isfinite(yo)
    assert np.array_equal(fin, np.isfinite(y))
    scale = float(np.abs(x[np.isfinite(x)].astype(np.float64)).max(initial=0.0))
    bound = 10 * c["sensitivity"] * scale
    diff = float(np.abs(y[fin].astype(np.float64) - yo[fin].astype(np.float64)).max(initial=0.0))
    assert diff <= bound, (diff, bound)


META, ARR = corpus()


@pytest.mark.parametrize("name", sorted(META))
def test_golden_corpus(engine, name):
    m = META[name]
    x, modes = ARR[f"{name}.x"], ARR[f"{name}.modes"]
    y, info = engine.decompose(x, return_info=True)
    assert y.shape == modes.shape
    assert [int(v) for v in info.windows] == m["windows"]
    assert [int(v) for v in info.sifts] == m["sifts"]
    bound = (m["sensitivity"] / 1e-12) * 1000 * 2.0**-53 * np.abs(x).max()
    assert np.abs(y - modes).max() <= bound
