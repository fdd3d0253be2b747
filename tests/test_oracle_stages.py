# SPDX-License-Identifier: Apache-2.0
"""The oracle's stage restatements against the definitions they restate (CPU, no GPU): the exact
selections against NumPy's median and "linear" quantile, the significant extrema against SciPy's
find_peaks and peak_prominences, the face-connected components against SciPy's ndimage.label
(labels renamed to the smallest index of each component). The reference pins the same stages
against the same definitions (cpp/tests/test_stats.cu:130-326 selections, :436-902 extrema with
SciPy twins, :966-1050 components against a BFS twin); the GPU stage tests then compare the engine
with these restatements bit for bit."""

from __future__ import annotations

import numpy as np
import pytest

import oracle

scipy_signal = pytest.importorskip("scipy.signal")
scipy_ndimage = pytest.importorskip("scipy.ndimage")


def _values(rng, n: int, kind: str) -> np.ndarray:
    if kind == "normal":
        return rng.standard_normal(n)
    if kind == "ties":
        return np.round(rng.standard_normal(n) * 3) / 3
    if kind == "zeros":
        v = rng.standard_normal(n)
        v[rng.integers(0, n, n // 3)] = 0.0
        v[rng.integers(0, n, n // 3)] = -0.0
        return v
    if kind == "subnormal":
        return rng.standard_normal(n) * 1e-310
    if kind == "wide":
        return rng.standard_normal(n) * np.exp(rng.uniform(-300, 300, n))
    raise ValueError(kind)


@pytest.mark.parametrize("kind", ["normal", "ties", "zeros", "subnormal", "wide"])
@pytest.mark.parametrize("n", [1, 2, 3, 10, 1001, 4096])
def test_select_matches_numpy(kind, n):
    rng = np.random.default_rng(n * 7 + len(kind))
    v = _values(rng, n, kind)
    got = oracle.select(v)
    want = float(np.median(v))
    assert got == want or (np.isnan(got) and np.isnan(want))
    for q in (0.0, 0.1, 0.25, 1 / 3, 0.5, 0.75, 0.9, 0.999, 1.0):
        got = oracle.select(v, q)
        want = float(np.quantile(v, q, method="linear"))
        assert got == want, (q, got, want)


def test_select_of_nothing_is_nan():
    assert np.isnan(oracle.select(np.zeros(0)))


def _scipy_flags(line: np.ndarray, tau: np.ndarray) -> np.ndarray:
    """SciPy's definition: peaks of line and of -line (plateau middles, no end points) whose
    topographic prominence, computed in double, is at least tau at the peak."""
    out = np.zeros(line.size, bool)
    x = line.astype(np.float64)
    for sgn in (1.0, -1.0):
        peaks, _ = scipy_signal.find_peaks(sgn * x)
        if peaks.size == 0:
            continue
        prom, _, _ = scipy_signal.peak_prominences(sgn * x, peaks)
        out[peaks[prom >= tau[peaks].astype(np.float64)]] = True
    return out


def _line(rng, n: int, kind: str, dtype) -> np.ndarray:
    t = np.arange(n)
    if kind == "smooth":
        x = np.sin(2 * np.pi * t / rng.uniform(5, 40)) + 0.3 * rng.standard_normal(n)
    elif kind == "plateaus":
        x = np.repeat(np.round(rng.standard_normal(n // 4 + 1) * 2), 4)[:n]
    elif kind == "ties":
        x = np.round(rng.standard_normal(n) * 2) / 2
    elif kind == "subnormal":
        x = rng.standard_normal(n) * 1e-41
    else:
        raise ValueError(kind)
    return x.astype(dtype)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("kind", ["smooth", "plateaus", "ties", "subnormal"])
@pytest.mark.parametrize("n", [3, 31, 32, 33, 64, 65, 257, 2000])
def test_flags_match_scipy(dtype, kind, n):
    rng = np.random.default_rng(n + 100 * len(kind))
    x = _line(rng, n, kind, dtype)
    scale = float(np.abs(x).max()) or 1.0
    for tau_kind in ("zero", "random", "const"):
        if tau_kind == "zero":
            tau = np.zeros(n, dtype)
        elif tau_kind == "const":
            tau = np.full(n, 0.5 * scale, dtype)
        else:
            tau = (rng.uniform(0, 1.5, n) * scale).astype(dtype)
        got, ext = oracle.flags(x, tau)
        want = _scipy_flags(x, tau)
        assert np.array_equal(got.astype(bool), want), (tau_kind, np.flatnonzero(got.astype(bool) != want))
        assert int(ext[0]) == int(want.sum())


def test_flags_tie_at_tau_is_decided_in_double():
    # the float32 difference of peak and base rounds to tau, the exact (double) difference is below it
    a = np.float32(1.0) + np.float32(2.0**-23)
    b = np.float32(2.0**-30)
    tau_val = np.float32(a - b)
    assert float(tau_val) > float(a) - float(b)
    x = np.array([b, a, b], np.float32)
    got, _ = oracle.flags(x, np.full(3, tau_val, np.float32))
    assert not got.any()
    got, _ = oracle.flags(x, np.full(3, np.float32(float(a) - float(b) - 1e-6), np.float32))
    assert got[1] == 1


@pytest.mark.parametrize("shape", [(9,), (1,), (7, 13), (33, 65), (5, 6, 7), (16, 9, 33)])
@pytest.mark.parametrize("density", [0.0, 0.3, 0.55, 1.0])
def test_components_match_scipy(shape, density):
    rng = np.random.default_rng(int(np.prod(shape)) + int(density * 100))
    mask = rng.uniform(size=shape) < density
    got = oracle.components(mask)
    lab, nlab = scipy_ndimage.label(mask)
    want = np.full(mask.shape, -1, np.int64)
    flat_lab = lab.reshape(-1)
    flat_want = want.reshape(-1)
    for k in range(1, nlab + 1):
        idx = np.flatnonzero(flat_lab == k)
        flat_want[idx] = idx.min()
    assert np.array_equal(got, want)
