# SPDX-License-Identifier: Apache-2.0
"""Parity and float64 error on the benchmarked configurations, through the public calls
eda.decompose and eda.decompose_ragged, on seeded samples made by the benchmark's own generators
(bench.py):

- 1-D: the 2048-sample three-tone signal;
- 2-D: two of the 64 images of 512 x 512 that the benchmark decomposes (the same seed);
- 3-D: two volumes of 128^3 made by the 256^3 recipe (the trend's width scaled by the side);
- 1-D ragged: eight signals of the ragged recipe, lengths 256 to 8192, and four of 8193 to 65536
  samples (lines beyond the shared-memory staging);
- 2-D ragged: four images of uneven sides, 64 to 640, by the ragged 2-D recipe.

For every element whose decisions are stable (unchanged by a one-ulp move of every sample, the
reference's stability probe), and at least half of every sample:
- the decisions (IMF count, windows, sift counts) equal the oracle's in float32, the dtype of the
  call;
- max |y - y64| / max |x| <= 1e-4, with y64 the oracle's decomposition of the same field in
  float64 (every rounding of the sift in double);
- and for every element, the rows add back up to x: max |sum_k y_k - x| / max |x| <= 1e-5.
"""

from __future__ import annotations

import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np
import pytest

import oracle

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
import bench  # noqa: E402

pytestmark = pytest.mark.gpu

REL_FP64 = 1e-4  # the sift's float32 rows against the float64 oracle, relative to max |x|
REL_SUM = 1e-5  # reconstruction, relative to max |x|


def _decisions(info) -> tuple:
    k = int(info["n_imfs"][0])
    return k, tuple(int(v) for v in info["windows"][0][:k]), tuple(int(v) for v in info["sifts"][0][:k])


def _oracle_both(fields: list[np.ndarray]):
    """Per field, on parallel threads: the oracle's float32 result, its float64 result, and whether
    the float32 decisions are stable (unchanged when every sample moves up by one ulp: the
    reference's own stability probe of its parity manifest)."""

    def one(x):
        r32 = oracle.decompose(x[None])
        up = oracle.decompose(np.nextafter(x, np.float32(np.inf))[None])
        return r32, oracle.decompose(x[None].astype(np.float64)), _decisions(r32[1]) == _decisions(up[1])

    with ThreadPoolExecutor(max_workers=min(len(fields), max(1, oracle.cores()))) as ex:
        return list(ex.map(one, fields))


def _check(fields, ys, infos):
    """fields: float32 arrays; ys[i]: rows (P, *shape) of field i; infos[i]: (n_imfs, windows, sifts).
    Elements whose decisions move with a one-ulp change of the input (unstable) are checked for
    reconstruction only: the engine's float32 log / exp (the reference's) and the oracle's host
    library may then take different windows. Most elements of every sample are stable."""
    worst = 0.0
    stable_count = 0
    for x, y, (k, win, sif), ((_, o32), (r64, o64), stable) in zip(fields, ys, infos, _oracle_both(fields)):
        y = np.asarray(y, dtype=np.float64)
        amax = float(np.abs(x).max())
        recon = float(np.abs(y.sum(axis=0) - x.astype(np.float64)).max()) / amax
        assert recon <= REL_SUM, recon
        if not stable:
            continue
        stable_count += 1
        assert k == int(o32["n_imfs"][0]), (k, o32["n_imfs"])
        assert list(win[:k]) == [int(v) for v in o32["windows"][0][:k]]
        assert list(sif[:k]) == [int(v) for v in o32["sifts"][0][:k]]
        # the float64 oracle takes the same decisions on these fields
        assert int(o64["n_imfs"][0]) == k and list(o64["windows"][0][:k]) == list(o32["windows"][0][:k])
        rel = float(np.abs(y[:k + 1] - r64[0, :k + 1]).max()) / amax
        assert rel <= REL_FP64, rel
        assert not np.any(y[k + 1:])
        worst = max(worst, rel)
    assert 2 * stable_count >= len(fields), (stable_count, len(fields))
    return worst


def _batch(engine, x: np.ndarray, axes):
    y, info = engine.decompose(x, axes=axes, return_info=True)
    ys = [y[b] for b in range(x.shape[0])]
    infos = [(int(info.n_imfs[b]), [int(v) for v in info.windows[b]], [int(v) for v in info.sifts[b]])
             for b in range(x.shape[0])]
    return ys, infos


def test_config_1d(engine):
    x = bench.signal_1d(2024)
    ys, infos = _batch(engine, x, (1,))
    _check([x[0]], ys, infos)


def test_config_2d_benchmark_images(engine):
    x = bench.workload(2, 1000)  # the benchmark's first two images (rank 0's seed)
    ys, infos = _batch(engine, x, (1, 2))
    _check(list(x), ys, infos)


def test_config_2d_on_device(engine):
    torch = pytest.importorskip("torch")
    x = bench.workload(2, 1000)
    y, info = engine.decompose(torch.from_numpy(x).cuda(), axes=(1, 2), return_info=True)
    y = np.asarray(y)
    infos = [(int(info.n_imfs[b]), [int(v) for v in info.windows[b]], [int(v) for v in info.sifts[b]]) for b in range(2)]
    _check(list(x), [y[b] for b in range(2)], infos)


def test_config_3d_stand_in(engine):
    x = bench.volumes_3d(2, 128, 2024)
    ys, infos = _batch(engine, x, (1, 2, 3))
    _check(list(x), ys, infos)


def test_config_ragged_1d(engine):
    xs = bench.signals_ragged(8, 256, 8192, 2024)
    rows, infos = engine.decompose_ragged(xs, return_info=True)
    _check(xs, rows, [(int(i.n_imfs), [int(v) for v in i.windows], [int(v) for v in i.sifts]) for i in infos])


def test_config_long_1d_signals(engine):
    """Signals of the 1-D ragged recipe beyond the 8192 samples that a pass stages in shared memory,
    up to the recipe's 65536: their lines fold in global memory."""
    xs = [x for x in bench.signals_ragged(40, 256, 65536, 77) if x.size > 8192][:3]
    xs.append(bench.signals_ragged(1, 65536, 65537, 5)[0])  # exp(U[ln 65536, ln 65537]) truncates to 65536
    assert all(x.size > 8192 for x in xs) and xs[-1].size == 65536
    rows, infos = engine.decompose_ragged(xs, return_info=True)
    _check(xs, rows, [(int(i.n_imfs), [int(v) for v in i.windows], [int(v) for v in i.sifts]) for i in infos])


def test_config_ragged_2d(engine):
    xs = bench.images_ragged(4, 64, 640, 2024)
    rows, infos = engine.decompose_ragged(xs, return_info=True)
    _check(xs, rows, [(int(i.n_imfs), [int(v) for v in i.windows], [int(v) for v in i.sifts]) for i in infos])
