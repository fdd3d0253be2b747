# SPDX-License-Identifier: Apache-2.0
"""Test configuration: the ``gpu`` marker (tests that need a B200), paths to the engine's Python
package and to the oracle (test infrastructure), and the committed fixtures."""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "eda-cuda_b200"))
sys.path.insert(0, str(ROOT / "oracle"))
GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built engine")
    config.addinivalue_line("markers", "slow: the larger fixture cases")


def parity_cases() -> dict:
    return json.loads((GOLDEN / "parity_expect.json").read_text())["cases"]


_inputs = None


def parity_input(case_id: str) -> np.ndarray:
    global _inputs
    if _inputs is None:
        _inputs = np.load(GOLDEN / "parity_inputs.npz", allow_pickle=False)
    return _inputs[case_id]


def corpus() -> tuple[dict, dict]:
    meta = json.loads((GOLDEN / "corpus.json").read_text())["cases"]
    arrays = np.load(GOLDEN / "corpus.npz", allow_pickle=False)
    return meta, arrays


def restore_order(ndim: int, batch_axes: tuple[int, ...], axes: tuple[int, ...], extra: int = 1) -> list[int]:
    nb = len(batch_axes)
    where = {a: nb + extra + k for k, a in enumerate(axes)}
    where.update({a: k for k, a in enumerate(batch_axes)})
    m = min(axes)
    return [where[f] for f in range(m)] + [nb + j for j in range(extra)] + [where[f] for f in range(m, ndim)]


def batched(x: np.ndarray, axes) -> tuple[np.ndarray, tuple, tuple, tuple]:
    """x as the C-contiguous (B, *spatial) array of a call, with batch axes, axes and batch shape."""
    ndim = x.ndim
    ax = tuple(range(ndim)) if axes is None else tuple(a % ndim for a in axes)
    bax = tuple(i for i in range(ndim) if i not in ax)
    xt = np.ascontiguousarray(x.transpose(list(bax) + list(ax)))
    bshape = tuple(x.shape[i] for i in bax)
    spatial = tuple(x.shape[a] for a in ax)
    return xt.reshape((int(np.prod(bshape, dtype=np.int64)),) + spatial), bax, ax, bshape


@pytest.fixture(scope="session")
def engine():
    """The eda package on the B200 engine (skips without a device)."""
    import eda

    if eda.device_count() < 1:
        pytest.skip("no CUDA device")
    return eda
