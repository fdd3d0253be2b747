# SPDX-License-Identifier: Apache-2.0
"""return_orientation (eda.decompose(..., return_orientation=True)): every mode's direction n and
coherence c as the method computes them at the start of the mode, with the reference's layout and
sign rule (src/eda/_api.py:65-83, cpp/src/method/orientation.cu:412-418 and 495-549 of eda-cuda).

- Against the oracle's orientation rows on the committed 2-D / 3-D fixture cases. Tolerances: the
  engine's float32 transforms run on the tensor cores (3xTF32) and the oracle's in double, and c =
  (mu1 - mu2) / (mu1 + mu2) is ill-conditioned where both eigenvalues of the energy tensor are tiny
  (flat or noise-only regions), where float32 rounding alone moves it (the float64 path, with the
  same kernels, meets 1e-6 everywhere). So for float32 at most 2.5 % of the samples may have
  |c - c_oracle| > 2e-3 or, where c_oracle > 0.05 (a direction exists), |n . n_oracle| <
  1 - 2e-3, and none may differ by more than 0.1 in c; float64 must hold
  |c - c_oracle| <= 1e-6 and |n . n_oracle| >= 1 - 1e-6 (c_oracle > 1e-3) everywhere.
- A stripe pattern's direction and coherence; unit directions with the canonical sign; zero rows
  beyond n_imfs; y and info unchanged by the request; the layout with batch axes between the
  spatial axes; device input.
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import batched, parity_cases, parity_input, restore_order

pytestmark = pytest.mark.gpu

CASES = parity_cases()
IDS_ND = sorted(c for c in CASES if len(CASES[c]["info_axes"]) > 1 and CASES[c]["conditioning_class"] == "stable")


def kwargs(c: dict) -> dict:
    return {"axes": c["axes"], "max_imf": c["max_imf"], "dtype": c["dtype"], "tie_tolerance": c["tie_tolerance"],
            "check_finite": c["check_finite"], "errors": "status"}


@pytest.mark.parametrize("cid", IDS_ND)
def test_orientation_agrees_with_the_oracle(engine, cid):
    c = CASES[cid]
    x = parity_input(cid)
    y, info, orient = engine.decompose(x, **kwargs(c), return_info=True, return_orientation=True)
    xb, bax, ax, bshape = batched(x.astype(c["dtype"]), c["axes"])
    D = len(ax)
    _, raw = oracle.decompose_raw(xb, max_imf=c["max_imf"], tie_tolerance=c["tie_tolerance"],
                                  check_finite=c["check_finite"], threads=8, orientation=True)
    K = info.windows.shape[-1]
    B = xb.shape[0]
    o = raw["orient"][:, :K]  # (B, K, D + 1, *spatial)
    ok = (raw["error"] == 0)[:, None] & (np.arange(K)[None, :] < raw["n_imfs"][:, None])
    o = np.where(ok.reshape((B, K) + (1,) * (D + 1)), o, 0)
    want_dir = o[:, :, :D].reshape(bshape + (K, D) + xb.shape[1:]).transpose(restore_order(x.ndim, bax, ax, 2))
    want_coh = o[:, :, D].reshape(bshape + (K,) + xb.shape[1:]).transpose(restore_order(x.ndim, bax, ax, 1))
    got_dir, got_coh = np.asarray(orient.direction), np.asarray(orient.coherence)
    assert got_dir.shape == want_dir.shape and got_coh.shape == want_coh.shape
    f32 = c["dtype"] == "float32"
    tol_c, min_c, tol_d = (2e-3, 0.05, 2e-3) if f32 else (1e-6, 1e-3, 1e-6)
    # the K axis sits at position m (m = min(axes)), the D-component axis at m + 1
    m = min(ax)
    dc = np.moveaxis(np.abs(got_coh.astype(np.float64) - want_coh), m, 0)
    gd = np.moveaxis(np.moveaxis(got_dir.astype(np.float64), m + 1, -1), m, 0)
    wd = np.moveaxis(np.moveaxis(want_dir.astype(np.float64), m + 1, -1), m, 0)
    live = np.moveaxis(np.asarray(want_coh), m, 0) > min_c
    bad_d = live & (np.abs(np.sum(gd * wd, axis=-1)) < 1 - tol_d)
    bad = (dc > tol_c) | bad_d
    if bad.size == 0:
        return  # no element has an IMF: no orientation row
    if f32:
        assert bad.mean() <= 2.5e-2 and dc.max() <= 0.1, (float(bad.mean()), float(dc.max()))
    else:
        assert not bad.any(), (float(dc.max()), int(bad_d.sum()))


def stripes(h: int, w: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w].astype(np.float64)
    return (np.cos(2 * np.pi * (0.8 * y + 0.6 * x) / 7) + 0.01 * rng.standard_normal((h, w))).astype(np.float32)


def test_stripes_have_their_direction(engine):
    x = np.stack([stripes(64, 72, s) for s in range(2)])
    y, info, orient = engine.decompose(x, axes=(1, 2), return_info=True, return_orientation=True)
    n = orient.direction[:, 0, :, 16:-16, 16:-16]  # mode 0, interior
    c = orient.coherence[:, 0, 16:-16, 16:-16]
    assert np.all(c > 0.9)
    assert np.allclose(n[:, 0], 0.8, atol=0.02) and np.allclose(n[:, 1], 0.6, atol=0.02)


def test_unit_directions_sign_rule_and_zero_rows(engine):
    x = np.stack([stripes(48, 40, s) + parity_input("d2-batch3-40x36.f32")[0, :1, :1].mean() for s in range(3)])
    x[1] = np.cos(np.arange(48)[:, None] / 3.0) * np.cos(np.arange(40)[None, :] / 5.0)
    y, info, orient = engine.decompose(x, axes=(1, 2), return_info=True, return_orientation=True)
    d, c = orient.direction, orient.coherence
    K = info.windows.shape[-1]
    zero = 2.0 ** -14
    for b in range(x.shape[0]):
        k = int(info.n_imfs[b])
        assert np.all(d[b, k:] == 0) and np.all(c[b, k:] == 0)
        for j in range(k):
            nb = d[b, j].astype(np.float64)
            norm = np.sqrt((nb ** 2).sum(axis=0))
            live = c[b, j] > 0
            assert np.allclose(norm[live], 1.0, atol=1e-4)
            first = np.where(np.abs(nb[0]) > zero, nb[0], nb[1])
            assert np.all(first[np.abs(first) > zero] > 0)
            assert np.all((c[b, j] >= 0) & (c[b, j] <= 1))
    assert d.shape == (x.shape[0], K, 2) + x.shape[1:]


def test_the_request_changes_neither_rows_nor_info(engine):
    x = parity_input("d2-batch3-40x36.f32")
    y0, i0 = engine.decompose(x, axes=(1, 2), return_info=True)
    y1, i1, _ = engine.decompose(x, axes=(1, 2), return_info=True, return_orientation=True)
    assert np.array_equal(np.asarray(y0).view(np.uint32), np.asarray(y1).view(np.uint32))
    for name in ("n_imfs", "error", "windows", "sifts", "spacing", "energy"):
        assert np.array_equal(getattr(i0, name), getattr(i1, name))


def test_layout_with_batch_axes_between(engine):
    x = parity_input("d2-batchmid-24x31.f32")  # (24, 3, 31), axes (0, 2)
    _, info, o = engine.decompose(x, axes=(0, 2), return_info=True, return_orientation=True)
    _, info2, o2 = engine.decompose(np.ascontiguousarray(np.moveaxis(x, 1, 0)), axes=(1, 2), return_info=True,
                                    return_orientation=True)
    K = info.windows.shape[-1]
    assert o.direction.shape == (K, 2, 24, 3, 31) and o.coherence.shape == (K, 24, 3, 31)
    assert np.array_equal(np.moveaxis(np.asarray(o.direction), 3, 0), np.asarray(o2.direction))
    assert np.array_equal(np.moveaxis(np.asarray(o.coherence), 2, 0), np.asarray(o2.coherence))


def test_device_input_returns_device_arrays(engine):
    import torch

    x = parity_input("d3-batch3-20x18x16.f32")
    _, _, oh = engine.decompose(x, axes=(1, 2, 3), return_info=True, return_orientation=True)
    _, _, od = engine.decompose(torch.from_numpy(x).cuda(), axes=(1, 2, 3), return_info=True,
                                return_orientation=True)
    assert isinstance(od.direction, engine.DeviceArray)
    assert np.array_equal(np.asarray(od.direction), oh.direction)
    assert np.array_equal(np.asarray(od.coherence), oh.coherence)
