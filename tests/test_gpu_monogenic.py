# SPDX-License-Identifier: Apache-2.0
"""eda.monogenic on the engine (src/eda/_api.py:356-426 and cpp/src/method/monogenic.cpp of
eda-cuda): against the oracle's restatement on the committed fixture fields, the plane-wave
behaviour the reference documents (amplitude 1, frequency |k|, direction k / |k|, coherence 1),
independence from the batch, device input and the non-finite rule.

Tolerances (the engine's float32 transforms run on the tensor cores in 3xTF32, the oracle's in
double): amplitude within 1e-4 (float32) / 1e-10 (float64) of the field's largest amplitude; where
the amplitude exceeds 5 % of its largest value (elsewhere phase and frequency, a quotient by the
squared amplitude, are ill-conditioned), phase within 2e-3 / 1e-8 rad and frequency within
5e-3 / 1e-8 cycles per sample; direction and
coherence as in the orientation test: float32 at most 2.5 % of the samples beyond 2e-3 (c) or
1 - 2e-3 (|n . n_oracle| where c > 0.05), float64 none beyond 1e-6.
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import batched, parity_cases, parity_input, restore_order

pytestmark = pytest.mark.gpu

CASES = parity_cases()
IDS = sorted(c for c in CASES if CASES[c]["conditioning_class"] == "stable" and "nan" not in c and "inf" not in c
             and CASES[c]["check_finite"])[::3]


def oracle_monogenic(x: np.ndarray, axes):
    xb, bax, ax, bshape = batched(x, axes)
    flat, bad = oracle.monogenic(xb)
    B, spatial = xb.shape[0], xb.shape[1:]
    D, n = len(spatial), xb.shape[0] * int(np.prod(spatial))
    out, off = [], 0
    for comps in ((0, 0, 0, D, 0) if D >= 2 else (0, 0, 0)):
        extra = (comps,) if comps else ()
        part = flat[off: off + n * max(comps, 1)].reshape(bshape + extra + spatial)
        out.append(part.transpose(restore_order(x.ndim, bax, ax, len(extra))))
        off += n * max(comps, 1)
    return out + ([None, None] if D == 1 else []), bad


def check(got, want, dtype, axis_m):
    amp, ph, fr, d, c = (np.asarray(v) if v is not None else None for v in got)
    wamp, wph, wfr, wd, wc = want
    f32 = dtype == np.float32
    scale = float(np.abs(wamp).max(initial=0.0)) or 1.0
    assert np.abs(amp - wamp).max(initial=0.0) <= (1e-4 if f32 else 1e-10) * scale
    live = wamp > 0.05 * scale
    dph = np.abs(np.angle(np.exp(1j * (ph.astype(np.float64) - wph))))
    assert dph[live].max(initial=0.0) <= (2e-3 if f32 else 1e-8)
    assert np.abs(fr.astype(np.float64) - wfr)[live].max(initial=0.0) <= (5e-3 if f32 else 1e-8)
    if d is None:
        return
    tol_c, min_c, tol_d = (2e-3, 0.05, 2e-3) if f32 else (1e-6, 1e-3, 1e-6)
    dc = np.abs(c.astype(np.float64) - wc)
    gd = np.moveaxis(d.astype(np.float64), axis_m, -1)
    wdd = np.moveaxis(wd.astype(np.float64), axis_m, -1)
    bad = (dc > tol_c) | ((wc > min_c) & (np.abs(np.sum(gd * wdd, axis=-1)) < 1 - tol_d))
    if f32:
        assert bad.mean() <= 2.5e-2 and dc.max(initial=0.0) <= 0.1, (float(bad.mean()), float(dc.max()))
    else:
        assert not bad.any(), float(dc.max(initial=0.0))


@pytest.mark.parametrize("cid", IDS)
def test_monogenic_agrees_with_the_oracle(engine, cid):
    c = CASES[cid]
    x = parity_input(cid).astype(c["dtype"])
    got = engine.monogenic(x, axes=c["axes"])
    want, bad = oracle_monogenic(x, c["axes"])
    assert not bad.any()
    _, _, ax, _ = batched(x, c["axes"])
    check((got.amplitude, got.phase, got.frequency, got.direction, got.coherence), want, x.dtype, min(ax))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_plane_waves(engine, dtype):
    h, w = 64, 80
    y, x = np.mgrid[0:h, 0:w].astype(np.float64)
    k = np.array([0.08, 0.06])
    f = np.cos(2 * np.pi * (k[0] * y + k[1] * x) + 0.3).astype(dtype)
    m = engine.monogenic(f)
    sl = (slice(12, -12), slice(12, -12))
    assert np.allclose(m.amplitude[sl], 1.0, atol=0.03)
    assert np.allclose(m.frequency[sl], 0.1, atol=0.003)
    assert np.allclose(m.direction[0][sl], 0.8, atol=0.01) and np.allclose(m.direction[1][sl], 0.6, atol=0.01)
    assert np.all(m.coherence[sl] > 0.99)
    t = np.arange(512.0)
    s = engine.monogenic(np.cos(2 * np.pi * 0.05 * t + 1.0).astype(dtype))
    assert s.direction is None and s.coherence is None
    assert np.allclose(s.amplitude[64:-64], 1.0, atol=0.05) and np.allclose(s.frequency[64:-64], 0.05, atol=0.002)


def test_fields_do_not_depend_on_their_batch(engine):
    x = parity_input("d2-batch3-40x36.f32")
    whole = engine.monogenic(x, axes=(1, 2))
    alone = engine.monogenic(np.ascontiguousarray(x[1]))
    for name in ("amplitude", "phase", "frequency", "coherence"):
        assert np.array_equal(getattr(whole, name)[1], getattr(alone, name))
    assert np.array_equal(whole.direction[1], alone.direction)


def test_device_input_and_the_non_finite_rule(engine):
    import torch

    x = parity_input("d3-batch3-20x18x16.f32")
    host = engine.monogenic(x, axes=(1, 2, 3))
    dev = engine.monogenic(torch.from_numpy(x).cuda(), axes=(1, 2, 3))
    assert isinstance(dev.amplitude, engine.DeviceArray)
    for name in ("amplitude", "phase", "frequency", "direction", "coherence"):
        assert np.array_equal(np.asarray(getattr(dev, name)), getattr(host, name))
    bad = x.copy()
    bad[2, 3, 4, 5] = np.nan
    with pytest.raises(ValueError, match="inf or NaN at batch index 2"):
        engine.monogenic(bad, axes=(1, 2, 3))
    m = engine.monogenic(bad, axes=(1, 2, 3), check_finite=False)
    assert np.array_equal(m.amplitude[:2], host.amplitude[:2])
