# SPDX-License-Identifier: Apache-2.0
"""Stage-level parity of the statistics on the GPU, through the C ABI's testing hooks
(include/eda_b200_testing.h), bit for bit against the oracle's restatements (which
tests/test_oracle_stages.py pins to NumPy and SciPy):

- exact selections (eda_testing_select): medians and "linear" quantiles of samples, of masked
  samples, of forward differences along axis sets, of |value - centre|; ties, signed zeros,
  subnormals, empty and one-item sets, 1-D to 3-D, float32 and float64, elements large enough for
  clusters of 8 CTAs (the reference's selection twins, cpp/tests/test_stats.cu:130-326);
- significant extrema (eda_testing_flags): plateaus, peaks at 32-sample block edges, ties of
  float32 differences with tau, subnormals, inf and NaN samples, lines of 8192 float32 / 4096
  float64 samples, rows and column axes (cpp/tests/test_stats.cu:436-902);
- face-connected components (eda_testing_components): labels equal to the smallest index of the
  component, in 1-D to 3-D, across tile borders, at densities around the percolation threshold
  (cpp/tests/test_stats.cu:966-1050)."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from eda import _native

    lib = ctypes.CDLL(str(_native.LIB))
    vp, i64p = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)
    lib.eda_testing_select.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int64, i64p, ctypes.c_int, ctypes.c_int,
                                       vp, ctypes.c_int, vp, ctypes.c_double, vp, vp, vp]
    lib.eda_testing_select.restype = ctypes.c_int
    lib.eda_testing_flags.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int64, i64p, vp, vp, vp]
    lib.eda_testing_flags.restype = ctypes.c_int
    lib.eda_testing_components.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int64, i64p, vp, vp]
    lib.eda_testing_components.restype = ctypes.c_int
    lib.eda_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    lib.eda_last_error.restype = ctypes.c_size_t
    return torch, lib


def _err(lib) -> str:
    buf = ctypes.create_string_buffer(1024)
    lib.eda_last_error(buf, len(buf))
    return buf.value.decode()


def _dims(shape):
    return np.asarray(shape, dtype=np.int64)


# ---------------------------------------------------------------------------------------------
# selections

def gpu_select(dev, x, src=0, axes=0, mask=None, bits=1, center=None, q=-1.0):
    torch, lib = dev
    B, n = x.shape[0], x.shape[1:]
    xd = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    md = torch.from_numpy(np.ascontiguousarray(mask)).cuda() if mask is not None else None
    out = np.zeros(B, np.float64)
    cnt = np.zeros(B, np.int64)
    c = np.ascontiguousarray(center, dtype=np.float64) if center is not None else None
    nn = _dims(n)
    st = lib.eda_testing_select(xd.data_ptr(), 0 if x.dtype == np.float32 else 1, len(n), B,
                                nn.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), src, axes,
                                md.data_ptr() if md is not None else None, bits,
                                c.ctypes.data if c is not None else None, q, out.ctypes.data, cnt.ctypes.data, None)
    assert st == 0, _err(lib)
    return out, cnt


def items(x1, src, axes, mask1, bits, center1):
    """The items of one element as doubles: samples (masked), or forward differences in the dtype."""
    if src == 0:
        v = x1 if mask1 is None else x1[(mask1 & bits) != 0]
        v = v.reshape(-1).astype(np.float64)
    else:
        parts = [np.diff(x1, axis=a).reshape(-1).astype(np.float64) for a in range(x1.ndim) if axes & (1 << a)]
        v = np.concatenate(parts)
    if center1 is not None:
        v = np.abs(v - center1)
    return v


def field(shape, dtype, seed, kind="ties"):
    rng = np.random.default_rng(seed)
    if kind == "ties":
        x = np.round(rng.standard_normal(shape) * 3) / 3
        flat = x.reshape(-1)
        flat[rng.integers(0, flat.size, max(1, flat.size // 7))] = -0.0
    elif kind == "subnormal":
        x = rng.standard_normal(shape) * (1e-41 if dtype == np.float32 else 1e-310)
    else:
        x = rng.standard_normal(shape) * np.exp(rng.uniform(-20, 20, shape))
    return x.astype(dtype)


SHAPES = [(2, 7), (3, 2048), (2, 64, 77), (2, 512, 512), (2, 16, 9, 33), (1, 64, 64, 64)]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("kind", ["ties", "subnormal", "wide"])
def test_select_samples(dev, dtype, shape, kind):
    x = field(shape, dtype, sum(shape) + len(kind), kind)
    for q in (-1.0, 0.0, 0.25, 0.5, 0.9, 1.0):
        out, cnt = gpu_select(dev, x, q=q)
        for b in range(shape[0]):
            v = items(x[b], 0, 0, None, 0, None)
            want = oracle.select(v, q)
            assert out[b] == want, (q, b, out[b], want)
            assert cnt[b] == v.size


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape", SHAPES)
def test_select_masked_and_centred(dev, dtype, shape):
    rng = np.random.default_rng(sum(shape))
    x = field(shape, dtype, sum(shape) + 5)
    mask = rng.integers(0, 4, shape).astype(np.uint8)
    mask[0] = 0  # element 0: nothing selected -> NaN, count 0
    center = rng.standard_normal(shape[0])
    for bits in (1, 2, 3):
        for c in (None, center):
            for q in (-1.0, 0.3):
                out, cnt = gpu_select(dev, x, mask=mask, bits=bits, center=c, q=q)
                for b in range(shape[0]):
                    v = items(x[b], 0, 0, mask[b], bits, None if c is None else c[b])
                    want = oracle.select(v, q)
                    assert (np.isnan(out[b]) and np.isnan(want)) or out[b] == want, (bits, q, b, out[b], want)
                    assert cnt[b] == v.size


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape", [(2, 2048), (2, 64, 77), (2, 512, 512), (2, 16, 9, 33)])
def test_select_differences(dev, dtype, shape):
    D = len(shape) - 1
    x = field(shape, dtype, sum(shape) + 9, "wide")
    rng = np.random.default_rng(3)
    center = rng.standard_normal(shape[0])
    for axes in range(1, 1 << D):
        for c in (None, center):
            out, cnt = gpu_select(dev, x, src=1, axes=axes, center=c)
            for b in range(shape[0]):
                v = items(x[b], 1, axes, None, 0, None if c is None else c[b])
                assert out[b] == oracle.select(v), (axes, b)
                assert cnt[b] == v.size


def test_select_single_item(dev):
    x = np.array([[3.5, 1.0], [-0.0, 2.0]], np.float32)
    mask = np.array([[1, 0], [1, 0]], np.uint8)
    out, cnt = gpu_select(dev, x, mask=mask)
    assert list(out) == [3.5, 0.0] and list(cnt) == [1, 1]
    assert not np.signbit(out[1])  # -0 selects as +0


# ---------------------------------------------------------------------------------------------
# significant extrema

def gpu_flags(dev, r, tau):
    torch, lib = dev
    B, n = r.shape[0], r.shape[1:]
    rd = torch.from_numpy(np.ascontiguousarray(r)).cuda()
    td = torch.from_numpy(np.ascontiguousarray(tau)).cuda()
    fd = torch.zeros(r.shape, dtype=torch.uint8, device="cuda")
    ext = np.zeros((B, len(n)), np.uint64)
    nn = _dims(n)
    st = lib.eda_testing_flags(rd.data_ptr(), td.data_ptr(), 0 if r.dtype == np.float32 else 1, len(n), B,
                               nn.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), fd.data_ptr(), ext.ctypes.data, None)
    assert st == 0, _err(lib)
    return fd.cpu().numpy(), ext


def lines(shape, dtype, seed, kind):
    rng = np.random.default_rng(seed)
    n = shape[-1]
    if kind == "smooth":
        t = np.arange(n)
        x = np.sin(2 * np.pi * t / rng.uniform(5, 40)) + 0.3 * rng.standard_normal(shape)
    elif kind == "plateaus":
        x = np.repeat(np.round(rng.standard_normal(shape[:-1] + (n // 4 + 1,)) * 2), 4, axis=-1)[..., :n]
    elif kind == "block_edges":
        x = 0.01 * rng.standard_normal(shape)
        for p in (31, 32, 63, 64, 95, 96):
            if p < n - 1:
                x[..., p] = 5.0 if p % 2 else -5.0
    elif kind == "subnormal":
        x = rng.standard_normal(shape) * (1e-41 if dtype == np.float32 else 1e-310)
    elif kind == "nonfinite":
        x = rng.standard_normal(shape)
        flat = x.reshape(-1)
        flat[rng.integers(0, flat.size, max(1, flat.size // 40))] = np.inf
        flat[rng.integers(0, flat.size, max(1, flat.size // 40))] = -np.inf
        flat[rng.integers(0, flat.size, max(1, flat.size // 40))] = np.nan
    else:
        raise ValueError(kind)
    return x.astype(dtype)


KINDS = ["smooth", "plateaus", "block_edges", "subnormal", "nonfinite"]


def check_flags(dev, r, tau):
    got, ext = gpu_flags(dev, r, tau)
    for b in range(r.shape[0]):
        want, wext = oracle.flags(r[b], tau[b])
        assert np.array_equal(got[b], want), np.argwhere(got[b] != want)[:5]
        assert [int(v) for v in ext[b]] == [int(v) for v in wext]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("shape", [(3, 3), (2, 33), (2, 100), (4, 2047), (2, 12000), (2, 64, 77), (2, 12, 10, 37)])
def test_flags(dev, dtype, kind, shape):
    r = lines(shape, dtype, sum(shape) + len(kind), kind)
    rng = np.random.default_rng(sum(shape))
    scale = float(np.nanmax(np.abs(r[np.isfinite(r)]))) if np.isfinite(r).any() else 1.0
    for tau in (np.zeros(shape, dtype), (rng.uniform(0, 1.2, shape) * scale).astype(dtype),
                np.full(shape, 0.5 * scale, dtype)):
        check_flags(dev, r, tau)


@pytest.mark.parametrize("dtype,n", [(np.float32, 8192), (np.float64, 4096), (np.float32, 20000), (np.float64, 65536),
                                     (np.float32, 65536)])
def test_flags_longest_lines(dev, dtype, n):
    r = lines((2, n), dtype, 11, "smooth")
    tau = np.full(r.shape, 0.4, dtype)
    check_flags(dev, r, tau)


def test_flags_tie_with_tau(dev):
    a = np.float32(1.0) + np.float32(2.0**-23)
    b = np.float32(2.0**-30)
    r = np.array([[b, a, b, a, b]], np.float32)
    tau = np.full(r.shape, np.float32(a - b), np.float32)  # the float difference ties, the double one is below
    got, _ = gpu_flags(dev, r, tau)
    assert not got.any()
    check_flags(dev, r, tau)


# ---------------------------------------------------------------------------------------------
# face-connected components

def gpu_components(dev, mask, bits=1):
    torch, lib = dev
    B, n = mask.shape[0], mask.shape[1:]
    md = torch.from_numpy(np.ascontiguousarray(mask.astype(np.uint8))).cuda()
    ld = torch.empty(mask.shape, dtype=torch.int32, device="cuda")
    nn = _dims(n)
    st = lib.eda_testing_components(md.data_ptr(), bits, len(n), B, nn.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                    ld.data_ptr(), None)
    assert st == 0, _err(lib)
    return ld.cpu().numpy()


@pytest.mark.parametrize("shape", [(2, 2), (2, 100), (3, 8192), (2, 20000), (1, 65536), (2, 7, 13), (2, 512, 512),
                                   (1, 3000, 70),
                                   (2, 5, 6, 7), (2, 16, 9, 33), (1, 64, 64, 64)])
@pytest.mark.parametrize("density", [0.0, 0.3, 0.5, 0.6, 1.0])
def test_components(dev, shape, density):
    rng = np.random.default_rng(int(np.prod(shape)) % 1000 + int(density * 10))
    mask = (rng.uniform(size=shape) < density).astype(np.uint8) * 2 + rng.integers(0, 2, shape).astype(np.uint8)
    for bits in (2, 1):
        got = gpu_components(dev, mask, bits)
        for b in range(shape[0]):
            want = oracle.components((mask[b] & bits) != 0)
            assert np.array_equal(got[b].astype(np.int64), want)


# Batches of 40 or more elements fill the GPU with clusters (one launch per selection); smaller
# batches take the grid-wide form (a counting and a pick launch per digit): both forms, every kind.
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape", [(40, 300), (48, 32, 48), (40, 6, 7, 9)])
def test_select_in_clusters(dev, dtype, shape):
    x = field(shape, dtype, sum(shape), "ties")
    rng = np.random.default_rng(1)
    mask = rng.integers(0, 2, shape).astype(np.uint8)
    center = rng.standard_normal(shape[0])
    for kw in ({}, {"mask": mask}, {"center": center}, {"src": 1, "axes": 1}, {"src": 1, "axes": (1 << (len(shape) - 1)) - 1}):
        for q in (-1.0, 0.25):
            out, cnt = gpu_select(dev, x, q=q, **kw)
            for b in range(shape[0]):
                v = items(x[b], kw.get("src", 0), kw.get("axes", 0), None if "mask" not in kw else mask[b], 1,
                          None if "center" not in kw else center[b])
                want = oracle.select(v, q)
                assert (np.isnan(out[b]) and np.isnan(want)) or out[b] == want, (kw, q, b)
                assert cnt[b] == v.size


# After its candidates' pass a selection reads the candidates (64-bit keys: the keys that share the
# first two digits, read from the fourth pass; 32-bit keys: the first digit, read in the third) when
# they fit a quarter of the items, else the items again: a constant field overflows the candidates,
# a field of many binades does not, one binade lies near the limit. Both forms.
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("batch", [2, 40])
def test_select_candidates_and_their_overflow(dev, dtype, batch):
    rng = np.random.default_rng(batch)
    shape = (batch, 96, 80)
    fields = {
        "constant": np.full(shape, 1.25),
        "one binade": 1.0 + rng.random(shape),
        "many binades": rng.standard_normal(shape) * np.exp(rng.uniform(-30, 30, shape)),
    }
    center = rng.standard_normal(batch)
    for name, x in fields.items():
        x = x.astype(dtype)
        for kw in ({}, {"center": center}, {"src": 1, "axes": 3}):
            for q in (-1.0, 0.75):
                out, cnt = gpu_select(dev, x, q=q, **kw)
                for b in range(batch):
                    v = items(x[b], kw.get("src", 0), kw.get("axes", 0), None, 0,
                              None if "center" not in kw else center[b])
                    assert out[b] == oracle.select(v, q), (name, kw, q, b)
                    assert cnt[b] == v.size
