# SPDX-License-Identifier: Apache-2.0
"""Stage-level parity on the GPU: the engine's cube filter (eda_testing_cube, through the C ABI)
bit for bit against the oracle's restatement of the reference's vHGW passes, as the reference's
own stage test checks its passes against its host twin (cpp/tests/test_cube.cu:52-205 of
eda-cuda): max, min, max+min and box means; 1-D, 2-D and 3-D; float32 and float64; windows
clamped by short axes (wider than the line), one-sample windows, window 0 (element skipped),
segments of more than 32 chunks (windows above 1024), elements with few rows (fewer lines per CTA),
and the rung launches (k = 1, 2, 5, 32 windows per element in one launch per pass) against k
one-rung cubes."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

OPS = {"max": 0, "min": 1, "maxmin": 2, "box": 3}


@pytest.fixture(scope="module")
def dev():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from eda import _native

    lib = ctypes.CDLL(str(_native.LIB))
    lib.eda_testing_cube.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int64,
                                     ctypes.POINTER(ctypes.c_int64), ctypes.c_int, ctypes.POINTER(ctypes.c_int32),
                                     ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.eda_testing_cube.restype = ctypes.c_int
    lib.eda_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    lib.eda_last_error.restype = ctypes.c_size_t
    return torch, lib


def field(shape, dtype, seed: int) -> np.ndarray:
    """Values with ties (a coarse grid), signed zeros and a smooth trend."""
    rng = np.random.default_rng(seed)
    x = np.round(rng.standard_normal(shape) * 4) / 4
    x = x + np.linspace(0, 1, x.size).reshape(shape) * (seed % 3)
    flat = x.reshape(-1)
    flat[rng.integers(0, flat.size, size=max(1, flat.size // 50))] = -0.0
    return x.astype(dtype)


def gpu_cube(dev, x: np.ndarray, op: str, wins: np.ndarray):
    """x (B, *n); wins [rungs][B] -> out0 (and out1 for maxmin) (rungs, B, *n)."""
    torch, lib = dev
    B, n = x.shape[0], x.shape[1:]
    rungs = wins.shape[0]
    xd = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    o0 = torch.empty((rungs,) + x.shape, dtype=xd.dtype, device="cuda")
    o1 = torch.empty_like(o0)
    nn = np.asarray(n, dtype=np.int64)
    w = np.ascontiguousarray(wins, dtype=np.int32)
    st = lib.eda_testing_cube(xd.data_ptr(), 0 if x.dtype == np.float32 else 1, len(n), B,
                              nn.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), OPS[op],
                              w.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), rungs, o0.data_ptr(),
                              o1.data_ptr(), None)
    if st != 0:
        buf = ctypes.create_string_buffer(512)
        lib.eda_last_error(buf, 512)
        raise AssertionError(f"eda_testing_cube: {st}: {buf.value.decode()}")
    torch.cuda.synchronize()
    return o0.cpu().numpy(), o1.cpu().numpy()


def same_bits(a: np.ndarray, b: np.ndarray) -> bool:
    u = np.uint32 if a.dtype == np.float32 else np.uint64
    return np.array_equal(np.ascontiguousarray(a).view(u), np.ascontiguousarray(b).view(u))


def check(dev, shape, op, wins, dtype, seed=1234):
    wins = np.asarray(wins, dtype=np.int32)
    if wins.ndim == 1:
        wins = wins[None, :]
    rungs, B = wins.shape
    x = np.stack([field(shape, dtype, seed + 7 * b) for b in range(B)])
    got0, got1 = gpu_cube(dev, x, op, wins)
    for j in range(rungs):
        for b in range(B):
            w = int(wins[j, b])
            if w < 1:
                assert np.isnan(got0[j, b]).all(), (shape, op, j, b)
                continue
            if op == "maxmin":
                want0, want1 = oracle.cube(x[b], "max", w), oracle.cube(x[b], "min", w)
                assert same_bits(got1[j, b], want1), (shape, op, "min", j, b, w)
            else:
                want0 = oracle.cube(x[b], op, w)
            assert same_bits(got0[j, b], want0), (shape, op, j, b, w,
                                                  float(np.nanmax(np.abs(got0[j, b] - want0))))


CASES = [
    ((300,), [1, 7, 0, 601]),
    ((2,), [1, 3, 5]),
    ((1500,), [1023, 1025, 1201, 2999]),
    ((37, 45), [9, 0, 3, 91]),
    ((5, 64), [13, 21]),
    ((1100, 5), [1025, 2201, 0]),
    ((3, 7), [5, 1, 15]),
    ((64, 96), [33, 65]),
    ((11, 9, 14), [5, 0, 27]),
    ((4, 16, 6), [9, 3]),
    ((40, 5, 36), [11, 7]),
]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("op", list(OPS))
@pytest.mark.parametrize("shape,wins", CASES, ids=[f"{'x'.join(map(str, s))}" for s, _ in CASES])
def test_cube_matches_the_oracle_bitwise(dev, shape, wins, op, dtype):
    check(dev, shape, op, wins, dtype)


def test_cube_on_benchmark_sized_images(dev):
    check(dev, (512, 512), "maxmin", [33, 101], np.float32)
    check(dev, (512, 512), "box", [7, 257], np.float32)


def test_cube_on_a_full_benchmark_batch(dev):
    """64 images of 512 x 512 with a different window per image (one skipped): every CTA runs
    several line groups, copying the next group while it folds the current one; and a 3-rung
    launch of the same batch (the first pass stages each group once for every rung)."""
    wins = np.array([9, 33, 65, 0, 257, 1, 129, 17] * 8, np.int32)
    check(dev, (512, 512), "maxmin", wins, np.float32)
    check(dev, (512, 512), "box", wins, np.float32)
    check(dev, (512, 512), "maxmin", np.stack([wins, np.roll(wins, 3), np.roll(wins, 5)]), np.float32, seed=77)


def test_cube_on_the_longest_lines(dev):
    check(dev, (8192,), "box", [4095, 16383, 1], np.float32)
    check(dev, (4096,), "maxmin", [2047, 9], np.float64)


# 1-D lines beyond the staged capacity (the long-line pass folds in global memory): every op,
# one-sample, one-chunk, multi-chunk and clamped windows, up to the 1-D limit of 65536 samples
LONG_WINS = [1, 3, 31, 33, 1025, 40001, 131071]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("op", list(OPS))
@pytest.mark.parametrize("n", [8193, 16384, 65536])
def test_cube_on_long_1d_lines(dev, n, op, dtype):
    check(dev, (n,), op, LONG_WINS[:4] if n == 8193 else LONG_WINS, dtype, seed=n)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("op", ["maxmin", "box"])
def test_cube_long_line_tiles(dev, op, dtype):
    """Long lines fold in tiles of 4096 outputs, each CTA staging the segments its outputs need,
    or (windows whose segments do not fit a tile's shared memory) the whole line in one CTA: a
    length that is no multiple of the tile, and windows on both sides of the limit."""
    check(dev, (20001,), op, [5, 65, 1501, 2049, 2501, 3001, 4097, 6001, 9001], dtype, seed=21)


def test_cube_rung_launch_on_long_lines(dev):
    rng = np.random.default_rng(5)
    wins = (2 * rng.integers(0, 3000, size=(4, 2)) + 1).astype(np.int32)
    wins[1, 0] = 0
    check(dev, (30000,), "maxmin", wins, np.float32, seed=3)
    check(dev, (30000,), "box", wins, np.float32, seed=4)


@pytest.mark.parametrize("k", [1, 2, 5, 32])
@pytest.mark.parametrize("op", ["maxmin", "box"])
@pytest.mark.parametrize("shape", [(37, 45), (300,), (11, 9, 14)], ids=["2d", "1d", "3d"])
def test_rung_launches_match_one_rung_cubes(dev, shape, op, k):
    rng = np.random.default_rng(k)
    B = 3
    wins = (2 * rng.integers(0, 40, size=(k, B)) + 1).astype(np.int32)
    wins[k // 2, 1] = 0  # a skipped element in one rung
    check(dev, shape, op, wins, np.float32, seed=99 + k)


# ---------------------------------------------------------------------------------------------
# The orientation's separable transforms (eda_testing_transform): the tensor-core passes (float32,
# 3xTF32) and the FP64 passes (float64) against the same orthonormal bases applied in float64 by
# numpy. Tolerance: float32 max|got - want| <= 2e-5 max|want| (3xTF32 keeps float32-level error,
# about 1e-6 relative for a 512-point axis); float64 1e-12 max|want|.

def basis(n: int, kind: int) -> np.ndarray:
    """Matrix M with out = M @ in along one axis: 0 forward DCT-II, 1 inverse cosine, 2 inverse sine."""
    k = np.arange(n)[:, None].astype(np.float64)
    x = np.arange(n)[None, :].astype(np.float64)
    ck = np.sqrt(np.where(k == 0, 1.0, 2.0) / n)
    C = ck * np.cos(np.pi * k * (2 * x + 1) / (2 * n))
    S = ck * np.sin(np.pi * k * (2 * x + 1) / (2 * n))
    return {0: C, 1: C.T, 2: S.T}[kind]


def gpu_transform(dev, x: np.ndarray, kinds) -> np.ndarray:
    torch, lib = dev
    lib.eda_testing_transform.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int64,
                                          ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32),
                                          ctypes.c_void_p, ctypes.c_void_p]
    lib.eda_testing_transform.restype = ctypes.c_int
    B, n = x.shape[0], x.shape[1:]
    xd = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    out = torch.empty_like(xd)
    nn = np.asarray(n, dtype=np.int64)
    kk = np.asarray(kinds, dtype=np.int32)
    st = lib.eda_testing_transform(xd.data_ptr(), 0 if x.dtype == np.float32 else 1, len(n), B,
                                   nn.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                   kk.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), out.data_ptr(), None)
    if st != 0:
        buf = ctypes.create_string_buffer(512)
        lib.eda_last_error(buf, 512)
        raise AssertionError(f"eda_testing_transform: {st}: {buf.value.decode()}")
    torch.cuda.synchronize()
    return out.cpu().numpy()


def host_transform(x: np.ndarray, kinds) -> np.ndarray:
    y = x.astype(np.float64)
    for a, kind in enumerate(kinds):
        M = basis(x.shape[1 + a], kind)
        y = np.moveaxis(np.tensordot(M, np.moveaxis(y, 1 + a, 0), axes=(1, 0)), 0, 1 + a)
    return y


TRANSFORMS = [
    ((37, 45), (0, 0)),
    ((64, 96), (1, 2)),
    ((130, 7), (2, 1)),
    ((128, 128), (2, 2)),
    ((512, 512), (0, 0)),
    ((5, 300), (1, 1)),
    ((11, 9, 14), (0, 0, 0)),
    ((32, 40, 36), (2, 1, 2)),
    ((17, 64, 33), (1, 2, 1)),
]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape,kinds", TRANSFORMS, ids=["x".join(map(str, s)) + "-" + "".join(map(str, k))
                                                          for s, k in TRANSFORMS])
def test_transform_matches_the_bases_in_float64(dev, shape, kinds, dtype):
    rng = np.random.default_rng(len(shape) * 100 + shape[0])
    B = 3
    x = rng.standard_normal((B,) + shape).astype(dtype)
    got = gpu_transform(dev, x, kinds)
    want = host_transform(x, kinds)
    err = np.max(np.abs(got - want))
    tol = (2e-5 if dtype == np.float32 else 1e-12) * np.max(np.abs(want))
    assert err <= tol, (shape, kinds, err, tol)


# the float32 transforms' products: their error against the float64 bases (relative to the
# result's largest magnitude) in every mode; the mode is process-wide, restored afterwards
PRECISION_TOL = {0: 2e-5, 1: 2e-4, 2: 2e-5}


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("shape,kinds", TRANSFORMS, ids=["x".join(map(str, s)) + "-" + "".join(map(str, k))
                                                          for s, k in TRANSFORMS])
def test_transform_precision_arms(dev, shape, kinds, mode):
    torch, lib = dev
    lib.eda_set_transform_precision.argtypes = [ctypes.c_int]
    lib.eda_transform_precision.restype = ctypes.c_int
    rng = np.random.default_rng(len(shape) * 100 + shape[0] + mode)
    x = rng.standard_normal((3,) + shape).astype(np.float32)
    assert lib.eda_set_transform_precision(mode) == 0
    try:
        assert lib.eda_transform_precision() == mode
        got = gpu_transform(dev, x, kinds)
    finally:
        lib.eda_set_transform_precision(0)
    want = host_transform(x, kinds)
    err = np.max(np.abs(got - want))
    tol = PRECISION_TOL[mode] * np.max(np.abs(want))
    assert err <= tol, (shape, kinds, mode, err, tol)


def test_transform_precision_rejects_unknown_modes(dev):
    torch, lib = dev
    lib.eda_set_transform_precision.argtypes = [ctypes.c_int]
    assert lib.eda_set_transform_precision(3) == 1
    assert lib.eda_set_transform_precision(-1) == 1


# Every launch shape the autotuner may choose gives the same bits: the cube filter under recorded
# shapes (lines per CTA, groups per CTA, segment share) against the oracle, then a tuned geometry's
# decomposition against the untuned one.
@pytest.mark.parametrize("lines,groups,share", [(2, 1, 2), (4, 2, 8), (8, 2, 2), (8, 1, 64)])
def test_cube_under_every_launch_shape(dev, tmp_path, lines, groups, share):
    import eda

    core = eda._native.core()
    shape = (48, 200)
    path = tmp_path / "tune.txt"
    path.write_text("".join(f"4 2 {shape[0]} {shape[1]} 1 {bucket} {lines} {groups} {share} 1 1\n" for bucket in range(4)))
    core.tuning_clear()
    core.tuning_load(str(path))
    try:
        check(dev, shape, "maxmin", [1, 5, 33, 63, 129], np.float32)
        check(dev, shape, "box", [3, 47, 95, 255], np.float32)
        check(dev, shape, "maxmin", np.stack([[7, 41, 99], [65, 0, 13]]), np.float32, seed=5)
    finally:
        core.tuning_clear()


def test_autotuned_geometry_decomposes_identically(dev, tmp_path):
    import eda

    rng = np.random.default_rng(4)
    yy, xx = np.mgrid[0:96, 0:120]
    x = np.stack([np.cos(2 * np.pi * (xx + k * yy) / 11) + 0.2 * rng.standard_normal((96, 120)) for k in (0.2, 0.5)])
    x = x.astype(np.float32)
    eda._native.core().tuning_clear()
    want, want_info = eda.decompose(x, axes=(1, 2), return_info=True)
    report = eda.autotune((96, 120), batch=2, cache=str(tmp_path / "t.txt"))
    assert report["us_best"] <= report["us_default"]
    got, info = eda.decompose(x, axes=(1, 2), return_info=True)
    assert np.array_equal(got, want) and np.array_equal(info.windows, want_info.windows)
    assert (tmp_path / "t.txt").read_text().count("\n") >= 2
    eda._native.core().tuning_clear()
