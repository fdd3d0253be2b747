# SPDX-License-Identifier: Apache-2.0
"""The allocation-free decomposition (eda_decompose_noalloc) through the C ABI: for callers that
cannot allocate device memory (plugin hosts whose allocator belongs to the host application, loops
that forbid allocation after start-up), it must return what eda_decompose returns, bit for bit
(the tolerance of the 1-D parity tests), on consecutive calls that share its scratch, take no
device memory on a warm call, and reject a call larger than its scratch or buffers that are not
device memory of the current device with a clear error. The test allocates the input and output
buffers itself; the entry point allocates nothing.

This file is collected last (tests/test_zz_*), so a run that stops at its first failure has run
every other test first; it also passes alone in a fresh process."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _signals(batch: int, n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    t = np.arange(n, dtype=np.float64)
    out = []
    for b in range(batch):
        p1, p2 = rng.uniform(5, 12), rng.uniform(40, 90)
        out.append(np.sin(2 * np.pi * t / p1) + 2 * np.sin(2 * np.pi * t / p2 + b) + 3 * np.sin(2 * np.pi * t / 512)
                   + 0.05 * rng.standard_normal(n))
    return np.asarray(out)


def _noalloc(lib, core, x: np.ndarray, capacity: int, torch):
    from eda._native import _Params

    B, n = x.shape
    dev = torch.device("cuda", 0)
    x_dev = torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    rows_dev = torch.full((B, capacity, n), 7.0, dtype=x_dev.dtype, device=dev)
    K = capacity - 1
    n_imfs = np.zeros(B, np.int32)
    error = np.zeros(B, np.int32)
    windows = np.zeros((B, K), np.int32)
    sifts = np.zeros((B, K), np.int32)
    spacing = np.zeros((B, K), np.float64)
    energy = np.zeros((B, K), np.float64)
    P = ctypes.c_int32(0)
    params = _Params(-1, -1.0, 3, 1, 0)
    stream = torch.cuda.current_stream(dev)
    st = lib.eda_decompose_noalloc(
        ctypes.c_void_p(x_dev.data_ptr()), 0 if x.dtype == np.float32 else 1, B, n, ctypes.byref(params),
        ctypes.c_void_p(rows_dev.data_ptr()), capacity, ctypes.byref(P),
        *(ctypes.c_void_p(a.ctypes.data) for a in (n_imfs, error, windows, sifts, spacing, energy)),
        ctypes.c_void_p(stream.cuda_stream))
    if st != 0:
        buf = ctypes.create_string_buffer(1024)
        lib.eda_last_error(buf, len(buf))
        return st, buf.value.decode(), None
    torch.cuda.synchronize(dev)
    info = {"n_imfs": n_imfs, "error": error, "windows": windows, "sifts": sifts, "spacing": spacing, "energy": energy}
    return st, P.value, (rows_dev.cpu().numpy(), info)


@pytest.fixture(scope="module")
def parts():
    torch = pytest.importorskip("torch")
    import eda
    from eda import _native

    if eda.device_count() < 1:
        pytest.skip("no CUDA device")
    core = _native.core()
    lib = core._lib
    vp, i32p = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)
    lib.eda_decompose_noalloc.argtypes = [vp, ctypes.c_int, ctypes.c_int64, ctypes.c_int64, vp, vp, ctypes.c_int32,
                                          i32p, vp, vp, vp, vp, vp, vp, vp]
    lib.eda_decompose_noalloc.restype = ctypes.c_int
    return torch, core, lib


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_noalloc_matches_eda_decompose_on_consecutive_calls(parts, dtype):
    torch, core, lib = parts
    capacity = 16
    for seed in (11, 12, 11):  # two different calls, then the first again: no state leaks through the scratch
        x = _signals(4, 2048, seed).astype(dtype)
        want_rows, want_info = core.decompose_host(x, -1, None, 3, True, False, 0)
        st, P, out = _noalloc(lib, core, x, capacity, torch)
        assert st == 0, P
        rows, info = out
        assert P == want_rows.shape[1]
        assert np.array_equal(rows[:, :P], want_rows)
        assert not rows[:, P:].any()
        K = want_info["windows"].shape[1]
        for name in ("n_imfs", "error"):
            assert np.array_equal(info[name], want_info[name]), name
        for name in ("windows", "sifts", "spacing", "energy"):
            assert np.array_equal(info[name][:, :K], want_info[name]), name
            assert not info[name][:, K:].any(), name


def test_noalloc_rejects_a_call_beyond_its_scratch(parts):
    torch, core, lib = parts
    x = _signals(64, 4096, 3).astype(np.float32)  # 262144 samples: beyond the 24 MiB scratch
    st, msg, _ = _noalloc(lib, core, x, 16, torch)
    assert st == 1 and "scratch" in msg
    # the library stays usable
    x = _signals(2, 512, 4).astype(np.float32)
    want_rows, _ = core.decompose_host(x, -1, None, 3, True, False, 0)
    st, P, (rows, _) = _noalloc(lib, core, x, 16, torch)
    assert st == 0 and np.array_equal(rows[:, :P], want_rows)


def test_noalloc_takes_no_device_memory(parts):
    """A warm call leaves the device's free memory unchanged (nothing allocated, nothing freed: no
    workspace, no pool, no library allocation); the buffers are made before the measurement."""
    torch, core, lib = parts
    from eda._native import _Params

    x = _signals(4, 2048, 21).astype(np.float32)
    B, n = x.shape
    dev = torch.device("cuda", 0)
    x_dev = torch.from_numpy(x).to(dev)
    rows_dev = torch.zeros((B, 16, n), dtype=torch.float32, device=dev)
    P = ctypes.c_int32(0)
    params = _Params(-1, -1.0, 3, 1, 0)
    stream = torch.cuda.current_stream(dev)

    def call():
        st = lib.eda_decompose_noalloc(ctypes.c_void_p(x_dev.data_ptr()), 0, B, n, ctypes.byref(params),
                                       ctypes.c_void_p(rows_dev.data_ptr()), 16, ctypes.byref(P),
                                       None, None, None, None, None, None, ctypes.c_void_p(stream.cuda_stream))
        torch.cuda.synchronize(dev)
        return st

    assert call() == 0  # warm: the kernels of the path are loaded
    free0, _ = torch.cuda.mem_get_info(dev)
    assert call() == 0
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0


def test_noalloc_rejects_host_buffers(parts):
    torch, core, lib = parts
    from eda._native import _Params

    x = _signals(2, 512, 5).astype(np.float32)
    rows = np.zeros((2, 16, 512), np.float32)
    P = ctypes.c_int32(0)
    params = _Params(-1, -1.0, 3, 1, 0)
    st = lib.eda_decompose_noalloc(ctypes.c_void_p(x.ctypes.data), 0, 2, 512, ctypes.byref(params),
                                   ctypes.c_void_p(rows.ctypes.data), 16, ctypes.byref(P),
                                   None, None, None, None, None, None, None)
    assert st == 1
    buf = ctypes.create_string_buffer(1024)
    lib.eda_last_error(buf, len(buf))
    assert "device memory" in buf.value.decode()
