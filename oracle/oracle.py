# SPDX-License-Identifier: Apache-2.0
"""TEST INFRASTRUCTURE ONLY: a ctypes wrapper of the CPU oracle (eda_oracle.cpp), the restatement of
eda-cuda's decomposition that the tests, the smoke check and the benchmark's CPU baseline compare
the CUDA path with. The product never imports this module.

``decompose(x, max_imf=-1, tie_tolerance=None, sifts=3, check_finite=True, threads=1)`` takes a
C-contiguous (B, *spatial) float32 or float64 array and returns ``(rows, info)`` with rows
(B, P, *spatial) (P = 1 + the largest IMF count of the elements without an error, NaN rows for
failed elements) and info the dict of the reference's native call (cpp/python/decompose.cpp:188-214):
n_imfs, error, windows, sifts, spacing, energy (B, K), K the largest IMF count.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
_lib = None


def build() -> Path:
    """Compiles the oracle (make) when the library is missing or older than its source."""
    src = HERE / "eda_oracle.cpp"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB))
        i64p = ctypes.POINTER(ctypes.c_int64)
        i32p = ctypes.POINTER(ctypes.c_int32)
        f64p = ctypes.POINTER(ctypes.c_double)
        L.eda_oracle_rows_cap.argtypes = [ctypes.c_int, i64p, ctypes.c_int32]
        L.eda_oracle_rows_cap.restype = ctypes.c_int
        L.eda_oracle_decompose.argtypes = [
            ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int64, i64p, ctypes.c_int32,
            ctypes.c_double, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
            i32p, i32p, i32p, i32p, f64p, f64p, i32p, ctypes.c_char_p, ctypes.c_int64,
        ]
        L.eda_oracle_decompose.restype = ctypes.c_int
        L.eda_oracle_decompose_orientation.argtypes = [
            ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int64, i64p, ctypes.c_int32,
            ctypes.c_double, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
            i32p, i32p, i32p, i32p, f64p, f64p, i32p, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int64,
        ]
        L.eda_oracle_decompose_orientation.restype = ctypes.c_int
        L.eda_oracle_monogenic.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int64, i64p,
                                           ctypes.c_void_p, i32p]
        L.eda_oracle_monogenic.restype = ctypes.c_int
        L.eda_oracle_rung_ladder.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int32, ctypes.c_int32, i32p]
        L.eda_oracle_rung_ladder.restype = ctypes.c_int
        L.eda_oracle_cube.argtypes = [ctypes.c_int, ctypes.c_int, i64p, ctypes.c_int, ctypes.c_int32, ctypes.c_void_p]
        L.eda_oracle_cube.restype = ctypes.c_int
        L.eda_oracle_select.argtypes = [f64p, ctypes.c_int64, ctypes.c_double, f64p]
        L.eda_oracle_select.restype = ctypes.c_int
        L.eda_oracle_flags.argtypes = [ctypes.c_int, ctypes.c_int, i64p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]
        L.eda_oracle_flags.restype = ctypes.c_int
        L.eda_oracle_components.argtypes = [ctypes.c_int, i64p, ctypes.c_void_p, i64p]
        L.eda_oracle_components.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def rows_cap(shape: tuple[int, ...], max_imf: int = -1) -> int:
    n = np.asarray(shape, dtype=np.int64)
    return lib().eda_oracle_rows_cap(len(shape), _p(n, ctypes.c_int64), max_imf)


def decompose_raw(x: np.ndarray, max_imf: int = -1, tie_tolerance: float | None = None, sifts: int = 3,
                  check_finite: bool = True, threads: int = 1, orientation: bool = False) -> tuple[np.ndarray, dict]:
    """The oracle on (B, *spatial): rows (B, cap, *spatial) and the raw per-element arrays; with
    ``orientation`` also ``orient`` (B, cap - 1, D + 1, *spatial): n (canonical sign) and c per mode."""
    x = np.ascontiguousarray(x)
    assert x.dtype in (np.float32, np.float64) and 2 <= x.ndim <= 4
    B, spatial = x.shape[0], x.shape[1:]
    n = np.asarray(spatial, dtype=np.int64)
    cap = rows_cap(spatial, max_imf)
    rows = np.zeros((B, cap) + spatial, dtype=x.dtype)
    he = cap - 1
    n_imfs = np.zeros(B, np.int32)
    error = np.zeros(B, np.int32)
    exps = np.zeros(B, np.int32)
    windows = np.zeros((B, he), np.int32)
    sifts_out = np.zeros((B, he), np.int32)
    spacing = np.zeros((B, he), np.float64)
    energy = np.zeros((B, he), np.float64)
    err = ctypes.create_string_buffer(512)
    orient = np.zeros((B, he, len(spatial) + 1) + spatial, dtype=x.dtype) if orientation else None
    rc = lib().eda_oracle_decompose_orientation(
        x.ctypes.data, 0 if x.dtype == np.float32 else 1, len(spatial), B, _p(n, ctypes.c_int64), max_imf,
        -1.0 if tie_tolerance is None else float(tie_tolerance), sifts, int(bool(check_finite)), threads,
        rows.ctypes.data, _p(n_imfs, ctypes.c_int32), _p(error, ctypes.c_int32), _p(windows, ctypes.c_int32),
        _p(sifts_out, ctypes.c_int32), _p(spacing, ctypes.c_double), _p(energy, ctypes.c_double),
        _p(exps, ctypes.c_int32), None if orient is None else orient.ctypes.data, err, 512)
    if rc != 0:
        raise RuntimeError(f"oracle: {err.value.decode()}")
    out = {"n_imfs": n_imfs, "error": error, "windows": windows, "sifts": sifts_out,
           "spacing": spacing, "energy": energy, "exp": exps}
    if orient is not None:
        out["orient"] = orient
    return rows, out


def decompose(x: np.ndarray, max_imf: int = -1, tie_tolerance: float | None = None, sifts: int = 3,
              check_finite: bool = True, threads: int = 1) -> tuple[np.ndarray, dict]:
    """The rows (B, P, *spatial) and the info dict of the reference's native call."""
    rows, raw = decompose_raw(x, max_imf, tie_tolerance, sifts, check_finite, threads)
    ok = raw["error"] == 0
    P = int(raw["n_imfs"][ok].max(initial=-1)) + 1 if ok.any() else 1
    P = max(P, 1)
    K = int(raw["n_imfs"].max(initial=0))
    info = {"n_imfs": raw["n_imfs"], "error": raw["error"]}
    for name in ("windows", "sifts", "spacing", "energy"):
        a = raw[name][:, :K].copy()
        a[~ok] = 0
        info[name] = a
    out = rows[:, :P].copy()
    return out, info


def monogenic(x: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """The monogenic signal of the fields of x (B, *spatial): the native planes (amplitude, phase,
    frequency (B, count) each, then in 2-D / 3-D direction (B, D, count) and coherence (B, count)),
    flattened, and the non-finite flags [B]."""
    x = np.ascontiguousarray(x)
    B, spatial = x.shape[0], x.shape[1:]
    D = len(spatial)
    count = int(np.prod(spatial))
    planes = 3 if D == 1 else 4 + D
    out = np.zeros(planes * B * count, dtype=x.dtype)
    bad = np.zeros(B, np.int32)
    n = np.asarray(spatial, dtype=np.int64)
    if lib().eda_oracle_monogenic(x.ctypes.data, 0 if x.dtype == np.float32 else 1, D, B, _p(n, ctypes.c_int64),
                                  out.ctypes.data, _p(bad, ctypes.c_int32)) != 0:
        raise RuntimeError("oracle: monogenic")
    return out, bad


def rung_ladder(d_min: float, d_max: float, w: int, n_max: int) -> list[int]:
    out = np.zeros(32, np.int32)
    k = lib().eda_oracle_rung_ladder(d_min, d_max, w, n_max, _p(out, ctypes.c_int32))
    if k < 0:
        raise ValueError("oracle: rung_ladder")
    return [int(v) for v in out[:k]]


def cube(f: np.ndarray, op: str, w: int) -> np.ndarray:
    """One cube filter (op 'max', 'min' or 'box') of one element f (*spatial)."""
    f = np.ascontiguousarray(f).copy()
    n = np.asarray(f.shape, dtype=np.int64)
    code = {"max": 0, "min": 1, "box": 3}[op]
    lib().eda_oracle_cube(0 if f.dtype == np.float32 else 1, f.ndim, _p(n, ctypes.c_int64), code, w, f.ctypes.data)
    return f


def select(values: np.ndarray, q: float = -1.0) -> float:
    """The exact median (q < 0) or NumPy "linear" quantile of the doubles in values (NaN if empty)."""
    v = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
    out = np.zeros(1, np.float64)
    lib().eda_oracle_select(_p(v, ctypes.c_double), v.size, float(q), _p(out, ctypes.c_double))
    return float(out[0])


def flags(r: np.ndarray, tau: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """The significant-extrema flags of one element r (*spatial) against the threshold field tau:
    u8 flags (bit a: an extremum of a line along axis a) and the counts per axis."""
    r = np.ascontiguousarray(r)
    tau = np.ascontiguousarray(tau, dtype=r.dtype)
    n = np.asarray(r.shape, dtype=np.int64)
    out = np.zeros(r.shape, np.uint8)
    ext = np.zeros(3, np.uint64)
    lib().eda_oracle_flags(0 if r.dtype == np.float32 else 1, r.ndim, _p(n, ctypes.c_int64), r.ctypes.data,
                           tau.ctypes.data, out.ctypes.data, _p(ext, ctypes.c_uint64))
    return out, ext[:r.ndim].copy()


def components(mask: np.ndarray) -> np.ndarray:
    """Face-connected components of mask != 0 of one element: the smallest index of the sample's
    component, -1 outside."""
    m = np.ascontiguousarray(mask != 0, dtype=np.uint8)
    n = np.asarray(m.shape, dtype=np.int64)
    out = np.zeros(m.shape, np.int64)
    lib().eda_oracle_components(m.ndim, _p(n, ctypes.c_int64), m.ctypes.data, _p(out, ctypes.c_int64))
    return out


def cores() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
