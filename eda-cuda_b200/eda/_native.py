# SPDX-License-Identifier: Apache-2.0
"""The ctypes binding of the engine's C ABI (include/eda_b200.h), loaded on first use.

``core()`` returns an object with the calls of the reference's extension module eda._core
(src/eda/_core.pyi of eda-cuda): ``build_info``, ``device_count``, ``device_info``,
``decompose_host`` and ``decompose_device``. There is no CPU fallback: without the compiled library
the first call raises ImportError.
"""

from __future__ import annotations

import ctypes
import json
from pathlib import Path
from typing import Any

import numpy as np

from ._errors import CudaError

LIB = Path(__file__).resolve().parent / "libeda_b200.so"
_core = None

EDA_OK, EDA_INVALID_ARGUMENT, EDA_OUT_OF_MEMORY, EDA_CUDA_ERROR, EDA_INTERNAL = range(5)


class _Params(ctypes.Structure):
    _fields_ = [
        ("max_imf", ctypes.c_int32),
        ("tie_tolerance", ctypes.c_double),
        ("sifts", ctypes.c_int32),
        ("check_finite", ctypes.c_int32),
        ("max_chunk", ctypes.c_int64),
        ("orientation", ctypes.c_int32),
    ]


class _Source(ctypes.Structure):
    """eda_source: a device input's element type and layout (strides in elements, either sign)."""

    _fields_ = [("type", ctypes.c_int32), ("batch_axes", ctypes.c_int32),
                ("batch_shape", ctypes.POINTER(ctypes.c_int64)), ("batch_stride", ctypes.POINTER(ctypes.c_int64)),
                ("stride", ctypes.POINTER(ctypes.c_int64))]


# EDA_SRC_* codes of include/eda_b200.h
SOURCE_TYPES = {"bool": 0, "int8": 1, "int16": 2, "int32": 3, "int64": 4, "uint8": 5, "uint16": 6, "uint32": 7,
                "uint64": 8, "float16": 9, "bfloat16": 10, "float32": 11, "float64": 12}


class Core:
    """The engine's entry points with the reference extension's Python signatures."""

    def __init__(self, path: Path) -> None:
        L = ctypes.CDLL(str(path))
        vp, i32, i64, f64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
        L.eda_decompose.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, i64, ctypes.POINTER(i64),
                                    ctypes.POINTER(_Params), vp, ctypes.POINTER(vp)]
        L.eda_decompose_strided.argtypes = [vp, ctypes.POINTER(_Source), ctypes.c_int, ctypes.c_int,
                                            ctypes.POINTER(i64), ctypes.POINTER(_Params), vp, ctypes.POINTER(vp)]
        L.eda_run_shape.argtypes = [vp, ctypes.POINTER(i64), ctypes.POINTER(i32), ctypes.POINTER(i32),
                                    ctypes.POINTER(i64), ctypes.POINTER(i64)]
        L.eda_run_info.argtypes = [vp] + [vp] * 6
        L.eda_run_collect.argtypes = [vp, vp, ctypes.c_int, vp]
        L.eda_run_collect_orientation.argtypes = [vp, vp, vp, ctypes.c_int, vp]
        L.eda_run_free.argtypes = [vp]
        L.eda_run_free.restype = None
        L.eda_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
        L.eda_last_error.restype = ctypes.c_size_t
        L.eda_build_info.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
        L.eda_device_info.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t]
        L.eda_decompose_ragged.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_int, ctypes.c_int, i64,
                                           ctypes.POINTER(i64), ctypes.POINTER(_Params), i32, vp, ctypes.POINTER(vp)]
        L.eda_ragged_element.argtypes = [vp, i64] + [vp] * 7
        L.eda_ragged_collect.argtypes = [vp, i64, vp, ctypes.c_int, vp]
        L.eda_ragged_collect_all.argtypes = [vp, vp, ctypes.c_int, ctypes.POINTER(i64), vp]
        L.eda_monogenic.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, i64, ctypes.POINTER(i64), i64, vp,
                                    ctypes.c_int, ctypes.POINTER(i32), vp]
        L.eda_ragged_free.argtypes = [vp]
        L.eda_ragged_free.restype = None
        L.eda_set_transform_precision.argtypes = [ctypes.c_int]
        L.eda_transform_precision.argtypes = []
        L.eda_set_length_classes.argtypes = [i32]
        L.eda_length_classes.argtypes = []
        L.eda_buffer_alloc.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.POINTER(vp), ctypes.POINTER(vp)]
        L.eda_buffer_release.argtypes = [vp]
        L.eda_buffer_release.restype = None
        L.eda_buffer_dlpack.argtypes = [vp, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(i64), ctypes.POINTER(i64), ctypes.POINTER(vp)]
        L.eda_copy_to_host.argtypes = [vp, vp, ctypes.c_size_t, ctypes.c_int]
        L.eda_pointer_device.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
        L.eda_autotune.argtypes = [ctypes.c_int, ctypes.c_int, i64, ctypes.POINTER(i64), ctypes.c_char_p,
                                   ctypes.c_char_p, ctypes.c_size_t]
        L.eda_tuning_load.argtypes = [ctypes.c_char_p]
        L.eda_tuning_dump.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
        L.eda_tuning_clear.argtypes = []
        self._lib = L
        self.path = str(path)

    # -- device buffers of results (no array library needed) ------------------------------------
    def buffer_alloc(self, device: int, nbytes: int) -> tuple[int, int]:
        h, p = ctypes.c_void_p(), ctypes.c_void_p()
        self._check(self._lib.eda_buffer_alloc(int(device), int(nbytes), ctypes.byref(h), ctypes.byref(p)))
        return int(h.value), int(p.value or 0)

    def buffer_release(self, handle: int) -> None:
        self._lib.eda_buffer_release(ctypes.c_void_p(handle))

    def buffer_dlpack(self, handle: int, byte_offset: int, code: int, bits: int, shape, strides) -> int:
        nd = len(shape)
        sh = (ctypes.c_int64 * max(nd, 1))(*[int(v) for v in shape])
        st = (ctypes.c_int64 * max(nd, 1))(*[int(v) for v in strides])
        out = ctypes.c_void_p()
        self._check(self._lib.eda_buffer_dlpack(ctypes.c_void_p(handle), int(byte_offset), int(code), int(bits), nd,
                                                sh, st, ctypes.byref(out)))
        return int(out.value)

    def copy_to_host(self, dst: int, src: int, nbytes: int, device: int) -> None:
        self._check(self._lib.eda_copy_to_host(ctypes.c_void_p(dst), ctypes.c_void_p(src), int(nbytes), int(device)))

    def pointer_device(self, ptr: int) -> int:
        d = ctypes.c_int()
        self._check(self._lib.eda_pointer_device(ctypes.c_void_p(ptr), ctypes.byref(d)))
        return int(d.value)

    # -- the cube passes' autotuner ------------------------------------------------------------
    def autotune(self, dtype: str, shape: tuple[int, ...], batch: int, cache: str | None) -> dict:
        n = (ctypes.c_int64 * 3)(*[int(v) for v in shape], *([1] * (3 - len(shape))))
        buf = ctypes.create_string_buffer(1024)
        code = 0 if np.dtype(dtype) == np.float32 else 1
        self._check(self._lib.eda_autotune(code, len(shape), int(batch), n,
                                           None if cache is None else str(cache).encode(), buf, len(buf)))
        return json.loads(buf.value.decode())

    def tuning_load(self, path: str) -> None:
        self._check(self._lib.eda_tuning_load(str(path).encode()))

    def tuning_dump(self) -> str:
        buf = ctypes.create_string_buffer(1 << 16)
        self._check(self._lib.eda_tuning_dump(buf, len(buf)))
        return buf.value.decode()

    def tuning_clear(self) -> None:
        self._check(self._lib.eda_tuning_clear())

    # -- the float32 transforms' product ------------------------------------------------------
    def set_transform_precision(self, mode: int) -> None:
        self._check(self._lib.eda_set_transform_precision(int(mode)))

    def transform_precision(self) -> int:
        return int(self._lib.eda_transform_precision())

    # -- how ragged 1-D batches group their signals -------------------------------------------
    def set_length_classes(self, on: bool) -> None:
        self._check(self._lib.eda_set_length_classes(1 if on else 0))

    def length_classes(self) -> bool:
        return bool(self._lib.eda_length_classes())

    # -- errors --------------------------------------------------------------------------------
    def _check(self, status: int) -> None:
        if status == EDA_OK:
            return
        buf = ctypes.create_string_buffer(4096)
        self._lib.eda_last_error(buf, len(buf))
        msg = buf.value.decode(errors="replace")
        if status == EDA_INVALID_ARGUMENT:
            raise ValueError(msg)
        if status == EDA_OUT_OF_MEMORY:
            raise MemoryError(msg)
        if status == EDA_CUDA_ERROR:
            name = None
            if "CUDA error " in msg:
                name = msg.split("CUDA error ", 1)[1].split(" ", 1)[0]
            raise CudaError(msg, None, name)
        raise RuntimeError(msg)

    # -- information ---------------------------------------------------------------------------
    def build_info(self) -> dict:
        buf = ctypes.create_string_buffer(2048)
        self._lib.eda_build_info(buf, len(buf))
        info = json.loads(buf.value.decode())
        info["library"] = self.path
        return info

    def device_count(self) -> int:
        return int(self._lib.eda_device_count())

    def device_info(self, device: int = 0) -> dict:
        buf = ctypes.create_string_buffer(2048)
        self._check(self._lib.eda_device_info(int(device), buf, len(buf)))
        return json.loads(buf.value.decode())

    # -- the decomposition ---------------------------------------------------------------------
    def _run(self, ptr: int, on_device: bool, dtype: np.dtype, shape: tuple[int, ...], max_imf: int,
             tie_tolerance: float | None, sifts: int, check_finite: bool, max_chunk: int, stream: int,
             orientation: bool = False, layout=None):
        p = _Params(int(max_imf), -1.0 if tie_tolerance is None else float(tie_tolerance), int(sifts),
                    int(bool(check_finite)), int(max_chunk), int(bool(orientation)))
        n = (ctypes.c_int64 * 3)(*[int(v) for v in shape[1:]], *([1] * (4 - len(shape))))
        run = ctypes.c_void_p()
        code = 0 if dtype == np.float32 else 1
        if layout is None:
            self._check(self._lib.eda_decompose(ctypes.c_void_p(ptr), int(on_device), code, len(shape) - 1,
                                                int(shape[0]), n, ctypes.byref(p), ctypes.c_void_p(stream),
                                                ctypes.byref(run)))
            return run
        src_type, batch_shape, batch_stride, stride = layout
        k = len(batch_shape)
        bs = (ctypes.c_int64 * max(k, 1))(*[int(v) for v in batch_shape])
        bt = (ctypes.c_int64 * max(k, 1))(*[int(v) for v in batch_stride])
        st = (ctypes.c_int64 * 3)(*[int(v) for v in stride], *([0] * (3 - len(stride))))
        src = _Source(SOURCE_TYPES[src_type], k, bs, bt, st)
        self._check(self._lib.eda_decompose_strided(ctypes.c_void_p(ptr), ctypes.byref(src), code, len(shape) - 1,
                                                    n, ctypes.byref(p), ctypes.c_void_p(stream), ctypes.byref(run)))
        return run

    def _info(self, run) -> tuple[dict, int, int, int]:
        B, P, K, count, chunk = (ctypes.c_int64(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64(),
                                 ctypes.c_int64())
        self._check(self._lib.eda_run_shape(run, ctypes.byref(B), ctypes.byref(P), ctypes.byref(K),
                                            ctypes.byref(count), ctypes.byref(chunk)))
        b, k = B.value, K.value
        arr = {"n_imfs": np.zeros(b, np.int32), "error": np.zeros(b, np.int32),
               "windows": np.zeros((b, k), np.int32), "sifts": np.zeros((b, k), np.int32),
               "spacing": np.zeros((b, k), np.float64), "energy": np.zeros((b, k), np.float64)}
        self._check(self._lib.eda_run_info(run, *(ctypes.c_void_p(arr[n].ctypes.data) for n in
                                                  ("n_imfs", "error", "windows", "sifts", "spacing", "energy"))))
        arr["chunk"] = int(chunk.value)
        return arr, P.value, b, count.value

    @staticmethod
    def _empty_info(B: int) -> dict:
        z = np.zeros((B, 0))
        return {"n_imfs": np.zeros(B, np.int32), "error": np.zeros(B, np.int32), "windows": z.astype(np.int32),
                "sifts": z.astype(np.int32), "spacing": z, "energy": z.copy(), "chunk": 0}

    def decompose_host(self, x: np.ndarray, max_imf: int, tie_tolerance: float | None, sifts: int,
                       check_finite: bool, orientation: bool, max_chunk: int) -> tuple:
        """Decomposes the C-contiguous host array x (B, *spatial) of float32 or float64:
        (rows (B, P, *spatial), info)."""
        if not (isinstance(x, np.ndarray) and x.flags.c_contiguous and x.dtype in (np.float32, np.float64)):
            raise TypeError("eda: decompose_host: expected a C-contiguous float32 or float64 array")
        if x.ndim < 2 or x.ndim > 4:
            raise ValueError("eda: decompose_host: x must have the shape (B, *spatial) with 1 to 3 spatial axes")
        if x.shape[0] == 0:
            self._validate_empty(x, max_imf, tie_tolerance, sifts, check_finite, max_chunk)
            return np.zeros((0, 1) + x.shape[1:], x.dtype), self._empty_info(0)
        run = self._run(x.ctypes.data, False, x.dtype, x.shape, max_imf, tie_tolerance, sifts, check_finite,
                        max_chunk, 0, orientation)
        try:
            info, P, B, count = self._info(run)
            rows = np.empty((B, P) + x.shape[1:], x.dtype)
            self._check(self._lib.eda_run_collect(run, ctypes.c_void_p(rows.ctypes.data), 0, None))
            if orientation:
                K, D = info["windows"].shape[1], x.ndim - 1
                info["direction"] = np.zeros((B, K, D) + x.shape[1:], x.dtype)
                info["coherence"] = np.zeros((B, K) + x.shape[1:], x.dtype)
                if K:
                    self._check(self._lib.eda_run_collect_orientation(
                        run, ctypes.c_void_p(info["direction"].ctypes.data),
                        ctypes.c_void_p(info["coherence"].ctypes.data), 0, None))
        finally:
            self._lib.eda_run_free(run)
        return rows, info

    def _validate_empty(self, x, max_imf, tie_tolerance, sifts, check_finite, max_chunk) -> None:
        # an empty batch is validated as one element and computes nothing
        one = np.zeros((1,) + x.shape[1:], x.dtype)
        p = _Params(int(max_imf), -1.0 if tie_tolerance is None else float(tie_tolerance), int(sifts),
                    int(bool(check_finite)), int(max_chunk))
        del one, p
        for n in x.shape[1:]:
            if n < 2:
                raise ValueError("eda: every spatial axis needs extent >= 2")

    def decompose_device(self, ptr: int, device: int, dtype: str, shape: tuple[int, ...], max_imf: int,
                         tie_tolerance: float | None, sifts: int, check_finite: bool, max_chunk: int,
                         stream: int, out_ptr_of, orient_of=None, layout=None) -> tuple:
        """Decomposes the C-contiguous device array at ptr (B, *spatial) in the compute dtype on its
        device, or with ``layout`` = (source dtype name, batch shape, batch strides, spatial strides;
        strides in elements) the array at ptr in that layout, converted by the engine chunk by chunk;
        ``out_ptr_of(P)`` allocates the (B, P, *spatial) output and returns it with its pointer; with
        ``orient_of`` (return_orientation), ``orient_of(K)`` allocates the direction
        (B, K, D, *spatial) and coherence (B, K, *spatial) outputs and returns them with their
        pointers, kept in info["direction"] / info["coherence"]."""
        run = self._run(ptr, True, np.dtype(dtype), shape, max_imf, tie_tolerance, sifts, check_finite,
                        max_chunk, stream, orient_of is not None, layout)
        try:
            info, P, B, count = self._info(run)
            out, out_ptr = out_ptr_of(P)
            self._check(self._lib.eda_run_collect(run, ctypes.c_void_p(out_ptr), 1, ctypes.c_void_p(stream)))
            if orient_of is not None:
                K = info["windows"].shape[1]
                (d, d_ptr), (c, c_ptr) = orient_of(K)
                if K:
                    self._check(self._lib.eda_run_collect_orientation(run, ctypes.c_void_p(d_ptr),
                                                                      ctypes.c_void_p(c_ptr), 1,
                                                                      ctypes.c_void_p(stream)))
                info["direction"], info["coherence"] = d, c
        finally:
            self._lib.eda_run_free(run)
        return out, info


    def decompose_ragged(self, ptrs: list[int], on_device: bool, dtype: str, shapes: list[tuple[int, ...]],
                         max_imf: int, tie_tolerance: float | None, sifts: int, check_finite: bool, workers: int,
                         stream: int, alloc) -> list[tuple[Any, dict]]:
        """Decomposes len(ptrs) C-contiguous arrays of one dtype and one number of axes, each of its own
        shape, on the host or on the current device (ready once ``stream`` reaches the call);
        ``alloc(total)`` allocates one flat output of ``total`` samples (a NumPy array or a tensor)
        and returns it with its pointer: every element's rows are collected into it at once, and
        element i's (P_i, *shape_i) rows are a view of it. Returns (rows, info) per element; info
        holds ``n_imfs``, ``error`` and the ``windows``, ``sifts``, ``spacing``, ``energy`` of its IMFs."""
        count = len(ptrs)
        dim = len(shapes[0]) if count else 1
        p = _Params(int(max_imf), -1.0 if tie_tolerance is None else float(tie_tolerance), int(sifts),
                    int(bool(check_finite)), 0)
        xs = (ctypes.c_void_p * max(count, 1))(*[ctypes.c_void_p(int(v)) for v in ptrs])
        flat = [int(v) for sh in shapes for v in sh]
        n = (ctypes.c_int64 * max(len(flat), 1))(*flat)
        run = ctypes.c_void_p()
        code = 0 if np.dtype(dtype) == np.float32 else 1
        self._check(self._lib.eda_decompose_ragged(xs, int(on_device), code, dim, count, n, ctypes.byref(p),
                                                   int(workers), ctypes.c_void_p(stream), ctypes.byref(run)))
        infos, rows_of = [], []
        try:
            for i in range(count):
                P, k, err = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
                self._check(self._lib.eda_ragged_element(run, i, ctypes.byref(P), ctypes.byref(k), ctypes.byref(err),
                                                         None, None, None, None))
                K = 0 if err.value else k.value
                info = {"n_imfs": int(k.value), "error": int(err.value), "windows": np.zeros(K, np.int32),
                        "sifts": np.zeros(K, np.int32), "spacing": np.zeros(K, np.float64),
                        "energy": np.zeros(K, np.float64)}
                if K:
                    self._check(self._lib.eda_ragged_element(
                        run, i, None, None, None, *(ctypes.c_void_p(info[f].ctypes.data) for f in
                                                    ("windows", "sifts", "spacing", "energy"))))
                infos.append(info)
                rows_of.append(int(P.value))
            sizes = [P * int(np.prod(sh)) for P, sh in zip(rows_of, shapes)]
            offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64) if count else np.zeros(1, np.int64)
            buf, ptr = alloc(int(offsets[-1]))
            if count:
                self._check(self._lib.eda_ragged_collect_all(
                    run, ctypes.c_void_p(ptr), int(on_device), offsets.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                    ctypes.c_void_p(stream)))
        finally:
            self._lib.eda_ragged_free(run)
        return [(buf[int(offsets[i]):int(offsets[i + 1])].reshape((rows_of[i],) + tuple(shapes[i])), infos[i])
                for i in range(count)]


    def monogenic(self, ptr: int, on_device: bool, dtype: str, shape: tuple[int, ...], stream: int, out_ptr: int,
                  max_chunk: int = 0) -> np.ndarray:
        """The monogenic planes of the C-contiguous (B, *spatial) array at ptr into the buffer at
        out_ptr (host memory, or device memory for device input); returns the non-finite flags [B]."""
        B = int(shape[0])
        n = (ctypes.c_int64 * 3)(*[int(v) for v in shape[1:]], *([1] * (4 - len(shape))))
        bad = np.zeros(max(B, 1), np.int32)
        code = 0 if np.dtype(dtype) == np.float32 else 1
        self._check(self._lib.eda_monogenic(ctypes.c_void_p(ptr), int(on_device), code, len(shape) - 1, B, n,
                                            int(max_chunk), ctypes.c_void_p(out_ptr), int(on_device),
                                            bad.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                            ctypes.c_void_p(stream)))
        return bad[:B]


def core() -> Core:
    """The engine, loaded on first use (ImportError when the library is not built)."""
    global _core
    if _core is None:
        if not LIB.exists():
            raise ImportError(
                f"eda: the B200 engine library is not built ({LIB}); build it with "
                "`python eda-cuda_b200/build.py` (nvcc for sm_100a)")
        try:
            _core = Core(LIB)
        except OSError as exc:
            raise ImportError(f"eda: the B200 engine library cannot be loaded: {exc}") from exc
    return _core
