# SPDX-License-Identifier: Apache-2.0
"""``eda.decompose`` on the B200 engine: the public argument rules, layouts, errors and result
types of the reference's call (src/eda/_api.py:184-353 of eda-cuda), written over this engine's
binding (_native.py)."""

from __future__ import annotations

import math
import operator
from collections.abc import Sequence
from dataclasses import dataclass
from typing import Any

import numpy as np

from . import _device, _native
from ._errors import DecompositionError

#: Error codes of an element (``DecompositionInfo.error``).
ERROR_NON_FINITE = 1
ERROR_NON_FINITE_RESULT = 2
ERROR_INTERNAL = 255
_MESSAGES = {
    ERROR_NON_FINITE: "the input has inf or NaN; check_finite=True",
    ERROR_NON_FINITE_RESULT: (
        "a non-finite intermediate or output row: the decomposition overflows the dtype's range, "
        "or the input has inf or NaN with check_finite=False"
    ),
}
_FLOATS = ("float32", "float64")
_INT32_MAX = 2**31 - 1


@dataclass(frozen=True, eq=False)
class DecompositionInfo:
    """Per-call information of ``eda.decompose(..., return_info=True)``: ``n_imfs`` and ``error`` of
    the batch shape; ``windows``, ``spacing``, ``sifts``, ``energy`` of the batch shape plus K (the
    largest IMF count), zero beyond an element's ``n_imfs`` and for a failed element; ``dtype``, the
    compute dtype; ``axes``, the spatial axes."""

    n_imfs: np.ndarray
    error: np.ndarray
    windows: np.ndarray
    spacing: np.ndarray
    sifts: np.ndarray
    energy: np.ndarray
    dtype: str
    axes: tuple[int, ...]


@dataclass(frozen=True, eq=False)
class Orientation:
    """Every mode's orientation, from ``eda.decompose(..., return_orientation=True)`` (2 or 3 spatial
    axes), laid out as the reference's (src/eda/_api.py:65-83 of eda-cuda): with ``m = min(axes)``
    and K the largest IMF count of the call, ``direction`` has the shape
    ``x.shape[:m] + (K, D) + x.shape[m:]`` (the unit direction n across the stripes that the method
    computes at the start of each mode, component a along the a-th axis of ``axes``, the first
    component of magnitude above the dtype's default tie tolerance positive) and ``coherence``
    ``x.shape[:m] + (K,) + x.shape[m:]`` (0: no direction, 1: perfect stripes). Rows beyond an
    element's ``n_imfs`` and all rows of a failed element are 0. NumPy arrays for host input,
    ``eda.DeviceArray`` for CUDA input, in the compute dtype."""

    direction: Any
    coherence: Any


@dataclass(frozen=True, eq=False)
class Monogenic:
    """The monogenic signal of every field, from ``eda.monogenic`` (the reference's type,
    src/eda/_api.py:86-102 of eda-cuda): ``amplitude``, ``phase`` in (-pi, pi] and ``frequency``
    (cycles per sample along ``direction``) of the shape of ``x``; in 2-D and 3-D ``direction`` of
    the shape ``x.shape[:m] + (D,) + x.shape[m:]`` (m = min(axes); the unit direction across the
    local stripes, its first component of magnitude above the dtype's default tie tolerance
    positive) and ``coherence`` of the shape of ``x`` (0: no direction, 1: perfect stripes);
    ``None`` in 1-D. NumPy arrays for host input, ``eda.DeviceArray`` for CUDA input."""

    amplitude: Any
    phase: Any
    frequency: Any
    direction: Any
    coherence: Any


def _int_arg(value: Any, name: str) -> int:
    if isinstance(value, (bool, np.bool_)):
        raise TypeError(f"eda: {name} must be an integer, not bool")
    try:
        return operator.index(value)
    except TypeError:
        raise TypeError(f"eda: {name} must be an integer, got {type(value).__name__}") from None


def _flag(value: Any, name: str) -> bool:
    if not isinstance(value, (bool, np.bool_)):
        raise TypeError(f"eda: {name} must be True or False, got {type(value).__name__}")
    return bool(value)


def _tie(value: Any) -> float | None:
    if value is None:
        return None
    if isinstance(value, (bool, np.bool_)) or not isinstance(value, (int, float, np.integer, np.floating)):
        raise TypeError(f"eda: tie_tolerance must be a real number or None, got {type(value).__name__}")
    try:
        number = float(value)
    except OverflowError:
        number = math.inf
    if not (math.isfinite(number) and number >= 0):
        raise ValueError(f"eda: tie_tolerance must be a finite number >= 0, got {value}")
    return number


def _axes(axes: Any, ndim: int) -> tuple[int, ...]:
    if ndim < 1:
        raise ValueError("eda: expected an array with at least one dimension")
    if axes is None:
        if ndim > 3:
            raise ValueError(f"eda: axes=None takes every axis and needs x.ndim <= 3, got {ndim}: name the "
                             "spatial axes (1 to 3) with axes=")
        return tuple(range(ndim))
    if isinstance(axes, (int, np.integer)) and not isinstance(axes, bool):
        axes = (axes,)
    try:
        listed = []
        for a in axes:
            if isinstance(a, (bool, np.bool_)):
                raise TypeError
            listed.append(operator.index(a))
    except TypeError:
        raise TypeError(f"eda: axes must be an int, a sequence of ints or None, got {type(axes).__name__}") from None
    out = []
    for a in listed:
        if not -ndim <= a < ndim:
            raise np.exceptions.AxisError(a, ndim, "eda")
        out.append(a % ndim)
    if len(set(out)) != len(out):
        raise ValueError(f"eda: axes must be unique, got {tuple(listed)}")
    if not 1 <= len(out) <= 3:
        raise ValueError(f"eda: 1 to 3 spatial axes, got {len(out)}")
    return tuple(out)


def _restore(ndim: int, batch_axes: tuple[int, ...], axes: tuple[int, ...], extra: int = 1) -> list[int]:
    """The permutation from the computed (*batch, *extra, *spatial in axes order) layout to the
    public one: x's axes in order, the extra axes just before min(axes)."""
    nb = len(batch_axes)
    where = {a: nb + extra + k for k, a in enumerate(axes)}
    where.update({a: k for k, a in enumerate(batch_axes)})
    m = min(axes)
    return [where[f] for f in range(m)] + [nb + j for j in range(extra)] + [where[f] for f in range(m, ndim)]


def _dtype_name(dtype: Any) -> str:
    try:
        return np.dtype(dtype).name
    except TypeError:
        return str(dtype).removeprefix("torch.")


def _stream_handle(stream: Any, default: int | None) -> int:
    """A raw CUDA stream handle from an int, a torch / CuPy stream object, or the default."""
    if stream is None:
        return int(default or 0)
    for attr in ("cuda_stream", "ptr", "handle"):
        if hasattr(stream, attr):
            return int(getattr(stream, attr))
    return int(stream)


def _c_contiguous(shape: Sequence[int], strides: Sequence[int]) -> bool:
    expect = 1
    for n, st in zip(reversed(list(shape)), reversed(list(strides))):
        if n != 1 and st != expect:
            return False
        expect *= n
    return True


def _wrap(a: Any) -> Any:
    return a if isinstance(a, _device.DeviceArray) else _device.DeviceArray(a)


def decompose(
    x: Any,
    axes: int | Sequence[int] | None = None,
    max_imf: int = -1,
    *,
    dtype: Any = None,
    tie_tolerance: float | None = None,
    sifts: int = 3,
    check_finite: bool = True,
    errors: str = "raise",
    stream: Any = None,
    return_info: bool = False,
    return_orientation: bool = False,
) -> Any:
    """Decompose every 1-D, 2-D or 3-D field of ``x`` into intrinsic mode functions (IMFs) and a
    residue, on the B200 engine. The arguments, the result layout
    (``x.shape[:m] + (P,) + x.shape[m:]``, ``m = min(axes)``; the IMFs fine to coarse, then the
    residue, then zero rows), the information, the orientation (``return_orientation``, 2 or 3 axes:
    an ``Orientation`` after the information) and the error rules are those of the reference's
    ``eda.decompose``; asking for the orientation does not change ``y`` or ``info``."""
    max_imf = max(-_INT32_MAX - 1, min(_int_arg(max_imf, "max_imf"), _INT32_MAX))
    tie = _tie(tie_tolerance)
    sifts = _int_arg(sifts, "sifts")
    if not 1 <= sifts <= _INT32_MAX:
        raise ValueError(f"eda: sifts must be an integer from 1 to {_INT32_MAX}, got {sifts}")
    check_finite = _flag(check_finite, "check_finite")
    return_info = _flag(return_info, "return_info")
    return_orientation = _flag(return_orientation, "return_orientation")
    if not isinstance(errors, str) or errors not in ("raise", "status"):
        raise ValueError(f"eda: errors={errors!r} is not one of 'raise', 'status'")
    on_device = _device.is_cuda_array(x)
    if on_device and not _device.is_torch(x):
        # any other CUDA array: read through the CUDA array interface or DLPack, without PyTorch
        cin = _device.intake(x)
        try:
            return _decompose_cuda(cin, axes, max_imf, dtype, tie, sifts, check_finite, errors, stream, return_info,
                                   return_orientation)
        finally:
            cin.release()
    if on_device:
        data = _device.as_tensor(x)
        src = _device.dtype_name(data)
        if src not in _device.SUPPORTED_DTYPES:
            raise TypeError(f"eda: arrays of dtype {src} are not supported (real bool, integer and float arrays only)")
    else:
        data = np.asarray(x)
        src = data.dtype.name
        if data.dtype.kind not in "biuf":
            raise TypeError(f"eda: arrays of dtype {src} are not supported (real bool, integer and float arrays only)")
    target = src if dtype is None else _dtype_name(dtype)
    if target not in _FLOATS:
        if dtype is None:
            raise TypeError(f"eda: expected a float32 or float64 array, got dtype {src} (pass dtype='float32' or "
                            "dtype='float64' to cast it)")
        raise TypeError(f"eda: dtype= must be float32 or float64, got {target}")
    ndim = len(data.shape)
    axes = _axes(axes, ndim)
    if return_orientation and len(axes) < 2:
        raise ValueError("eda: return_orientation=True needs 2 or 3 spatial axes, got 1 (the method has no "
                         "orientation in 1-D)")
    batch_axes = tuple(i for i in range(ndim) if i not in axes)
    batch_shape = tuple(int(data.shape[i]) for i in batch_axes)
    spatial = tuple(int(data.shape[a]) for a in axes)
    B = math.prod(batch_shape)
    order = list(batch_axes) + list(axes)
    core = _native.core()
    if on_device:
        torch = _device._torch()
        tdt = getattr(torch, target)
        t = data.permute(order) if order != list(range(ndim)) else data
        layout = None
        if t.dtype == tdt and t.is_contiguous():
            t = t.reshape((B,) + spatial)  # read in place
        else:
            # any other element type or layout: the engine gathers and casts each chunk itself
            # (cpp/src/field/convert.cu:69-170 of the reference), no converted copy of x is made
            layout = (src, batch_shape, tuple(int(data.stride(i)) for i in batch_axes),
                      tuple(int(data.stride(a)) for a in axes))
        dev = t.device
        if B == 0:
            rows_t, raw = torch.zeros((0, 1) + spatial, dtype=tdt, device=dev), core._empty_info(0)
        else:
            with torch.cuda.device(dev):
                st = torch.cuda.current_stream(dev)

                def alloc(P):
                    out = torch.empty((B, P) + spatial, dtype=tdt, device=dev)
                    return out, out.data_ptr()

                def orient_of(K):
                    d = torch.zeros((B, K, len(spatial)) + spatial, dtype=tdt, device=dev)
                    c = torch.zeros((B, K) + spatial, dtype=tdt, device=dev)
                    return (d, d.data_ptr()), (c, c.data_ptr())

                rows_t, raw = core.decompose_device(t.data_ptr(), dev.index or 0, target, (B,) + spatial, max_imf,
                                                    tie, sifts, check_finite, 0, st.cuda_stream, alloc,
                                                    orient_of if return_orientation else None, layout)
    else:
        xc = data if data.dtype == np.dtype(target) else data.astype(target)
        xt = np.ascontiguousarray(xc.transpose(order)) if order != list(range(ndim)) else xc
        xb = np.ascontiguousarray(xt).reshape((B,) + spatial)
        rows, raw = core.decompose_host(xb, max_imf, tie, sifts, check_finite, return_orientation, 0)
    return _finish(raw, rows_t if on_device else rows, on_device, batch_shape, batch_axes, axes, spatial, ndim, target,
                   errors, return_info, return_orientation)


def _decompose_cuda(cin, axes, max_imf, dtype, tie, sifts, check_finite, errors, stream, return_info,
                    return_orientation):
    """eda.decompose of a CUDA array that is not a torch tensor (DLPack or the CUDA array interface):
    read in place where it is a C-contiguous array of the compute dtype, else gathered and cast by the
    engine chunk by chunk (eda_decompose_strided); the results in engine-allocated DeviceArrays. The
    engine runs on the array's stream (the CUDA array interface's, else ``stream``, else the legacy
    default stream), so it is ordered after the producer's work."""
    src = cin.dtype
    if src not in _device.SUPPORTED_DTYPES:
        raise TypeError(f"eda: arrays of dtype {src} are not supported (real bool, integer and float arrays only)")
    target = src if dtype is None else _dtype_name(dtype)
    if target not in _FLOATS:
        if dtype is None:
            raise TypeError(f"eda: expected a float32 or float64 array, got dtype {src} (pass dtype='float32' or "
                            "dtype='float64' to cast it)")
        raise TypeError(f"eda: dtype= must be float32 or float64, got {target}")
    ndim = len(cin.shape)
    axes = _axes(axes, ndim)
    if return_orientation and len(axes) < 2:
        raise ValueError("eda: return_orientation=True needs 2 or 3 spatial axes, got 1 (the method has no "
                         "orientation in 1-D)")
    batch_axes = tuple(i for i in range(ndim) if i not in axes)
    batch_shape = tuple(int(cin.shape[i]) for i in batch_axes)
    spatial = tuple(int(cin.shape[a]) for a in axes)
    B = math.prod(batch_shape)
    order = list(batch_axes) + list(axes)
    layout = None
    if not (src == target and _c_contiguous([cin.shape[i] for i in order], [cin.strides[i] for i in order])):
        layout = (src, batch_shape, tuple(int(cin.strides[i]) for i in batch_axes),
                  tuple(int(cin.strides[a]) for a in axes))
    core = _native.core()
    dev = cin.device
    if B == 0:
        rows_t, raw = _device.DeviceArray.empty((0, 1) + spatial, target, dev), core._empty_info(0)
    else:
        def alloc(P):
            out = _device.DeviceArray.empty((B, P) + spatial, target, dev)
            return out, out.ptr

        def orient_of(K):
            d = _device.DeviceArray.empty((B, K, len(spatial)) + spatial, target, dev)
            c = _device.DeviceArray.empty((B, K) + spatial, target, dev)
            return (d, d.ptr), (c, c.ptr)

        rows_t, raw = core.decompose_device(cin.ptr, dev, target, (B,) + spatial, max_imf, tie, sifts, check_finite,
                                            0, _stream_handle(stream, cin.stream), alloc,
                                            orient_of if return_orientation else None, layout)
    return _finish(raw, rows_t, True, batch_shape, batch_axes, axes, spatial, ndim, target, errors, return_info,
                   return_orientation)


def _finish(raw, rows, on_device, batch_shape, batch_axes, axes, spatial, ndim, target, errors, return_info,
            return_orientation):
    """The result of a call: the information, the error policy, the rows in the caller's layout and
    the orientation."""
    rows_t = rows
    info = DecompositionInfo(
        n_imfs=np.asarray(raw["n_imfs"], np.int32).reshape(batch_shape),
        error=np.asarray(raw["error"], np.int32).reshape(batch_shape),
        windows=np.asarray(raw["windows"], np.int32).reshape(batch_shape + raw["windows"].shape[1:]),
        spacing=np.asarray(raw["spacing"], np.float64).reshape(batch_shape + raw["spacing"].shape[1:]),
        sifts=np.asarray(raw["sifts"], np.int32).reshape(batch_shape + raw["sifts"].shape[1:]),
        energy=np.asarray(raw["energy"], np.float64).reshape(batch_shape + raw["energy"].shape[1:]),
        dtype=target,
        axes=axes,
    )
    codes = info.error.reshape(-1)
    internal = np.flatnonzero(codes == ERROR_INTERNAL)
    if internal.size:
        raise RuntimeError("eda: an internal invariant failed (error code 255) for batch index "
                           f"{', '.join(str(int(i)) for i in internal[:8])}: this is a bug in eda")
    failed = np.flatnonzero(codes != 0)
    if failed.size and errors == "raise":
        parts = []
        for code in sorted({int(c) for c in codes[failed]}):
            where = failed[codes[failed] == code]
            shown = ", ".join(str(int(i)) for i in where[:8]) + (", ..." if where.size > 8 else "")
            parts.append(f"code {code} ({_MESSAGES.get(code, f'error code {code}')}) at batch index {shown}")
        raise DecompositionError(
            f"eda: the decomposition failed for {failed.size} of {codes.size} element(s): " + "; ".join(parts),
            indices=failed, codes=codes[failed], info=info)
    perm = _restore(ndim, batch_axes, axes)
    if on_device:
        P = rows_t.shape[1]
        y_t = rows_t.reshape(batch_shape + (P,) + spatial)
        if perm != list(range(ndim + 1)):
            y_t = y_t.permute(perm)
        y = _wrap(y_t)
    else:
        P = rows.shape[1]
        y = rows.reshape(batch_shape + (P,) + spatial)
        if perm != list(range(ndim + 1)):
            y = y.transpose(perm)
    out: tuple = (y,)
    if return_info:
        out += (info,)
    if return_orientation:
        K = info.windows.shape[-1]
        D = len(spatial)
        parts = []
        for name, extra, shape in (("direction", 2, batch_shape + (K, D) + spatial),
                                   ("coherence", 1, batch_shape + (K,) + spatial)):
            a = raw[name]
            p2 = _restore(ndim, batch_axes, axes, extra)
            if on_device:
                a = a.reshape(shape)
                parts.append(_wrap(a.permute(p2) if p2 != list(range(len(p2))) else a))
            else:
                a = np.asarray(a).reshape(shape)
                parts.append(a.transpose(p2) if p2 != list(range(len(p2))) else a)
        out += (Orientation(*parts),)
    return out if len(out) > 1 else y


def decompose_ragged(
    xs: Sequence[Any],
    max_imf: int = -1,
    *,
    dtype: Any = None,
    tie_tolerance: float | None = None,
    sifts: int = 3,
    check_finite: bool = True,
    errors: str = "raise",
    return_info: bool = False,
    workers: int = 8,
) -> Any:
    """Decompose a ragged batch: ``xs`` is a sequence of fields of different shapes (each one field
    with 1, 2 or 3 axes, all with the same number of axes, all NumPy arrays or all CUDA arrays on
    one device). Returns the list of each field's rows ``(P_i, *x_i.shape)`` (P_i = its IMF count
    plus the residue; a failed field's row is NaN), and with ``return_info`` the list of its
    ``DecompositionInfo`` (batch shape ``()``). Every field's result is the one ``eda.decompose``
    gives for it alone; the fields are grouped (2-D and 3-D fields by shape; 1-D signals by length
    class [2^k, 2^(k+1)), each class one batch of uneven lengths, see ``eda.set_length_classes``)
    and up to ``workers`` groups run concurrently on the GPU. The argument and error rules are those of ``eda.decompose``
    (``errors='raise'`` raises DecompositionError naming the failed indices)."""
    max_imf = max(-_INT32_MAX - 1, min(_int_arg(max_imf, "max_imf"), _INT32_MAX))
    tie = _tie(tie_tolerance)
    sifts = _int_arg(sifts, "sifts")
    if not 1 <= sifts <= _INT32_MAX:
        raise ValueError(f"eda: sifts must be an integer from 1 to {_INT32_MAX}, got {sifts}")
    check_finite = _flag(check_finite, "check_finite")
    return_info = _flag(return_info, "return_info")
    workers = _int_arg(workers, "workers")
    if workers < 1:
        raise ValueError(f"eda: workers must be >= 1, got {workers}")
    if not isinstance(errors, str) or errors not in ("raise", "status"):
        raise ValueError(f"eda: errors={errors!r} is not one of 'raise', 'status'")
    if isinstance(xs, np.ndarray) or not isinstance(xs, Sequence):
        raise TypeError("eda: decompose_ragged expects a sequence of arrays (a list or tuple)")
    items = list(xs)
    if not items:
        return ([], []) if return_info else []
    on_device = [_device.is_cuda_array(x) for x in items]
    if any(on_device) and not all(on_device):
        raise ValueError("eda: decompose_ragged needs all fields on the host or all on one CUDA device")
    dev = all(on_device)
    fields, srcs = [], []
    for x in items:
        if dev:
            data = _device.as_tensor(x)
            src = _device.dtype_name(data)
            if src not in _device.SUPPORTED_DTYPES:
                raise TypeError(f"eda: arrays of dtype {src} are not supported (real bool, integer and float arrays only)")
        else:
            data = np.asarray(x)
            src = data.dtype.name
            if data.dtype.kind not in "biuf":
                raise TypeError(f"eda: arrays of dtype {src} are not supported (real bool, integer and float arrays only)")
        fields.append(data)
        srcs.append(src)
    if dtype is None and len(set(srcs)) != 1:
        raise TypeError(f"eda: the fields have different dtypes {sorted(set(srcs))}; pass dtype= to cast them")
    target = srcs[0] if dtype is None else _dtype_name(dtype)
    if target not in _FLOATS:
        if dtype is None:
            raise TypeError(f"eda: expected float32 or float64 arrays, got dtype {target} (pass dtype='float32' or "
                            "dtype='float64' to cast them)")
        raise TypeError(f"eda: dtype= must be float32 or float64, got {target}")
    ndims = {len(f.shape) for f in fields}
    if len(ndims) != 1 or not 1 <= next(iter(ndims)) <= 3:
        raise ValueError("eda: every field of a ragged batch has the same number of axes, 1 to 3")
    core = _native.core()
    shapes = [tuple(int(v) for v in f.shape) for f in fields]
    if dev:
        torch = _device._torch()
        tdt = getattr(torch, target)
        ts = [f.to(tdt).contiguous() for f in fields]
        device = ts[0].device
        if any(t.device != device for t in ts):
            raise ValueError("eda: decompose_ragged needs all CUDA fields on one device")
        with torch.cuda.device(device):
            st = torch.cuda.current_stream(device)

            def alloc(total):
                out = torch.empty((max(total, 1),), dtype=tdt, device=device)
                return out, out.data_ptr()

            res = core.decompose_ragged([t.data_ptr() for t in ts], True, target, shapes, max_imf, tie, sifts,
                                        check_finite, workers, st.cuda_stream, alloc)
        rows = [_device.DeviceArray(r) for r, _ in res]
    else:
        hs = [np.ascontiguousarray(f if f.dtype == np.dtype(target) else f.astype(target)) for f in fields]

        def alloc(total):
            out = np.empty((max(total, 1),), target)
            return out, out.ctypes.data

        res = core.decompose_ragged([h.ctypes.data for h in hs], False, target, shapes, max_imf, tie, sifts,
                                    check_finite, workers, 0, alloc)
        rows = [r for r, _ in res]
    infos = []
    for (_, raw), shape in zip(res, shapes):
        infos.append(DecompositionInfo(
            n_imfs=np.asarray(raw["n_imfs"], np.int32), error=np.asarray(raw["error"], np.int32),
            windows=raw["windows"], spacing=raw["spacing"], sifts=raw["sifts"], energy=raw["energy"],
            dtype=target, axes=tuple(range(len(shape)))))
    codes = np.asarray([int(i.error) for i in infos], np.int32)
    internal = np.flatnonzero(codes == ERROR_INTERNAL)
    if internal.size:
        raise RuntimeError("eda: an internal invariant failed (error code 255) for field index "
                           f"{', '.join(str(int(i)) for i in internal[:8])}: this is a bug in eda")
    failed = np.flatnonzero(codes != 0)
    if failed.size and errors == "raise":
        parts = []
        for code in sorted({int(c) for c in codes[failed]}):
            where = failed[codes[failed] == code]
            shown = ", ".join(str(int(i)) for i in where[:8]) + (", ..." if where.size > 8 else "")
            parts.append(f"code {code} ({_MESSAGES.get(code, f'error code {code}')}) at field index {shown}")
        raise DecompositionError(
            f"eda: the decomposition failed for {failed.size} of {codes.size} field(s): " + "; ".join(parts),
            indices=failed, codes=codes[failed], info=infos)
    return (rows, infos) if return_info else rows


def monogenic(
    x: Any,
    axes: int | Sequence[int] | None = None,
    *,
    dtype: Any = None,
    check_finite: bool = True,
    stream: Any = None,
) -> Monogenic:
    """The monogenic signal of every 1-D, 2-D or 3-D field of ``x`` (the reference's
    ``eda.monogenic``, src/eda/_api.py:356-426 of eda-cuda): with R1 the first-order and R2 the
    second-order Riesz transforms (half-sample symmetric extension), n the top eigenvector of
    T = R1 R1^T + R2 R2^T (1 in 1-D) and q = n . R1: amplitude sqrt(f^2 + |R1|^2), phase
    atan2(q, f), frequency (f dq/dn - q df/dn) / (2 pi amplitude^2) (0 where the amplitude vanishes),
    direction n and coherence (mu1 - mu2) / (mu1 + mu2). ``x``, ``axes``, ``dtype`` and
    ``check_finite`` follow ``eda.decompose``; a field with inf or NaN raises ValueError with
    ``check_finite=True``. Each field's result does not depend on the batch around it."""
    check_finite = _flag(check_finite, "check_finite")
    on_device = _device.is_cuda_array(x)
    if on_device:
        data = _device.as_tensor(x)
        src = _device.dtype_name(data)
        if src not in _device.SUPPORTED_DTYPES:
            raise TypeError(f"eda: arrays of dtype {src} are not supported (real bool, integer and float arrays only)")
    else:
        data = np.asarray(x)
        src = data.dtype.name
        if data.dtype.kind not in "biuf":
            raise TypeError(f"eda: arrays of dtype {src} are not supported (real bool, integer and float arrays only)")
    target = src if dtype is None else _dtype_name(dtype)
    if target not in _FLOATS:
        if dtype is None:
            raise TypeError(f"eda: expected a float32 or float64 array, got dtype {src} (pass dtype='float32' or "
                            "dtype='float64' to cast it)")
        raise TypeError(f"eda: dtype= must be float32 or float64, got {target}")
    ndim = len(data.shape)
    axes = _axes(axes, ndim)
    batch_axes = tuple(i for i in range(ndim) if i not in axes)
    batch_shape = tuple(int(data.shape[i]) for i in batch_axes)
    spatial = tuple(int(data.shape[a]) for a in axes)
    B = math.prod(batch_shape)
    D = len(spatial)
    count = math.prod(spatial)
    order = list(batch_axes) + list(axes)
    core = _native.core()
    planes = 3 if D == 1 else 4 + D
    if on_device:
        torch = _device._torch()
        tdt = getattr(torch, target)
        t = data.permute(order) if order != list(range(ndim)) else data
        # the monogenic call reads C-contiguous arrays of the compute dtype: any other element type
        # or layout is cast and copied first
        t = t.to(tdt).contiguous().reshape((B,) + spatial)
        dev = t.device
        flat = torch.empty(planes * B * count, dtype=tdt, device=dev)
        if B:
            with torch.cuda.device(dev):
                st = torch.cuda.current_stream(dev)
                bad = core.monogenic(t.data_ptr(), True, target, (B,) + spatial, st.cuda_stream, flat.data_ptr())
        else:
            bad = np.zeros(0, np.int32)
    else:
        xc = data if data.dtype == np.dtype(target) else data.astype(target)
        xt = np.ascontiguousarray(xc.transpose(order)) if order != list(range(ndim)) else xc
        xb = np.ascontiguousarray(xt).reshape((B,) + spatial)
        flat = np.empty(planes * B * count, target)
        bad = core.monogenic(xb.ctypes.data, False, target, (B,) + spatial, 0, flat.ctypes.data) if B else \
            np.zeros(0, np.int32)
    idx = np.flatnonzero(bad)
    if check_finite and idx.size:
        shown = ", ".join(str(int(i)) for i in idx[:8]) + (", ..." if idx.size > 8 else "")
        raise ValueError(f"eda: the input has inf or NaN at batch index {shown} ({idx.size} of {B} field(s)); "
                         "check_finite=True")
    out, offset = [], 0
    n = B * count
    for comps in ((0, 0, 0, D, 0) if D >= 2 else (0, 0, 0)):
        extra = (comps,) if comps else ()
        shape = batch_shape + extra + spatial
        perm = _restore(ndim, batch_axes, axes, len(extra)) if extra else _restore(ndim, batch_axes, axes, 0)
        part = flat[offset: offset + n * max(comps, 1)].reshape(shape)
        if on_device:
            out.append(_device.DeviceArray(part.permute(perm) if perm != list(range(len(perm))) else part))
        else:
            out.append(part.transpose(perm) if perm != list(range(len(perm))) else part)
        offset += n * max(comps, 1)
    return Monogenic(*out) if D >= 2 else Monogenic(*out, None, None)
