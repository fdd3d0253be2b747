# SPDX-License-Identifier: Apache-2.0
"""CUDA arrays in and out, as the reference's device layer does (src/eda/_device.py:99-334 of
eda-cuda). A torch tensor is read through PyTorch (its current stream, no copy). Any other CUDA
array (CuPy, Numba, JAX, another library's DLPack export) is read by ``eda.decompose`` directly,
without PyTorch, through the CUDA array interface (versions 2 and 3, with its stream) or DLPack (the
capsule's DLManagedTensor, consumed and released after the call). Results of CUDA input are
``DeviceArray`` objects that export DLPack and the CUDA array interface; for torch input they wrap a
torch tensor, otherwise a buffer allocated by the engine (libeda_b200.so) that lives as long as the
array, its views, or any tensor exported from it."""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from typing import Any

import numpy as np

#: The dtype names a CUDA array may have (cast to the compute dtype on the GPU).
SUPPORTED_DTYPES = frozenset(("bool", "int8", "int16", "int32", "int64", "uint8", "uint16", "uint32", "uint64",
                              "float16", "bfloat16", "float32", "float64"))

_KDL_CUDA, _KDL_CUDA_MANAGED = 2, 13


def _torch():
    import torch

    return torch


def is_torch(x: Any) -> bool:
    return type(x).__module__.startswith("torch") and hasattr(x, "is_cuda")


def is_cuda_array(x: Any) -> bool:
    """Whether x is a CUDA array (device input)."""
    if is_torch(x):
        return bool(x.is_cuda)
    if hasattr(x, "__dlpack_device__"):
        try:
            dev_type, _ = x.__dlpack_device__()
            return int(dev_type) in (_KDL_CUDA, _KDL_CUDA_MANAGED)
        except Exception:
            return False
    return hasattr(x, "__cuda_array_interface__")


def as_tensor(x: Any):
    """The CUDA array x as a torch tensor (no copy): x itself for a torch tensor, else through DLPack
    or the CUDA array interface (the PyTorch path of decompose_ragged and monogenic)."""
    if is_torch(x):
        return x
    torch = _torch()
    if hasattr(x, "__dlpack__"):
        return torch.from_dlpack(x)
    return torch.as_tensor(x, device="cuda")


def dtype_name(t: Any) -> str:
    return str(t.dtype).removeprefix("torch.")


def c_strides(shape: tuple[int, ...]) -> tuple[int, ...]:
    """The strides (elements) of a C-contiguous array of this shape."""
    out, acc = [], 1
    for n in reversed(shape):
        out.append(acc)
        acc *= max(int(n), 1)
    return tuple(reversed(out))


# ---------------------------------------------------------------------------------------------
# intake without PyTorch

_TYPESTR = {"b1": "bool", "i1": "int8", "i2": "int16", "i4": "int32", "i8": "int64", "u1": "uint8", "u2": "uint16",
            "u4": "uint32", "u8": "uint64", "f2": "float16", "f4": "float32", "f8": "float64"}
_DL_TYPES = {(0, 8): "int8", (0, 16): "int16", (0, 32): "int32", (0, 64): "int64", (1, 8): "uint8", (1, 16): "uint16",
             (1, 32): "uint32", (1, 64): "uint64", (2, 16): "float16", (2, 32): "float32", (2, 64): "float64",
             (4, 16): "bfloat16", (6, 8): "bool"}
_DL_CODES = {v: k for k, v in _DL_TYPES.items()}
_ITEMSIZE = {"bool": 1, "int8": 1, "uint8": 1, "int16": 2, "uint16": 2, "float16": 2, "bfloat16": 2, "int32": 4,
             "uint32": 4, "float32": 4, "int64": 8, "uint64": 8, "float64": 8}


class _DLDevice(ctypes.Structure):
    _fields_ = [("device_type", ctypes.c_int32), ("device_id", ctypes.c_int32)]


class _DLDataType(ctypes.Structure):
    _fields_ = [("code", ctypes.c_uint8), ("bits", ctypes.c_uint8), ("lanes", ctypes.c_uint16)]


class _DLTensor(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("device", _DLDevice), ("ndim", ctypes.c_int32), ("dtype", _DLDataType),
                ("shape", ctypes.POINTER(ctypes.c_int64)), ("strides", ctypes.POINTER(ctypes.c_int64)),
                ("byte_offset", ctypes.c_uint64)]


_DELETER = ctypes.CFUNCTYPE(None, ctypes.c_void_p)


class _DLManagedTensor(ctypes.Structure):
    _fields_ = [("dl_tensor", _DLTensor), ("manager_ctx", ctypes.c_void_p), ("deleter", _DELETER)]


def _pyapi(name: str, restype, *argtypes):
    return ctypes.PYFUNCTYPE(restype, *argtypes)((name, ctypes.pythonapi))


_capsule_get = _pyapi("PyCapsule_GetPointer", ctypes.c_void_p, ctypes.py_object, ctypes.c_char_p)
_capsule_rename = _pyapi("PyCapsule_SetName", ctypes.c_int, ctypes.py_object, ctypes.c_char_p)
_capsule_valid = _pyapi("PyCapsule_IsValid", ctypes.c_int, ctypes.py_object, ctypes.c_char_p)
# the destructor handles a capsule that is being deallocated by its raw address only
_capsule_valid_raw = _pyapi("PyCapsule_IsValid", ctypes.c_int, ctypes.c_void_p, ctypes.c_char_p)
_capsule_get_raw = _pyapi("PyCapsule_GetPointer", ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p)
_capsule_new = _pyapi("PyCapsule_New", ctypes.py_object, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p)
_NAME = b"dltensor"
_USED = b"used_dltensor"


def _release_managed(addr: int) -> None:
    m = _DLManagedTensor.from_address(addr)
    if m.deleter:
        m.deleter(addr)


@dataclass
class CudaInput:
    """A CUDA array read without PyTorch: the address of its first element, its device, element
    type, shape, strides in elements, the stream its producer orders it on (None: ready now), and
    what keeps it alive until release()."""

    ptr: int
    device: int
    dtype: str
    shape: tuple[int, ...]
    strides: tuple[int, ...]
    stream: int | None
    keep: Any = None
    managed: int | None = None

    def release(self) -> None:
        """Gives a consumed DLPack tensor back to its producer (its deleter)."""
        if self.managed:
            addr, self.managed = self.managed, None
            _release_managed(addr)
        self.keep = None


def intake(x: Any) -> CudaInput:
    """x (a CUDA array that is not a torch tensor) through the CUDA array interface or DLPack."""
    cai = getattr(x, "__cuda_array_interface__", None)
    if cai is not None:
        typestr = cai["typestr"]
        name = _TYPESTR.get(typestr[1:])
        if name is None or (typestr[0] == ">" and _ITEMSIZE[name] > 1):
            raise TypeError(f"eda: CUDA arrays of typestr {typestr!r} are not supported")
        shape = tuple(int(v) for v in cai["shape"])
        size = _ITEMSIZE[name]
        if cai.get("strides") is None:
            strides = c_strides(shape)
        else:
            bs = tuple(int(v) for v in cai["strides"])
            if any(v % size for v in bs):
                raise ValueError("eda: CUDA array strides must be multiples of the element size")
            strides = tuple(v // size for v in bs)
        ptr = int(cai["data"][0]) if cai.get("data") else 0
        s = cai.get("stream")  # version 3: the producer's stream (1: legacy default, 2: per-thread)
        if s is not None and int(s) == 0:
            raise ValueError("eda: __cuda_array_interface__ stream 0 is disallowed by the protocol")
        dev = _pointer_device(ptr) if ptr and math.prod(shape) else 0
        return CudaInput(ptr, dev, name, shape, strides, None if s is None else int(s), keep=x)
    if hasattr(x, "__dlpack__"):
        cap = x.__dlpack__()
        if not _capsule_valid(cap, _NAME):
            raise TypeError("eda: __dlpack__ did not return an unconsumed DLPack capsule")
        addr = _capsule_get(cap, _NAME)
        _capsule_rename(cap, _USED)
        t = _DLManagedTensor.from_address(addr).dl_tensor
        shape = tuple(int(t.shape[i]) for i in range(t.ndim))
        strides = c_strides(shape) if not t.strides else tuple(int(t.strides[i]) for i in range(t.ndim))
        cin = CudaInput(int(t.data or 0) + int(t.byte_offset), int(t.device.device_id),
                        _DL_TYPES.get((int(t.dtype.code), int(t.dtype.bits)), ""), shape, strides, None, keep=x,
                        managed=addr)
        if t.device.device_type not in (_KDL_CUDA, _KDL_CUDA_MANAGED) or t.dtype.lanes != 1 or not cin.dtype:
            cin.release()
            raise TypeError(f"eda: the DLPack tensor is not a CUDA array of supported scalars (device type "
                            f"{t.device.device_type}, dtype code {t.dtype.code}, bits {t.dtype.bits}, lanes "
                            f"{t.dtype.lanes})")
        return cin
    raise TypeError("eda: expected a CUDA array (DLPack or the CUDA array interface)")


def _pointer_device(ptr: int) -> int:
    from . import _native

    return _native.core().pointer_device(ptr)


# ---------------------------------------------------------------------------------------------
# results

class _Buffer:
    """One reference to an engine-allocated device buffer (eda_buffer)."""

    def __init__(self, device: int, nbytes: int) -> None:
        from . import _native

        self._core = _native.core()
        self.handle, self.ptr = self._core.buffer_alloc(device, nbytes)
        self.device = device
        self.nbytes = nbytes

    def __del__(self) -> None:
        h, self.handle = getattr(self, "handle", None), None
        if h:
            try:
                self._core.buffer_release(h)
            except Exception:
                pass


def _capsule_destructor(capsule_ptr: int) -> None:
    # an exported capsule that no consumer took (still named "dltensor"): its tensor is released
    if capsule_ptr and _capsule_valid_raw(capsule_ptr, _NAME):
        addr = _capsule_get_raw(capsule_ptr, _NAME)
        if addr:
            _release_managed(addr)


_DESTRUCTOR = ctypes.CFUNCTYPE(None, ctypes.c_void_p)(_capsule_destructor)


class DeviceArray:
    """A result on the GPU: shape, strides (bytes), dtype, device; readable without a copy through
    DLPack (``torch.from_dlpack``, ``cupy.from_dlpack``, ...) and the CUDA array interface;
    ``numpy.asarray`` copies it to the host."""

    def __init__(self, tensor: Any = None, *, buffer: _Buffer | None = None, offset: int = 0,
                 shape: tuple[int, ...] = (), strides: tuple[int, ...] = (), dtype: str = "float32") -> None:
        self._t = tensor
        self._buf = buffer
        if tensor is not None:
            self.shape = tuple(int(s) for s in tensor.shape)
            self.dtype = np.dtype(dtype_name(tensor))
            self.strides = tuple(int(s) * self.dtype.itemsize for s in tensor.stride())
            self.device = int(tensor.device.index or 0)
            self.ptr = int(tensor.data_ptr())
            self._offset = 0
        else:
            self.dtype = np.dtype(dtype)
            self.shape = tuple(int(s) for s in shape)
            self.strides = tuple(int(s) * self.dtype.itemsize for s in strides)
            self.device = buffer.device
            self._offset = int(offset)
            self.ptr = int(buffer.ptr) + self._offset * self.dtype.itemsize

    @classmethod
    def empty(cls, shape: tuple[int, ...], dtype: str, device: int) -> DeviceArray:
        """A C-contiguous array in an engine-allocated buffer."""
        nbytes = math.prod(shape) * np.dtype(dtype).itemsize
        return cls(buffer=_Buffer(device, nbytes), shape=shape, strides=c_strides(shape), dtype=dtype)

    def _elem_strides(self) -> tuple[int, ...]:
        return tuple(s // self.dtype.itemsize for s in self.strides)

    def reshape(self, shape: tuple[int, ...]) -> DeviceArray:
        """A C-contiguous array as another shape of the same size (a view)."""
        shape = tuple(int(v) for v in shape)
        if self._t is not None:
            return DeviceArray(self._t.reshape(shape))
        if self._elem_strides() != c_strides(self.shape) or math.prod(shape) != self.size:
            raise ValueError("eda: reshape of a non-contiguous DeviceArray")
        return DeviceArray(buffer=self._buf, offset=self._offset, shape=shape, strides=c_strides(shape),
                           dtype=self.dtype.name)

    def permute(self, perm: list[int]) -> DeviceArray:
        """The axes reordered (a view)."""
        if self._t is not None:
            return DeviceArray(self._t.permute(perm))
        es = self._elem_strides()
        return DeviceArray(buffer=self._buf, offset=self._offset, shape=tuple(self.shape[p] for p in perm),
                           strides=tuple(es[p] for p in perm), dtype=self.dtype.name)

    def narrow(self, start: int, length: int) -> DeviceArray:
        """Elements [start, start + length) of a 1-D array (a view)."""
        if self._t is not None:
            return DeviceArray(self._t[start:start + length])
        return DeviceArray(buffer=self._buf, offset=self._offset + start * self._elem_strides()[0], shape=(length,),
                           strides=self._elem_strides(), dtype=self.dtype.name)

    def __getitem__(self, index: int) -> DeviceArray:
        """Element `index` along the first axis (a view)."""
        if self._t is not None:
            return DeviceArray(self._t[index])
        i = int(index)
        n = self.shape[0]
        if not -n <= i < n:
            raise IndexError(f"eda: index {index} out of range for axis 0 of size {n}")
        es = self._elem_strides()
        return DeviceArray(buffer=self._buf, offset=self._offset + (i % n) * es[0], shape=self.shape[1:],
                           strides=es[1:], dtype=self.dtype.name)

    @property
    def ndim(self) -> int:
        return len(self.shape)

    @property
    def size(self) -> int:
        return math.prod(self.shape)

    @property
    def nbytes(self) -> int:
        return self.size * self.dtype.itemsize

    @property
    def __cuda_array_interface__(self) -> dict[str, Any]:
        if self._t is not None:
            return self._t.__cuda_array_interface__
        contiguous = self._elem_strides() == c_strides(self.shape)
        # the data is complete when the call that made it returned: no stream to order on
        return {"shape": self.shape, "typestr": self.dtype.str, "data": (self.ptr, False), "version": 3,
                "strides": None if contiguous else self.strides, "stream": None}

    def __dlpack_device__(self) -> tuple[int, int]:
        return (_KDL_CUDA, self.device)

    def __dlpack__(self, *args: Any, **kwargs: Any) -> Any:
        if self._t is not None:
            return self._t.__dlpack__(*args, **kwargs)
        code, bits = _DL_CODES[self.dtype.name]
        addr = self._buf._core.buffer_dlpack(self._buf.handle, self._offset * self.dtype.itemsize, code, bits,
                                             self.shape, self._elem_strides())
        return _capsule_new(addr, _NAME, ctypes.cast(_DESTRUCTOR, ctypes.c_void_p))

    def __array__(self, dtype: Any = None, copy: Any = None) -> np.ndarray:
        if self._t is not None:
            out = self._t.detach().cpu().numpy()
        elif self.size == 0:
            out = np.zeros(self.shape, self.dtype)
        else:
            es = self._elem_strides()
            lo = sum(min(0, (n - 1) * s) for n, s in zip(self.shape, es))
            hi = sum(max(0, (n - 1) * s) for n, s in zip(self.shape, es))
            span = np.empty(hi - lo + 1, self.dtype)
            self._buf._core.copy_to_host(span.ctypes.data, self.ptr + lo * self.dtype.itemsize, span.nbytes,
                                         self.device)
            out = np.lib.stride_tricks.as_strided(span[-lo:], self.shape, self.strides).copy()
        return out if dtype is None else out.astype(dtype)

    def torch(self):
        """The result as a torch tensor (no copy)."""
        if self._t is not None:
            return self._t
        return _torch().from_dlpack(self)

    def __repr__(self) -> str:
        return f"DeviceArray(shape={self.shape}, dtype={self.dtype}, device={self.device})"
