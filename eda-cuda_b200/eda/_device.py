# SPDX-License-Identifier: Apache-2.0
"""CUDA arrays in and out. A CUDA array (a torch tensor, or anything with DLPack or the CUDA array
interface) is taken through PyTorch; the result of CUDA input is a ``DeviceArray`` that exports
DLPack and the CUDA array interface, as the reference's result type (src/eda/_device.py:228-334 of
eda-cuda)."""

from __future__ import annotations

import math
from typing import Any

import numpy as np

#: The dtype names a CUDA array may have (cast to the compute dtype on the GPU).
SUPPORTED_DTYPES = frozenset(("bool", "int8", "int16", "int32", "int64", "uint8", "uint16", "uint32", "uint64",
                              "float16", "bfloat16", "float32", "float64"))


def _torch():
    import torch

    return torch


def is_cuda_array(x: Any) -> bool:
    """Whether x is a CUDA array (device input)."""
    if type(x).__module__.startswith("torch") and hasattr(x, "is_cuda"):
        return bool(x.is_cuda)
    if hasattr(x, "__dlpack_device__"):
        try:
            dev_type, _ = x.__dlpack_device__()
            return int(dev_type) in (2, 13)  # kDLCUDA, kDLCUDAManaged
        except Exception:
            return False
    return hasattr(x, "__cuda_array_interface__")


def as_tensor(x: Any):
    """The CUDA array x as a torch tensor (no copy)."""
    torch = _torch()
    if isinstance(x, torch.Tensor):
        return x
    if hasattr(x, "__dlpack__"):
        return torch.from_dlpack(x)
    return torch.as_tensor(x, device="cuda")


def dtype_name(t: Any) -> str:
    return str(t.dtype).removeprefix("torch.")


class DeviceArray:
    """A result on the GPU: shape, strides (bytes), dtype, device; readable without a copy through
    DLPack (``torch.from_dlpack``) and the CUDA array interface; ``numpy.asarray`` copies it to the
    host."""

    def __init__(self, tensor: Any) -> None:
        self._t = tensor
        self.shape = tuple(int(s) for s in tensor.shape)
        self.dtype = np.dtype(dtype_name(tensor))
        self.strides = tuple(int(s) * self.dtype.itemsize for s in tensor.stride())
        self.device = int(tensor.device.index or 0)
        self.ptr = int(tensor.data_ptr())

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
        return self._t.__cuda_array_interface__

    def __dlpack_device__(self) -> tuple[int, int]:
        return (2, self.device)

    def __dlpack__(self, *args: Any, **kwargs: Any) -> Any:
        return self._t.__dlpack__(*args, **kwargs)

    def __array__(self, *args: Any, **kwargs: Any) -> np.ndarray:
        return np.asarray(self._t.detach().cpu().numpy(), *args, **kwargs)

    def torch(self):
        """The result as a torch tensor (no copy)."""
        return self._t

    def __repr__(self) -> str:
        return f"DeviceArray(shape={self.shape}, dtype={self.dtype}, device={self.device})"
