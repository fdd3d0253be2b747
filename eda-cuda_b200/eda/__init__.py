# SPDX-License-Identifier: Apache-2.0
"""eda on B200: the sifting hot path of eda-cuda's empirical decomposition behind the same public
call, ``eda.decompose``, computed by this package's sm_100a engine (libeda_b200.so). Importing the
package needs neither a GPU nor the compiled engine; the engine loads on the first call that needs
it, and there is no CPU fallback."""

from __future__ import annotations

import operator

import numpy as np
from typing import Any

from . import _native
from ._api import DecompositionInfo, Monogenic, Orientation, decompose, decompose_ragged, monogenic
from ._device import DeviceArray
from ._errors import CudaError, DecompositionError

__version__ = "0.1.0"

__all__ = [
    "CudaError",
    "DecompositionError",
    "DecompositionInfo",
    "DeviceArray",
    "Monogenic",
    "Orientation",
    "__version__",
    "build_info",
    "decompose",
    "decompose_ragged",
    "device_count",
    "device_info",
    "autotune",
    "load_tuning",
    "monogenic",
    "length_classes",
    "set_length_classes",
    "set_transform_precision",
    "transform_precision",
]

#: The products of the float32 orientation transforms (2-D / 3-D): split products on the tensor
#: cores ("tf32x3", the default; "bf16x3") or the plain float32 product ("fp32").
TRANSFORM_PRECISIONS = ("tf32x3", "bf16x3", "fp32")


def set_transform_precision(name: str) -> None:
    """Selects the product of the float32 orientation transforms for the whole process: "tf32x3"
    (3xTF32 split products on the tensor cores, the default), "bf16x3" (BF16x3 split products on
    the tensor cores) or "fp32" (the plain float32 product). Float64 input always uses float64. This
    engine's extension: the reference computes the transforms with cuFFT in float32."""
    if name not in TRANSFORM_PRECISIONS:
        raise ValueError(f"eda: transform precision must be one of {TRANSFORM_PRECISIONS}, got {name!r}")
    _native.core().set_transform_precision(TRANSFORM_PRECISIONS.index(name))


def transform_precision() -> str:
    """The current product of the float32 orientation transforms (see set_transform_precision)."""
    return TRANSFORM_PRECISIONS[_native.core().transform_precision()]


def set_length_classes(on: bool) -> None:
    """How decompose_ragged groups 1-D signals, for the whole process: True (the default) decomposes
    the signals whose lengths share a class [2^k, 2^(k+1)) together as one batch of uneven lengths,
    False groups them by exact length. Results are the same either way (every signal's rows and
    information are those of a call on that signal alone). This engine's extension: the reference
    takes one shape per call."""
    _native.core().set_length_classes(bool(on))


def length_classes() -> bool:
    """Whether decompose_ragged groups 1-D signals by length class (see set_length_classes)."""
    return _native.core().length_classes()


def build_info() -> dict[str, Any]:
    """How the engine was built (CUDA toolkit, runtime and driver, architectures); works without a GPU."""
    return _native.core().build_info()


def device_count() -> int:
    """The number of visible CUDA devices; 0 without a driver or device."""
    return _native.core().device_count()


def device_info(device: int = 0) -> dict[str, Any]:
    """Properties of a visible CUDA device; ValueError for a device that is not visible."""
    if isinstance(device, bool):
        raise TypeError("eda: device must be an integer, not bool")
    try:
        number = operator.index(device)
    except TypeError:
        raise TypeError(f"eda: device must be an integer, got {type(device).__name__}") from None
    if not -(2**31) <= number < 2**31:
        raise ValueError(f"eda: CUDA device {number} is not visible")
    return _native.core().device_info(number)



def autotune(shape: Any, batch: int = 1, dtype: Any = "float32", cache: str | None = None) -> dict[str, Any]:
    """Times the launch shapes of the cube passes for fields of ``shape`` (1 to 3 axes) in batches of
    ``batch`` on the current device and keeps the fastest for every later call with that geometry
    (the results do not change, only the speed); with ``cache``, all kept shapes are written to that
    file, which ``load_tuning`` (or the environment variable EDA_TUNING_CACHE) reads in a later
    process. Returns the chosen shape and the timings (microseconds, default and tuned). This
    engine's addition: the reference's launch shapes are fixed."""
    dims = tuple(operator.index(v) for v in (shape if isinstance(shape, (tuple, list)) else (shape,)))
    name = np.dtype(dtype).name if not isinstance(dtype, str) else dtype
    if name not in ("float32", "float64"):
        raise ValueError(f"eda: autotune dtype must be float32 or float64, got {dtype!r}")
    return _native.core().autotune(name, dims, operator.index(batch), cache)


def load_tuning(path: str) -> None:
    """Reads launch shapes saved by ``autotune(..., cache=path)``."""
    _native.core().tuning_load(path)