# SPDX-License-Identifier: Apache-2.0
"""The exceptions of eda (importable without the compiled engine): the same classes, attributes and
pickling as the reference's src/eda/_errors.py."""

from __future__ import annotations

from typing import Any


class CudaError(RuntimeError):
    """A CUDA call or kernel launch failed inside eda, or no usable GPU was found. ``code`` is the
    numeric ``cudaError_t`` and ``name`` its symbolic name, None when unknown."""

    def __init__(self, message: str, code: int | None = None, name: str | None = None) -> None:
        super().__init__(message)
        self.code = code
        self.name = name or None

    def __reduce__(self) -> tuple[type, tuple[str, int | None, str | None]]:
        return (type(self), (str(self), self.code, self.name))


class DecompositionError(ValueError):
    """Elements of an ``eda.decompose`` call with ``errors="raise"`` failed: ``indices`` holds their
    flat batch indices, ``codes`` their error codes and ``info`` the call's information."""

    def __init__(self, message: str, indices: Any = (), codes: Any = (), info: Any = None) -> None:
        super().__init__(message)
        self.indices = indices
        self.codes = codes
        self.info = info

    def __reduce__(self) -> tuple[type, tuple[str, Any, Any, Any]]:
        return (type(self), (str(self), self.indices, self.codes, self.info))
