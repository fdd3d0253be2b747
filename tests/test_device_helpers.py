# SPDX-License-Identifier: Apache-2.0
"""The host-side rules of the device layer (no GPU): strides of C-contiguous arrays, the contiguity
test that decides between reading a CUDA array in place and gathering it, and the stream handle of
a call."""

from __future__ import annotations

import eda._api as api
from eda import _device


class _Stream:
    def __init__(self, **kw):
        self.__dict__.update(kw)


def test_c_strides():
    assert _device.c_strides((4, 5, 6)) == (30, 6, 1)
    assert _device.c_strides((7,)) == (1,)
    assert _device.c_strides((0, 3)) == (3, 1)


def test_contiguity_ignores_unit_axes():
    assert api._c_contiguous((4, 5), (5, 1))
    assert api._c_contiguous((4, 1, 5), (5, 99, 1))
    assert not api._c_contiguous((4, 5), (1, 4))
    assert not api._c_contiguous((4, 5), (10, 2))


def test_stream_handles():
    assert api._stream_handle(None, None) == 0
    assert api._stream_handle(None, 7) == 7
    assert api._stream_handle(12, 7) == 12
    assert api._stream_handle(_Stream(cuda_stream=33), None) == 33
    assert api._stream_handle(_Stream(ptr=44), None) == 44


def test_a_torch_free_object_is_a_cuda_array():
    class Cai:
        __cuda_array_interface__ = {"shape": (2,), "typestr": "<f4", "data": (0, False), "version": 3}

    assert _device.is_cuda_array(Cai())
    assert not _device.is_torch(Cai())
