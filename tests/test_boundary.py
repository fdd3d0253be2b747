# SPDX-License-Identifier: Apache-2.0
"""The C ABI boundary without a GPU: the engine library loads, exports every entry point that
include/eda_b200.h declares, and its host-side argument rules and error mapping work; the Python
surface mirrors the reference's argument rules (tests/python/test_api.py of eda-cuda)."""

from __future__ import annotations

import ctypes
import re

import numpy as np
import pytest

from conftest import ROOT


def declared() -> list[str]:
    names = []
    for header in sorted((ROOT / "include").glob("*.h")):
        names += re.findall(r"EDA_API\s+[\w\s\*]+?\b(eda_\w+)\s*\(", header.read_text())
    return names


def test_the_library_exports_every_declared_entry_point():
    import eda
    from eda import _native

    lib = ctypes.CDLL(str(_native.LIB))
    names = declared()
    assert len(names) >= 10
    for name in names:
        assert hasattr(lib, name), name


def test_build_info_works_without_a_gpu():
    import eda

    info = eda.build_info()
    assert info["cuda_architectures"] == "100a" and info["sass"] == ["sm_100a"]


def test_device_count_is_an_integer():
    import eda

    assert isinstance(eda.device_count(), int)


@pytest.mark.parametrize("kwargs,exc", [
    ({"max_imf": True}, TypeError),
    ({"max_imf": 1.5}, TypeError),
    ({"sifts": 0}, ValueError),
    ({"sifts": True}, TypeError),
    ({"tie_tolerance": -1.0}, ValueError),
    ({"tie_tolerance": float("nan")}, ValueError),
    ({"tie_tolerance": "x"}, TypeError),
    ({"check_finite": 1}, TypeError),
    ({"errors": "ignore"}, ValueError),
    ({"return_info": None}, TypeError),
    ({"axes": (0, 0)}, ValueError),
    ({"axes": 3}, np.exceptions.AxisError),
    ({"dtype": "int32"}, TypeError),
])
def test_argument_rules(kwargs, exc):
    import eda

    with pytest.raises(exc):
        eda.decompose(np.zeros((4, 5), np.float32), **kwargs)


def test_integer_input_needs_a_dtype():
    import eda

    with pytest.raises(TypeError, match="float32 or float64"):
        eda.decompose(np.zeros(16, np.int32))


def test_orientation_needs_two_axes():
    import eda

    with pytest.raises(ValueError, match="2 or 3 spatial axes"):
        eda.decompose(np.zeros(16, np.float32), return_orientation=True)


def test_axis_rules_of_the_native_layer():
    from eda import _native

    core = _native.Core(_native.LIB)
    with pytest.raises(ValueError, match="at least 2 samples"):
        core.decompose_host(np.zeros((1, 1), np.float32), -1, None, 3, True, False, 0)
    with pytest.raises(ValueError, match="extent >= 2"):
        core.decompose_host(np.zeros((1, 5, 1), np.float32), -1, None, 3, True, False, 0)


def test_empty_batch_computes_nothing():
    import eda

    y, info = eda.decompose(np.zeros((0, 8), np.float32), axes=1, return_info=True)
    assert y.shape == (0, 1, 8) and info.windows.shape == (0, 0)


@pytest.mark.parametrize("xs,exc", [
    (np.zeros(10), TypeError),
    ([np.zeros(10), np.zeros((4, 4))], ValueError),
    ([np.zeros(10, np.float32), np.zeros(12, np.float64)], TypeError),
    ([np.zeros(10, np.int32)], TypeError),
    ([np.zeros((2, 2, 2, 2))], ValueError),
])
def test_ragged_argument_rules(xs, exc):
    import eda

    with pytest.raises(exc):
        eda.decompose_ragged(xs)


def test_ragged_empty_batch():
    import eda

    assert eda.decompose_ragged([]) == []
    assert eda.decompose_ragged([], return_info=True) == ([], [])


@pytest.mark.parametrize("case,message", [
    ("type", "unknown source element type"),
    ("axes", "at most 64 batch axes"),
    ("dim", "D must be 1, 2 or 3"),
    ("null", "null"),
    ("extent", "batch extent is negative"),
])
def test_strided_argument_rules(case, message):
    """eda_decompose_strided rejects a bad layout before it touches the device."""
    from eda import _native

    core = _native.core()
    lib = core._lib
    shape = (ctypes.c_int64 * 1)(-1 if case == "extent" else 2)
    bstride = (ctypes.c_int64 * 1)(64)
    stride = (ctypes.c_int64 * 3)(8, 1, 0)
    src = _native._Source(13 if case == "type" else 11, 65 if case == "axes" else 1, shape, bstride, stride)
    n = (ctypes.c_int64 * 3)(8, 8, 1)
    p = _native._Params(-1, -1.0, 3, 1, 0, 0)
    run = ctypes.c_void_p()
    src_arg = None if case == "null" else ctypes.byref(src)
    st = lib.eda_decompose_strided(ctypes.c_void_p(1), src_arg, 0, 4 if case == "dim" else 2, n, ctypes.byref(p),
                                   None, ctypes.byref(run))
    assert st == 1  # EDA_INVALID_ARGUMENT
    buf = ctypes.create_string_buffer(512)
    lib.eda_last_error(buf, 512)
    assert message in buf.value.decode()


def test_length_classes_setting_round_trips():
    """How ragged 1-D batches group their signals is a process-wide host setting (no GPU needed)."""
    import eda

    assert eda.length_classes() is True  # the default
    try:
        eda.set_length_classes(False)
        assert eda.length_classes() is False
    finally:
        eda.set_length_classes(True)
    assert eda.length_classes() is True


def test_ragged_collect_all_rejects_a_null_run():
    from eda import _native

    lib = _native.core()._lib
    st = lib.eda_ragged_collect_all(None, None, 0, None, None)
    assert st != 0
