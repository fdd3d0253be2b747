# SPDX-License-Identifier: Apache-2.0
"""CUDA arrays that are not torch tensors through eda.decompose (the reference's device layer,
src/eda/_device.py:99-334 of eda-cuda): an object that offers only the CUDA array interface, and one
that offers only DLPack, are read without PyTorch; the results are engine-allocated DeviceArrays
that export DLPack and the CUDA array interface. Results are bit for bit those of the host call on
the same values (float32 / float64, C-contiguous, strided and cast input, return_orientation), and
the exported tensors outlive the DeviceArray they came from. The test allocates its inputs with
PyTorch only to have device memory; the objects handed to eda hide that."""

from __future__ import annotations

import gc

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


class CaiOnly:
    """A CUDA array seen only through __cuda_array_interface__ (version 3)."""

    def __init__(self, t, stream=None):
        self._t = t
        d = dict(t.__cuda_array_interface__)
        d["version"] = 3
        d["stream"] = stream
        self.__cuda_array_interface__ = d


class DlpackOnly:
    """A CUDA array seen only through DLPack."""

    def __init__(self, t):
        self._t = t

    def __dlpack__(self, *args, **kwargs):
        return self._t.__dlpack__(*args, **kwargs)

    def __dlpack_device__(self):
        return self._t.__dlpack_device__()


@pytest.fixture(scope="module")
def torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def signals(shape, dtype, seed=3):
    rng = np.random.default_rng(seed)
    t = np.arange(shape[-1])
    x = np.sin(2 * np.pi * t / 9) + 2 * np.sin(2 * np.pi * t / 71) + 0.05 * rng.standard_normal(shape)
    return x.astype(dtype)


def same(a, b) -> bool:
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and a.dtype == b.dtype and np.array_equal(a, b, equal_nan=True)


@pytest.mark.parametrize("wrap", [CaiOnly, DlpackOnly], ids=["cai", "dlpack"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_non_torch_input_matches_the_host_call(torch, wrap, dtype):
    import eda

    x = signals((3, 1500), dtype)
    want, want_info = eda.decompose(x, return_info=True)
    y, info = eda.decompose(wrap(torch.from_numpy(x).cuda()), return_info=True)
    assert isinstance(y, eda.DeviceArray) and y._t is None  # an engine buffer, not a torch tensor
    assert same(y, want)
    assert np.array_equal(info.windows, want_info.windows) and np.array_equal(info.n_imfs, want_info.n_imfs)
    back = torch.from_dlpack(y)
    assert same(back.cpu().numpy(), want)
    cai = y.__cuda_array_interface__
    assert cai["shape"] == want.shape and cai["data"][0] == back.data_ptr()


def test_strided_and_cast_input(torch):
    import eda

    base = signals((700, 4), np.float64)  # signals along axis 0, a transposed view, cast to float32
    t = torch.from_numpy(base).cuda()
    want = eda.decompose(base.astype(np.float32), axes=0)
    got = eda.decompose(CaiOnly(t), axes=0, dtype="float32")
    assert same(got, want)


def test_orientation_of_a_non_torch_image(torch):
    import eda

    rng = np.random.default_rng(5)
    yy, xx = np.mgrid[0:64, 0:80]
    img = (np.cos(2 * np.pi * (xx + 0.3 * yy) / 9) + 0.1 * rng.standard_normal((64, 80))).astype(np.float32)
    want_y, want_o = eda.decompose(img, return_orientation=True)
    got_y, got_o = eda.decompose(DlpackOnly(torch.from_numpy(img).cuda()), return_orientation=True)
    assert same(got_y, want_y)
    assert same(got_o.direction, want_o.direction) and same(got_o.coherence, want_o.coherence)


def test_exported_tensors_outlive_the_array(torch):
    import eda

    x = signals((2, 900), np.float32)
    y = eda.decompose(CaiOnly(torch.from_numpy(x).cuda(), stream=1))
    want = np.asarray(y)
    unused = y.__dlpack__()  # a capsule nobody consumes: released when it is collected
    del unused
    t = torch.from_dlpack(y)
    del y
    gc.collect()
    torch.cuda.synchronize()
    assert np.array_equal(t.cpu().numpy(), want)
