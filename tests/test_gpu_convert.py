# SPDX-License-Identifier: Apache-2.0
"""Device input in any element type and layout (eda_decompose_strided; the reference's strided
gather and cast, cpp/src/field/convert.cu:69-170, and its input tests, tests/python/test_input.py):
the engine reads a CUDA array where it lies and casts each chunk in a kernel. Every case must give
rows and information bit for bit equal to decomposing the same array after PyTorch's cast to the
compute dtype and a contiguous copy (both casts round to nearest even), for all 13 element types,
permuted, sliced, broadcast and transposed layouts, and negative strides through the C ABI."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

DTYPES = ["bool", "int8", "int16", "int32", "int64", "uint8", "uint16", "uint32", "uint64", "float16", "bfloat16",
          "float32", "float64"]


def field(shape, dtype: str, seed: int):
    """Structured values with noise, representable in the element type (a copy on the device)."""
    rng = np.random.default_rng(seed)
    grids = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in shape[-2:]], indexing="ij")
    base = np.cos(2 * np.pi * grids[0] / 9.0) + np.sin(2 * np.pi * grids[-1] / 7.0)
    v = base + 0.3 * rng.standard_normal(shape)
    if dtype == "bool":
        a = v > 0.2
    elif dtype.startswith("int") or dtype.startswith("uint"):
        lo = 0 if dtype.startswith("uint") else -40
        a = np.clip(np.round(20 * v + (40 if lo == 0 else 0)), lo, 100).astype(np.int64)
        if dtype in ("int64", "uint64"):
            a = a * (1 << 40) + 12345  # beyond float32 and float64 precision: rounding matters
    else:
        a = v * 3.7
    t = torch.from_numpy(np.asarray(a)).cuda()
    return t.to(getattr(torch, dtype))


def assert_same(engine, got, want):
    y1, i1 = got
    y2, i2 = want
    a, b = np.asarray(y1), np.asarray(y2)
    assert a.dtype == b.dtype and a.shape == b.shape
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
    for name in ("n_imfs", "error", "windows", "sifts", "spacing", "energy"):
        assert np.array_equal(getattr(i1, name), getattr(i2, name)), name


@pytest.mark.parametrize("target", ["float32", "float64"])
@pytest.mark.parametrize("dtype", DTYPES)
def test_every_element_type_matches_the_cast_copy(engine, dtype, target):
    x = field((3, 40, 36), dtype, 7)
    got = engine.decompose(x, axes=(1, 2), dtype=target, errors="status", return_info=True)
    want = engine.decompose(x.to(getattr(torch, target)).contiguous(), axes=(1, 2), errors="status",
                            return_info=True)
    assert_same(engine, got, want)


@pytest.mark.parametrize("case", ["permuted", "sliced", "broadcast", "transposed", "1d-strided", "3d-middle"])
def test_layouts_match_the_contiguous_copy(engine, case):
    if case == "permuted":      # spatial axes first, batch last
        x = field((40, 36, 3), "float32", 1)
        axes = (0, 1)
    elif case == "sliced":      # every other row and column of a larger array
        x = field((3, 80, 72), "float32", 2)[:, ::2, 1::2]
        axes = (1, 2)
    elif case == "broadcast":   # one field repeated over a batch axis of stride 0
        x = field((1, 40, 36), "float64", 3).expand(4, 40, 36)
        axes = (1, 2)
    elif case == "transposed":  # the spatial axes in the other order
        x = field((2, 40, 36), "int16", 4)
        axes = (2, 1)
    elif case == "1d-strided":  # 1-D signals along the middle axis of a 3-D array
        x = field((3, 300, 2), "float16", 5)
        axes = (1,)
    else:                       # two batch axes around a 2-D field
        x = field((2, 24, 20, 3), "float32", 6)
        axes = (1, 2)
    got = engine.decompose(x, axes=axes, dtype="float32", errors="status", return_info=True)
    # the reference: the cast, permuted to (batch..., spatial in axes order), contiguous, read in place
    batch_axes = tuple(i for i in range(x.dim()) if i not in axes)
    nb = len(batch_axes)
    c = x.to(torch.float32).permute(list(batch_axes) + list(axes)).contiguous()
    want = engine.decompose(c, axes=tuple(range(nb, x.dim())), errors="status", return_info=True)
    # the result's public layout is the computed (batch..., P, spatial...) one permuted by the API's
    # restore rule: undo it
    from eda._api import _restore

    perm = _restore(x.dim(), batch_axes, axes)
    y_got = np.transpose(np.asarray(got[0]), np.argsort(perm))
    y_want = np.asarray(want[0])
    assert y_got.shape == y_want.shape
    assert np.array_equal(y_got.view(np.uint32), y_want.view(np.uint32))
    for name in ("n_imfs", "error", "windows", "sifts", "spacing", "energy"):
        assert np.array_equal(np.asarray(getattr(got[1], name)), np.asarray(getattr(want[1], name))), name


def test_negative_strides_through_the_c_abi(engine):
    """A field read backwards along both axes (a pointer at its last sample, negative strides) gives
    the rows of the flipped field."""
    from eda import _native

    x = field((2, 40, 36), "float32", 8).contiguous()
    core = _native.core()
    B, n0, n1 = x.shape
    item = x.element_size()
    last = x.data_ptr() + ((n0 - 1) * n1 + (n1 - 1)) * item
    layout = ("float32", (B,), (n0 * n1,), (-n1, -1))
    st = torch.cuda.current_stream()

    def alloc(P):
        out = torch.empty((B, P, n0, n1), dtype=torch.float32, device=x.device)
        return out, out.data_ptr()

    rows, info = core.decompose_device(last, x.device.index or 0, "float32", (B, n0, n1), -1, None, 3, True, 0,
                                       st.cuda_stream, alloc, None, layout)
    torch.cuda.synchronize()
    want = engine.decompose(torch.flip(x, dims=(1, 2)).contiguous(), axes=(1, 2), return_info=True)
    assert np.array_equal(rows.cpu().numpy().view(np.uint32), np.asarray(want[0]).view(np.uint32))
    assert np.array_equal(info["n_imfs"], np.asarray(want[1].n_imfs))


def test_argument_rules(engine):
    x = field((2, 16, 16), "int32", 9)
    with pytest.raises(TypeError):
        engine.decompose(x, axes=(1, 2))  # an integer array needs dtype=
    y = engine.decompose(x[:0], axes=(1, 2), dtype="float32")
    assert np.asarray(y).shape[0] == 0
