# SPDX-License-Identifier: Apache-2.0
"""Ragged batches (eda.decompose_ragged / eda_decompose_ragged): fields of different shapes in one
call. Every field's rows and information must equal, bit for bit, what eda.decompose gives for it
alone (the reference's way to run a ragged workload: one call per shape), whatever the grouping,
the order of the fields and the number of concurrent workers."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    if not t.cuda.is_available():
        pytest.skip("no CUDA device")
    return t


def signal(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    t = np.arange(n, dtype=np.float64)
    f0 = rng.uniform(0.002, 0.01)
    return (np.cos(2 * np.pi * (f0 * t + 0.5 * (0.2 - f0) / n * t * t)) + 0.8 * np.cos(rng.uniform(0.05, 0.3) * t)
            + rng.uniform(-1e-3, 1e-3) * t + 0.01 * rng.standard_normal(n))


def image(h: int, w: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w].astype(np.float64)
    cy, cx = rng.uniform(0, h), rng.uniform(0, w)
    return (np.cos(2 * np.pi * np.hypot(y - cy, x - cx) / 6) + 1.5 * np.cos(2 * np.pi * x / 24)
            + 3 * np.exp(-((y - h / 2) ** 2 + (x - w / 3) ** 2) / (2 * (h / 4) ** 2)) + 0.02 * rng.standard_normal((h, w)))


def alone(eda, x: np.ndarray):
    rows, info = eda.decompose(x[None], axes=tuple(range(1, x.ndim + 1)), return_info=True, errors="status")
    k = int(info.n_imfs[0]) if int(info.error[0]) == 0 else 0
    return rows[0, : (k + 1 if int(info.error[0]) == 0 else 1)], info, k


def same(a: np.ndarray, b: np.ndarray) -> bool:
    u = np.uint32 if a.dtype == np.float32 else np.uint64
    return a.shape == b.shape and np.array_equal(np.ascontiguousarray(a).view(u), np.ascontiguousarray(b).view(u))


def check_against_alone(eda, xs, rows, infos):
    assert len(rows) == len(xs) == len(infos)
    for i, x in enumerate(xs):
        want, winfo, k = alone(eda, x)
        assert same(np.asarray(rows[i]), np.asarray(want)), i
        assert int(infos[i].n_imfs) == int(winfo.n_imfs[0]) and int(infos[i].error) == int(winfo.error[0])
        np.testing.assert_array_equal(infos[i].windows, winfo.windows[0, :k])
        np.testing.assert_array_equal(infos[i].sifts, winfo.sifts[0, :k])
        np.testing.assert_array_equal(infos[i].spacing, winfo.spacing[0, :k])
        np.testing.assert_array_equal(infos[i].energy, winfo.energy[0, :k])


def test_ragged_1d_equals_one_call_per_field(torch):
    import eda

    lengths = [300, 2048, 511, 1024, 300, 777, 4096, 1024, 2, 300, 6000, 513]
    xs = [signal(n, 7 + i).astype(np.float32) for i, n in enumerate(lengths)]
    rows, infos = eda.decompose_ragged(xs, return_info=True)
    check_against_alone(eda, xs, rows, infos)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_ragged_2d_equals_one_call_per_field(torch, dtype):
    import eda

    shapes = [(40, 56), (64, 64), (40, 56), (33, 90), (64, 64), (96, 128), (40, 56)]
    xs = [image(h, w, 3 + i).astype(dtype) for i, (h, w) in enumerate(shapes)]
    rows, infos = eda.decompose_ragged(xs, return_info=True)
    check_against_alone(eda, xs, rows, infos)


def test_ragged_results_do_not_depend_on_the_workers(torch):
    import eda

    lengths = [700, 900, 700, 1500, 900, 64, 3000]
    xs = [signal(n, 100 + i) for i, n in enumerate(lengths)]
    one = eda.decompose_ragged(xs, workers=1)
    many = eda.decompose_ragged(xs, workers=8)
    for a, b in zip(one, many):
        assert same(a, b)


def test_ragged_device_input(torch):
    import eda

    lengths = [500, 1200, 500, 2500]
    xs = [signal(n, 40 + i).astype(np.float32) for i, n in enumerate(lengths)]
    xd = [torch.from_numpy(x).cuda() for x in xs]
    rows = eda.decompose_ragged(xd)
    host = eda.decompose_ragged(xs)
    for r, h in zip(rows, host):
        assert same(r.cpu().numpy() if hasattr(r, "cpu") else np.asarray(r), h)


def test_ragged_failed_field(torch):
    import eda

    xs = [signal(400, 1), signal(500, 2), signal(400, 3)]
    xs[1][17] = np.nan
    with pytest.raises(eda.DecompositionError) as e:
        eda.decompose_ragged(xs)
    assert list(e.value.indices) == [1]
    rows, infos = eda.decompose_ragged(xs, errors="status", return_info=True)
    assert rows[1].shape == (1, 500) and np.isnan(rows[1]).all() and int(infos[1].error) == 1
    check_against_alone(eda, [xs[0], xs[2]], [rows[0], rows[2]], [infos[0], infos[2]])


def test_ragged_rejects_a_field_beyond_the_axis_limit(torch):
    import eda

    with pytest.raises(ValueError, match="exceeds the limit"):
        eda.decompose_ragged([signal(300, 1).astype(np.float32), signal(65537, 2).astype(np.float32)])
    with pytest.raises(ValueError, match="exceeds the limit"):
        eda.decompose_ragged([np.zeros((8193, 4), np.float32), np.zeros((6, 4), np.float32)])


def test_fresh_workspaces_are_zeroed_on_the_workers_streams(torch):
    """Each ragged call starts new worker threads, which lease workspaces (allocated and zeroed when
    the pool has none idle; released here first). With the caller on a non-blocking stream and the
    legacy default stream kept busy by other work, a zeroing queued on the legacy stream would land
    in the middle of the workers' kernels (which run on their own non-blocking streams) and corrupt
    their inputs; zeroed on the workers' own streams, every field must still equal its one-field
    call."""
    import eda

    xs = [signal(400, 11), signal(400, 13), signal(520, 12), signal(520, 14)]
    wants = [alone(eda, x) for x in xs]
    xd = [torch.from_numpy(x).cuda() for x in xs]  # device fields: the workers follow the caller's stream
    side = torch.cuda.Stream()
    a = torch.randn(8192, 8192, device="cuda")
    for _ in range(3):
        torch.cuda.synchronize()
        assert eda._native.core()._lib.eda_release_workspace() == 0  # fresh workspaces for the workers
        busy = a
        for _ in range(24):  # tens of milliseconds of work on the legacy default stream
            busy = busy @ a
        with torch.cuda.stream(side):
            rows, infos = eda.decompose_ragged(xd, workers=2, return_info=True, errors="status")
            side.synchronize()
        for i, (want, winfo, k) in enumerate(wants):
            assert same(np.asarray(rows[i]), np.asarray(want)), i
            assert int(infos[i].n_imfs) == int(winfo.n_imfs[0])
    torch.cuda.synchronize()


@pytest.fixture
def exact_lengths():
    """Runs a test body with 1-D signals grouped by exact length, restoring length classes after."""
    import eda

    eda.set_length_classes(False)
    try:
        yield
    finally:
        eda.set_length_classes(True)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_length_classes_equal_exact_length_groups(torch, dtype):
    """Signals of one length class run as one batch of uneven lengths (every kernel reading each
    signal's own length); grouped by exact length every signal runs alone. Both must agree bit for
    bit, and with one call per signal."""
    import eda

    assert eda.length_classes()
    lengths = [2, 3, 31, 32, 33, 63, 64, 65, 100, 127, 250, 256, 300, 511, 640, 1000, 1023]
    xs = [signal(n, 500 + i).astype(dtype) for i, n in enumerate(lengths)]
    rows_c, infos_c = eda.decompose_ragged(xs, return_info=True)
    eda.set_length_classes(False)
    try:
        rows_e, infos_e = eda.decompose_ragged(xs, return_info=True)
    finally:
        eda.set_length_classes(True)
    for i in range(len(xs)):
        assert same(np.asarray(rows_c[i]), np.asarray(rows_e[i])), lengths[i]
        assert int(infos_c[i].n_imfs) == int(infos_e[i].n_imfs)
        np.testing.assert_array_equal(infos_c[i].windows, infos_e[i].windows)
        np.testing.assert_array_equal(infos_c[i].energy, infos_e[i].energy)
    check_against_alone(eda, xs[::4], rows_c[::4], infos_c[::4])


def test_length_class_across_the_staged_capacity(torch):
    """A class whose longest signal folds its lines in global memory (beyond the shared-memory
    capacity of a staged cube pass) runs every signal of the class that way, signals that alone
    would be staged included: the canonical folds make both give the same bits."""
    import eda

    lengths = [16400, 20000, 16384, 18000, 30000]
    xs = [signal(n, 900 + i).astype(np.float32) for i, n in enumerate(lengths)]
    rows, infos = eda.decompose_ragged(xs, return_info=True)
    check_against_alone(eda, xs, rows, infos)


def test_length_class_of_the_longest_signals(torch):
    """The class [32768, 65536]: global-memory folds, the global-memory extrema pass (lines beyond
    the staged extrema capacity) and column tiles in the components."""
    import eda

    lengths = [65536, 40000, 52000, 33000]
    xs = [signal(n, 1300 + i).astype(np.float32) for i, n in enumerate(lengths)]
    rows, infos = eda.decompose_ragged(xs, return_info=True, workers=2)
    check_against_alone(eda, xs, rows, infos)


def test_length_class_device_input_and_failed_signal(torch):
    import eda

    lengths = [600, 900, 1000, 513, 700]
    xs = [signal(n, 70 + i).astype(np.float32) for i, n in enumerate(lengths)]
    xs[2][400] = np.inf
    xd = [torch.from_numpy(x).cuda() for x in xs]
    rows, infos = eda.decompose_ragged(xd, return_info=True, errors="status")
    assert int(infos[2].error) == 1 and rows[2].shape == (1, 1000)
    host, hinfos = eda.decompose_ragged(xs, return_info=True, errors="status")
    for i in range(len(xs)):
        r = rows[i].cpu().numpy() if hasattr(rows[i], "cpu") else np.asarray(rows[i])
        assert same(r, np.asarray(host[i])), i
    keep = [0, 1, 3, 4]
    check_against_alone(eda, [xs[i] for i in keep], [host[i] for i in keep], [hinfos[i] for i in keep])


def test_exact_length_groups_still_equal_one_call_per_field(torch, exact_lengths):
    import eda

    lengths = [300, 511, 300, 777, 513]
    xs = [signal(n, 31 + i).astype(np.float32) for i, n in enumerate(lengths)]
    rows, infos = eda.decompose_ragged(xs, return_info=True)
    check_against_alone(eda, xs, rows, infos)


def test_length_classes_in_cluster_selections(torch):
    """Classes of many signals (the exact selections run as thread-block clusters, one per
    signal, from several host threads at once) still equal one call per signal."""
    import eda

    rng = np.random.default_rng(77)
    lengths = [int(v) for v in rng.integers(256, 1024, size=96)]
    xs = [signal(n, 2000 + i).astype(np.float32) for i, n in enumerate(lengths)]
    rows, infos = eda.decompose_ragged(xs, return_info=True, workers=8)
    check_against_alone(eda, xs, rows, infos)
