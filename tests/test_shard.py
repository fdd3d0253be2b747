# SPDX-License-Identifier: Apache-2.0
"""Element sharding across ranks (the multi-GPU path): two gloo ranks on the CPU each decompose
their shard of a batch (the oracle stands in for the GPU engine) and gather the rows; the result
equals the single-process decomposition of the whole batch bit for bit, since elements are
independent."""

from __future__ import annotations

import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def test_shard_bounds_cover_the_batch():
    from eda._shard import shard_bounds

    for batch in (0, 1, 5, 64, 67):
        for world in (1, 2, 3, 8):
            spans = [shard_bounds(batch, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == batch
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1


def _batch() -> np.ndarray:
    rng = np.random.default_rng(5)
    t = np.arange(300)
    x = np.stack([np.sin(2 * np.pi * t / p) + 0.3 * rng.standard_normal(300) for p in (7, 13, 29, 41, 61)])
    x[3, 17] = np.nan  # a failed element (check_finite) on one rank
    return x.astype(np.float32)


def _worker(rank: int, world: int, port: int, out: dict) -> None:
    sys.path.insert(0, str(ROOT / "eda-cuda_b200"))
    sys.path.insert(0, str(ROOT / "oracle"))
    import torch.distributed as dist

    import oracle
    from eda._shard import decompose_sharded

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        y, info = decompose_sharded(_batch(), decompose=lambda xs, **kw: oracle.decompose(xs))
        out[rank] = (y, {k: v for k, v in info.items()})
    finally:
        dist.destroy_process_group()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_gather_the_single_process_result():
    import oracle

    ctx = mp.get_context("spawn")
    with ctx.Manager() as manager:
        out = manager.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs)
        res = dict(out)
    want_rows, want_info = oracle.decompose(_batch())
    for rank in (0, 1):
        y, info = res[rank]
        assert y.shape == want_rows.shape
        assert np.array_equal(y, want_rows, equal_nan=True)
        for k in ("n_imfs", "error", "windows", "sifts", "spacing", "energy"):
            assert np.array_equal(info[k], want_info[k]), k
    assert want_info["error"][3] == 1


def test_mode_bound_matches_the_oracle():
    import oracle
    from eda._shard import mode_bound

    for n in (2, 3, 4, 9, 100, 512, 2048, 8192, 65536):
        assert mode_bound(n) + 2 == oracle.rows_cap((n,))


def test_ragged_assignment_balances_the_work():
    from eda._shard import mode_bound, ragged_assignment

    rng = np.random.default_rng(3)
    shapes = [(int(np.exp(rng.uniform(np.log(256), np.log(65536)))),) for _ in range(300)]
    for world in (1, 2, 3, 8):
        owner = ragged_assignment(shapes, world)
        load = [0] * world
        for s, r in zip(shapes, owner):
            load[r] += s[0] * mode_bound(s[0])
        heaviest = max(s[0] * mode_bound(s[0]) for s in shapes)
        assert max(load) - min(load) <= heaviest  # the longest-processing-time bound


def _ragged_fields() -> list[np.ndarray]:
    rng = np.random.default_rng(9)
    out = []
    for n in (300, 1200, 77, 640, 2000, 150):
        t = np.arange(n)
        out.append((np.sin(2 * np.pi * t / 11) + 0.5 * np.sin(2 * np.pi * t / 57) + 0.1 * rng.standard_normal(n))
                   .astype(np.float32))
    return out


def _oracle_ragged(fields, **kw):
    import oracle

    rows, infos = [], []
    for x in fields:
        r, info = oracle.decompose(x[None])
        rows.append(r[0])
        infos.append({k: v[0] for k, v in info.items()})
    return rows, infos


def _ragged_worker(rank: int, world: int, port: int, out: dict) -> None:
    sys.path.insert(0, str(ROOT / "eda-cuda_b200"))
    sys.path.insert(0, str(ROOT / "oracle"))
    import torch.distributed as dist

    from eda._shard import decompose_ragged_sharded

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out[rank] = decompose_ragged_sharded(_ragged_fields(), decompose=_oracle_ragged)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_share_a_ragged_batch():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as manager:
        out = manager.dict()
        port = _free_port()
        procs = [ctx.Process(target=_ragged_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs)
        res = dict(out)
    want_rows, want_infos = _oracle_ragged(_ragged_fields())
    for rank in (0, 1):
        rows, infos = res[rank]
        for got, want in zip(rows, want_rows):
            assert np.array_equal(got, want, equal_nan=True)
        for got, want in zip(infos, want_infos):
            for k in ("n_imfs", "error", "windows", "sifts"):
                assert np.array_equal(np.asarray(got[k]), np.asarray(want[k])), k
