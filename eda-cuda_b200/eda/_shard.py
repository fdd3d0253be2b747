# SPDX-License-Identifier: Apache-2.0
"""Element sharding across processes (one per GPU). Every element of a batch is decomposed on its
own, bit for bit independent of the others, so a batch splits into contiguous shards with no
exchange during the decomposition; the rows are gathered afterwards only when the caller asks
(an all-gather of the padded rows and the information arrays over torch.distributed: NCCL between
GPUs, gloo on the CPU in the tests)."""

from __future__ import annotations

from typing import Any, Callable

import numpy as np


def shard_bounds(batch: int, world: int, rank: int) -> tuple[int, int]:
    """The contiguous shard [lo, hi) of `rank`: the first batch % world ranks hold one element more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("eda: rank out of range")
    base, extra = divmod(batch, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


_INFO = ("n_imfs", "error", "windows", "sifts", "spacing", "energy")


def decompose_sharded(x: np.ndarray, group: Any = None, gather: bool = True,
                      decompose: Callable[..., tuple[np.ndarray, dict]] | None = None,
                      **kwargs: Any) -> tuple[np.ndarray, dict]:
    """Decompose this rank's shard of the host batch x (B, *spatial) and, with gather, return the
    whole batch's rows (B, P, *spatial) and information on every rank (else the shard's). The
    compute call is `decompose(x_shard, **kwargs) -> (rows, info)` (default: the engine's
    ``eda._native.core().decompose_host`` arguments in keyword form)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    lo, hi = shard_bounds(x.shape[0], world, rank)
    if decompose is None:
        from . import _native

        def decompose(xs, **kw):
            return _native.core().decompose_host(np.ascontiguousarray(xs), kw.get("max_imf", -1), kw.get("tie_tolerance"),
                                                 kw.get("sifts", 3), kw.get("check_finite", True), False, 0)
    rows, info = decompose(np.ascontiguousarray(x[lo:hi]), **kwargs)
    if not gather or world == 1:
        return rows, info
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    # the common padded shapes: shard size, P and K
    dims = torch.tensor([hi - lo, rows.shape[1], info["windows"].shape[1]], dtype=torch.int64, device=dev)
    dist.all_reduce(dims, op=dist.ReduceOp.MAX, group=group)
    nmax, P, K = (int(v) for v in dims.tolist())
    spatial = x.shape[1:]

    def padded(a: np.ndarray, shape: tuple[int, ...]) -> torch.Tensor:
        out = np.zeros(shape, a.dtype)
        out[tuple(slice(0, s) for s in a.shape)] = a
        return torch.from_numpy(out).to(dev)

    def all_gather(t: torch.Tensor) -> list[torch.Tensor]:
        parts = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(parts, t, group=group)
        return parts

    row_parts = all_gather(padded(rows, (nmax, P) + spatial))
    info_parts = {k: all_gather(padded(np.asarray(info[k]), (nmax,) + ((K,) if np.asarray(info[k]).ndim == 2 else ())))
                  for k in _INFO}
    out_rows, out_info = [], {k: [] for k in _INFO}
    for r in range(world):
        a, b = shard_bounds(x.shape[0], world, r)
        out_rows.append(row_parts[r][: b - a].cpu().numpy())
        for k in _INFO:
            out_info[k].append(info_parts[k][r][: b - a].cpu().numpy())
    merged = {k: np.concatenate(v, axis=0) for k, v in out_info.items()}
    # rows beyond an element's residue are zero; failed elements' padded rows stay NaN
    y = np.concatenate(out_rows, axis=0)
    ok = merged["error"] == 0
    Pw = int(merged["n_imfs"][ok].max(initial=-1)) + 1 if ok.any() else 1
    y = y[:, : max(Pw, 1)]
    for i in np.flatnonzero(~ok):
        y[i] = np.nan
    Kw = int(merged["n_imfs"].max(initial=0))
    for k in ("windows", "sifts", "spacing", "energy"):
        merged[k] = merged[k][:, :Kw]
    return y, merged


def mode_bound(n_max: int) -> int:
    """The largest number of modes of a field whose longest axis has n_max samples (the window rule
    of cpp/src/method/driver.cpp:128-140: windows from 3, at least the previous + 2, at least twice
    the previous from the third mode on, while within n_max)."""
    w_prev, count = 1, 0
    k = 0
    while True:
        w = max(3, w_prev + 2)
        if k >= 2:
            w = max(w, 2 * (int(2.0 * w_prev) // 2) + 1)
        if w > n_max:
            return count
        count += 1
        w_prev = w
        k += 1


def ragged_assignment(shapes: list[tuple[int, ...]], world: int) -> list[int]:
    """The rank of every field of a ragged batch: the fields' costs (samples x mode bound, the
    sift's work) spread over the ranks by longest-processing-time first (each field, heaviest
    first, to the least loaded rank; ties to the lowest rank), so every rank gets about the same
    work however uneven the fields are."""
    if world < 1:
        raise ValueError("eda: world must be >= 1")
    cost = [int(np.prod(s)) * max(1, mode_bound(max(s))) for s in shapes]
    order = sorted(range(len(shapes)), key=lambda i: (-cost[i], i))
    load = [0] * world
    rank = [0] * len(shapes)
    for i in order:
        r = min(range(world), key=lambda j: (load[j], j))
        rank[i] = r
        load[r] += cost[i]
    return rank


def decompose_ragged_sharded(xs: list[np.ndarray], group: Any = None, gather: bool = True,
                             decompose: Callable[..., tuple[list, list]] | None = None,
                             **kwargs: Any) -> tuple[list, list]:
    """Decompose this rank's share of the ragged batch xs (host fields of different shapes, the
    share from ragged_assignment) and, with gather, return every field's rows and information on
    every rank, in input order (else this rank's, None elsewhere). The compute call is
    ``decompose(fields, **kwargs) -> (rows list, infos list)`` (default: eda.decompose_ragged with
    return_info). The results are collected with all_gather_object (pickled host arrays)."""
    import torch.distributed as dist

    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    owner = ragged_assignment([tuple(np.shape(x)) for x in xs], world)
    mine = [i for i in range(len(xs)) if owner[i] == rank]
    if decompose is None:
        from ._api import decompose_ragged

        def decompose(fields, **kw):
            return decompose_ragged(fields, return_info=True, **kw)
    rows_m, infos_m = decompose([xs[i] for i in mine], **kwargs) if mine else ([], [])
    rows: list = [None] * len(xs)
    infos: list = [None] * len(xs)
    for j, i in enumerate(mine):
        rows[i], infos[i] = rows_m[j], infos_m[j]
    if not gather or world == 1:
        return rows, infos
    parts: list = [None] * world
    dist.all_gather_object(parts, [(i, np.asarray(rows[i]), infos[i]) for i in mine], group=group)
    for part in parts:
        for i, r, inf in part:
            rows[i], infos[i] = r, inf
    return rows, infos
