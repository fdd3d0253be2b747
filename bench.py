# SPDX-License-Identifier: Apache-2.0
"""Benchmark of the decomposition on B200: decompositions per second of the 2-D workload of 64
float32 images of 512 x 512 (rings, wavy stripes, two Gaussian blobs and noise, seeded synthetic
inputs with the shapes and value ranges of the workload), one decomposition call of the batch per
step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU (torchrun for N > 1); every rank decomposes its own 64 images (weak scaling,
no collective on the data path); the time of a step is the maximum over ranks. Prints one JSON line
on rank 0:

- value: decompositions/s with the inputs resident in HBM (CUDA events around each call, the L2
  flushed between steps by writing a 256 MiB buffer);
- e2e: the same through the public call with host input in pinned memory, the host-to-device copy
  of the images and the device-to-host copy of the rows inside every step;
- roofline: the dominant kernel (the cube-filter passes): its algorithmic bytes over its summed
  CUDA-event time across the timed region against the measured copy bandwidth; traffic: DRAM bytes
  per launch from the committed ncu summary (profiles/), when one exists;
- cpu_baseline: the oracle (the CPU restatement of the method) on the host cores, one image per
  thread.

--impl reference times the reference's computation on the host cores: the reference ships no CPU
implementation of the path and its GPU build needs its own CMake build with cuFFT, so this arm runs
the oracle port of the same method (one image per host thread per step).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "eda-cuda_b200"))

BATCH = 64
SIDE = 512
METRIC = "decompositions/s (2-D 64 x 512^2 float32, sifts 3)"
UNIT = "decompositions/s"
PEAKS = ROOT / "MEASURED_PEAKS.json"
TRAFFIC = ROOT / "profiles" / "cube_pass_traffic.json"


def workload(batch: int, seed: int) -> np.ndarray:
    """The seeded synthetic images (batch, 512, 512) float32."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:SIDE, 0:SIDE].astype(np.float64)
    out = np.empty((batch, SIDE, SIDE), np.float32)
    stripes = 1.5 * np.cos(2 * np.pi * (x + 4 * np.sin(2 * np.pi * y / 128)) / 24)
    for b in range(batch):
        cy, cx = rng.uniform(0, SIDE, 2)
        f = np.cos(2 * np.pi * np.hypot(y - cy, x - cx) / 6) + stripes
        for _ in range(2):
            by, bx = rng.uniform(0, SIDE, 2)
            f = f + 3 * np.exp(-((y - by) ** 2 + (x - bx) ** 2) / (2 * 80.0**2))
        f = f + 0.02 * rng.standard_normal((SIDE, SIDE))
        out[b] = f.astype(np.float32)
    return out


def peak_hbm() -> tuple[float, str]:
    if PEAKS.exists():
        return float(json.loads(PEAKS.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples of the SM clock and the throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int) -> None:
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]
        return False

    def summary(self) -> dict:
        sm, mx, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in getattr(self, "lines", []):
            p = [v.strip() for v in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = max(mx, float(p[2]))
            except ValueError:
                continue
            for name, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_oracle(images: np.ndarray, threads: int, results: list | None = None) -> float:
    """Seconds for the oracle to decompose `images` with `threads` host threads; its (rows, info)
    are appended to `results` when given."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    t0 = time.perf_counter()
    out = oracle.decompose(images, threads=threads)
    secs = time.perf_counter() - t0
    if results is not None:
        results.append(out)
    return secs


def decisions_match(info, oinfo, count: int) -> int:
    """Elements among the first `count` whose IMF count, windows and sift counts equal the oracle's."""
    same = 0
    for b in range(count):
        k = int(info.n_imfs[b])
        if k != int(oinfo["n_imfs"][b]):
            continue
        if (np.array_equal(np.asarray(info.windows[b][:k]), oinfo["windows"][b][:k])
                and np.array_equal(np.asarray(info.sifts[b][:k]), oinfo["sifts"][b][:k])):
            same += 1
    return same


def host_cores() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


def dist_env() -> tuple[int, int, int]:
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def run_reference(args) -> None:
    rank, world, _ = dist_env()
    if rank != 0:
        return
    cores = host_cores()
    threads = max(1, min(cores, BATCH))
    images = workload(threads, 1234)
    for _ in range(args.warmup):
        cpu_oracle(images, threads)
    times = [cpu_oracle(images, threads) for _ in range(args.steps)]
    value = threads * len(times) / sum(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * sum(times) / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"2-D {BATCH} x {SIDE}x{SIDE} float32 images (rings, wavy stripes, blobs, noise)",
                   "sample_per_step": f"{threads} of the images, one per host thread"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{threads} images of {SIDE}x{SIDE} per step, one per thread; the reference has "
                                   "no CPU implementation of the path, so the oracle port runs its method"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args) -> None:
    import torch

    import eda
    from eda import _native

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
        pg = dist
    lib = _native.core()._lib
    lib.eda_profile_read.argtypes = [ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                                     ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    batch = args.batch
    x_host = workload(batch, 1000 + rank)
    x_dev = torch.from_numpy(x_host).to(dev)
    flush = torch.empty(64 << 20, dtype=torch.float32, device=dev)  # 256 MiB > L2
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize(dev)

    # the cube passes' launch shapes for this geometry (the autotuner; outside the timed region)
    tuned = eda.autotune((SIDE, SIDE), batch=batch) if args.tune else None
    # the clock sampler starts before the warm-up, so that its start-up stays out of the timed steps
    clk = Clocks(local).__enter__()
    # warm-up (device input)
    for _ in range(args.warmup):
        eda.decompose(x_dev, axes=(1, 2))
    barrier()
    # timed: device-resident inputs, events around each call, L2 flushed between calls
    lib.eda_profile(1)
    ms = []
    try:
        for _ in range(args.steps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            y = eda.decompose(x_dev, axes=(1, 2))
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
    finally:
        clk.__exit__(None, None, None)
    launches, cl, cb, cms = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_double(), ctypes.c_double()
    lib.eda_profile_read(ctypes.byref(launches), ctypes.byref(cl), ctypes.byref(cb), ctypes.byref(cms))
    lib.eda_profile(0)
    P = y.shape[1]
    barrier()
    total_ms = sum(ms)
    if pg is not None:
        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms = float(t.item())
    value = batch * world * args.steps / (total_ms / 1000.0)
    # end to end: host input from pinned memory, rows back to the host, every step
    pinned = torch.empty(x_host.shape, dtype=torch.float32).pin_memory()
    pinned.numpy()[...] = x_host
    xp = pinned.numpy()
    e2e_ms = []
    d2h = 0
    for _ in range(0 if args.no_e2e else args.warmup):
        eda.decompose(xp, axes=(1, 2))  # untimed: the host path's first-use allocations
    for _ in range(0 if args.no_e2e else args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        rows = eda.decompose(xp, axes=(1, 2))
        e2e_ms.append(1000 * (time.perf_counter() - t0))
        d2h = rows.nbytes
    e2e_total = sum(e2e_ms) if e2e_ms else float("nan")
    if pg is not None:
        t = torch.tensor([e2e_total], device=dev, dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e = batch * world * args.steps / (e2e_total / 1000.0)
    cpu = None
    check = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = max(1, min(host_cores(), batch))
        got = []
        secs = cpu_oracle(x_host[:threads], threads, got)
        cpu = {"value": threads / secs, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{threads} of the {batch} images ({SIDE}x{SIDE} float32), one per host thread, "
                         f"{secs:.1f} s"}
        # correctness on the benchmarked workload, outside the timed region: the decisions of the
        # oracle's images against the engine's, and the rows of a seeded subset against the oracle
        # run in float64
        y_chk, info_chk = eda.decompose(x_dev[:threads], axes=(1, 2), return_info=True)
        y_chk = y_chk.cpu().numpy() if hasattr(y_chk, "cpu") else np.asarray(y_chk)
        n64 = min(4, threads)
        check = {"decisions_equal": decisions_match(info_chk, got[0][1], threads), "decisions_checked": threads,
                 "fp64_err": fp64_error([x_host[b] for b in range(n64)], [y_chk[b] for b in range(n64)], n64)}
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    if rank != 0:
        return
    peak, peak_kind = peak_hbm()
    achieved = (cb.value / (cms.value / 1000.0)) / 1e9 if cms.value > 0 else None
    traffic = None
    if TRAFFIC.exists():
        traffic = json.loads(TRAFFIC.read_text()).get("dram_bytes_per_launch")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "step_ms": {"min": min(ms), "median": statistics.median(ms), "max": max(ms),
                    "all": [round(v, 3) for v in ms]} if ms else None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"2-D {batch} x {SIDE}x{SIDE} float32 images per GPU (rings, wavy stripes, blobs, "
                               "noise), sifts 3", "l2": "flushed between steps (256 MiB write)",
                   "rows_per_element": int(P), "parallelism": f"replicas x{world}",
                   "cube_launch_shape": tuned},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(x_host.nbytes), "d2h_bytes_per_step": int(d2h)},
        "roofline": {"bound": "hbm", "kernel": "cube_pass", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "peak_kind": peak_kind,
                     "traffic": traffic, "launches": int(cl.value),
                     "algorithmic_bytes_per_launch": (cb.value / cl.value) if cl.value else None,
                     "share_of_step": (cms.value / total_ms) if total_ms else None},
        "gpu_launches": int(launches.value),
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
        "parity": check,
        "fp64_err": check["fp64_err"] if check else None,
    }
    print(json.dumps(line), flush=True)


def signal_1d(seed: int) -> np.ndarray:
    """The 1-D configuration: one 2048-sample float32 signal (three tones and noise), shape (1, 2048)."""
    rng = np.random.default_rng(seed)
    t = np.arange(2048, dtype=np.float64)
    x = np.sin(2 * np.pi * t / 8) + 2 * np.sin(2 * np.pi * t / 64) + 3 * np.sin(2 * np.pi * t / 512)
    return (x + 0.01 * rng.standard_normal(t.size)).astype(np.float32)[None]


def volumes_3d(batch: int, n: int, seed: int) -> np.ndarray:
    """The 3-D configuration at side n (256 in the benchmark): spherical shells cos(2 pi r / 8), a plane
    wave along z with its period rising from 32 to 64 voxels, a Gaussian trend of sigma 90 n / 256,
    noise 0.01 N(0, 1); (batch, n, n, n) float32."""
    rng = np.random.default_rng(seed)
    z, y, x = np.mgrid[0:n, 0:n, 0:n].astype(np.float32)
    out = np.empty((batch, n, n, n), np.float32)
    period = 32 + 32 * z / (n - 1)
    sigma = 90.0 * n / 256
    for b in range(batch):
        c = rng.uniform(0, n, 3)
        r = np.sqrt((z - c[0]) ** 2 + (y - c[1]) ** 2 + (x - c[2]) ** 2)
        g = rng.uniform(0, n, 3)
        f = np.cos(2 * np.pi * r / 8) + np.cos(2 * np.pi * z / period)
        f += 3 * np.exp(-((z - g[0]) ** 2 + (y - g[1]) ** 2 + (x - g[2]) ** 2) / (2 * sigma ** 2))
        out[b] = f + 0.01 * rng.standard_normal((n, n, n)).astype(np.float32)
    return out


def signals_ragged(count: int, lo: int, hi: int, seed: int) -> list[np.ndarray]:
    """The 1-D ragged configuration: lengths exp(U[ln lo, ln hi]); a linear chirp 0.002 -> 0.2
    cycles/sample, 0.8 cos(w t + 0.8 sin w t) with w ~ U[0.05, 0.3], a slope ~ U[-1e-3, 1e-3], noise."""
    rng = np.random.default_rng(seed)
    xs = []
    for _ in range(count):
        n = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        t = np.arange(n, dtype=np.float64)
        w = rng.uniform(0.05, 0.3)
        f = np.cos(2 * np.pi * (0.002 * t + 0.5 * (0.2 - 0.002) / n * t * t)) + 0.8 * np.cos(w * t + 0.8 * np.sin(w * t))
        f += rng.uniform(-1e-3, 1e-3) * t + 0.01 * rng.standard_normal(n)
        xs.append(f.astype(np.float32))
    return xs


def images_ragged(count: int, lo: int, hi: int, seed: int) -> list[np.ndarray]:
    """The 2-D ragged configuration: height and width each U[lo, hi]; the 2-D recipe with the ring and
    stripe periods and the blob width scaled by side / 512."""
    rng = np.random.default_rng(seed)
    xs = []
    for _ in range(count):
        h, w = (int(v) for v in rng.integers(lo, hi + 1, 2))
        s = np.sqrt(h * w) / 512
        y, x = np.mgrid[0:h, 0:w].astype(np.float32)
        cy, cx = rng.uniform(0, h), rng.uniform(0, w)
        f = np.cos(2 * np.pi * np.hypot(y - cy, x - cx) / (6 * s))
        f += 1.5 * np.cos(2 * np.pi * (x + 4 * s * np.sin(2 * np.pi * y / (128 * s))) / (24 * s))
        for _ in range(2):
            by, bx = rng.uniform(0, h), rng.uniform(0, w)
            f += 3 * np.exp(-((y - by) ** 2 + (x - bx) ** 2) / (2 * (80 * s) ** 2))
        xs.append((f + 0.02 * rng.standard_normal((h, w))).astype(np.float32))
    return xs


def other_workload(name: str, seed: int):
    """The other configurations of the method's benchmark suite (seeded synthetic stand-ins):
    returns (description, list of fields or one batch array, axes, elements)."""
    if name == "1d":
        return "1-D 1 x 2048 float32 (three tones and noise), sifts 3", signal_1d(seed), (1,), 1
    if name == "3d":
        return ("3-D 4 x 256^3 float32 (spherical waves, chirped plane wave, trend, noise), sifts 3",
                volumes_3d(4, 256, seed), (1, 2, 3), 4)
    if name == "ragged1d":
        return ("1-D ragged 1024 signals, lengths exp(U[ln 256, ln 65536]) float32 (chirp, FM tone, slope, noise), "
                "sifts 3", signals_ragged(1024, 256, 65536, seed), None, 1024)
    if name == "ragged1d-short":
        return ("1-D ragged 1024 signals, lengths exp(U[ln 256, ln 8192]) float32 (chirp, FM tone, slope, noise), "
                "sifts 3", signals_ragged(1024, 256, 8192, seed), None, 1024)
    if name == "ragged2d":
        return ("2-D ragged 256 images, sides U[64, 2048] float32 (the 2-D recipe scaled by side / 512), sifts 3",
                images_ragged(256, 64, 2048, seed), None, 256)
    raise ValueError(name)


def fp64_error(fields: list[np.ndarray], results: list[np.ndarray], threads: int) -> dict:
    """The FP64 error of float32 results: each field is decomposed again by the oracle in float64
    (the same sift, every rounding in double) and max |y - y64| over the rows is taken, rel = that
    over max |x|; the worst element is reported. Elements whose float64 decisions (IMF count,
    windows) differ from the float32 result's are counted apart (their rows are not comparable)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    from concurrent.futures import ThreadPoolExecutor

    def one(i):
        x = fields[i]
        rows64, info64 = oracle.decompose(x[None].astype(np.float64))
        y = np.asarray(results[i], dtype=np.float64)
        k = int(info64["n_imfs"][0]) + 1
        if y.shape[0] < k or np.any(y[k:] != 0):
            return None
        d = float(np.abs(y[:k] - rows64[0, :k]).max())
        return d, d / float(np.abs(x).max())

    with ThreadPoolExecutor(max_workers=max(1, threads)) as ex:
        out = list(ex.map(one, range(len(fields))))
    ok = [o for o in out if o is not None]
    return {"max_abs": max((o[0] for o in ok), default=None), "rel": max((o[1] for o in ok), default=None),
            "n_checked": len(ok), "decisions_differ": len(out) - len(ok), "oracle": "float64 restatement of the sift"}


def check_fields(name: str, data) -> tuple[list[np.ndarray], tuple | None, str]:
    """The seeded subset whose rows are checked against the float64 oracle, with its axes (None:
    ragged) and a description: the whole 1-D workload; one 128^3 volume of the 3-D recipe (a 256^3
    volume takes the oracle minutes); four fields of the ragged workloads (the shortest)."""
    if name == "1d":
        return [data[0]], (1,), "the signal"
    if name == "3d":
        return [volumes_3d(1, 128, 7)[0]], (1, 2, 3), "one 128^3 volume of the same recipe (seed 7)"
    order = sorted(range(len(data)), key=lambda i: data[i].size)[:4]
    return [data[i] for i in order], None, "the four smallest fields of the batch"


def run_other(args) -> None:
    """One JSON line for a configuration other than the 2-D benchmark (1 GPU): decompositions/s with
    device-resident inputs (CUDA events around each call) and through host inputs (e2e). For 2-D and
    3-D workloads every product of the float32 orientation transforms is timed too ("arms": 3xTF32
    and BF16x3 split products on the tensor cores, plain float32), each with its float64 error; the
    line's value is the default arm's (3xTF32)."""
    import torch

    import eda

    dev = torch.device("cuda", 0)
    desc, data, axes, elements = other_workload(args.workload, 2024)
    if args.length_class is not None:  # one length class of a ragged 1-D workload (profiling)
        if axes is not None or data[0].ndim != 1:
            raise SystemExit("--length-class applies to the ragged 1-D workloads")
        k = args.length_class
        data = [x for x in data if (1 << k) <= x.size < (2 << k)]
        if not data:
            raise SystemExit(f"no signal of the workload has a length in [2^{k}, 2^{k + 1})")
        desc += f"; only the {len(data)} signals of lengths [2^{k}, 2^{k + 1})"
        elements = len(data)
    ragged = axes is None
    if ragged:
        eda.set_length_classes(not args.exact_lengths)
        on_dev = [torch.from_numpy(x).to(dev) for x in data]
        call_dev = lambda: eda.decompose_ragged(on_dev, workers=args.workers)  # noqa: E731
        call_host = lambda: eda.decompose_ragged(data, workers=args.workers)  # noqa: E731
        h2d = sum(x.nbytes for x in data)
    else:
        on_dev = torch.from_numpy(data).to(dev)
        call_dev = lambda: eda.decompose(on_dev, axes=axes)  # noqa: E731
        call_host = lambda: eda.decompose(data, axes=axes)  # noqa: E731
        h2d = data.nbytes
    flush = torch.empty(64 << 20, dtype=torch.float32, device=dev)
    if args.tune and not ragged:
        eda.autotune(data.shape[1:], batch=data.shape[0])
    clk = Clocks(0).__enter__()  # started before the warm-up (its start-up stays out of the timed steps)
    for _ in range(args.warmup):
        call_dev()
    torch.cuda.synchronize(dev)
    ms = []
    try:
        for _ in range(args.steps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            call_dev()
            e1.record()
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
    finally:
        clk.__exit__(None, None, None)
    for _ in range(0 if args.no_e2e else args.warmup):
        call_host()
    wall, d2h = [], 0
    for _ in range(0 if args.no_e2e else args.steps):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        out = call_host()
        wall.append(1000 * (time.perf_counter() - t0))
        d2h = sum(np.asarray(r).nbytes for r in out) if ragged else out.nbytes
    total = sum(ms)
    # the float64 error of a seeded subset, outside the timed regions
    fields, faxes, fdesc = check_fields(args.workload, data)

    def subset_err():
        if faxes is None:
            ys = eda.decompose_ragged(fields)
        else:
            y = eda.decompose(np.stack(fields), axes=faxes)
            ys = [y[b] for b in range(len(fields))]
        err = fp64_error(fields, ys, max(1, min(host_cores(), len(fields))))
        err["sample"] = fdesc
        return err

    arms = None
    spatial_dims = len(axes) if axes is not None else data[0].ndim
    if spatial_dims >= 2 and not args.no_cpu:
        arms = {}
        for arm in eda.TRANSFORM_PRECISIONS:
            eda.set_transform_precision(arm)
            for _ in range(max(1, args.warmup)):
                call_dev()
            torch.cuda.synchronize(dev)
            am = []
            for _ in range(args.steps):
                flush.fill_(1.0)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                call_dev()
                e1.record()
                e1.synchronize()
                am.append(e0.elapsed_time(e1))
            arms[arm] = {"value": elements * args.steps / (sum(am) / 1000.0), "ms_per_step": sum(am) / args.steps,
                         "fp64_err": subset_err()}
        eda.set_transform_precision("tf32x3")
        arms["ratio_tf32x3_vs_fp32"] = arms["tf32x3"]["value"] / arms["fp32"]["value"]
        arms["ratio_bf16x3_vs_fp32"] = arms["bf16x3"]["value"] / arms["fp32"]["value"]
    err = arms["tf32x3"]["fp64_err"] if arms else (subset_err() if not args.no_cpu else None)
    line = {
        "metric": f"decompositions/s ({args.workload})", "value": elements * args.steps / (total / 1000.0),
        "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": desc, "l2": "flushed between steps (256 MiB write)",
                   **({"workers": args.workers,
                       "grouping": "exact shapes" if args.exact_lengths or data[0].ndim > 1 else "1-D length classes"}
                      if ragged else {})},
        "e2e": {"value": elements * args.steps / (sum(wall) / 1000.0) if wall else None, "unit": UNIT,
                "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "clocks": clk.summary(),
        "fp64_err": err,
        "arms": arms,
    }
    print(json.dumps(line), flush=True)


import ctypes  # noqa: E402


def write_traffic(csv_path: Path) -> None:
    """Sums dram__bytes_read.sum + dram__bytes_write.sum over the cube-pass launches of an ncu CSV
    log (one row per metric and launch) into the per-launch DRAM traffic the roofline reports."""
    import csv

    rows = list(csv.reader(csv_path.open()))
    h = next(i for i, r in enumerate(rows) if "Kernel Name" in r)
    hdr = rows[h]
    ki, mi, vi, ui, ii = (hdr.index(k) for k in ("Kernel Name", "Metric Name", "Metric Value", "Metric Unit", "ID"))
    scale = {"byte": 1.0, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9}
    per: dict[str, float] = {}
    for r in rows[h + 1:]:
        if "cube_pass" in r[ki] and r[mi] in ("dram__bytes_read.sum", "dram__bytes_write.sum"):
            per[r[ii]] = per.get(r[ii], 0.0) + float(r[vi].replace(",", "")) * scale[r[ui]]
    if not per:
        raise SystemExit(f"{csv_path}: no cube_pass DRAM metrics")
    out = {"kernel": "cube_pass", "launches": len(per), "dram_bytes": sum(per.values()),
           "dram_bytes_per_launch": sum(per.values()) / len(per)}
    TRAFFIC.write_text(json.dumps(out, indent=1) + "\n")
    print(json.dumps(out))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end loop (profiling runs)")
    ap.add_argument("--workers", type=int, default=8,
                    help="concurrent shape groups of the ragged workloads (host threads with their own streams)")
    ap.add_argument("--length-class", type=int, default=None, metavar="K",
                    help="ragged 1-D workloads: only the signals of lengths [2^K, 2^(K+1)) (profiling one class)")
    ap.add_argument("--exact-lengths", action="store_true",
                    help="ragged 1-D workloads: group the signals by exact length instead of length class")
    ap.add_argument("--tune", action="store_true",
                    help="autotune the cube passes' launch shapes for the workload's geometry before the warm-up "
                         "(on the 2-D workload the tuner keeps the default shape)")
    ap.add_argument("--batch", type=int, default=BATCH,
                    help="images per GPU of the 2-D benchmark (64; smaller only for profiling captures)")
    ap.add_argument("--workload", default="2d", choices=("2d", "1d", "3d", "ragged1d", "ragged1d-short", "ragged2d"),
                    help="2d: the benchmark (default); the others measure the remaining configurations on 1 GPU")
    ap.add_argument("--traffic-from", metavar="CSV",
                    help="write the cube passes' DRAM bytes per launch from an ncu --csv log of "
                         "dram__bytes_read.sum and dram__bytes_write.sum to profiles/ and exit")
    args = ap.parse_args()
    if args.traffic_from:
        write_traffic(Path(args.traffic_from))
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload != "2d":
        run_other(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
