"""Autotuner for the brick-major projector and backprojector.

The brick kernels have three launch parameters whose best values depend on
the box size, the batch and the orientation distribution: the brick edge
(pixels per brick-slice pair versus shared memory per CTA), the threads per
CTA (latency hiding versus CTAs per SM) and the slices per work item (load
balance versus how often a brick is flushed to the volume).  `tune_project`
and `tune_backproject` time every candidate on the caller's own data with
CUDA events and install the fastest with set_brick_tuning; results can be
kept in a JSON file keyed by GPU, box and batch.

Candidates whose shared memory does not fit a CTA are skipped (the library
rejects them).  Timing is on the current stream, after one untimed call per
candidate; each candidate is timed `reps` times and its median kept.
"""
from __future__ import annotations

import itertools
import json
import statistics
from pathlib import Path
from typing import Callable, Iterable

import torch

from . import _lib
from .relion import set_brick_tuning, set_path

EDGES = (16, 20, 24, 26, 28, 29)
THREADS = (256, 512, 1024)
CHUNKS = (512, 2048, 8192)


def _smem(op: str, edge: int) -> int:
    return 8 * (edge + 1) ** 3 if op == "project" else 12 * edge * (edge + 1) ** 2


def candidates(op: str, edges: Iterable[int] = EDGES, threads: Iterable[int] = THREADS,
               chunks: Iterable[int] = CHUNKS) -> list[tuple[int, int, int]]:
    return [(e, t, c) for e, t, c in itertools.product(edges, threads, chunks)
            if _smem(op, e) <= 227 * 1024]


def _time(fn: Callable[[], None], reps: int) -> float:
    fn()
    ts = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return statistics.median(ts)


def tune(op: str, run: Callable[[], None], cands=None, reps: int = 3, path: str = "segment") -> dict:
    """Times `run` (one call of the op) under every candidate launch shape of
    the brick-major `path` ("segment", the default variant, or "brick") and
    installs the fastest.  Returns {"best": (edge, threads, chunk), "ms": ...,
    "table": [(edge, threads, chunk, ms), ...]}."""
    set_path(op, path)
    table = []
    try:
        for e, t, c in (cands or candidates(op)):
            try:
                set_brick_tuning(op, e, t, c)
            except _lib.GtomError:
                continue
            table.append((e, t, c, _time(run, reps)))
    finally:
        set_path(op, "auto")
    best = min(table, key=lambda r: r[3])
    set_brick_tuning(op, *best[:3])
    return {"best": best[:3], "ms": best[3], "table": table}


def save(path: str | Path, key: str, result: dict) -> None:
    p = Path(path)
    data = json.loads(p.read_text()) if p.exists() else {}
    data[key] = {"best": list(result["best"]), "ms": result["ms"]}
    p.write_text(json.dumps(data, indent=1))


def load(path: str | Path, key: str, op: str) -> bool:
    """Installs a saved best shape for `key`; returns whether one was found."""
    p = Path(path)
    if not p.exists():
        return False
    entry = json.loads(p.read_text()).get(key)
    if not entry:
        return False
    set_brick_tuning(op, *entry["best"])
    return True


def cache_key(op: str, box: int, pad: int, batch: int) -> str:
    return f"{torch.cuda.get_device_name()}|{op}|box{box}|pad{pad}|batch{batch}"
