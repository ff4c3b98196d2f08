"""Batched reconstruction of many volumes of uneven box size.

`BatchReconstructor` wraps gtomrln_batch_create / _run / _destroy: every
slice of every subvolume is inserted by one persistent kernel launch and
each box size is gridding-corrected as a stack, the whole run captured once
in a CUDA graph and replayed.  `reconstruct_separately` is the same work as
one d_rlnBackproject + d_ReconstructGridding call pair per subvolume (what a
caller of the reference does), and `autotune` picks the insertion launch
shape by timing the caller's own batch.
"""
from __future__ import annotations

import ctypes as C
import itertools
import statistics
from dataclasses import dataclass

import torch

from . import _lib
from .relion import _dev_ptr, _stream, d_ReconstructGridding, d_rlnBackproject


class _Subvolume(C.Structure):
    _fields_ = [("box", C.c_int), ("nslices", C.c_int), ("d_projft", C.c_void_p),
                ("d_projweights", C.c_void_p), ("d_matrices", C.c_void_p), ("d_out", C.c_void_p)]


@dataclass
class Subvolume:
    """One reconstruction: `nslices` half-complex box x box slices (complex64,
    or None for value 1), their weights (float32, or None for 1), their
    rotation matrices (nslices x 9, as d_rlnBackproject's, supersampled by
    the padding factor) and the box^3 float32 output map."""
    box: int
    projft: torch.Tensor | None
    projweights: torch.Tensor | None
    matrices: torch.Tensor
    out: torch.Tensor

    @property
    def nslices(self) -> int:
        return self.matrices.numel() // 9


class BatchReconstructor:
    def __init__(self, subvolumes: list[Subvolume], paddingfactor: int = 2, iterations: int = 10):
        self.subvolumes = list(subvolumes)  # keeps the tensors alive for the handle
        self.paddingfactor = int(paddingfactor)
        self.iterations = int(iterations)
        arr = (_Subvolume * len(self.subvolumes))()
        for k, s in enumerate(self.subvolumes):
            e = (s.box // 2 + 1) * s.box * s.nslices
            arr[k] = _Subvolume(
                int(s.box), int(s.nslices),
                _dev_ptr(s.projft, "projft", torch.complex64, e, optional=True).value,
                _dev_ptr(s.projweights, "projweights", torch.float32, e, optional=True).value,
                _dev_ptr(s.matrices, "matrices", torch.float32, 9 * s.nslices).value,
                _dev_ptr(s.out, "out", torch.float32, s.box ** 3).value)
        h = C.c_void_p()
        _lib.call("gtomrln_batch_create", C.cast(arr, C.c_void_p), len(self.subvolumes),
                  self.paddingfactor, self.iterations, C.byref(h))
        self._handle = h
        self.tuning = (256, 4, 4)

    def set_tuning(self, threads: int = 0, slices_per_item: int = 0, blocks_per_sm: int = 0) -> None:
        _lib.call("gtomrln_batch_set_tuning", self._handle, int(threads), int(slices_per_item),
                  int(blocks_per_sm))
        t = list(self.tuning)
        for i, v in enumerate((threads, slices_per_item, blocks_per_sm)):
            if v:
                t[i] = int(v)
        self.tuning = tuple(t)

    def run(self, use_graph: bool = True, stream=None) -> None:
        _lib.call("gtomrln_batch_run", self._handle, int(bool(use_graph)), _stream(stream))

    def close(self) -> None:
        if getattr(self, "_handle", None) is not None and self._handle.value:
            _lib.load().gtomrln_batch_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def reconstruct_separately(subvolumes: list[Subvolume], paddingfactor: int = 2,
                           iterations: int = 10, scratch: dict | None = None) -> None:
    """One d_rlnBackproject + d_ReconstructGridding pair per subvolume, into
    zeroed centred accumulators (the reference caller's loop).  `scratch`
    may hold accumulators by box to reuse across calls."""
    scratch = {} if scratch is None else scratch
    for s in subvolumes:
        P = s.box * paddingfactor
        D = P + 1
        nvol = (D // 2 + 1) * D * D
        if s.box not in scratch:
            dev = s.matrices.device
            scratch[s.box] = (torch.empty(nvol, dtype=torch.complex64, device=dev),
                              torch.empty(nvol, dtype=torch.float32, device=dev))
        acc_ft, acc_w = scratch[s.box]
        acc_ft.zero_()
        acc_w.zero_()
        d_rlnBackproject(acc_ft, acc_w, (D, D, D), s.projft, s.projweights, (s.box, s.box, 1), s.box // 2,
                         s.matrices.reshape(-1), None, (1, 0, 0, 1), 0.0, False, False, s.nslices)
        d_ReconstructGridding(acc_ft, acc_w, s.out, (s.box,) * 3, (D, D, D), paddingfactor, 0, 0, iterations)


THREADS = (128, 256, 512)
SLICES = (1, 2, 4, 8)
BLOCKS_PER_SM = (2, 4, 8)


def autotune(rec: BatchReconstructor, threads=THREADS, slices=SLICES, blocks=BLOCKS_PER_SM,
             reps: int = 3) -> dict:
    """Times a whole graph run (capture excluded) under every launch shape of
    the insertion kernel and installs the fastest.  Returns {"best": (threads,
    slices per item, CTAs per SM), "ms": ..., "table": [...]}."""
    table = []
    for t, s, b in itertools.product(threads, slices, blocks):
        rec.set_tuning(t, s, b)
        rec.run()  # capture + one untimed run
        ts = []
        for _ in range(reps):
            a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            rec.run()
            e.record()
            e.synchronize()
            ts.append(a.elapsed_time(e))
        table.append((t, s, b, statistics.median(ts)))
    best = min(table, key=lambda r: r[3])
    rec.set_tuning(*best[:3])
    return {"best": best[:3], "ms": best[3], "table": table}
