"""Child process of tests/test_device_reset_gpu.py (run as a script, never
collected by pytest).

gtom's own test harness resets the device around every test
(GTOMTest/Norm.cpp:7,55,58: cudaDeviceReset()), so a drop-in library must
keep working after a caller destroys its context.  This process touches the
GPU only through the CUDA runtime (cuda-python) and the library's C ABI, no
torch, so that nothing but the library holds device state across the reset.

It runs every cached path once (the row-segment projector and
backprojector with their plan scratch and brick orders, the host-angle
overloads' kernel-parameter upload, the allocation-free projector's fixed
array, the gridding with its cuFFT plans and blob table, the fused-FFT
gridding with its twiddle table and launch attributes, the particle
preprocessing with its R2C plan), then:

  1. gtomrln_release_caches(), cudaDeviceReset(), and everything again;
  2. cudaDeviceReset() without releasing anything (the caches notice the new
     context by its id), and everything again;

and prints one JSON line with the largest differences to the first run.
Case 2 runs only when the driver reports a new context id after the reset;
otherwise the line says so.
"""
from __future__ import annotations

import ctypes as C
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from cuda.bindings import driver as drv  # noqa: E402
from cuda.bindings import runtime as rt  # noqa: E402

from gtom_b200 import _lib  # noqa: E402
from tests.synthdata import blob_volume_ft, random_angles  # noqa: E402

H2D = rt.cudaMemcpyKind.cudaMemcpyHostToDevice
D2H = rt.cudaMemcpyKind.cudaMemcpyDeviceToHost


def ok(res):
    err = res[0] if isinstance(res, tuple) else res
    if err != rt.cudaError_t.cudaSuccess:
        raise RuntimeError(f"CUDA runtime: {err}")
    return res[1] if isinstance(res, tuple) and len(res) > 1 else None


class Buf:
    def __init__(self, nbytes: int):
        self.nbytes = nbytes
        self.ptr = int(ok(rt.cudaMalloc(nbytes)))
        ok(rt.cudaMemset(self.ptr, 0, nbytes))

    def put(self, a: np.ndarray) -> "Buf":
        a = np.ascontiguousarray(a)
        assert a.nbytes <= self.nbytes
        ok(rt.cudaMemcpy(self.ptr, a.ctypes.data, a.nbytes, H2D))
        return self

    def get(self, dtype, count: int) -> np.ndarray:
        out = np.empty(count, dtype)
        ok(rt.cudaMemcpy(out.ctypes.data, self.ptr, out.nbytes, D2H))
        return out

    def free(self) -> None:
        ok(rt.cudaFree(self.ptr))


def context_id() -> int:
    err, ctx = drv.cuCtxGetCurrent()
    if err != drv.CUresult.CUDA_SUCCESS or int(ctx) == 0:
        return 0
    err, cid = drv.cuCtxGetId(ctx)
    return int(cid) if err == drv.CUresult.CUDA_SUCCESS else 0


def check(L, st: int, what: str) -> None:
    if st != 0:
        raise RuntimeError(f"{what}: status {st}: {L.gtomrln_last_error()}")


def run_all(L) -> dict[str, np.ndarray]:
    n, pad, batch = 32, 2, 64
    P, D = n * pad, n * pad + 1
    e = (n // 2 + 1) * n
    rng = np.random.default_rng(5)
    vol = blob_volume_ft(rng, n, P, 6)
    ang = np.ascontiguousarray(random_angles(rng, batch), np.float32)
    mats = np.empty((batch, 9), np.float32)
    check(L, L.gtomrln_matrices_from_angles(ang.ctypes.data, 2.0, batch, mats.ctypes.data), "matrices")
    out = {}
    bufs = []

    def buf(nbytes):
        b = Buf(nbytes)
        bufs.append(b)
        return b

    dvol = buf(vol.nbytes).put(vol)
    dmat = buf(mats.nbytes).put(mats)
    proj = buf(batch * e * 8)
    check(L, L.gtomrln_project(dvol.ptr, P, P, P, proj.ptr, n, n, 1, n // 2, dmat.ptr, batch, None), "project")
    out["project"] = proj.get(np.complex64, batch * e)
    proj2 = buf(batch * e * 8)
    check(L, L.gtomrln_project_angles(dvol.ptr, P, P, P, proj2.ptr, n, n, 1, ang.ctypes.data, C.c_float(2.0), batch,
                                      None), "project_angles")
    out["project_angles"] = proj2.get(np.complex64, batch * e)
    proj3 = buf(batch * e * 8)
    check(L, L.gtomrln_project_angles_noalloc(dvol.ptr, P, P, P, proj3.ptr, n, n, 1, ang.ctypes.data, C.c_float(2.0),
                                              batch, None), "project_angles_noalloc")
    out["project_noalloc"] = proj3.get(np.complex64, batch * e)

    nv = (D // 2 + 1) * D * D
    vf, vw = buf(nv * 8), buf(nv * 4)
    check(L, L.gtomrln_backproject(vf.ptr, vw.ptr, D, D, D, proj.ptr, None, n, n, 1, n // 2, dmat.ptr, None, 1.0, 0.0,
                                   0.0, 1.0, 0.0, 0, 0, batch, None), "backproject")
    out["backproject_data"] = vf.get(np.complex64, nv)
    out["backproject_weights"] = vw.get(np.float32, nv)

    rec = buf(n ** 3 * 4)
    for path, key in ((0, "gridding"), (4, "gridding_fused")):
        check(L, L.gtomrln_set_path(2, path), "set_path")
        check(L, L.gtomrln_reconstruct_gridding(vf.ptr, vw.ptr, rec.ptr, n, n, n, D, D, D, pad, 0, 0, 10, 1.9, 0, 15.0,
                                                None), key)
        out[key] = rec.get(np.float32, n ** 3)
    check(L, L.gtomrln_set_path(2, 0), "set_path")

    imgs = rng.normal(size=(batch, n, n)).astype(np.float32)
    dimg = buf(imgs.nbytes).put(imgs)
    pft, pw = buf(batch * e * 8), buf(batch * e * 4)
    check(L, L.gtomrln_preprocess_particles(dimg.ptr, n, batch, None, pft.ptr, pw.ptr, None), "preprocess")
    out["preprocess"] = pft.get(np.complex64, batch * e)

    ok(rt.cudaDeviceSynchronize())
    for b in bufs:
        b.free()
    return out


def rel(a: np.ndarray, b: np.ndarray) -> float:
    a64, b64 = a.astype(np.complex128), b.astype(np.complex128)
    den = np.linalg.norm(b64)
    return float(np.linalg.norm(a64 - b64) / (den if den > 0 else 1.0))


def compare(first, again) -> dict[str, float]:
    return {k: rel(again[k], first[k]) for k in first}


def main() -> None:
    L = _lib.load()
    ok(rt.cudaSetDevice(0))
    first = run_all(L)
    res = {"keys": sorted(first)}

    check(L, L.gtomrln_release_caches(), "release_caches")
    before = context_id()
    ok(rt.cudaDeviceReset())
    ok(rt.cudaSetDevice(0))
    after_release = run_all(L)
    res["released_then_reset"] = compare(first, after_release)
    res["context_changed_1"] = context_id() != before

    before = context_id()
    ok(rt.cudaDeviceReset())
    ok(rt.cudaFree(0))  # the runtime re-creates the primary context
    after = context_id()
    if after != before and after != 0:
        res["reset_without_release"] = compare(first, run_all(L))
    else:
        res["reset_without_release"] = f"skipped: context id {before} -> {after}"
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
