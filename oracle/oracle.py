"""CPU oracle for the RELION-style projector / backprojector / gridding path.

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as
the checker, and by bench.py's CPU-baseline leg.  The product library
(gtom_b200/) never imports it.

* project / backproject: ctypes over oracle_core.cpp (FP64 oracle, plus the
  FP32 OpenMP port used as the CPU baseline), built by oracle/Makefile.
* reconstruct_gridding: d_ReconstructGridding (src/Reconstruction/
  RecFourier.cu:98-241) restated in float64 numpy, with numpy's pocketfft
  for the transforms (normalisation as in src/FFT/IFFT.cu:36-56).

Parity pin: the restatement is checked against the reference's own CUDA path
(oracle/_ref/libgtomref.so, built from the reference sources by
`make -C oracle ref`) through the fixtures in tests/golden/.
"""
from __future__ import annotations

import ctypes as C
import subprocess
import threading
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"
REF_PATH = HERE / "_ref" / "libgtomref.so"

_lock = threading.Lock()
_lib = None


def lib() -> C.CDLL:
    """Loads (building if needed) liboracle.so."""
    global _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                subprocess.run(["make", "-C", str(HERE)], check=True, capture_output=True)
            L = C.CDLL(str(LIB_PATH))
            p, i, f, d = C.c_void_p, C.c_int, C.c_float, C.c_double
            L.orc_matrices_f64.argtypes = [p, i, d, p]
            L.orc_project_f64.argtypes = [p, i, p, i, i, i, p, i]
            L.orc_project_f32.argtypes = [p, i, p, i, i, i, p, i]
            bp = [p, p, i, p, p, i, i, i, p, p, p, f, i, i, i, i]
            L.orc_backproject_f64.argtypes = bp
            L.orc_backproject_f32.argtypes = bp
            L.orc_project_shifted_f64.argtypes = [p, i, p, i, i, i, p, p, p, i]
            L.orc_backproject_shifted_f64.argtypes = [p, p, i, p, p, i, i, i, p, p, p, i]
            L.orc_kaiser_fourier_value.argtypes = [d, d, d, i]
            L.orc_kaiser_fourier_value.restype = d
            L.orc_kb_table.argtypes = [d, d, i, i, p]
            L.orc_num_threads.restype = i
            L.orc_set_threads.argtypes = [i]
            _lib = L
    return _lib


def elements_fft(n: int, ndims: int = 2) -> int:
    return (n // 2 + 1) * n * (n if ndims == 3 else 1)


def _ptr(a) -> int:
    return 0 if a is None else a.ctypes.data


def _c(a, dtype) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=dtype)


def matrices_f64(angles: np.ndarray, supersample: float) -> np.ndarray:
    """s * A^T per slice, (batch, 9) column-major, float64 (Euler.cu:39-68)."""
    ang = _c(angles, np.float32).reshape(-1, 3)
    out = np.empty((ang.shape[0], 9), np.float64)
    lib().orc_matrices_f64(ang.ctypes.data, ang.shape[0], float(supersample), out.ctypes.data)
    return out


def project(volume: np.ndarray, P: int, n: int, rmax: int, mats: np.ndarray, ndims: int = 2,
            fp32: bool = False) -> np.ndarray:
    """Project3DArraytoNDKernel (Project.cu:89-177).  volume: complex64
    decentred half volume of P; mats: (batch, 9) float32.  Returns
    (batch, elements) complex128 (complex64 with fp32=True)."""
    vol = _c(volume, np.complex64)
    m = _c(mats, np.float32).reshape(-1, 9)
    batch = m.shape[0]
    e = elements_fft(n, ndims)
    rmax = min(int(rmax), n // 2)
    if fp32:
        out = np.zeros((batch, e), np.complex64)
        lib().orc_project_f32(vol.ctypes.data, P, out.ctypes.data, n, ndims, rmax, m.ctypes.data, batch)
    else:
        out = np.zeros((batch, e), np.complex128)
        lib().orc_project_f64(vol.ctypes.data, P, out.ctypes.data, n, ndims, rmax, m.ctypes.data, batch)
    return out


def backproject(volft: np.ndarray | None, volw: np.ndarray | None, P: int, projft, projw,
                n: int, rmax: int, mats: np.ndarray, ivolume=None, magnification=(1, 0, 0, 1),
                ewaldradiussuper: float = 0.0, decentered: bool = True, square: bool = False,
                half_weights: bool = True, ndims: int = 2, fp32: bool = False) -> None:
    """Backproject3DtoNDKernel (Backproject.cu:126-322), accumulating in place
    into volft (complex128, or complex64 with fp32) and volw (float64 /
    float32).  half_weights rounds the trilinear weights through binary16 as
    the reference does."""
    m = _c(mats, np.float32).reshape(-1, 9)
    batch = m.shape[0]
    pf = None if projft is None else _c(projft, np.complex64)
    pw = None if projw is None else _c(projw, np.float32)
    iv = None if ivolume is None else _c(ivolume, np.int32)
    mag = np.asarray(magnification, np.float32)
    rmax = min(int(rmax), n // 2)
    ewinv = 0.0 if ewaldradiussuper == 0 else float(np.float32(1.0) / (np.float32(2.0) * np.float32(ewaldradiussuper)))
    fn = lib().orc_backproject_f32 if fp32 else lib().orc_backproject_f64
    for a, dt in ((volft, np.complex64 if fp32 else np.complex128), (volw, np.float32 if fp32 else np.float64)):
        if a is not None and (a.dtype != dt or not a.flags.c_contiguous):
            raise ValueError(f"accumulator must be contiguous {dt}")
    fn(_ptr(volft), _ptr(volw), P, _ptr(pf), _ptr(pw), n, ndims, rmax, m.ctypes.data, _ptr(iv),
       mag.ctypes.data, C.c_float(ewinv), int(decentered), int(square), int(half_weights), batch)


def scaled_shifts(h_shifts, n: int) -> np.ndarray:
    """The matrix overloads' shifts: pixels * 2 pi / n in float32, as the
    h_angles overloads compute them (ProjectShifted.cu:40-44)."""
    h = np.asarray(h_shifts, np.float32).reshape(-1, 3)
    return (h * np.float32(6.283185307179586) / np.float32(n)).astype(np.float32)


def project_shifted(volume: np.ndarray, P: int, n: int, rmax: int, mats: np.ndarray, shifts,
                    globalweights, ndims: int = 2) -> np.ndarray:
    """ProjectShifted3DArraytoNDKernel (ProjectShifted.cu:124-224) in
    float64: the projection times exp(-i (x sx + y sy [+ z sz])) times the
    slice's global weight.  shifts: (batch, 3) already scaled by 2 pi / n."""
    vol = _c(volume, np.complex64)
    m = _c(mats, np.float32).reshape(-1, 9)
    batch = m.shape[0]
    sh = _c(shifts, np.float32).reshape(batch, 3)
    gw = _c(globalweights, np.float32).reshape(batch)
    out = np.zeros((batch, elements_fft(n, ndims)), np.complex128)
    lib().orc_project_shifted_f64(vol.ctypes.data, P, out.ctypes.data, n, ndims, min(int(rmax), n // 2),
                                  m.ctypes.data, sh.ctypes.data, gw.ctypes.data, batch)
    return out


def backproject_shifted(volft, volw, V: int, projft, projw, n: int, rmax: int, mats, shifts,
                        globalweights, ndims: int = 2) -> None:
    """BackprojectShifted3DtoNDKernel (BackprojectShifted.cu:67-186) in
    float64, accumulating into volft (complex128) / volw (float64), centred
    volumes of V; indices clamped as in the unshifted backprojector."""
    m = _c(mats, np.float32).reshape(-1, 9)
    batch = m.shape[0]
    pf = None if projft is None else _c(projft, np.complex64)
    pw = None if projw is None else _c(projw, np.float32)
    sh = _c(shifts, np.float32).reshape(batch, 3)
    gw = _c(globalweights, np.float32).reshape(batch)
    for a, dt in ((volft, np.complex128), (volw, np.float64)):
        if a is not None and (a.dtype != dt or not a.flags.c_contiguous):
            raise ValueError(f"accumulator must be contiguous {dt}")
    lib().orc_backproject_shifted_f64(_ptr(volft), _ptr(volw), V, _ptr(pf), _ptr(pw), n, ndims,
                                      min(int(rmax), n // 2), m.ctypes.data, sh.ctypes.data, gw.ctypes.data,
                                      batch)


def kb_table(radius: float, alpha: float, order: int = 0, nsamples: int = 10000) -> np.ndarray:
    out = np.empty(nsamples, np.float64)
    lib().orc_kb_table(float(radius), float(alpha), int(order), int(nsamples), out.ctypes.data)
    return out


def kaiser_fourier_value(w: float, a: float, alpha: float, m: int) -> float:
    return lib().orc_kaiser_fourier_value(float(w), float(a), float(alpha), int(m))


# --------------------------------------------------------------- gridding --
def _decenter(src: np.ndarray, P: int, old: tuple[int, int, int]) -> np.ndarray:
    """DecenterKernel (RecFourier.cu:264-285) onto the P-grid half volume, with
    reads outside the centred input counted as 0."""
    ox, oy, oz = old
    src = src.reshape(oz, oy, ox // 2 + 1)
    z = np.arange(P)
    zp = np.where(z < P // 2 + 1, z, z - P)
    x = np.arange(P // 2 + 1)
    rr = zp[:, None, None] ** 2 + zp[None, :, None] ** 2 + x[None, None, :] ** 2
    mask = (rr < (P * P) // 4).astype(np.float64)
    zi = zp + oz // 2
    yi = zp + oy // 2
    valid = ((zi >= 0) & (zi < oz))[:, None, None] & ((yi >= 0) & (yi < oy))[None, :, None] \
        & (x < ox // 2 + 1)[None, None, :]
    zc = np.clip(zi, 0, oz - 1)
    yc = np.clip(yi, 0, oy - 1)
    xc = np.clip(x, 0, ox // 2)
    out = src[zc[:, None, None], yc[None, :, None], xc[None, None, :]].astype(
        np.complex128 if np.iscomplexobj(src) else np.float64)
    return np.where(valid, out, 0) * mask


def reconstruct_gridding(dataft: np.ndarray, weight: np.ndarray, ori: int, dimspadded,
                         pad: int = 2, iterations: int = 10, blobradius: float = 1.9,
                         bloborder: int = 0, blobalpha: float = 15.0,
                         return_weights: bool = False):
    """d_ReconstructGridding in float64.  dataft (complex) / weight (real) are
    centred half volumes of dimspadded; returns the real ori^3 map
    (z, y, x), and the final gridding weights when return_weights."""
    old = tuple(int(v) for v in dimspadded)
    P = ori * pad
    nsamp = 10000
    sampling = 0.5 / nsamp
    table = kb_table(blobradius * pad, blobalpha, bloborder, nsamp)
    k = np.arange(P)
    kp = np.where(k < P // 2, k, k - P).astype(np.float64)
    r = np.sqrt(kp[:, None, None] ** 2 + kp[None, :, None] ** 2 + kp[None, None, :] ** 2) / P / sampling
    blob = table[np.minimum(nsamp - 1, r.astype(np.int64))]

    Fw = _decenter(np.asarray(weight, np.float64), P, old).real
    zs = np.arange(P)
    zsp = np.where(zs < P // 2 + 1, zs, zs - P)
    x = np.arange(P // 2 + 1)
    r2 = zsp[:, None, None] ** 2 + zsp[None, :, None] ** 2 + x[None, None, :] ** 2
    rmaxp = (ori // 2) * pad
    Fnw = (r2 < rmaxp * rmaxp).astype(np.float64)
    for _ in range(iterations):
        conv = np.fft.irfftn(Fw * Fnw, s=(P, P, P), axes=(0, 1, 2))  # normalised 1/P^3
        conv *= blob
        convft = np.fft.rfftn(conv, axes=(0, 1, 2))
        Fnw = np.minimum(1e20, Fnw / np.maximum(1e-4, convft.real))
    data = _decenter(np.asarray(dataft, np.complex128), P, old)
    if iterations == 0:
        data = data / np.maximum(np.abs(Fw), 1e-4)
    else:
        data = data * Fnw
    sign = 1 - 2 * ((zs[:, None, None] + zs[None, :, None] + x[None, None, :]) & 1)
    data = data * sign
    vol = np.fft.irfftn(data, s=(P, P, P), axes=(0, 1, 2)) * (P ** 3)  # unnormalised C2R
    off = P // 2 - ori // 2
    vol = vol[off:off + ori, off:off + ori, off:off + ori].copy()
    c = np.arange(ori) - ori // 2
    rr = np.sqrt(c[:, None, None] ** 2 + c[None, :, None] ** 2 + c[None, None, :] ** 2) / P
    s = np.where(np.abs(rr) <= 1e-4, 1.0, np.sinc(rr))  # np.sinc(x) = sin(pi x)/(pi x)
    vol = np.where(rr > 0, vol / (s * s), vol)
    vol = vol / (pad ** 3 * ori)
    if return_weights:
        return vol, Fnw
    return vol


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def num_threads() -> int:
    return lib().orc_num_threads()
