"""Python mirror of gtom's RELION projector / backprojector / gridding API.

The functions keep the reference's names, argument order and meaning
(include/Relion.cuh:9-10,34-37 and include/Reconstruction.cuh:16 of
dtegunov/gtom); C++ overloads become one function that dispatches on the
kind of its arguments.  Device buffers are CUDA torch tensors (complex64 for
``tcomplex*``, float32 for ``tfloat*``), host arrays are numpy arrays, dims
are 3-tuples (x, y, z).  Every call goes through the C ABI of
libgtomrln.so (gtom_b200/_lib.py) on torch's current stream; a non-zero
status raises GtomError where the reference would throw.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np
import torch

from . import _lib

Dims = Sequence[int]


def elements_fft(dims: Dims) -> int:
    """ElementsFFT (include/Prerequisites.cuh:224): (x/2+1) * y * z."""
    return (dims[0] // 2 + 1) * dims[1] * max(dims[2], 1)


def _stream(stream) -> C.c_void_p:
    if stream is None:
        stream = torch.cuda.current_stream()
    if isinstance(stream, torch.cuda.Stream):
        return C.c_void_p(stream.cuda_stream)
    return C.c_void_p(int(stream))


def _dev_ptr(t, name: str, dtype: torch.dtype | None = None, min_numel: int = 0,
             optional: bool = False) -> C.c_void_p:
    if t is None:
        if optional:
            return C.c_void_p(0)
        raise ValueError(f"{name} must be a CUDA tensor")
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if dtype is not None and t.dtype != dtype:
        raise ValueError(f"{name} must be {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if t.numel() < min_numel:
        raise ValueError(f"{name} holds {t.numel()} elements, needs {min_numel}")
    return C.c_void_p(t.data_ptr())


def _host_f32(a, name: str, min_numel: int) -> np.ndarray:
    arr = np.ascontiguousarray(np.asarray(a if not isinstance(a, torch.Tensor) else a.cpu().numpy(),
                                          dtype=np.float32))
    if arr.size < min_numel:
        raise ValueError(f"{name} holds {arr.size} values, needs {min_numel}")
    return arr


def _is_host(a) -> bool:
    return isinstance(a, (np.ndarray, list, tuple)) or (isinstance(a, torch.Tensor) and not a.is_cuda)


def matrices_from_angles(h_angles, supersample: float = 1.0) -> np.ndarray:
    """transpose(Matrix3Euler(angles)) * supersample per slice, (batch, 9)
    column-major float32 (src/Relion/Project.cu:14-16)."""
    ang = _host_f32(h_angles, "h_angles", 0).reshape(-1, 3)
    out = np.empty((ang.shape[0], 9), np.float32)
    _lib.call("gtomrln_matrices_from_angles", ang.ctypes.data, C.c_float(supersample),
              ang.shape[0], out.ctypes.data)
    return out


def d_rlnProject(volumeft, dimsvolume: Dims, proj: torch.Tensor, dimsproj: Dims, *args,
                 stream=None) -> None:
    """Central-slice gather (include/Relion.cuh:34-37).

    Overloads, after ``(volumeft, dimsvolume, d_proj, dimsproj)``:
      ``(h_angles, supersample, batch)``  — Project.cu:12-23
      ``(rmax, d_matrices, batch)``       — Project.cu:25-43
    ``volumeft`` is a complex64 CUDA tensor of the decentred half volume, or
    a ``(t_volumeRe, t_volumeIm)`` pair of texture object handles
    (Project.cu:45-87).
    """
    if len(args) != 3:
        raise TypeError("d_rlnProject expects (h_angles, supersample, batch) or "
                        "(rmax, d_matrices, batch) after dimsproj")
    vx, vy, vz = (int(v) for v in dimsvolume)
    px, py, pz = (int(v) for v in dimsproj)
    batch = int(args[2])
    e = elements_fft((px, py, pz))
    pp = _dev_ptr(proj, "d_proj", torch.complex64, e * batch)
    tex = isinstance(volumeft, tuple)
    if not tex:
        vp = _dev_ptr(volumeft, "d_volumeft", torch.complex64, elements_fft((vx, vy, vz)))
    s = _stream(stream)
    if _is_host(args[0]):
        ang = _host_f32(args[0], "h_angles", 3 * batch)
        if tex:
            _lib.call("gtomrln_project_tex_angles", int(volumeft[0]), int(volumeft[1]), vx, vy, vz,
                      pp, px, py, pz, ang.ctypes.data, C.c_float(args[1]), batch, s)
        else:
            _lib.call("gtomrln_project_angles", vp, vx, vy, vz, pp, px, py, pz, ang.ctypes.data,
                      C.c_float(args[1]), batch, s)
    else:
        rmax = int(args[0])
        mp = _dev_ptr(args[1], "d_matrices", torch.float32, 9 * batch)
        if tex:
            _lib.call("gtomrln_project_tex", int(volumeft[0]), int(volumeft[1]), vx, vy, vz, pp, px,
                      py, pz, rmax, mp, batch, s)
        else:
            _lib.call("gtomrln_project", vp, vx, vy, vz, pp, px, py, pz, rmax, mp, batch, s)


def d_rlnProjectShifted(volumeft, dimsvolume: Dims, proj: torch.Tensor, dimsproj: Dims, *args,
                        stream=None) -> None:
    """Central-slice gather times a per-slice phase shift and global weight
    (include/Relion.cuh:40-43).

    Overloads, after ``(volumeft, dimsvolume, d_proj, dimsproj)``:
      ``(h_angles, h_shifts, h_globalweights, supersample, batch)`` — ProjectShifted.cu:32-56
      ``(rmax, d_matrices, d_shifts, d_globalweights, batch)``     — ProjectShifted.cu:58-75
    h_shifts are in pixels; d_shifts already scaled by 2 pi / dimsproj.x.
    ``volumeft`` may be a ``(t_volumeRe, t_volumeIm)`` texture pair
    (ProjectShifted.cu:78-122).
    """
    if len(args) != 5:
        raise TypeError("d_rlnProjectShifted expects (h_angles, h_shifts, h_globalweights, supersample, "
                        "batch) or (rmax, d_matrices, d_shifts, d_globalweights, batch)")
    vx, vy, vz = (int(v) for v in dimsvolume)
    px, py, pz = (int(v) for v in dimsproj)
    batch = int(args[4])
    pp = _dev_ptr(proj, "d_proj", torch.complex64, elements_fft((px, py, pz)) * batch)
    tex = isinstance(volumeft, tuple)
    vol = (int(volumeft[0]), int(volumeft[1])) if tex else \
        (_dev_ptr(volumeft, "d_volumeft", torch.complex64, elements_fft((vx, vy, vz))),)
    s = _stream(stream)
    if _is_host(args[0]):
        ang = _host_f32(args[0], "h_angles", 3 * batch)
        sh = _host_f32(args[1], "h_shifts", 3 * batch)
        gw = _host_f32(args[2], "h_globalweights", batch)
        _lib.call("gtomrln_project_shifted_tex_angles" if tex else "gtomrln_project_shifted_angles",
                  *vol, vx, vy, vz, pp, px, py, pz, ang.ctypes.data, sh.ctypes.data, gw.ctypes.data,
                  C.c_float(args[3]), batch, s)
    else:
        mp = _dev_ptr(args[1], "d_matrices", torch.float32, 9 * batch)
        sp = _dev_ptr(args[2], "d_shifts", torch.float32, 3 * batch)
        wp = _dev_ptr(args[3], "d_globalweights", torch.float32, batch)
        _lib.call("gtomrln_project_shifted_tex" if tex else "gtomrln_project_shifted", *vol, vx, vy, vz,
                  pp, px, py, pz, int(args[0]), mp, sp, wp, batch, s)


def d_rlnBackprojectShifted(volumeft, volumeweights, dimsvolume: Dims, projft, projweights,
                            dimsproj: Dims, rmax: int, *args, stream=None) -> None:
    """Shifted, globally weighted insertion (include/Relion.cuh:17-18), into
    centred accumulators.

    Overloads, after ``(..., dimsproj, rmax)``:
      ``(h_angles, h_shifts, h_globalweights, supersample, batch)`` — BackprojectShifted.cu:11-35
      ``(d_matrices, d_shifts, d_globalweights, batch)``            — BackprojectShifted.cu:37-58
    """
    vx, vy, vz = (int(v) for v in dimsvolume)
    px, py, pz = (int(v) for v in dimsproj)
    nvol = elements_fft((vx, vy, vz))
    s = _stream(stream)
    if len(args) == 5:
        batch = int(args[4])
    elif len(args) == 4:
        batch = int(args[3])
    else:
        raise TypeError("d_rlnBackprojectShifted expects (h_angles, h_shifts, h_globalweights, "
                        "supersample, batch) or (d_matrices, d_shifts, d_globalweights, batch)")
    e = elements_fft((px, py, pz)) * batch
    common = (_dev_ptr(volumeft, "d_volumeft", torch.complex64, nvol, optional=True),
              _dev_ptr(volumeweights, "d_volumeweights", torch.float32, nvol, optional=True),
              vx, vy, vz, _dev_ptr(projft, "d_projft", torch.complex64, e, optional=True),
              _dev_ptr(projweights, "d_projweights", torch.float32, e, optional=True),
              px, py, pz, int(rmax))
    if len(args) == 5:
        ang = _host_f32(args[0], "h_angles", 3 * batch)
        sh = _host_f32(args[1], "h_shifts", 3 * batch)
        gw = _host_f32(args[2], "h_globalweights", batch)
        _lib.call("gtomrln_backproject_shifted_angles", *common, ang.ctypes.data, sh.ctypes.data,
                  gw.ctypes.data, C.c_float(args[3]), batch, s)
    else:
        _lib.call("gtomrln_backproject_shifted", *common,
                  _dev_ptr(args[0], "d_matrices", torch.float32, 9 * batch),
                  _dev_ptr(args[1], "d_shifts", torch.float32, 3 * batch),
                  _dev_ptr(args[2], "d_globalweights", torch.float32, batch), batch, s)


def d_BackprojectTomo(volumeft, dimsvolume: Dims, projft, projweights, dimsproj: Dims, rmax: int, angles_or_matrices,
                      batch: int, stream=None) -> None:
    """Lanczos-5 gather insertion for tomograms (include/Relion.cuh:13-14):
    host Euler angles (BackprojectTomo.cu:11-28) or device matrices
    (:30-46)."""
    vx, vy, vz = (int(v) for v in dimsvolume)
    px, py, pz = (int(v) for v in dimsproj)
    batch = int(batch)
    e = elements_fft((px, py, pz)) * batch
    common = (_dev_ptr(volumeft, "d_volumeft", torch.complex64, elements_fft((vx, vy, vz))), vx, vy, vz,
              _dev_ptr(projft, "d_projft", torch.complex64, e), _dev_ptr(projweights, "d_projweights", torch.float32, e),
              px, py, pz, int(rmax))
    if _is_host(angles_or_matrices):
        ang = _host_f32(angles_or_matrices, "h_angles", 3 * batch)
        _lib.call("gtomrln_backproject_tomo_angles", *common, ang.ctypes.data, batch, _stream(stream))
    else:
        _lib.call("gtomrln_backproject_tomo", *common,
                  _dev_ptr(angles_or_matrices, "d_matrices", torch.float32, 9 * batch), batch, _stream(stream))


def d_rlnBackproject(volumeft, volumeweights, dimsvolume: Dims, projft, projweights,
                     dimsproj: Dims, rmax: int, *args, stream=None) -> None:
    """Trilinear scatter-insert, accumulating in place (include/Relion.cuh:9-10).

    Overloads, after ``(..., dimsproj, rmax)``:
      ``(d_matrices, d_ivolume, magnification, ewaldradiussuper,
         outputdecentered, squareinterpweights, batch)``     — Backproject.cu:48-124
      ``(h_angles, h_ivolume, magnification, ewaldradius, supersample,
         outputdecentered, squareinterpweights, batch)``     — Backproject.cu:23-46
    ``magnification`` is the float4 (x, y, z, w) of the 2x2 matrix columns.
    """
    vx, vy, vz = (int(v) for v in dimsvolume)
    px, py, pz = (int(v) for v in dimsproj)
    nvol = elements_fft((vx, vy, vz))
    s = _stream(stream)
    if len(args) == 7:
        mats, ivol, mag, ewald, dec, sq, batch = args
        batch = int(batch)
        e = elements_fft((px, py, pz))
        _lib.call("gtomrln_backproject",
                  _dev_ptr(volumeft, "d_volumeft", torch.complex64, nvol, optional=True),
                  _dev_ptr(volumeweights, "d_volumeweights", torch.float32, nvol, optional=True),
                  vx, vy, vz,
                  _dev_ptr(projft, "d_projft", torch.complex64, e * batch, optional=True),
                  _dev_ptr(projweights, "d_projweights", torch.float32, e * batch, optional=True),
                  px, py, pz, int(rmax),
                  _dev_ptr(mats, "d_matrices", torch.float32, 9 * batch),
                  _dev_ptr(ivol, "d_ivolume", torch.int32, batch, optional=True),
                  *(C.c_float(float(m)) for m in mag), C.c_float(float(ewald)), int(bool(dec)),
                  int(bool(sq)), batch, s)
    elif len(args) == 8:
        ang, ivol, mag, ewald, ss, dec, sq, batch = args
        batch = int(batch)
        e = elements_fft((px, py, pz))
        ang = _host_f32(ang, "h_angles", 3 * batch)
        iv = None
        if ivol is not None:
            iv = np.ascontiguousarray(np.asarray(ivol, dtype=np.int32))
            if iv.size < batch:
                raise ValueError("h_ivolume shorter than batch")
        _lib.call("gtomrln_backproject_angles",
                  _dev_ptr(volumeft, "d_volumeft", torch.complex64, nvol, optional=True),
                  _dev_ptr(volumeweights, "d_volumeweights", torch.float32, nvol, optional=True),
                  vx, vy, vz,
                  _dev_ptr(projft, "d_projft", torch.complex64, e * batch, optional=True),
                  _dev_ptr(projweights, "d_projweights", torch.float32, e * batch, optional=True),
                  px, py, pz, int(rmax), ang.ctypes.data,
                  C.c_void_p(iv.ctypes.data if iv is not None else 0),
                  *(C.c_float(float(m)) for m in mag), C.c_float(float(ewald)),
                  C.c_float(float(ss)), int(bool(dec)), int(bool(sq)), batch, s)
    else:
        raise TypeError("d_rlnBackproject: unexpected number of arguments")


def d_ReconstructGridding(dataft, weight, reconstructed, dimsori: Dims, dimspadded: Dims,
                          paddingfactor: int = 2, pre_planforw: int = 0, pre_planback: int = 0,
                          iterations: int = 10, blobradius: float = 1.9, bloborder: int = 0,
                          blobalpha: float = 15.0, stream=None) -> None:
    """Gridding-corrected reconstruction (include/Reconstruction.cuh:16)."""
    ox, oy, oz = (int(v) for v in dimsori)
    qx, qy, qz = (int(v) for v in dimspadded)
    npad = elements_fft((qx, qy, qz))
    _lib.call("gtomrln_reconstruct_gridding",
              _dev_ptr(dataft, "d_dataft", torch.complex64, npad),
              _dev_ptr(weight, "d_weight", torch.float32, npad),
              _dev_ptr(reconstructed, "d_reconstructed", torch.float32, ox * oy * oz),
              ox, oy, oz, qx, qy, qz, int(paddingfactor), int(pre_planforw or 0),
              int(pre_planback or 0), int(iterations), float(blobradius), int(bloborder),
              float(blobalpha), _stream(stream))


def reconstruct_gridding_tol(dataft, weight, reconstructed, dimsori: Dims, dimspadded: Dims,
                             paddingfactor: int = 2, max_iterations: int = 100,
                             tolerance: float = 1e-4, blobradius: float = 1.9,
                             bloborder: int = 0, blobalpha: float = 15.0,
                             stream=None) -> tuple[int, float]:
    """d_ReconstructGridding with a convergence test on the relative change of
    the gridding weights; returns (iterations run, last relative change)."""
    ox, oy, oz = (int(v) for v in dimsori)
    qx, qy, qz = (int(v) for v in dimspadded)
    npad = elements_fft((qx, qy, qz))
    it = C.c_int(0)
    ch = C.c_double(0)
    _lib.call("gtomrln_reconstruct_gridding_tol",
              _dev_ptr(dataft, "d_dataft", torch.complex64, npad),
              _dev_ptr(weight, "d_weight", torch.float32, npad),
              _dev_ptr(reconstructed, "d_reconstructed", torch.float32, ox * oy * oz),
              ox, oy, oz, qx, qy, qz, int(paddingfactor), int(max_iterations), float(tolerance),
              float(blobradius), int(bloborder), float(blobalpha), C.byref(it), C.byref(ch),
              _stream(stream))
    return it.value, ch.value


def reconstruct_gridding_warm(dataft, weight, reconstructed, dimsori: Dims, dimspadded: Dims,
                              mlp_params=None, paddingfactor: int = 2, max_iterations: int = 1000,
                              tolerance: float = 1e-4, momentum: float = 0.0,
                              residual_limit: float = 0.5, blobradius: float = 1.9,
                              bloborder: int = 0, blobalpha: float = 15.0,
                              stream=None) -> tuple[int, float, bool]:
    """Gridding reconstruction from the MLP's predicted start (mlp_params, a
    CUDA float32 tensor of mlp_param_count() values; None for the
    sphere-mask start) and/or with momentum (gtomrln_reconstruct_gridding_warm).
    Returns (iterations run, last relative change, predicted start kept)."""
    ox, oy, oz = (int(v) for v in dimsori)
    qx, qy, qz = (int(v) for v in dimspadded)
    npad = elements_fft((qx, qy, qz))
    it, ch, used = C.c_int(0), C.c_double(0), C.c_int(0)
    _lib.call("gtomrln_reconstruct_gridding_warm",
              _dev_ptr(dataft, "d_dataft", torch.complex64, npad),
              _dev_ptr(weight, "d_weight", torch.float32, npad),
              _dev_ptr(reconstructed, "d_reconstructed", torch.float32, ox * oy * oz),
              ox, oy, oz, qx, qy, qz, int(paddingfactor), int(max_iterations), float(tolerance),
              C.c_float(float(momentum)),
              _dev_ptr(mlp_params, "d_mlp_params", torch.float32, mlp_param_count(), optional=True),
              C.c_float(float(residual_limit)), float(blobradius), int(bloborder), float(blobalpha),
              C.byref(it), C.byref(ch), C.byref(used), _stream(stream))
    return it.value, ch.value, bool(used.value)


def gridding_weights(weight, dimspadded: Dims, ori: int, paddingfactor: int = 2,
                     max_iterations: int = 1000, tolerance: float = 1e-4, momentum: float = 0.0,
                     mlp_params=None, residual_limit: float = 0.5, blobradius: float = 1.9,
                     bloborder: int = 0, blobalpha: float = 15.0, fw_out=None, fnw_out=None,
                     stream=None, ref_fnw=None, ref_tolerance: float = 0.0, return_distance: bool = False):
    """The gridding weights only (gtomrln_gridding_weights).  Returns
    (Fnewweight, Fweight, iterations, last change, predicted start kept);
    the weights are flat float32 CUDA tensors on the decentred
    (P/2+1) x P x P grid, P = ori * paddingfactor.  With ref_fnw (weights on
    that grid) the loop also stops once ||Fw (Fnw - ref)|| / ||Fw ref|| <=
    ref_tolerance; return_distance appends the last such distance."""
    qx, qy, qz = (int(v) for v in dimspadded)
    P = int(ori) * int(paddingfactor)
    nc = (P // 2 + 1) * P * P
    dev = weight.device
    fnw = fnw_out if fnw_out is not None else torch.empty(nc, dtype=torch.float32, device=dev)
    fw = fw_out if fw_out is not None else torch.empty(nc, dtype=torch.float32, device=dev)
    it, ch, used, dist = C.c_int(0), C.c_double(0), C.c_int(0), C.c_double(0)
    _lib.call("gtomrln_gridding_weights",
              _dev_ptr(weight, "d_weight", torch.float32, elements_fft((qx, qy, qz))),
              qx, qy, qz, int(ori), int(paddingfactor), int(max_iterations), float(tolerance),
              C.c_float(float(momentum)),
              _dev_ptr(mlp_params, "d_mlp_params", torch.float32, mlp_param_count(), optional=True),
              C.c_float(float(residual_limit)), float(blobradius), int(bloborder), float(blobalpha),
              _dev_ptr(fw, "d_fw", torch.float32, nc), _dev_ptr(fnw, "d_fnw", torch.float32, nc),
              C.byref(it), C.byref(ch), C.byref(used),
              _dev_ptr(ref_fnw, "ref_fnw", torch.float32, nc, optional=True), float(ref_tolerance),
              C.byref(dist), _stream(stream))
    if return_distance:
        return fnw, fw, it.value, ch.value, bool(used.value), dist.value
    return fnw, fw, it.value, ch.value, bool(used.value)


def mlp_param_count() -> int:
    """Floats in the warm-start MLP's parameter block."""
    return int(_lib.load().gtomrln_mlp_param_count())


_OPS = {"project": 0, "backproject": 1, "gridding": 2}
_PATHS = {"auto": 0, "direct": 1, "brick": 2, "segment": 3, "fused": 4, "segment_fp32": 5, "symmetric": 6}


def set_path(op: str, path: str) -> None:
    """Selects the implementation of "project" or "backproject" for this
    process: "auto" (default), "direct", "brick" (pixels binned per brick) or
    "segment" (pixels found per brick by row segments; the backprojector's
    accumulates each work item in fixed point first), for "backproject" also
    "segment_fp32" (row segments, FP32 atomics only); of "gridding": "auto"
    (default: "symmetric" on power-of-two grids P = 64 .. 512, cuFFT
    elsewhere), "direct" (cuFFT transforms), "fused" (two fused passes per
    iteration with the library's own transforms on power-of-two grids) or
    "symmetric" (four passes over the Hermitian half along z of the real
    iterated spectrum, the library's own transforms) (gtomrln_set_path)."""
    _lib.call("gtomrln_set_path", _OPS[op], _PATHS[path])


def set_brick_tuning(op: str, edge: int = 0, threads: int = 0, chunk: int = 0) -> None:
    """Launch shape of the brick-major kernels of "project" or "backproject"
    (gtomrln_set_brick_tuning); 0 keeps the default for a field."""
    _lib.call("gtomrln_set_brick_tuning", _OPS[op], int(edge), int(threads), int(chunk))


def kaiser_bessel_table(radius: float, alpha: float, order: int = 0,
                        nsamples: int = 10000) -> np.ndarray:
    """The normalised blob table of the gridding correction."""
    out = np.empty(nsamples, np.float32)
    _lib.call("gtomrln_kaiser_bessel_table", float(radius), float(alpha), int(order),
              int(nsamples), out.ctypes.data)
    return out
