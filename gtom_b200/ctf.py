"""CTF simulation and particle preprocessing (mirror of gtom's
d_CTFSimulate, include/CTF.cuh:317, and the step before d_rlnBackproject),
over the C ABI of gtom_b200/csrc/ctf.cu."""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .relion import _dev_ptr, _stream

FIELDS = ("pixelsize", "pixeldelta", "pixelangle", "Cs", "voltage", "defocus", "astigmatismangle",
          "defocusdelta", "amplitude", "Bfactor", "Bfactordelta", "Bfactorangle", "scale", "phaseshift")
# gtom::CTFParams() defaults (include/CTF.cuh:28-42): metres, volts, radians
DEFAULTS = dict(pixelsize=1e-10, pixeldelta=0.0, pixelangle=0.0, Cs=2e-3, voltage=300e3, defocus=-3e-6,
                astigmatismangle=0.0, defocusdelta=0.0, amplitude=0.07, Bfactor=0.0, Bfactordelta=0.0,
                Bfactorangle=0.0, scale=1.0, phaseshift=0.0)


class CTFParams(C.Structure):
    _fields_ = [(f, C.c_float) for f in FIELDS]


def ctf_params(items) -> "C.Array":
    """A CTFParams array from dicts (missing fields take gtom's defaults) or
    from a (batch, 14) array in field order."""
    if isinstance(items, np.ndarray):
        rows = [dict(zip(FIELDS, r)) for r in np.asarray(items, np.float32).reshape(-1, 14)]
    else:
        rows = [{**DEFAULTS, **d} for d in items]
    arr = (CTFParams * len(rows))()
    for i, r in enumerate(rows):
        for f in FIELDS:
            setattr(arr[i], f, float(r[f]))
    return arr


def d_CTFSimulate(h_params, d_addresses: torch.Tensor, d_gammacorrection, d_output: torch.Tensor, n: int,
                  amplitudesquared: bool = False, ignorefirstpeak: bool = False, batch: int = 1,
                  stream=None) -> None:
    """CTF values at n points (d_addresses: n float2 = (frequency in 1/pixel,
    azimuth)) for `batch` parameter sets into d_output (batch x n)."""
    arr = h_params if isinstance(h_params, C.Array) else ctf_params(h_params)
    if len(arr) < batch:
        raise ValueError(f"{len(arr)} CTF parameter sets for a batch of {batch}")
    _lib.call("gtomrln_ctf_simulate", C.cast(arr, C.c_void_p),
              _dev_ptr(d_addresses, "d_addresses", torch.float32, 2 * n),
              _dev_ptr(d_gammacorrection, "d_gammacorrection", torch.float32, n, optional=True),
              _dev_ptr(d_output, "d_output", torch.float32, n * batch), int(n), int(bool(amplitudesquared)),
              int(bool(ignorefirstpeak)), int(batch), _stream(stream))


def preprocess_particles(images: torch.Tensor, params=None, weights: bool = True, stream=None):
    """CTF * FT and CTF^2 (half-complex, flat per particle) of centred real
    particles (batch, n, n) float32 on the GPU; params: CTF parameter sets
    (dicts or a (batch, 14) array) or None for no CTF."""
    b, n = images.shape[0], images.shape[-1]
    e = (n // 2 + 1) * n
    projft = torch.empty(b * e, dtype=torch.complex64, device=images.device)
    projw = torch.empty(b * e, dtype=torch.float32, device=images.device) if weights else None
    arr = None if params is None else (params if isinstance(params, C.Array) else ctf_params(params))
    _lib.call("gtomrln_preprocess_particles", _dev_ptr(images, "images", torch.float32, b * n * n),
              int(n), int(b), None if arr is None else C.cast(arr, C.c_void_p),
              _dev_ptr(projft, "projft", torch.complex64, b * e),
              _dev_ptr(projw, "projweights", torch.float32, b * e, optional=True), _stream(stream))
    return projft, projw
