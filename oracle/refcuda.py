"""ctypes binding of the reference's own CUDA implementation.

TEST INFRASTRUCTURE ONLY: oracle/_ref/libgtomref.so is compiled from the
reference sources by `make -C oracle ref REF=<reference tree>` (through the
wrappers of oracle/ref_harness.cu, each calling one reference overload
unchanged).  It is used by tests/golden/make_golden.py (fixtures), by the
GPU parity tests that run the reference beside the library on the same
inputs, and by bench.py's reference arm.  The product library (gtom_b200/)
never loads it.

Buffers handed to the reference projector need 64 spare elements past the
volume: its x1 = P/2+1 read (src/Relion/Project.cu:155) can touch one
element past the end.
"""
from __future__ import annotations

import ctypes as C
import threading

from .oracle import REF_PATH

_p, _i, _f, _d = C.c_void_p, C.c_int, C.c_float, C.c_double

SIGNATURES = {
    "ref_matrices": [_p, _f, _i, _p],
    "ref_project": [_p, _i, _p, _i, _i, _i, _p, _i],
    "ref_project_angles": [_p, _i, _p, _i, _i, _p, _f, _i],
    "ref_backproject": [_p, _p, _i, _p, _p, _i, _i, _i, _p, _p, _f, _f, _f, _f, _f, _i, _i, _i],
    "ref_backproject_angles": [_p, _p, _i, _p, _p, _i, _i, _i, _p, _p, _f, _f, _f, _f, _f, _f, _i, _i, _i],
    "ref_reconstruct_gridding": [_p, _p, _p, _i, _i, _i, _i, _d, _i, _d],
    "ref_project_shifted": [_p, _i, _p, _i, _i, _i, _p, _p, _p, _i],
    "ref_backproject_shifted": [_p, _p, _i, _p, _p, _i, _i, _i, _p, _p, _p, _i],
    "ref_ctf_simulate": [_p, _p, _p, _p, _i, _i, _i, _i],
    "ref_convert_weights_dense": [_p, _i, _i, _i, _i, _p, _p, _p],
    "ref_backproject_tomo": [_p, _i, _p, _p, _i, _i, _p, _i],
    "ref_convert_weights_sparse": [_p, _p, _p, _i, _i, _i, _p, _p, _p],
    "ref_diff_remap_dense": [_p, _p, _p, _i, _i, _i, _i, _i, _i, _i, _p, _p, _i],
    "ref_diff_remap_sparse": [_p, _p, _p, _p, _p, _i, _i, _i, _i, _p, _p, _i],
    "ref_create_minvsigma2s": [_p, _p, _i, _p, _f],
    "ref_store_weights_add": [_p, _p, _p, _p, _p, _i, _i, _p, _f, _f, _p, _p, _p, _p, _p, _p, _p, _i],
}

_lock = threading.Lock()
_ref = None


def available() -> bool:
    return REF_PATH.exists()


def lib() -> C.CDLL:
    """Loads oracle/_ref/libgtomref.so (raises FileNotFoundError if it was
    not built)."""
    global _ref
    with _lock:
        if _ref is None:
            if not REF_PATH.exists():
                raise FileNotFoundError(f"{REF_PATH} is not built (make -C oracle ref REF=<reference tree>)")
            L = C.CDLL(str(REF_PATH))
            for name, args in SIGNATURES.items():
                getattr(L, name).argtypes = args
            _ref = L
    return _ref


def check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"{what}: CUDA error {rc}")


def matrices(angles, supersample: float):
    """The reference's own host matrices for (batch, 3) float32 Euler angles
    (radians): (batch, 9) float32, glm column-major."""
    import numpy as np
    a = np.ascontiguousarray(angles, np.float32)
    out = np.empty((a.shape[0], 9), np.float32)
    check(lib().ref_matrices(a.ctypes.data, float(supersample), a.shape[0], out.ctypes.data), "ref_matrices")
    return out
