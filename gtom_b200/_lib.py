"""ctypes binding of libgtomrln.so (the C ABI declared in include/gtomrln.h).

The library is loaded from gtom_b200/lib/ only.  There is no fallback: if
the shared library is missing, importing a compute entry point raises
GtomLibraryMissing, so a GPU run can never silently execute anything but
the CUDA kernels.
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libgtomrln.so"

GTOMRLN_OK = 0
GTOMRLN_ERR_INVALID = -1
GTOMRLN_ERR_CUDA = -2
GTOMRLN_ERR_CUFFT = -3
GTOMRLN_ERR_ALLOC = -4


class GtomLibraryMissing(RuntimeError):
    pass


class GtomError(RuntimeError):
    """A gtomrln entry point returned a non-zero status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"gtomrln status {status}: {message}")
        self.status = status


_f = C.c_float
_d = C.c_double
_i = C.c_int
_u = C.c_uint
_p = C.c_void_p
_ull = C.c_ulonglong
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)

# name -> argtypes (restype is int unless listed in _RESTYPES)
SIGNATURES: dict[str, list] = {
    "gtomrln_version": [],
    "gtomrln_last_error": [],
    "gtomrln_release_caches": [],
    "gtomrln_set_path": [_i, _i],
    "gtomrln_set_brick_tuning": [_i, _i, _i, _i],
    "gtomrln_matrices_from_angles": [_p, _f, _u, _p],
    "gtomrln_project": [_p, _i, _i, _i, _p, _i, _i, _i, _u, _p, _u, _p],
    "gtomrln_project_angles": [_p, _i, _i, _i, _p, _i, _i, _i, _p, _f, _u, _p],
    "gtomrln_project_angles_noalloc": [_p, _i, _i, _i, _p, _i, _i, _i, _p, _f, _u, _p],
    "gtomrln_project_tex": [_ull, _ull, _i, _i, _i, _p, _i, _i, _i, _u, _p, _u, _p],
    "gtomrln_project_tex_angles": [_ull, _ull, _i, _i, _i, _p, _i, _i, _i, _p, _f, _u, _p],
    "gtomrln_backproject": [_p, _p, _i, _i, _i, _p, _p, _i, _i, _i, _u, _p, _p,
                            _f, _f, _f, _f, _f, _i, _i, _u, _p],
    "gtomrln_backproject_angles": [_p, _p, _i, _i, _i, _p, _p, _i, _i, _i, _u, _p, _p,
                                   _f, _f, _f, _f, _f, _f, _i, _i, _u, _p],
    "gtomrln_backproject_tomo": [_p, _i, _i, _i, _p, _p, _i, _i, _i, _u, _p, _u, _p],
    "gtomrln_backproject_tomo_angles": [_p, _i, _i, _i, _p, _p, _i, _i, _i, _u, _p, _u, _p],
    "gtomrln_project_shifted": [_p, _i, _i, _i, _p, _i, _i, _i, _u, _p, _p, _p, _u, _p],
    "gtomrln_project_shifted_angles": [_p, _i, _i, _i, _p, _i, _i, _i, _p, _p, _p, _f, _u, _p],
    "gtomrln_project_shifted_tex": [_ull, _ull, _i, _i, _i, _p, _i, _i, _i, _u, _p, _p, _p, _u, _p],
    "gtomrln_project_shifted_tex_angles": [_ull, _ull, _i, _i, _i, _p, _i, _i, _i, _p, _p, _p, _f, _u,
                                           _p],
    "gtomrln_backproject_shifted": [_p, _p, _i, _i, _i, _p, _p, _i, _i, _i, _u, _p, _p, _p, _u, _p],
    "gtomrln_backproject_shifted_angles": [_p, _p, _i, _i, _i, _p, _p, _i, _i, _i, _u, _p, _p, _p, _f,
                                           _u, _p],
    "gtomrln_reconstruct_gridding": [_p, _p, _p, _i, _i, _i, _i, _i, _i, _i, _i, _i, _i,
                                     _d, _i, _d, _p],
    "gtomrln_reconstruct_gridding_tol": [_p, _p, _p, _i, _i, _i, _i, _i, _i, _i, _i, _d,
                                         _d, _i, _d, _ip, _dp, _p],
    "gtomrln_reconstruct_gridding_warm": [_p, _p, _p, _i, _i, _i, _i, _i, _i, _i, _i, _d, _f, _p,
                                          _f, _d, _i, _d, _ip, _dp, _ip, _p],
    "gtomrln_gridding_weights": [_p, _i, _i, _i, _i, _i, _i, _d, _f, _p, _f, _d, _i, _d, _p, _p,
                                 _ip, _dp, _ip, _p, _d, _dp, _p],
    "gtomrln_kaiser_bessel_table": [_d, _d, _i, _i, _p],
    "gtomrln_ctf_simulate": [_p, _p, _p, _p, _u, _i, _i, _i, _p],
    "gtomrln_preprocess_particles": [_p, _i, _u, _p, _p, _p, _p],
    "gtomrln_squared_differences_sparse": [_p, _p, _p, _i, _i, _i, _p, _p, _p, _p, _u, _u, _i, _p],
    "gtomrln_squared_differences": [_p, _p, _p, _i, _i, _i, _u, _p, _u, _p, _u, _u, _p, _i, _p],
    "gtomrln_convert_weights_dense": [_p, _u, _u, _u, _u, _p, _p, _p, _p],
    "gtomrln_convert_weights_sparse": [_p, _p, _p, _u, _u, _u, _p, _p, _p, _p],
    "gtomrln_convert_weights_sort": [_p, _u, _p],
    "gtomrln_convert_weights_compact": [_p, _p, C.POINTER(C.c_uint), _p],
    "gtomrln_diff_remap_dense": [_p, _p, _p, _u, _u, _u, _u, _u, _u, _u, _p, _p, _i, _p],
    "gtomrln_diff_remap_sparse": [_p, _p, _p, _p, _p, _u, _u, _u, _u, _p, _p, _i, _p],
    "gtomrln_create_minvsigma2s": [_p, _p, _u, _p, _f, _p],
    "gtomrln_store_weights_add": [_p, _p, _p, _p, _p, _u, _u, _p, _f, _f, _p, _p, _p, _p, _p, _p, _p, _i, _p],
    "gtomrln_batch_create": [_p, _i, _i, _i, _p],
    "gtomrln_batch_set_tuning": [_p, _i, _i, _i],
    "gtomrln_batch_run": [_p, _i, _p],
    "gtomrln_batch_destroy": [_p],
    "gtomrln_mlp_param_count": [],
    "gtomrln_mlp_forward": [_p, _p, _i, _p, _p],
    "gtomrln_mlp_volume_features": [_p, _i, _p, _p, _i, _p, _p],
    "gtomrln_mlp_gradients": [_p, _p, _p, _p, _i, _f, _p, _p, _p],
    "gtomrln_mlp_train_batch": [_p, _p, _p, _p, _p, _i, _p, _i, _f, _p, _p, _p],
    "gtomrln_mlp_adam": [_p, _p, _p, _p, _i, _f, _f, _f, _f, _p],
}
_RESTYPES = {"gtomrln_last_error": C.c_char_p}

_lock = threading.Lock()
_lib: C.CDLL | None = None


def load() -> C.CDLL:
    """Loads libgtomrln.so once and declares every entry point's signature."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise GtomLibraryMissing(
                f"{LIB_PATH} is not built; run `python -m gtom_b200.build` "
                "(the CUDA library is the only implementation)")
        lib = C.CDLL(str(LIB_PATH))
        for name, args in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = _RESTYPES.get(name, C.c_int)
        _lib = lib
        return lib


def check(status: int) -> None:
    if status != GTOMRLN_OK:
        msg = load().gtomrln_last_error()
        raise GtomError(status, msg.decode() if msg else "")


def call(name: str, *args) -> None:
    """Calls an entry point and raises GtomError on a non-zero status."""
    check(getattr(load(), name)(*args))
