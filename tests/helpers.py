"""Small numeric helpers for the parity tests."""
from __future__ import annotations

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def rel_l2(a, b) -> float:
    """||a - b|| / ||b|| in float64."""
    a = np.asarray(a, np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(b) else np.float64)
    b = np.asarray(b, a.dtype)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))


def load_golden(name: str):
    return np.load(GOLDEN / f"{name}.npz")


def fsc(a: np.ndarray, b: np.ndarray, nshells: int | None = None) -> np.ndarray:
    """Fourier shell correlation of two real cubes, one value per integer shell
    up to Nyquist."""
    n = a.shape[0]
    # float64 throughout: the shell sums of |F|^2 of large maps overflow float32
    fa, fb = np.fft.rfftn(np.asarray(a, np.float64)), np.fft.rfftn(np.asarray(b, np.float64))
    k = np.fft.fftfreq(n) * n
    kx = np.arange(n // 2 + 1)
    r = np.sqrt(k[:, None, None] ** 2 + k[None, :, None] ** 2 + kx[None, None, :] ** 2)
    shell = np.rint(r).astype(int)
    nsh = nshells or n // 2
    out = np.zeros(nsh)
    for s in range(1, nsh + 1):
        m = shell == s
        num = np.real(np.sum(fa[m] * np.conj(fb[m])))
        den = np.sqrt(np.sum(np.abs(fa[m]) ** 2) * np.sum(np.abs(fb[m]) ** 2))
        out[s - 1] = num / den if den > 0 else 1.0
    return out
