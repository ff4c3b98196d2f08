"""Test infrastructure: float64 numpy restatement of gtom's d_BackprojectTomo
(src/Relion/BackprojectTomo.cu:48-153): for every voxel of the decentred
half volume inside rmax, a Lanczos-5 weighted gather over every pixel of
every slice whose plane passes within 5 voxels.  Brute force over all
pixels, as the reference does; only tests may import it."""
from __future__ import annotations

import numpy as np


def _sinc(x):
    return np.where(np.abs(x) <= 1e-4, 1.0, np.sin(np.pi * x) / (np.pi * np.where(x == 0, 1, x)))


def backproject_tomo(volume: np.ndarray, V: int, projft, projw, n: int, rmax: int, mats) -> np.ndarray:
    """Returns a copy of `volume` ((V/2+1) V V complex) with the written voxels."""
    out = np.array(volume, np.complex128).reshape(-1)
    rmax = min(int(rmax), V // 2)
    m = np.asarray(mats, np.float64).reshape(-1, 3, 3).transpose(0, 2, 1)  # column-major -> M[r][c]
    proj = np.asarray(projft, np.complex128).reshape(len(m), -1)
    pw = np.asarray(projw, np.float64).reshape(len(m), -1)
    dimft = n // 2 + 1
    idy, idx = np.divmod(np.arange(dimft * n), dimft)
    px = idx.astype(np.float64)
    py = np.where(idy <= n // 2, idy, idy - n).astype(np.float64)
    rowlen = V // 2 + 1
    for i in range(out.size):
        x = i % rowlen
        y = (i // rowlen) % V
        z = i // (rowlen * V)
        v = np.array([x, y if y < V // 2 else y - V, z if z < V // 2 else z - V], np.float64)
        if np.sqrt(v @ v) >= rmax:
            continue
        vs = 0j
        ws = ss = 0.0
        for b in range(len(m)):
            if abs((m[b].T @ v)[2]) > 5:
                continue
            pos = m[b][:, 0][:, None] * px[None] + m[b][:, 1][:, None] * py[None]  # (3, pixels)
            neg = pos[0] < 0
            pos = np.where(neg[None], -pos, pos)
            d = v[:, None] - pos
            ok = np.all(np.abs(d) <= 5, axis=0)
            s = (_sinc(d[0]) * _sinc(d[0] / 5) * _sinc(d[1]) * _sinc(d[1] / 5) * _sinc(d[2]) * _sinc(d[2] / 5))[ok]
            val = np.where(neg, np.conj(proj[b]), proj[b])[ok]
            ss += s.sum()
            ws += (s * pw[b][ok]).sum()
            vs += (s * val).sum()
        if abs(ss) > 1e-3:
            out[i] = vs / ws * min(1.0, max(-1.0, ss))
    return out
