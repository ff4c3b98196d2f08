"""Seeded synthetic inputs shared by the tests and the golden-fixture script:
uniform SO(3) orientations and Fourier transforms of Gaussian-blob volumes."""
from __future__ import annotations

import numpy as np


def random_angles(rng, batch: int) -> np.ndarray:
    """Uniform SO(3) (Shoemake quaternions) -> ZYZ Euler (rot, tilt, psi)."""
    u = rng.random((batch, 3))
    q = np.stack([np.sqrt(1 - u[:, 0]) * np.sin(2 * np.pi * u[:, 1]),
                  np.sqrt(1 - u[:, 0]) * np.cos(2 * np.pi * u[:, 1]),
                  np.sqrt(u[:, 0]) * np.sin(2 * np.pi * u[:, 2]),
                  np.sqrt(u[:, 0]) * np.cos(2 * np.pi * u[:, 2])], 1)
    w, x, y, z = q.T
    R = np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w),
                  2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
                  2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], 1).reshape(-1, 3, 3)
    tilt = np.arccos(np.clip(R[:, 2, 2], -1, 1))
    rot = np.arctan2(R[:, 2, 1], R[:, 2, 0])
    psi = np.arctan2(R[:, 1, 2], -R[:, 0, 2])
    return np.stack([rot, tilt, psi], 1).astype(np.float32)


def blob_volume_ft(rng, n: int, P: int, nblobs: int) -> np.ndarray:
    """Decentred half-complex FT (P, P, P/2+1) of n^3 Gaussian blobs padded to P."""
    c = np.arange(n) - n // 2
    vol = np.zeros((n, n, n))
    for _ in range(nblobs):
        ctr = rng.normal(size=3)
        ctr = ctr / np.linalg.norm(ctr) * rng.random() ** (1 / 3) * 0.4 * n
        s = rng.uniform(0.6, 1.6) * n / 32
        a = rng.uniform(0.2, 1.0)
        d2 = (c[:, None, None] - ctr[2]) ** 2 + (c[None, :, None] - ctr[1]) ** 2 + (c[None, None, :] - ctr[0]) ** 2
        vol += a * np.exp(-d2 / (2 * s * s))
    padded = np.zeros((P, P, P))
    o = P // 2 - n // 2
    padded[o:o + n, o:o + n, o:o + n] = vol
    return np.fft.rfftn(np.fft.ifftshift(padded)).astype(np.complex64)
