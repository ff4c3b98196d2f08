"""Seeded synthetic single-particle workloads, generated on the GPU.

Stand-ins for real cryo-EM data with the shapes and value distributions of
the benchmark configurations: a Gaussian-blob volume, orientations from a
von Mises-Fisher mixture plus a uniform part, a CTF per particle (the gtom
formula, include/CTF.cuh:195-223 of dtegunov/gtom), and white noise at a
given SNR.  Everything here prepares inputs; the timed work is in the CUDA
library.
"""
from __future__ import annotations

import math

import numpy as np
import torch


def blob_volume(n: int, nblobs: int, seed: int, device, radius_frac: float = 0.44,
                sigma_range=(1.5, 4.0)) -> torch.Tensor:
    """n^3 float32 volume of isotropic Gaussians with centres uniform in a
    ball of radius radius_frac * n, sigma ~ U(sigma_range) * n / 64 voxels and
    amplitude ~ U(0.2, 1)."""
    rng = np.random.default_rng(seed)
    vol = torch.zeros((n, n, n), dtype=torch.float32, device=device)
    scale = n / 64.0
    for _ in range(nblobs):
        d = rng.normal(size=3)
        c = d / np.linalg.norm(d) * rng.random() ** (1 / 3) * radius_frac * n + n / 2
        s = rng.uniform(*sigma_range) * scale
        a = rng.uniform(0.2, 1.0)
        h = int(math.ceil(4 * s))
        lo = [max(0, int(math.floor(ci)) - h) for ci in c]
        hi = [min(n, int(math.floor(ci)) + h + 1) for ci in c]
        zz = torch.arange(lo[2], hi[2], device=device, dtype=torch.float32) - float(c[2])
        yy = torch.arange(lo[1], hi[1], device=device, dtype=torch.float32) - float(c[1])
        xx = torch.arange(lo[0], hi[0], device=device, dtype=torch.float32) - float(c[0])
        g = torch.exp(-(zz[:, None, None] ** 2 + yy[None, :, None] ** 2 + xx[None, None, :] ** 2) / (2 * s * s))
        vol[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] += a * g
    return vol


def padded_half_ft(vol: torch.Tensor, pad: int = 2) -> torch.Tensor:
    """Decentred half-complex FT (P, P, P/2+1), P = pad * n, of the volume
    zero-padded about its centre: the layout d_rlnProject reads."""
    n = vol.shape[0]
    P = pad * n
    big = torch.zeros((P, P, P), dtype=torch.float32, device=vol.device)
    o = P // 2 - n // 2
    big[o:o + n, o:o + n, o:o + n] = vol
    big = torch.fft.ifftshift(big)
    ft = torch.fft.rfftn(big)
    del big
    return ft.to(torch.complex64).contiguous()


def _euler_from_view(d: np.ndarray, psi: np.ndarray) -> np.ndarray:
    """ZYZ (rot, tilt, psi) whose projection direction (third row of the
    RELION matrix A) is the unit vector d."""
    d = d / np.linalg.norm(d, axis=1, keepdims=True)
    tilt = np.arccos(np.clip(d[:, 2], -1, 1))
    rot = np.arctan2(d[:, 1], d[:, 0])
    return np.stack([rot, tilt, psi], 1).astype(np.float32)


def sample_vmf(rng, mu: np.ndarray, kappa: float, count: int) -> np.ndarray:
    """Samples from a von Mises-Fisher distribution on S^2 (Wood's method)."""
    mu = mu / np.linalg.norm(mu)
    u = rng.random(count)
    if kappa < 1e-6:
        w = 2 * u - 1
    else:
        w = 1 + np.log(u + (1 - u) * np.exp(-2 * kappa)) / kappa
    th = rng.uniform(0, 2 * np.pi, count)
    a = np.array([1.0, 0, 0]) if abs(mu[0]) < 0.9 else np.array([0, 1.0, 0])
    v1 = np.cross(mu, a)
    v1 /= np.linalg.norm(v1)
    v2 = np.cross(mu, v1)
    s = np.sqrt(np.clip(1 - w * w, 0, None))
    return w[:, None] * mu + s[:, None] * (np.cos(th)[:, None] * v1 + np.sin(th)[:, None] * v2)


def vmf_mixture_angles(rng, count: int, lobes: int = 3, kappa_range=(5.0, 40.0),
                       uniform_frac: float = 0.3) -> np.ndarray:
    """Euler angles (count, 3) float32 radians: `lobes` vMF preferred views with
    kappa ~ U(kappa_range), a uniform_frac isotropic part, psi uniform."""
    nu = int(round(uniform_frac * count))
    dirs = [rng.normal(size=(nu, 3))]
    rest = count - nu
    split = rng.multinomial(rest, np.ones(lobes) / lobes)
    for k in range(lobes):
        mu = rng.normal(size=3)
        dirs.append(sample_vmf(rng, mu, rng.uniform(*kappa_range), int(split[k])))
    d = np.concatenate(dirs, 0)
    d = d[rng.permutation(count)]
    psi = rng.uniform(-np.pi, np.pi, count)
    return _euler_from_view(d, psi)


def ctf_half(n: int, defocus_um: torch.Tensor, astig_um: torch.Tensor, astig_angle: torch.Tensor,
             pixel_a: float = 1.0, voltage_kv: float = 300.0, cs_mm: float = 2.7,
             amplitude: float = 0.07) -> torch.Tensor:
    """CTF on the half-complex n x n grid (FFT order in y) for a batch of
    particles, (batch, n, n/2+1) float32.  gamma = K1 df r^2 + K2 r^4 - K3,
    CTF = -sin(gamma) with K1 = pi lambda, K2 = pi/2 Cs lambda^3,
    K3 = atan(A / sqrt(1 - A^2)); r in 1/Angstrom."""
    dev = defocus_um.device
    v = voltage_kv * 1e3
    lam = 12.2643247 / math.sqrt(v * (1.0 + v * 0.978466e-6))
    K1 = math.pi * lam
    K2 = math.pi / 2 * (cs_mm * 1e7) * lam ** 3
    K3 = math.atan(amplitude / math.sqrt(1 - amplitude * amplitude))
    x = torch.arange(n // 2 + 1, device=dev, dtype=torch.float32)
    y = torch.arange(n, device=dev, dtype=torch.float32)
    y = torch.where(y <= n // 2, y, y - n)
    kx = x[None, :] / (n * pixel_a)
    ky = y[:, None] / (n * pixel_a)
    r2 = kx * kx + ky * ky
    ang = torch.atan2(ky, kx)
    df = -(defocus_um[:, None, None] * 1e4
           + 0.5 * astig_um[:, None, None] * 1e4 * torch.cos(2 * (ang[None] - astig_angle[:, None, None])))
    gamma = K1 * df * r2[None] + K2 * r2[None] ** 2 - K3
    return (-torch.sin(gamma)).contiguous()


def in_disk_mask(n: int, rmax: int, device) -> torch.Tensor:
    x = torch.arange(n // 2 + 1, device=device)
    y = torch.arange(n, device=device)
    y = torch.where(y <= n // 2, y, y - n)
    return (x[None, :] ** 2 + y[:, None] ** 2) <= rmax * rmax
