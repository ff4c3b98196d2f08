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


def tilt_matrices(euler: np.ndarray, tilts_deg: np.ndarray, supersample: float) -> np.ndarray:
    """(ntilts, 9) float32 matrices (the library's layout, glm column-major)
    of a tilt series: the subvolume's rotation E (ZYZ Euler, radians), then a
    rotation by each tilt angle about y; M = s (T E)^T."""
    from .relion import matrices_from_angles
    Es_t = matrices_from_angles(np.asarray(euler, np.float32)[None], 1.0)[0].reshape(3, 3).T  # E^T
    out = np.empty((len(tilts_deg), 9), np.float32)
    for k, t in enumerate(np.deg2rad(np.asarray(tilts_deg, np.float64))):
        c, s = math.cos(t), math.sin(t)
        T = np.array([[c, 0, -s], [0, 1, 0], [s, 0, c]])
        M = supersample * (Es_t.astype(np.float64) @ T.T)
        out[k] = M.T.ravel()
    return out


def tilt_series_batch(count: int, seed: int, device, boxes=(32, 48, 64, 96, 128), pad: int = 2,
                      tilt_range: float = 60.0, tilt_step: float = 3.0, max_dose: float = 120.0,
                      snr: float = 0.1, pixel_a: float = 1.0):
    """Synthetic sub-tomogram batch: per subvolume a box from `boxes`
    (uniform), a volume of Gaussian blobs, a random rotation and a tilt
    series over +-tilt_range in tilt_step steps (41 tilts by default); per
    tilt a CTF (300 kV, Cs 2.7 mm, defocus U(2, 5) um) and the dose filter
    exp(-N k^2 / 4), N the dose accumulated in dose-symmetric order up to
    max_dose e/A^2, and white noise at `snr`.  Returns a list of dicts with
    box, projft (CTF- and dose-weighted noisy slices), projweights (their
    squared weights), matrices and an output map buffer."""
    from .relion import d_rlnProject
    rng = np.random.default_rng(seed)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    tilts = np.arange(-tilt_range, tilt_range + 1e-6, tilt_step)
    nt = len(tilts)
    order = np.argsort(np.abs(tilts), kind="stable")  # dose-symmetric acquisition
    dose = np.empty(nt)
    dose[order] = (np.arange(nt) + 1) * max_dose / nt
    out = []
    for i in range(count):
        n = int(rng.choice(boxes))
        P = n * pad
        e = (n // 2 + 1) * n
        vol = blob_volume(n, max(20, n // 2), int(rng.integers(1 << 31)), device)
        volft = padded_half_ft(vol, pad).reshape(-1)
        euler = _euler_from_view(rng.normal(size=(1, 3)), rng.uniform(-np.pi, np.pi, 1))[0]
        mats = torch.from_numpy(tilt_matrices(euler, tilts, float(pad))).to(device)
        proj = torch.empty(nt * e, dtype=torch.complex64, device=device)
        d_rlnProject(volft, (P, P, P), proj, (n, n, 1), n // 2, mats.reshape(-1), nt)
        df = torch.from_numpy(rng.uniform(2.0, 5.0, nt).astype(np.float32)).to(device)
        zero = torch.zeros(nt, dtype=torch.float32, device=device)
        ctf = ctf_half(n, df, zero, zero, pixel_a=pixel_a).reshape(nt, e)
        x = torch.arange(n // 2 + 1, device=device, dtype=torch.float32)
        y = torch.arange(n, device=device, dtype=torch.float32)
        y = torch.where(y <= n // 2, y, y - n)
        k2 = ((x[None, :] ** 2 + y[:, None] ** 2) / (n * pixel_a) ** 2).reshape(-1)
        filt = ctf * torch.exp(-torch.from_numpy(dose.astype(np.float32)).to(device)[:, None] * k2[None] / 4)
        sig = proj.reshape(nt, e) * filt
        disk = in_disk_mask(n, n // 2, device).reshape(-1)
        pw = (sig.abs() ** 2 * disk).sum(1, keepdim=True) / disk.sum()
        sd = torch.sqrt(pw / snr / 2)
        noise = torch.complex(torch.randn((nt, e), device=device, generator=gen),
                              torch.randn((nt, e), device=device, generator=gen)) * sd
        out.append(dict(box=n, projft=((sig + noise) * filt).contiguous().reshape(-1),
                        projweights=(filt * filt).contiguous().reshape(-1), matrices=mats.reshape(-1),
                        out=torch.empty(n ** 3, dtype=torch.float32, device=device)))
        del vol, volft, proj
    return out
