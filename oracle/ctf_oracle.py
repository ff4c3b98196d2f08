"""Test infrastructure: a float64 numpy restatement of the CTF simulation
(gtom's d_CTFSimulate: include/CTF.cuh:100-137 for the parameter
conversion, :195-223 for d_GetCTF, src/CTF/Simulate.cu:117-139 for the
per-point kernel) and of the particle preprocessing the library builds on
it (gtom_b200/csrc/ctf.cu: R2C of the centred particle, CTF multiply,
squared CTF as weights).  Only tests may import it.
"""
from __future__ import annotations

import numpy as np

FIELDS = ("pixelsize", "pixeldelta", "pixelangle", "Cs", "voltage", "defocus", "astigmatismangle",
          "defocusdelta", "amplitude", "Bfactor", "Bfactordelta", "Bfactorangle", "scale", "phaseshift")
DEFAULTS = dict(pixelsize=1e-10, pixeldelta=0.0, pixelangle=0.0, Cs=2e-3, voltage=300e3, defocus=-3e-6,
                astigmatismangle=0.0, defocusdelta=0.0, amplitude=0.07, Bfactor=0.0, Bfactordelta=0.0,
                Bfactorangle=0.0, scale=1.0, phaseshift=0.0)


def params_array(params: list[dict]) -> np.ndarray:
    """(batch, 14) float32 in CTFParams' field order, defaults filled in."""
    return np.array([[float(np.float32({**DEFAULTS, **p}[f])) for f in FIELDS] for p in params], np.float32)


def lean(p: np.ndarray) -> dict:
    """CTFParamsLean in float64 (Angstrom units)."""
    d = dict(zip(FIELDS, (float(v) for v in p)))
    lam = 12.2643247 / np.sqrt(d["voltage"] * (1.0 + d["voltage"] * 0.978466e-6))
    return dict(pixelsize=d["pixelsize"] * 1e10, pixeldelta=d["pixeldelta"] * 0.5e10, pixelangle=d["pixelangle"],
                defocus=d["defocus"] * 1e10, astigmatismangle=d["astigmatismangle"],
                defocusdelta=d["defocusdelta"] * 0.5e10, scale=d["scale"], phaseshift=d["phaseshift"],
                K1=np.pi * lam, K2=np.pi / 2 * d["Cs"] * 1e10 * lam ** 3,
                K3=np.arctan(d["amplitude"] / np.sqrt(1 - d["amplitude"] ** 2)),
                Bfactor=d["Bfactor"] * 0.25e20, Bfactordelta=d["Bfactordelta"] * 0.25e20,
                Bfactorangle=d["Bfactorangle"])


def ctf(k: np.ndarray, angle: np.ndarray, L: dict, gammacorr=0.0, amplitudesquared=False,
        ignorefirstpeak=False) -> np.ndarray:
    """d_GetCTF at spatial frequency k (1/Angstrom) and azimuth angle."""
    r2 = k * k
    deltaf = L["defocus"] + L["defocusdelta"] * np.cos(2 * (angle - L["astigmatismangle"]))
    gamma = L["K1"] * deltaf * r2 + L["K2"] * r2 * r2 - L["phaseshift"] - L["K3"] + gammacorr
    v = -np.sin(gamma)
    if ignorefirstpeak:
        v = np.where(np.abs(gamma) < np.pi / 2, 1.0, v)
    if L["Bfactor"] != 0 or L["Bfactordelta"] != 0:
        b = L["Bfactor"] + (L["Bfactordelta"] * np.cos(2 * (angle - L["Bfactorangle"]))
                            if L["Bfactordelta"] != 0 else 0.0)
        v = v * np.exp(b * r2)
    if amplitudesquared:
        v = np.abs(v)
    return v * L["scale"]


def simulate(params: np.ndarray, addresses: np.ndarray, gammacorr=None, amplitudesquared=False,
             ignorefirstpeak=False) -> np.ndarray:
    """d_CTFSimulate: (batch, n) values at addresses (n, 2) = (frequency in
    1/pixel, angle); the pixel size varies with the angle by pixeldelta."""
    a = np.asarray(addresses, np.float64).reshape(-1, 2)
    g = 0.0 if gammacorr is None else np.asarray(gammacorr, np.float64)
    out = []
    for p in np.asarray(params, np.float32).reshape(-1, 14):
        L = lean(p)
        ps = L["pixelsize"] + L["pixeldelta"] * np.cos(2 * (a[:, 1] - L["pixelangle"]))
        out.append(ctf(a[:, 0] / ps, a[:, 1], L, g, amplitudesquared, ignorefirstpeak))
    return np.array(out)


def half_grid_addresses(n: int) -> np.ndarray:
    """(n * (n/2+1), 2) addresses of the half-complex n x n grid, y in FFT
    order: (sqrt(x^2 + y^2) / n, atan2(y, x))."""
    x = np.arange(n // 2 + 1)
    y = np.arange(n)
    y = np.where(y <= n // 2, y, y - n)
    X, Y = np.meshgrid(x, y)
    return np.stack([np.sqrt(X ** 2 + Y ** 2) / n, np.arctan2(Y, X)], -1).reshape(-1, 2)


def preprocess(images: np.ndarray, params: np.ndarray | None):
    """(CTF * FT, CTF^2) of centred real particles (batch, n, n): FT is the
    unnormalised R2C of the particle moved to the origin."""
    imgs = np.asarray(images, np.float64)
    n = imgs.shape[-1]
    ft = np.fft.rfft2(np.fft.ifftshift(imgs, axes=(-2, -1))).reshape(len(imgs), -1)
    if params is None:
        return ft, np.ones(ft.shape)
    c = simulate(params, half_grid_addresses(n))
    return ft * c, c * c
