"""CPU checks of the oracle itself: closed-form Bessel values against scipy,
known-answer projections, the FP32 port against the FP64 restatement, and
the gridding restatement's behaviour on uniform sampling."""
import numpy as np
import pytest
import scipy.special as sp

from oracle import oracle as O
from tests.helpers import fsc, rel_l2
from tests.synthdata import blob_volume_ft, random_angles


@pytest.mark.parametrize("order", [0, 2])
@pytest.mark.parametrize("w", [0.0, 0.013, 0.1, 0.25, 0.4999, 0.63, 0.9])
def test_kaiser_bessel_against_scipy(order, w):
    a, alpha = 3.8, 15.0
    t = 2 * np.pi * a * w
    sigma = np.sqrt(abs(alpha ** 2 - t ** 2))
    nu = 1.5 if order == 0 else 3.5
    bes = sp.jv(nu, sigma) if t > alpha else sp.iv(nu, sigma)
    ref = (2 * np.pi) ** 1.5 * a ** 3 * (alpha ** 2 if order == 2 else 1) * bes / (sp.i0(alpha) * sigma ** nu)
    assert O.kaiser_fourier_value(w, a, alpha, order) == pytest.approx(ref, rel=1e-9, abs=1e-14)


def test_kb_table_normalised_and_monotone_in_band():
    t = O.kb_table(3.8, 15.0, 0, 10000)
    assert t[0] == 1.0
    assert np.all(np.diff(t[:4000]) < 0)


def test_project_constant_volume_gives_constant_slice():
    """KAT: a delta at the real-space origin has a constant spectrum, so every
    sample inside rmax interpolates to exactly 1 and outside is 0."""
    P, n = 32, 16
    vol = np.ones((P, P, P // 2 + 1), np.complex64)
    mats = O.matrices_f64(random_angles(np.random.default_rng(1), 7), 2.0).astype(np.float32)
    out = O.project(vol, P, n, n // 2, mats)
    x = np.arange(n // 2 + 1)
    y = np.where(np.arange(n) <= n // 2, np.arange(n), np.arange(n) - n)
    inside = (x[None, :] ** 2 + y[:, None] ** 2 <= (n // 2) ** 2).ravel()
    assert np.allclose(out[:, inside], 1.0, atol=1e-12)
    assert np.all(out[:, ~inside] == 0)


def test_project_identity_reads_the_central_plane():
    """KAT: with M = 2 I the slice samples the z = 0 plane at even voxels."""
    rng = np.random.default_rng(2)
    P, n = 32, 16
    vol = (rng.normal(size=(P, P, P // 2 + 1)) + 1j * rng.normal(size=(P, P, P // 2 + 1))).astype(np.complex64)
    m = np.array([[2, 0, 0, 0, 2, 0, 0, 0, 2]], np.float32)
    out = O.project(vol, P, n, n // 2, m)[0].reshape(n, n // 2 + 1)
    for yi in range(n):
        y = yi if yi <= n // 2 else yi - n
        for x in range(n // 2 + 1):
            if x * x + y * y > (n // 2) ** 2:
                continue
            assert out[yi, x] == pytest.approx(vol[0, (2 * y) % P, 2 * x], abs=1e-6)


def test_project_hermitian_pairs():
    """Samples on the x = 0 column at +y and -y are conjugate mates."""
    rng = np.random.default_rng(3)
    P, n = 32, 16
    vol = blob_volume_ft(rng, n, P, 8)
    mats = O.matrices_f64(random_angles(rng, 5), 2.0).astype(np.float32)
    out = O.project(vol, P, n, n // 2, mats).reshape(5, n, n // 2 + 1)
    for y in range(1, n // 2):
        a, b = out[:, y, 0], out[:, n - y, 0]
        assert np.allclose(a, np.conj(b), atol=1e-3 * np.abs(out).max())


def test_fp32_port_matches_fp64_oracle():
    rng = np.random.default_rng(4)
    P, n = 64, 32
    vol = blob_volume_ft(rng, n, P, 20)
    mats = O.matrices_f64(random_angles(rng, 20), 2.0).astype(np.float32)
    a = O.project(vol, P, n, n // 2, mats)
    b = O.project(vol, P, n, n // 2, mats, fp32=True)
    assert rel_l2(b, a) < 1e-5
    proj = a.astype(np.complex64)
    w = rng.uniform(0.1, 1, size=proj.shape).astype(np.float32)
    nv = (P // 2 + 1) * P * P
    # With binary16 weights a few weights round to the neighbouring binary16
    # value when the single- and double-precision products straddle a
    # rounding boundary (one binary16 ulp is ~4.9e-4 relative), so that mode
    # agrees to 1e-4; with full-precision weights to 1e-5.
    for half, tol in ((True, 1e-4), (False, 1e-5)):
        v64, w64 = np.zeros(nv, np.complex128), np.zeros(nv)
        v32, w32 = np.zeros(nv, np.complex64), np.zeros(nv, np.float32)
        O.backproject(v64, w64, P, proj, w, n, n // 2, mats, half_weights=half)
        O.backproject(v32, w32, P, proj, w, n, n // 2, mats, fp32=True, half_weights=half)
        assert rel_l2(v32, v64) < tol
        assert rel_l2(w32, w64) < tol


def test_backproject_weights_sum_to_slice_weight():
    """Without binary16 rounding the 8 trilinear weights of a sample sum to 1,
    and each sample lands once more for every x = 0 neighbour mirrored onto
    the plane's other half; with a flat slice of weight 1 the total inserted
    weight therefore equals the inserted samples plus the x = 0 duplicates."""
    P, n = 32, 16
    m = np.array([[2, 0, 0, 0, 2, 0, 0, 0, 2]], np.float32)  # samples on even voxels, fx = 0
    nv = (P // 2 + 1) * P * P
    w = np.zeros(nv)
    O.backproject(None, w, P, None, None, n, n // 2, m, half_weights=False)
    x = np.arange(n // 2 + 1)
    y = np.where(np.arange(n) <= n // 2, np.arange(n), np.arange(n) - n)
    X, Y = np.meshgrid(x, y)
    ins = (X * X + Y * Y < (n // 2) ** 2) & ~((X == 0) & (Y < 0))
    dup = ins & (X == 0) & (Y != 0)
    assert w.sum() == pytest.approx(ins.sum() + dup.sum())


def test_gridding_uniform_weights_converge_to_constant():
    """KAT: a flat sampling density makes the gridding weights converge to a
    constant inside the mask (the blob convolution of a constant is flat)."""
    ori, pad = 16, 2
    P = ori * pad
    D = P + 1
    weight = np.ones((D, D, D // 2 + 1), np.float32)
    data = np.zeros((D, D, D // 2 + 1), np.complex64)
    _, Fnw = O.reconstruct_gridding(data, weight, ori, (D, D, D), pad, iterations=20, return_weights=True)
    z = np.arange(P)
    zp = np.where(z < P // 2 + 1, z, z - P)
    x = np.arange(P // 2 + 1)
    r = np.sqrt(zp[:, None, None] ** 2 + zp[None, :, None] ** 2 + x[None, None, :] ** 2)
    core = Fnw[r < P / 4]
    assert core.std() / core.mean() < 2e-2


def test_gridding_reconstructs_blob_volume():
    """End-to-end on the oracle: dense projections of a blob volume, centred
    backprojection, gridding; the map agrees with the truth shell by shell up
    to one shell below Nyquist."""
    rng = np.random.default_rng(5)
    ori, pad = 16, 2
    P = ori * pad
    D = P + 1
    vol_ft = blob_volume_ft(rng, ori, P, 6)
    mats = O.matrices_f64(random_angles(rng, 1500), float(pad)).astype(np.float32)
    proj = O.project(vol_ft, P, ori, ori // 2, mats).astype(np.complex64)
    nv = (D // 2 + 1) * D * D
    data, w = np.zeros(nv, np.complex128), np.zeros(nv)
    O.backproject(data, w, D, proj, None, ori, ori // 2, mats, decentered=False)
    rec = O.reconstruct_gridding(data.reshape(D, D, D // 2 + 1), w.reshape(D, D, D // 2 + 1), ori, (D, D, D), pad)
    truth = np.fft.fftshift(np.fft.irfftn(vol_ft, s=(P, P, P), axes=(0, 1, 2)))
    o = P // 2 - ori // 2
    truth = truth[o:o + ori, o:o + ori, o:o + ori]
    assert np.all(fsc(rec, truth)[: ori // 2 - 1] > 0.98)
