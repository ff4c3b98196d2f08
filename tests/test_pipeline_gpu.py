"""End to end on the GPU, through the default paths (row-segment brick
projector and insertion, cuFFT gridding): a blob volume is projected at
dense uniform orientations, the projections are inserted (plain and CTF-
weighted, with the CTF squared as the weights), and the gridded maps must
agree with the truth shell by shell up to just below Nyquist, as the
oracle's own end-to-end test does at a smaller size.  The blobs are sharp
(0.5-1 voxel) so that the outer shells carry signal."""
import numpy as np
import pytest
import torch

import gtom_b200 as G
from tests.helpers import fsc
from tests.synthdata import random_angles

pytestmark = pytest.mark.gpu


def _sharp_blobs_ft(rng, n, P, nblobs):
    """Decentred half FT of n^3 Gaussian blobs of 0.5-1 voxel, padded to P:
    sharp enough that every shell up to Nyquist carries signal (smooth blobs
    leave the outer shells at 1e-4 of the power and their FSC meaningless)."""
    c = np.arange(n) - n // 2
    vol = np.zeros((n, n, n))
    for _ in range(nblobs):
        ctr = rng.normal(size=3)
        ctr = ctr / np.linalg.norm(ctr) * rng.random() ** (1 / 3) * 0.4 * n
        s = rng.uniform(0.5, 1.0)
        d2 = (c[:, None, None] - ctr[2]) ** 2 + (c[None, :, None] - ctr[1]) ** 2 + (c[None, None, :] - ctr[0]) ** 2
        vol += rng.uniform(0.2, 1.0) * np.exp(-d2 / (2 * s * s))
    padded = np.zeros((P, P, P))
    o = P // 2 - n // 2
    padded[o:o + n, o:o + n, o:o + n] = vol
    return np.fft.rfftn(np.fft.ifftshift(padded)).astype(np.complex64)


def _truth(vol_ft, ori, P):
    truth = np.fft.fftshift(np.fft.irfftn(vol_ft, s=(P, P, P), axes=(0, 1, 2)))
    o = P // 2 - ori // 2
    return truth[o:o + ori, o:o + ori, o:o + ori]


@pytest.mark.parametrize("ctf", [False, True])
def test_dense_projection_insertion_gridding_recovers_the_volume(gtom_lib, cuda, ctf):
    rng = np.random.default_rng(11 + ctf)
    ori, pad, batch = 64, 2, 8000
    P, D = ori * pad, ori * pad + 1
    vol_ft = _sharp_blobs_ft(rng, ori, P, 40)
    mats = torch.from_numpy(G.matrices_from_angles(random_angles(rng, batch), float(pad))).cuda().reshape(-1)
    e = (ori // 2 + 1) * ori
    proj = torch.empty(batch * e, dtype=torch.complex64, device="cuda")
    G.d_rlnProject(torch.from_numpy(vol_ft.astype(np.complex64)).cuda().reshape(-1), (P, P, P), proj,
                   (ori, ori, 1), ori // 2, mats, batch)
    weights = None
    if ctf:  # a CTF-like modulation c with zeros: the image is c * proj, and the
        # caller inserts c * image with weights c^2 (the backprojector takes both as given)
        y = np.fft.fftfreq(ori) * ori
        x = np.arange(ori // 2 + 1)
        r2 = (y[:, None] ** 2 + x[None, :] ** 2).ravel()
        df = rng.uniform(0.5, 2.0, batch)
        c = np.cos(np.outer(df, r2) * (np.pi / (ori * ori)) * 6.0).astype(np.float32) * 0.9 + 0.1
        cc = torch.from_numpy(c).cuda().reshape(-1)
        proj = proj * (cc * cc)
        weights = (cc * cc).contiguous()
    nv = (D // 2 + 1) * D * D
    vf = torch.zeros(nv, dtype=torch.complex64, device="cuda")
    vw = torch.zeros(nv, dtype=torch.float32, device="cuda")
    G.d_rlnBackproject(vf, vw, (D, D, D), proj.contiguous(), weights, (ori, ori, 1), ori // 2, mats, None,
                       (1, 0, 0, 1), 0.0, False, False, batch)
    rec = torch.zeros(ori ** 3, dtype=torch.float32, device="cuda")
    G.d_ReconstructGridding(vf, vw, rec, (ori,) * 3, (D,) * 3, pad, 0, 0, 10)
    torch.cuda.synchronize()
    f = fsc(rec.cpu().numpy().reshape(ori, ori, ori), _truth(vol_ft, ori, P))
    # trilinear interpolation at padding 2 costs the last shells below
    # Nyquist a little correlation; everything to 0.9 Nyquist is near-exact
    assert np.all(f[: int(0.9 * ori // 2) + 1] > 0.99), np.round(f, 4)
    assert np.all(f[: ori // 2 - 1] > 0.97), np.round(f, 4)
