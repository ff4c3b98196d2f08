"""The fused FFT iteration of the gridding reconstructor (gtom_b200/csrc/
gridfft.cu: two passes per iteration with the library's own transforms)
against the cuFFT path on the same inputs.  Both compute the reference's
iteration; the transforms round differently in FP32, and the iteration's
division by the convolved weights carries that into the maps, so the maps
agree to relative L2 1e-4 and the iteration counts to the convergence test
exactly or within one.  Parity of either path with the reference and the
FP64 oracle is tested in test_parity_gpu.py (which runs the default path)."""
import numpy as np
import pytest
import torch

import gtom_b200 as G
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


def _inputs(ori, pad=2, seed=0):
    """Centred accumulators of a synthetic backprojection: blob data, smooth
    positive weights inside the padded sphere."""
    rng = np.random.default_rng(seed + ori)
    D = ori * pad + 1
    z, y, x = np.meshgrid(np.arange(D) - D // 2, np.arange(D) - D // 2, np.arange(D // 2 + 1), indexing="ij")
    r = np.sqrt(x ** 2 + y ** 2 + z ** 2)
    w = (np.where(r < ori * pad / 2, 1.0 + 30.0 * np.exp(-r / (ori / 3)), 0.0)
         * rng.uniform(0.8, 1.2, r.shape)).astype(np.float32)
    data = ((rng.normal(size=r.shape) + 1j * rng.normal(size=r.shape)) * w * np.exp(-r / ori)).astype(np.complex64)
    return torch.from_numpy(data).cuda().reshape(-1), torch.from_numpy(w).cuda().reshape(-1), D


def _run(path, fn):
    G.set_path("gridding", path)
    try:
        out = fn()
        torch.cuda.synchronize()
        return out
    finally:
        G.set_path("gridding", "auto")


@pytest.mark.parametrize("ori", [32, 64, 128, 256])
def test_fused_gridding_matches_cufft(gtom_lib, cuda, ori):
    data, w, D = _inputs(ori)
    maps = {}
    for path in ("direct", "fused"):
        out = torch.full((ori ** 3,), float("nan"), device="cuda")
        _run(path, lambda: G.d_ReconstructGridding(data, w, out, (ori,) * 3, (D,) * 3, 2, 0, 0, 10))
        maps[path] = out.cpu().numpy()
    assert np.all(np.isfinite(maps["fused"]))
    assert rel_l2(maps["fused"], maps["direct"]) <= 1e-4


@pytest.mark.parametrize("momentum", [0.0, 0.9])
def test_fused_gridding_long_runs_match_cufft(gtom_lib, cuda, momentum):
    """60 iterations (plain and with momentum), then to a change of 1e-4:
    the two paths may stop one iteration apart, and one iteration moves the
    weights by ~1e-4, so the stopped maps agree to 1e-3."""
    ori = 64
    data, w, D = _inputs(ori, seed=5)
    res = {}
    for path in ("direct", "fused"):
        fixed = torch.zeros(ori ** 3, device="cuda")
        _run(path, lambda: G.reconstruct_gridding_warm(data, w, fixed, (ori,) * 3, (D,) * 3, None, 2, 60, 0.0,
                                                       momentum))
        out = torch.zeros(ori ** 3, device="cuda")
        it, ch, _ = _run(path, lambda: G.reconstruct_gridding_warm(data, w, out, (ori,) * 3, (D,) * 3, None, 2, 400,
                                                                   1e-4, momentum))
        res[path] = (it, ch, out.cpu().numpy(), fixed.cpu().numpy())
    assert rel_l2(res["fused"][3], res["direct"][3]) <= 1e-4
    assert abs(res["fused"][0] - res["direct"][0]) <= 1
    assert res["fused"][1] <= 1e-4 and res["direct"][1] <= 1e-4
    assert rel_l2(res["fused"][2], res["direct"][2]) <= 1e-3


def test_gridding_path_switch_rejects_brick(gtom_lib):
    with pytest.raises(G.GtomError):
        G.set_path("gridding", "brick")
