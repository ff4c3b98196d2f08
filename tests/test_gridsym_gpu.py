"""The symmetric-spectrum gridding iteration (gtom_b200/csrc/gridsym.cu:
four passes per iteration over the Hermitian half along z of the real
iterated spectrum, with the library's own transforms) against the cuFFT path
and the FP64 oracle on the same inputs, on every grid it takes: powers of two
P = 64 .. 512 and the mixed-radix P = 96, 192 (radix 3) and 800 (radix 5).

Both paths compute the reference's iteration (RecFourier.cu:158-171); they
differ only in how the FP32 transforms round, so the weights after one
iteration agree to ~1e-6 and the maps after 10 iterations to relative L2
1e-5 (the bar here, tighter than the 1e-4 of reconstructions against the
reference).  Against the FP64 oracle the bar is the reconstructions' 1e-4."""
import numpy as np
import pytest
import torch

import gtom_b200 as G
from oracle import oracle as O
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


def _inputs(ori, pad=2, seed=0, hermitian=True):
    """Centred accumulators of a synthetic backprojection: blob data, smooth
    positive weights inside the padded sphere, both Hermitian on the x = 0
    plane (w(-y, -z) = w(y, z), data(-y, -z) = conj data(y, z)), as the
    backprojector's second insertions make them; hermitian=False leaves the
    data's x = 0 plane as drawn."""
    rng = np.random.default_rng(seed + ori)
    D = ori * pad + 1
    z, y, x = np.meshgrid(np.arange(D) - D // 2, np.arange(D) - D // 2, np.arange(D // 2 + 1), indexing="ij")
    r = np.sqrt(x ** 2 + y ** 2 + z ** 2)
    w = (np.where(r < ori * pad / 2, 1.0 + 30.0 * np.exp(-r / (ori / 3)), 0.0)
         * rng.uniform(0.8, 1.2, r.shape)).astype(np.float32)
    w[:, :, 0] = 0.5 * (w[:, :, 0] + w[::-1, ::-1, 0])
    data = ((rng.normal(size=r.shape) + 1j * rng.normal(size=r.shape)) * w * np.exp(-r / ori)).astype(np.complex64)
    if hermitian:
        data[:, :, 0] = 0.5 * (data[:, :, 0] + np.conj(data[::-1, ::-1, 0]))
    return data, w, D


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda().reshape(-1)


def _on(path, fn):
    G.set_path("gridding", path)
    try:
        out = fn()
        torch.cuda.synchronize()
        return out
    finally:
        G.set_path("gridding", "auto")


@pytest.mark.parametrize("ori", [32, 48, 64, 96, 128, 256])
def test_symmetric_gridding_matches_cufft(gtom_lib, cuda, ori):
    data, w, D = _inputs(ori)
    d_data, d_w = _dev(data), _dev(w)
    maps = {}
    for path in ("direct", "symmetric"):
        out = torch.full((ori ** 3,), float("nan"), device="cuda")
        _on(path, lambda: G.d_ReconstructGridding(d_data, d_w, out, (ori,) * 3, (D,) * 3, 2, 0, 0, 10))
        maps[path] = out.cpu().numpy()
    assert np.all(np.isfinite(maps["symmetric"]))
    assert rel_l2(maps["symmetric"], maps["direct"]) <= 1e-5


@pytest.mark.parametrize("iterations", [1, 3])
def test_symmetric_weights_match_cufft(gtom_lib, cuda, iterations):
    """The gridding weights themselves after a few iterations."""
    ori = 64
    data, w, D = _inputs(ori, seed=3)
    d_w = _dev(w)
    fnw = {}
    for path in ("direct", "symmetric"):
        fnw[path] = _on(path, lambda: G.gridding_weights(d_w, (D,) * 3, ori, 2, iterations, 0.0))[0].cpu().numpy()
    assert rel_l2(fnw["symmetric"], fnw["direct"]) <= 2e-6


@pytest.mark.parametrize("ori,iterations", [(16, 10), (24, 3), (32, 10), (32, 0), (48, 2)])
def test_symmetric_gridding_matches_oracle(gtom_lib, cuda, ori, iterations):
    """FP64 oracle (numpy pocketfft restatement of RecFourier.cu:98-241);
    ori 24 is a grid the path does not take (P = 48): cuFFT runs there.
    0 iterations: the final map divides by max(|Fw|, 1e-4)."""
    data, w, D = _inputs(ori, seed=7)
    out = torch.zeros(ori ** 3, device="cuda")
    _on("symmetric", lambda: G.d_ReconstructGridding(_dev(data), _dev(w), out, (ori,) * 3, (D,) * 3, 2, 0, 0,
                                                     iterations))
    ref = O.reconstruct_gridding(data, w, ori, (D, D, D), 2, iterations=iterations)
    assert rel_l2(out.cpu().numpy().reshape(ori, ori, ori), ref) <= 1e-4


@pytest.mark.parametrize("momentum", [0.0, 0.9])
def test_symmetric_long_runs_match_cufft(gtom_lib, cuda, momentum):
    """60 iterations (plain and with momentum), then to a change of 1e-4:
    the two paths may stop one iteration apart, and one iteration moves the
    weights by ~1e-4, so the stopped maps agree to 1e-3."""
    ori = 64
    data, w, D = _inputs(ori, seed=5)
    d_data, d_w = _dev(data), _dev(w)
    res = {}
    for path in ("direct", "symmetric"):
        fixed = torch.zeros(ori ** 3, device="cuda")
        _on(path, lambda: G.reconstruct_gridding_warm(d_data, d_w, fixed, (ori,) * 3, (D,) * 3, None, 2, 60, 0.0,
                                                      momentum))
        out = torch.zeros(ori ** 3, device="cuda")
        it, ch, _ = _on(path, lambda: G.reconstruct_gridding_warm(d_data, d_w, out, (ori,) * 3, (D,) * 3, None, 2,
                                                                  400, 1e-4, momentum))
        res[path] = (it, ch, out.cpu().numpy(), fixed.cpu().numpy())
    assert rel_l2(res["symmetric"][3], res["direct"][3]) <= 1e-4
    assert abs(res["symmetric"][0] - res["direct"][0]) <= 1
    assert res["symmetric"][1] <= 1e-4 and res["direct"][1] <= 1e-4
    assert rel_l2(res["symmetric"][2], res["direct"][2]) <= 1e-3


def test_symmetric_distance_to_reference_weights(gtom_lib, cuda):
    """The distance measure ||Fw (Fnw - ref)|| / ||Fw ref|| accumulated by
    the z pass equals the cuFFT path's update kernel's, and stops the loop at
    the same iteration (within one)."""
    ori = 64
    data, w, D = _inputs(ori, seed=9)
    d_w = _dev(w)
    ref = _on("direct", lambda: G.gridding_weights(d_w, (D,) * 3, ori, 2, 400, 0.0, momentum=0.9))[0]
    got = {}
    for path in ("direct", "symmetric"):
        got[path] = _on(path, lambda: G.gridding_weights(d_w, (D,) * 3, ori, 2, 1000, 0.0, ref_fnw=ref,
                                                         ref_tolerance=1e-2, return_distance=True))
    it_d, it_s = got["direct"][2], got["symmetric"][2]
    assert abs(it_d - it_s) <= 1 and it_d < 1000
    assert got["symmetric"][5] <= 1e-2


def test_symmetric_warm_start(gtom_lib, cuda):
    """The learned start (the committed 128^3 network) on the symmetric
    path: same decision on the predicted start and the same map as cuFFT's
    within the long-run bar."""
    from gtom_b200 import warmstart as WS
    ori = 64
    data, w, D = _inputs(ori, seed=11)
    d_data, d_w = _dev(data), _dev(w)
    params = WS.load_params(128, torch.device("cuda"))
    res = {}
    for path in ("direct", "symmetric"):
        out = torch.zeros(ori ** 3, device="cuda")
        it, ch, used = _on(path, lambda: G.reconstruct_gridding_warm(d_data, d_w, out, (ori,) * 3, (D,) * 3, params,
                                                                     2, 30, 0.0, 0.9))
        res[path] = (used, out.cpu().numpy())
    assert res["symmetric"][0] == res["direct"][0]
    assert rel_l2(res["symmetric"][1], res["direct"][1]) <= 1e-4


def test_symmetric_gridding_matches_cufft_at_800(gtom_lib, cuda):
    """P = 800 (400^3 at padding 2, the large combined configuration's grid;
    radix-5 transforms, rows of the x pass spanning warps), 3 iterations;
    inputs made on the GPU (2.6 GB of accumulators), Hermitian on x = 0."""
    ori, pad = 400, 2
    D = ori * pad + 1
    g = torch.Generator(device="cuda")
    g.manual_seed(800)
    z = torch.arange(D, device="cuda", dtype=torch.float32) - D // 2
    x = torch.arange(D // 2 + 1, device="cuda", dtype=torch.float32)
    r = torch.sqrt(z[:, None, None] ** 2 + z[None, :, None] ** 2 + x[None, None, :] ** 2)
    w = torch.where(r < ori * pad / 2, 1.0 + 30.0 * torch.exp(-r / (ori / 3)), torch.zeros_like(r))
    w = w * (0.8 + 0.4 * torch.rand(w.shape, device="cuda", generator=g))
    w[:, :, 0] = 0.5 * (w[:, :, 0] + torch.flip(w[:, :, 0], (0, 1)))
    data = torch.complex(torch.randn(w.shape, device="cuda", generator=g),
                         torch.randn(w.shape, device="cuda", generator=g)) * (w * torch.exp(-r / ori))
    data[:, :, 0] = 0.5 * (data[:, :, 0] + torch.flip(data[:, :, 0], (0, 1)).conj())
    del r
    d_w, d_data = w.reshape(-1).contiguous(), data.reshape(-1).contiguous()
    del w, data
    maps = {}
    for path in ("direct", "symmetric"):
        out = torch.full((ori ** 3,), float("nan"), device="cuda")
        _on(path, lambda: G.d_ReconstructGridding(d_data, d_w, out, (ori,) * 3, (D,) * 3, pad, 0, 0, 3))
        maps[path] = out
    assert torch.isfinite(maps["symmetric"]).all()
    err = (torch.linalg.vector_norm(maps["symmetric"] - maps["direct"]) /
           torch.linalg.vector_norm(maps["direct"])).item()
    assert err <= 1e-5, err


def test_symmetric_gridding_takes_asymmetric_weights_as_the_oracle(gtom_lib, cuda):
    """Weights whose x = 0 plane is not symmetric (a caller's own, not a
    backprojection's): every C2R of the path takes the x = 0 and x = P/2
    terms of each transformed row as real, i.e. transforms the Hermitian part
    of the plane, as numpy's irfftn in the oracle does."""
    ori = 32
    data, w, D = _inputs(ori, seed=13)
    rng = np.random.default_rng(13)
    w = w.copy()
    w[:, :, 0] *= rng.uniform(0.7, 1.3, w[:, :, 0].shape).astype(np.float32)
    out = torch.full((ori ** 3,), float("nan"), device="cuda")
    _on("symmetric", lambda: G.d_ReconstructGridding(_dev(data), _dev(w), out, (ori,) * 3, (D,) * 3, 2, 0, 0, 10))
    ref = O.reconstruct_gridding(data, w, ori, (D, D, D), 2, iterations=10)
    got = out.cpu().numpy().reshape(ori, ori, ori)
    assert np.all(np.isfinite(got))
    assert rel_l2(got, ref) <= 1e-4


def test_symmetric_final_map_of_non_hermitian_data_follows_the_oracle(gtom_lib, cuda):
    """Data whose x = 0 plane is not Hermitian: the final transform takes its
    Hermitian part, as numpy's irfftn in the oracle does.  (cuFFT's 3D C2R
    is not specified on such input, and its result differs from the oracle's
    at P = 128 and 256; a backprojection's data is Hermitian there.)"""
    ori = 64
    data, w, D = _inputs(ori, seed=17, hermitian=False)
    out = torch.full((ori ** 3,), float("nan"), device="cuda")
    _on("symmetric", lambda: G.d_ReconstructGridding(_dev(data), _dev(w), out, (ori,) * 3, (D,) * 3, 2, 0, 0, 2))
    ref = O.reconstruct_gridding(data, w, ori, (D, D, D), 2, iterations=2)
    got = out.cpu().numpy().reshape(ori, ori, ori)
    assert np.all(np.isfinite(got))
    assert rel_l2(got, ref) <= 1e-4


def test_symmetric_gridding_on_concurrent_streams(gtom_lib, cuda):
    """Two reconstructions enqueued on two streams at once, three times over
    (each call has its own work array, whose padding holds the y pass's work
    counter): the maps equal, bit for bit, those of the same calls made one
    after the other (the path has no atomics on values)."""
    ori = 64
    runs = []
    for seed in (21, 22):
        data, w, D = _inputs(ori, seed=seed)
        runs.append((_dev(data), _dev(w), D))
    serial = []
    for d_data, d_w, D in runs:
        out = torch.zeros(ori ** 3, device="cuda")
        G.d_ReconstructGridding(d_data, d_w, out, (ori,) * 3, (D,) * 3, 2, 0, 0, 10)
        serial.append(out)
    torch.cuda.synchronize()
    streams = [torch.cuda.Stream() for _ in runs]
    outs = [torch.full((ori ** 3,), float("nan"), device="cuda") for _ in runs]
    for _ in range(3):
        for (d_data, d_w, D), s, out in zip(runs, streams, outs):
            s.wait_stream(torch.cuda.current_stream())
            G.d_ReconstructGridding(d_data, d_w, out, (ori,) * 3, (D,) * 3, 2, 0, 0, 10, stream=s)
    torch.cuda.synchronize()
    for got, want in zip(outs, serial):
        assert torch.equal(got, want)
