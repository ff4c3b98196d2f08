"""The brick-major kernels against the direct ones on larger batches.

The brick projector evaluates every pixel with the direct kernel's
arithmetic on the same voxel values, so the two must agree bit for bit.  The
brick backprojector sums the same contributions in another order (shared
memory first, then one reduction per brick), so the two agree to FP32
rounding of the sums."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.helpers import rel_l2
from tests.synthdata import blob_volume_ft, random_angles

pytestmark = pytest.mark.gpu


def _paths(p, b):
    from gtom_b200 import set_path
    set_path("project", p)
    set_path("backproject", b)


@pytest.fixture(autouse=True)
def _reset(gtom_lib):
    yield
    _paths("auto", "auto")


def _angles(rng, batch, kind):
    if kind == "uniform":
        return random_angles(rng, batch)
    if kind == "near_identity":  # planes close to z = 0: many samples on the x = 0 plane boundary
        return (rng.normal(size=(batch, 3)) * 0.05).astype(np.float32)
    if kind == "axis_aligned":  # exact multiples of 90 degrees: samples on voxel faces
        return (rng.integers(0, 4, size=(batch, 3)) * (np.pi / 2)).astype(np.float32)
    raise ValueError(kind)


@pytest.mark.parametrize("n,scale,batch,kind", [(64, 2, 300, "uniform"), (32, 2, 200, "near_identity"),
                                                 (32, 2, 64, "axis_aligned"), (48, 3, 100, "uniform"),
                                                 (96, 2, 64, "uniform")])
def test_brick_projector_is_bit_identical(cuda, n, scale, batch, kind):
    from gtom_b200 import d_rlnProject, matrices_from_angles
    rng = np.random.default_rng(n * 7 + batch)
    P = scale * n
    vol = blob_volume_ft(rng, n, P, 20)
    vol = (vol + 0.01 * np.abs(vol).max() * (rng.normal(size=vol.shape) + 1j * rng.normal(size=vol.shape))).astype(np.complex64)
    mats = torch.from_numpy(matrices_from_angles(_angles(rng, batch, kind), float(scale))).cuda().reshape(-1)
    e = (n // 2 + 1) * n
    dv = torch.from_numpy(vol).cuda().reshape(-1)
    outs = {}
    for p in ("direct", "brick", "segment"):
        _paths(p, "auto")
        out = torch.full((batch * e,), complex(np.nan, np.nan), dtype=torch.complex64, device="cuda")
        d_rlnProject(dv, (P, P, P), out, (n, n, 1), n // 2, mats, batch)
        torch.cuda.synchronize()
        outs[p] = out
    for p in ("brick", "segment"):
        assert torch.isfinite(torch.view_as_real(outs[p])).all(), p
        assert torch.equal(outs["direct"], outs[p]), p


@pytest.mark.parametrize("n,V,batch,kind,dec,sq", [(64, 129, 300, "uniform", False, False),
                                                   (64, 128, 300, "uniform", True, False),
                                                   (32, 64, 200, "near_identity", True, True),
                                                   (32, 65, 64, "axis_aligned", False, False),
                                                   (48, 97, 100, "uniform", False, True),
                                                   (32, 64, 64, "uniform", False, False)])
def test_brick_backprojector_matches_direct(cuda, n, V, batch, kind, dec, sq):
    from gtom_b200 import d_rlnBackproject, matrices_from_angles
    rng = np.random.default_rng(n * 11 + batch)
    e = (n // 2 + 1) * n
    scale = 2.0 if V < 3 * n else 3.0
    ang = _angles(rng, batch, kind)
    m_host = matrices_from_angles(ang, scale)
    mats = torch.from_numpy(m_host).cuda().reshape(-1)
    projft = (rng.normal(size=(batch, e)) + 1j * rng.normal(size=(batch, e))).astype(np.complex64)
    projw = rng.uniform(0.1, 1, size=(batch, e)).astype(np.float32)
    dpf = torch.from_numpy(projft).cuda().reshape(-1)
    dpw = torch.from_numpy(projw).cuda().reshape(-1)
    nv = (V // 2 + 1) * V * V
    res = {}
    for b in ("direct", "brick", "segment_fp32", "segment"):
        _paths("auto", b)
        vf = torch.zeros(nv, dtype=torch.complex64, device="cuda")
        vw = torch.zeros(nv, dtype=torch.float32, device="cuda")
        d_rlnBackproject(vf, vw, (V, V, V), dpf, dpw, (n, n, 1), n // 2, mats, None, (1, 0, 0, 1), 0.0, dec, sq,
                         batch)
        torch.cuda.synchronize()
        res[b] = (vf.cpu().numpy(), vw.cpu().numpy())
    of, ow = np.zeros(nv, np.complex64), np.zeros(nv, np.float32)
    O.backproject(of, ow, V, projft, projw, n, n // 2, m_host, decentered=dec, square=sq, fp32=True)
    for p in ("brick", "segment_fp32", "segment"):
        assert rel_l2(res[p][0], res["direct"][0]) <= 1e-6, p
        assert rel_l2(res[p][1], res["direct"][1]) <= 1e-6, p
        assert rel_l2(res[p][0], of) <= 1e-5 and rel_l2(res[p][1], ow) <= 1e-5, p
        if p != "segment":
            # the voxels that received nothing are exactly the same ones
            assert np.array_equal(res[p][1] == 0, res["direct"][1] == 0), p
        else:
            # fixed point: a voxel that received only terms below half a
            # step (2^-26 of the largest weight) may stay exactly zero
            differ = (res[p][1] == 0) != (res["direct"][1] == 0)
            assert np.all(np.abs(res["direct"][1][differ]) <= 2.0 ** -25 * np.abs(ow).max()), p


def test_brick_backprojector_accumulates_across_calls(cuda):
    """Two calls into the same accumulators equal one call over both batches."""
    from gtom_b200 import d_rlnBackproject, matrices_from_angles
    rng = np.random.default_rng(5)
    n, V, batch = 32, 65, 120
    e = (n // 2 + 1) * n
    mats = torch.from_numpy(matrices_from_angles(random_angles(rng, batch), 2.0)).cuda()
    pf = torch.from_numpy((rng.normal(size=(batch, e)) + 1j * rng.normal(size=(batch, e))).astype(np.complex64)).cuda()
    nv = (V // 2 + 1) * V * V
    _paths("auto", "brick")
    a_f = torch.zeros(nv, dtype=torch.complex64, device="cuda")
    a_w = torch.zeros(nv, dtype=torch.float32, device="cuda")
    h = batch // 2
    for s in (slice(0, h), slice(h, batch)):
        d_rlnBackproject(a_f, a_w, (V, V, V), pf[s].reshape(-1), None, (n, n, 1), n // 2,
                         mats[s].reshape(-1).contiguous(), None, (1, 0, 0, 1), 0.0, False, False, s.stop - s.start)
    b_f = torch.zeros_like(a_f)
    b_w = torch.zeros_like(a_w)
    d_rlnBackproject(b_f, b_w, (V, V, V), pf.reshape(-1), None, (n, n, 1), n // 2, mats.reshape(-1), None,
                     (1, 0, 0, 1), 0.0, False, False, batch)
    torch.cuda.synchronize()
    assert rel_l2(a_f.cpu().numpy(), b_f.cpu().numpy()) <= 1e-6
    assert rel_l2(a_w.cpu().numpy(), b_w.cpu().numpy()) <= 1e-6


@pytest.mark.parametrize("kind,edge", [("unit_scale", 0), ("unit_scale", 12), ("sheared", 0), ("sheared", 9),
                                       ("odd_size", 0)])
def test_segment_paths_on_general_geometry(cuda, kind, edge):
    """The segment variants against the direct kernels where the row
    segments are least regular: a pixel spacing of one voxel (a brick spans
    more than 32 slice rows, so the rows come in several batches), sheared
    non-orthogonal slice matrices (the row range uses the full inverse of
    the columns' Gram matrix), an odd slice size (rows -n/2 .. n/2) and small
    bricks (many pairs per slice)."""
    from gtom_b200 import d_rlnBackproject, d_rlnProject, matrices_from_angles, set_brick_tuning
    rng = np.random.default_rng(91 + edge + len(kind))
    n = 63 if kind == "odd_size" else 64
    scale = 1.0 if kind == "unit_scale" else 2.0
    batch = 96
    m_host = matrices_from_angles(random_angles(rng, batch), scale).reshape(batch, 9)
    if kind == "sheared":
        m_host = (m_host + rng.normal(scale=0.15, size=m_host.shape) * scale).astype(np.float32)
        m_host *= 0.8  # keep every sample inside the brick grids
    mats = torch.from_numpy(np.ascontiguousarray(m_host)).cuda().reshape(-1)
    try:
        if edge:
            set_brick_tuning("project", edge=edge)
            set_brick_tuning("backproject", edge=edge)
        P = int(scale * n)
        vol = blob_volume_ft(rng, n, P, 12)
        dv = torch.from_numpy(vol.astype(np.complex64)).cuda().reshape(-1)
        e = (n // 2 + 1) * n
        outs = {}
        for p in ("direct", "segment"):
            _paths(p, "auto")
            out = torch.full((batch * e,), complex(np.nan, np.nan), dtype=torch.complex64, device="cuda")
            d_rlnProject(dv, (P, P, P), out, (n, n, 1), n // 2, mats, batch)
            torch.cuda.synchronize()
            outs[p] = out
        assert torch.equal(outs["direct"], outs["segment"])
        V = P + 1
        projft = (rng.normal(size=(batch, e)) + 1j * rng.normal(size=(batch, e))).astype(np.complex64)
        projw = rng.uniform(0.1, 1, size=(batch, e)).astype(np.float32)
        dpf = torch.from_numpy(projft).cuda().reshape(-1)
        dpw = torch.from_numpy(projw).cuda().reshape(-1)
        nv = (V // 2 + 1) * V * V
        res = {}
        for b in ("direct", "segment"):
            _paths("auto", b)
            vf = torch.zeros(nv, dtype=torch.complex64, device="cuda")
            vw = torch.zeros(nv, dtype=torch.float32, device="cuda")
            d_rlnBackproject(vf, vw, (V, V, V), dpf, dpw, (n, n, 1), n // 2, mats, None, (1, 0, 0, 1), 0.0, False,
                             False, batch)
            torch.cuda.synchronize()
            res[b] = (vf.cpu().numpy(), vw.cpu().numpy())
        assert rel_l2(res["segment"][0], res["direct"][0]) <= 1e-6
        assert rel_l2(res["segment"][1], res["direct"][1]) <= 1e-6
        # fixed point: only voxels whose terms all fell below half a step may
        # differ in being exactly zero
        differ = (res["segment"][1] == 0) != (res["direct"][1] == 0)
        assert np.all(np.abs(res["direct"][1][differ]) <= 2.0 ** -25 * np.abs(res["direct"][1]).max())
    finally:
        set_brick_tuning("project")
        set_brick_tuning("backproject")


@pytest.mark.parametrize("case", [
    dict(mag=(1.03, 0.02, -0.01, 0.97)),
    dict(ewald=30.0),
    dict(nvol=3),
    dict(mag=(0.98, -0.015, 0.02, 1.025), ewald=-45.0, nvol=2, sq=True),
    dict(mag=(1.01, 0.0, 0.0, 1.01), ewald=60.0, nvol=4, n=64, V=129, batch=200),
])
def test_segment_backprojector_general_geometry(cuda, case):
    """Magnification, Ewald curvature and per-slice volumes on the row-segment
    backprojector (centred output): the same contributions as the oracle's
    single-precision port of Backproject3DtoNDKernel, including the samples
    that come within one voxel of the volume's edge (folded by the clamps)."""
    from gtom_b200 import d_rlnBackproject
    c = dict(mag=(1, 0, 0, 1), ewald=0.0, nvol=1, sq=False, n=48, V=97, batch=300)
    c.update(case)
    n, V, batch, nvol = c["n"], c["V"], c["batch"], c["nvol"]
    rng = np.random.default_rng(n + batch + nvol)
    mats = O.matrices_f64(random_angles(rng, batch), 2.0).astype(np.float32)
    e = O.elements_fft(n)
    projft = (rng.normal(size=(batch, e)) + 1j * rng.normal(size=(batch, e))).astype(np.complex64)
    projw = rng.uniform(0.1, 1, size=(batch, e)).astype(np.float32)
    ivol = rng.integers(0, nvol, batch).astype(np.int32) if nvol > 1 else None
    nv = (V // 2 + 1) * V * V * nvol
    got = {}
    for path in ("direct", "segment"):
        _paths("auto", path)
        vf = torch.zeros(nv, dtype=torch.complex64, device="cuda")
        vw = torch.zeros(nv, dtype=torch.float32, device="cuda")
        d_rlnBackproject(vf, vw, (V, V, V), torch.from_numpy(projft).cuda().reshape(-1),
                         torch.from_numpy(projw).cuda().reshape(-1), (n, n, 1), n // 2,
                         torch.from_numpy(mats).cuda().reshape(-1),
                         None if ivol is None else torch.from_numpy(ivol).cuda(), c["mag"], c["ewald"], False,
                         c["sq"], batch)
        torch.cuda.synchronize()
        got[path] = (vf.cpu().numpy(), vw.cpu().numpy())
    of, ow = np.zeros(nv, np.complex64), np.zeros(nv, np.float32)
    O.backproject(of, ow, V, projft, projw, n, n // 2, mats, ivolume=ivol, magnification=c["mag"],
                  ewaldradiussuper=c["ewald"], decentered=False, square=c["sq"], fp32=True)
    for path, (gf, gw) in got.items():
        assert rel_l2(gf, of) <= 1e-5, path
        assert rel_l2(gw, ow) <= 1e-5, path


def _bp_segment(path, V, n, mats, projft, projw, dec=False):
    from gtom_b200 import d_rlnBackproject
    _paths("auto", path)
    batch = mats.shape[0]
    nv = (V // 2 + 1) * V * V
    vf = torch.zeros(nv, dtype=torch.complex64, device="cuda")
    vw = torch.zeros(nv, dtype=torch.float32, device="cuda")
    d_rlnBackproject(vf, vw, (V, V, V), torch.from_numpy(projft).cuda().reshape(-1),
                     torch.from_numpy(projw).cuda().reshape(-1), (n, n, 1), n // 2,
                     torch.from_numpy(mats).cuda().reshape(-1), None, (1, 0, 0, 1), 0.0, dec, False, batch)
    torch.cuda.synchronize()
    return vf.cpu().numpy(), vw.cpu().numpy()


@pytest.mark.parametrize("dec", [False, True])
def test_fixed_point_insertion_matches_fp32(cuda, dec):
    """The segment backprojector's fixed-point work items (int32 atomics of
    round(w v S)) against its FP32 ones and the oracle's port on the same
    2 000 slices of random data: the two agree to FP32 rounding of the sums."""
    rng = np.random.default_rng(1234 + dec)
    n, batch = 96, 2000
    V = 2 * n + (0 if dec else 1)
    mats = O.matrices_f64(random_angles(rng, batch), 2.0).astype(np.float32)
    e = O.elements_fft(n)
    projft = (rng.normal(size=(batch, e)) + 1j * rng.normal(size=(batch, e))).astype(np.complex64)
    projw = rng.uniform(0.0, 1.0, size=(batch, e)).astype(np.float32)
    fx = _bp_segment("segment", V, n, mats, projft, projw, dec)
    fp = _bp_segment("segment_fp32", V, n, mats, projft, projw, dec)
    assert rel_l2(fx[0], fp[0]) <= 1e-6 and rel_l2(fx[1], fp[1]) <= 1e-6
    of, ow = np.zeros_like(fx[0]), np.zeros_like(fx[1])
    O.backproject(of, ow, V, projft, projw, n, n // 2, mats, decentered=dec, fp32=True)
    assert rel_l2(fx[0], of) <= 1e-5 and rel_l2(fx[1], ow) <= 1e-5


@pytest.mark.parametrize("kind", ["outlier", "coherent"])
def test_fixed_point_falls_back_to_fp32(cuda, kind):
    """Items whose fixed-point sums could overflow are accumulated again in
    FP32: a single pixel 1e7 times larger than the rest (the magnitude sample
    does not see it, its terms exceed the fixed-point range), and 1 500
    slices of one orientation with identical data (every voxel near the
    plane sums 1 500 equal terms)."""
    rng = np.random.default_rng(77)
    n, V = 64, 129
    e = O.elements_fft(n)
    if kind == "outlier":
        batch = 1200
        mats = O.matrices_f64(random_angles(rng, batch), 2.0).astype(np.float32)
        projft = (rng.normal(size=(batch, e)) + 1j * rng.normal(size=(batch, e))).astype(np.complex64)
        projft[517, 300] = 1e7 + 3e6j
    else:
        batch = 1500
        mats = np.repeat(O.matrices_f64(random_angles(rng, 1), 2.0).astype(np.float32), batch, axis=0)
        one = (rng.normal(size=e) + 1j * rng.normal(size=e)).astype(np.complex64)
        projft = np.repeat(one[None], batch, axis=0)
    projw = rng.uniform(0.5, 1.0, size=(batch, e)).astype(np.float32)
    fx = _bp_segment("segment", V, n, mats, projft, projw)
    of, ow = np.zeros_like(fx[0]), np.zeros_like(fx[1])
    O.backproject(of, ow, V, projft, projw, n, n // 2, mats, decentered=False, fp32=True)
    assert np.all(np.isfinite(fx[0])) and np.all(np.isfinite(fx[1]))
    assert rel_l2(fx[0], of) <= 1e-5 and rel_l2(fx[1], ow) <= 1e-5
