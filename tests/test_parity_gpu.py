"""Parity of the CUDA library (through its C ABI) with the oracle and with the
reference's own CUDA results (tests/golden/, made by make_golden.py).

Tolerances (relative L2 unless stated):
  projections     <= 1e-5 against the FP64 oracle; <= 1e-6 against the
                     reference (same single-precision arithmetic).
  backprojection  <= 1e-5 against the oracle's single-precision port (same
                     binary16 weights; only the atomic summation order
                     differs); <= 1e-4 against the FP64 oracle (a few
                     binary16 weights round the other way when the FP64 and
                     FP32 products straddle a rounding boundary); <= 1e-5
                     against the reference.
  reconstruction  <= 1e-4 against the FP64 oracle and against the
                     reference, FSC >= 0.999 in every shell to Nyquist.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.helpers import fsc, load_golden, rel_l2
from tests.synthdata import blob_volume_ft, random_angles

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["direct", "brick", "segment"])
def impl(request, gtom_lib):
    """Runs a test once per implementation of the projector / backprojector."""
    from gtom_b200 import set_path
    set_path("project", request.param)
    set_path("backproject", request.param)
    yield request.param
    set_path("project", "auto")
    set_path("backproject", "auto")


def cu(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def noisy_volume(rng, n, P):
    vol = blob_volume_ft(rng, n, P, 12)
    noise = (rng.normal(size=vol.shape) + 1j * rng.normal(size=vol.shape)) * 0.02 * np.abs(vol).max()
    return (vol + noise).astype(np.complex64)


def gpu_project(vol, P, n, ndims, rmax, mats):
    from gtom_b200 import d_rlnProject, elements_fft
    batch = mats.shape[0]
    e = elements_fft((n, n, n if ndims == 3 else 1))
    out = torch.full((batch * e,), complex(np.nan, np.nan), dtype=torch.complex64, device="cuda")
    d_rlnProject(cu(vol).reshape(-1), (P, P, P), out, (n, n, n if ndims == 3 else 1), rmax,
                 cu(mats).reshape(-1), batch)
    torch.cuda.synchronize()
    return out.cpu().numpy().reshape(batch, e)


# ----------------------------------------------------------------- project --
@pytest.mark.parametrize("n,ndims,batch,scale", [(16, 2, 30, 2), (32, 2, 50, 2), (64, 2, 40, 2),
                                                 (16, 2, 20, 3), (8, 3, 2, 2), (16, 3, 2, 2)])
def test_project_matches_oracle(gtom_lib, cuda, impl, n, ndims, batch, scale):
    rng = np.random.default_rng(100 + n + ndims)
    P = scale * n
    vol = noisy_volume(rng, n, P)
    mats = O.matrices_f64(random_angles(rng, batch), float(scale)).astype(np.float32)
    got = gpu_project(vol, P, n, ndims, n // 2, mats)
    ref = O.project(vol, P, n, n // 2, mats, ndims=ndims)
    assert rel_l2(got, ref) <= 1e-5
    assert np.all(np.isfinite(got))


@pytest.mark.parametrize("rmax", [0, 3, 8, 100])
def test_project_rmax(gtom_lib, cuda, impl, rmax):
    rng = np.random.default_rng(7)
    n, P = 16, 32
    vol = noisy_volume(rng, n, P)
    mats = O.matrices_f64(random_angles(rng, 10), 2.0).astype(np.float32)
    got = gpu_project(vol, P, n, 2, rmax, mats)
    ref = O.project(vol, P, n, rmax, mats)
    assert rel_l2(got, ref) <= 1e-5
    assert np.array_equal(got == 0, ref == 0) or rmax == 0


def test_project_angles_overload_equals_matrix_overload(gtom_lib, cuda, impl):
    from gtom_b200 import d_rlnProject, matrices_from_angles
    rng = np.random.default_rng(8)
    n, P, batch = 32, 64, 25
    vol = noisy_volume(rng, n, P)
    ang = random_angles(rng, batch)
    e = (n // 2 + 1) * n
    a = torch.zeros(batch * e, dtype=torch.complex64, device="cuda")
    b = torch.zeros_like(a)
    dv = cu(vol).reshape(-1)
    d_rlnProject(dv, (P, P, P), a, (n, n, 1), ang, 2.0, batch)
    d_rlnProject(dv, (P, P, P), b, (n, n, 1), n // 2, cu(matrices_from_angles(ang, 2.0)).reshape(-1), batch)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    ref = O.project(vol, P, n, n // 2, O.matrices_f64(ang, 2.0).astype(np.float32))
    assert rel_l2(a.cpu().numpy().reshape(batch, e), ref) <= 1e-5


@pytest.mark.parametrize("name", ["project_2d", "project_2d_rmax", "project_3d"])
def test_project_matches_reference_golden(gtom_lib, cuda, impl, name):
    g = load_golden(name)
    P, n, nd, rmax = int(g["P"]), int(g["n"]), int(g["ndims"]), int(g["rmax"])
    got = gpu_project(g["volume"], P, n, nd, rmax, g["matrices"])
    assert rel_l2(got, g["proj"]) <= 1e-6
    assert np.array_equal(got == 0, g["proj"] == 0)


def test_project_texture_overload(gtom_lib, cuda):
    """Texture objects built like d_BindTextureTo3DArray (point filtering,
    wrap addressing) give the array path's result."""
    from cuda.bindings import runtime as rt
    from gtom_b200 import d_rlnProject
    rng = np.random.default_rng(9)
    n, P, batch = 16, 32, 12
    vol = noisy_volume(rng, n, P)
    mats = O.matrices_f64(random_angles(rng, batch), 2.0).astype(np.float32)
    texs, arrays = [], []
    for part in (vol.real, vol.imag):
        host = np.ascontiguousarray(part.astype(np.float32))
        desc = rt.cudaCreateChannelDesc(32, 0, 0, 0, rt.cudaChannelFormatKind.cudaChannelFormatKindFloat)[1]
        ext = rt.make_cudaExtent(P // 2 + 1, P, P)
        err, arr = rt.cudaMalloc3DArray(desc, ext, 0)
        assert err == rt.cudaError_t.cudaSuccess
        p = rt.cudaMemcpy3DParms()
        p.srcPtr = rt.make_cudaPitchedPtr(host.ctypes.data, (P // 2 + 1) * 4, P // 2 + 1, P)
        p.dstArray = arr
        p.extent = ext
        p.kind = rt.cudaMemcpyKind.cudaMemcpyHostToDevice
        assert rt.cudaMemcpy3D(p)[0] == rt.cudaError_t.cudaSuccess
        res = rt.cudaResourceDesc()
        res.resType = rt.cudaResourceType.cudaResourceTypeArray
        res.res.array.array = arr
        td = rt.cudaTextureDesc()
        td.filterMode = rt.cudaTextureFilterMode.cudaFilterModePoint
        td.readMode = rt.cudaTextureReadMode.cudaReadModeElementType
        td.normalizedCoords = 0
        td.addressMode = [rt.cudaTextureAddressMode.cudaAddressModeWrap] * 3
        err, tex = rt.cudaCreateTextureObject(res, td, None)
        assert err == rt.cudaError_t.cudaSuccess
        texs.append(int(tex))
        arrays.append(arr)
    e = (n // 2 + 1) * n
    out = torch.zeros(batch * e, dtype=torch.complex64, device="cuda")
    d_rlnProject((texs[0], texs[1]), (P, P, P), out, (n, n, 1), n // 2, cu(mats).reshape(-1), batch)
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(batch, e)
    # against the FP64 oracle, at the projector's tolerance
    ref = O.project(vol, P, n, n // 2, mats)
    assert rel_l2(got, ref) <= 1e-5
    assert np.array_equal(got == 0, ref == 0)
    arr_path = gpu_project(vol, P, n, 2, n // 2, mats)
    # Identical to the array path except where it reads x1 = P/2+1 (the next
    # row's first element) and the wrapping texture reads x = 0 of the same
    # row; those samples carry a weight |fx| <= 1e-5.
    assert rel_l2(got, arr_path) <= 1e-6
    for t in texs:
        rt.cudaDestroyTextureObject(t)
    for a in arrays:
        rt.cudaFreeArray(a)


# ------------------------------------------------------------- backproject --
def gpu_backproject(P, n, ndims, rmax, mats, projft, projw, ivol=None, nvol=1, mag=(1, 0, 0, 1),
                    ewald=0.0, dec=True, sq=False, want=(True, True)):
    from gtom_b200 import d_rlnBackproject
    nv = (P // 2 + 1) * P * P * nvol
    vf = torch.zeros(nv, dtype=torch.complex64, device="cuda") if want[0] else None
    vw = torch.zeros(nv, dtype=torch.float32, device="cuda") if want[1] else None
    d_rlnBackproject(vf, vw, (P, P, P), None if projft is None else cu(projft).reshape(-1),
                     None if projw is None else cu(projw).reshape(-1), (n, n, n if ndims == 3 else 1),
                     rmax, cu(mats).reshape(-1), None if ivol is None else cu(ivol), mag, ewald, dec, sq,
                     mats.shape[0])
    torch.cuda.synchronize()
    return (None if vf is None else vf.cpu().numpy(), None if vw is None else vw.cpu().numpy())


def oracle_backproject(P, n, ndims, rmax, mats, projft, projw, ivol=None, nvol=1, mag=(1, 0, 0, 1),
                       ewald=0.0, dec=True, sq=False, fp32=False):
    nv = (P // 2 + 1) * P * P * nvol
    vf = np.zeros(nv, np.complex64 if fp32 else np.complex128)
    vw = np.zeros(nv, np.float32 if fp32 else np.float64)
    O.backproject(vf, vw, P, projft, projw, n, rmax, mats, ivolume=ivol, magnification=mag,
                  ewaldradiussuper=ewald, decentered=dec, square=sq, ndims=ndims, fp32=fp32)
    return vf, vw


@pytest.mark.parametrize("case", [
    dict(n=16, P=32, ndims=2, batch=40),
    dict(n=32, P=64, ndims=2, batch=60),
    dict(n=64, P=128, ndims=2, batch=30),
    dict(n=16, P=33, ndims=2, batch=40, dec=False, sq=True),
    dict(n=16, P=32, ndims=2, batch=40, mag=(1.03, 0.02, -0.01, 0.97), ewald=40.0),
    dict(n=16, P=32, ndims=2, batch=40, nvol=3),
    dict(n=8, P=16, ndims=3, batch=3),
])
def test_backproject_matches_oracle(gtom_lib, cuda, impl, case):
    c = dict(dec=True, sq=False, mag=(1, 0, 0, 1), ewald=0.0, nvol=1)
    c.update(case)
    rng = np.random.default_rng(c["n"] + c["P"] + c["batch"])
    n, P, nd, batch = c["n"], c["P"], c["ndims"], c["batch"]
    mats = O.matrices_f64(random_angles(rng, batch), 2.0).astype(np.float32)
    e = O.elements_fft(n, nd)
    projft = (rng.normal(size=(batch, e)) + 1j * rng.normal(size=(batch, e))).astype(np.complex64)
    projw = rng.uniform(0.1, 1, size=(batch, e)).astype(np.float32)
    ivol = rng.integers(0, c["nvol"], batch).astype(np.int32) if c["nvol"] > 1 else None
    kw = dict(ivol=ivol, nvol=c["nvol"], mag=c["mag"], ewald=c["ewald"], dec=c["dec"], sq=c["sq"])
    gf, gw = gpu_backproject(P, n, nd, n // 2, mats, projft, projw, **kw)
    of32, ow32 = oracle_backproject(P, n, nd, n // 2, mats, projft, projw, fp32=True, **kw)
    of, ow = oracle_backproject(P, n, nd, n // 2, mats, projft, projw, **kw)
    assert rel_l2(gf, of32) <= 1e-5 and rel_l2(gw, ow32) <= 1e-5
    assert rel_l2(gf, of) <= 1e-4 and rel_l2(gw, ow) <= 1e-4


def test_backproject_null_inputs_and_outputs(gtom_lib, cuda, impl):
    rng = np.random.default_rng(11)
    n, P, batch = 16, 32, 20
    mats = O.matrices_f64(random_angles(rng, batch), 2.0).astype(np.float32)
    gf, gw = gpu_backproject(P, n, 2, n // 2, mats, None, None)
    of, ow = oracle_backproject(P, n, 2, n // 2, mats, None, None, fp32=True)
    assert rel_l2(gf, of) <= 1e-5 and rel_l2(gw, ow) <= 1e-5
    gf2, gw2 = gpu_backproject(P, n, 2, n // 2, mats, None, None, want=(False, True))
    assert gf2 is None and rel_l2(gw2, ow) <= 1e-5


def test_backproject_angles_overload(gtom_lib, cuda, impl):
    from gtom_b200 import d_rlnBackproject
    rng = np.random.default_rng(12)
    n, P, batch = 16, 32, 24
    ang = random_angles(rng, batch)
    e = O.elements_fft(n)
    projft = (rng.normal(size=(batch, e)) + 1j * rng.normal(size=(batch, e))).astype(np.complex64)
    nv = (P // 2 + 1) * P * P * 2
    ivol = rng.integers(0, 2, batch).astype(np.int32)
    vf = torch.zeros(nv, dtype=torch.complex64, device="cuda")
    vw = torch.zeros(nv, dtype=torch.float32, device="cuda")
    d_rlnBackproject(vf, vw, (P, P, P), cu(projft).reshape(-1), None, (n, n, 1), n // 2, ang, ivol,
                     (1, 0, 0, 1), 0.0, 2.0, True, False, batch)
    torch.cuda.synchronize()
    # same single-precision host matrices as the h_angles overload builds
    from gtom_b200 import matrices_from_angles
    of, ow = oracle_backproject(P, n, 2, n // 2, matrices_from_angles(ang, 2.0), projft, None,
                                ivol=ivol, nvol=2, fp32=True)
    assert rel_l2(vf.cpu().numpy(), of) <= 1e-5 and rel_l2(vw.cpu().numpy(), ow) <= 1e-5


@pytest.mark.parametrize("name", ["bp_dec", "bp_cen_sq_mag", "bp_3d"])
def test_backproject_matches_reference_golden(gtom_lib, cuda, impl, name):
    g = load_golden(name)
    P, n, nd = int(g["P"]), int(g["n"]), int(g["ndims"])
    ivol = g["ivolume"] if g["ivolume"].size else None
    gf, gw = gpu_backproject(P, n, nd, int(g["rmax"]), g["matrices"], g["projft"], g["projw"], ivol=ivol,
                             nvol=int(g["nvol"]), mag=tuple(g["mag"]), ewald=float(g["ewald"]),
                             dec=bool(g["decentered"]), sq=bool(g["square"]))
    assert rel_l2(gf, g["volft"]) <= 1e-5
    assert rel_l2(gw, g["volw"]) <= 1e-5


# ---------------------------------------------------------------- gridding --
def gpu_gridding(dataft, weight, ori, dpad, pad, iters):
    from gtom_b200 import d_ReconstructGridding
    out = torch.zeros(ori ** 3, dtype=torch.float32, device="cuda")
    d_ReconstructGridding(cu(dataft).reshape(-1), cu(weight).reshape(-1), out, (ori, ori, ori),
                          (dpad, dpad, dpad), pad, 0, 0, iters)
    torch.cuda.synchronize()
    return out.cpu().numpy().reshape(ori, ori, ori)


def make_gridding_input(rng, ori, pad, nproj):
    P = ori * pad
    D = P + 1
    vol = blob_volume_ft(rng, ori, P, 8)
    mats = O.matrices_f64(random_angles(rng, nproj), float(pad)).astype(np.float32)
    proj = O.project(vol, P, ori, ori // 2, mats).astype(np.complex64)
    nv = (D // 2 + 1) * D * D
    data, w = np.zeros(nv, np.complex64), np.zeros(nv, np.float32)
    O.backproject(data, w, D, proj, None, ori, ori // 2, mats, decentered=False, fp32=True)
    return data.reshape(D, D, D // 2 + 1), w.reshape(D, D, D // 2 + 1), D


@pytest.mark.parametrize("ori,pad,iters", [(16, 2, 10), (32, 2, 10), (16, 2, 0), (12, 3, 3), (32, 2, 1)])
def test_gridding_matches_oracle(gtom_lib, cuda, ori, pad, iters):
    rng = np.random.default_rng(ori * 10 + pad + iters)
    data, w, D = make_gridding_input(rng, ori, pad, 400)
    got = gpu_gridding(data, w, ori, D, pad, iters)
    ref = O.reconstruct_gridding(data, w, ori, (D, D, D), pad, iterations=iters)
    assert rel_l2(got, ref) <= 1e-4
    assert np.all(fsc(got, ref) >= 0.999)


@pytest.mark.parametrize("name", ["grid_it10", "grid_it0", "grid_it3_pad3"])
def test_gridding_matches_reference_golden(gtom_lib, cuda, name):
    g = load_golden(name)
    ori, pad, dpad, iters = int(g["ori"]), int(g["pad"]), int(g["dimspadded"]), int(g["iterations"])
    nv = (dpad // 2 + 1) * dpad * dpad
    got = gpu_gridding(g["dataft"][:nv], g["weight"][:nv], ori, dpad, pad, iters)
    ref = g["reconstructed"]
    assert np.all(fsc(got, ref) >= 0.999)
    assert rel_l2(got, ref) <= 1e-4


def test_gridding_tolerance_variant(gtom_lib, cuda):
    from gtom_b200 import reconstruct_gridding_tol
    rng = np.random.default_rng(21)
    ori, pad = 16, 2
    data, w, D = make_gridding_input(rng, ori, pad, 300)
    out = torch.zeros(ori ** 3, dtype=torch.float32, device="cuda")
    it, ch = reconstruct_gridding_tol(cu(data).reshape(-1), cu(w).reshape(-1), out, (ori,) * 3, (D,) * 3,
                                      pad, max_iterations=10, tolerance=0.0)
    assert it == 10
    ref10 = gpu_gridding(data, w, ori, D, pad, 10)
    assert np.array_equal(out.cpu().numpy().reshape(ref10.shape), ref10)
    # the gridding iteration converges slowly (change ~ 1/iteration), so the
    # early exit is exercised at a loose tolerance
    it, ch = reconstruct_gridding_tol(cu(data).reshape(-1), cu(w).reshape(-1), out, (ori,) * 3, (D,) * 3,
                                      pad, max_iterations=300, tolerance=5e-3)
    assert 10 < it < 300 and ch <= 5e-3
