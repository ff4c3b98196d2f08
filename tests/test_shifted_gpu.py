"""d_rlnProjectShifted / d_rlnBackprojectShifted on the GPU against the
reference's own results (tests/golden/) and the float64 oracle, through the
matrix and h_angles overloads and the texture overload."""
import numpy as np
import pytest
import torch

import gtom_b200 as G
from oracle import oracle as O
from tests.helpers import load_golden, rel_l2

pytestmark = pytest.mark.gpu


def cu(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    return (t if dtype is None else t.to(dtype)).cuda()


@pytest.fixture(params=["auto", "segment"])
def path(request, gtom_lib):
    """The small golden batches take the direct kernels under "auto"; forcing
    "segment" runs the same cases through the brick-major segment kernels."""
    G.set_path("project", request.param)
    G.set_path("backproject", request.param)
    yield request.param
    G.set_path("project", "auto")
    G.set_path("backproject", "auto")


@pytest.mark.parametrize("name", ["project_shifted_2d", "project_shifted_3d"])
def test_project_shifted_matches_reference(gtom_lib, cuda, name, path):
    g = load_golden(name)
    P, n, nd, rmax = int(g["P"]), int(g["n"]), int(g["ndims"]), int(g["rmax"])
    batch = g["matrices"].shape[0]
    dims = (n, n, n if nd == 3 else 1)
    e = O.elements_fft(n, nd)
    vol = cu(g["volume"]).reshape(-1)
    out = torch.full((batch * e,), complex(np.nan, np.nan), dtype=torch.complex64, device="cuda")
    G.d_rlnProjectShifted(vol, (P, P, P), out, dims, rmax, cu(g["matrices"]).reshape(-1),
                          cu(g["shifts"]).reshape(-1), cu(g["globalweights"]), batch)
    got = out.cpu().numpy().reshape(batch, e)
    assert rel_l2(got, g["proj"]) <= 1e-6  # same arithmetic, same fast sine/cosine
    want = O.project_shifted(g["volume"], P, n, rmax, g["matrices"], g["shifts"], g["globalweights"], ndims=nd)
    assert rel_l2(got, want) <= 1e-5
    if nd == 2:  # h_angles overload: pixels in, rmax = n/2, FP32 host matrices
        out2 = torch.zeros_like(out)
        G.d_rlnProjectShifted(vol, (P, P, P), out2, dims, g["angles"], g["shifts_px"], g["globalweights"], 2.0,
                              batch)
        want2 = O.project_shifted(g["volume"], P, n, n // 2, O.matrices_f64(g["angles"], 2.0).astype(np.float32),
                                  O.scaled_shifts(g["shifts_px"], n), g["globalweights"])
        assert rel_l2(out2.cpu().numpy().reshape(batch, e), want2) <= 1e-5


def test_project_shifted_texture_overload(gtom_lib, cuda):
    from cuda.bindings import runtime as rt
    g = load_golden("project_shifted_2d")
    P, n, rmax = int(g["P"]), int(g["n"]), int(g["rmax"])
    batch = g["matrices"].shape[0]
    vol = g["volume"].reshape(P, P, P // 2 + 1)
    texs, arrays = [], []
    for part in (np.ascontiguousarray(vol.real.astype(np.float32)), np.ascontiguousarray(vol.imag.astype(np.float32))):
        desc = rt.cudaCreateChannelDesc(32, 0, 0, 0, rt.cudaChannelFormatKind.cudaChannelFormatKindFloat)[1]
        err, arr = rt.cudaMalloc3DArray(desc, rt.make_cudaExtent(P // 2 + 1, P, P), 0)
        assert err == rt.cudaError_t.cudaSuccess
        p = rt.cudaMemcpy3DParms()
        p.srcPtr = rt.make_cudaPitchedPtr(part.ctypes.data, (P // 2 + 1) * 4, P // 2 + 1, P)
        p.dstArray = arr
        p.extent = rt.make_cudaExtent(P // 2 + 1, P, P)
        p.kind = rt.cudaMemcpyKind.cudaMemcpyHostToDevice
        assert rt.cudaMemcpy3D(p)[0] == rt.cudaError_t.cudaSuccess
        res = rt.cudaResourceDesc()
        res.resType = rt.cudaResourceType.cudaResourceTypeArray
        res.res.array.array = arr
        td = rt.cudaTextureDesc()
        td.addressMode = [rt.cudaTextureAddressMode.cudaAddressModeWrap] * 3
        td.filterMode = rt.cudaTextureFilterMode.cudaFilterModePoint
        td.readMode = rt.cudaTextureReadMode.cudaReadModeElementType
        td.normalizedCoords = 0
        err, tex = rt.cudaCreateTextureObject(res, td, None)
        assert err == rt.cudaError_t.cudaSuccess
        texs.append(int(tex))
        arrays.append(arr)
    e = O.elements_fft(n)
    out = torch.zeros(batch * e, dtype=torch.complex64, device="cuda")
    G.d_rlnProjectShifted((texs[0], texs[1]), (P, P, P), out, (n, n, 1), rmax, cu(g["matrices"]).reshape(-1),
                          cu(g["shifts"]).reshape(-1), cu(g["globalweights"]), batch)
    torch.cuda.synchronize()
    for t, a in zip(texs, arrays):
        rt.cudaDestroyTextureObject(t)
        rt.cudaFreeArray(a)
    # as the array path except where that reads x1 = P/2+1 (the next row's
    # first element) and the wrapping texture reads x = 0 of the same row;
    # those samples carry a weight |fx| <= 1e-5
    want = O.project_shifted(g["volume"], P, n, rmax, g["matrices"], g["shifts"], g["globalweights"])
    assert rel_l2(out.cpu().numpy().reshape(batch, e), want) <= 1e-5


@pytest.mark.parametrize("name", ["bp_shifted_2d", "bp_shifted_3d"])
def test_backproject_shifted_matches_reference(gtom_lib, cuda, name, path):
    g = load_golden(name)
    V, n, nd, rmax = int(g["V"]), int(g["n"]), int(g["ndims"]), int(g["rmax"])
    batch = g["matrices"].shape[0]
    nv = (V // 2 + 1) * V * V
    vf = torch.zeros(nv, dtype=torch.complex64, device="cuda")
    vw = torch.zeros(nv, dtype=torch.float32, device="cuda")
    G.d_rlnBackprojectShifted(vf, vw, (V, V, V), cu(g["projft"]).reshape(-1), cu(g["projw"]).reshape(-1),
                              (n, n, n if nd == 3 else 1), rmax, cu(g["matrices"]).reshape(-1),
                              cu(g["shifts"]).reshape(-1), cu(g["globalweights"]), batch)
    got_f, got_w = vf.cpu().numpy(), vw.cpu().numpy()
    assert rel_l2(got_f, g["volft"]) <= 1e-6  # float atomics: order of the sums only
    assert rel_l2(got_w, g["volw"]) <= 1e-6
    if nd == 2:  # h_angles overload
        vf2 = torch.zeros_like(vf)
        vw2 = torch.zeros_like(vw)
        G.d_rlnBackprojectShifted(vf2, vw2, (V, V, V), cu(g["projft"]).reshape(-1), cu(g["projw"]).reshape(-1),
                                  (n, n, 1), rmax, g["angles"], g["shifts_px"], g["globalweights"], 2.0, batch)
        of = np.zeros(nv, np.complex128)
        ow = np.zeros(nv, np.float64)
        O.backproject_shifted(of, ow, V, g["projft"], g["projw"], n, rmax,
                              O.matrices_f64(g["angles"], 2.0).astype(np.float32),
                              O.scaled_shifts(g["shifts_px"], n), g["globalweights"])
        assert rel_l2(vf2.cpu().numpy(), of) <= 1e-5
        assert rel_l2(vw2.cpu().numpy(), ow) <= 1e-5


def test_shifted_rejects_bad_dims(gtom_lib, cuda):
    v = torch.zeros(12, dtype=torch.complex64, device="cuda")
    w = torch.zeros(12, dtype=torch.float32, device="cuda")
    m = torch.zeros(9, dtype=torch.float32, device="cuda")
    with pytest.raises(G.GtomError):  # a 2D volume: the reference throws
        G.d_rlnBackprojectShifted(v, w, (4, 4, 1), None, None, (4, 4, 1), 2, m, m[:3], m[:1], 1)


@pytest.mark.parametrize("V,sheared", [(129, False), (128, False), (129, True)])
def test_shifted_segment_paths_match_direct(gtom_lib, cuda, V, sheared):
    """The segment kernels of both shifted operators against their direct
    kernels on a batch above the brick threshold: the projector bit for bit
    (same arithmetic, same fast sine and cosine), the insertion to FP32
    rounding of the sums (odd and even centred volumes, sheared matrices)."""
    from tests.synthdata import blob_volume_ft, random_angles
    rng = np.random.default_rng(V + 7 * sheared)
    n, batch = 64, 160
    e = (n // 2 + 1) * n
    m = G.matrices_from_angles(random_angles(rng, batch), 2.0).reshape(batch, 9)
    if sheared:
        m = ((m + rng.normal(scale=0.3, size=m.shape)) * 0.8).astype(np.float32)
    shifts = rng.normal(scale=0.2, size=(batch, 3)).astype(np.float32)
    gws = rng.uniform(0.5, 1.5, batch).astype(np.float32)
    P = 2 * n
    vol = cu(blob_volume_ft(rng, n, P, 12).astype(np.complex64)).reshape(-1)
    outs = {}
    try:
        for p in ("direct", "segment"):
            G.set_path("project", p)
            out = torch.full((batch * e,), complex(np.nan, np.nan), dtype=torch.complex64, device="cuda")
            G.d_rlnProjectShifted(vol, (P, P, P), out, (n, n, 1), n // 2, cu(m).reshape(-1), cu(shifts).reshape(-1),
                                  cu(gws), batch)
            torch.cuda.synchronize()
            outs[p] = out
        assert torch.equal(outs["direct"], outs["segment"])
        pf = (rng.normal(size=(batch, e)) + 1j * rng.normal(size=(batch, e))).astype(np.complex64)
        pw = rng.uniform(0.1, 1, size=(batch, e)).astype(np.float32)
        nv = (V // 2 + 1) * V * V
        res = {}
        for p in ("direct", "segment"):
            G.set_path("backproject", p)
            vf = torch.zeros(nv, dtype=torch.complex64, device="cuda")
            vw = torch.zeros(nv, dtype=torch.float32, device="cuda")
            G.d_rlnBackprojectShifted(vf, vw, (V, V, V), cu(pf).reshape(-1), cu(pw).reshape(-1), (n, n, 1), n // 2,
                                      cu(m).reshape(-1), cu(shifts).reshape(-1), cu(gws), batch)
            torch.cuda.synchronize()
            res[p] = (vf.cpu().numpy(), vw.cpu().numpy())
        assert rel_l2(res["segment"][0], res["direct"][0]) <= 1e-6
        assert rel_l2(res["segment"][1], res["direct"][1]) <= 1e-6
        assert np.array_equal(res["segment"][1] == 0, res["direct"][1] == 0)
    finally:
        G.set_path("project", "auto")
        G.set_path("backproject", "auto")
