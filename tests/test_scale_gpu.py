"""Parity with the reference itself at the benchmark's sizes.

The reference's own CUDA implementation (oracle/_ref/libgtomref.so, compiled
from its sources) and this library run on the same seeded inputs:

* the small plain configuration in full: a 64^3 volume of 200 Gaussian
  blobs, padding 2, 1 000 slices at uniform SO(3) orientations, projected,
  inserted with unit CTF and weights, and reconstructed with 10 gridding
  iterations;
* the single-particle configuration at 256^3 (2 000 blobs, padding 2,
  P = 512): 5 000 CTF-weighted noisy particles from the benchmark's
  orientation mixture, projected, inserted (the central bricks then take
  more pairs than one work item holds, so the flush that adds several items
  into one brick with L2 reductions runs), and reconstructed at P = 512;
* several work items per brick forced at a small size (pairs per item cut
  to 16), checked against the oracle's single-precision port.

Tolerances (relative L2): projections <= 1e-6 against the reference (the
same single-precision arithmetic; zeros identical); backprojection <= 1e-5
against the reference; reconstructions <= 1e-4 against the reference with
FSC >= 0.999 in every shell.  The reference's insertion sums with FP32
atomics in whatever order its threads arrive, so it differs from itself run
to run: `test_reference_noise_floor` measures that floor (two runs of the
reference on the same inputs) on the small configuration and on a 128^3
sub-tomogram-sized case, and the tests print it beside the library's
distance from the reference.
"""
import math

import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import refcuda
from tests.helpers import fsc, rel_l2

pytestmark = pytest.mark.gpu

PAD = 2


@pytest.fixture(scope="module")
def ref():
    if not refcuda.available():
        pytest.skip("the reference build (oracle/_ref/libgtomref.so) is not present")
    return refcuda.lib()


def vol_buffer(ft):
    """The decentred volume followed by 64 zeros (the reference projector's
    x1 = P/2+1 read can touch one element past the end)."""
    buf = torch.zeros(ft.numel() + 64, dtype=torch.complex64, device="cuda")
    buf[:ft.numel()] = ft.reshape(-1)
    return buf


def ref_project(ref, vbuf, P, n, mats, rmax):
    batch = mats.shape[0]
    out = torch.empty(batch * (n // 2 + 1) * n, dtype=torch.complex64, device="cuda")
    refcuda.check(ref.ref_project(vbuf.data_ptr(), P, out.data_ptr(), n, 2, rmax, mats.data_ptr(), batch),
                  "reference project")
    return out


def ref_backproject(ref, D, n, rmax, mats, data, wts):
    nv = (D // 2 + 1) * D * D
    vf = torch.zeros(nv, dtype=torch.complex64, device="cuda")
    vw = torch.zeros(nv, dtype=torch.float32, device="cuda")
    refcuda.check(ref.ref_backproject(vf.data_ptr(), vw.data_ptr(), D, data.data_ptr(),
                                      None if wts is None else wts.data_ptr(), n, 2, rmax, mats.data_ptr(),
                                      None, 1, 0, 0, 1, 0.0, 0, 0, mats.shape[0]), "reference backproject")
    return vf, vw


def ref_gridding(ref, vf, vw, ori, D, iters=10):
    out = torch.empty(ori ** 3, dtype=torch.float32, device="cuda")
    refcuda.check(ref.ref_reconstruct_gridding(vf.data_ptr(), vw.data_ptr(), out.data_ptr(), ori, D, PAD, iters,
                                               1.9, 0, 15.0), "reference gridding")
    return out


def our_project(vbuf, nv_in, P, n, mats, rmax):
    from gtom_b200 import d_rlnProject
    batch = mats.shape[0]
    out = torch.full((batch * (n // 2 + 1) * n,), complex(math.nan, math.nan), dtype=torch.complex64,
                     device="cuda")
    d_rlnProject(vbuf[:nv_in], (P, P, P), out, (n, n, 1), rmax, mats.reshape(-1), batch)
    return out


def our_backproject(D, n, rmax, mats, data, wts):
    from gtom_b200 import d_rlnBackproject
    nv = (D // 2 + 1) * D * D
    vf = torch.zeros(nv, dtype=torch.complex64, device="cuda")
    vw = torch.zeros(nv, dtype=torch.float32, device="cuda")
    d_rlnBackproject(vf, vw, (D, D, D), data, wts, (n, n, 1), rmax, mats.reshape(-1), None, (1, 0, 0, 1), 0.0,
                     False, False, mats.shape[0])
    return vf, vw


def our_gridding(vf, vw, ori, D, iters=10):
    from gtom_b200 import d_ReconstructGridding
    out = torch.empty(ori ** 3, dtype=torch.float32, device="cuda")
    d_ReconstructGridding(vf, vw, out, (ori,) * 3, (D,) * 3, PAD, 0, 0, iters)
    return out


def cube(t, n):
    return t.cpu().numpy().reshape(n, n, n)


def check_reconstruction(got, want, n, tol=1e-4):
    g, w = cube(got, n), cube(want, n)
    err = rel_l2(g, w)
    shells = fsc(g, w)
    assert err <= tol, f"reconstruction rel L2 {err:.3e}"
    assert np.all(shells >= 0.999), f"min FSC {shells.min():.6f}"
    return err, float(shells.min())


def blob_workload(n, nblobs, radius, count, seed, uniform=True, ctf=False, snr=None):
    """Volume, matrices (the reference's host expression) and, with ctf,
    CTF-weighted noisy particles with CTF^2 weights, on the GPU."""
    from gtom_b200 import d_rlnProject, synth
    rng = np.random.default_rng(seed)
    P = n * PAD
    vol = synth.blob_volume(n, nblobs, seed, "cuda", radius_frac=radius / n)
    ft = synth.padded_half_ft(vol, PAD).reshape(-1)
    del vol
    ang = (synth.vmf_mixture_angles(rng, count, uniform_frac=1.0) if uniform
           else synth.vmf_mixture_angles(rng, count))
    mats = torch.from_numpy(refcuda.matrices(ang, float(PAD))).cuda()
    vbuf = vol_buffer(ft)
    out = dict(vbuf=vbuf, nv=ft.numel(), mats=mats)
    if ctf:
        e = (n // 2 + 1) * n
        proj = torch.empty(count * e, dtype=torch.complex64, device="cuda")
        d_rlnProject(ft, (P, P, P), proj, (n, n, 1), n // 2, mats.reshape(-1), count)
        proj = proj.reshape(count, e)
        df = torch.from_numpy(rng.uniform(0.5, 3.0, count).astype(np.float32)).cuda()
        da = torch.from_numpy(rng.uniform(0.0, 0.1, count).astype(np.float32)).cuda()
        aa = torch.from_numpy(rng.uniform(0.0, np.pi, count).astype(np.float32)).cuda()
        c = synth.ctf_half(n, df, da, aa).reshape(count, e)
        disk = synth.in_disk_mask(n, n // 2, "cuda").reshape(-1)
        sig = proj * c
        pw = (sig.abs() ** 2 * disk).sum(1, keepdim=True) / disk.sum()
        gen = torch.Generator(device="cuda")
        gen.manual_seed(seed)
        noise = torch.complex(torch.randn((count, e), device="cuda", generator=gen),
                              torch.randn((count, e), device="cuda", generator=gen)) * torch.sqrt(pw / snr / 2)
        out["data"] = ((sig + noise) * c).contiguous().reshape(-1)
        out["wts"] = (c * c).contiguous().reshape(-1)
    return out


def test_small_configuration_in_full_against_reference(gtom_lib, cuda, ref):
    """64^3, 200 blobs within radius 28, padding 2, 1 000 uniform slices:
    project -> backproject (unit CTF and weights) -> 10 gridding iterations,
    each stage against the reference on the same inputs."""
    n, rmax = 64, 32
    P, D = n * PAD, n * PAD + 1
    w = blob_workload(n, 200, 28.0, 1000, 1001)
    mats = w["mats"]
    p_ref = ref_project(ref, w["vbuf"], P, n, mats, rmax)
    p_our = our_project(w["vbuf"], w["nv"], P, n, mats, rmax)
    torch.cuda.synchronize()
    a, b = p_our.cpu().numpy(), p_ref.cpu().numpy()
    assert rel_l2(a, b) <= 1e-6
    assert np.array_equal(a == 0, b == 0)

    vf_r, vw_r = ref_backproject(ref, D, n, rmax, mats, p_ref, None)
    vf_o, vw_o = our_backproject(D, n, rmax, mats, p_ref, None)
    torch.cuda.synchronize()
    e_f = rel_l2(vf_o.cpu().numpy(), vf_r.cpu().numpy())
    e_w = rel_l2(vw_o.cpu().numpy(), vw_r.cpu().numpy())
    assert e_f <= 1e-5 and e_w <= 1e-5, (e_f, e_w)

    rec_r = ref_gridding(ref, vf_r, vw_r, n, D)
    rec_o = our_gridding(vf_o, vw_o, n, D)
    rec_o_on_ref = our_gridding(vf_r, vw_r, n, D)
    torch.cuda.synchronize()
    err, fmin = check_reconstruction(rec_o, rec_r, n)
    err2, _ = check_reconstruction(rec_o_on_ref, rec_r, n)
    print(f"small config vs reference: backprojection {e_f:.2e} / {e_w:.2e}, "
          f"reconstruction {err:.2e} (min FSC {fmin:.7f}), gridding alone {err2:.2e}")


def test_single_particle_256_against_reference(gtom_lib, cuda, ref):
    """256^3, 2 000 blobs, padding 2 (P = 512), 5 000 CTF-weighted particles
    at SNR 0.05 from the benchmark's orientation mixture: projections,
    accumulators and the P = 512 reconstruction against the reference."""
    n, rmax, count = 256, 128, 5000
    P, D = n * PAD, n * PAD + 1
    w = blob_workload(n, 2000, 0.44 * n, count, 1002, uniform=False, ctf=True, snr=0.05)
    mats = w["mats"]
    p_ref = ref_project(ref, w["vbuf"], P, n, mats, rmax)
    p_our = our_project(w["vbuf"], w["nv"], P, n, mats, rmax)
    torch.cuda.synchronize()
    assert torch.equal(torch.isnan(p_our), torch.zeros_like(p_our, dtype=torch.bool))
    a, b = p_our.cpu().numpy(), p_ref.cpu().numpy()
    del p_our, p_ref
    assert rel_l2(a, b) <= 1e-6
    assert np.array_equal(a == 0, b == 0)
    del a, b

    vf_r, vw_r = ref_backproject(ref, D, n, rmax, mats, w["data"], w["wts"])
    vf_o, vw_o = our_backproject(D, n, rmax, mats, w["data"], w["wts"])
    torch.cuda.synchronize()
    e_f = rel_l2(vf_o.cpu().numpy(), vf_r.cpu().numpy())
    e_w = rel_l2(vw_o.cpu().numpy(), vw_r.cpu().numpy())
    assert e_f <= 1e-5 and e_w <= 1e-5, (e_f, e_w)

    rec_r = ref_gridding(ref, vf_r, vw_r, n, D)
    rec_o = our_gridding(vf_o, vw_o, n, D)
    torch.cuda.synchronize()
    err, fmin = check_reconstruction(rec_o, rec_r, n)
    print(f"256^3 vs reference: backprojection {e_f:.2e} / {e_w:.2e}, reconstruction {err:.2e} "
          f"(min FSC {fmin:.7f})")


@pytest.mark.parametrize("path", ["segment", "brick"])
def test_several_items_per_brick(gtom_lib, cuda, path):
    """Work items cut to 16 pairs, so every brick crossed by more than 16 of
    the 300 slices is added by several items with L2 reductions: the result
    equals the oracle's single-precision port."""
    from gtom_b200 import set_brick_tuning, set_path
    from tests.synthdata import random_angles
    rng = np.random.default_rng(77)
    n, P, batch = 48, 96, 300
    mats = O.matrices_f64(random_angles(rng, batch), 2.0).astype(np.float32)
    e = O.elements_fft(n)
    projft = (rng.normal(size=(batch, e)) + 1j * rng.normal(size=(batch, e))).astype(np.complex64)
    projw = rng.uniform(0.1, 1, size=(batch, e)).astype(np.float32)
    set_path("backproject", path)
    set_brick_tuning("backproject", edge=12, chunk=16)
    try:
        for dec in (True, False):
            V = P if dec else P + 1
            from gtom_b200 import d_rlnBackproject
            nv = (V // 2 + 1) * V * V
            vf = torch.zeros(nv, dtype=torch.complex64, device="cuda")
            vw = torch.zeros(nv, dtype=torch.float32, device="cuda")
            d_rlnBackproject(vf, vw, (V, V, V), torch.from_numpy(projft).cuda().reshape(-1),
                             torch.from_numpy(projw).cuda().reshape(-1), (n, n, 1), n // 2,
                             torch.from_numpy(mats).cuda().reshape(-1), None, (1, 0, 0, 1), 0.0, dec, False, batch)
            torch.cuda.synchronize()
            of, ow = np.zeros(nv, np.complex64), np.zeros(nv, np.float32)
            O.backproject(of, ow, V, projft, projw, n, n // 2, mats, decentered=dec, fp32=True)
            assert rel_l2(vf.cpu().numpy(), of) <= 1e-5
            assert rel_l2(vw.cpu().numpy(), ow) <= 1e-5
    finally:
        set_brick_tuning("backproject")
        set_path("backproject", "auto")


def test_reference_noise_floor(gtom_lib, cuda, ref):
    """The reference against itself: two runs of its insertion (FP32 atomics
    in arrival order) on the same inputs, then its gridding of each, on the
    small configuration and on a 128^3 case (padding 2, 2 000 CTF-weighted
    particles).  The library's distance from the reference is printed beside
    the floor; the library must stay within max(tolerance, floor)."""
    rows = []
    for n, nblobs, count, ctf in ((64, 200, 1000, False), (128, 500, 2000, True)):
        rmax, D = n // 2, n * PAD + 1
        w = blob_workload(n, nblobs, 0.44 * n, count, 2000 + n, uniform=not ctf, ctf=ctf, snr=0.1)
        mats = w["mats"]
        if ctf:
            data, wts = w["data"], w["wts"]
        else:
            data, wts = ref_project(ref, w["vbuf"], n * PAD, n, mats, rmax), None
        r1 = ref_backproject(ref, D, n, rmax, mats, data, wts)
        r2 = ref_backproject(ref, D, n, rmax, mats, data, wts)
        ours = our_backproject(D, n, rmax, mats, data, wts)
        g1, g2 = ref_gridding(ref, *r1, n, D), ref_gridding(ref, *r2, n, D)
        go = our_gridding(*ours, n, D)
        torch.cuda.synchronize()
        floor_bp = rel_l2(r2[0].cpu().numpy(), r1[0].cpu().numpy())
        floor_rec = rel_l2(cube(g2, n), cube(g1, n))
        ours_bp = rel_l2(ours[0].cpu().numpy(), r1[0].cpu().numpy())
        ours_rec = rel_l2(cube(go, n), cube(g1, n))
        rows.append((n, floor_bp, floor_rec, ours_bp, ours_rec))
        assert ours_bp <= max(1e-5, 4 * floor_bp)
        assert ours_rec <= max(1e-4, 4 * floor_rec)
        assert np.all(fsc(cube(go, n), cube(g1, n)) >= 0.999)
    for n, fb, fr, ob, orr in rows:
        print(f"{n}^3: reference vs itself: backprojection {fb:.2e}, reconstruction {fr:.2e}; "
              f"library vs reference: {ob:.2e}, {orr:.2e}")


def test_general_geometry_256_against_reference(gtom_lib, cuda, ref):
    """The general insertion at 256^3 against the reference: anisotropic
    magnification (1.2 % / 0.7 % with shear), the Ewald curvature of 300 kV
    electrons at 1 A/pixel (sphere radius 256 / 0.0197 pixels, supersampled
    by 2) and two target volumes (half-maps) chosen per particle, 3 000
    CTF-weighted particles into centred 513^3 accumulators.  The library
    takes its row-segment kernel here (volume beyond L2, batch >= 300)."""
    n, rmax, count = 256, 128, 3000
    D = n * PAD + 1
    w = blob_workload(n, 2000, 0.44 * n, count, 1005, uniform=False, ctf=True, snr=0.05)
    mats = w["mats"]
    iv = torch.from_numpy(np.random.default_rng(9).integers(0, 2, count).astype(np.int32)).cuda()
    mag = (1.012, 0.004, -0.006, 0.993)
    ewald = 2.0 * 256.0 / 0.0197
    nv = (D // 2 + 1) * D * D * 2
    vf_r = torch.zeros(nv, dtype=torch.complex64, device="cuda")
    vw_r = torch.zeros(nv, dtype=torch.float32, device="cuda")
    refcuda.check(ref.ref_backproject(vf_r.data_ptr(), vw_r.data_ptr(), D, w["data"].data_ptr(), w["wts"].data_ptr(),
                                      n, 2, rmax, mats.data_ptr(), iv.data_ptr(), *mag, ewald, 0, 0, count),
                  "reference backproject")
    from gtom_b200 import d_rlnBackproject
    vf_o = torch.zeros_like(vf_r)
    vw_o = torch.zeros_like(vw_r)
    d_rlnBackproject(vf_o, vw_o, (D, D, D), w["data"], w["wts"], (n, n, 1), rmax, mats.reshape(-1), iv, mag, ewald,
                     False, False, count)
    torch.cuda.synchronize()
    e_f = rel_l2(vf_o.cpu().numpy(), vf_r.cpu().numpy())
    e_w = rel_l2(vw_o.cpu().numpy(), vw_r.cpu().numpy())
    print(f"general geometry 256^3 vs reference: {e_f:.2e} / {e_w:.2e}")
    assert e_f <= 1e-5 and e_w <= 1e-5, (e_f, e_w)
