"""Generates the golden fixtures of tests/golden/ from the reference itself.

Runs the reference's own CUDA implementation (oracle/_ref/libgtomref.so,
compiled from the reference sources by `make -C oracle ref`) on seeded
inputs and stores inputs and outputs as compressed .npz files:

    python tests/golden/make_golden.py [outdir]      # needs a GPU

The fixtures pin the CPU oracle (tests/test_oracle_golden.py) and the CUDA
library (tests/test_parity_gpu.py) to the reference's results.  Buffers
handed to the reference projector are over-allocated by 64 elements because
its x1 = P/2+1 read (src/Relion/Project.cu:155) can touch one element past
the end of the volume; the extra elements are zero and never reach a result
that the fixtures keep.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from oracle import refcuda  # noqa: E402
from tests.synthdata import blob_volume_ft, random_angles  # noqa: E402

REF = refcuda.lib()
_ok = refcuda.check


def dev(a: np.ndarray, extra: int = 0) -> torch.Tensor:
    flat = torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1).copy())
    t = torch.zeros(flat.numel() + extra * 8, dtype=torch.uint8, device="cuda")
    t[: flat.numel()] = flat.cuda()
    return t


def host(t: torch.Tensor, dtype, count: int) -> np.ndarray:
    return t.cpu().numpy().view(dtype)[:count].copy()


def gen_project(out: Path, rng) -> None:
    for name, n, ndims, batch, rmax in (("project_2d", 16, 2, 24, 8), ("project_2d_rmax", 16, 2, 12, 5),
                                        ("project_3d", 8, 3, 3, 4)):
        P = 2 * n
        vol = blob_volume_ft(rng, n, P, 12)
        vol = (vol + (rng.normal(size=vol.shape) + 1j * rng.normal(size=vol.shape)).astype(np.complex64) * 0.05 * np.abs(vol).max()).astype(np.complex64)
        ang = random_angles(rng, batch)
        mats = O.matrices_f64(ang, 2.0).astype(np.float32)
        e = O.elements_fft(n, ndims)
        dv = dev(vol, extra=64)
        dm = dev(mats)
        dp = torch.zeros(e * batch * 8, dtype=torch.uint8, device="cuda")
        _ok(REF.ref_project(dv.data_ptr(), P, dp.data_ptr(), n, ndims, rmax, dm.data_ptr(), batch), name)
        proj = host(dp, np.complex64, e * batch).reshape(batch, e)
        dp2 = torch.zeros_like(dp)
        _ok(REF.ref_project_angles(dv.data_ptr(), P, dp2.data_ptr(), n, ndims, ang.ctypes.data, 2.0, batch),
            name + "_angles")
        proj_ang = host(dp2, np.complex64, e * batch).reshape(batch, e)
        np.savez_compressed(out / f"{name}.npz", volume=vol, P=P, n=n, ndims=ndims, rmax=rmax,
                            angles=ang, matrices=mats, proj=proj, proj_angles=proj_ang)
        print(name, np.abs(proj).max())


def gen_backproject(out: Path, rng) -> None:
    cases = (
        # name, n, ndims, P, batch, decentred, square, mag, ewaldradius(super), nvol
        ("bp_dec", 16, 2, 32, 40, True, False, (1, 0, 0, 1), 0.0, 1),
        ("bp_cen_sq_mag", 16, 2, 33, 40, False, True, (1.03, 0.02, -0.01, 0.97), 40.0, 2),
        ("bp_3d", 8, 3, 16, 3, True, False, (1, 0, 0, 1), 0.0, 1),
    )
    for name, n, ndims, P, batch, dec, sq, mag, ewald, nvol in cases:
        ang = random_angles(rng, batch)
        mats = O.matrices_f64(ang, 2.0).astype(np.float32)
        e = O.elements_fft(n, ndims)
        projft = (rng.normal(size=(batch, e)) + 1j * rng.normal(size=(batch, e))).astype(np.complex64)
        projw = rng.uniform(0.1, 1.0, size=(batch, e)).astype(np.float32)
        ivol = rng.integers(0, nvol, size=batch).astype(np.int32) if nvol > 1 else None
        nv = (P // 2 + 1) * P * P
        dvf = torch.zeros(nv * nvol * 8, dtype=torch.uint8, device="cuda")
        dvw = torch.zeros(nv * nvol * 4, dtype=torch.uint8, device="cuda")
        dpf, dpw, dm = dev(projft), dev(projw), dev(mats)
        div = dev(ivol) if ivol is not None else None
        rmax = n // 2
        _ok(REF.ref_backproject(dvf.data_ptr(), dvw.data_ptr(), P, dpf.data_ptr(), dpw.data_ptr(), n, ndims,
                                rmax, dm.data_ptr(), div.data_ptr() if div is not None else None,
                                *mag, ewald, int(dec), int(sq), batch), name)
        volft = host(dvf, np.complex64, nv * nvol)
        volw = host(dvw, np.float32, nv * nvol)
        np.savez_compressed(out / f"{name}.npz", P=P, n=n, ndims=ndims, rmax=rmax, angles=ang, matrices=mats,
                            projft=projft, projw=projw, ivolume=ivol if ivol is not None else np.zeros(0, np.int32),
                            nvol=nvol, mag=np.array(mag, np.float32), ewald=ewald, decentered=dec,
                            square=sq, volft=volft, volw=volw)
        print(name, np.abs(volft).max(), volw.max())


def gen_gridding(out: Path, rng) -> None:
    for name, ori, pad, nproj, iters in (("grid_it10", 16, 2, 300, 10), ("grid_it0", 16, 2, 300, 0),
                                         ("grid_it3_pad3", 12, 3, 200, 3)):
        P = ori * pad
        dpad = P + 1
        vol = blob_volume_ft(rng, ori, P, 10)
        ang = random_angles(rng, nproj)
        mats = O.matrices_f64(ang, float(pad)).astype(np.float32)
        e = O.elements_fft(ori)
        dv = dev(vol, extra=64)
        dm = dev(mats)
        dp = torch.zeros(e * nproj * 8, dtype=torch.uint8, device="cuda")
        _ok(REF.ref_project(dv.data_ptr(), P, dp.data_ptr(), ori, 2, ori // 2, dm.data_ptr(), nproj), name)
        nv = (dpad // 2 + 1) * dpad * dpad
        dvf = torch.zeros(nv * 8, dtype=torch.uint8, device="cuda")
        dvw = torch.zeros(nv * 4, dtype=torch.uint8, device="cuda")
        _ok(REF.ref_backproject(dvf.data_ptr(), dvw.data_ptr(), dpad, dp.data_ptr(), None, ori, 2, ori // 2,
                                dm.data_ptr(), None, 1, 0, 0, 1, 0.0, 0, 0, nproj), name + " bp")
        dataft = host(dvf, np.complex64, nv)
        weight = host(dvw, np.float32, nv)
        drec = torch.zeros(ori ** 3 * 4, dtype=torch.uint8, device="cuda")
        _ok(REF.ref_reconstruct_gridding(dvf.data_ptr(), dvw.data_ptr(), drec.data_ptr(), ori, dpad, pad,
                                         iters, 1.9, 0, 15.0), name + " grid")
        rec = host(drec, np.float32, ori ** 3).reshape(ori, ori, ori)
        np.savez_compressed(out / f"{name}.npz", ori=ori, pad=pad, dimspadded=dpad, iterations=iters,
                            dataft=dataft, weight=weight, reconstructed=rec)
        print(name, np.abs(rec).max())


def gen_shifted(out: Path, rng) -> None:
    """d_rlnProjectShifted / d_rlnBackprojectShifted (matrix overloads).  The
    backprojection cases keep rmax * supersample below the centred box's
    half-width: the reference writes without bounds checks."""
    for name, n, ndims, batch, rmax in (("project_shifted_2d", 16, 2, 12, 8), ("project_shifted_3d", 8, 3, 3, 4)):
        P = 2 * n
        vol = blob_volume_ft(rng, n, P, 12)
        ang = random_angles(rng, batch)
        mats = O.matrices_f64(ang, 2.0).astype(np.float32)
        shifts_px = rng.uniform(-3, 3, (batch, 3)).astype(np.float32)
        shifts = O.scaled_shifts(shifts_px, n)
        gw = rng.uniform(0.5, 1.5, batch).astype(np.float32)
        e = O.elements_fft(n, ndims)
        dv, dm, ds, dw = dev(vol, extra=64), dev(mats), dev(shifts), dev(gw)
        dp = torch.zeros(e * batch * 8, dtype=torch.uint8, device="cuda")
        _ok(REF.ref_project_shifted(dv.data_ptr(), P, dp.data_ptr(), n, ndims, rmax, dm.data_ptr(), ds.data_ptr(),
                                    dw.data_ptr(), batch), name)
        proj = host(dp, np.complex64, e * batch).reshape(batch, e)
        np.savez_compressed(out / f"{name}.npz", volume=vol, P=P, n=n, ndims=ndims, rmax=rmax, angles=ang,
                            matrices=mats, shifts_px=shifts_px, shifts=shifts, globalweights=gw, proj=proj)
        print(name, np.abs(proj).max())
    for name, n, ndims, V, batch, rmax in (("bp_shifted_2d", 16, 2, 33, 30, 7), ("bp_shifted_3d", 8, 3, 17, 3, 3)):
        ang = random_angles(rng, batch)
        mats = O.matrices_f64(ang, 2.0).astype(np.float32)
        shifts_px = rng.uniform(-3, 3, (batch, 3)).astype(np.float32)
        shifts = O.scaled_shifts(shifts_px, n)
        gw = rng.uniform(0.5, 1.5, batch).astype(np.float32)
        e = O.elements_fft(n, ndims)
        projft = (rng.normal(size=(batch, e)) + 1j * rng.normal(size=(batch, e))).astype(np.complex64)
        projw = rng.uniform(0.1, 1.0, size=(batch, e)).astype(np.float32)
        nv = (V // 2 + 1) * V * V
        dvf = torch.zeros(nv * 8, dtype=torch.uint8, device="cuda")
        dvw = torch.zeros(nv * 4, dtype=torch.uint8, device="cuda")
        dpf, dpw, dm, ds, dw = dev(projft), dev(projw), dev(mats), dev(shifts), dev(gw)
        _ok(REF.ref_backproject_shifted(dvf.data_ptr(), dvw.data_ptr(), V, dpf.data_ptr(), dpw.data_ptr(), n, ndims,
                                        rmax, dm.data_ptr(), ds.data_ptr(), dw.data_ptr(), batch), name)
        volft = host(dvf, np.complex64, nv)
        volw = host(dvw, np.float32, nv)
        np.savez_compressed(out / f"{name}.npz", V=V, n=n, ndims=ndims, rmax=rmax, angles=ang, matrices=mats,
                            shifts_px=shifts_px, shifts=shifts, globalweights=gw, projft=projft, projw=projw,
                            volft=volft, volw=volw)
        print(name, np.abs(volft).max(), volw.max())


def gen_ctf(out: Path, rng) -> None:
    """d_CTFSimulate on the half-complex grid of 32 (frequencies up to
    0.25/pixel at 1-1.5 A/pixel keep the phase below ~60 rad) and on random
    points, with and without amplitude squaring / first-peak flattening,
    astigmatism, anisotropic pixels, B-factors, phase shift and a gamma
    correction."""
    from oracle import ctf_oracle as CO
    batch = 6
    params = CO.params_array([dict(pixelsize=rng.uniform(1.0, 1.5) * 1e-10, pixeldelta=rng.uniform(0, 0.02) * 1e-10,
                                   pixelangle=rng.uniform(0, np.pi), defocus=-rng.uniform(0.3, 1.5) * 1e-6,
                                   defocusdelta=rng.uniform(0, 0.1) * 1e-6, astigmatismangle=rng.uniform(0, np.pi),
                                   Bfactor=-rng.uniform(0, 60) * 1e-20 if i % 2 else 0.0,
                                   Bfactordelta=rng.uniform(0, 10) * 1e-20 if i % 3 == 0 else 0.0,
                                   Bfactorangle=rng.uniform(0, np.pi), phaseshift=rng.uniform(0, 0.5),
                                   scale=rng.uniform(0.8, 1.2)) for i in range(batch)])
    grid = CO.half_grid_addresses(32)
    grid = grid[grid[:, 0] <= 0.25]
    pts = np.stack([rng.uniform(0, 0.25, 300), rng.uniform(-np.pi, np.pi, 300)], -1)
    addresses = np.concatenate([grid, pts]).astype(np.float32)
    n = len(addresses)
    gcorr = rng.uniform(-0.2, 0.2, n).astype(np.float32)
    da, dg = dev(addresses), dev(gcorr)
    res = {}
    for sq in (0, 1):
        for ign in (0, 1):
            for gc in (0, 1):
                do = torch.zeros(n * batch * 4, dtype=torch.uint8, device="cuda")
                _ok(REF.ref_ctf_simulate(params.ctypes.data, da.data_ptr(), dg.data_ptr() if gc else None,
                                         do.data_ptr(), n, sq, ign, batch), "ctf")
                res[f"out_sq{sq}_ign{ign}_gc{gc}"] = host(do, np.float32, n * batch).reshape(batch, n)
    np.savez_compressed(out / "ctf_simulate.npz", params=params, addresses=addresses, gammacorrection=gcorr, **res)
    print("ctf_simulate", {k: float(np.abs(v).max()) for k, v in res.items()})


def gen_estep(out: Path, rng) -> None:
    """The reference's E-step consumers on random inputs.  Every device
    buffer handed to the reference is held in `keep` until the calls are
    done (a temporary's memory would go back to torch's allocator and be
    reused by the next argument)."""
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    keep = []

    def D(a) -> int:
        t = dev(a)
        keep.append(t)
        return t.data_ptr()

    res = {}
    # ConvertWeightsDense
    npart, ncls, nrot, ntr = 3, 2, 20, 7
    w = f32(rng.uniform(0, 5, npart * ncls * nrot * ntr))
    pr, pt, md = f32(rng.uniform(0, 1, ncls * nrot)), f32(rng.uniform(0, 1, npart * ncls * ntr)), f32(rng.uniform(0, 1, npart))
    dw = dev(w)
    _ok(REF.ref_convert_weights_dense(dw.data_ptr(), npart, ncls, nrot, ntr, D(pr), D(pt),
                                      D(md)), "convert dense")
    res.update(cd_in=w, cd_pdfrot=pr, cd_pdftrans=pt, cd_mindiff2=md, cd_out=host(dw, np.float32, w.size),
               cd_shape=np.array([npart, ncls, nrot, ntr]))
    # ConvertWeightsSparse
    nsp, ndense = 100, 500
    comb = np.stack([rng.integers(0, ncls, nsp), rng.integers(0, nrot, nsp), rng.integers(0, ntr, nsp),
                     rng.permutation(ndense)[:nsp]], 1).astype(np.uint32)
    dense = f32(rng.uniform(0, 5, ndense))
    pt2 = f32(rng.uniform(0, 1, ncls * ntr))
    md1 = f32([0.5])
    dd, dsp = dev(dense), torch.zeros(nsp * 4, dtype=torch.uint8, device="cuda")
    _ok(REF.ref_convert_weights_sparse(dd.data_ptr(), dsp.data_ptr(), D(comb), nsp, nrot, ntr,
                                       D(pr), D(pt2), D(md1)), "convert sparse")
    res.update(cs_dense=dense, cs_comb=comb, cs_pdftrans=pt2, cs_mindiff2=md1, cs_out_dense=host(dd, np.float32, ndense),
               cs_out_sparse=host(dsp, np.float32, nsp))
    # DiffRemapDense, both modes
    norient, iclass, nrot2, ntr2, ntp = 10, 1, 12, 5, 8
    orient = np.stack([np.zeros(norient), rng.permutation(nrot2)[:norient], np.zeros(norient)], 1).astype(np.uint32)
    inp = f32(rng.uniform(0, 5, norient * npart * ntp))
    xi2, sq = f32(rng.uniform(1, 2, npart)), f32(rng.uniform(0.5, 1, npart))
    for cc in (0, 1):
        o0 = f32(rng.uniform(0, 1, npart * ncls * nrot2 * ntr2))
        do = dev(o0)
        _ok(REF.ref_diff_remap_dense(D(inp), do.data_ptr(), D(orient), norient, iclass, npart,
                                     ncls, nrot2, ntr2, ntp, D(xi2), D(sq), cc), "remap dense")
        res[f"rd_out0_cc{cc}"] = o0
        res[f"rd_out_cc{cc}"] = host(do, np.float32, o0.size)
    res.update(rd_in=inp, rd_orient=orient, rd_xi2=xi2, rd_sqrtxi2=sq,
               rd_shape=np.array([norient, iclass, npart, ncls, nrot2, ntr2, ntp]))
    # DiffRemapSparse, both modes
    nel, tile, wpp = 208, 16, 256
    combs = np.stack([np.zeros(nel // tile), rng.integers(0, npart, nel // tile), np.zeros(nel // tile)], 1).astype(np.uint32)
    # hidden indices unique within each particle (the reference writes them without ordering)
    perms, used = [rng.permutation(wpp) for _ in range(npart)], [0] * npart
    hid = []
    for c in combs:
        p_ = int(c[1])
        hid.append(perms[p_][used[p_]:used[p_] + tile])
        used[p_] += tile
    hid = np.concatenate(hid).astype(np.uint32)
    inp2 = f32(rng.uniform(-1, 5, nel))
    for cc in (0, 1):
        o0 = f32(np.zeros(npart * wpp))
        m0 = f32(np.full(npart, 1e30))
        do, dm = dev(o0), dev(m0)
        _ok(REF.ref_diff_remap_sparse(D(inp2), do.data_ptr(), dm.data_ptr(), D(combs),
                                      D(hid), nel, tile, wpp, npart, D(xi2), D(sq),
                                      cc), "remap sparse")
        res[f"rs_out_cc{cc}"] = host(do, np.float32, o0.size)
        res[f"rs_min_cc{cc}"] = host(dm, np.float32, npart)
    res.update(rs_in=inp2, rs_comb=combs, rs_hidden=hid, rs_shape=np.array([nel, tile, wpp, npart]))
    # CreateMinvsigma2s
    nm = 500
    mres = rng.integers(-1, 21, nm).astype(np.int32)
    s2 = f32(rng.uniform(0.5, 2, 21))
    dmo = torch.zeros(nm * 4, dtype=torch.uint8, device="cuda")
    _ok(REF.ref_create_minvsigma2s(dmo.data_ptr(), D(mres), nm, D(s2), 1.3), "minvsigma2s")
    res.update(mv_mresol=mres, mv_sigma2=s2, mv_out=host(dmo, np.float32, nm))
    # StoreWeightsAdd, both modes
    ne, nt = 300, 4
    inp3 = (rng.normal(size=(nt, ne)) + 1j * rng.normal(size=(nt, ne))).astype(np.complex64)
    ctf = f32(rng.uniform(-1, 1, ne))
    ref = (rng.normal(size=ne) + 1j * rng.normal(size=ne)).astype(np.complex64)
    mv = f32(rng.uniform(0.1, 1, ne))
    mr = rng.integers(-1, 16, ne).astype(np.int32)
    wts = f32([0.3, 0.0001, 0.5, 0.2])
    prior = f32(rng.uniform(0, 6, 16))
    res.update(sw_in=inp3, sw_ctf=ctf, sw_ref=ref, sw_minvsigma2=mv, sw_mresol=mr, sw_weights=wts, sw_prior=prior)
    for sc in (0, 1):
        o0 = (rng.normal(size=(nt, ne)) + 1j * rng.normal(size=(nt, ne))).astype(np.complex64)
        ow0 = f32(rng.uniform(0, 1, (nt, ne)))
        s20, nc0, xa0, aa0 = f32(rng.uniform(0, 1, 16)), f32([0.25]), f32(rng.uniform(0, 1, 16)), f32(rng.uniform(0, 1, 16))
        do, dow, ds2, dnc, dxa, daa = dev(o0), dev(ow0), dev(s20), dev(nc0), dev(xa0), dev(aa0)
        _ok(REF.ref_store_weights_add(D(inp3), D(ctf), D(ref), D(mv),
                                      D(mr), ne, nt, D(wts), 0.001, 1.7, do.data_ptr(),
                                      dow.data_ptr(), ds2.data_ptr(), dnc.data_ptr(), D(prior),
                                      dxa.data_ptr(), daa.data_ptr(), sc), "store weights")
        res.update({f"sw{sc}_out0": o0, f"sw{sc}_ow0": ow0, f"sw{sc}_s20": s20, f"sw{sc}_nc0": nc0,
                    f"sw{sc}_xa0": xa0, f"sw{sc}_aa0": aa0,
                    f"sw{sc}_out": host(do, np.complex64, nt * ne), f"sw{sc}_ow": host(dow, np.float32, nt * ne),
                    f"sw{sc}_s2": host(ds2, np.float32, 16), f"sw{sc}_nc": host(dnc, np.float32, 1),
                    f"sw{sc}_xa": host(dxa, np.float32, 16), f"sw{sc}_aa": host(daa, np.float32, 16)})
    np.savez_compressed(out / "estep.npz", **res)
    print("estep", len(res), "arrays")


def gen_tomo(out: Path, rng) -> None:
    """d_BackprojectTomo: a 16^3 half volume from 7 tilted 16^2 slices (a
    tilt series about y under a random rotation), volume pre-filled so that
    the voxels it leaves alone are visible."""
    from tests.synthdata import random_angles
    V, n, batch, rmax = 16, 16, 7, 7
    base = random_angles(rng, 1)[0]
    ang = np.array([[base[0], base[1] + t, base[2]] for t in np.deg2rad(np.linspace(-45, 45, batch))], np.float32)
    mats = O.matrices_f64(ang, 1.0).astype(np.float32)
    e = O.elements_fft(n)
    projft = (rng.normal(size=(batch, e)) + 1j * rng.normal(size=(batch, e))).astype(np.complex64)
    projw = rng.uniform(0.5, 1.0, size=(batch, e)).astype(np.float32)
    nv = (V // 2 + 1) * V * V
    vol0 = np.full(nv, 7 + 7j, np.complex64)
    dv, dpf, dpw, dm = dev(vol0), dev(projft), dev(projw), dev(mats)
    _ok(REF.ref_backproject_tomo(dv.data_ptr(), V, dpf.data_ptr(), dpw.data_ptr(), n, rmax, dm.data_ptr(), batch),
        "tomo")
    np.savez_compressed(out / "bp_tomo.npz", V=V, n=n, rmax=rmax, angles=ang, matrices=mats, projft=projft,
                        projw=projw, volume0=vol0, volume=host(dv, np.complex64, nv))
    print("bp_tomo", np.abs(host(dv, np.complex64, nv)).max())


def main() -> None:
    """make_golden.py [outdir] [--only project|backproject|gridding|shifted|ctf|estep|tomo ...]"""
    args = sys.argv[1:]
    only = set(args[args.index("--only") + 1:]) if "--only" in args else None
    args = args[:args.index("--only")] if "--only" in args else args
    out = Path(args[0]) if args else Path(__file__).resolve().parent
    out.mkdir(parents=True, exist_ok=True)
    rng = np.random.default_rng(20261203)
    for key, fn in (("project", gen_project), ("backproject", gen_backproject), ("gridding", gen_gridding)):
        if only is None or key in only:
            fn(out, rng)
    if only is None or "shifted" in only:
        gen_shifted(out, np.random.default_rng(20261204))
    if only is None or "ctf" in only:
        gen_ctf(out, np.random.default_rng(20261205))
    if only is None or "estep" in only:
        gen_estep(out, np.random.default_rng(20261206))
    if only is None or "tomo" in only:
        gen_tomo(out, np.random.default_rng(20261207))


if __name__ == "__main__":
    main()
