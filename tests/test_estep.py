"""RELION E-step consumers: the float64 oracle against the reference's own
results (tests/golden/estep.npz, CPU), the library against both (GPU),
and the squared differences (no reference source) against the oracle and
the case of GTOMTest/RelionSquaredDiff.cpp."""
import numpy as np
import pytest
import torch

from oracle import estep_oracle as E
from tests.helpers import load_golden, rel_l2


def g():
    return load_golden("estep")


def test_oracle_convert_and_remap_match_reference():
    d = g()
    npart, ncls, nrot, ntr = (int(v) for v in d["cd_shape"])
    got = E.convert_weights_dense(d["cd_in"], npart, ncls, nrot, ntr, d["cd_pdfrot"], d["cd_pdftrans"], d["cd_mindiff2"])
    assert rel_l2(got, d["cd_out"]) <= 1e-5
    dense, sparse = E.convert_weights_sparse(d["cs_dense"], d["cs_comb"], nrot, ntr, d["cd_pdfrot"], d["cs_pdftrans"],
                                             d["cs_mindiff2"][0])
    assert rel_l2(sparse, d["cs_out_sparse"]) <= 1e-5 and rel_l2(dense, d["cs_out_dense"]) <= 1e-5
    norient, iclass, np_, ncls2, nrot2, ntr2, ntp = (int(v) for v in d["rd_shape"])
    for cc in (0, 1):
        got = E.diff_remap_dense(d["rd_in"], d["rd_orient"], iclass, np_, ncls2, nrot2, ntr2, ntp, d["rd_xi2"],
                                 d["rd_sqrtxi2"], cc, d[f"rd_out0_cc{cc}"])
        assert rel_l2(got, d[f"rd_out_cc{cc}"]) <= 1e-6
    nel, tile, wpp, npart3 = (int(v) for v in d["rs_shape"])
    for cc in (0, 1):
        out, md = E.diff_remap_sparse(d["rs_in"], d["rs_comb"], d["rs_hidden"], tile, wpp, d["rd_xi2"], d["rd_sqrtxi2"],
                                      cc, np.zeros(npart3 * wpp), np.full(npart3, 1e30))
        assert rel_l2(out, d[f"rs_out_cc{cc}"]) <= 1e-6
        np.testing.assert_allclose(md, d[f"rs_min_cc{cc}"], rtol=1e-6)
    got = E.create_minvsigma2s(d["mv_mresol"], d["mv_sigma2"], np.float32(1.3))
    np.testing.assert_allclose(got, d["mv_out"], rtol=1e-6)


@pytest.mark.parametrize("sc", [0, 1])
def test_oracle_store_weights_matches_reference(sc):
    d = g()
    nt, ne = d["sw_in"].shape
    r = E.store_weights_add(d["sw_in"], d["sw_ctf"], d["sw_ref"], d["sw_minvsigma2"], d["sw_mresol"], d["sw_weights"],
                            0.001, 1.7, d[f"sw{sc}_out0"], d[f"sw{sc}_ow0"], d[f"sw{sc}_s20"], d[f"sw{sc}_nc0"],
                            d["sw_prior"], d[f"sw{sc}_xa0"], d[f"sw{sc}_aa0"], sc)
    for got, key in zip(r, ("out", "ow", "s2", "nc", "xa", "aa")):
        assert rel_l2(np.ravel(got), d[f"sw{sc}_{key}"].ravel()) <= 1e-5, key


def test_oracle_squared_differences_on_the_gtomtest_case():
    """GTOMTest/RelionSquaredDiff.cpp, case 1 scaled down (16 refs, 16
    shifts): the particle is 1+1i, shift s is (i % (s+1) / 2, 1), ref r is
    (2, i % (r+1) / 2) with integer division."""
    n, nr, ns, tile = 64, 16, 16, 4
    e = (n // 2 + 1) * n
    i = np.arange(e)
    part = np.full((1, e), 1 + 1j)
    shifts = np.array([(i % (s + 1)) // 2 + 1j for s in range(ns)])
    refs = np.array([2 + 1j * ((i % (r + 1)) // 2) for r in range(nr)])
    combos = [(s, 0, r) for r in range(0, nr, tile) for s in range(0, ns, tile)]
    got = E.squared_differences_sparse(part, None, None, shifts, refs, combos, tile)
    want = []
    for s0, _, r0 in combos:
        for r in range(tile):
            for s in range(tile):
                d = refs[r0 + r] - part[0] * shifts[s0 + s]
                want.append(0.5 * np.sum(d.real ** 2 + d.imag ** 2))
    np.testing.assert_allclose(got, want, rtol=1e-12)


# --------------------------------------------------------------------- GPU --
def cu(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return t if dtype is None else t.to(dtype)


@pytest.mark.gpu
@pytest.mark.parametrize("cc", [False, True])
@pytest.mark.parametrize("group", [1, 4, 8])
def test_squared_differences_match_oracle(gtom_lib, cuda, cc, group):
    from gtom_b200.estep import d_rlnSquaredDifferences, d_rlnSquaredDifferencesSparse
    rng = np.random.default_rng(group + 10 * cc)
    n, npart, nr, ns = 32, 2, 2 * group, 3 * group
    e = (n // 2 + 1) * n
    cplx = lambda *s: (rng.normal(size=s) + 1j * rng.normal(size=s)).astype(np.complex64)
    part, shifts, refs = cplx(npart, e), cplx(ns, e), cplx(nr, e)
    w = rng.uniform(0.2, 1.0, e).astype(np.float32)
    ctf = rng.uniform(-1, 1, (npart, e)).astype(np.float32)
    combos = np.array([(s, p, r) for p in range(npart) for r in range(0, nr, group) for s in range(0, ns, group)],
                      np.uint32)
    out = torch.zeros(len(combos) * group * group, device="cuda")
    d_rlnSquaredDifferencesSparse(cu(part), cu(w), cu(ctf), (n, n, 1), cu(shifts), cu(refs), out, cu(combos),
                                  out.numel(), group, cc)
    want = E.squared_differences_sparse(part, w, ctf, shifts, refs, combos, group, cc)
    assert rel_l2(out.cpu().numpy(), want) <= 1e-5
    dense = torch.zeros(npart * nr * ns, device="cuda")
    d_rlnSquaredDifferences(cu(part), cu(w), cu(ctf), (n, n, 1), npart, cu(shifts), ns, cu(refs), nr, group, dense, cc)
    want_d = E.squared_differences_dense(part, w, ctf, shifts, refs, cc)
    assert rel_l2(dense.cpu().numpy(), want_d.ravel()) <= 1e-5


@pytest.mark.gpu
def test_convert_remap_minvsigma_match_reference(gtom_lib, cuda):
    from gtom_b200 import estep as S
    d = g()
    npart, ncls, nrot, ntr = (int(v) for v in d["cd_shape"])
    w = cu(d["cd_in"])
    S.d_rlnConvertWeightsDense(w, npart, ncls, nrot, ntr, cu(d["cd_pdfrot"]), cu(d["cd_pdftrans"]), cu(d["cd_mindiff2"]))
    assert rel_l2(w.cpu().numpy(), d["cd_out"]) <= 1e-5
    dense = cu(d["cs_dense"])
    sparse = torch.zeros(len(d["cs_comb"]), device="cuda")
    S.d_rlnConvertWeightsSparse(dense, sparse, cu(d["cs_comb"].astype(np.int32)), len(d["cs_comb"]), nrot, ntr,
                                cu(d["cd_pdfrot"]), cu(d["cs_pdftrans"]), cu(d["cs_mindiff2"]))
    assert rel_l2(sparse.cpu().numpy(), d["cs_out_sparse"]) <= 1e-5
    assert rel_l2(dense.cpu().numpy(), d["cs_out_dense"]) <= 1e-5
    norient, iclass, np_, ncls2, nrot2, ntr2, ntp = (int(v) for v in d["rd_shape"])
    nel, tile, wpp, npart3 = (int(v) for v in d["rs_shape"])
    for cc in (0, 1):
        out = cu(d[f"rd_out0_cc{cc}"])
        S.d_rlnDiffRemapDense(cu(d["rd_in"]), out, cu(d["rd_orient"].astype(np.int32)), norient, iclass, np_, ncls2,
                              nrot2, ntr2, ntp, cu(d["rd_xi2"]), cu(d["rd_sqrtxi2"]), bool(cc))
        np.testing.assert_array_equal(out.cpu().numpy(), d[f"rd_out_cc{cc}"])
        out = torch.zeros(npart3 * wpp, device="cuda")
        md = torch.full((npart3,), 1e30, device="cuda")
        S.d_rlnDiffRemapSparse(cu(d["rs_in"]), out, md, cu(d["rs_comb"].astype(np.int32)),
                               cu(d["rs_hidden"].astype(np.int32)), nel, tile, wpp, npart3, cu(d["rd_xi2"]),
                               cu(d["rd_sqrtxi2"]), bool(cc))
        np.testing.assert_array_equal(out.cpu().numpy(), d[f"rs_out_cc{cc}"])
        np.testing.assert_array_equal(md.cpu().numpy(), d[f"rs_min_cc{cc}"])
    mv = torch.zeros(len(d["mv_mresol"]), device="cuda")
    S.d_rlnCreateMinvsigma2s(mv, cu(d["mv_mresol"]), len(d["mv_mresol"]), cu(d["mv_sigma2"]), 1.3)
    np.testing.assert_allclose(mv.cpu().numpy(), d["mv_out"], rtol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("sc", [0, 1])
def test_store_weights_match_reference(gtom_lib, cuda, sc):
    from gtom_b200 import estep as S
    d = g()
    nt, ne = d["sw_in"].shape
    out, ow = cu(d[f"sw{sc}_out0"]).reshape(-1), cu(d[f"sw{sc}_ow0"]).reshape(-1)
    s2, nc, xa, aa = cu(d[f"sw{sc}_s20"]), cu(d[f"sw{sc}_nc0"]), cu(d[f"sw{sc}_xa0"]), cu(d[f"sw{sc}_aa0"])
    S.d_rlnStoreWeightsAdd(cu(d["sw_in"]).reshape(-1), cu(d["sw_ctf"]), cu(d["sw_ref"]), cu(d["sw_minvsigma2"]),
                           cu(d["sw_mresol"]), ne, nt, cu(d["sw_weights"]), 0.001, 1.7, out, ow, s2, nc, cu(d["sw_prior"]),
                           xa, aa, bool(sc))
    for t, key in ((out, "out"), (ow, "ow"), (s2, "s2"), (nc, "nc"), (xa, "xa"), (aa, "aa")):
        assert rel_l2(t.cpu().numpy().ravel(), d[f"sw{sc}_{key}"].ravel()) <= 1e-5, key


@pytest.mark.gpu
def test_sort_and_compact(gtom_lib, cuda):
    from gtom_b200 import estep as S
    rng = np.random.default_rng(3)
    x = rng.normal(size=10007).astype(np.float32)
    t = cu(x)
    S.d_rlnConvertWeightsSort(t, x.size)
    np.testing.assert_array_equal(t.cpu().numpy(), np.sort(x))
    out = torch.zeros_like(t)
    n = S.d_rlnConvertWeightsCompact(cu(x), out, x.size)
    np.testing.assert_array_equal(out.cpu().numpy()[:n], x[x > 0])


@pytest.mark.gpu
def test_squared_differences_close_match_accuracy(gtom_lib, cuda):
    """A particle equal to CTF * reference 0 up to 1e-3 noise, identity
    shift: its squared difference to that reference is ~1e-6 of the
    operands' weighted power, and the dense (tiled) kernel still gives it to
    1e-3 of the FP64 oracle (no cancelling expansion of |a - b|^2)."""
    from gtom_b200.estep import d_rlnSquaredDifferences
    rng = np.random.default_rng(7)
    n, nr, ns = 64, 70, 66
    e = (n // 2 + 1) * n
    cplx = lambda *s: (rng.normal(size=s) + 1j * rng.normal(size=s)).astype(np.complex64)
    refs = cplx(nr, e)
    shifts = cplx(ns, e)
    shifts[0] = 1.0
    ctf = rng.uniform(-1, 1, (1, e)).astype(np.float32)
    part = (ctf[0] * refs[0] + 1e-3 * cplx(e)).astype(np.complex64)[None]
    w = rng.uniform(0.2, 1.0, e).astype(np.float32)
    dense = torch.zeros(nr * ns, device="cuda")
    d_rlnSquaredDifferences(cu(part), cu(w), cu(ctf), (n, n, 1), 1, cu(shifts), ns, cu(refs), nr, 1, dense, False)
    want = E.squared_differences_dense(part, w, ctf, shifts, refs, False).ravel()
    got = dense.cpu().numpy()
    assert got[0] == pytest.approx(want[0], rel=1e-3)
    assert want[0] < 1e-5 * np.median(want)
    assert rel_l2(got, want) <= 1e-5
