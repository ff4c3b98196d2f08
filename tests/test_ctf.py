"""CTF simulation (gtom's d_CTFSimulate) and particle preprocessing.

CPU: the float64 oracle against the reference's own results
(tests/golden/ctf_simulate.npz) and a known answer (zero frequency).
GPU: gtomrln_ctf_simulate against the reference's results and the oracle;
gtomrln_preprocess_particles against the oracle's FFT + CTF, and inserting
its output equals inserting the CTF-weighted slices made on the host."""
import numpy as np
import pytest
import torch

from oracle import ctf_oracle as CO
from tests.helpers import load_golden, rel_l2

CASES = [(sq, ign, gc) for sq in (0, 1) for ign in (0, 1) for gc in (0, 1)]


@pytest.mark.parametrize("sq,ign,gc", CASES)
def test_oracle_ctf_matches_reference(sq, ign, gc):
    """The reference evaluates with the fast hardware sine/cosine/exp in
    float; the oracle in float64.  Phases stay below ~60 rad here."""
    g = load_golden("ctf_simulate")
    want = g[f"out_sq{sq}_ign{ign}_gc{gc}"]
    got = CO.simulate(g["params"], g["addresses"], g["gammacorrection"] if gc else None, bool(sq), bool(ign))
    assert np.max(np.abs(got - want)) <= 2e-4


def test_oracle_ctf_zero_frequency():
    """At k = 0 the CTF is -sin(-phaseshift - K3) * scale, K3 = atan(A/sqrt(1-A^2))."""
    p = CO.params_array([dict(amplitude=0.1, phaseshift=0.3, scale=2.0)])
    v = CO.simulate(p, np.zeros((1, 2)))[0, 0]
    assert v == pytest.approx(-np.sin(-0.3 - np.arcsin(np.float32(0.1))) * 2.0, rel=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("sq,ign,gc", CASES)
def test_ctf_simulate_matches_reference(gtom_lib, cuda, sq, ign, gc):
    from gtom_b200.ctf import d_CTFSimulate
    g = load_golden("ctf_simulate")
    want = g[f"out_sq{sq}_ign{ign}_gc{gc}"]
    batch, n = want.shape
    out = torch.full((batch * n,), np.nan, dtype=torch.float32, device="cuda")
    d_CTFSimulate(g["params"], torch.from_numpy(g["addresses"]).cuda().reshape(-1),
                  torch.from_numpy(g["gammacorrection"]).cuda() if gc else None, out, n, bool(sq), bool(ign),
                  batch)
    got = out.cpu().numpy().reshape(batch, n)
    assert np.max(np.abs(got - want)) <= 2e-5  # same float arithmetic and intrinsics
    oracle = CO.simulate(g["params"], g["addresses"], g["gammacorrection"] if gc else None, bool(sq), bool(ign))
    assert np.max(np.abs(got - oracle)) <= 2e-4


@pytest.mark.gpu
def test_preprocess_particles_matches_oracle(gtom_lib, cuda):
    from gtom_b200.ctf import preprocess_particles
    rng = np.random.default_rng(12)
    n, b = 48, 7
    imgs = rng.normal(size=(b, n, n)).astype(np.float32)
    params = CO.params_array([dict(pixelsize=1.2e-10, defocus=-rng.uniform(0.5, 1.5) * 1e-6,
                                   defocusdelta=0.05e-6, astigmatismangle=0.4, Bfactor=-20e-20)
                              for _ in range(b)])
    ft, w = preprocess_particles(torch.from_numpy(imgs).cuda(), params)
    want_ft, want_w = CO.preprocess(imgs, params)
    assert rel_l2(ft.cpu().numpy().reshape(b, -1), want_ft) <= 1e-5
    assert rel_l2(w.cpu().numpy().reshape(b, -1), want_w) <= 1e-5
    ft0, w0 = preprocess_particles(torch.from_numpy(imgs).cuda(), None)
    assert rel_l2(ft0.cpu().numpy().reshape(b, -1), CO.preprocess(imgs, None)[0]) <= 1e-6
    assert torch.all(w0 == 1)


@pytest.mark.gpu
def test_preprocessed_particles_insert_like_host_weighted_slices(gtom_lib, cuda):
    """Preprocess + d_rlnBackproject equals d_rlnBackproject of slices
    weighted on the host with the oracle's CTF (same FFT convention)."""
    import gtom_b200 as G
    from gtom_b200.ctf import preprocess_particles
    from oracle import oracle as O
    from tests.synthdata import random_angles
    rng = np.random.default_rng(5)
    n, b = 32, 40
    imgs = rng.normal(size=(b, n, n)).astype(np.float32)
    params = CO.params_array([dict(defocus=-rng.uniform(0.5, 2) * 1e-6) for _ in range(b)])
    mats = torch.from_numpy(O.matrices_f64(random_angles(rng, b), 2.0).astype(np.float32)).cuda().reshape(-1)
    D = 2 * n + 1
    nv = (D // 2 + 1) * D * D
    ft, w = preprocess_particles(torch.from_numpy(imgs).cuda(), params)
    a_f, a_w = torch.zeros(nv, dtype=torch.complex64, device="cuda"), torch.zeros(nv, device="cuda")
    G.d_rlnBackproject(a_f, a_w, (D, D, D), ft, w, (n, n, 1), n // 2, mats, None, (1, 0, 0, 1), 0.0, False, False, b)
    hf, hw = CO.preprocess(imgs, params)
    b_f, b_w = torch.zeros_like(a_f), torch.zeros_like(a_w)
    G.d_rlnBackproject(b_f, b_w, (D, D, D), torch.from_numpy(hf.astype(np.complex64)).cuda().reshape(-1),
                       torch.from_numpy(hw.astype(np.float32)).cuda().reshape(-1), (n, n, 1), n // 2, mats, None,
                       (1, 0, 0, 1), 0.0, False, False, b)
    # the two inputs differ by the fast-intrinsic CTF against the float64 one
    # (<= 1e-5 relative, previous test); insertion is linear in them
    assert rel_l2(a_f.cpu().numpy(), b_f.cpu().numpy()) <= 5e-5
    assert rel_l2(a_w.cpu().numpy(), b_w.cpu().numpy()) <= 5e-5
