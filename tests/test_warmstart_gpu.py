"""The learned warm start on the GPU, against the CPU oracle
(oracle/mlp_oracle.py): features, forward pass, gradients of the training
kernel, Adam, the predicted start with one gridding iteration, the momentum
iteration, the residual check's fallback to the cold start, and what a
network trained here on the GPU gains over the cold start on held-out
orientation distributions."""
import ctypes as C

import numpy as np
import pytest
import torch

import gtom_b200 as G
from gtom_b200 import warmstart as W
from oracle import mlp_oracle as M
from oracle import oracle as O
from tests.helpers import rel_l2
from tests.synthdata import random_angles

pytestmark = pytest.mark.gpu


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dev(a):
    return torch.tensor(np.asarray(a), dtype=torch.float32, device="cuda")


def _params(seed=5):
    rng = np.random.default_rng(seed)
    p = M.init_params(rng, shift=rng.normal(-1, 1, M.N_IN), scale=rng.uniform(0.3, 1.5, M.N_IN))
    p[M.OFF_B1:M.OFF_W2] = rng.normal(0, 0.2, M.N_HID)
    p[M.OFF_B2:M.OFF_W3] = rng.normal(0, 0.2, M.N_HID)
    p[M.OFF_B3] = 0.3
    return p


def _weights(P, views=600, seed=2):
    rng = np.random.default_rng(seed)
    n = P // 2
    mats = O.matrices_f64(random_angles(rng, views), 2.0).astype(np.float32)
    e = (n // 2 + 1) * n
    w = rng.uniform(0.2, 1.0, (views, e)).astype(np.float32)
    D = P + 1
    vol = np.zeros((D // 2 + 1) * D * D, np.float32)
    O.backproject(None, vol, D, None, w, n, n // 2, mats, decentered=False, fp32=True)
    return vol, D


def _gridding(weight, D, ori, iters, tol=0.0, momentum=0.0, params=None, limit=0.5):
    return G.gridding_weights(weight, (D, D, D), ori, 2, iters, tol, momentum, mlp_params=params,
                              residual_limit=limit)


def test_forward_matches_oracle(gtom_lib, cuda):
    rng = np.random.default_rng(1)
    p = _params()
    f = rng.normal(-2, 2, (3000, M.N_IN))
    f[:, 27] = rng.uniform(0, 1, 3000)
    want = M.forward(p, f)
    dp, df = _dev(p), _dev(f)
    out = torch.empty(3000, dtype=torch.float32, device="cuda")
    assert gtom_lib.gtomrln_mlp_forward(C.c_void_p(dp.data_ptr()), C.c_void_p(df.data_ptr()), 3000,
                                        C.c_void_p(out.data_ptr()), _stream()) == 0
    got = out.cpu().numpy()
    assert np.max(np.abs(got - want)) <= 1e-4 * max(1.0, np.max(np.abs(want)))


def test_gradients_match_oracle(gtom_lib, cuda):
    """The training kernel's gradients against the oracle's analytic ones
    (which the CPU suite checks against finite differences), over several
    blocks including a partial last block."""
    rng = np.random.default_rng(2)
    p = _params(7)
    n = 1000
    f = rng.normal(-2, 2, (n, M.N_IN))
    t = rng.normal(0, 1, n)
    w = rng.uniform(0.1, 2, n)
    loss_ref, g_ref = M.gradients(p, f, t, w, 1 / n)
    dp, df, dt, dw = _dev(p), _dev(f), _dev(t), _dev(w)
    grad = torch.zeros(M.N_PARAMS, dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    assert gtom_lib.gtomrln_mlp_gradients(C.c_void_p(dp.data_ptr()), C.c_void_p(df.data_ptr()),
                                          C.c_void_p(dt.data_ptr()), C.c_void_p(dw.data_ptr()), n,
                                          C.c_float(1 / n), C.c_void_p(grad.data_ptr()),
                                          C.c_void_p(loss.data_ptr()), _stream()) == 0
    g = grad.cpu().numpy().astype(np.float64)
    assert loss.item() == pytest.approx(loss_ref, rel=1e-4)
    assert np.all(g[:M.OFF_W1] == 0)
    for a, b in ((M.OFF_W1, M.OFF_B1), (M.OFF_B1, M.OFF_W2), (M.OFF_W2, M.OFF_B2), (M.OFF_B2, M.OFF_W3),
                 (M.OFF_W3, M.OFF_B3), (M.OFF_B3, M.N_PARAMS)):
        assert rel_l2(g[a:b], g_ref[a:b]) <= 1e-4, (a, b)


def test_adam_matches_oracle(gtom_lib, cuda):
    rng = np.random.default_rng(4)
    p = _params(3)
    m = rng.normal(0, 0.01, M.N_PARAMS)
    v = rng.uniform(0, 0.01, M.N_PARAMS)
    g = rng.normal(0, 1, M.N_PARAMS)
    pw, mw, vw = M.adam(p, g, m, v, 7, 3e-3)
    dp, dg, dm, dv = _dev(p), _dev(g), _dev(m), _dev(v)
    assert gtom_lib.gtomrln_mlp_adam(C.c_void_p(dp.data_ptr()), C.c_void_p(dg.data_ptr()),
                                     C.c_void_p(dm.data_ptr()), C.c_void_p(dv.data_ptr()), 7, C.c_float(3e-3),
                                     C.c_float(0.9), C.c_float(0.999), C.c_float(1e-8), _stream()) == 0
    np.testing.assert_allclose(dp.cpu().numpy(), pw, rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(dm.cpu().numpy()[M.OFF_W1:], mw[M.OFF_W1:], rtol=1e-5, atol=1e-7)
    assert np.all(dg.cpu().numpy()[M.OFF_W1:] == 0)


def test_volume_features_match_oracle(cuda):
    P = 32
    vol, D = _weights(P)
    fw = O._decenter(vol.astype(np.float64), P, (D, D, D)).real.ravel().astype(np.float32)
    nc = fw.size
    rng = np.random.default_rng(8)
    rowlen = P // 2 + 1
    idx = np.concatenate([rng.integers(0, nc, 500), np.arange(0, nc, rowlen)[:200]])  # incl. x = 0
    stack = np.concatenate([fw, 2 * fw])
    index = np.concatenate([idx, idx + nc]).astype(np.int64)
    want = np.concatenate([M.features(fw, P, 0.7, idx), M.features(2 * fw, P, 0.35, idx)])
    ts = W.TrainingSet(P=P, fw=_dev(stack), target=None, weight=None,
                       inv_scale=_dev([0.7, 0.35]), eligible=None)
    got = W.volume_features(ts, torch.tensor(index, device="cuda")).cpu().numpy()
    assert np.max(np.abs(got - want)) <= 2e-5 * np.max(np.abs(want))


def test_predicted_start_and_one_iteration_match_oracle(cuda):
    P = 32
    vol, D = _weights(P)
    p = _params(11)
    p[M.OFF_B3] = 0.0
    fw = O._decenter(vol.astype(np.float64), P, (D, D, D)).real.ravel()
    start = M.predict_start(p, fw, P, (P // 2) ** 2)
    want, ch = M.gridding_iterations(fw, start, P, 2, 1)
    fnw, gfw, it, change, used = _gridding(_dev(vol), D, P // 2, 1, params=_dev(p), limit=1e30)
    assert used and it == 1
    np.testing.assert_allclose(gfw.cpu().numpy(), fw, rtol=1e-6, atol=0)
    sel = fw > 0
    assert rel_l2(fnw.cpu().numpy()[sel], want[sel]) <= 1e-4
    assert change == pytest.approx(ch[0], rel=1e-3)


@pytest.mark.parametrize("momentum", [0.0, 0.9])
def test_iteration_matches_oracle(cuda, momentum):
    P = 32
    vol, D = _weights(P, seed=6)
    fw = O._decenter(vol.astype(np.float64), P, (D, D, D)).real.ravel()
    start = M.predict_start(M.init_params(np.random.default_rng(0)), np.zeros_like(fw), P, (P // 2) ** 2)
    want, ch = M.gridding_iterations(fw, start, P, 2, 25, momentum=momentum)
    # a tolerance far below reach makes every iteration report its change
    fnw, _, it, change, used = _gridding(_dev(vol), D, P // 2, 25, tol=1e-12, momentum=momentum)
    assert it == 25 and not used
    got = fnw.cpu().numpy()
    d = np.sqrt(np.sum((fw * (got - want)) ** 2) / np.sum((fw * want) ** 2))
    assert d <= 1e-4, d
    assert change == pytest.approx(ch[-1], rel=2e-2), (change, ch[-1])


def test_rejected_start_falls_back_to_the_cold_start(cuda):
    """A network whose start is far off (output + 40 in the log) fails the
    residual check; the result must then be exactly the cold-start result."""
    P = 32
    vol, D = _weights(P, seed=9)
    p = _params(1)
    p[M.OFF_B3] = 40.0
    dw = _dev(vol)
    cold, _, it_c, ch_c, _ = _gridding(dw, D, P // 2, 200, tol=1e-3)
    warm, _, it_w, ch_w, used = _gridding(dw, D, P // 2, 200, tol=1e-3, params=_dev(p))
    assert not used
    assert it_w == it_c + 1  # the rejected iteration counts
    assert torch.equal(warm, cold)
    assert ch_w == pytest.approx(ch_c, rel=1e-9)  # change sums are reduced by atomics


def test_trained_network_beats_the_cold_start(cuda):
    """Train on 12 distributions at box 32 (P = 64) with the library's own
    kernels; then on 4 held-out distributions the predicted start must be
    closer to the converged weights than the cold start after the same
    number of plain iterations (10: the criterion of the converged weights,
    measured early, where the network's gain lies), and reach the 1e-4
    change in no more iterations (plain and momentum forms).  What it does
    not gain is asserted nowhere because it is not there: to within 1e-4 of
    the converged weights the learned start takes as long as the cold one
    (1.00x plain, 0.95x with momentum on the 200 held-out distributions of
    the 128^3 workload), the remaining error being the iteration's slow,
    non-local modes."""
    box, pad = 32, 2
    D = box * pad + 1
    rng = np.random.default_rng(2024)
    dists = [W.random_distribution(rng, views_range=(3000, 12000)) for _ in range(16)]
    vols = [W.sampling_weights(box, d, pad) for d in dists]
    ts = W.make_training_set(vols[:12], box, pad, tolerance=1e-6, max_iterations=4000)
    params = W.init_params(ts, seed=1)
    losses = W.train(ts, params, steps=600, batch=16384, lr=3e-3, lr_final=1e-4, log_every=100)
    assert losses[-1] < 0.5 * losses[0]
    gains = []
    for w in vols[12:]:
        ref, fw, _, _, _ = _gridding(w, D, box, 4000, tol=1e-7, momentum=0.9)
        cold10, _, _, _, _ = _gridding(w, D, box, 10)
        warm10, _, _, _, used = _gridding(w, D, box, 10, params=params)
        assert used
        gains.append(W.weighted_distance(fw, cold10, ref) / W.weighted_distance(fw, warm10, ref))
        for mom in (0.0, 0.9):
            _, _, it_c, _, _ = _gridding(w, D, box, 3000, tol=1e-4, momentum=mom)
            _, _, it_w, _, _ = _gridding(w, D, box, 3000, tol=1e-4, momentum=mom, params=params)
            assert it_w <= it_c, (mom, it_w, it_c)
    assert min(gains) > 1.2, gains


@pytest.mark.parametrize("momentum", [0.0, 0.9])
def test_distance_to_reference_weights_stops_the_loop(cuda, momentum):
    """gtomrln_gridding_weights with reference weights: the library's
    distance ||Fw (Fnw - ref)|| / ||Fw ref|| equals the one measured on the
    returned weights, the loop stops at the first iteration within the
    tolerance, and one iteration fewer is not within it."""
    P = 64
    vol, D = _weights(P)
    w = torch.from_numpy(vol).cuda()
    ref, fw, _, _, _ = _gridding(w, D, P // 2, 3000, 1e-6, 0.9)
    tol = 1e-3
    fnw, fw2, k, _, _, dist = G.gridding_weights(w, (D, D, D), P // 2, 2, 5000, 0.0, momentum, ref_fnw=ref,
                                                 ref_tolerance=tol, return_distance=True)
    assert 1 < k < 5000
    assert dist <= tol
    assert dist == pytest.approx(W.weighted_distance(fw2, fnw, ref), rel=1e-5)
    _, _, k1, _, _, d1 = G.gridding_weights(w, (D, D, D), P // 2, 2, k - 1, 0.0, momentum, ref_fnw=ref,
                                            ref_tolerance=0.0, return_distance=True)
    assert k1 == k - 1 and d1 > tol
