"""CPU checks of the warm-start oracle (oracle/mlp_oracle.py): its analytic
gradients against finite differences, Adam, the Hermitian symmetry of the
features and of the predicted start, and that the momentum form of the
gridding iteration reaches the plain iteration's fixed point."""
import numpy as np
import pytest

from oracle import mlp_oracle as M
from oracle import oracle as O
from tests.synthdata import random_angles


def _params(rng):
    p = M.init_params(rng, shift=rng.normal(0, 1, M.N_IN), scale=rng.uniform(0.5, 2, M.N_IN))
    p[M.OFF_B1:M.OFF_W2] = rng.normal(0, 0.1, M.N_HID)
    p[M.OFF_B2:M.OFF_W3] = rng.normal(0, 0.1, M.N_HID)
    return p


def test_layout_matches_the_kernel_block():
    assert M.N_PARAMS == 6137
    assert (M.OFF_W1, M.OFF_B1, M.OFF_W2, M.OFF_B2, M.OFF_W3, M.OFF_B3) == (56, 1848, 1912, 6008, 6072, 6136)


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(11)
    p = _params(rng)
    n = 40
    f = rng.normal(0, 1, (n, M.N_IN))
    t = rng.normal(0, 1, n)
    w = rng.uniform(0.1, 2, n)
    loss, g = M.gradients(p, f, t, w, 1 / n)
    idx = np.concatenate([rng.choice(np.arange(M.OFF_W1, M.N_PARAMS), 60, replace=False), [M.OFF_B3]])
    h = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += h
        lp, _ = M.gradients(q, f, t, w, 1 / n)
        q[i] -= 2 * h
        lm, _ = M.gradients(q, f, t, w, 1 / n)
        fd = (lp - lm) / (2 * h)
        assert g[i] == pytest.approx(fd, rel=1e-5, abs=1e-8), i
    assert np.all(g[:M.OFF_W1] == 0)


def test_adam_step_matches_its_definition():
    rng = np.random.default_rng(3)
    p = _params(rng)
    g = rng.normal(0, 1, M.N_PARAMS)
    m = np.zeros(M.N_PARAMS)
    v = np.zeros(M.N_PARAMS)
    p1, m1, v1 = M.adam(p, g, m, v, 1, 1e-3)
    s = slice(M.OFF_W1, None)
    # first step: m/(1-b1) = g, v/(1-b2) = g^2, so the step is lr * sign(g) (up to eps)
    np.testing.assert_allclose(p1[s], p[s] - 1e-3 * g[s] / (np.abs(g[s]) + 1e-8), rtol=1e-12)
    np.testing.assert_array_equal(p1[:M.OFF_W1], p[:M.OFF_W1])


def _weights(P, views=300, seed=2):
    rng = np.random.default_rng(seed)
    n = P // 2
    mats = O.matrices_f64(random_angles(rng, views), 2.0).astype(np.float32)
    e = (n // 2 + 1) * n
    w = rng.uniform(0.2, 1.0, (views, e)).astype(np.float32)
    D = P + 1
    vol = np.zeros((D // 2 + 1) * D * D, np.float32)
    O.backproject(None, vol, D, None, w, n, n // 2, mats, decentered=False, fp32=True)
    return vol, D


def _decentred(vol, P, D):
    return O._decenter(vol.astype(np.float64), P, (D, D, D)).real.ravel()


def test_features_see_hermitian_mates_on_the_x0_plane():
    P = 16
    vol, D = _weights(P)
    fw = _decentred(vol, P, D)
    rowlen = P // 2 + 1
    y, z = 3, 5
    a = z * P * rowlen + y * rowlen
    b = ((-z) % P) * P * rowlen + ((-y) % P) * rowlen
    fa, fb = M.features(fw, P, 1.0, [a, b])
    # neighbour (dz, dy, dx) of a voxel on x = 0 is neighbour (-dz, -dy, -dx)
    # of its Hermitian mate
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                ka = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)
                kb = (-dz + 1) * 9 + (-dy + 1) * 3 + (-dx + 1)
                assert fa[ka] == fb[kb]
    assert fa[27] == fb[27]


def test_predicted_start_is_hermitian_on_x0():
    P = 16
    vol, D = _weights(P)
    fw = _decentred(vol, P, D)
    p = _params(np.random.default_rng(9))
    s = M.predict_start(p, fw, P, (P // 2) ** 2).reshape(P, P, P // 2 + 1)
    idx = (-np.arange(P)) % P
    np.testing.assert_array_equal(s[:, :, 0], s[idx][:, idx][:, :, 0])
    assert (s > 0).sum() > 0 and np.all(np.isfinite(s))


def test_momentum_reaches_the_plain_fixed_point():
    P = 24
    vol, D = _weights(P, views=400)
    fw = _decentred(vol, P, D)
    start = M.predict_start(M.init_params(np.random.default_rng(0)), np.zeros_like(fw), P, (P // 2) ** 2)
    plain_ref, _ = M.gridding_iterations(fw, start, P, 2, 20000)
    mom_ref, _ = M.gridding_iterations(fw, start, P, 2, 3000, momentum=0.9)

    def dist(a, ref):
        return np.sqrt(np.sum((fw * (a - ref)) ** 2) / np.sum((fw * ref) ** 2))
    assert dist(mom_ref, plain_ref) < 1e-4  # the same fixed point
    plain, ch_plain = M.gridding_iterations(fw, start, P, 2, 150)
    mom, ch_mom = M.gridding_iterations(fw, start, P, 2, 150, momentum=0.9)
    assert dist(mom, plain_ref) < 0.1 * dist(plain, plain_ref)
    assert ch_mom[-1] < ch_plain[-1]


def test_warm_start_summary_of_the_converged_criterion():
    """gtom_b200.warmstart.summarise: medians per mode, and the speed-up to
    the converged weights taken only over distributions where both the mode
    and the plain run reached the criterion (a run that did not is counted
    in `reached`, not timed)."""
    from gtom_b200 import warmstart as W

    def mode(it, ms, conv_it, conv_ms, reached=True):
        return {"iterations": it, "ms": ms, "distance_to_converged": 0.01, "fsc_min_to_plain": 1.0,
                "fsc_min_to_converged": 0.99, "warm_used": True,
                "to_converged": {"iterations": conv_it, "distance": 1e-4 if reached else 3e-4,
                                 "reached": reached, **({"ms": conv_ms} if reached else {})}}

    rows = [{"plain": mode(300, 100.0, 3000, 1000.0), "momentum": mode(90, 30.0, 300, 100.0)},
            {"plain": mode(280, 90.0, 3400, 1200.0), "momentum": mode(80, 30.0, 320, 80.0)},
            {"plain": mode(290, 95.0, 8000, None, reached=False), "momentum": mode(85, 30.0, 310, 90.0)}]
    out = W.summarise(rows)
    assert out["plain"]["to_converged"]["reached"] == 2 and out["plain"]["to_converged"]["of"] == 3
    assert out["momentum"]["to_converged"]["reached"] == 3
    assert out["momentum"]["to_converged"]["iterations"] == 310
    # speed-ups over the two rows where plain reached it: 10x and 15x
    assert out["momentum"]["to_converged"]["speedup_vs_plain"] == pytest.approx(12.5)
    assert out["plain"]["to_converged"]["speedup_vs_plain"] == pytest.approx(1.0)
    assert out["momentum"]["speedup_vs_plain"] == pytest.approx(np.median([100 / 30, 90 / 30, 95 / 30]))
