"""CPU model of the symmetric-spectrum gridding iteration (gtom_b200/csrc/
gridsym.cu), written with the kernels' own index logic, against numpy's full
C2R -> blob -> R2C of the cuFFT path (RecFourier.cu:158-171), and of its
final map (three passes keeping only the crop) against irfftn and the crop
(RecFourier.cu:175-216, Padding.cu:22-42).

It pins what the GPU kernels rely on: that a real half spectrum's transforms
stay Hermitian in z, so the planes z <= P/2 carry the whole iteration; the
pre- and post-twiddles of the half-length real transforms; the four-step
decomposition with thread t holding elements t + N2 m before and after; and
the Hermitian partners H - k (element N1-1-m of thread N2-t, or element N1-m
/ the extra element H of thread 0)."""
import numpy as np
import pytest

SPLITS = {16: (4, 4), 32: (8, 4), 48: (12, 4), 64: (8, 8), 96: (24, 4), 128: (16, 8), 192: (24, 8)}


def e(x):
    return np.exp(2j * np.pi * x)


def four_step(cols, inverse):
    """The kernels' four-step transform of each row of `cols` (N = N1 N2):
    thread t holds v[t][m] = x[t + N2 m]; an N1-point DFT over m, the
    twiddle e(-+t k1 / N), the exchange (thread t takes k1 = t + N2 j), and
    N2-point DFTs over the threads; thread t then holds X[k1 + N1 k2] at
    m' = j + (N1/N2) k2, which is X[t + N2 m'] (checked)."""
    n = cols.shape[-1]
    n1, n2 = SPLITS[n]
    jc = n1 // n2
    for t in range(n2):
        for j in range(jc):
            for k2 in range(n2):
                assert (t + n2 * j) + n1 * k2 == t + n2 * (j + jc * k2)
    sg = 1 if inverse else -1
    v = cols.reshape(-1, n1, n2).transpose(0, 2, 1)  # v[c, t, m] = x[c, t + N2 m]
    f1 = e(sg * np.outer(np.arange(n1), np.arange(n1)) / n1)
    y = v @ f1  # y[c, t, k1]
    y = y * e(sg * np.outer(np.arange(n2), np.arange(n1)) / n)
    f2 = e(sg * np.outer(np.arange(n2), np.arange(n2)) / n2)
    z = np.einsum("cnk,nq->ckq", y, f2)  # z[c, k1, k2] = X[k1 + N1 k2]
    return z.transpose(0, 2, 1).reshape(cols.shape)


def partners(h, n2, n1):
    """For each k = t + N2 m: where the kernels find X(H - k) (pre-twiddle)
    and Z((H - k) mod H) (post-twiddle)."""
    pre, post = {}, {}
    for t in range(n2):
        for m in range(n1):
            k = t + n2 * m
            if t != 0:
                src = (n2 - t) + n2 * (n1 - 1 - m)
                pre[k] = post[k] = src
            else:
                pre[k] = h if m == 0 else n2 * (n1 - m)
                post[k] = 0 if m == 0 else n2 * (n1 - m)
    return pre, post


def c2r_rows(X, plus):
    """Hermitian half X(0..H) -> x(0..P-1) (unnormalised; PLUS: exp(+))."""
    h = X.shape[-1] - 1
    n1, n2 = SPLITS[h]
    pre, _ = partners(h, n2, n1)
    k = np.arange(h)
    xm = X[:, [pre[i] for i in k]]
    assert np.array_equal([pre[i] for i in k], h - k)
    sg = 1 if plus else -1
    a, b = X[:, :h] + np.conj(xm), X[:, :h] - np.conj(xm)
    z = four_step(a + 1j * e(sg * k / (2 * h)) * b, inverse=plus)
    out = np.empty((X.shape[0], 2 * h))
    out[:, 0::2], out[:, 1::2] = z.real, z.imag
    return out


def r2c_rows(x, plus):
    """Real x(0..P-1) -> Y(0..H) (PLUS: exp(+))."""
    h = x.shape[-1] // 2
    n1, n2 = SPLITS[h]
    _, post = partners(h, n2, n1)
    sg = 1 if plus else -1
    z = four_step(x[:, 0::2] + 1j * x[:, 1::2], inverse=plus)
    k = np.arange(h)
    km = [post[i] for i in k]
    assert np.array_equal(km, (h - k) % h)
    zm = z[:, km]
    out = np.empty((x.shape[0], h + 1), complex)
    out[:, :h] = 0.5 * (z + np.conj(zm)) - 0.5j * e(sg * k / (2 * h)) * (z - np.conj(zm))
    out[:, h] = z[:, 0].real - z[:, 0].imag
    return out


@pytest.mark.parametrize("P", [32, 64, 96, 128])
def test_symmetric_iteration_model_equals_full_transforms(P):
    rng = np.random.default_rng(P)
    H = P // 2
    # real half spectrum S[kz][ky][kx], symmetric on the kx = 0 and kx = H planes
    S = rng.standard_normal((P, P, H + 1))
    idx = (-np.arange(P)) % P
    for kx in (0, H):
        S[:, :, kx] = 0.5 * (S[:, :, kx] + S[idx][:, idx][:, :, kx])
    blob = rng.uniform(0.1, 1.0, (P, P, P))
    blob = 0.5 * (blob + blob[idx][:, idx][:, :, idx])  # radial blobs are point-symmetric

    # the cuFFT path: unnormalised C2R, x blob / P^3, R2C, real part
    conv = np.fft.irfftn(S.astype(complex), s=(P, P, P), axes=(0, 1, 2)) * P ** 3
    want = np.fft.rfftn(conv * blob / P ** 3, axes=(0, 1, 2)).real

    # z pass (first): per column (kx, ky), real-to-Hermitian along z with exp(+)
    cols = S.transpose(1, 2, 0).reshape(-1, P)          # (ky, kx) x kz
    T1 = r2c_rows(cols, plus=True).reshape(P, H + 1, H + 1).transpose(2, 0, 1)
    # y inverse: columns along y of W[z][y][x]
    W = T1.transpose(0, 2, 1).reshape(-1, P)
    W = four_step(W, inverse=True).reshape(H + 1, H + 1, P).transpose(0, 2, 1)
    # x pass: rows (z <= H, y): C2R, blob / P^3, R2C
    rows = W.reshape(-1, H + 1)
    f = c2r_rows(rows, plus=True)
    f = f * blob[:H + 1].reshape(-1, P) / P ** 3
    W = r2c_rows(f, plus=False).reshape(H + 1, P, H + 1)
    # y forward
    W = four_step(W.transpose(0, 2, 1).reshape(-1, P), inverse=False).reshape(H + 1, H + 1, P).transpose(0, 2, 1)
    # z pass: Hermitian-to-real along z with exp(-)
    cols = W.transpose(1, 2, 0).reshape(-1, H + 1)      # (y, x) x z
    got = c2r_rows(cols, plus=False).reshape(P, H + 1, P).transpose(2, 0, 1)
    assert np.abs(got - want).max() <= 1e-9 * np.abs(want).max()


@pytest.mark.parametrize("P,ori", [(32, 16), (64, 32), (64, 20), (96, 48), (96, 30)])
def test_final_map_model_equals_irfftn_crop(P, ori):
    """The final map's three passes (gridsym_final_{z,y,x}_kernel) with the
    kernels' transforms: the inverse transform along z keeping only the
    crop's planes, along y keeping only its rows, then the C2R along x with
    the x = 0 and x = P/2 terms taken as real, keeping the crop's x; equal to
    numpy's irfftn (unnormalised) cropped to the central ori^3 — on a
    spectrum that is not Hermitian anywhere, which irfftn's last-axis C2R
    treats the same way."""
    rng = np.random.default_rng(P + ori)
    H = P // 2
    S = rng.standard_normal((P, P, H + 1)) + 1j * rng.standard_normal((P, P, H + 1))  # [kz][ky][kx]
    off = P // 2 - ori // 2
    want = np.fft.irfftn(S, s=(P, P, P), axes=(0, 1, 2)) * P ** 3
    want = want[off:off + ori, off:off + ori, off:off + ori]
    # z pass: every (y, x) column along z, the crop's planes kept -> T[zc][y][x]
    cols = S.transpose(1, 2, 0).reshape(-1, P)
    T = four_step(cols, inverse=True).reshape(P, H + 1, P).transpose(2, 0, 1)[off:off + ori]
    # y pass: every (zc, x) column along y, the crop's rows kept -> T[zc][yc][x]
    cols = T.transpose(0, 2, 1).reshape(-1, P)
    T = four_step(cols, inverse=True).reshape(ori, H + 1, P).transpose(0, 2, 1)[:, off:off + ori]
    # x pass: C2R of each kept row, the crop's x
    rows = T.reshape(-1, H + 1).copy()
    rows[:, 0] = rows[:, 0].real
    rows[:, H] = rows[:, H].real
    got = c2r_rows(rows, plus=True).reshape(ori, ori, P)[:, :, off:off + ori]
    assert np.abs(got - want).max() <= 1e-9 * np.abs(want).max()
