"""Test infrastructure: a float64 numpy restatement of the learned gridding
warm start (gtom_b200/csrc/mlp.cuh, mlp.cu) and of the momentum form of the
gridding iteration (gtom_b200/csrc/gridding.cu, grid_update_momentum_kernel).

Neither exists in the reference, whose gridding always starts from the
sphere mask and applies the plain update (src/Reconstruction/RecFourier.cu:
149-167, 287-308); this file is the CPU definition of the extension that
the CUDA kernels are checked against: features, forward pass, analytic
gradients (themselves checked here against finite differences), Adam, the
predicted start with its Hermitian symmetrisation, and the iteration.
Only tests may import it.
"""
from __future__ import annotations

import numpy as np

N_IN, N_HID = 28, 64
OFF_SHIFT, OFF_SCALE = 0, N_IN
OFF_W1 = 2 * N_IN
OFF_B1 = OFF_W1 + N_HID * N_IN
OFF_W2 = OFF_B1 + N_HID
OFF_B2 = OFF_W2 + N_HID * N_HID
OFF_W3 = OFF_B2 + N_HID
OFF_B3 = OFF_W3 + N_HID
N_PARAMS = OFF_B3 + 1
WEIGHT_FLOOR = 1e-6


def unpack(p: np.ndarray):
    p = np.asarray(p, np.float64)
    return dict(shift=p[OFF_SHIFT:OFF_SHIFT + N_IN], scale=p[OFF_SCALE:OFF_SCALE + N_IN],
                W1=p[OFF_W1:OFF_B1].reshape(N_HID, N_IN), b1=p[OFF_B1:OFF_W2],
                W2=p[OFF_W2:OFF_B2].reshape(N_HID, N_HID), b2=p[OFF_B2:OFF_W3],
                W3=p[OFF_W3:OFF_B3], b3=p[OFF_B3])


def init_params(rng, shift=None, scale=None) -> np.ndarray:
    """He-initialised weights, zero biases, the given input standardisation."""
    p = np.zeros(N_PARAMS, np.float64)
    p[OFF_SHIFT:OFF_SHIFT + N_IN] = 0 if shift is None else shift
    p[OFF_SCALE:OFF_SCALE + N_IN] = 1 if scale is None else scale
    p[OFF_W1:OFF_B1] = rng.normal(0, np.sqrt(2 / N_IN), N_HID * N_IN)
    p[OFF_W2:OFF_B2] = rng.normal(0, np.sqrt(2 / N_HID), N_HID * N_HID)
    p[OFF_W3:OFF_B3] = rng.normal(0, np.sqrt(1 / N_HID), N_HID)
    return p


def voxel_xyz(e, P: int):
    rowlen = P // 2 + 1
    e = np.asarray(e, np.int64)
    return e % rowlen, (e // rowlen) % P, e // (rowlen * P)


def features(fw: np.ndarray, P: int, inv_scale: float, index) -> np.ndarray:
    """Raw features (n, 28) of voxels `index` (flat element indices) of the
    decentred half grid fw ((P/2+1) * P * P values): log(Fw/s + 1e-6) of the
    3x3x3 neighbours in (dz, dy, dx) order, dx fastest, the x = -1 neighbour
    of the x = 0 plane being the Hermitian mate (1, -y, -z); then the radius
    over P/2."""
    fw = np.asarray(fw, np.float64).reshape(P, P, P // 2 + 1)
    x, y, z = voxel_xyz(index, P)
    out = np.empty((len(x), N_IN), np.float64)
    k = 0
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                xx, yy, zz = x + dx, y + dy, z + dz
                neg = xx < 0
                xx = np.where(neg, -xx, xx)
                yy = np.where(neg, -yy, yy) % P
                zz = np.where(neg, -zz, zz) % P
                xx = np.minimum(xx, P // 2)
                out[:, k] = np.log(fw[zz, yy, xx] * inv_scale + WEIGHT_FLOOR)
                k += 1
    yp = np.where(y < P // 2 + 1, y, y - P)
    zp = np.where(z < P // 2 + 1, z, z - P)
    out[:, 27] = np.sqrt(x * x + yp * yp + zp * zp) / (P // 2)
    return out


def forward(p: np.ndarray, feats: np.ndarray, cache: bool = False):
    q = unpack(p)
    X = (np.asarray(feats, np.float64) - q["shift"]) * q["scale"]
    A1 = X @ q["W1"].T + q["b1"]
    H1 = np.maximum(A1, 0)
    A2 = H1 @ q["W2"].T + q["b2"]
    H2 = np.maximum(A2, 0)
    out = H2 @ q["W3"] + q["b3"]
    if cache:
        return out, (X, A1, H1, A2, H2)
    return out


def gradients(p: np.ndarray, feats, targets, weights, loss_scale: float):
    """(loss, dloss/dp) of L = loss_scale * sum w (out - t)^2; the input
    standardisation entries of the gradient are zero."""
    q = unpack(p)
    out, (X, A1, H1, A2, H2) = forward(p, feats, cache=True)
    d = out - np.asarray(targets, np.float64)
    w = np.asarray(weights, np.float64)
    loss = loss_scale * np.sum(w * d * d)
    dout = 2 * loss_scale * w * d
    g = np.zeros(N_PARAMS, np.float64)
    g[OFF_W3:OFF_B3] = dout @ H2
    g[OFF_B3] = dout.sum()
    G2 = dout[:, None] * q["W3"][None, :] * (A2 > 0)
    g[OFF_W2:OFF_B2] = (G2.T @ H1).ravel()
    g[OFF_B2:OFF_W3] = G2.sum(0)
    G1 = (G2 @ q["W2"]) * (A1 > 0)
    g[OFF_W1:OFF_B1] = (G1.T @ X).ravel()
    g[OFF_B1:OFF_W2] = G1.sum(0)
    return loss, g


def adam(p, grad, m, v, step: int, lr: float, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam step on the trained entries; returns (p, m, v)."""
    p, m, v = (np.array(a, np.float64) for a in (p, m, v))
    s = slice(OFF_W1, N_PARAMS)
    g = np.asarray(grad, np.float64)[s]
    m[s] = beta1 * m[s] + (1 - beta1) * g
    v[s] = beta2 * v[s] + (1 - beta2) * g * g
    mh = m[s] / (1 - beta1 ** step)
    vh = v[s] / (1 - beta2 ** step)
    p[s] -= lr * mh / (np.sqrt(vh) + eps)
    return p, m, v


def weight_scale(fw: np.ndarray, P: int, maskr2: int) -> float:
    """Mean of the non-zero weights with x^2 + y^2 + z^2 < maskr2."""
    e = np.arange((P // 2 + 1) * P * P)
    x, y, z = voxel_xyz(e, P)
    yp = np.where(y < P // 2 + 1, y, y - P)
    zp = np.where(z < P // 2 + 1, z, z - P)
    fw = np.asarray(fw, np.float64).ravel()
    sel = (fw > 0) & (x * x + yp * yp + zp * zp < maskr2)
    return fw[sel].sum() / sel.sum() if sel.any() else 1.0


def predict_start(p: np.ndarray, fw: np.ndarray, P: int, maskr2: int) -> np.ndarray:
    """The predicted gridding start (mlp_start_kernel): 0 outside the
    sphere, 1 where Fw = 0 inside it, exp(out) / s elsewhere, the two
    Hermitian mates of the x = 0 plane sharing the mean of their outputs."""
    fw = np.asarray(fw, np.float64).ravel()
    e = np.arange(fw.size)
    x, y, z = voxel_xyz(e, P)
    yp = np.where(y < P // 2 + 1, y, y - P)
    zp = np.where(z < P // 2 + 1, z, z - P)
    inside = x * x + yp * yp + zp * zp < maskr2
    s = weight_scale(fw, P, maskr2)
    start = np.where(inside, 1.0, 0.0)
    sel = np.nonzero(inside & (fw > 0))[0]
    out = forward(p, features(fw, P, 1 / s, sel))
    x0 = (x[sel] == 0) & ((yp[sel] != 0) | (zp[sel] != 0))
    if x0.any():
        my = (-y[sel][x0]) % P
        mz = (-z[sel][x0]) % P
        mate = mz * (P * (P // 2 + 1)) + my * (P // 2 + 1)
        out[x0] = 0.5 * (out[x0] + forward(p, features(fw, P, 1 / s, mate)))
    start[sel] = np.minimum(1e20, np.exp(out) / s)
    return start


def gridding_iterations(fw: np.ndarray, start: np.ndarray, P: int, pad: int, iterations: int,
                        momentum: float = 0.0, blobradius: float = 1.9, blobalpha: float = 15.0):
    """Iterates the gridding update on the decentred half grid of P from
    `start` (momentum 0: RecFourier.cu:287-308's update; else the momentum
    form), returning (Fnewweight, list of the relative changes)."""
    from oracle import oracle as O
    nsamp = 10000
    table = O.kb_table(blobradius * pad, blobalpha, 0, nsamp)
    k = np.arange(P)
    kp = np.where(k < P // 2, k, k - P).astype(np.float64)
    r = np.sqrt(kp[:, None, None] ** 2 + kp[None, :, None] ** 2 + kp[None, None, :] ** 2) / P / (0.5 / nsamp)
    blob = table[np.minimum(nsamp - 1, r.astype(np.int64))]
    Fw = np.asarray(fw, np.float64).reshape(P, P, P // 2 + 1)
    F = np.asarray(start, np.float64).reshape(P, P, P // 2 + 1).copy()
    V = F.copy()
    changes = []
    for _ in range(iterations):
        c = np.fft.rfftn(np.fft.irfftn(Fw * V, s=(P, P, P), axes=(0, 1, 2)) * blob, axes=(0, 1, 2)).real
        new = np.minimum(1e20, V / np.maximum(1e-4, c))
        if momentum > 0:
            ok = (F > 0) & (new > 0)
            ratio = np.where(ok, new / np.where(ok, F, 1), 1)
            V = np.where(ok, np.minimum(1e20, new * ratio ** momentum), new)
        else:
            V = new
        num = np.sum((Fw * (new - F)) ** 2)
        den = np.sum((Fw * F) ** 2)
        changes.append(np.sqrt(num / den) if den > 0 else 0.0)
        F = new
    return F.ravel(), changes
