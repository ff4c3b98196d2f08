"""Learned warm start of the gridding reconstruction: training data,
training loop and the trained parameters.

The per-voxel MLP (gtom_b200/csrc/mlp.cuh) predicts the converged gridding
correction Fnewweight of d_ReconstructGridding's iteration
(src/Reconstruction/RecFourier.cu:158-168) from the 27 log-weights around
each voxel and its radius.  Training pairs come from the library itself:
sampling-weight volumes are made by backprojecting CTF^2 weights of
synthetic orientation distributions (d_rlnBackproject without data), and
their converged corrections by running the gridding iteration to a tight
tolerance (gtomrln_gridding_weights; the momentum form has the same fixed
points and gets there in far fewer iterations).  Training runs on the GPU
through the library's own forward/backward kernel (gtomrln_mlp_train_batch)
and Adam kernel (gtomrln_mlp_adam); torch only holds the device buffers and
draws the minibatch indices.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np
import torch

from . import _lib, synth
from .relion import d_rlnBackproject, gridding_weights, matrices_from_angles, mlp_param_count

DATA_DIR = Path(__file__).resolve().parent / "data"
N_IN = 28
N_HID = 64
OFF_W1 = 2 * N_IN
LOG_FLOOR = -12.0


def params_path(box: int) -> Path:
    return DATA_DIR / f"warmstart_mlp_box{box}.npy"


def load_params(box: int, device="cuda") -> torch.Tensor | None:
    """The trained parameter block for a box size, or None if none was saved."""
    p = params_path(box)
    if not p.exists():
        return None
    a = np.load(p).astype(np.float32)
    if a.size != mlp_param_count():
        raise ValueError(f"{p} holds {a.size} values, expected {mlp_param_count()}")
    return torch.from_numpy(a).to(device)


def save_params(params: torch.Tensor, box: int) -> Path:
    DATA_DIR.mkdir(parents=True, exist_ok=True)
    p = params_path(box)
    np.save(p, params.detach().float().cpu().numpy())
    return p


# --------------------------------------------------------------- sampling --
@dataclass
class Distribution:
    """One synthetic orientation distribution: vMF lobes plus a uniform part."""
    views: int
    lobes: int
    kappa_range: tuple
    uniform_frac: float
    seed: int


def random_distribution(rng, views_range=(5000, 200000), lobes_range=(1, 5),
                        kappa_range=(0.0, 50.0), uniform_range=(0.0, 0.5)) -> Distribution:
    return Distribution(views=int(rng.integers(views_range[0], views_range[1] + 1)),
                        lobes=int(rng.integers(lobes_range[0], lobes_range[1] + 1)),
                        kappa_range=tuple(kappa_range),
                        uniform_frac=float(rng.uniform(*uniform_range)),
                        seed=int(rng.integers(1 << 31)))


def sampling_weights(box: int, dist: Distribution, pad: int = 2, device="cuda",
                     chunk: int = 8192) -> torch.Tensor:
    """Centred weight half volume of P + 1 (P = box * pad) accumulated from
    the CTF^2 weights of dist.views particles (300 kV, Cs 2.7 mm, 1 A/px,
    defocus U(0.5, 3) um, astigmatism U(0, 0.1) um) at the distribution's
    orientations."""
    rng = np.random.default_rng(dist.seed)
    n = box
    D = box * pad + 1
    nvol = (D // 2 + 1) * D * D
    acc = torch.zeros(nvol, dtype=torch.float32, device=device)
    ang = synth.vmf_mixture_angles(rng, dist.views, lobes=dist.lobes, kappa_range=dist.kappa_range,
                                   uniform_frac=dist.uniform_frac)
    mats = torch.from_numpy(matrices_from_angles(ang, float(pad))).to(device)
    e = (n // 2 + 1) * n
    for c0 in range(0, dist.views, chunk):
        c = min(chunk, dist.views - c0)
        df = torch.from_numpy(rng.uniform(0.5, 3.0, c).astype(np.float32)).to(device)
        da = torch.from_numpy(rng.uniform(0.0, 0.1, c).astype(np.float32)).to(device)
        aa = torch.from_numpy(rng.uniform(0.0, np.pi, c).astype(np.float32)).to(device)
        ctf = synth.ctf_half(n, df, da, aa).reshape(c, e)
        w = (ctf * ctf).contiguous()
        d_rlnBackproject(None, acc, (D, D, D), None, w.reshape(-1), (n, n, 1), n // 2,
                         mats[c0:c0 + c].reshape(-1), None, (1, 0, 0, 1), 0.0, False, False, c)
    return acc


def sphere_mask(P: int, device) -> torch.Tensor:
    """r^2 < (P/2)^2 on the decentred half grid of P (the gridding sphere)."""
    z = torch.arange(P, device=device)
    zp = torch.where(z < P // 2 + 1, z, z - P)
    x = torch.arange(P // 2 + 1, device=device)
    r2 = zp[:, None, None] ** 2 + zp[None, :, None] ** 2 + x[None, None, :] ** 2
    return (r2 < (P // 2) ** 2).reshape(-1)


def weighted_distance(fw: torch.Tensor, a: torch.Tensor, b: torch.Tensor) -> float:
    """||Fw (a - b)|| / ||Fw b||: the distance of gridding weights a from b
    in the measure of the convergence test."""
    fw = fw.double()
    num = torch.sum((fw * (a.double() - b.double())) ** 2)
    den = torch.sum((fw * b.double()) ** 2)
    return float(torch.sqrt(num / den)) if den > 0 else 0.0


# -------------------------------------------------------------- training --
@dataclass
class TrainingSet:
    """Stacks of the training volumes on the decentred half grid of P."""
    P: int
    fw: torch.Tensor          # (ndist * nc) sampling weights
    target: torch.Tensor      # log(Fnw * s), clamped at LOG_FLOOR
    weight: torch.Tensor      # loss weight (Fw Fnw)^2, mean 1 per distribution
    inv_scale: torch.Tensor   # (ndist,) 1 / s
    eligible: torch.Tensor    # int64 flat indices of trained voxels
    converged: list = field(default_factory=list)  # (iterations, change) per distribution


def make_training_set(weights: list, ori: int, pad: int = 2, tolerance: float = 1e-6,
                      max_iterations: int = 5000, momentum: float = 0.9) -> TrainingSet:
    """Converged gridding weights of each centred weight volume (dims P+1)
    and the tensors the training kernel reads."""
    P = ori * pad
    D = P + 1
    nc = (P // 2 + 1) * P * P
    dev = weights[0].device
    mask = sphere_mask(P, dev)
    nd = len(weights)
    fw_all = torch.empty(nd * nc, dtype=torch.float32, device=dev)
    tg_all = torch.empty(nd * nc, dtype=torch.float32, device=dev)
    lw_all = torch.zeros(nd * nc, dtype=torch.float32, device=dev)
    inv = torch.empty(nd, dtype=torch.float32, device=dev)
    elig = []
    conv = []
    for d, w in enumerate(weights):
        fw = fw_all[d * nc:(d + 1) * nc]
        fnw, _, it, ch, _ = gridding_weights(w, (D, D, D), ori, pad, max_iterations, tolerance, momentum,
                                             fw_out=fw)
        conv.append((it, ch))
        sel = mask & (fw > 0)
        s = float(fw[sel].double().mean()) if bool(sel.any()) else 1.0
        inv[d] = 1.0 / s
        tg_all[d * nc:(d + 1) * nc] = torch.log(torch.clamp(fnw * s, min=math.exp(LOG_FLOOR)))
        lw = torch.where(sel, (fw * fnw) ** 2, torch.zeros_like(fw))
        m = lw[sel].double().mean() if bool(sel.any()) else 0.0
        if m > 0:
            lw_all[d * nc:(d + 1) * nc] = (lw / m).float()
        elig.append(torch.nonzero(sel).squeeze(1) + d * nc)
    return TrainingSet(P=P, fw=fw_all, target=tg_all, weight=lw_all, inv_scale=inv,
                       eligible=torch.cat(elig), converged=conv)


def volume_features(ts: TrainingSet, index: torch.Tensor) -> torch.Tensor:
    """Raw features (n, 28) of stack voxels `index` (int64 CUDA tensor)."""
    n = index.numel()
    out = torch.empty((n, N_IN), dtype=torch.float32, device=index.device)
    _lib.call("gtomrln_mlp_volume_features", C.c_void_p(ts.fw.data_ptr()), ts.P,
              C.c_void_p(ts.inv_scale.data_ptr()), C.c_void_p(index.data_ptr()), n,
              C.c_void_p(out.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return out


def init_params(ts: TrainingSet, seed: int = 0, sample: int = 200000) -> torch.Tensor:
    """He-initialised parameters whose input standardisation is the mean and
    standard deviation of the features of a random sample of trained voxels."""
    g = torch.Generator(device=ts.fw.device)
    g.manual_seed(seed)
    pick = ts.eligible[torch.randint(ts.eligible.numel(), (min(sample, ts.eligible.numel()),),
                                     generator=g, device=ts.fw.device)]
    f = volume_features(ts, pick).double()
    mu = f.mean(0)
    sd = f.std(0).clamp_min(1e-3)
    rng = np.random.default_rng(seed)
    p = np.zeros(mlp_param_count(), np.float32)
    p[:N_IN] = mu.cpu().numpy()
    p[N_IN:2 * N_IN] = (1.0 / sd).cpu().numpy()
    o = OFF_W1
    p[o:o + N_HID * N_IN] = rng.normal(0, math.sqrt(2 / N_IN), N_HID * N_IN)
    o += N_HID * N_IN + N_HID
    p[o:o + N_HID * N_HID] = rng.normal(0, math.sqrt(2 / N_HID), N_HID * N_HID)
    o += N_HID * N_HID + N_HID
    p[o:o + N_HID] = rng.normal(0, math.sqrt(1 / N_HID), N_HID)
    return torch.from_numpy(p).to(ts.fw.device)


def train(ts: TrainingSet, params: torch.Tensor, steps: int = 2000, batch: int = 32768,
          lr: float = 2e-3, lr_final: float = 1e-4, seed: int = 0, log_every: int = 0) -> list:
    """Adam (cosine learning-rate decay) on the weighted squared error of the
    log correction; returns the minibatch losses read back every log_every
    steps and at the end."""
    dev = params.device
    n = mlp_param_count()
    grad = torch.zeros(n, dtype=torch.float32, device=dev)
    m = torch.zeros(n, dtype=torch.float32, device=dev)
    v = torch.zeros(n, dtype=torch.float32, device=dev)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    losses = []
    ne = ts.eligible.numel()
    for step in range(1, steps + 1):
        idx = ts.eligible[torch.randint(ne, (batch,), generator=g, device=dev)]
        loss.zero_()
        _lib.call("gtomrln_mlp_train_batch", C.c_void_p(params.data_ptr()), C.c_void_p(ts.fw.data_ptr()),
                  C.c_void_p(ts.target.data_ptr()), C.c_void_p(ts.weight.data_ptr()),
                  C.c_void_p(ts.inv_scale.data_ptr()), ts.P, C.c_void_p(idx.data_ptr()), batch,
                  C.c_float(1.0 / batch), C.c_void_p(grad.data_ptr()), C.c_void_p(loss.data_ptr()), stream)
        t = (step - 1) / max(1, steps - 1)
        rate = lr_final + 0.5 * (lr - lr_final) * (1 + math.cos(math.pi * t))
        _lib.call("gtomrln_mlp_adam", C.c_void_p(params.data_ptr()), C.c_void_p(grad.data_ptr()),
                  C.c_void_p(m.data_ptr()), C.c_void_p(v.data_ptr()), step, C.c_float(rate),
                  C.c_float(0.9), C.c_float(0.999), C.c_float(1e-8), stream)
        if (log_every and step % log_every == 0) or step == steps:
            losses.append(float(loss.item()))
    return losses
