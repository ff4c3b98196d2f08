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


def insert_distribution(box: int, dist: Distribution, pad: int = 2, device="cuda",
                        chunk: int = 8192, volft: torch.Tensor | None = None):
    """Centred half volumes of P + 1 (P = box * pad) accumulated from
    dist.views particles at the distribution's orientations, each with a CTF
    (300 kV, Cs 2.7 mm, 1 A/px, defocus U(0.5, 3) um, astigmatism
    U(0, 0.1) um): the CTF^2 weights, and, when volft (the decentred padded
    half transform of a box^3 volume) is given, the CTF-weighted central
    slices of it.  Returns (data or None, weights)."""
    from .relion import d_rlnProject
    rng = np.random.default_rng(dist.seed)
    n = box
    P = box * pad
    D = P + 1
    nvol = (D // 2 + 1) * D * D
    acc = torch.zeros(nvol, dtype=torch.float32, device=device)
    data = None if volft is None else torch.zeros(nvol, dtype=torch.complex64, device=device)
    ang = synth.vmf_mixture_angles(rng, dist.views, lobes=dist.lobes, kappa_range=dist.kappa_range,
                                   uniform_frac=dist.uniform_frac)
    mats = torch.from_numpy(matrices_from_angles(ang, float(pad))).to(device)
    e = (n // 2 + 1) * n
    proj = None if volft is None else torch.empty(min(chunk, dist.views) * e, dtype=torch.complex64,
                                                  device=device)
    for c0 in range(0, dist.views, chunk):
        c = min(chunk, dist.views - c0)
        m = mats[c0:c0 + c].reshape(-1)
        df = torch.from_numpy(rng.uniform(0.5, 3.0, c).astype(np.float32)).to(device)
        da = torch.from_numpy(rng.uniform(0.0, 0.1, c).astype(np.float32)).to(device)
        aa = torch.from_numpy(rng.uniform(0.0, np.pi, c).astype(np.float32)).to(device)
        ctf = synth.ctf_half(n, df, da, aa).reshape(c, e)
        w = (ctf * ctf).contiguous()
        slices = None
        if volft is not None:
            d_rlnProject(volft, (P, P, P), proj, (n, n, 1), n // 2, m, c)
            slices = (proj[:c * e].reshape(c, e) * ctf).contiguous().reshape(-1)
        d_rlnBackproject(data, acc, (D, D, D), slices, w.reshape(-1), (n, n, 1), n // 2, m, None,
                         (1, 0, 0, 1), 0.0, False, False, c)
    return data, acc


def sampling_weights(box: int, dist: Distribution, pad: int = 2, device="cuda",
                     chunk: int = 8192) -> torch.Tensor:
    """The CTF^2 weight volume of insert_distribution."""
    return insert_distribution(box, dist, pad, device, chunk)[1]


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


def make_training_set(weights, ori: int, pad: int = 2, tolerance: float = 1e-6,
                      max_iterations: int = 5000, momentum: float = 0.9, count: int | None = None,
                      device="cuda", max_voxels: int | None = None) -> TrainingSet:
    """Converged gridding weights of each centred weight volume (dims P+1)
    and the tensors the training kernel reads.  weights: a list of volumes,
    or any iterable of `count` volumes (made one at a time)."""
    P = ori * pad
    D = P + 1
    nc = (P // 2 + 1) * P * P
    nd = len(weights) if count is None else int(count)
    dev = torch.device(device)
    mask = sphere_mask(P, dev)
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
        idx = torch.nonzero(sel).squeeze(1)
        if max_voxels and idx.numel() > max_voxels:  # a random subset keeps the index list small
            g = torch.Generator(device=dev)
            g.manual_seed(d)
            idx = idx[torch.randperm(idx.numel(), generator=g, device=dev)[:max_voxels]]
        elig.append(idx + d * nc)
    return TrainingSet(P=P, fw=fw_all, target=tg_all, weight=lw_all, inv_scale=inv,
                       eligible=torch.cat(elig), converged=conv)


@dataclass
class FeatureRows:
    """Training rows sampled from many distributions: raw features (n, 28),
    targets log(Fnw * s) and loss weights (mean 1 per distribution)."""
    X: torch.Tensor
    target: torch.Tensor
    weight: torch.Tensor
    converged: list = field(default_factory=list)


def make_feature_rows(weights, ori: int, pad: int = 2, rows_per_dist: int = 60000, tolerance: float = 1e-6,
                      max_iterations: int = 5000, momentum: float = 0.9, count: int | None = None,
                      device="cuda", seed: int = 0) -> FeatureRows:
    """As make_training_set, but keeping only `rows_per_dist` randomly chosen
    trained voxels of each distribution, as feature rows, so that thousands
    of distributions fit in memory (a full stack takes ~100 MB per
    distribution at P = 256; 60 000 rows take 7 MB)."""
    P = ori * pad
    D = P + 1
    nd = len(weights) if count is None else int(count)
    dev = torch.device(device)
    mask = sphere_mask(P, dev)
    X = torch.zeros((nd * rows_per_dist, N_IN), dtype=torch.float32, device=dev)
    T = torch.zeros(nd * rows_per_dist, dtype=torch.float32, device=dev)
    Wt = torch.zeros(nd * rows_per_dist, dtype=torch.float32, device=dev)
    g = torch.Generator(device=dev)
    conv = []
    for d, w in enumerate(weights):
        fnw, fw, it, ch, _ = gridding_weights(w, (D, D, D), ori, pad, max_iterations, tolerance, momentum)
        conv.append((it, ch))
        sel = mask & (fw > 0)
        idx = torch.nonzero(sel).squeeze(1)
        if idx.numel() == 0:
            continue
        s = float(fw[sel].double().mean())
        g.manual_seed(seed * 100003 + d)
        pick = idx[torch.randint(idx.numel(), (rows_per_dist,), generator=g, device=dev)]
        one = TrainingSet(P=P, fw=fw, target=fnw, weight=fnw, inv_scale=torch.tensor([1.0 / s], device=dev),
                          eligible=pick)
        lo = d * rows_per_dist
        X[lo:lo + rows_per_dist] = volume_features(one, pick)
        T[lo:lo + rows_per_dist] = torch.log(torch.clamp(fnw[pick] * s, min=math.exp(LOG_FLOOR)))
        lw = (fw[sel] * fnw[sel]) ** 2
        m = float(lw.double().mean())
        if m > 0:
            Wt[lo:lo + rows_per_dist] = (fw[pick] * fnw[pick]) ** 2 / m
    return FeatureRows(X=X, target=T, weight=Wt, converged=conv)


def init_params_rows(rows: FeatureRows, seed: int = 0, sample: int = 200000) -> torch.Tensor:
    """init_params on feature rows."""
    g = torch.Generator(device=rows.X.device)
    g.manual_seed(seed)
    pick = torch.randint(rows.X.shape[0], (min(sample, rows.X.shape[0]),), generator=g, device=rows.X.device)
    f = rows.X[pick].double()
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
    return torch.from_numpy(p).to(rows.X.device)


def train_rows(rows: FeatureRows, params: torch.Tensor, steps: int = 3000, batch: int = 32768,
               lr: float = 2e-3, lr_final: float = 1e-4, seed: int = 0, log_every: int = 0) -> list:
    """train() on feature rows: minibatches gathered from the rows, gradients
    by the library's hand-written backward kernel (gtomrln_mlp_gradients)."""
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
    nr = rows.X.shape[0]
    for step in range(1, steps + 1):
        idx = torch.randint(nr, (batch,), generator=g, device=dev)
        xb, tb, wb = rows.X[idx].contiguous(), rows.target[idx].contiguous(), rows.weight[idx].contiguous()
        loss.zero_()
        _lib.call("gtomrln_mlp_gradients", C.c_void_p(params.data_ptr()), C.c_void_p(xb.data_ptr()),
                  C.c_void_p(tb.data_ptr()), C.c_void_p(wb.data_ptr()), batch, C.c_float(1.0 / batch),
                  C.c_void_p(grad.data_ptr()), C.c_void_p(loss.data_ptr()), stream)
        t = (step - 1) / max(1, steps - 1)
        rate = lr_final + 0.5 * (lr - lr_final) * (1 + math.cos(math.pi * t))
        _lib.call("gtomrln_mlp_adam", C.c_void_p(params.data_ptr()), C.c_void_p(grad.data_ptr()),
                  C.c_void_p(m.data_ptr()), C.c_void_p(v.data_ptr()), step, C.c_float(rate),
                  C.c_float(0.9), C.c_float(0.999), C.c_float(1e-8), stream)
        if (log_every and step % log_every == 0) or step == steps:
            losses.append(float(loss.item()))
    return losses


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


# ------------------------------------------------------------ evaluation --
# (name, momentum, use the network)
MODES = (("plain", 0.0, False), ("plain+mlp", 0.0, True), ("momentum", 0.9, False),
         ("momentum+mlp", 0.9, True))


def fsc_min(a: torch.Tensor, b: torch.Tensor, box: int) -> float:
    """Minimum over Fourier shells 1 .. box/2 of the correlation of two
    box^3 maps."""
    fa = torch.fft.rfftn(a.reshape(box, box, box).double())
    fb = torch.fft.rfftn(b.reshape(box, box, box).double())
    k = torch.fft.fftfreq(box, device=a.device) * box
    kx = torch.fft.rfftfreq(box, device=a.device) * box
    r = torch.sqrt(k[:, None, None] ** 2 + k[None, :, None] ** 2 + kx[None, None, :] ** 2).round().long()
    num = torch.zeros(box, dtype=torch.float64, device=a.device)
    da = torch.zeros_like(num)
    db = torch.zeros_like(num)
    keep = r < box
    rr = r[keep]
    num.index_add_(0, rr, (fa * fb.conj()).real[keep])
    da.index_add_(0, rr, (fa.abs() ** 2)[keep])
    db.index_add_(0, rr, (fb.abs() ** 2)[keep])
    f = num[1:box // 2 + 1] / torch.sqrt(da[1:box // 2 + 1] * db[1:box // 2 + 1]).clamp_min(1e-300)
    return float(f.min())


def evaluate(params: torch.Tensor | None, box: int, dists: list, pad: int = 2,
             tolerance: float = 1e-4, max_iterations: int = 5000, volft=None,
             converged_tolerance: float = 1e-4, converge_max: int = 20000) -> list:
    """For each distribution: the converged weights (momentum, relative
    change 1e-6, about the float32 floor of the change measure), then for each of MODES the iterations to `tolerance`, the
    weighted distance of the stopped weights from the converged ones, the
    wall time of the whole reconstruction through reconstruct_gridding_warm
    (CUDA events around the call, which synchronises once per iteration),
    and the map's minimum FSC to the plain map and to the map made with the
    converged weights.  Under "to_converged": the iterations the mode needs
    to bring the weights within `converged_tolerance` (weighted relative L2)
    of the converged ones, found with the library's distance measure, and
    the wall time of the whole reconstruction run for exactly that many
    iterations (no convergence test, so no per-iteration synchronisation)."""
    from .relion import reconstruct_gridding_warm
    P = box * pad
    D = P + 1
    rows = []
    for dist in dists:
        data, w = insert_distribution(box, dist, pad, volft=volft)
        if data is None:
            data = torch.complex(w, torch.zeros_like(w)).contiguous()
        ref, fw, it_ref, ch_ref, _ = gridding_weights(w, (D, D, D), box, pad, 5000, 1e-6, 0.9)
        row = {"views": dist.views, "lobes": dist.lobes, "uniform_frac": round(dist.uniform_frac, 3),
               "reference": {"iterations": it_ref, "change": ch_ref}}
        out = torch.empty(box ** 3, dtype=torch.float32, device=w.device)
        reconstruct_gridding_warm(data, w, out, (box,) * 3, (D,) * 3, None, pad, 2, 0.0)  # plans
        converged_map = torch.empty_like(out)
        reconstruct_gridding_warm(data, w, converged_map, (box,) * 3, (D,) * 3, None, pad, 5000, 1e-6, 0.9)
        maps = {}
        for name, mom, use in MODES:
            p = params if use else None
            if use and p is None:
                continue
            fnw, _, it, ch, used = gridding_weights(w, (D, D, D), box, pad, max_iterations, tolerance, mom,
                                                    mlp_params=p)
            res = {"iterations": it, "change": ch, "warm_used": used,
                   "distance_to_converged": weighted_distance(fw, fnw, ref)}
            m = torch.empty_like(out)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record()
            reconstruct_gridding_warm(data, w, m, (box,) * 3, (D,) * 3, p, pad, max_iterations, tolerance,
                                      mom)
            b.record()
            torch.cuda.synchronize()
            res["ms"] = a.elapsed_time(b)
            maps[name] = m
            _, _, k, _, _, dist = gridding_weights(w, (D, D, D), box, pad, converge_max, 0.0, mom, mlp_params=p,
                                                   ref_fnw=ref, ref_tolerance=converged_tolerance,
                                                   return_distance=True)
            conv = {"iterations": k, "distance": dist, "reached": bool(dist <= converged_tolerance)}
            if conv["reached"]:
                m2 = torch.empty_like(out)
                torch.cuda.synchronize()
                a.record()
                reconstruct_gridding_warm(data, w, m2, (box,) * 3, (D,) * 3, p, pad, k, 0.0, mom)
                b.record()
                torch.cuda.synchronize()
                conv["ms"] = a.elapsed_time(b)
            res["to_converged"] = conv
            row[name] = res
        for name, m in maps.items():
            row[name]["fsc_min_to_plain"] = fsc_min(m, maps["plain"], box)
            row[name]["fsc_min_to_converged"] = fsc_min(m, converged_map, box)
        rows.append(row)
    return rows


def summarise(rows: list) -> dict:
    """Medians over distributions per mode, and the wall-time and iteration
    ratios of each mode against the plain cold start."""
    out = {}
    for name, _, _ in MODES:
        have = [r[name] for r in rows if name in r]
        if not have:
            continue
        med = lambda k: float(np.median([h[k] for h in have]))
        out[name] = {"iterations": med("iterations"), "ms": med("ms"),
                     "distance_to_converged": med("distance_to_converged"),
                     "fsc_min_to_plain": float(min(h["fsc_min_to_plain"] for h in have)),
                     "fsc_min_to_converged": float(min(h["fsc_min_to_converged"] for h in have)),
                     "warm_rejected": int(sum(1 for h in have if not h["warm_used"]))
                     if name.endswith("+mlp") else 0,
                     "speedup_vs_plain": float(np.median([r["plain"]["ms"] / r[name]["ms"] for r in rows
                                                          if name in r]))}
        both = [r for r in rows if name in r and r[name]["to_converged"]["reached"]
                and r["plain"]["to_converged"]["reached"]]
        tc = [h["to_converged"] for h in have]
        out[name]["to_converged"] = {
            "reached": int(sum(1 for c in tc if c["reached"])), "of": len(tc),
            "iterations": float(np.median([c["iterations"] for c in tc])),
            "ms": float(np.median([c["ms"] for c in tc if c["reached"]])) if any(c["reached"] for c in tc) else None,
            "speedup_vs_plain": float(np.median([r["plain"]["to_converged"]["ms"] / r[name]["to_converged"]["ms"]
                                                 for r in both])) if both else None}
    return out


def main(argv=None) -> None:
    """Make the training set, train, save the parameters for the box size,
    evaluate on held-out distributions and write a JSON report.

        python -m gtom_b200.warmstart --box 128 --train 400 --held-out 100 \\
            --eval 16 --steps 3000 --save --report out.json
    """
    import argparse
    import json
    import time
    ap = argparse.ArgumentParser()
    ap.add_argument("--box", type=int, default=128)
    ap.add_argument("--pad", type=int, default=2)
    ap.add_argument("--train", type=int, default=400, help="training distributions")
    ap.add_argument("--held-out", type=int, default=100, help="held-out distributions")
    ap.add_argument("--eval", type=int, default=16, help="held-out distributions evaluated")
    ap.add_argument("--views", type=int, nargs=2, default=(5000, 200000))
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=32768)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--max-voxels", type=int, default=400000, help="trained voxels kept per distribution")
    ap.add_argument("--rows-per-dist", type=int, default=0,
                    help="train on this many sampled feature rows per distribution instead of whole stacks "
                         "(fits thousands of distributions)")
    ap.add_argument("--seed", type=int, default=1004)
    ap.add_argument("--save", action="store_true", help="store the parameters under gtom_b200/data/")
    ap.add_argument("--load", action="store_true", help="evaluate the stored parameters (no training)")
    ap.add_argument("--report", default=None)
    a = ap.parse_args(argv)
    rng = np.random.default_rng(a.seed)
    dists = [random_distribution(rng, views_range=tuple(a.views)) for _ in range(a.train + a.held_out)]
    train_d, held = dists[:a.train], dists[a.train:]
    rep = {"box": a.box, "pad": a.pad, "train": a.train, "held_out": a.held_out, "seed": a.seed,
           "views_range": list(a.views)}
    if a.load:
        params = load_params(a.box)
        if params is None:
            raise SystemExit(f"no stored parameters for box {a.box}")
        return _evaluate_and_report(a, params, held, rep)
    t0 = time.perf_counter()
    if a.rows_per_dist:
        ts = make_feature_rows((sampling_weights(a.box, d, a.pad) for d in train_d), a.box, a.pad,
                               rows_per_dist=a.rows_per_dist, count=len(train_d), seed=a.seed)
        rep["rows"] = int(ts.X.shape[0])
    else:
        ts = make_training_set((sampling_weights(a.box, d, a.pad) for d in train_d), a.box, a.pad,
                               count=len(train_d), max_voxels=a.max_voxels)
    torch.cuda.synchronize()
    rep["make_training_set_s"] = round(time.perf_counter() - t0, 1)
    rep["reference_iterations_median"] = float(np.median([c[0] for c in ts.converged]))
    t0 = time.perf_counter()
    if a.rows_per_dist:
        params = init_params_rows(ts, seed=a.seed)
        losses = train_rows(ts, params, steps=a.steps, batch=a.batch, lr=a.lr, log_every=max(1, a.steps // 20))
    else:
        params = init_params(ts, seed=a.seed)
        losses = train(ts, params, steps=a.steps, batch=a.batch, lr=a.lr, log_every=max(1, a.steps // 20))
    torch.cuda.synchronize()
    rep["train_s"] = round(time.perf_counter() - t0, 1)
    rep["losses"] = [round(x, 5) for x in losses]
    del ts
    torch.cuda.empty_cache()
    if a.save:
        rep["saved"] = str(save_params(params, a.box).name)
    _evaluate_and_report(a, params, held, rep)


def _evaluate_and_report(a, params, held, rep) -> None:
    import json
    from .synth import blob_volume, padded_half_ft
    volft = padded_half_ft(blob_volume(a.box, 2000 if a.box >= 128 else 200, a.seed, "cuda"), a.pad).reshape(-1)
    rows = evaluate(params, a.box, held[:a.eval], a.pad, volft=volft)
    rep["summary"] = summarise(rows)
    rep["rows"] = rows
    text = json.dumps(rep, indent=1)
    if a.report:
        Path(a.report).write_text(text)
    print(json.dumps({"summary": rep["summary"], "train_s": rep.get("train_s"),
                      "make_training_set_s": rep.get("make_training_set_s")}))


if __name__ == "__main__":
    main()
