"""Batched uneven-box reconstruction (one persistent insertion launch, the
gridding of each box size as a stack, all captured in a CUDA graph) against
the same reconstructions done one subvolume at a time through
d_rlnBackproject + d_ReconstructGridding, whose parity with the reference
the other GPU tests establish."""
import numpy as np
import pytest
import torch

from gtom_b200 import _lib, synth
from gtom_b200.batch import BatchReconstructor, Subvolume, autotune, reconstruct_separately
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

# Reconstructions: relative L2 <= 3e-4.  The two paths add the same
# insertion terms in different orders (one persistent direct kernel here,
# the row-segment brick kernel per subvolume there; their accumulators agree
# to ~1e-7, test_brick_gpu.py); ten gridding iterations divide by the
# accumulated weights and amplify those rounding differences where the
# weights are small (observed 3e-5 to 1.1e-4 over launch shapes).
TOL = 3e-4


def _batch(count, seed, boxes):
    raw = synth.tilt_series_batch(count, seed, "cuda", boxes=boxes)
    return [Subvolume(r["box"], r["projft"], r["projweights"], r["matrices"], r["out"]) for r in raw]


def _separate(subs, iterations=10):
    ref = [Subvolume(s.box, s.projft, s.projweights, s.matrices, torch.empty_like(s.out)) for s in subs]
    reconstruct_separately(ref, 2, iterations)
    torch.cuda.synchronize()
    return [r.out.cpu().numpy() for r in ref]


@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_equals_separate_calls(cuda, use_graph):
    subs = _batch(9, 31, (16, 24, 32))
    want = _separate(subs)
    rec = BatchReconstructor(subs, 2, 10)
    for _ in range(2):  # a second run (graph replay) starts from zeroed accumulators again
        for s in subs:
            s.out.fill_(float("nan"))
        rec.run(use_graph=use_graph)
        torch.cuda.synchronize()
        for s, w in zip(subs, want):
            got = s.out.cpu().numpy()
            assert np.all(np.isfinite(got))
            assert rel_l2(got, w) <= TOL, s.box
    rec.close()


def test_batch_tuning_and_untouched_slices(cuda):
    """Every launch shape the autotuner tries gives the same maps, and a
    subvolume without slices reconstructs to zero."""
    subs = _batch(5, 7, (16, 32))
    empty = Subvolume(24, None, None, torch.zeros(0, dtype=torch.float32, device="cuda"),
                      torch.full((24 ** 3,), 7.0, device="cuda"))
    want = _separate(subs)
    rec = BatchReconstructor(subs + [empty], 2, 10)
    res = autotune(rec, threads=(128, 512), slices=(1, 8), blocks=(2, 8), reps=1)
    assert len(res["table"]) == 8
    for t in res["table"]:
        rec.set_tuning(*t[:3])
        rec.run()
        torch.cuda.synchronize()
        for s, w in zip(subs, want):
            assert rel_l2(s.out.cpu().numpy(), w) <= TOL
        assert torch.count_nonzero(empty.out).item() == 0
    rec.close()


def test_batch_rejects_bad_input(cuda):
    s = _batch(1, 3, (16,))[0]
    bad = Subvolume(15, s.projft, s.projweights, s.matrices, s.out)
    with pytest.raises(_lib.GtomError):
        BatchReconstructor([bad])
    rec = BatchReconstructor([s])
    with pytest.raises(_lib.GtomError):
        rec.set_tuning(threads=100)
    rec.close()


def test_batch_against_reference_with_its_noise_floor(cuda):
    """Each sub-tomogram of a batch (boxes 32 to 128, 41 tilts over +-60
    degrees, CTF, dose filter, SNR 0.1) against the reference's own
    d_rlnBackproject + d_ReconstructGridding (10 iterations), with the
    difference taken apart:

    * insertion order: the reference against itself with its slices inserted
      in reverse order (the same terms summed in another order);
    * the gridding stage: this library's d_ReconstructGridding run on the
      reference's own accumulators against the reference's reconstruction.
      The reference computes the final centring shift with fast-math
      sin/cos of phases up to ~2 pi (x + y + z) / 2 (hundreds of radians;
      built with -use_fast_math), the library with the exact sign
      (-1)^(x+y+z); with a missing wedge many voxels carry almost no weight
      and the gridding's division there makes the map more sensitive to
      such differences than a single-particle map.

    The batch must stay within max(1e-4, 2 x (order floor + gridding
    difference)) of the reference, with FSC >= 0.999."""
    from oracle import refcuda
    from gtom_b200 import d_ReconstructGridding
    from tests.helpers import fsc
    if not refcuda.available():
        pytest.skip("the reference build is not present")
    ref = refcuda.lib()
    subs = _batch(6, 57, (32, 48, 64, 96, 128))
    rec = BatchReconstructor(subs, 2, 10)
    rec.run(use_graph=True)
    torch.cuda.synchronize()
    rows = []
    for s in subs:
        n, ns = s.box, s.nslices
        D = 2 * n + 1
        nv = (D // 2 + 1) * D * D
        e = (n // 2 + 1) * n
        order = [(s.projft, s.projweights, s.matrices),
                 (s.projft.reshape(ns, e).flip(0).contiguous(), s.projweights.reshape(ns, e).flip(0).contiguous(),
                  s.matrices.reshape(ns, 9).flip(0).contiguous())]
        outs, accs = [], []
        for pf, pw, mt in order:
            vf = torch.zeros(nv, dtype=torch.complex64, device="cuda")
            vw = torch.zeros(nv, dtype=torch.float32, device="cuda")
            refcuda.check(ref.ref_backproject(vf.data_ptr(), vw.data_ptr(), D, pf.data_ptr(), pw.data_ptr(), n, 2,
                                              n // 2, mt.data_ptr(), None, 1, 0, 0, 1, 0.0, 0, 0, ns),
                          "reference backproject")
            out = torch.empty(n ** 3, dtype=torch.float32, device="cuda")
            refcuda.check(ref.ref_reconstruct_gridding(vf.data_ptr(), vw.data_ptr(), out.data_ptr(), n, D, 2, 10, 1.9,
                                                       0, 15.0), "reference gridding")
            outs.append(out.cpu().numpy().reshape(n, n, n))
            accs.append((vf, vw))
        lib_on_ref = torch.empty(n ** 3, dtype=torch.float32, device="cuda")
        d_ReconstructGridding(accs[0][0], accs[0][1], lib_on_ref, (n,) * 3, (D,) * 3, 2, 0, 0, 10)
        torch.cuda.synchronize()
        got = s.out.cpu().numpy().reshape(n, n, n)
        floor = rel_l2(outs[1], outs[0])
        grid = rel_l2(lib_on_ref.cpu().numpy().reshape(n, n, n), outs[0])
        err = rel_l2(got, outs[0])
        rows.append((n, floor, grid, err))
        assert err <= max(1e-4, 2 * (floor + grid)), (n, err, floor, grid)
        assert np.all(fsc(got, outs[0]) >= 0.999), n
    rec.close()
    for n, floor, grid, err in rows:
        print(f"box {n}: reference vs itself in reverse order {floor:.2e}, library gridding of the reference's "
              f"accumulators {grid:.2e}, batch vs reference {err:.2e}")
