"""Multi-rank insertion on CPU: two gloo ranks shard the slices, insert their
shares into private accumulators (the oracle's FP32 port stands in for the
GPU kernel, whose per-slice arithmetic it matches), sum them with the one
all-reduce of gtom_b200.shard.Accumulators, and must reproduce the
single-process insertion of the whole batch up to FP32 summation order."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from gtom_b200.shard import Accumulators, broadcast_reference, slice_range, volumes_for_rank
from oracle import oracle as O
from tests.helpers import rel_l2
from tests.synthdata import random_angles

N_SLICES, BOX, PAD = 37, 16, 2


def _inputs():
    rng = np.random.default_rng(77)
    n = BOX
    e = (n // 2 + 1) * n
    data = (rng.standard_normal((N_SLICES, e)) + 1j * rng.standard_normal((N_SLICES, e))).astype(np.complex64)
    wts = rng.uniform(0.1, 1.0, (N_SLICES, e)).astype(np.float32)
    mats = O.matrices_f64(random_angles(rng, N_SLICES), float(PAD)).astype(np.float32)
    return data, wts, mats


def _insert(acc_data: np.ndarray, acc_w: np.ndarray, data, wts, mats):
    P = BOX * PAD
    O.backproject(acc_data, acc_w, P + 1, data, wts, BOX, BOX // 2, mats, decentered=False, fp32=True)


def _nvox():
    D = BOX * PAD + 1
    return (D // 2 + 1) * D * D


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, outdir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        # the reference volume, built on rank 0 only, reaches every rank
        ref = torch.zeros(6, 5, 4, dtype=torch.complex64)
        if rank == 0:
            ref = torch.complex(torch.arange(120.).reshape(6, 5, 4), -torch.arange(120.).reshape(6, 5, 4))
        broadcast_reference(ref)
        np.save(os.path.join(outdir, f"ref{rank}.npy"), ref.numpy())
        data, wts, mats = _inputs()
        first, count = slice_range(N_SLICES, rank, world)
        acc = Accumulators(_nvox(), "cpu")
        _insert(acc.data.numpy(), acc.weights.numpy(), data[first:first + count], wts[first:first + count],
                mats[first:first + count])
        acc.all_reduce()
        np.save(os.path.join(outdir, f"acc{rank}.npy"), acc.buffer.numpy())
    finally:
        dist.destroy_process_group()


def test_slice_range_partitions_the_batch():
    for total in (0, 1, 7, 100, 10001):
        for world in (1, 2, 3, 8):
            spans = [slice_range(total, r, world) for r in range(world)]
            assert sum(c for _, c in spans) == total
            assert spans[0][0] == 0
            for (f0, c0), (f1, _) in zip(spans, spans[1:]):
                assert f1 == f0 + c0
            assert max(c for _, c in spans) - min(c for _, c in spans) <= 1
    with pytest.raises(ValueError):
        slice_range(10, 2, 2)


def test_accumulator_views_share_one_buffer():
    acc = Accumulators(5, "cpu")
    acc.data[3] = 2 + 3j
    acc.weights[4] = 7
    assert acc.buffer[6].item() == 2 and acc.buffer[7].item() == 3 and acc.buffer[14].item() == 7
    acc.all_reduce()  # no process group: leaves the sums alone
    assert acc.weights[4].item() == 7
    assert acc.zero_().buffer.abs().sum().item() == 0


@pytest.mark.timeout(180)
def test_two_rank_insertion_equals_single_process():
    data, wts, mats = _inputs()
    ref = Accumulators(_nvox(), "cpu")
    _insert(ref.data.numpy(), ref.weights.numpy(), data, wts, mats)
    world = 2
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_rank_main, args=(world, _free_port(), d), nprocs=world, join=True,
                           start_method="spawn")
        got = [np.load(os.path.join(d, f"acc{r}.npy")) for r in range(world)]
        refs = [np.load(os.path.join(d, f"ref{r}.npy")) for r in range(world)]
    want = ref.buffer.numpy()
    assert np.abs(want).max() > 0
    for g in got:  # every rank holds the full sums after the all-reduce
        assert rel_l2(g, want) <= 1e-6
    np.testing.assert_array_equal(got[0], got[1])
    expect = np.arange(120.).reshape(6, 5, 4) * (1 - 1j)
    for r in refs:  # the broadcast reference volume
        np.testing.assert_array_equal(r, expect.astype(np.complex64))


def test_volumes_for_rank_partitions_the_volumes():
    for n, world in ((0, 1), (1, 3), (8, 2), (9, 4), (512, 8)):
        parts = [volumes_for_rank(n, r, world) for r in range(world)]
        assert sorted(sum(parts, [])) == list(range(n))
        assert max(map(len, parts)) - min(map(len, parts)) <= 1
    with pytest.raises(ValueError):
        volumes_for_rank(4, 2, 2)


def test_sharded_projection_concatenates_to_the_full_batch():
    """The projector shards without any exchange: the ranks' slices,
    concatenated in rank order, are the whole batch's slices."""
    rng = np.random.default_rng(5)
    P, n = BOX * PAD, BOX
    vol = (rng.standard_normal((P, P, P // 2 + 1)) + 1j * rng.standard_normal((P, P, P // 2 + 1))).astype(
        np.complex64)
    mats = O.matrices_f64(random_angles(rng, 11), float(PAD)).astype(np.float32)
    full = O.project(vol, P, n, n // 2, mats, fp32=True)
    parts = []
    for r in range(3):
        f, c = slice_range(11, r, 3)
        parts.append(O.project(vol, P, n, n // 2, mats[f:f + c], fp32=True))
    np.testing.assert_array_equal(np.concatenate(parts), full)
