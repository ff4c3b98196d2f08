"""The allocation-free projector entry point, through the C ABI.

gtomrln_project_angles_noalloc serves callers that cannot allocate device
memory (their device memory belongs to another allocator or a fixed budget,
or an allocation must not synchronise the device mid-pipeline).  It keeps
the rotation matrices in a fixed array inside the library instead of
allocating them.  Its results must equal gtomrln_project_angles's on the
same inputs, call after call, and batches beyond the array's capacity must
be refused with an error rather than overrun it.

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from tests.synthdata import blob_volume_ft, random_angles

pytestmark = pytest.mark.gpu

MAX_BATCH = 4096  # the fixed capacity documented in include/gtomrln.h


def _project(lib, name, vol, P, n, ang, supersample, out):
    batch = ang.shape[0]
    a = np.ascontiguousarray(ang, np.float32)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = getattr(lib, name)(C.c_void_p(vol.data_ptr()), P, P, P, C.c_void_p(out.data_ptr()), n, n, 1,
                            a.ctypes.data, C.c_float(supersample), batch, stream)
    return rc


def _empty(batch, e):
    return torch.full((batch * e,), complex(np.nan, np.nan), dtype=torch.complex64, device="cuda")


def test_noalloc_projection_equals_allocating_entry_point(gtom_lib, cuda):
    """Two calls in a row on one stream, with no host synchronisation
    between them: the second call's matrices replace the first's in the
    shared array only after the first projection has read them (stream
    order), so both results equal the allocating entry point's bit for bit
    (the direct and row-segment projector kernels agree exactly)."""
    rng = np.random.default_rng(4242)
    n, P = 64, 128
    vol = torch.from_numpy(blob_volume_ft(rng, n, P, 16)).cuda().reshape(-1)
    e = (n // 2 + 1) * n
    angs = [random_angles(rng, b) for b in (300, 57)]
    got = [_empty(a.shape[0], e) for a in angs]
    for a, g in zip(angs, got):
        assert _project(gtom_lib, "gtomrln_project_angles_noalloc", vol, P, n, a, 2.0, g) == 0
    ref = [torch.zeros(a.shape[0] * e, dtype=torch.complex64, device="cuda") for a in angs]
    for a, r in zip(angs, ref):
        assert _project(gtom_lib, "gtomrln_project_angles", vol, P, n, a, 2.0, r) == 0
    torch.cuda.synchronize()
    for g, r in zip(got, ref):
        assert torch.isfinite(torch.view_as_real(g)).all()
        assert torch.equal(g, r)


def test_noalloc_full_capacity_batch(gtom_lib, cuda):
    """A batch of exactly the array's capacity fills it completely."""
    rng = np.random.default_rng(4343)
    n, P = 16, 32
    vol = torch.from_numpy(blob_volume_ft(rng, n, P, 6)).cuda().reshape(-1)
    e = (n // 2 + 1) * n
    ang = random_angles(rng, MAX_BATCH)
    got, ref = _empty(MAX_BATCH, e), torch.zeros(MAX_BATCH * e, dtype=torch.complex64, device="cuda")
    assert _project(gtom_lib, "gtomrln_project_angles_noalloc", vol, P, n, ang, 2.0, got) == 0
    assert _project(gtom_lib, "gtomrln_project_angles", vol, P, n, ang, 2.0, ref) == 0
    torch.cuda.synchronize()
    assert torch.equal(got, ref)


def test_noalloc_3d_projection(gtom_lib, cuda):
    """3D projections (a rotated n^3 half-volume per orientation) through the
    fixed array equal the allocating entry point's."""
    import ctypes as C
    rng = np.random.default_rng(4444)
    n, P, batch = 16, 32, 3
    vol = torch.from_numpy(blob_volume_ft(rng, n, P, 6)).cuda().reshape(-1)
    e = (n // 2 + 1) * n * n
    ang = np.ascontiguousarray(random_angles(rng, batch), np.float32)
    got, ref = _empty(batch, e), torch.zeros(batch * e, dtype=torch.complex64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for name, out in (("gtomrln_project_angles_noalloc", got), ("gtomrln_project_angles", ref)):
        rc = getattr(gtom_lib, name)(C.c_void_p(vol.data_ptr()), P, P, P, C.c_void_p(out.data_ptr()), n, n, n,
                                     ang.ctypes.data, C.c_float(2.0), batch, stream)
        assert rc == 0
    torch.cuda.synchronize()
    assert torch.equal(got, ref)


def test_noalloc_refuses_batches_beyond_capacity(gtom_lib, cuda):
    n, P = 16, 32
    vol = torch.zeros((P // 2 + 1) * P * P, dtype=torch.complex64, device="cuda")
    ang = np.zeros((MAX_BATCH + 1, 3), np.float32)
    out = torch.zeros((MAX_BATCH + 1) * (n // 2 + 1) * n, dtype=torch.complex64, device="cuda")
    rc = _project(gtom_lib, "gtomrln_project_angles_noalloc", vol, P, n, ang, 2.0, out)
    assert rc == -1
    assert b"capacity" in gtom_lib.gtomrln_last_error()
    assert _project(gtom_lib, "gtomrln_project_angles_noalloc", vol, P, n, ang[:0], 2.0, out) == 0
