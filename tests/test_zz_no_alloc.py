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

from tests.helpers import rel_l2
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


def test_noalloc_projection_equals_allocating_entry_point(gtom_lib, cuda):
    rng = np.random.default_rng(4242)
    n, P = 64, 128
    vol = torch.from_numpy(blob_volume_ft(rng, n, P, 16)).cuda().reshape(-1)
    e = (n // 2 + 1) * n
    for batch in (300, 57):  # two calls in a row through the shared array
        ang = random_angles(rng, batch)
        ref = torch.zeros(batch * e, dtype=torch.complex64, device="cuda")
        got = torch.full((batch * e,), complex(np.nan, np.nan), dtype=torch.complex64, device="cuda")
        assert _project(gtom_lib, "gtomrln_project_angles", vol, P, n, ang, 2.0, ref) == 0
        assert _project(gtom_lib, "gtomrln_project_angles_noalloc", vol, P, n, ang, 2.0, got) == 0
        torch.cuda.synchronize()
        g, r = got.cpu().numpy(), ref.cpu().numpy()
        assert np.all(np.isfinite(g))
        assert rel_l2(g, r) <= 1e-6


def test_noalloc_refuses_batches_beyond_capacity(gtom_lib, cuda):
    n, P = 16, 32
    vol = torch.zeros((P // 2 + 1) * P * P, dtype=torch.complex64, device="cuda")
    ang = np.zeros((MAX_BATCH + 1, 3), np.float32)
    out = torch.zeros((MAX_BATCH + 1) * (n // 2 + 1) * n, dtype=torch.complex64, device="cuda")
    rc = _project(gtom_lib, "gtomrln_project_angles_noalloc", vol, P, n, ang, 2.0, out)
    assert rc == -1
    assert b"capacity" in gtom_lib.gtomrln_last_error()
    assert _project(gtom_lib, "gtomrln_project_angles_noalloc", vol, P, n, ang[:0], 2.0, out) == 0
