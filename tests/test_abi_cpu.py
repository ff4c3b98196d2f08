"""CPU checks of the C ABI: the library loads, exports exactly what
include/gtomrln.h declares, and its host-side logic (matrices, blob table,
argument validation) matches the oracle without touching a GPU."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from tests.synthdata import random_angles

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols() -> set[str]:
    text = (ROOT / "include" / "gtomrln.h").read_text()
    return set(re.findall(r"GTOMRLN_API\s+[\w\s\*]*?\b(gtomrln_\w+)\s*\(", text))


def exported_symbols(path: Path) -> set[str]:
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", str(path)], capture_output=True, text=True,
                         check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if " T " in ln}


def test_library_exports_every_declared_symbol(gtom_lib):
    from gtom_b200 import _lib
    decl = declared_symbols()
    assert len(decl) >= 13
    exported = exported_symbols(_lib.LIB_PATH)
    assert decl <= exported, decl - exported
    # nothing beyond the C ABI leaks out of the library
    assert {s for s in exported if s.startswith("gtomrln_")} == decl
    for name in decl:
        assert hasattr(gtom_lib, name)
    assert set(_lib.SIGNATURES) == decl


def test_version_and_error_state(gtom_lib):
    assert gtom_lib.gtomrln_version() == 100


def test_matrices_match_fp64_oracle(gtom_lib):
    from gtom_b200 import matrices_from_angles
    ang = random_angles(np.random.default_rng(0), 200)
    for s in (1.0, 2.0, 1.5):
        a = matrices_from_angles(ang, s)
        b = O.matrices_f64(ang, s)
        assert np.max(np.abs(a - b)) < 4e-7 * s


def test_blob_table_matches_oracle(gtom_lib):
    from gtom_b200 import kaiser_bessel_table
    for order in (0, 2):
        a = kaiser_bessel_table(3.8, 15.0, order, 10000)
        b = O.kb_table(3.8, 15.0, order, 10000)
        assert np.max(np.abs(a - b)) < 2e-7
    with pytest.raises(Exception):
        kaiser_bessel_table(3.8, 15.0, 1, 100)


def test_invalid_dimensions_return_error_not_terminate(gtom_lib):
    """The reference calls `throw;` (std::terminate) when the volume has fewer
    dimensions than the projections; the C ABI returns GTOMRLN_ERR_INVALID
    with a message, before any device work."""
    rc = gtom_lib.gtomrln_project(None, 32, 32, 1, None, 16, 16, 16, 8, None, 1, None)
    assert rc == -1
    assert b"dimensions" in gtom_lib.gtomrln_last_error()
    rc = gtom_lib.gtomrln_backproject(None, None, 32, 32, 1, None, None, 16, 16, 16, 8, None, None,
                                      1.0, 0.0, 0.0, 1.0, 0.0, 1, 0, 1, None)
    assert rc == -1
    rc = gtom_lib.gtomrln_reconstruct_gridding(None, None, None, 16, 16, 16, 33, 33, 33, 2, 0, 0, 10,
                                               1.9, 0, 15.0, None)
    assert rc == -1


def test_zero_batch_is_a_no_op(gtom_lib):
    assert gtom_lib.gtomrln_project(None, 32, 32, 32, None, 16, 16, 1, 8, None, 0, None) == 0
    assert gtom_lib.gtomrln_backproject(None, None, 32, 32, 32, None, None, 16, 16, 1, 8, None, None,
                                        1.0, 0.0, 0.0, 1.0, 0.0, 1, 0, 0, None) == 0


def test_python_mirror_rejects_host_buffers(gtom_lib):
    import torch
    from gtom_b200 import d_rlnProject
    vol = torch.zeros(17 * 32 * 32, dtype=torch.complex64)
    proj = torch.zeros(9 * 16, dtype=torch.complex64)
    with pytest.raises(ValueError):
        d_rlnProject(vol, (32, 32, 32), proj, (16, 16, 1), 8, torch.zeros(9), 1)
