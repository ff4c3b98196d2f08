"""The library keeps working after the caller resets the device.

gtom's own tests call cudaDeviceReset() around every test
(GTOMTest/Norm.cpp:7,55,58), which destroys every allocation, plan and
loaded module of the process's context.  The library's caches (memory
pool, plan scratch, staging slots, cuFFT plans, blob and twiddle tables,
brick orders, fused-FFT launch attributes) are keyed on the context's
unique id, and gtomrln_release_caches() frees them; the fixed array of the
allocation-free projector is looked up on every call.  The check runs in a
child process that uses only the CUDA runtime and the library's C ABI
(tests/device_reset_child.py): every cached path before a reset, after
gtomrln_release_caches() + cudaDeviceReset(), and after a bare
cudaDeviceReset(), with the same results (projections and preprocessing
bit for bit; accumulations and reconstructions up to the FP32 atomics'
summation order).
"""
import json
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

CHILD = Path(__file__).resolve().parent / "device_reset_child.py"
EXACT = ("project", "project_angles", "project_noalloc", "preprocess")


def check(diffs: dict) -> None:
    for k, v in diffs.items():
        tol = 0.0 if k in EXACT else 1e-5
        assert v <= tol, f"{k}: {v:.3e} after the reset"


def test_entry_points_after_device_reset(gtom_lib, cuda):
    r = subprocess.run([sys.executable, str(CHILD)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert len(res["keys"]) == 8
    check(res["released_then_reset"])
    print("reset without release:", res["reset_without_release"])
    if isinstance(res["reset_without_release"], dict):
        check(res["reset_without_release"])
