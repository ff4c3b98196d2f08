"""Pins the CPU oracle to the reference's own CUDA results (tests/golden/,
produced by make_golden.py from the reference sources rebuilt for sm_100a).

The single-precision port follows the reference's arithmetic operation for
operation (same fused multiply-adds, same binary16 weight rounding), so it
reproduces the reference's projections exactly and its backprojection up to
the order of the floating-point atomic sums.  The FP64 oracle differs only
by the reference's single-precision rounding (and, in the backprojector,
weights that round to the neighbouring binary16 value)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import fsc, load_golden, rel_l2


@pytest.mark.parametrize("name", ["project_2d", "project_2d_rmax", "project_3d"])
def test_oracle_project_matches_reference(name):
    g = load_golden(name)
    P, n, nd, rmax = int(g["P"]), int(g["n"]), int(g["ndims"]), int(g["rmax"])
    port = O.project(g["volume"], P, n, rmax, g["matrices"], ndims=nd, fp32=True)
    assert rel_l2(port, g["proj"]) <= 1e-7
    f64 = O.project(g["volume"], P, n, rmax, g["matrices"], ndims=nd)
    assert rel_l2(f64, g["proj"]) <= 1e-6
    # the h_angles overload uses rmax = n/2 and FP32 host matrices
    f64a = O.project(g["volume"], P, n, n // 2, O.matrices_f64(g["angles"], 2.0).astype(np.float32), ndims=nd)
    assert rel_l2(f64a, g["proj_angles"]) <= 1e-5


@pytest.mark.parametrize("name", ["bp_dec", "bp_cen_sq_mag", "bp_3d"])
def test_oracle_backproject_matches_reference(name):
    g = load_golden(name)
    P, n, nd, nvol = int(g["P"]), int(g["n"]), int(g["ndims"]), int(g["nvol"])
    nv = (P // 2 + 1) * P * P * nvol
    iv = g["ivolume"] if g["ivolume"].size else None
    for fp32, tol in ((True, 1e-6), (False, 1e-4)):
        vf = np.zeros(nv, np.complex64 if fp32 else np.complex128)
        vw = np.zeros(nv, np.float32 if fp32 else np.float64)
        O.backproject(vf, vw, P, g["projft"], g["projw"], n, int(g["rmax"]), g["matrices"], ivolume=iv,
                      magnification=tuple(g["mag"]), ewaldradiussuper=float(g["ewald"]),
                      decentered=bool(g["decentered"]), square=bool(g["square"]), ndims=nd, fp32=fp32)
        assert rel_l2(vf, g["volft"]) <= tol
        assert rel_l2(vw, g["volw"]) <= tol


@pytest.mark.parametrize("name", ["grid_it10", "grid_it0", "grid_it3_pad3"])
def test_oracle_gridding_matches_reference(name):
    g = load_golden(name)
    ori, pad, dp, it = int(g["ori"]), int(g["pad"]), int(g["dimspadded"]), int(g["iterations"])
    rec = O.reconstruct_gridding(g["dataft"].reshape(dp, dp, dp // 2 + 1), g["weight"].reshape(dp, dp, dp // 2 + 1),
                                 ori, (dp,) * 3, pad, iterations=it)
    assert rel_l2(rec, g["reconstructed"]) <= 1e-5
    assert fsc(rec, g["reconstructed"]).min() >= 0.9999


@pytest.mark.parametrize("name", ["project_shifted_2d", "project_shifted_3d"])
def test_oracle_project_shifted_matches_reference(name):
    """The reference multiplies by the phase with the fast hardware sine and
    cosine (ProjectShifted.cu:217); the float64 oracle with exact ones."""
    g = load_golden(name)
    out = O.project_shifted(g["volume"], int(g["P"]), int(g["n"]), int(g["rmax"]), g["matrices"], g["shifts"],
                            g["globalweights"], ndims=int(g["ndims"]))
    assert rel_l2(out, g["proj"]) <= 1e-5
    np.testing.assert_array_equal(O.scaled_shifts(g["shifts_px"], int(g["n"])), g["shifts"])


@pytest.mark.parametrize("name", ["bp_shifted_2d", "bp_shifted_3d"])
def test_oracle_backproject_shifted_matches_reference(name):
    g = load_golden(name)
    V = int(g["V"])
    nv = (V // 2 + 1) * V * V
    vf = np.zeros(nv, np.complex128)
    vw = np.zeros(nv, np.float64)
    O.backproject_shifted(vf, vw, V, g["projft"], g["projw"], int(g["n"]), int(g["rmax"]), g["matrices"],
                          g["shifts"], g["globalweights"], ndims=int(g["ndims"]))
    assert rel_l2(vf, g["volft"]) <= 1e-5
    assert rel_l2(vw, g["volw"]) <= 1e-5
