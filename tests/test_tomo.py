"""d_BackprojectTomo (Lanczos-5 gather insertion): the float64 oracle
against the reference's own result (CPU), and the library against both
(GPU), through the matrix and h_angles overloads."""
import numpy as np
import pytest
import torch

from oracle import tomo_oracle as T
from tests.helpers import load_golden, rel_l2


def test_oracle_tomo_matches_reference():
    g = load_golden("bp_tomo")
    got = T.backproject_tomo(g["volume0"], int(g["V"]), g["projft"], g["projw"], int(g["n"]), int(g["rmax"]),
                             g["matrices"])
    # the reference evaluates the sincs with the fast hardware sine (arguments
    # up to 5 pi) in float and divides by the weight sums: 4e-4 from exact
    assert rel_l2(got, g["volume"]) <= 1e-3
    assert np.count_nonzero(got != g["volume0"]) > 0


@pytest.mark.gpu
@pytest.mark.parametrize("overload", ["matrices", "angles"])
def test_tomo_matches_reference(gtom_lib, cuda, overload):
    import gtom_b200 as G
    g = load_golden("bp_tomo")
    V, n, rmax = int(g["V"]), int(g["n"]), int(g["rmax"])
    batch = g["matrices"].shape[0]
    vol = torch.from_numpy(g["volume0"]).cuda()
    arg = g["angles"] if overload == "angles" else torch.from_numpy(g["matrices"]).cuda().reshape(-1)
    G.d_BackprojectTomo(vol, (V, V, V), torch.from_numpy(g["projft"]).cuda().reshape(-1),
                        torch.from_numpy(g["projw"]).cuda().reshape(-1), (n, n, 1), rmax, arg, batch)
    got = vol.cpu().numpy()
    written = got != g["volume0"]
    np.testing.assert_array_equal(written, g["volume"] != g["volume0"])
    assert rel_l2(got, g["volume"]) <= 1e-4  # fast sine / division in both; sums in another order
