"""Pins the oracle's one-thread restatement of the reference's colourings
(Oracle.colour_perm for "SC", "PC", "PC_BAL", Oracle.colours_valid) against
the reference's own Utils::generate_perm run on one OpenMP thread
(Reference.generate_perm): identical permutations and level pointers, which
fix every row's colour."""
import numpy as np
import pytest

from oracle.oracle import Oracle, Reference, reference_available
from smaxkernels_b200 import matrices as M

O = Oracle()
needs_ref = pytest.mark.skipif(not reference_available(), reason="oracle/_ref not built")

CASES = {
    "laplace2d_9": lambda: M.laplace2d_5pt(9),
    "laplace3d_6": lambda: M.laplace3d_7pt(6),
    "stencil27_5": lambda: M.stencil27(5),
    "poisson2d_app_7": lambda: M.poisson2d_app(7),
    "lognormal_2000": lambda: M.lognormal_random(2000, seed=3),  # PC_BAL moves 664 rows here
    "lower_lognormal_1500": lambda: M.lower_triangle(*M.lognormal_random(1500, seed=5)),
}


@needs_ref
@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("type_", ["SC", "PC", "PC_BAL"])
def test_colourings_equal_the_reference_on_one_thread(name, type_):
    rp, col, _ = CASES[name]()
    R = Reference()
    R.set_threads(1)
    perm, inv, lvl_ptr, colour = O.colour_perm(rp, col, type_)
    rperm, rinv, rlvl = R.generate_perm(rp, col, type_)
    np.testing.assert_array_equal(perm, rperm)
    np.testing.assert_array_equal(inv, rinv)
    np.testing.assert_array_equal(lvl_ptr, rlvl)
    assert O.colours_valid(rp, col, colour)


def test_balance_moves_rows_on_an_irregular_pattern():
    rp, col, _ = CASES["lognormal_2000"]()
    _, _, _, c_pc = O.colour_perm(rp, col, "PC")
    _, _, _, c_bal = O.colour_perm(rp, col, "PC_BAL")
    assert (c_pc != c_bal).sum() > 0
    assert np.bincount(c_bal).max() < np.bincount(c_pc).max()


def test_sanity_check_ignores_colour_zero():
    rp = np.array([0, 1, 3, 5], np.int32)
    col = np.array([0, 0, 1, 1, 2], np.int32)
    assert O.colours_valid(rp, col, [0, 0, 1])      # 1-0 share colour 0: not a conflict
    assert not O.colours_valid(rp, col, [0, 2, 2])  # rows 2 and 1 share colour 2
