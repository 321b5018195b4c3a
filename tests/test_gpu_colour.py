"""GPU colourings (generate_perm "SC", "PC", "PC_BAL") and sanity_check_perm
against the oracle's one-thread restatement (pinned to the reference by
tests/test_colour_oracle.py): identical permutations and level pointers.
Then multicolour Gauss-Seidel: the solver on the PC-permuted Poisson matrix,
whose D+L solve has one level per colour, against the oracle."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from smaxkernels_b200 import Interface
from smaxkernels_b200 import matrices as M

pytestmark = pytest.mark.gpu
O = Oracle()

CASES = {
    "laplace2d_9": lambda: M.laplace2d_5pt(9),
    "stencil27_5": lambda: M.stencil27(5),
    "poisson2d_app_7": lambda: M.poisson2d_app(7),
    "lognormal_2000": lambda: M.lognormal_random(2000, seed=3),
    "lower_lognormal_1500": lambda: M.lower_triangle(*M.lognormal_random(1500, seed=5)),
    "laplace2d_300": lambda: M.laplace2d_5pt(300),          # 599 small levels in one CTA
    "stencil27_24": lambda: M.stencil27(24),                # wide SC levels
    "lognormal_30000": lambda: M.lognormal_random(30000, seed=9),
    "laplace3d_80": lambda: M.laplace3d_7pt(80),            # levels wider than 4096 rows
}


def gpu_perm(rp, col, type_):
    smax = Interface()
    n = len(rp) - 1
    perm = np.zeros(n, np.int32)
    inv = np.zeros(n, np.int32)
    smax.utils.generate_perm(n, rp, col, perm, inv, type_)
    lvl = np.array([smax.get_level_ptr_at(i) for i in range(smax.get_n_levels() + 1)], np.int32)
    smax.close()
    return perm, inv, lvl


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("type_", ["SC", "PC", "PC_BAL"])
def test_colourings_equal_the_oracle(name, type_):
    rp, col, _ = CASES[name]()
    perm, inv, lvl = gpu_perm(rp, col, type_)
    operm, oinv, olvl, colour = O.colour_perm(rp, col, type_)
    np.testing.assert_array_equal(lvl, olvl)
    np.testing.assert_array_equal(perm, operm)
    np.testing.assert_array_equal(inv, oinv)


def test_sanity_check_perm():
    rp, col, _ = M.lognormal_random(3000, seed=4)
    smax = Interface()
    n = len(rp) - 1
    _, _, _, colour = O.colour_perm(rp, col, "PC")
    assert smax.utils.sanity_check_perm(n, rp, col, colour)
    # plant a conflict: give a row the colour of a lower neighbour (colour != 0)
    bad = colour.copy()
    for r in range(n):
        lower = [int(c) for c in col[rp[r]:rp[r + 1]] if c < r and colour[c] != 0]
        if lower:
            bad[r] = colour[lower[0]]
            break
    assert not O.colours_valid(rp, col, bad)
    assert not smax.utils.sanity_check_perm(n, rp, col, bad)
    # every row colour 0 is accepted, as the reference's check skips colour 0
    assert smax.utils.sanity_check_perm(n, rp, col, np.zeros(n, np.int32))
    smax.close()


def test_empty_pattern():
    for t in ("SC", "PC", "PC_BAL"):
        perm, inv, lvl = gpu_perm(np.zeros(1, np.int32), np.zeros(0, np.int32), t)
        assert len(perm) == 0 and lvl.tolist() == [0, 0]


def test_multicolour_gauss_seidel():
    from smaxkernels_b200.solvers import Solver
    rp, col, val = M.poisson2d_app(24)
    n = len(rp) - 1
    perm, inv, lvl = gpu_perm(rp, col, "PC")
    assert len(lvl) == 3  # red-black
    prp, pcol, pval = O.apply_mat_perm(rp, col, val, perm, inv)
    b = M.uniform_vector(n, 12)
    x = np.zeros(n)
    with Solver("gauss_seidel", prp, pcol, pval) as s:
        st = s.solve(b, x, tol=1e-8, max_iters=3000)
    xo, n_o, norm_o, _ = O.gauss_seidel_app(prp, pcol, pval, b, np.zeros(n), 1e-8, 3000, 5)
    assert st["n_iters"] == n_o and st["converged"] == int(norm_o < 1e-8) == 1
    assert np.linalg.norm(x - xo) <= 1e-12 * np.linalg.norm(xo)
