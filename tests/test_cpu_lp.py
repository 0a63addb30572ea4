"""LP blocks (negative block sizes) at the interface, on the host side: the checks of
brisk_solve_data on LP entries (problem.c's problem_from_sdpa_data: an LP block takes diagonal
entries only) run before any GPU work, so they are tested without a GPU.  The solves themselves
are in tests/test_gpu_solve.py."""
import numpy as np

import brisk_b200
from brisk_b200 import problems


def test_off_diagonal_lp_entry_is_refused():
    d = problems.sdp_lp_problem(blocks=(5, -4), m=6, seed=1)
    a = [np.asarray(x).copy() for x in d.args()]
    lp = np.nonzero((a[3] == 2) & (a[2] > 0))[0][0]   # an LP entry of a constraint
    a[5][lp] = a[4][lp] % 4 + 1                        # column != row
    res = brisk_b200.solve_sdpa(*a, verbose=False)
    assert res.exit_code == 2
    assert "off-diagonal entry in LP block" in res.log


def test_generator_lp_blocks_are_diagonal_and_feasible():
    """The generator's LP blocks hold diagonal entries only, and b = A(I, 1)."""
    d = problems.sdp_lp_problem(blocks=(6, -5, 3), m=8, seed=2)
    assert d.bs.tolist() == [6, -5, 3]
    lp = d.blk == 2
    assert np.all(d.i[lp] == d.j[lp])
    C, A = d.dense_blocks()
    b = sum(np.trace(A[k], axis1=1, axis2=2) for k in range(3))
    np.testing.assert_allclose(b, d.c, rtol=1e-12, atol=1e-12)
    assert np.all(np.diag(C[1]) > 0)
