"""The LP route (the reference's schur_lp, solver.c:3233) on a B200: M += A diag(x_p / z_p) A' over
the variables of one LP block, one launch per LP block, through the C ABI (bgpu_schur_lp), and
whole solves of LP blocks whose rows join every variable, against the reference's runs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import brisk_b200  # noqa: E402
from brisk_b200 import step  # noqa: E402
from test_gpu_solve import FP64, check, make  # noqa: E402


def lp_lists(A):
    """The route's lists of a dense nc x N matrix A (zeros are absent): per constraint its
    (variable, value) pairs by ascending variable, per variable its (constraint, value) pairs by
    ascending constraint."""
    nc, N = A.shape
    t_idx, p_idx = np.nonzero(A)                 # row-major: by constraint, then variable
    aptr = np.zeros(nc + 1, np.int64)
    np.add.at(aptr, t_idx + 1, 1)
    aptr = np.cumsum(aptr)
    avar, aval = p_idx.astype(np.int32), A[t_idx, p_idx]
    p2, t2 = np.nonzero(A.T)                     # by variable, then constraint
    vptr = np.zeros(N + 1, np.int64)
    np.add.at(vptr, p2 + 1, 1)
    vptr = np.cumsum(vptr)
    return aptr, avar, aval, vptr, t2.astype(np.int32), A[t2, p2]


@pytest.mark.parametrize("N,nc,m,per,dense", [(300, 50, 80, 5, 2), (1, 3, 3, 1, 0), (1000, 200, 1000, 3, 1)])
def test_schur_lp_matches_numpy(cuda, N, nc, m, per, dense):
    rng = np.random.default_rng(N + nc)
    A = np.zeros((nc, N))
    for t in range(nc):
        q = N if t < dense else min(per, N)
        var = rng.choice(N, size=q, replace=False)
        A[t, var] = rng.standard_normal(q)
    A[:, N // 2] = 0.0                           # a variable in no constraint
    gcon = np.sort(rng.choice(m, size=nc, replace=False)).astype(np.int32)
    x = rng.uniform(0.1, 2.0, N)
    zi = 1.0 / rng.uniform(0.1, 2.0, N)
    M0 = rng.standard_normal((m, m))
    M0 = M0 + M0.T
    aptr, avar, aval, vptr, vcon, vval = lp_lists(A)
    d = {k: torch.as_tensor(np.ascontiguousarray(v), device=cuda) for k, v in
         dict(gcon=gcon, aptr=aptr, avar=avar, aval=aval, vptr=vptr, vcon=vcon, vval=vval, x=x, zi=zi).items()}
    M = torch.as_tensor(np.ascontiguousarray(M0.T), device=cuda).contiguous()   # column-major
    step.call("schur_lp", m, N, nc, int(aval.size), *(d[k].data_ptr() for k in
              ("gcon", "aptr", "avar", "aval", "vptr", "vcon", "vval", "x", "zi")), M.data_ptr(), None)
    step.call("sync", None)
    got = M.cpu().numpy().T
    Ag = np.zeros((m, N))
    Ag[gcon] = A
    want = M0 + Ag @ np.diag(x * zi) @ Ag.T
    scale = np.abs(Ag).max() ** 2 * (x * zi).max() * max(1, np.count_nonzero(A, axis=1).max())
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-14 * scale + 1e-14 * np.abs(M0).max())
    assert np.array_equal(got, got.T)            # both triangles from the same sums


@pytest.mark.parametrize("run,opts", [("default", FP64), ("init0", FP64 + ["-init", "0"]),
                                      ("nt", ["-nohsd", "-dir", "nt", "-mixed", "0", "-tol", "1e-7"])])
def test_lp_block_with_rows_over_all_variables(golden, run, opts):
    """lp_dense: an LP block of 300 variables, two of whose 80 rows join every variable, beside an
    SDP block of order 20.  The LP route takes the block in one launch per assembly (the small-block
    route needed a launch per variable: every variable shares a constraint with every other).
    Status, objectives and DIMACS errors as the reference's run; the iteration count within one."""
    e = golden["lp_dense"]
    res = brisk_b200.solve_sdpa(*make(e).args(), options=opts + ["-vv"], verbose=False)
    ref = e["runs"][run]
    check(res, ref)
    assert abs(res.iterations - ref["iterations"]) <= 1, (res.iterations, ref["iterations"])
    assert "300 variables over 80 constraints by the LP route" in res.log
