"""The low-rank Schur route (the reference's schur_lowrank, solver.c:1862-1934) on a B200: M from
the factors A_t = sum sig_k w_k w_k' (P = W'XW, Q = W'ZiW by DMMA, one launch over the pairs of
constraints) against M_tu = <A_t, X A_u Zi> computed plainly in FP64, to the north star's 1e-10
relative; whole solves of low-rank problems through the route against the reference's runs (which
take its own low-rank route on them), and the same problems through the other routes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import brisk_b200  # noqa: E402
from brisk_b200 import problems, step  # noqa: E402
from test_cpu_lowrank import full_lists, random_lowrank  # noqa: E402
from test_gpu_solve import FP64, check, make  # noqa: E402


def spd(rng, n, cond):
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    return (Q * np.logspace(0, np.log10(cond), n)) @ Q.T


@pytest.mark.parametrize("n,ncon,support", [(80, 120, 0), (100, 60, 20), (65, 40, 65)])
def test_lowrank_schur_matches_dense_formula(cuda, n, ncon, support):
    rng = np.random.default_rng(n + ncon)
    mats = [random_lowrank(rng, n, int(rng.integers(1, 4)), support or n) for _ in range(ncon)]
    X, Zi = spd(rng, n, 1e3), spd(rng, n, 1e4)
    m = ncon + 7
    con = np.sort(rng.choice(m, size=ncon, replace=False)).astype(np.int32)
    cptr, cpos, cval = full_lists(mats, n)
    M0 = rng.standard_normal((m, m))
    M0 = M0 + M0.T
    dM = torch.as_tensor(np.ascontiguousarray(M0.T), device=cuda).contiguous()
    dX = torch.as_tensor(np.ascontiguousarray(X.T), device=cuda).contiguous()
    dZ = torch.as_tensor(np.ascontiguousarray(Zi.T), device=cuda).contiguous()
    dcon = torch.as_tensor(con, device=cuda)
    rank = np.zeros(1, np.int32)
    step.call("schur_lowrank", n, m, ncon, dcon.data_ptr(), cptr.ctypes.data, cpos.ctypes.data, cval.ctypes.data,
              dX.data_ptr(), dZ.data_ptr(), dM.data_ptr(), rank.ctypes.data, None)
    assert rank[0] == sum(np.linalg.matrix_rank(a) for a in mats)
    got = dM.cpu().numpy().T - M0
    Ms = np.zeros((ncon, ncon))
    for u in range(ncon):
        G = X @ mats[u] @ Zi
        for t in range(ncon):
            Ms[t, u] = np.sum(mats[t] * G)
    want = np.zeros((m, m))
    want[np.ix_(con, con)] = Ms
    err = np.abs(got - want).max() / np.abs(want).max()
    assert err <= 1e-10, err
    assert np.array_equal(got, got.T)


def test_lowrank_route_refuses_a_full_rank_block(cuda):
    n = 50
    rng = np.random.default_rng(5)
    B = rng.standard_normal((n, n))
    mats = [random_lowrank(rng, n, 1, n), B + B.T]
    cptr, cpos, cval = full_lists(mats, n)
    dM = torch.zeros(4, dtype=torch.float64, device=cuda)
    dX = torch.eye(n, dtype=torch.float64, device=cuda)
    dcon = torch.arange(2, dtype=torch.int32, device=cuda)
    rank = np.zeros(1, np.int32)
    with pytest.raises(step.BgpuError) as e:
        step.call("schur_lowrank", n, 2, 2, dcon.data_ptr(), cptr.ctypes.data, cpos.ctypes.data, cval.ctypes.data,
                  dX.data_ptr(), dX.data_ptr(), dM.data_ptr(), rank.ctypes.data, None)
    assert e.value.rc == -6
    assert float(dM.abs().sum()) == 0.0


NT = ["-nohsd", "-dir", "nt", "-mixed", "0", "-tol", "1e-7"]


@pytest.mark.parametrize("name", ["lowrank80", "lowrank80s"])
@pytest.mark.parametrize("run,opts", [("default", FP64), ("init0", FP64 + ["-init", "0"]), ("nt", NT)])
def test_lowrank_solves_match_reference(golden, name, run, opts):
    """Constraints of rank 1-3 (lowrank80: dense vectors; lowrank80s: vectors on 20 of 80 rows):
    the route is taken (its -v line), and status, objectives and DIMACS errors are the reference's
    (whose own low-rank route solves them); the iteration count within one of its."""
    e = golden[name]
    ref = e["runs"][run]
    res = brisk_b200.solve_sdpa(*make(e).args(), options=opts + ["-v"], verbose=False)
    assert "low-rank route" in res.log
    check(res, ref)
    assert abs(res.iterations - ref["iterations"]) <= 1, (res.iterations, ref["iterations"])


def test_lowrank_route_equals_other_routes():
    """-lowrank 0 (the row-product route) and -lowrank 1 give the same solve to DIMACS accuracy."""
    d = problems.lowrank_sdp(n=80, m=150, max_rank=2, support=20, seed=7)
    a = brisk_b200.solve_sdpa(*d.args(), options=FP64 + ["-lowrank", "1", "-v"], verbose=False)
    b = brisk_b200.solve_sdpa(*d.args(), options=FP64 + ["-lowrank", "0", "-v"], verbose=False)
    assert "low-rank route" in a.log and "low-rank route" not in b.log
    assert a.status_str == b.status_str == "OPTIMAL"
    assert abs(a.pobj - b.pobj) <= 1e-7 * (1 + abs(b.pobj))
    assert abs(a.dobj - b.dobj) <= 1e-7 * (1 + abs(b.dobj))
