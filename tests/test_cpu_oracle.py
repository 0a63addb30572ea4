"""The oracle (oracle/restate.py) against the reference's own runs (tests/golden/ref_runs.json)
and the reference's published golden value, plus the host-side problem plumbing."""
import os

import numpy as np
import pytest

from brisk_b200 import problems
from oracle import restate
from refdir import REF_DIR

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SMALL = ["theta30", "rand30", "rand60"]


def make(entry):
    fn = getattr(problems, entry["generator"])
    return fn(**entry["kwargs"])


@pytest.mark.parametrize("name", ["theta30", "theta50", "rand30", "rand60", "rand100"])
def test_oracle_scaling_and_start_match_reference_iteration0(golden, name):
    """Scaling (problem_prepare) and the SDPT3 start pinned: the reference's iteration-0 row
    (printed to 9 significant digits in pobj/dobj, 3 in the rest) is reproduced."""
    if name not in golden:
        pytest.skip("instance not in the fixtures")
    e = golden[name]
    d = make(e)
    S = restate.scale_problem(d)
    X, Z, y, xi, eta = restate.start_point(S)
    sc = S.bs * S.cs
    n = X[0].shape[0]
    pobj = sc * sum(float(np.sum(C * Xk)) for C, Xk in zip(S.C, X))
    mu = sc * sum(float(np.sum(Xk * Zk)) for Xk, Zk in zip(X, Z)) / n
    rp = S.b - restate.aop(S.A, X)
    pinf = np.linalg.norm(rp * S.du) / (1 + S.normb2)
    row = e["runs"]["init0"]["rows"][0]
    assert -pobj == pytest.approx(row["pobj"], rel=1e-8, abs=1e-8)
    assert mu == pytest.approx(row["mu"], rel=6e-3)
    assert pinf == pytest.approx(row["pinf"], rel=6e-3, abs=1e-15)


def test_oracle_first_schur_is_gram_at_the_start(golden):
    """M0 = (xi/eta) <A_i, A_j> on the scaled data (X0 = xi I, Z0 = eta I)."""
    d = make(golden["rand30"])
    S = restate.scale_problem(d)
    X, Z, y, xi, eta = restate.start_point(S)
    M0 = restate.schur(S.A, X, [np.linalg.inv(Zk) for Zk in Z])
    G = np.einsum("ipq,jpq->ij", S.A[0], S.A[0])
    np.testing.assert_allclose(M0, xi[0] / eta[0] * G, rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("name", SMALL)
def test_oracle_solve_matches_reference(golden, name):
    """Same status, objectives within 1e-7 relative, DIMACS errors <= 1e-7 (the reference's
    -init 0 run: the oracle restates the SDPT3 start).  "Relative" uses the DIMACS gap's
    denominator 1 + |<C,X>| + |b'y|: each solve is only that accurate."""
    e = golden[name]
    ref = e["runs"]["init0"]
    out = restate.solve(make(e), tol=1e-7)
    assert out["status_str"] == ref["status"] == "OPTIMAL"
    den = 1 + abs(ref["pobj"]) + abs(ref["dobj"])
    assert abs(out["pobj"] - ref["pobj"]) <= 1e-7 * den
    assert abs(out["dobj"] - ref["dobj"]) <= 1e-7 * den
    assert np.max(np.abs(out["dimacs"])) <= 1e-7
    assert max(abs(x) for x in ref["dimacs"]) <= 1e-7


@pytest.mark.parametrize("name", ["theta30", "rand30", "rand60", "mom8"])
def test_oracle_nt_solve_matches_reference(golden, name):
    """The restated NT loop against the reference's -dir nt -init 0 run: same status, objectives
    within 1e-7 relative, DIMACS errors <= 1e-7, iterations within 2, and the first rows of the
    iteration table: three rows where every block has order <= 32 (the reference then takes exact
    step lengths, as the oracle does), else the start's row (above 32 the reference's step
    lengths are Lanczos estimates)."""
    e = golden[name]
    ref = e["runs"]["nt_init0"]
    out = restate.solve(make(e), tol=1e-7, direction="nt")
    assert out["status_str"] == ref["status"] == "OPTIMAL"
    den = 1 + abs(ref["pobj"]) + abs(ref["dobj"])
    assert abs(out["pobj"] - ref["pobj"]) <= 1e-7 * den
    assert abs(out["dobj"] - ref["dobj"]) <= 1e-7 * den
    assert np.max(np.abs(out["dimacs"])) <= 1e-7
    assert abs(out["iterations"] - ref["iterations"]) <= 2
    d = make(e)
    nrows = 3 if max(int(b) for b in d.bs) <= 32 else 1
    for mine, theirs in zip(out["table"][:nrows], ref["rows"][:nrows]):
        assert mine["pobj"] == pytest.approx(theirs["pobj"], rel=1e-6, abs=1e-8)
        assert mine["dobj"] == pytest.approx(theirs["dobj"], rel=1e-6, abs=1e-8)


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_DIR, "examples", "theta1.dat-s")), reason="reference tree absent")
def test_oracle_theta1_published_value():
    """theta1 -> 2.2999999997e+01 (the reference's INSTALL.md:44-45)."""
    d = problems.read_sdpa(os.path.join(REF_DIR, "examples", "theta1.dat-s"))
    out = restate.solve(d, tol=1e-8)
    assert out["status_str"] == "OPTIMAL"
    assert -out["pobj"] == pytest.approx(23.0, rel=1e-7)


def test_sdpa_roundtrip(tmp_path):
    d = problems.random_sdp(n=12, m=20, density=0.2, seed=5)
    p = tmp_path / "x.dat-s"
    problems.write_sdpa(d, str(p))
    e = problems.read_sdpa(str(p))
    assert e.m == d.m and list(e.bs) == list(d.bs)
    np.testing.assert_array_equal(e.c, d.c)
    np.testing.assert_array_equal(e.v, d.v)
    np.testing.assert_array_equal(e.i, d.i)
    np.testing.assert_array_equal(e.mat, d.mat)


def test_generators_match_workload_shapes():
    d = problems.theta_problem(n=50, p=0.5, seed=1)
    assert d.m == 588 and int(d.bs[0]) == 50
    d = problems.random_sdp(n=40, m=30, density=0.01 * 20, seed=0)
    k = int(round(0.2 * 40 * 41 / 2))
    assert d.meta["upper_per_con"] == k
    # b_i = <A_i, I>
    C, A = d.dense_blocks()
    np.testing.assert_allclose(np.trace(A[0], axis1=1, axis2=2), d.c, rtol=1e-12, atol=1e-12)
    # C = G G'/n + I is positive definite
    assert np.linalg.eigvalsh(C[0]).min() > 0.99
    sizes = problems.random_dense_batch(count=64, seed=0, sizes_only=True)
    for n, m in sizes:
        assert 8 <= n <= 64 and n <= m <= n * (n + 1) // 4


@pytest.mark.parametrize("name", ["lp_mixed", "lp_only"])
@pytest.mark.parametrize("run,direction", [("init0", "hkm"), ("nt_init0", "nt")])
def test_oracle_lp_blocks_match_reference(golden, name, run, direction):
    """LP blocks (negative sizes) in the restatement: a dense block with diagonal data, whose
    iterates stay diagonal (the LP's own iteration), and the reference's sigma rule for problems
    with LP blocks only (cubic, solver.c:14848-14851).  The reference's -init 0 runs are followed
    to every printed digit: same status and iterations, the first four table rows."""
    e = golden[name]
    ref = e["runs"][run]
    out = restate.solve(make(e), tol=1e-7, direction=direction)
    assert out["status_str"] == ref["status"] == "OPTIMAL"
    assert out["iterations"] == ref["iterations"]
    den = 1 + abs(ref["pobj"]) + abs(ref["dobj"])
    assert abs(out["pobj"] - ref["pobj"]) <= 1e-9 * den
    assert abs(out["dobj"] - ref["dobj"]) <= 1e-9 * den
    for mine, theirs in zip(out["table"][:4], ref["rows"][:4]):
        assert mine["pobj"] == pytest.approx(theirs["pobj"], rel=1e-8, abs=1e-8)
        assert mine["dobj"] == pytest.approx(theirs["dobj"], rel=1e-8, abs=1e-8)


ROW_BY_ROW = ["theta30", "theta50", "rand30", "rand60", "rand100", "mom8", "mom60", "dense24", "dense48", "lp_mixed",
              "lp_only", "lp_dense", "lowrank80", "lowrank80s", "batch_q0", "batch_q1", "batch_q2", "batch_q3",
              "batch_q4", "batch_q5", "batch_q6", "batch_q7", "batch_q8", "batch_q9", "batch_q10", "batch_q11",
              "batch_q3339"]


@pytest.mark.parametrize("name", ROW_BY_ROW)
@pytest.mark.parametrize("run,direction,init", [("default", "hkm", 1), ("nt", "nt", 1), ("init0", "hkm", 0),
                                                ("nt_init0", "nt", 0)])
def test_oracle_follows_reference_row_by_row(golden, name, run, direction, init):
    """The restatement follows the reference's runs row by row over the whole iteration table,
    from both starts (the least-squares start, the reference's default, solver.c:13939-14198; the
    SDPT3 start, -init 0) and in both directions: the same status and iterations, pobj and dobj of
    every row to the printed digits, and its gap, mu, pinf and dinf to theirs (three significant
    digits, to 1 %; in the last rows, at the rounding floor of the residuals, pinf to 1e-11 and
    dinf to 1e-13 absolute: the largest differences over these 95 runs are 4.5e-12 and 3.2e-14).
    Row 0 of a least-squares start also allows pinf 1e-10 and gap 1e-11 absolute: the reference
    solves that start by CG to 1e-10 where the restatement solves it exactly (lowrank80s: pinf
    6.2e-11 against 4.6e-16).  Blocks of order <= 32 take exact eigenvalues, larger ones the
    reference's Lanczos estimate (batch_q2: n = 37, batch_q1: n = 44, theta50, rand60, rand100,
    lowrank80), in the step lengths and in the least-squares start's shifts."""
    e = golden[name]
    if run not in e["runs"]:
        pytest.skip("run not in the fixtures")
    ref = e["runs"][run]
    d = make(e)
    out = restate.solve(d, tol=1e-7, direction=direction, init=init)
    assert out["status_str"] == ref["status"] == "OPTIMAL"
    assert out["iterations"] == ref["iterations"]
    assert len(out["table"]) == len(ref["rows"])
    for mine, theirs in zip(out["table"], ref["rows"]):
        start = init == 1 and theirs["it"] == 0
        assert mine["pobj"] == pytest.approx(theirs["pobj"], rel=1e-7, abs=1e-8)
        assert mine["dobj"] == pytest.approx(theirs["dobj"], rel=1e-7, abs=1e-8)
        assert mine["gap"] == pytest.approx(theirs["gap"], rel=1e-2, abs=1e-11 if start else 1e-14), ("gap", theirs["it"])
        assert mine["mu"] == pytest.approx(theirs["mu"], rel=1e-2, abs=1e-14), ("mu", theirs["it"])
        assert mine["dinf"] == pytest.approx(theirs["dinf"], rel=6e-3, abs=1e-13), ("dinf", theirs["it"])
        assert mine["pinf"] == pytest.approx(theirs["pinf"], rel=6e-3, abs=1e-10 if start else 1e-11), \
            ("pinf", theirs["it"])


@pytest.mark.parametrize("name,status", [("infeas_p", "PRIMAL INFEASIBLE"), ("infeas_d", "DUAL INFEASIBLE")])
@pytest.mark.parametrize("run,direction,init", [("default", "hkm", 1), ("nt", "nt", 1), ("init0", "hkm", 0),
                                                ("nt_init0", "nt", 0)])
def test_oracle_infeasible_method_on_infeasible_problems(golden, name, status, run, direction, init):
    """The infeasible-start method on the two infeasible problems: the reference's status (its
    tests of b'y against |A'y + Z| and of <C,X> against |A(X)|, solver.c:14575-14581) at its
    iteration, and its first five rows to the printed digits; beyond them the iterates diverge
    (objectives of 1e9 to 1e14), and the rows agree only to about 1e-5."""
    e = golden[name]
    if run not in e["runs"]:
        pytest.skip("run not in the fixtures")
    ref = e["runs"][run]
    out = restate.solve(make(e), tol=1e-7, direction=direction, init=init)
    assert out["status_str"] == ref["status"] == status
    assert out["iterations"] == ref["iterations"]
    for mine, theirs in zip(out["table"][:5], ref["rows"][:5]):
        assert mine["pobj"] == pytest.approx(theirs["pobj"], rel=1e-7, abs=1e-8), ("pobj", theirs["it"])
        assert mine["dobj"] == pytest.approx(theirs["dobj"], rel=1e-7, abs=1e-8), ("dobj", theirs["it"])
