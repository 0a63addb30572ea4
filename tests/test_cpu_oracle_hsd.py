"""The oracle's restatement of the self-dual embedding (oracle/restate.py: solve_hsd, the method
of Solver::run_hsd) against the reference's own runs of its embedding (tests/golden/ref_runs.json
"hsd_auto": without -nohsd the reference's rule, solver.c:13519-13560, picks the embedding on
these problems).  The two embeddings take different iterates (the reference's adds correctors
and end phases: 4-7 iterations against 8-12), so the bar is the outcome: the same status, the
objectives by parity.objectives_close, DIMACS errors <= 1e-7, and for the infeasible instances
the same certificate.  The CUDA path's runs are compared with this restatement in
tests/test_gpu_hsd.py."""
import numpy as np
import pytest

from oracle import restate
from parity import objectives_close
from test_cpu_oracle import make

SOLVED = ["theta30", "theta50", "rand30", "rand60", "rand100", "mom8", "dense24", "batch_q0", "batch_q5",
          "lowrank80", "lowrank80s", "lp_dense", "lp_mixed", "lp_only"]


@pytest.mark.parametrize("name", SOLVED)
def test_oracle_embedding_matches_the_reference_embedding(golden, name):
    e = golden[name]
    ref = e["runs"]["hsd_auto"]
    out = restate.solve_hsd(make(e), tol=1e-7)
    assert out["status_str"] == ref["status"] == "OPTIMAL"
    objectives_close(out["pobj"], out["dobj"], ref["pobj"], ref["dobj"])
    assert np.max(np.abs(out["dimacs"])) <= 1e-7, out["dimacs"]
    assert ref["iterations"] < out["iterations"] <= 12


@pytest.mark.parametrize("name,status", [("infeas_p", "PRIMAL INFEASIBLE"), ("infeas_d", "DUAL INFEASIBLE")])
def test_oracle_embedding_certifies_infeasibility(golden, name, status):
    """tau -> 0 with kappa > 1e8 tau: b'y > 0 certifies primal infeasibility, <C,X> < 0 dual
    infeasibility, the reference's embedding's status on the same problems."""
    e = golden[name]
    assert e["runs"]["hsd_auto"]["status"] == status
    out = restate.solve_hsd(make(e), tol=1e-7)
    assert out["status_str"] == status
    assert out["kappa"] > 1e8 * out["tau"]
    last = out["table"][-1]
    if status == "PRIMAL INFEASIBLE":
        assert last["dobj"] < 0          # the table's sign convention: -b'y / tau, b'y > 0
    else:
        assert last["pobj"] > 0          # -<C,X> / tau, <C,X> < 0


def test_oracle_embedding_residuals_fall_together(golden):
    """One step length for every variable: the embedding's residuals rp = b tau - A(X) and
    Rd = C tau - A'y - Z fall by the same factor 1 - eta alpha an iteration (the Newton equations
    A(dX) - b dtau = eta rp and A'dy + dZ - C dtau = eta Rd), so pinf / dinf, the ratio of their
    norms, is constant along the solve (to rounding) until the last rows."""
    e = golden["rand30"]
    out = restate.solve_hsd(make(e), tol=1e-7)
    rows = out["table"]
    r = [row["pinf"] / row["dinf"] for row in rows[:6]]
    assert max(r) / min(r) < 1 + 1e-6, r


@pytest.mark.parametrize("name", ["rand30", "theta50", "mom8", "lp_mixed"])
def test_oracle_embedding_solves_its_newton_system(golden, name):
    """Every direction the restatement takes satisfies the embedding's linearised equations
    (solve_hsd's check).  The dual equation A'dy + dZ = C dtau + eta Rd and the tau-kappa one
    hold to rounding by construction.  The primal one and the gap equation pass through the
    Schur solves, whose residual is eps cond(M): 1e-16 to 1e-13 while mu >= 1e-2, growing like
    1/mu^2 near the end (up to 3e-6 relative at mu ~ 1e-7 on lp_mixed)."""
    out = restate.solve_hsd(make(golden[name]), tol=1e-7, check=True)
    assert out["status_str"] == "OPTIMAL"
    assert len(out["newton"]) == 2 * out["iterations"]          # a predictor and a corrector each
    for it, e1, e2, e3, e4 in out["newton"]:
        assert e2 <= 1e-14 and e4 <= 1e-14, (it, e2, e4)
        bound = 1e-12 if out["table"][it]["mu"] >= 1e-2 else 1e-4
        assert e1 <= bound and e3 <= bound, (it, e1, e3)
