"""The self-dual embedding on a B200 (Solver::run_hsd: this build's homogeneous self-dual
predictor-corrector in the HKM direction, the reference's method choice hsd_run, solver.c:9803)
against the reference's own runs of its embedding (tests/golden/ref_runs.json "hsd_auto": no
-nohsd, the reference's automatic rule picks the embedding on these problems).  Parity: the same
status and exit code, (pobj + dobj) / 2 within 1e-7 relative and each objective within 1e-7 of
the DIMACS denominator (parity.objectives_close: the two embeddings stop at different iterates),
DIMACS errors <= 1e-7.  The reference's embedding, with its correctors and end phases, takes 4-7
iterations here; this one 8-12 (the infeasible method 9-14).  Row by row, the CUDA path is
compared with the oracle's restatement of its own method (oracle solve_hsd), which these
instances pin against the reference's runs on CPU."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import brisk_b200  # noqa: E402
from parity import objectives_close  # noqa: E402
from test_gpu_solve import make  # noqa: E402

HSD = ["-hsd", "-mixed", "0", "-tol", "1e-7"]
SOLVED = ["theta30", "theta50", "rand30", "rand60", "rand100", "mom8", "dense24", "batch_q0", "batch_q5",
          "lowrank80", "lowrank80s", "lp_dense", "lp_mixed"]


@pytest.mark.parametrize("name", SOLVED)
def test_embedding_matches_the_reference_embedding(golden, name):
    e = golden[name]
    ref = e["runs"]["hsd_auto"]
    res = brisk_b200.solve_sdpa(*make(e).args(), options=HSD + ["-v"], verbose=False)
    assert "self-dual embedding, HKM direction" in res.log, res.log
    assert res.status_str == ref["status"] == "OPTIMAL", res.log
    assert res.exit_code == ref["exit_code"] == 0
    objectives_close(res.pobj, res.dobj, ref["pobj"], ref["dobj"])
    assert np.max(np.abs(res.dimacs)) <= 1e-7, res.dimacs


@pytest.mark.parametrize("name,status,code", [("infeas_p", "PRIMAL INFEASIBLE", 11), ("infeas_d", "DUAL INFEASIBLE", 12)])
def test_embedding_certifies_infeasibility(golden, name, status, code):
    """tau -> 0 with kappa > 0: b'y > 0 certifies a primal infeasible problem, <C,X> < 0 a dual
    infeasible one, as the reference's embedding reports them (status and exit code)."""
    e = golden[name]
    for run in ("hsd_auto", "default"):
        assert e["runs"][run]["status"] == status and e["runs"][run]["exit_code"] == code
    for opts in (HSD, ["-mixed", "0", "-tol", "1e-7"]):      # asked for, and the default rule
        res = brisk_b200.solve_sdpa(*make(e).args(), options=opts + ["-v"], verbose=False)
        assert res.status_str == status, res.log
        assert res.exit_code == code
        assert "self-dual embedding" in res.log


@pytest.mark.parametrize("name", ["theta30", "theta50", "rand30", "rand60", "mom8", "dense24", "batch_q0", "batch_q5",
                                  "lp_dense", "lp_mixed", "lp_only", "infeas_p", "infeas_d"])
def test_embedding_follows_the_oracle_restatement(golden, name):
    """The CUDA path's embedding against its numpy FP64 restatement (oracle solve_hsd: the same
    start, Newton system, step rule and stops): the same status and iteration count, and on the
    solved instances the same objectives to 1e-8 relative (they agree to about ten digits).  The
    instances whose blocks all have order <= 64 or are LP blocks: their step lengths are exact
    eigenvalues on both sides, where a larger block's Lanczos estimate, summed in another order
    on the device, could move a marginal stop by an iteration."""
    from oracle import restate
    e = golden[name]
    out = restate.solve_hsd(make(e), tol=1e-7)
    res = brisk_b200.solve_sdpa(*make(e).args(), options=HSD, verbose=False)
    assert res.status_str == out["status_str"], res.log
    assert res.iterations == out["iterations"]
    if out["status_str"] == "OPTIMAL":
        for got, want in ((res.pobj, out["pobj"]), (res.dobj, out["dobj"])):
            assert abs(got - want) <= 1e-8 * max(1.0, abs(want)), (got, want)


def test_default_rule_and_nohsd():
    """Without -hsd or -nohsd the reference's rule (solver.c:13519-13560) picks the embedding for
    problems whose dense work is small next to the Schur factor (a 30 x 30 block, m = 60);
    -nohsd keeps the infeasible-start method.  Both reach the same optimum."""
    e = dict(generator="random_sdp", kwargs=dict(n=30, m=60, density=0.1, seed=1))
    a = brisk_b200.solve_sdpa(*make(e).args(), options=["-mixed", "0", "-tol", "1e-7", "-v"], verbose=False)
    b = brisk_b200.solve_sdpa(*make(e).args(), options=["-nohsd", "-mixed", "0", "-tol", "1e-7", "-v"], verbose=False)
    assert "self-dual embedding first" in a.log and "self-dual embedding, HKM direction" in a.log
    assert "self-dual embedding" not in b.log and "infeasible start" in b.log
    assert a.status_str == b.status_str == "OPTIMAL"
    objectives_close(a.pobj, a.dobj, b.pobj, b.dobj)


def test_embedding_on_the_mixed_path():
    """rand100 by the embedding with the default precision rule (-mixed -1) and with the 3xTF32
    assembly: the same optimum as the reference's embedding."""
    from brisk_b200 import problems
    d = problems.random_sdp(n=100, m=300, density=0.02, seed=3)
    for extra in ([], ["-asmprec", "tf32x3"]):
        res = brisk_b200.solve_sdpa(*d.args(), options=["-hsd", "-tol", "1e-7"] + extra, verbose=False)
        assert res.status_str == "OPTIMAL", res.log
        assert np.max(np.abs(res.dimacs)) <= 1e-7
