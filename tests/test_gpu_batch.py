"""The batch entry point (bgpu_batch_solve) on a B200: instances of the uneven 4096-instance
batch (n ~ U{8..64}, m ~ U{n..n(n+1)/4}, dense N(0,1) A_i, b = A(I), C = G G'/n + I) solved
in one call, each checked against the reference's own solve of that instance and against its
own stand-alone solve through brisk_solve_data.  The default (lockstep) form advances every
instance together with batched kernels; the concurrent form runs the stand-alone solver per
instance on worker streams and gives its bits."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import brisk_b200  # noqa: E402
from brisk_b200 import problems  # noqa: E402
from parity import objectives_close  # noqa: E402

FP64 = ["-nohsd", "-dir", "hkm", "-mixed", "0", "-tol", "1e-7"]
GOLDEN_Q = list(range(12)) + [3339]


def check(res, ref, each=False):
    """Same status; objectives within 1e-7 relative (parity.objectives_close); DIMACS <= 1e-7."""
    assert res.status_str == ref["status"]
    objectives_close(res.pobj, res.dobj, ref["pobj"], ref["dobj"], each=each)
    assert np.max(np.abs(res.dimacs)) <= 1e-7, res.dimacs


@pytest.mark.parametrize("mode", ["lockstep", "concurrent"])
def test_batch_matches_reference(golden, mode):
    """Thirteen instances (the first twelve and the largest, n = 64, m = 1038) in one call.  The
    concurrent form runs each instance's stand-alone solve: where it ends at the reference's
    iteration count, pobj and dobj each within 1e-7 relative.  The lockstep form computes in
    another order (packed rows, one launch over every instance) and may end at another iterate of
    the same accuracy: its (pobj + dobj) / 2 within 1e-7 relative, pobj and dobj each within 1e-7
    of the DIMACS denominator (parity.objectives_close gives the argument)."""
    insts = [problems.batch_instance(q) for q in GOLDEN_Q]
    out = brisk_b200.solve_batch(insts, options=FP64 + ["-batchmode", mode], workers=6)
    assert len(out) == len(insts)
    for q, res in zip(GOLDEN_Q, out):
        assert res.exit_code == 0, (q, res.exit_code)
        ref = golden[f"batch_q{q}"]["runs"]["default"]
        check(res, ref, each=(mode == "concurrent" and res.iterations == ref["iterations"]))


def test_lockstep_batch_matches_standalone_solves():
    """96 instances in lockstep: each has its stand-alone solve's status, DIMACS errors <= 1e-7
    and objectives within 1e-7 of it (the lockstep bar of test_batch_matches_reference)."""
    insts = [problems.batch_instance(q) for q in range(100, 196)]
    out = brisk_b200.solve_batch(insts, options=FP64)
    for d, res in zip(insts, out):
        ref = brisk_b200.solve_sdpa(*d.args(), options=FP64, verbose=False)
        assert res.status == ref.status and res.exit_code == 0
        objectives_close(res.pobj, res.dobj, ref.pobj, ref.dobj, each=False)
        assert np.max(np.abs(res.dimacs)) <= 1e-7
        assert abs(res.iterations - ref.iterations) <= 2


def test_lockstep_bad_instance_does_not_stop_the_others():
    """An entry outside its block gives that problem exit code 2; the lockstep batch solves the rest."""
    good = [problems.batch_instance(q) for q in (5, 6, 7)]
    arrs = brisk_b200.concat_problems(good)
    arrs["i"] = arrs["i"].copy()
    first1 = int(arrs["nnz"][0])
    arrs["i"][first1 + 3] = 99                 # instance 1: row 99 of a 12 x 12 block
    out = brisk_b200.solve_batch_arrays(**arrs, options=FP64)
    assert out[1].exit_code == 2
    assert out[0].status_str == "OPTIMAL" and out[2].status_str == "OPTIMAL"


def test_batch_equals_standalone_solves():
    """Each instance's result in a concurrent batch is bit for bit its stand-alone solve's:
    the workers run the same kernels in the same order on their own streams."""
    insts = [problems.batch_instance(q) for q in range(12, 44)]
    out = brisk_b200.solve_batch(insts, options=FP64 + ["-batchmode", "concurrent"], workers=8)
    for d, res in zip(insts, out):
        ref = brisk_b200.solve_sdpa(*d.args(), options=FP64, verbose=False)
        assert res.exit_code == ref.exit_code and res.status == ref.status
        assert res.iterations == ref.iterations
        assert res.pobj == ref.pobj and res.dobj == ref.dobj
        np.testing.assert_array_equal(res.y, ref.y)
        np.testing.assert_array_equal(res.X[0], ref.X[0])
        np.testing.assert_array_equal(res.dimacs, ref.dimacs)


def test_batch_bad_instance_does_not_stop_the_others():
    """A problem with a bad block size gets exit code 2; the rest of the batch solves."""
    good = [problems.batch_instance(q) for q in (5, 6, 7)]
    arrs = brisk_b200.concat_problems(good)
    arrs["bs"] = arrs["bs"].copy()
    arrs["bs"][1] = 0                        # instance 1: a block of order 0
    out = brisk_b200.solve_batch_arrays(**arrs, options=FP64, workers=2)
    assert out[1].exit_code == 2
    assert out[0].exit_code == 0 and out[2].exit_code == 0
    assert out[0].status_str == "OPTIMAL" and out[2].status_str == "OPTIMAL"


def test_batch_rejects_bad_options():
    d = problems.batch_instance(5)
    with pytest.raises(RuntimeError):
        brisk_b200.solve_batch([d], options=["-tol", "abc"])


def test_resident_batch_runs_twice_like_the_one_call_batch():
    """bgpu_batch_create + bgpu_batch_run (resident) gives the bits of bgpu_batch_solve, run after run."""
    arrs = brisk_b200.concat_problems([problems.batch_instance(q) for q in range(200, 240)])
    ref = brisk_b200.solve_batch_arrays(**arrs, options=FP64)
    sess = brisk_b200.BatchSession(**arrs, options=FP64)
    for _ in range(2):
        out = sess.run()
        for a, b in zip(out, ref):
            assert a.status == b.status and a.iterations == b.iterations
            assert a.pobj == b.pobj and a.dobj == b.dobj
            np.testing.assert_array_equal(a.y, b.y)
    sess.close()


NT = ["-nohsd", "-dir", "nt", "-mixed", "0", "-tol", "1e-7"]


@pytest.mark.parametrize("mode", ["lockstep", "concurrent"])
def test_nt_batch_matches_reference(golden, mode):
    """The NT direction in both batch forms against the reference's -dir nt solves."""
    insts = [problems.batch_instance(q) for q in GOLDEN_Q]
    out = brisk_b200.solve_batch(insts, options=NT + ["-batchmode", mode], workers=6)
    for q, res in zip(GOLDEN_Q, out):
        ref = golden[f"batch_q{q}"]["runs"]["nt"]
        assert res.exit_code == 0, (q, res.exit_code)
        check(res, ref)
        assert abs(res.iterations - ref["iterations"]) <= 2, (q, res.iterations, ref["iterations"])


def test_default_direction_batch_is_nt_in_lockstep():
    """Without -dir the batch's blocks (order <= 64) take NT, as the reference's rule does, and the
    resident lockstep batch gives the bits of the one-call batch with -dir nt."""
    arrs = brisk_b200.concat_problems([problems.batch_instance(q) for q in range(200, 232)])
    ref = brisk_b200.solve_batch_arrays(**arrs, options=NT)
    sess = brisk_b200.BatchSession(**arrs, options=["-nohsd", "-mixed", "0", "-tol", "1e-7"])
    out = sess.run()
    sess.close()
    for a, b in zip(out, ref):
        assert a.status == b.status and a.iterations == b.iterations
        assert a.pobj == b.pobj and a.dobj == b.dobj


def test_every_instance_of_the_4096_batch_matches_its_own_solve():
    """The whole uneven batch, 4096 instances in one lockstep call, each checked against its own
    stand-alone FP64 solve (the concurrent form, which gives brisk_solve_data's bits per instance):
    the same status (all OPTIMAL), DIMACS errors <= 1e-7 in both, objectives within 1e-7 by the
    lockstep bar (parity.objectives_close) and the iteration count within 2."""
    full = problems.batch_arrays(4096)
    lock = brisk_b200.solve_batch_arrays(**full, options=FP64)
    own = brisk_b200.solve_batch_arrays(**full, options=FP64 + ["-batchmode", "concurrent"], workers=16)
    assert len(lock) == len(own) == 4096
    worst = 0.0
    for q, (a, b) in enumerate(zip(lock, own)):
        assert a.exit_code == b.exit_code == 0, (q, a.exit_code, b.exit_code)
        assert a.status_str == b.status_str == "OPTIMAL", q
        objectives_close(a.pobj, a.dobj, b.pobj, b.dobj, each=False)
        worst = max(worst, float(np.max(np.abs(a.dimacs))), float(np.max(np.abs(b.dimacs))))
        assert abs(a.iterations - b.iterations) <= 2, (q, a.iterations, b.iterations)
    assert worst <= 1e-7, worst


def test_batch_work_item_autotuner_keeps_the_bits():
    """The lockstep batch's autotuner times the Q form's work-item sizes on the batch's own data and
    keeps the fastest per block-order class; every size computes each constraint's row alone, so
    the tuned batch gives the bits of the untuned one (-batchtune 0: 8 constraints a CTA)."""
    insts = [problems.batch_instance(q) for q in range(200, 264)]
    tuned = brisk_b200.solve_batch(insts, options=FP64 + ["-batchtune", "1"])
    fixed = brisk_b200.solve_batch(insts, options=FP64 + ["-batchtune", "0"])
    for a, b in zip(tuned, fixed):
        assert a.exit_code == b.exit_code == 0
        assert (a.pobj, a.dobj, a.iterations) == (b.pobj, b.dobj, b.iterations)
        np.testing.assert_array_equal(a.y, b.y)
