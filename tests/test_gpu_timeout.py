"""Failure detection on the GPU without a fault: a bounded device wait that runs out.

The triangular solves chain their block rows by flags: the CTA of block row r waits (a bounded
number of polls) for the flags of the rows before it.  bgpu_test_hold_trsv_row(r) makes the CTA
of row r compute its rows but never publish its flag, so the rows after it wait for a flag that
nothing sets; with a short bound (bgpu_set_wait_limit) they give up, the solve sets its error
flag, every CTA returns, and the host reads BGPU_ERR_TIMEOUT.  The context stays usable: the
same solve then runs normally and gives the right answer.  No GPU fault, trap or hang is
involved."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from brisk_b200 import _core, problems, step  # noqa: E402

SHORT = 2000   # polls of 64 ns: about 0.1-0.3 ms before a waiting block row gives up


@pytest.fixture
def held_row():
    L = step.lib()
    L.bgpu_set_wait_limit.argtypes = [ctypes.c_uint]
    L.bgpu_set_wait_limit.restype = None
    L.bgpu_test_hold_trsv_row.argtypes = [ctypes.c_int]
    L.bgpu_test_hold_trsv_row.restype = None

    def hold(r, limit=SHORT):
        L.bgpu_set_wait_limit(limit)
        L.bgpu_test_hold_trsv_row(r)
    yield hold
    L.bgpu_test_hold_trsv_row(-1)
    L.bgpu_set_wait_limit(0)


def factor(n, seed):
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    A = (Q * np.logspace(0, 2, n)) @ Q.T
    cuda = torch.device("cuda:0")
    L = torch.as_tensor(np.ascontiguousarray(A.T), device=cuda).contiguous()
    nb = (n + 63) // 64
    dinv = torch.zeros(nb * 4096, dtype=torch.float64, device=cuda)
    info = torch.zeros(1, dtype=torch.int32, device=cuda)
    pmin = torch.zeros(1, dtype=torch.float64, device=cuda)
    step.call("potrf", n, L.data_ptr(), n, dinv.data_ptr(), info.data_ptr(), pmin.data_ptr(), None)
    step.call("sync", None)
    assert int(info.item()) == 0
    return A, L, dinv


@pytest.mark.parametrize("trans", [0, 1])
def test_trsv_wait_runs_out_and_the_context_stays_usable(held_row, trans):
    n = 64 * 6
    A, L, dinv = factor(n, 3)
    cuda = torch.device("cuda:0")
    flags = torch.zeros((n + 63) // 64, dtype=torch.int32, device=cuda)
    err = torch.zeros(1, dtype=torch.int32, device=cuda)
    b = np.random.default_rng(5).standard_normal(n)
    x = torch.as_tensor(b, device=cuda).clone()
    # trans 0 runs the block rows top-down (row 2 held: rows 3..5 wait on it); trans 1 bottom-up
    held_row(2 if trans == 0 else 3)
    step.call("trsv", n, L.data_ptr(), n, dinv.data_ptr(), x.data_ptr(), trans, flags.data_ptr(), 1,
              err.data_ptr(), None)
    step.call("sync", None)
    assert int(err.item()) == 1
    # the entry point that reads the flag back itself returns BGPU_ERR_TIMEOUT
    with pytest.raises(step.BgpuError) as e:
        step.call("trsv_noalloc", n, L.data_ptr(), n, dinv.data_ptr(), x.data_ptr(), trans, None)
    assert e.value.rc == -4
    # back to normal solves: the same context gives the right answer
    held_row(-1, 0)
    err.zero_()
    x = torch.as_tensor(b, device=cuda).clone()
    step.call("trsv", n, L.data_ptr(), n, dinv.data_ptr(), x.data_ptr(), 0, flags.data_ptr(), 2, err.data_ptr(), None)
    step.call("trsv", n, L.data_ptr(), n, dinv.data_ptr(), x.data_ptr(), 1, flags.data_ptr(), 3, err.data_ptr(), None)
    step.call("sync", None)
    assert int(err.item()) == 0
    np.testing.assert_allclose(x.cpu().numpy(), np.linalg.solve(A, b), rtol=1e-9, atol=1e-11)


def test_solve_reports_the_timeout_and_the_next_solve_succeeds(held_row):
    """Inside a whole solve (the PCG preconditioner's triangular solves of the dense factor of
    M, m = 200: 4 block rows): brisk_solve_data returns the abort exit code -3 with a GPU-failure
    message naming the timeout code (-4), and the next solve on the same context is OPTIMAL."""
    d = problems.random_sdp(n=30, m=200, density=0.1, seed=1)
    opts = ["-nohsd", "-dir", "hkm", "-tol", "1e-7", "-mixed", "0", "-init", "0"]
    held_row(1)
    with pytest.raises(RuntimeError) as e:   # the binding raises on an aborted solve (exit code < 0)
        _core.solve_sdpa(*d.args(), options=opts, verbose=False)
    assert "aborted (code -3)" in str(e.value) and "GPU failure (code -4" in str(e.value), str(e.value)
    held_row(-1, 0)
    r = _core.solve_sdpa(*d.args(), options=opts, verbose=False)
    assert r.status_str == "OPTIMAL", r.log
