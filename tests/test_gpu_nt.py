"""The NT direction on a B200 through the C interface: the scaling kernels (bgpu_nt_scaling, the
one-CTA form for n <= 64 and block Jacobi above) against the oracle's nt_scaling
(oracle/restate.py, solver.c:7824-7912), and NT solves against the reference's own runs with
-dir nt (tests/golden/ref_runs.json, runs "nt", made from oracle/_ref)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import brisk_b200  # noqa: E402
from brisk_b200 import problems, step  # noqa: E402
from oracle import restate  # noqa: E402
from parity import objectives_close  # noqa: E402

NT = ["-nohsd", "-dir", "nt", "-mixed", "0", "-tol", "1e-7"]


def spd(rng, n, lo, hi):
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    return (Q * np.geomspace(lo, hi, n)) @ Q.T


def colmajor(A, cuda):
    return torch.as_tensor(np.ascontiguousarray(np.asarray(A).T)).to(cuda)


def from_colmajor(t, n):
    return t.cpu().numpy().reshape(n, n).T


def scaling(X, Z, cuda):
    n = X.shape[0]
    LX, LZ = np.linalg.cholesky(X), np.linalg.cholesky(Z)
    # the strict upper triangles hold garbage: the kernels must read the lower ones only
    junk = np.triu(np.full((n, n), 7.0), 1)
    G, lam, W, sweeps = step.nt_scaling(colmajor(LX + junk, cuda), colmajor(LZ - junk, cuda))
    torch.cuda.synchronize()
    return from_colmajor(G, n), lam.cpu().numpy(), from_colmajor(W, n), sweeps, LX, LZ


@pytest.mark.parametrize("n,lo,hi", [(1, 2.0, 2.0), (2, 0.5, 2.0), (15, 1e-2, 10.0), (33, 1e-4, 1.0),
                                     (64, 1e-3, 10.0), (65, 1e-3, 10.0), (130, 1e-4, 1.0), (400, 1e-3, 10.0),
                                     (1201, 1e-2, 1.0)])
def test_nt_scaling_matches_oracle(cuda, n, lo, hi):
    rng = np.random.default_rng(1000 + n)
    X, Z = spd(rng, n, lo, hi), spd(rng, n, lo, hi)
    G, lam, W, sweeps, LX, LZ = scaling(X, Z, cuda)
    Go, lamo, Wo = restate.nt_scaling(LX, LZ)
    np.testing.assert_allclose(np.sort(lam)[::-1], lamo, rtol=1e-9, atol=1e-13 * lamo[0])
    assert np.linalg.norm(W - Wo) <= 1e-9 * np.linalg.norm(Wo)
    assert np.array_equal(W, W.T)
    # the device G itself: G' Z G = diag(lam), G G' = W
    assert np.linalg.norm(G.T @ Z @ G - np.diag(lam)) <= 1e-10 * np.sqrt(n) * lam.max()
    assert np.linalg.norm(G @ G.T - W) <= 1e-12 * np.linalg.norm(W)
    if n > 64:
        assert 1 <= sweeps <= 40
    else:
        assert sweeps == 0


@pytest.mark.parametrize("n", [20, 200])
def test_nt_scaling_on_the_central_path(cuda, n):
    """Z = mu X^-1: X Z = mu I, every lam = sqrt(mu) (one cluster) and W = X / sqrt(mu)."""
    rng = np.random.default_rng(n)
    X = spd(rng, n, 1e-3, 1e3)
    mu = 1e-8
    Z = mu * np.linalg.inv(X)
    Z = 0.5 * (Z + Z.T)
    G, lam, W, sweeps, LX, LZ = scaling(X, Z, cuda)
    np.testing.assert_allclose(lam, np.sqrt(mu), rtol=1e-7)
    assert np.linalg.norm(W - X / np.sqrt(mu)) <= 1e-7 * np.linalg.norm(X / np.sqrt(mu))


def test_nt_scaling_graph_replay_matches_direct_launches(cuda):
    """On a created stream each sweep is a cached CUDA graph; on the default stream the rounds are
    launched one by one: the same bits either way, and on a second (cached) replay."""
    rng = np.random.default_rng(77)
    n = 300
    X, Z = spd(rng, n, 1e-4, 1.0), spd(rng, n, 1e-4, 1.0)
    LX, LZ = colmajor(np.linalg.cholesky(X), cuda), colmajor(np.linalg.cholesky(Z), cuda)
    G0, lam0, W0, s0 = step.nt_scaling(LX, LZ)
    torch.cuda.synchronize()
    st = torch.cuda.Stream()
    for _ in range(2):
        G1, lam1, W1, s1 = step.nt_scaling(LX, LZ, st.cuda_stream)
        torch.cuda.synchronize()
        assert s1 == s0
        assert torch.equal(G0, G1) and torch.equal(lam0, lam1) and torch.equal(W0, W1)


def test_nt_scaling_rejects_bad_arguments(cuda):
    z = torch.zeros((4, 4), dtype=torch.float64, device=cuda)
    rc = step.lib().bgpu_nt_scaling(0, z.data_ptr(), z.data_ptr(), z.data_ptr(), z.data_ptr(), z.data_ptr(),
                                    z.data_ptr(), 256, None, None)
    assert rc == -2
    rc = step.lib().bgpu_nt_scaling(100, z.data_ptr(), z.data_ptr(), z.data_ptr(), z.data_ptr(), z.data_ptr(),
                                    z.data_ptr(), 256, None, None)   # workspace too small for n = 100
    assert rc == -2


def make(entry):
    return getattr(problems, entry["generator"])(**entry["kwargs"])


def check(res, ref):
    """Same status; objectives within 1e-7 relative (parity.objectives_close); DIMACS <= 1e-7."""
    assert res.status_str == ref["status"], res.log
    objectives_close(res.pobj, res.dobj, ref["pobj"], ref["dobj"], each=res.iterations == ref["iterations"])
    assert np.max(np.abs(res.dimacs)) <= 1e-7, res.dimacs


@pytest.mark.parametrize("name", ["theta30", "theta50", "rand30", "rand60", "rand100", "mom8", "mom60", "dense24",
                                  "dense48", "batch_q5", "batch_q3339"])
def test_nt_solve_matches_reference(golden, name):
    e = golden[name]
    ref = e["runs"]["nt"]
    res = brisk_b200.solve_sdpa(*make(e).args(), options=NT, verbose=False)
    check(res, ref)
    assert abs(res.iterations - ref["iterations"]) <= 2, (res.iterations, ref["iterations"])


def test_nt_solve_full_size(golden):
    """The n = 400, m = 2000 workload with the NT direction against the reference's NT solve."""
    e = golden["rand400"]
    res = brisk_b200.solve_sdpa(*make(e).args(), options=NT, verbose=False)
    check(res, e["runs"]["nt"])


def test_auto_direction_takes_nt_on_small_blocks(golden):
    """-dir auto (the default) takes NT where 15 sum n^3 <= 1e8 (solver.c:13585-13591): rand60's
    solve without -dir is the -dir nt solve, bit for bit; rand400 (m = 2000, n = 400) stays HKM."""
    d = make(golden["rand60"])
    auto = brisk_b200.solve_sdpa(*d.args(), options=["-nohsd", "-mixed", "0", "-tol", "1e-7"], verbose=False)
    nt = brisk_b200.solve_sdpa(*d.args(), options=NT, verbose=False)
    assert auto.iterations == nt.iterations and auto.pobj == nt.pobj and auto.dobj == nt.dobj
    np.testing.assert_array_equal(auto.y, nt.y)
    assert "NT direction" in auto.log
    big = brisk_b200.solve_sdpa(*make(golden["rand400"]).args(), options=["-nohsd", "-mixed", "0", "-tol", "1e-7"],
                                verbose=False)
    assert "HKM direction" in big.log
    check(big, golden["rand400"]["runs"]["default"])
