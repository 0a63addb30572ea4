"""The supernodal sparse Schur factor on a B200 (bgpu_schol_factor / bgpu_schol_solve): the
factor of D M D + reg I on the clique pattern solves like numpy's dense solve, a matrix that is
not positive definite is reported (no fault), and the moment relaxation solves to the
reference's result with the sparse factor."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import brisk_b200  # noqa: E402
from brisk_b200 import problems, step  # noqa: E402
from parity import objectives_close  # noqa: E402

FP64 = ["-nohsd", "-dir", "hkm", "-mixed", "0", "-tol", "1e-7"]


def cliques_of(d):
    return [np.unique(d.mat[(d.blk == k) & (d.mat >= 1)] - 1).tolist() for k in range(1, d.nblk + 1)]


def pattern_spd(m, cliques, seed, shift=1e-3):
    """A symmetric positive definite matrix whose pattern is the union of the cliques."""
    rng = np.random.default_rng(seed)
    M = np.zeros((m, m))
    for cl in cliques:
        B = rng.standard_normal((len(cl), len(cl)))
        M[np.ix_(cl, cl)] += B @ B.T / len(cl)
    M += shift * np.eye(m)
    return M


def factor_solve(S, M, cuda, reg=0.0):
    m = M.shape[0]
    dM = torch.as_tensor(M.T.copy().ravel(), device=cuda)
    D = 1.0 / np.sqrt(np.abs(np.diag(M)))
    dD = torch.as_tensor(D, device=cuda)
    info, pmin = ctypes.c_int(0), ctypes.c_double(0)
    step.call("schol_factor", S.h, dM.data_ptr(), m, dD.data_ptr(), reg, ctypes.addressof(info),
              ctypes.addressof(pmin), None)
    return dM, dD, D, info.value, pmin.value


@pytest.mark.parametrize("name,nv", [("mom8", 8), ("mom60", 60)])
def test_sparse_factor_solves_like_dense(cuda, name, nv):
    d = problems.moment_relaxation(nvars=nv, clique=4, seed=1 if nv == 8 else 0)
    cl = cliques_of(d)
    S = step.SparseCholesky(d.m, cl)
    M = pattern_spd(d.m, cl, 3)
    dM, dD, D, info, pmin = factor_solve(S, M, cuda)
    assert info == 0 and 0 < pmin <= 1
    b = np.random.default_rng(4).standard_normal(d.m)
    x = torch.as_tensor(b, device=cuda)
    step.call("schol_solve", S.h, dD.data_ptr(), x.data_ptr(), None)
    step.call("sync", None)
    want = np.linalg.solve(M, b)
    got = x.cpu().numpy()
    assert np.linalg.norm(got - want) <= 1e-12 * np.linalg.cond(M) * np.linalg.norm(want)
    # the smallest pivot of the scaled matrix: the dense Cholesky's, to rounding
    Ms = D[:, None] * M * D[None, :]
    perm = S.perm()
    Lp = np.linalg.cholesky(Ms[np.ix_(perm, perm)])
    assert pmin == pytest.approx(np.min(np.diag(Lp)) ** 2, rel=1e-8)
    S.close()


def test_sparse_factor_reports_indefinite(cuda):
    d = problems.moment_relaxation(nvars=8, clique=4, seed=1)
    cl = cliques_of(d)
    S = step.SparseCholesky(d.m, cl)
    M = pattern_spd(d.m, cl, 5)
    M[np.ix_(cl[2], cl[2])] -= 3.0 * np.eye(len(cl[2]))   # indefinite on one clique
    _, _, _, info, _ = factor_solve(S, M, cuda)
    assert info > 0
    # the same handle factors a positive definite matrix again
    _, _, _, info2, _ = factor_solve(S, pattern_spd(d.m, cl, 6), cuda)
    assert info2 == 0
    S.close()


@pytest.mark.parametrize("sparse", ["1", "-1"])
def test_moment_relaxation_sparse_factor_matches_reference(golden, sparse):
    """mom60 (57 moment blocks of 15, m = 2029) with the sparse Schur factor (forced, and the
    automatic choice, which takes it) against the reference's solve."""
    e = golden["mom60"]
    d = problems.moment_relaxation(**e["kwargs"])
    res = brisk_b200.solve_sdpa(*d.args(), options=FP64 + ["-sparse", sparse, "-v"], verbose=False)
    assert "sparse Cholesky" in res.log
    ref = e["runs"]["default"]
    assert res.status_str == ref["status"]
    objectives_close(res.pobj, res.dobj, ref["pobj"], ref["dobj"], each=res.iterations == ref["iterations"])
    assert np.max(np.abs(res.dimacs)) <= 1e-7


def test_large_moment_relaxation_sparse_matches_reference(golden):
    """The chain moment relaxation in 700 variables (697 blocks of 15, m = 24429): the automatic
    choice takes the sparse factor; the result matches the reference's."""
    e = golden["mom700"]
    d = problems.moment_relaxation(**e["kwargs"])
    res = brisk_b200.solve_sdpa(*d.args(), options=FP64 + ["-v"], verbose=False)
    assert "sparse Cholesky" in res.log
    ref = e["runs"]["default"]
    assert res.status_str == ref["status"]
    objectives_close(res.pobj, res.dobj, ref["pobj"], ref["dobj"], each=res.iterations == ref["iterations"])
    assert np.max(np.abs(res.dimacs)) <= 1e-7


@pytest.mark.parametrize("name,nv", [("mom8", 8), ("mom60", 60)])
def test_sparse_factor_f32_solves_like_dense(cuda, name, nv):
    """bgpu_schol_factor_f32: the fronts, L and the update matrices in FP32.  The solve agrees with
    numpy's FP64 solve within the FP32 factor's error (a few ulps of FP32 times the condition
    number of the scaled matrix), and the smallest pivot with the FP64 factor's to FP32 rounding."""
    d = problems.moment_relaxation(nvars=nv, clique=4, seed=1 if nv == 8 else 0)
    cl = cliques_of(d)
    S = step.SparseCholesky(d.m, cl)
    M = pattern_spd(d.m, cl, 3)
    _, _, D, info64, pmin64 = factor_solve(S, M, cuda)
    assert info64 == 0
    dM = torch.as_tensor(M.T.copy().ravel(), device=cuda)
    dD = torch.as_tensor(D, device=cuda)
    info, pmin = ctypes.c_int(0), ctypes.c_double(0)
    step.call("schol_factor_f32", S.h, dM.data_ptr(), d.m, dD.data_ptr(), 0.0, ctypes.addressof(info),
              ctypes.addressof(pmin), None)
    assert info.value == 0
    assert pmin.value == pytest.approx(pmin64, rel=1e-4)
    b = np.random.default_rng(4).standard_normal(d.m)
    x = torch.as_tensor(b, device=cuda)
    step.call("schol_solve", S.h, dD.data_ptr(), x.data_ptr(), None)
    step.call("sync", None)
    want = np.linalg.solve(M, b)
    cond_s = np.linalg.cond(D[:, None] * M * D[None, :])
    err = np.linalg.norm(x.cpu().numpy() - want) / np.linalg.norm(want)
    assert err <= 64 * 2.0 ** -24 * cond_s, (err, cond_s)
    assert err > 1e-12   # it is the FP32 factor that solved
    # the next FP64 factor on the same handle solves to FP64 accuracy again
    _, dD2, _, info2, _ = factor_solve(S, M, cuda)
    x = torch.as_tensor(b, device=cuda)
    step.call("schol_solve", S.h, dD2.data_ptr(), x.data_ptr(), None)
    step.call("sync", None)
    assert info2 == 0
    assert np.linalg.norm(x.cpu().numpy() - want) <= 1e-12 * np.linalg.cond(M) * np.linalg.norm(want)
    S.close()


@pytest.mark.parametrize("name", ["mom60", "mom700"])
def test_moment_relaxation_fp32_early_sparse_factor_matches_reference(golden, name):
    """The mixed form of the sparse path (-mixed 1; the default for m >= 1000): FP32 fronts while
    mu >= 1e-4, FP64 after, PCG against the FP64 M throughout.  Against the reference's FP64
    solve: the same status, objectives by the parity bar, DIMACS <= 1e-7; the log shows both
    factor types."""
    e = golden[name]
    d = problems.moment_relaxation(**e["kwargs"])
    opts = ["-nohsd", "-dir", "hkm", "-mixed", "1", "-tol", "1e-7", "-sparse", "1", "-vv"]
    res = brisk_b200.solve_sdpa(*d.args(), options=opts, verbose=False)
    assert "sparse Cholesky" in res.log
    assert "factor fp32" in res.log and "factor fp64" in res.log, res.log
    ref = e["runs"]["default"]
    assert res.status_str == ref["status"]
    objectives_close(res.pobj, res.dobj, ref["pobj"], ref["dobj"], each=res.iterations == ref["iterations"])
    assert np.max(np.abs(res.dimacs)) <= 1e-7
