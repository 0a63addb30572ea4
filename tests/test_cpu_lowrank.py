"""The host half of the low-rank Schur route (bgpu_lowrank_factor, no GPU): every constraint of a
block factored as A_t = sum_k sig_k w_k w_k' with unit w_k, from its full-expansion lists, by
exact Jacobi on supports of up to 32 rows and by a checked random range sketch above; constraints
without a factor of rank below 28 make the block keep its other routes."""
import ctypes

import numpy as np
import pytest

from brisk_b200 import problems, step


def full_lists(mats, n):
    """cptr, cpos (p + q n, ascending), cval of symmetric n x n matrices (both triangles)."""
    cptr, cpos, cval = [0], [], []
    for A in mats:
        q, p = np.nonzero(A.T)                   # column-major order: by column q, then row p
        pos = p + q * n
        order = np.argsort(pos)
        cpos.append(pos[order].astype(np.int32))
        cval.append(A[p, q][order])
        cptr.append(cptr[-1] + pos.size)
    return (np.array(cptr, np.int64), np.concatenate(cpos) if cpos else np.zeros(0, np.int32),
            np.concatenate(cval) if cval else np.zeros(0))


def factor(mats, n, max_rank=4096):
    cptr, cpos, cval = full_lists(mats, n)
    ncon = len(mats)
    off = np.zeros(ncon + 1, np.int32)
    W = np.zeros(n * max_rank)
    sig = np.zeros(max_rank)
    L = step.lib()
    R = L.bgpu_lowrank_factor(n, ncon, cptr.ctypes.data, cpos.ctypes.data, cval.ctypes.data, max_rank,
                              off.ctypes.data, W.ctypes.data, sig.ctypes.data)
    if R < 0:
        return R, None, None, None
    return R, off, W[:n * R].reshape(R, n).T, sig[:R]


def random_lowrank(rng, n, rank, support):
    A = np.zeros((n, n))
    for _ in range(rank):
        g = np.zeros(n)
        rows = rng.choice(n, size=support, replace=False)
        g[rows] = rng.standard_normal(support)
        A += rng.choice([-1.0, 1.0]) * np.outer(g, g)
    return A


@pytest.mark.parametrize("n,support", [(40, 6), (60, 60), (200, 150), (33, 33)])
def test_factors_reproduce_each_constraint(libpath, n, support):
    rng = np.random.default_rng(n + support)
    mats = [random_lowrank(rng, n, int(rng.integers(1, 6)), support) for _ in range(25)]
    mats.append(np.zeros((n, n)))                       # a constraint with no entry in the block
    e = np.zeros((n, n)); e[3, 5] = e[5, 3] = 1.0       # X_ij = 0: rank 2, values +-1
    mats.append(e)
    R, off, W, sig = factor(mats, n)
    assert R > 0
    np.testing.assert_allclose(np.linalg.norm(W, axis=0), 1.0, rtol=1e-12)
    for t, A in enumerate(mats):
        cols = slice(off[t], off[t + 1])
        got = (W[:, cols] * sig[cols]) @ W[:, cols].T
        np.testing.assert_allclose(got, A, rtol=0, atol=1e-12 * max(1.0, np.abs(A).max()))
        assert off[t + 1] - off[t] == np.linalg.matrix_rank(A)
    assert off[-2] == off[-3]                           # the empty constraint has rank 0


def test_full_rank_constraint_is_refused(libpath):
    rng = np.random.default_rng(3)
    n = 50
    B = rng.standard_normal((n, n))
    mats = [random_lowrank(rng, n, 2, n), B + B.T]
    R, *_ = factor(mats, n)
    assert R == -6
    # and the rank limit
    R, *_ = factor([random_lowrank(rng, n, 3, n) for _ in range(4)], n, max_rank=10)
    assert R == -6


def test_generator_constraints_factor_with_their_ranks(libpath):
    d = problems.lowrank_sdp(n=30, m=12, max_rank=3, support=0, seed=2)
    _, A = d.dense_blocks()
    mats = list(A[0])
    R, off, W, sig = factor(mats, 30)
    assert R == sum(np.linalg.matrix_rank(a) for a in mats)
    np.testing.assert_allclose(d.c, [np.trace(a) for a in mats], rtol=1e-12)   # b = A(I)
