"""Symbolic phase of the sparse Schur Cholesky (bgpu_schol_analyze, host code: no GPU needed):
the ordering is a permutation, the supernodes partition it, and the predicted structure of L is
exactly the structural Cholesky fill of the clique pattern in that order."""
import numpy as np
import pytest

from brisk_b200 import problems, step


def cliques_of(d):
    """The constraint set of every block (the cliques whose union is the pattern of M)."""
    return [np.unique(d.mat[(d.blk == k) & (d.mat >= 1)] - 1).tolist() for k in range(1, d.nblk + 1)]


def symbolic_fill(m, cliques, perm):
    """Structural Cholesky of the clique pattern in the order perm (dense boolean elimination)."""
    iperm = np.empty(m, int)
    iperm[perm] = np.arange(m)
    A = np.eye(m, dtype=bool)
    for cl in cliques:
        idx = iperm[np.asarray(cl, int)]
        A[np.ix_(idx, idx)] = True
    for k in range(m):
        nz = np.nonzero(A[k + 1:, k])[0] + k + 1
        if nz.size:
            A[np.ix_(nz, nz)] = True
    return np.tril(A)


def analysis_pattern(S):
    sfirst, parent, rptr, rows = S.supernodes()
    m = S.m
    Lp = np.zeros((m, m), dtype=bool)
    for s in range(len(sfirst) - 1):
        r = rows[rptr[s]:rptr[s + 1]]
        for k in range(sfirst[s], sfirst[s + 1]):
            Lp[r[r >= k], k] = True
    return Lp


def random_cliques(m, count, lo, hi, seed):
    rng = np.random.default_rng(seed)
    return [sorted(rng.choice(m, size=int(rng.integers(lo, hi + 1)), replace=False).tolist()) for _ in range(count)]


CASES = {
    "mom8": lambda: (lambda d: (d.m, cliques_of(d)))(problems.moment_relaxation(nvars=8, clique=4, seed=1)),
    "random": lambda: (150, random_cliques(150, 30, 3, 12, 5)),
    "one_clique": lambda: (40, [list(range(40))]),
    "disjoint_and_isolated": lambda: (60, [list(range(0, 10)), list(range(20, 35)), [40, 41]]),
    "chain": lambda: (90, [list(range(i, i + 12)) for i in range(0, 79, 6)]),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_analysis_structure_is_the_exact_fill(name):
    m, cl = CASES[name]()
    S = step.SparseCholesky(m, cl)
    perm = S.perm()
    assert sorted(perm.tolist()) == list(range(m))
    sfirst, parent, rptr, rows = S.supernodes()
    assert sfirst[0] == 0 and sfirst[-1] == m and np.all(np.diff(sfirst) > 0)
    for s in range(len(sfirst) - 1):
        r = rows[rptr[s]:rptr[s + 1]]
        ns = sfirst[s + 1] - sfirst[s]
        assert np.array_equal(r[:ns], np.arange(sfirst[s], sfirst[s + 1]))   # own columns first
        assert np.all(np.diff(r) > 0)
        if r.size > ns:   # the parent holds the first off-diagonal row; parents come later
            t = parent[s]
            assert sfirst[t] <= r[ns] < sfirst[t + 1] and t > s
        else:
            assert parent[s] == -1
    want = symbolic_fill(m, cl, perm)
    got = analysis_pattern(S)
    assert np.array_equal(got, want)
    inf = S.info()
    assert inf["nnz"] == want.sum()
    # the pattern of M below the diagonal
    P = np.zeros((m, m), dtype=bool)
    for c in cl:
        P[np.ix_(c, c)] = True
    assert inf["pattern"] == np.tril(P, -1).sum()
    S.close()


def test_moment_relaxation_factor_is_cheap_and_shallow():
    """The chain-clique moment relaxation (57 blocks of 15, m = 2029): the multiple-elimination
    ordering keeps the factor near the pattern (fill below 50 %), far below the dense flops, and
    the supernode tree shallow (a chain of 57 cliques in at most 8 levels); strict minimum degree
    (delta 0) has less fill and a tall tree."""
    d = problems.moment_relaxation(nvars=60, clique=4, seed=0)
    S = step.SparseCholesky(d.m, cliques_of(d))
    inf = S.info()
    assert inf["nnz"] <= 1.5 * (inf["pattern"] + d.m)
    assert inf["flops"] < 0.01 * d.m ** 3 / 3
    assert inf["levels"] <= 8
    S.close()
    step.lib().bgpu_schol_set_delta(0.0)
    try:
        S0 = step.SparseCholesky(d.m, cliques_of(d))
        inf0 = S0.info()
        S0.close()
    finally:
        step.lib().bgpu_schol_set_delta(1.0)
    assert inf0["nnz"] <= inf["nnz"] and inf0["levels"] > inf["levels"]
    S.close()


def test_bad_cliques_are_rejected():
    with pytest.raises(step.BgpuError):
        step.SparseCholesky(5, [[0, 7]])
