"""The oracle's NT scaling (oracle/restate.py: nt_scaling, solver.c:7824-7912) on the CPU: the
scaling point's defining identities, W Z W = X and G' Z G = G^-1 X G^-T = diag(lam), and lam^2
the eigenvalues of X Z."""
import numpy as np
import pytest

from oracle import restate


def spd(rng, n, lo, hi):
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    return (Q * np.geomspace(lo, hi, n)) @ Q.T


@pytest.mark.parametrize("n,lo,hi", [(5, 0.5, 2.0), (30, 1e-3, 10.0), (64, 1e-6, 1.0)])
def test_oracle_nt_scaling_identities(n, lo, hi):
    rng = np.random.default_rng(n)
    X, Z = spd(rng, n, lo, hi), spd(rng, n, lo, hi)
    G, lam, W = restate.nt_scaling(np.linalg.cholesky(X), np.linalg.cholesky(Z))
    assert np.all(np.diff(lam) <= 0)
    sc = np.linalg.norm(X)
    assert np.linalg.norm(W @ Z @ W - X) <= 1e-9 * sc
    assert np.linalg.norm(G.T @ Z @ G - np.diag(lam)) <= 1e-9 * np.linalg.norm(lam)
    Gi = np.linalg.inv(G)
    assert np.linalg.norm(Gi @ X @ Gi.T - np.diag(lam)) <= 1e-9 * np.linalg.norm(lam)
    ev = np.sort(np.linalg.eigvals(X @ Z).real)[::-1]
    np.testing.assert_allclose(lam ** 2, ev, rtol=1e-8, atol=1e-12 * ev[0])   # eigvals of X Z: absolute accuracy
