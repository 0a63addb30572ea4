"""Oracle: a CPU (numpy, FP64) restatement of the reference's SDP interior-point Newton step.

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg may import this module, and only as the checker; the product (brisk_b200/libbrisk.so) never
calls it and has no CPU path.

It restates, on dense matrices (small sizes: tests), the reference BRISK 1.7 algorithm:

* problem_prepare        row equilibration and b/C scaling         problem.c:1866-1910
* start_sdpt3            X0 = xi I, Z0 = eta I, y = 0 (-init 0)     solver.c:6622-6661
* the least-squares start (the default) from A A' and shifts         solver.c:13939-14198
* schur (HKM)            M_ij = <A_i, X A_j Z^-1>                    solver.c:1969, 2339-3021
* the infeasible-start predictor-corrector loop, HKM or NT          solver.c:14394-15188
  (residuals 14423-14484, theta R0 recurrence 14317-14326 / 14587-14607, rhs pieces
  14715-14735, predictor 14787-14818, sigma rule 14829-14873, corrector 14998-15050,
  refinement of A(dX) = rp 15058-15105, try_step 6393-6447)
* maxstep                the largest alpha with V + alpha dV >= 0     solver.c:6300-6390
  (exact eigenvalues up to order 32 and for LP blocks; above, the Lanczos   solver.c:6083-6225
  estimate theta - residual, as the reference takes it)
* LP blocks (negative sizes) as dense blocks of diagonal data, their iterates diagonal, and the
  cubic sigma rule for problems of LP blocks only                      solver.c:14848-14851
* nt_scaling             the NT scaling G, lam, W = G G' from the     solver.c:7824-7912
                         factors of X and Z (eigenvectors of Mb' Mb,
                         Mb = L_Z' L_X; lam descending)
* DIMACS errors on the data as given                                  postsolve.c:2880-2897
* the final status rule                                               main.c:2349-2362
* solve_hsd: the CUDA path's self-dual embedding (its own method in the place of hsd_run,
  solver.c:9803), which the reference's embedding does not follow row by row

Pinned against the reference's own runs on the same seeded inputs (tests/golden/, made by
tests/golden/make_golden.py from oracle/_ref/brisk_ref, the reference compiled by
oracle/Makefile): their iteration tables are followed row by row, from both starts and in both
directions (tests/test_cpu_oracle.py); solve_hsd by outcome (status, objectives, certificates:
tests/test_cpu_oracle_hsd.py); and against the reference's published golden value for theta1
(INSTALL.md:44-45).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
from scipy.linalg import cho_factor, cho_solve


@dataclass
class Scaled:
    """The scaled problem (problem_prepare): dense blocks, one list entry per block."""
    m: int
    C: list                 # scaled C per block (n x n)
    A: list                 # per block: (m, n, n) scaled A_i (zero for constraints not in the block)
    b: np.ndarray           # scaled b
    b0: np.ndarray          # b as given
    d: np.ndarray
    du: np.ndarray
    bs: float
    cs: float
    normb1: float
    normb2: float
    normC1: float
    normC2: float
    C0: list = field(default_factory=list)   # C as given
    A0: list = field(default_factory=list)   # A as given


def scale_problem(data) -> Scaled:
    """problem_prepare (problem.c:1866-1910) on dense blocks."""
    C0, A0 = data.dense_blocks()
    m = data.m
    b0 = np.array(data.c, dtype=np.float64)
    nrm2 = np.zeros(m)
    c2 = c1 = 0.0
    for Ck, Ak in zip(C0, A0):
        nrm2 += np.einsum("tij,tij->t", Ak, Ak)            # sum of squares of the full expansion
        c2 += float(np.sum(Ck * Ck))
        c1 += float(np.sum(np.abs(Ck)))
    normC2, normC1 = np.sqrt(c2), c1
    normb1, normb2 = float(np.sum(np.abs(b0))), float(np.sqrt(np.sum(b0 * b0)))
    d = np.where(nrm2 > 0, 1.0 / np.sqrt(np.where(nrm2 > 0, nrm2, 1.0)), 1.0)
    nb = float(np.sqrt(np.sum((d * b0) ** 2)))
    bs = nb if nb > 1 else 1.0
    A = [Ak * d[:, None, None] for Ak in A0]
    b = b0 * d
    du = bs / d
    cs = normC2 if normC2 > 1 else 1.0
    b = b / bs
    C = [Ck / cs for Ck in C0]
    return Scaled(m, C, A, b, b0, d, du, bs, cs, normb1, normb2, normC1, normC2, C0, A0)


def start_point(S: Scaled):
    """start_sdpt3 (solver.c:6622-6661): per block xi, eta; X0 = xi I, Z0 = eta I, y0 = 0."""
    X, Z, xis, etas = [], [], [], []
    for Ck, Ak in zip(S.C, S.A):
        n = Ck.shape[0]
        nC = float(np.sqrt(np.sum(Ck * Ck)))
        a = np.sqrt(np.einsum("tij,tij->t", Ak, Ak))
        inb = a > 0                                            # constraints touching the block
        maxA = float(a[inb].max()) if inb.any() else 0.0
        ratio = float(((1 + np.abs(S.b[inb])) / (1 + a[inb])).max()) if inb.any() else 0.0
        xi = max(10.0, max(np.sqrt(n), n * ratio))
        eta = max(10.0, max(np.sqrt(n), max(maxA, nC)))
        X.append(xi * np.eye(n))
        Z.append(eta * np.eye(n))
        xis.append(xi)
        etas.append(eta)
    return X, Z, np.zeros(S.m), xis, etas


def start_least_squares(S: Scaled, lp=None):
    """The least-squares start (init 1, the default, solver.c:13939-14198), with exact solves and
    exact eigenvalues: dy = (A A')^-1 b and y = (A A')^-1 A(C) (A A' the Schur complement at
    X = Zi = I); with ax, az the largest -lambda_min over the blocks of X0 = A'dy and Z0 = C - A'y,
    X0 is shifted by 1 + ax when ax >= -1e-8 (else kept) and Z0 by max(0, 1 + az)
    (solver.c:14099-14104); then each block's X0, Z0 is raised by 1e-8, 1e-7, ... on the diagonal
    until a Cholesky factor exists (solver.c:14190-14199).  None when A A' has no Cholesky factor (the
    reference then takes the SDPT3 start).  The reference solves by CG to 1e-10 first (its direct
    solve when that misses 1e-3) and takes lmin by Lanczos for blocks above order 32: the same
    start to that accuracy, exactly the same shifts where every block has order <= 32."""
    eye = [np.eye(Ck.shape[0]) for Ck in S.C]
    G = schur(S.A, eye, eye)
    try:
        np.linalg.cholesky(G)
    except np.linalg.LinAlgError:
        return None
    dy = np.linalg.solve(G, S.b)
    y = np.linalg.solve(G, aop(S.A, S.C))
    X = atop(S.A, dy)
    Z = [Ck - a for Ck, a in zip(S.C, atop(S.A, y))]
    lp = lp if lp is not None else [False] * len(X)
    ax = max(-block_lam_min(None, Xk, f) for Xk, f in zip(X, lp))
    az = max(-block_lam_min(None, Zk, f) for Zk, f in zip(Z, lp))
    shx = 1.0 + ax if ax >= -1e-8 else 0.0
    shz = max(0.0, 1.0 + az)
    X = [Xk + shx * I for Xk, I in zip(X, eye)]
    Z = [Zk + shz * I for Zk, I in zip(Z, eye)]
    for V in (X, Z):
        for k, I in enumerate(eye):
            extra = 1e-8
            while True:
                try:
                    np.linalg.cholesky(V[k])
                    break
                except np.linalg.LinAlgError:
                    V[k] = V[k] + extra * I
                    extra *= 10
    return X, Z, y


def schur(A_blocks, X_blocks, Zi_blocks):
    """M_ij = sum_blocks <A_i, X A_j Zi> (the HKM Schur complement, dense formula)."""
    m = A_blocks[0].shape[0]
    M = np.zeros((m, m))
    for Ak, Xk, Zik in zip(A_blocks, X_blocks, Zi_blocks):
        # the constraints that touch the block (the others add exact zeros)
        idx = np.flatnonzero(np.any(Ak.reshape(m, -1) != 0, axis=1))
        if idx.size == 0:
            continue
        Ai = Ak[idx]
        G = Xk[None] @ Ai @ Zik[None]                       # G_j = X A_j Zi (batched products)
        M[np.ix_(idx, idx)] += Ai.reshape(idx.size, -1) @ G.reshape(idx.size, -1).T
    return M


def aop(A_blocks, D_blocks):
    return sum(np.einsum("tij,ij->t", Ak, Dk) for Ak, Dk in zip(A_blocks, D_blocks))


def atop(A_blocks, y):
    return [np.einsum("t,tij->ij", y, Ak) for Ak in A_blocks]


SMALL_BLOCK = 32     # solver.c:5944: exact eigenvalues up to this order
SMALL_N_MAX = 64     # the CUDA path's small-block kernel (exact eigenvalues) up to this order
LANCZOS_K = 30       # solver.c:81, and the default -lanczos (solver.c:122)
LZ_TOL = 0.02        # solver.c:6041: the relative Ritz accuracy that ends the Lanczos steps


def lam_min(L, D):
    """lambda_min(L^-1 D L^-T) (exact)."""
    Li = np.linalg.inv(L)
    B = Li @ D @ Li.T
    return float(np.linalg.eigvalsh(0.5 * (B + B.T))[0])


def _ritz_bound(alpha, beta, kk):
    """ritz_bound (solver.c:6030-6039): theta, the smallest eigenvalue of the tridiagonal
    T_kk, and |beta_kk z_kk| for its unit eigenvector z."""
    T = np.diag(alpha[:kk]) + np.diag(beta[:kk - 1], 1) + np.diag(beta[:kk - 1], -1)
    w, V = np.linalg.eigh(T)
    return abs(beta[kk - 1] * V[kk - 1, 0]), float(w[0])


def lam_min_lanczos(L, D, kmax=LANCZOS_K):
    """sdp_maxstep_lam for blocks above SMALL_BLOCK (solver.c:6083-6225), cold start: Lanczos on
    L^-1 D L^-T (on D when L is None; D read by its lower triangle, as dsymv) from the fixed
    vector q_i = 1 + 0.5 sin(1.7 i + 0.3), normalised; each new vector orthogonalised twice against
    all earlier ones; stopped when beta <= 1e-12 max|alpha|, or from the sixth step every third
    step when the Ritz bound res <= 0.02 |theta| + 1e-14 max|alpha|.  Returns theta - res, the
    reference's conservative estimate of lambda_min."""
    from scipy.linalg import solve_triangular
    n = D.shape[0]
    K = min(n, kmax, LANCZOS_K)
    Dl = np.tril(D) + np.tril(D, -1).T
    i = np.arange(n)
    q = 1.0 + 0.5 * np.sin(1.7 * i + 0.3)
    Q = [q / np.linalg.norm(q)]
    alpha, beta = [], []
    scale, kk = 0.0, 0
    for j in range(K):
        v = Q[j] if L is None else solve_triangular(L, Q[j], trans="T", lower=True)
        w = Dl @ v
        if L is not None:
            w = solve_triangular(L, w, lower=True)
        a = float(Q[j] @ w)
        alpha.append(a)
        for _ in range(2):
            for qi in Q[:j + 1]:
                w = w - float(qi @ w) * qi
        b = float(np.linalg.norm(w))
        beta.append(b)
        kk = j + 1
        scale = max(scale, abs(a))
        if b <= 1e-12 * (scale + 1e-300):
            beta[j] = 0.0
            break
        if kk >= 6 and kk % 3 == 0:
            res, theta = _ritz_bound(alpha, beta, kk)
            if res <= LZ_TOL * abs(theta) + 1e-14 * scale:
                break
        if j + 1 < K:
            Q.append(w / b)
    res, theta = _ritz_bound(alpha, beta, kk)
    return theta - res


def block_lam_min(L, D, lp=False, exact_n=SMALL_BLOCK):
    """The reference's lambda_min of L^-1 D L^-T for one block: exact up to order SMALL_BLOCK
    (small_lammin) and for an LP block (the ratio test of lp_maxstep, solver.c:6227-6235, on its
    diagonal), the Lanczos estimate above (sdp_maxstep_lam).  L None: of D itself.  exact_n:
    the largest order with exact eigenvalues (the CUDA path's small-block kernel takes 64)."""
    n = D.shape[0]
    if n <= exact_n or lp:
        if L is None:
            return float(np.linalg.eigvalsh(0.5 * (D + D.T))[0])
        return lam_min(L, D)
    return lam_min_lanczos(L, D)


def maxstep(Ls, dVs, lp=None, exact_n=SMALL_BLOCK):
    """maxstep (solver.c:6300-6390): 1e30 when unbounded.  lp[k]: block k is an LP block."""
    a = 1e30
    for k, (L, dV) in enumerate(zip(Ls, dVs)):
        lam = block_lam_min(L, dV, bool(lp[k]) if lp is not None else False, exact_n)
        ak = 1e30 if lam >= 0 else -1.0 / lam
        a = min(a, ak)
    return a


def nt_scaling(LX, LZ):
    """nt_scaling (solver.c:7824-7912) on dense factors: Mb = L_Z' L_X, the eigenvectors V of
    H = Mb' Mb with lam = sqrt of its eigenvalues in descending order (dsyevd's ascending order
    reversed, solver.c:7853-7858), G = L_X V diag(lam)^-1/2 and W = G G' (solver.c:7886-7893).
    Returns (G, lam, W), or None where an eigenvalue is not positive (the reference then tries
    dgesdd; the oracle does not)."""
    LX, LZ = np.tril(LX), np.tril(LZ)
    Mb = LZ.T @ LX
    w, Q = np.linalg.eigh(Mb.T @ Mb)
    if not w[0] > 0:
        return None
    lam = np.sqrt(w[::-1])
    V = Q[:, ::-1]
    G = (LX @ V) / np.sqrt(lam)[None, :]
    return G, lam, G @ G.T


def try_step(Vs, dVs, alpha):
    """try_step (solver.c:6393-6447): alpha *= 0.8 until every V + alpha dV is Cholesky-definite."""
    a = alpha
    for _ in range(40):
        new = [V + a * dV for V, dV in zip(Vs, dVs)]
        try:
            Ls = [np.linalg.cholesky(V) for V in new]
            return True, a, new, Ls
        except np.linalg.LinAlgError:
            a *= 0.8
    return False, a, Vs, None


def dimacs(S: Scaled, Xs, y):
    """DIMACS errors 1..6 of (X, y) on the data as given, with Z = C - A'y
    (postsolve.c:2880-2897); X, y in the scaled problem's units."""
    Xo = [S.bs * X for X in Xs]
    yo = S.cs * S.d * y
    Zo = [Ck - Ak_y for Ck, Ak_y in zip(S.C0, atop(S.A0, yo))]
    pobj = sum(float(np.sum(Ck * Xk)) for Ck, Xk in zip(S.C0, Xo))
    dobj = float(S.b0 @ yo)
    r = aop(S.A0, Xo) - S.b0
    xz = sum(float(np.sum(Xk * Zk)) for Xk, Zk in zip(Xo, Zo))
    lamx = min(float(np.linalg.eigvalsh(Xk)[0]) for Xk in Xo)
    lamz = min(float(np.linalg.eigvalsh(Zk)[0]) for Zk in Zo)
    den = 1 + abs(pobj) + abs(dobj)
    err = np.array([np.linalg.norm(r) / (1 + S.normb1), max(0.0, -lamx) / (1 + S.normb1), 0.0,
                    max(0.0, -lamz) / (1 + S.normC1), (pobj - dobj) / den, xz / den])
    return err, pobj, dobj, Xo, yo, Zo


STATUS = {0: "OPTIMAL", 1: "PRIMAL INFEASIBLE", 2: "DUAL INFEASIBLE", 3: "ITERATION LIMIT",
          4: "NUMERICAL DIFFICULTIES", 5: "REDUCED ACCURACY", 6: "TIME LIMIT"}


def solve(data, tol=1e-8, maxit=100, gamma_max=0.99, red_acc=None, log=None, direction="hkm", init=0):
    """The infeasible-start predictor-corrector loop (solver.c:14394-15188), FP64, dense, with the
    HKM direction or (direction="nt") the NT direction in the scaled space: the scaling W = G G'
    from nt_scaling each iteration (solver.c:14403-14410), the Schur complement at X = Zi = W
    (nt_view), h = A(W theta R0 W), the predictor dXt = -lam - G' dZ G (solver.c:14740-14792), the
    corrector Rt = L_lam^-1(smu I - lam^2 - sym(dXt dZt)), rhs = b + h - A(G (Rt + lam) G'),
    dX = G (Rt - G' dZ G) G' (solver.c:14876-14996) and the refinement with W A'w W.

    Returns a dict with status, iterations, pobj, dobj, dimacs (errors 1..6), the iteration-0
    measures (it0: pobj, dobj, pinf, dinf, gap, mu in the reference's -v table convention) and
    the first Schur complement M0 (scaled problem)."""
    if red_acc is None:
        red_acc = max(1e-6, 100 * tol)
    lp = [int(b) < 0 for b in data.bs]          # LP blocks (negative sizes)
    lp_only = all(lp)
    S = scale_problem(data)
    Xs, Zs, y, xis, etas = start_point(S)
    if init >= 1 and S.m > 0:   # the least-squares start (the reference's default)
        ls = start_least_squares(S, lp)
        if ls is not None:
            Xs, Zs, y = ls
    LX = [np.linalg.cholesky(X) for X in Xs]
    LZ = [np.linalg.cholesky(Z) for Z in Zs]
    m = S.m
    Ntot = sum(X.shape[0] for X in Xs)
    R0 = [Ck - Zk - Ak for Ck, Zk, Ak in zip(S.C, Zs, atop(S.A, y))]
    theta = 1.0
    r0norm = float(np.sqrt(sum(np.sum(R * R) for R in R0)))
    nbs = float(np.linalg.norm(S.b))
    best_score, it_best, best, ybest, XZbest = np.inf, 0, None, y.copy(), None
    status, stall, alp, ald, sigma = -1, 0, 0.0, 0.0, 0.0
    out = {"M0": None, "it0": None, "table": []}
    it = 0
    nt = direction == "nt"
    sym = lambda A: 0.5 * (A + A.T)   # noqa: E731
    for it in range(maxit + 1):
        if nt:
            scal = [nt_scaling(Lx, Lz) for Lx, Lz in zip(LX, LZ)]
            if any(sc_ is None for sc_ in scal):
                status = 4
                break
            Gn = [sc_[0] for sc_ in scal]
            lamn = [sc_[1] for sc_ in scal]
            Zi = [sym(sc_[2]) for sc_ in scal]
        else:
            Zi = [np.linalg.inv(L).T @ np.linalg.inv(L) for L in LZ]
            Zi = [0.5 * (Q + Q.T) for Q in Zi]
        Xv = Zi if nt else None   # the X the products read: W under NT
        rp = S.b - aop(S.A, Xs)
        ATy = atop(S.A, y)
        Fs = [a + Zk for a, Zk in zip(ATy, Zs)]
        nCR2 = sum(float(np.sum(F * F)) for F in Fs)
        Fd = [F - Ck for F, Ck in zip(Fs, S.C)]
        pobj = sum(float(np.sum(Ck * Xk)) for Ck, Xk in zip(S.C, Xs))
        xz = sum(float(np.sum(Xk * Zk)) for Xk, Zk in zip(Xs, Zs))
        rdn2 = sum(float(np.sum(F * F)) for F in Fd)
        dev2 = sum(float(np.sum((F + theta * R) ** 2)) for F, R in zip(Fd, R0))
        dobj = float(S.b @ y)
        mu = xz / Ntot
        rpo = float(np.linalg.norm(rp * S.du))
        rdo = S.cs * np.sqrt(rdn2)
        sc = S.bs * S.cs
        po, dob = sc * pobj, sc * dobj
        pinf = rpo / (1 + S.normb2)
        dinf = rdo / (1 + S.normC2)
        oden = 1 + abs(po) + abs(dob)
        relgap = abs(po - dob) / oden
        relcomp = sc * xz / oden
        row = dict(it=it, pobj=-po, dobj=-dob, pinf=pinf, dinf=dinf, gap=relgap, mu=sc * mu)
        out["table"].append(row)
        if it == 0:
            out["it0"] = row
        if log:
            log(f"{it:3d} {-po:+.8e} {-dob:+.8e} {pinf:.2e} {dinf:.2e} {relgap:.2e} {sc * mu:.2e} "
                f"{alp:.3f} {ald:.3f} {sigma:.3f}")
        score = max(relgap, relcomp, pinf, dinf)
        err_it = (rpo / (1 + S.normb1), rdo / (1 + S.normC1), (po - dob) / oden, sc * xz / oden)
        if score < best_score:
            best_score, it_best, ybest = score, it, y.copy()
            best = err_it
            XZbest = ([X.copy() for X in Xs], [Z.copy() for Z in Zs])
        if score < tol:
            status = 0
            break
        if it > it_best and max(abs(e) for e in best) <= 0.5 * tol:
            status = 4
            break
        if dobj > 0 and np.sqrt(nCR2) / dobj < 1e-8 and it > 5:
            status = 1
            break
        nAX = float(np.linalg.norm(S.b - rp))
        if pobj < 0 and nAX / (-pobj) < 1e-8 and it > 5:
            status = 2
            break
        if it == maxit:
            status = 3
            break
        if stall >= 3 or (it - it_best >= 5 and best_score < 1e-6) or (it - it_best >= 8 and best_score < 1e-4) \
                or it - it_best >= 12:
            status = 4
            break
        dev = np.sqrt(dev2)
        if dev > 1e-10 * (1.0 + theta * r0norm) and dev > 1e-12:
            theta, r0norm = 1.0, float(np.sqrt(rdn2))
            R0 = [-F for F in Fd]
        if theta * r0norm <= 1e-13:
            theta = 0.0
        Xp = Xv if nt else Xs
        M = schur(S.A, Xp, Zi)
        if out["M0"] is None:
            out["M0"] = M.copy()
        # M's Cholesky factor and triangular solves (schur_factor / schur_solve, solver.c:14671,
        # 14796): an explicit inverse leaves A(dX) - rp at eps cond(M) |rp|, which held the late
        # rows' primal residual near 1e-10 where the reference's reaches 1e-13
        try:
            Mc = cho_factor(M, lower=True)
            msolve = lambda v: cho_solve(Mc, v)   # noqa: E731
        except np.linalg.LinAlgError:   # numerically indefinite: partial-pivoting LU
            msolve = lambda v: np.linalg.solve(M, v)   # noqa: E731
        a0 = aop(S.A, Zi)
        h = aop(S.A, [theta * Zk @ R @ Xk for Zk, R, Xk in zip(Zi, R0, Xp)]) if theta > 0 else np.zeros(m)
        dy = msolve(S.b + h)
        dZ = [-a + theta * R for a, R in zip(atop(S.A, dy), R0)]
        dX = []
        if nt:
            dXt, dZt = [], []
            for Gk, lk, dZk in zip(Gn, lamn, dZ):
                zt = sym(Gk.T @ dZk @ Gk)
                xt = -np.diag(lk) - zt
                dZt.append(zt)
                dXt.append(xt)
                dX.append(sym(Gk @ xt @ Gk.T))
        else:
            for Zk, dZk, Xk in zip(Zi, dZ, Xs):
                G = Zk @ dZk @ Xk
                dX.append(-0.5 * (G + G.T) - Xk)
        ap = min(1.0, maxstep(LX, dX, lp))
        ad = min(1.0, maxstep(LZ, dZ, lp))
        xdz = sum(float(np.sum(a * b)) for a, b in zip(Xs, dZ))
        dxz = sum(float(np.sum(a * b)) for a, b in zip(dX, Zs))
        dxdz = sum(float(np.sum(a * b)) for a, b in zip(dX, dZ))
        mu_a = (xz + ap * dxz + ad * xdz + ap * ad * dxdz) / Ntot
        frac = max(0.0, mu_a / mu)
        mina = min(ap, ad)
        # the default sigma rule (solver.c:14848-14855): cubic when the problem has no SDP block
        # (only LP blocks), else adaptive
        if lp_only:
            expon = 3.0
        else:
            expon = max(1.0, 3 * mina * mina) if relgap > 1e-6 else 3.0
        sigma = min(1.0, frac ** expon)
        gamma = 0.9 + (gamma_max - 0.9) * mina
        smu = sigma * mu
        if nt:
            Rt = []
            for lk, xt, zt in zip(lamn, dXt, dZt):
                H = sym(xt @ zt)
                L2 = lk[:, None] + lk[None, :]
                R_ = -2.0 * H / L2
                R_[np.diag_indices_from(R_)] += smu / lk - lk
                Rt.append(R_)
            Gt = [sym(Gk @ (R_ + np.diag(lk)) @ Gk.T) for Gk, R_, lk in zip(Gn, Rt, lamn)]
            rhs = S.b + h - aop(S.A, Gt)
        else:
            Q = [Zk @ dZk @ dXk for Zk, dZk, dXk in zip(Zi, dZ, dX)]
            rhs = S.b - smu * a0 + aop(S.A, Q) + h
        dy = msolve(rhs)
        dZ = [-a + theta * R for a, R in zip(atop(S.A, dy), R0)]
        dX = []
        if nt:
            for Gk, R_, dZk in zip(Gn, Rt, dZ):
                dX.append(sym(Gk @ (R_ - sym(Gk.T @ dZk @ Gk)) @ Gk.T))
        else:
            for Zk, dZk, Xk, Qk in zip(Zi, dZ, Xs, Q):
                G = Zk @ dZk @ Xk + Qk
                dX.append(-0.5 * (G + G.T) + smu * Zk - Xk)
        for _ in range(3):
            ev = rp - aop(S.A, dX)
            ne, nrp = np.linalg.norm(ev), np.linalg.norm(rp)
            if not (ne > 1e-2 * nrp and ne > 1e-3 * tol * (1 + nbs)):
                break
            wv = msolve(ev)
            Qd = atop(S.A, wv)
            Gs = []
            for Zk, Qk, Xk in zip(Zi, Qd, Xp):
                G = Zk @ Qk @ Xk
                Gs.append(0.5 * (G + G.T))
            ne2 = np.linalg.norm(ev - aop(S.A, Gs))
            if not (ne2 < 0.5 * ne):
                break
            dy = dy + wv
            dZ = [a - b for a, b in zip(dZ, Qd)]
            dX = [a + b for a, b in zip(dX, Gs)]
        apr = min(1.0, maxstep(LX, dX, lp))
        adr = min(1.0, maxstep(LZ, dZ, lp))
        apn, adn = min(1.0, gamma * apr), min(1.0, gamma * adr)
        if pinf < 1e-6:
            ev = rp - aop(S.A, dX)
            nrp, nev = np.linalg.norm(rp), np.linalg.norm(ev)
            lim = max(1e3, 1e-6 / max(pinf, 1e-300)) * nrp
            if nev > lim and nrp > 0:
                apn = min(apn, lim / nev)
        okp, apn, Xs, LXn = try_step(Xs, dX, apn)
        okd, adn, Zs, LZn = try_step(Zs, dZ, adn)
        if not okp or not okd:
            status = 4
            break
        LX, LZ = LXn, LZn
        y = y + adn * dy
        theta *= (1.0 - adn)
        alp, ald = apn, adn
        stall = stall + 1 if (apn < 1e-6 and adn < 1e-6) else 0
    if status not in (0, 1, 2) and XZbest is not None and best_score < score:
        y = ybest
        Xs, Zs = XZbest
    err, pobj_o, dobj_o, Xo, yo, Zo = dimacs(S, Xs, y)
    acc = max(err[0], err[1], err[3], abs(err[4]), abs(err[5]))
    if status in (0, 3, 4, 5, 6):
        if acc <= tol:
            status = 0
        elif acc <= red_acc:
            status = 5
        elif status in (0, 5):
            status = 4
    out.update(status=status, status_str=STATUS.get(status, "?"), iterations=it, pobj=pobj_o, dobj=dobj_o,
               dimacs=err, X=Xo, y=yo, Z=Zo, xi=xis, eta=etas, scaled=S)
    return out


def solve_hsd(data, tol=1e-8, maxit=100, gamma_max=0.99, red_acc=None, log=None, exact_n=SMALL_N_MAX, check=False):
    """The homogeneous self-dual embedding as the CUDA path runs it (Solver::run_hsd, which stands
    for the reference's hsd_run, solver.c:9803, as a method of its own: HKM direction, one
    Mehrotra predictor-corrector step an iteration, no extra correctors or end phases), FP64,
    dense.  With tau, kappa >= 0 the scaled problem is embedded as
        A(X) - b tau = 0,   A'y + Z - C tau = 0,   b'y - <C,X> - kappa = 0,
    X Z = mu I, tau kappa = mu, mu = (<X,Z> + tau kappa) / (N + 1), from X = Z = I, y = 0,
    tau = kappa = 1 on the equilibrated problem.  The Newton system reduces to the infeasible
    method's Schur complement M: dy = u + (v1 + w) dtau with M v1 = A(Zi C X), M w = b and M u
    = eta rp - sigma mu A(Zi) + A(X) + eta A(Zi Rd X) + A(Q); dtau from the third equation in
    its cancellation-free form, den = b'w + <R, Zi R X> + kappa / tau with R = C - A'v1.  One
    step length for every variable (Z's Cholesky test first, then X's, Z moved back when X's is
    shorter); the step lengths take exact eigenvalues up to order exact_n (the CUDA path's
    small-block kernel: 64) and the Lanczos estimate above.  kappa > 1e8 tau ends the solve with a certificate: b'y > 0 primal infeasible,
    <C,X> < 0 dual infeasible.  The solution is X / tau, y / tau.

    The reference's own embedding takes 4-7 iterations on the parity instances where this one
    takes 8-12 (its extra correctors), so the two agree in status and objectives, not row by
    row.  Returns the dict of solve() (status, iterations, pobj, dobj, dimacs, the table with
    tau and kappa per row); with check, also "newton": per direction the relative residuals of
    the four linearised equations A(dX) - b dtau = eta rp, A'dy + dZ - C dtau = eta Rd,
    b'dy - <C,dX> - dkappa = eta rg and kappa dtau + tau dkappa = sigma mu - tau kappa - dtau_p
    dkappa_p (each over the sum of its terms' norms)."""
    if red_acc is None:
        red_acc = max(1e-6, 100 * tol)
    lp = [int(b) < 0 for b in data.bs]
    S = scale_problem(data)
    m = S.m
    C, A, b = S.C, S.A, S.b
    Xs = [np.eye(Ck.shape[0]) for Ck in C]
    Zs = [np.eye(Ck.shape[0]) for Ck in C]
    LX = [np.eye(Ck.shape[0]) for Ck in C]
    LZ = [np.eye(Ck.shape[0]) for Ck in C]
    y = np.zeros(m)
    N = sum(Ck.shape[0] for Ck in C)
    tau = 1.0
    kap = sum(float(np.sum(X * Z)) for X, Z in zip(Xs, Zs)) / N

    def ip(P_, Q_):
        return sum(float(np.sum(p * q)) for p, q in zip(P_, Q_))

    def prod(P_, Q_, R_):
        return [p @ q @ r for p, q, r in zip(P_, Q_, R_)]

    def ratio(x, dx):
        return -x / dx if dx < 0 else 1e30

    status, stall, it, it_best = -1, 0, 0, 0
    best_score, best, saved = np.inf, None, None
    sigma = alpha = 0.0
    out = {"table": [], "newton": []}
    for it in range(maxit + 1):
        Zi = [np.linalg.inv(L).T @ np.linalg.inv(L) for L in LZ]
        Zi = [0.5 * (Q + Q.T) for Q in Zi]
        AX = aop(A, Xs)
        rp = b * tau - AX
        Rd = [Ck * tau - a - Zk for Ck, a, Zk in zip(C, atop(A, y), Zs)]
        cx, xz, rd2 = ip(C, Xs), ip(Xs, Zs), ip(Rd, Rd)
        by = float(b @ y)
        rg = kap - by + cx
        mu = (xz + tau * kap) / (N + 1)
        sc = S.bs * S.cs
        rpo = float(np.linalg.norm(rp * S.du)) / tau
        rdo = S.cs * np.sqrt(rd2) / tau
        po, dob = sc * cx / tau, sc * by / tau
        pinf, dinf = rpo / (1 + S.normb2), rdo / (1 + S.normC2)
        oden = 1 + abs(po) + abs(dob)
        relgap = abs(po - dob) / oden
        relcomp = sc * xz / (tau * tau) / oden
        row = dict(it=it, pobj=-po, dobj=-dob, pinf=pinf, dinf=dinf, gap=relgap, mu=sc * xz / (tau * tau * N),
                   tau=tau, kappa=kap)
        out["table"].append(row)
        if log:
            log(f"{it:3d} {-po:+.8e} {-dob:+.8e} {pinf:.2e} {dinf:.2e} {relgap:.2e} {row['mu']:.2e} "
                f"{alpha:.3f} {sigma:.3f} tau {tau:.3e} kappa {kap:.3e}")
        if not (np.isfinite(po) and np.isfinite(dob) and tau > 0 and kap > 0):
            status = 4
            break
        score = max(relgap, relcomp, pinf, dinf)
        err_it = (rpo / (1 + S.normb1), rdo / (1 + S.normC1), (po - dob) / oden, relcomp)
        if score < best_score:
            best_score, it_best, best = score, it, err_it
            saved = ([X.copy() for X in Xs], [Z.copy() for Z in Zs], y.copy(), tau)
        if score < tol:
            status = 0
            break
        if it > it_best and max(abs(e) for e in best) <= 0.5 * tol:
            status = 4
            break
        if kap > 1e8 * tau:
            status = 1 if by > 0 else (2 if cx < 0 else 4)
            break
        if it == maxit:
            status = 3
            break
        if stall >= 3 or (it - it_best >= 5 and best_score < 1e-6) or it - it_best >= 12:
            status = 4
            break
        M = schur(A, Xs, Zi)
        try:
            Mc = cho_factor(M, lower=True)
        except np.linalg.LinAlgError:
            status = 4
            break
        msolve = lambda v: cho_solve(Mc, v)   # noqa: E731
        a0 = aop(A, Zi)
        pv = aop(A, prod(Zi, C, Xs))
        hv = aop(A, prod(Zi, Rd, Xs))
        v1 = msolve(pv)
        w = msolve(b)
        Rm = [Ck - a for Ck, a in zip(C, atop(A, v1))]            # R = C - A'v1
        G = prod(Zi, Rm, Xs)
        rwr, rzi, rx, rw = ip(Rm, G), ip(Rm, Zi), ip(Rm, Xs), ip(Rd, G)
        den = float(b @ w) + rwr + kap / tau
        if not (den > 0 and np.isfinite(den)):
            status = 4
            break
        v1rp = float(v1 @ rp)
        v = v1 + w

        def direction(smu, eta, Q, qv, rq, dtdk):
            rhs = eta * rp - smu * a0 + AX + eta * hv + (qv if Q is not None else 0.0)
            u = msolve(rhs)
            num = eta * rg + (smu - tau * kap - dtdk) / tau - float(b @ u) + eta * v1rp + smu * rzi - rx \
                - eta * rw - rq
            dt = num / den
            dy = u + v * dt
            dZ = [Ck * dt - a + eta * R for Ck, a, R in zip(C, atop(A, dy), Rd)]
            Gd = prod(Zi, dZ, Xs)
            if Q is not None:
                Gd = [g + q for g, q in zip(Gd, Q)]
            dX = [-0.5 * (g + g.T) + smu * zi - x for g, zi, x in zip(Gd, Zi, Xs)]
            dk = (smu - tau * kap - dtdk - kap * dt) / tau
            if check:
                nrm = lambda V: float(np.sqrt(ip(V, V)))   # noqa: E731
                ad, aty, bd = aop(A, dX), atop(A, dy), b * dt
                e1 = float(np.linalg.norm(ad - bd - eta * rp)) / (
                    np.linalg.norm(ad) + np.linalg.norm(bd) + eta * np.linalg.norm(rp))
                e2 = nrm([a + z - Ck * dt - eta * R for a, z, Ck, R in zip(aty, dZ, C, Rd)]) / (
                    nrm(aty) + nrm(dZ) + abs(dt) * nrm(C) + eta * nrm(Rd))
                t3 = (float(b @ dy), ip(C, dX), dk, eta * rg)
                e3 = abs(t3[0] - t3[1] - t3[2] - t3[3]) / sum(abs(t) for t in t3)
                t4 = (kap * dt, tau * dk, smu - tau * kap - dtdk)
                e4 = abs(t4[0] + t4[1] - t4[2]) / max(sum(abs(t) for t in t4), 1e-300)
                out["newton"].append((it, e1, e2, e3, e4))
            return dX, dy, dZ, dt, dk

        dXp, _, dZp, dtp, dkp = direction(0.0, 1.0, None, None, 0.0, 0.0)
        ap = min(1.0, maxstep(LX, dXp, lp, exact_n), maxstep(LZ, dZp, lp, exact_n), ratio(tau, dtp), ratio(kap, dkp))
        xdz, dxz, dxdz = ip(Xs, dZp), ip(dXp, Zs), ip(dXp, dZp)
        mu_a = (xz + ap * (xdz + dxz) + ap * ap * dxdz + (tau + ap * dtp) * (kap + ap * dkp)) / (N + 1)
        expon = max(1.0, 3.0 * ap * ap) if relgap > 1e-6 else 3.0
        sigma = min(1.0, max(0.0, mu_a / mu) ** expon)
        Q = prod(Zi, dZp, dXp)
        dX, dy, dZ, dt, dk = direction(sigma * mu, 1.0 - sigma, Q, aop(A, Q), ip(Rm, Q), dtp * dkp)
        amax = min(maxstep(LX, dX, lp, exact_n), maxstep(LZ, dZ, lp, exact_n), ratio(tau, dt), ratio(kap, dk))
        gamma = 0.9 + (gamma_max - 0.9) * min(1.0, amax)
        a = min(1.0, gamma * amax)
        okz, a, Zn, LZn = try_step(Zs, dZ, a)
        a_z = a
        okx = False
        if okz:
            okx, a, Xn, LXn = try_step(Xs, dX, a)
            if okx and a < a_z:
                a_x = a
                okz, a, Zn, LZn = try_step(Zs, dZ, a)
                if okz and a < a_x:
                    okx, a, Xn, LXn = try_step(Xs, dX, a)
        if not (okz and okx):
            status = 4
            break
        Xs, Zs, LX, LZ = Xn, Zn, LXn, LZn
        y = y + a * dy
        tau += a * dt
        kap += a * dk
        alpha = a
        stall = stall + 1 if a < 1e-6 else 0
    if status not in (0, 1, 2) and saved is not None and best_score < score:
        Xs, Zs, y, tau = saved
    err, pobj_o, dobj_o, Xo, yo, Zo = dimacs(S, [X / tau for X in Xs], y / tau)
    acc = max(err[0], err[1], err[3], abs(err[4]), abs(err[5]))
    if status in (0, 3, 4, 5, 6):
        if acc <= tol:
            status = 0
        elif acc <= red_acc:
            status = 5
        elif status in (0, 5):
            status = 4
    out.update(status=status, status_str=STATUS.get(status, "?"), iterations=it, pobj=pobj_o, dobj=dobj_o,
               dimacs=err, X=Xo, y=yo, Z=Zo, scaled=S, tau=tau, kappa=kap)
    return out
