"""Seeded synthetic SDP instances in the numbers of an SDPA sparse file.

A problem is what BRISK's C interface takes (``brisk_solve_data``, capi.c:175): block sizes
``bs`` (LP blocks negative), the right-hand side ``c`` (m entries) and the entries
``(mat, blk, i, j, v)``, 1-based as in the file, ``mat`` 0 being F0 = -C and 1..m the A_i
(brisk.h:128-140).  BRISK solves (P) min <C,X> s.t. <A_i,X> = b_i, X >= 0 with C = -F0,
A_i = F_i, b = c.

The generators follow the workload descriptions the solver is measured on:

* ``theta_problem``     Lovasz theta of a seeded G(n, p): one n x n block, C = -J,
                        tr(X) = 1 and X_ij = 0 per edge (the SDPA form of the reference's
                        tools/timelimit_test.sh:16-27, with n = 50, p = 0.5).
* ``random_sdp``        one n x n block, m constraints, each A_i symmetric with
                        round(density * n(n+1)/2) upper entries at uniform distinct positions
                        and N(0,1) values, b_i = <A_i, I> (X0 = I is feasible),
                        C = G G'/n + I with G ~ N(0,1) (n=400, m=2000, 1 %; n=1000, m=8000,
                        0.5 %).
* ``random_dense_batch`` independent small instances: n ~ U{8..64},
                        m ~ U{n..floor(n(n+1)/4)}, dense N(0,1) symmetric A_i, b = A(I),
                        C = G G'/n + I.

All randomness comes from ``numpy.random.default_rng(seed)`` (or Python's ``random`` for the
graph, as the reference's generator does), so the same seed gives the same bits everywhere.
"""
from __future__ import annotations

import random as _pyrandom
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np


@dataclass
class SdpaData:
    """An SDP in SDPA sparse numbers (1-based entries; mat 0 is F0 = -C)."""
    bs: np.ndarray          # int32 block sizes
    c: np.ndarray           # float64, m
    mat: np.ndarray         # int32
    blk: np.ndarray         # int32
    i: np.ndarray           # int32 (1-based, i <= j after normalisation)
    j: np.ndarray           # int32
    v: np.ndarray           # float64
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def m(self) -> int:
        return int(self.c.size)

    @property
    def nblk(self) -> int:
        return int(self.bs.size)

    @property
    def nnz(self) -> int:
        return int(self.v.size)

    def args(self):
        """The positional arguments of ``solve_sdpa`` (blocksizes, c, mat, blk, i, j, v)."""
        return (self.bs, self.c, self.mat, self.blk, self.i, self.j, self.v)

    # ---- dense views (small problems only: tests and the oracle) ----
    def dense_blocks(self):
        """C and A_1..A_m as dense symmetric matrices, one list per block:
        returns (C[k], A[k][t]) with A[k] a (m, n, n) array for SDP block k."""
        Cs, As = [], []
        for k, n in enumerate(self.bs):
            n = abs(int(n))
            Ck = np.zeros((n, n))
            Ak = np.zeros((self.m, n, n))
            sel = self.blk == k + 1
            for mt, ii, jj, vv in zip(self.mat[sel], self.i[sel] - 1, self.j[sel] - 1, self.v[sel]):
                if mt == 0:
                    Ck[ii, jj] = -vv
                    Ck[jj, ii] = -vv
                else:
                    Ak[mt - 1, ii, jj] = vv
                    Ak[mt - 1, jj, ii] = vv
            Cs.append(Ck)
            As.append(Ak)
        return Cs, As


def _normalise(mat, blk, i, j, v):
    i = np.asarray(i, dtype=np.int32)
    j = np.asarray(j, dtype=np.int32)
    lo, hi = np.minimum(i, j), np.maximum(i, j)
    return (np.asarray(mat, dtype=np.int32), np.asarray(blk, dtype=np.int32), lo, hi,
            np.asarray(v, dtype=np.float64))


def theta_problem(n: int = 50, p: float = 0.5, seed: int = 1) -> SdpaData:
    """Lovasz theta SDP of a seeded Erdos-Renyi graph G(n, p).

    max <J, X> s.t. tr X = 1, X_ij = 0 for each edge ij, X >= 0; in BRISK form
    C = -J (F0 = J), A_1 = I (b_1 = 1), A_k = E_ij + E_ji (b_k = 0).  The edge list is
    drawn with Python's ``random.Random(seed)`` in the order of the reference's generator.
    """
    rng = _pyrandom.Random(seed)
    E = [(a, b) for a in range(1, n + 1) for b in range(a + 1, n + 1) if rng.random() < p]
    m = 1 + len(E)
    iu, ju = np.triu_indices(n)
    mats = [np.zeros(iu.size, np.int32), np.ones(n, np.int32), np.arange(2, m + 1, dtype=np.int32)]
    ii = [iu + 1, np.arange(1, n + 1), np.array([e[0] for e in E], np.int32)]
    jj = [ju + 1, np.arange(1, n + 1), np.array([e[1] for e in E], np.int32)]
    vv = [np.ones(iu.size), np.ones(n), np.ones(len(E))]
    mat = np.concatenate(mats)
    d = _normalise(mat, np.ones(mat.size, np.int32), np.concatenate(ii), np.concatenate(jj), np.concatenate(vv))
    c = np.zeros(m)
    c[0] = 1.0
    return SdpaData(np.array([n], np.int32), c, *d, name=f"theta_G({n},{p})_seed{seed}",
                    meta=dict(kind="theta", n=n, p=p, seed=seed, edges=len(E)))


def _random_upper_positions(rng, n, k):
    """k distinct uniform positions of the upper triangle (with diagonal) of an n x n matrix."""
    tot = n * (n + 1) // 2
    lin = rng.choice(tot, size=k, replace=False)
    lin.sort()
    # invert the column-major upper packing: column j holds rows 0..j, starting at j(j+1)/2
    jcol = ((np.sqrt(8.0 * lin + 1.0) - 1.0) / 2.0).astype(np.int64)
    jcol -= (jcol * (jcol + 1) // 2 > lin)
    jcol += ((jcol + 1) * (jcol + 2) // 2 <= lin)
    irow = lin - jcol * (jcol + 1) // 2
    return irow, jcol


def random_sdp(n: int = 400, m: int = 2000, density: float = 0.01, seed: int = 0) -> SdpaData:
    """Dense-C random SDP with sparse N(0,1) constraints (one n x n block).

    Each A_i has round(density * n(n+1)/2) upper-triangle entries at distinct uniform
    positions with N(0,1) values; b_i = <A_i, I> so X0 = I is feasible; C = G G'/n + I.
    """
    rng = np.random.default_rng(seed)
    k = int(round(density * n * (n + 1) / 2))
    G = rng.standard_normal((n, n))
    C = G @ G.T / n + np.eye(n)
    mats, ii, jj, vv = [], [], [], []
    iu, ju = np.triu_indices(n)
    mats.append(np.zeros(iu.size, np.int32))
    ii.append(iu + 1)
    jj.append(ju + 1)
    vv.append(-C[iu, ju])
    b = np.zeros(m)
    for t in range(m):
        r, cc = _random_upper_positions(rng, n, k)
        val = rng.standard_normal(k)
        mats.append(np.full(k, t + 1, np.int32))
        ii.append(r + 1)
        jj.append(cc + 1)
        vv.append(val)
        b[t] = val[r == cc].sum()
    mat = np.concatenate(mats)
    d = _normalise(mat, np.ones(mat.size, np.int32), np.concatenate(ii), np.concatenate(jj), np.concatenate(vv))
    return SdpaData(np.array([n], np.int32), b, *d, name=f"random_sdp_n{n}_m{m}_d{density}_seed{seed}",
                    meta=dict(kind="random", n=n, m=m, density=density, seed=seed, upper_per_con=k))


def sdp_lp_problem(blocks=(30, -40, 6), m: int = 50, density: float = 0.1, lp_per_con: int = 4,
                   seed: int = 0, dense_rows: int = 0) -> SdpaData:
    """A random problem with LP blocks (negative sizes) among SDP blocks.

    SDP block of order n: C = G G'/n + I, each A_i with round(density n(n+1)/2) N(0,1) upper
    entries at distinct positions.  LP block of size N: c ~ U(0.5, 1.5), each A_i with
    min(lp_per_con, N) N(0,1) entries on distinct variables; the first dense_rows constraints
    instead hold all N variables (rows that join every variable of the block).  b = A(I, 1, ...),
    so X = I, x = 1 is feasible, and y = 0 gives Z = C > 0, z = c > 0: both sides strictly
    feasible.
    """
    rng = np.random.default_rng(seed)
    mats, blks, ii, jj, vv = [], [], [], [], []
    b = np.zeros(m)
    for kb, sz in enumerate(blocks, start=1):
        if sz > 0:
            n = sz
            G = rng.standard_normal((n, n))
            C = G @ G.T / n + np.eye(n)
            iu, ju = np.triu_indices(n)
            mats.append(np.zeros(iu.size, np.int32)); blks.append(np.full(iu.size, kb, np.int32))
            ii.append(iu + 1); jj.append(ju + 1); vv.append(-C[iu, ju])
            k = max(1, int(round(density * n * (n + 1) / 2)))
            for t in range(m):
                r, cc = _random_upper_positions(rng, n, k)
                val = rng.standard_normal(k)
                mats.append(np.full(k, t + 1, np.int32)); blks.append(np.full(k, kb, np.int32))
                ii.append(r + 1); jj.append(cc + 1); vv.append(val)
                b[t] += val[r == cc].sum()
        else:
            N = -sz
            c = rng.uniform(0.5, 1.5, N)
            idx = np.arange(1, N + 1)
            mats.append(np.zeros(N, np.int32)); blks.append(np.full(N, kb, np.int32))
            ii.append(idx); jj.append(idx); vv.append(-c)
            for t in range(m):
                q = N if t < dense_rows else min(lp_per_con, N)
                var = rng.choice(N, size=q, replace=False) + 1
                val = rng.standard_normal(q)
                mats.append(np.full(q, t + 1, np.int32)); blks.append(np.full(q, kb, np.int32))
                ii.append(var); jj.append(var); vv.append(val)
                b[t] += val.sum()
    d = _normalise(np.concatenate(mats), np.concatenate(blks), np.concatenate(ii), np.concatenate(jj),
                   np.concatenate(vv))
    return SdpaData(np.array(blocks, np.int32), b, *d, name=f"sdp_lp_{'_'.join(map(str, blocks))}_m{m}_seed{seed}",
                    meta=dict(kind="sdp_lp", blocks=list(blocks), m=m, seed=seed, dense_rows=dense_rows))


def lowrank_sdp(n: int = 100, m: int = 300, max_rank: int = 3, support: int = 0, seed: int = 0) -> SdpaData:
    """A random SDP whose constraints have low rank (one n x n block): A_i = sum_k s_k g_k g_k'
    with 1..max_rank terms, s_k = +-1, g_k ~ N(0,1) on `support` random rows (0: all n rows,
    dense data).  b = A(I), C = G G'/n + I: X = I and y = 0 are strictly feasible."""
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((n, n))
    C = G @ G.T / n + np.eye(n)
    iu, ju = np.triu_indices(n)
    mats, ii, jj, vv = [np.zeros(iu.size, np.int32)], [iu + 1], [ju + 1], [-C[iu, ju]]
    b = np.zeros(m)
    for t in range(m):
        r = int(rng.integers(1, max_rank + 1))
        A = np.zeros((n, n))
        for _ in range(r):
            g = np.zeros(n)
            rows = np.arange(n) if support <= 0 else rng.choice(n, size=min(support, n), replace=False)
            g[rows] = rng.standard_normal(rows.size)
            A += (1.0 if rng.random() < 0.7 else -1.0) * np.outer(g, g)
        nzr, nzc = np.nonzero(np.triu(A))
        mats.append(np.full(nzr.size, t + 1, np.int32)); ii.append(nzr + 1); jj.append(nzc + 1); vv.append(A[nzr, nzc])
        b[t] = np.trace(A)
    mat = np.concatenate(mats)
    d = _normalise(mat, np.ones(mat.size, np.int32), np.concatenate(ii), np.concatenate(jj), np.concatenate(vv))
    return SdpaData(np.array([n], np.int32), b, *d, name=f"lowrank_sdp_n{n}_m{m}_r{max_rank}_s{support}_seed{seed}",
                    meta=dict(kind="lowrank", n=n, m=m, max_rank=max_rank, support=support, seed=seed))


def infeasible_sdp(kind: str = "primal", n: int = 6, m: int = 8, seed: int = 0) -> SdpaData:
    """A seeded infeasible SDP (one n x n block).  kind "primal": A_1 = I with b_1 = -1 (no X >= 0
    has a negative trace) and m - 1 random sparse constraints b = A(I); the dual is unbounded.
    kind "dual": C = -E_11 (minimize -X_11) with constraints that leave X_11 free to grow (m
    random constraints on the other rows and columns, b = A(I)); the primal is unbounded, the dual
    infeasible.  C otherwise G G'/n + I."""
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((n, n))
    C = G @ G.T / n + np.eye(n)
    if kind == "dual":
        C = np.zeros((n, n))
        C[0, 0] = -1.0
    iu, ju = np.triu_indices(n)
    keep = C[iu, ju] != 0
    mats, ii, jj, vv = [np.zeros(int(keep.sum()), np.int32)], [iu[keep] + 1], [ju[keep] + 1], [-C[iu, ju][keep]]
    b = np.zeros(m)
    for t in range(m):
        A = np.zeros((n, n))
        if kind == "primal" and t == 0:
            A = np.eye(n)
        else:
            lo = 1 if kind == "dual" else 0
            for _ in range(3):
                p, q = rng.integers(lo, n, size=2)
                v = rng.standard_normal()
                A[p, q] += v
                A[q, p] = A[p, q]
        nzr, nzc = np.nonzero(np.triu(A))
        mats.append(np.full(nzr.size, t + 1, np.int32)); ii.append(nzr + 1); jj.append(nzc + 1); vv.append(A[nzr, nzc])
        b[t] = -1.0 if (kind == "primal" and t == 0) else np.trace(A)
    mat = np.concatenate(mats)
    d = _normalise(mat, np.ones(mat.size, np.int32), np.concatenate(ii), np.concatenate(jj), np.concatenate(vv))
    return SdpaData(np.array([n], np.int32), b, *d, name=f"infeasible_{kind}_n{n}_m{m}_seed{seed}",
                    meta=dict(kind="infeasible", which=kind, n=n, m=m, seed=seed))


def random_dense_instance(rng, n: int, m: int, name: str = "") -> SdpaData:
    """One small dense instance: A_i dense N(0,1) symmetric, b = A(I), C = G G'/n + I."""
    iu, ju = np.triu_indices(n)
    G = rng.standard_normal((n, n))
    C = G @ G.T / n + np.eye(n)
    U = rng.standard_normal((m, iu.size))             # upper entries of each A_i
    b = U[:, iu == ju].sum(axis=1)
    mat = np.concatenate([np.zeros(iu.size, np.int32), np.repeat(np.arange(1, m + 1, dtype=np.int32), iu.size)])
    i = np.concatenate([iu + 1, np.tile(iu + 1, m)])
    j = np.concatenate([ju + 1, np.tile(ju + 1, m)])
    v = np.concatenate([-C[iu, ju], U.ravel()])
    d = _normalise(mat, np.ones(mat.size, np.int32), i, j, v)
    return SdpaData(np.array([n], np.int32), b, *d, name=name, meta=dict(kind="dense", n=n, m=m))


def dense_instance(n: int, m: int, seed: int = 0) -> SdpaData:
    """One seeded small dense instance (random_dense_instance with default_rng(seed))."""
    return random_dense_instance(np.random.default_rng(seed), n, m, name=f"dense_n{n}_m{m}_seed{seed}")


def random_dense_batch(count: int = 4096, nmin: int = 8, nmax: int = 64, seed: int = 0,
                       sizes_only: bool = False):
    """The uneven batch: n ~ U{nmin..nmax}, m ~ U{n..floor(n(n+1)/4)} per instance.

    Returns the list of (n, m) when ``sizes_only``; else the list of SdpaData instances."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(nmin, nmax + 1, size=count)
    ms = np.array([rng.integers(n, n * (n + 1) // 4 + 1) for n in ns])
    if sizes_only:
        return list(zip(ns.tolist(), ms.tolist()))
    out = []
    for q, (n, m) in enumerate(zip(ns, ms)):
        sub = np.random.default_rng([seed, q])
        out.append(random_dense_instance(sub, int(n), int(m), name=f"batch{seed}_{q}"))
    return out


def batch_arrays(count: int = 4096, nmin: int = 8, nmax: int = 64, seed: int = 0, first: int = 0,
                 total: int = 4096):
    """Instances first .. first+count-1 of random_dense_batch(total, ...) (batch_instance(q)) as
    the concatenated arrays of solve_batch_arrays, filled one instance at a time (peak memory:
    the arrays plus one instance)."""
    sizes = random_dense_batch(max(total, first + count), nmin, nmax, seed, sizes_only=True)[first:first + count]
    tri = [n * (n + 1) // 2 for n, _ in sizes]
    nnz = np.array([t * (m + 1) for t, (_, m) in zip(tri, sizes)], np.int64)
    tot = int(nnz.sum())
    out = dict(m=np.array([m for _, m in sizes], np.intc), nblk=np.ones(count, np.intc),
               bs=np.array([n for n, _ in sizes], np.intc), c=np.empty(sum(m for _, m in sizes)),
               nnz=nnz, mat=np.empty(tot, np.intc), blk=np.ones(tot, np.intc), i=np.empty(tot, np.intc),
               j=np.empty(tot, np.intc), v=np.empty(tot))
    e = cc = 0
    for q, (n, m) in enumerate(sizes):
        d = random_dense_instance(np.random.default_rng([seed, first + q]), int(n), int(m))
        k = d.v.size
        if k != nnz[q]:
            raise RuntimeError("batch instance size mismatch")
        out["mat"][e:e + k] = d.mat
        out["i"][e:e + k] = d.i
        out["j"][e:e + k] = d.j
        out["v"][e:e + k] = d.v
        out["c"][cc:cc + m] = d.c
        e += k
        cc += m
    return out


def batch_instance(q: int, count: int = 4096, nmin: int = 8, nmax: int = 64, seed: int = 0) -> SdpaData:
    """Instance q of random_dense_batch(count, nmin, nmax, seed), made without the others."""
    n, m = random_dense_batch(count, nmin, nmax, seed, sizes_only=True)[q]
    return random_dense_instance(np.random.default_rng([seed, q]), int(n), int(m), name=f"batch{seed}_{q}")


# ---------------------------------------------------------------------------------------
# SDPA sparse files
# ---------------------------------------------------------------------------------------
def write_sdpa(d: SdpaData, path: str) -> None:
    """Write an SDPA sparse file (values with 17 significant digits: reading it back gives
    the same doubles)."""
    with open(path, "w") as f:
        f.write(f'"{d.name}"\n{d.m}\n{d.nblk}\n')
        f.write(" ".join(str(int(b)) for b in d.bs) + "\n")
        f.write(" ".join(repr(float(x)) for x in d.c) + "\n")
        arr = np.empty(d.nnz, dtype=[("mat", "i4"), ("blk", "i4"), ("i", "i4"), ("j", "i4"), ("v", "f8")])
        arr["mat"], arr["blk"], arr["i"], arr["j"], arr["v"] = d.mat, d.blk, d.i, d.j, d.v
        np.savetxt(f, arr, fmt=["%d", "%d", "%d", "%d", "%.17g"])


def read_sdpa(path: str) -> SdpaData:
    """Read an SDPA sparse file (comments '"' / '*' lines, separators , ( ) { })."""
    with open(path) as f:
        toks = []
        body = []
        header_done = False
        for line in f:
            s = line.strip()
            if not s or s[0] in '"*':
                continue
            s = s.translate(str.maketrans(",(){}", "     "))
            if not header_done:
                toks.extend(s.split())
                if len(toks) >= 2:
                    m, nb = int(float(toks[0])), int(float(toks[1]))
                    if len(toks) >= 2 + nb + m:
                        header_done = True
                        rest = toks[2 + nb + m:]
                        if rest:
                            body.append(" ".join(rest))
                continue
            body.append(s)
    m, nb = int(float(toks[0])), int(float(toks[1]))
    bs = np.array([int(float(x)) for x in toks[2:2 + nb]], np.int32)
    c = np.array([float(x) for x in toks[2 + nb:2 + nb + m]])
    vals = np.array(" ".join(body).split(), dtype=np.float64).reshape(-1, 5) if body else np.zeros((0, 5))
    d = _normalise(vals[:, 0].astype(np.int32), vals[:, 1].astype(np.int32), vals[:, 2].astype(np.int32),
                   vals[:, 3].astype(np.int32), vals[:, 4])
    keep = d[4] != 0
    return SdpaData(bs, c, *(a[keep] for a in d), name=path)


WORKLOADS = {
    "theta50": dict(fn=theta_problem, kw=dict(n=50, p=0.5, seed=1)),
    "rand400": dict(fn=random_sdp, kw=dict(n=400, m=2000, density=0.01, seed=0)),
    "rand1000": dict(fn=random_sdp, kw=dict(n=1000, m=8000, density=0.005, seed=0)),
}


def workload(name: str, **over) -> SdpaData:
    w = WORKLOADS[name]
    kw = dict(w["kw"])
    kw.update(over)
    return w["fn"](**kw)


def _monomials_upto(vars_, deg):
    """Monomials of degree <= deg in the given variables, as sorted tuples (graded order)."""
    out = [()]
    frontier = [()]
    for _ in range(deg):
        nxt = []
        for mono in frontier:
            start = vars_.index(mono[-1]) if mono else 0
            for v in vars_[start:]:
                nxt.append(mono + (v,))
        out.extend(nxt)
        frontier = nxt
    return out


def moment_relaxation(nvars: int = 60, clique: int = 4, seed: int = 0) -> SdpaData:
    """Degree-2 (order-2) sparse moment relaxation of a seeded random quartic with chain cliques.

    f(x) = sum of c_alpha x^alpha over every monomial of degree <= 4 supported on one of the
    cliques {i, ..., i+clique-1} (i = 0..nvars-clique), c_alpha ~ N(0,1), except that each x_i^4
    gets 1 + the sum of |c| of the other quartic monomials containing x_i, so f is bounded
    below and the relaxation has an optimum.  The relaxation
    min sum c_alpha y_alpha  s.t.  M_2(y, I_k) >= 0 for every clique, y_0 = 1
    has one moment block per clique, indexed by the monomials of degree <= 2 in its variables
    (15 x 15 for cliques of 4), and one free moment y_alpha per monomial alpha != 0.  In BRISK's
    form max b'y s.t. C - sum y_i A_i = Z >= 0: C = B_0, A_i = -B_alpha_i, b_i = -c_alpha_i, where
    B_alpha has a 1 at (u, v) of block k whenever u + v = alpha.  The optimal value is
    c_0 - (the SDP's b'y)."""
    rng = np.random.default_rng(seed)
    cliques = [tuple(range(i, i + clique)) for i in range(nvars - clique + 1)]
    index = {}

    def mono_id(mono):
        if mono not in index:
            index[mono] = len(index)
        return index[mono]

    mono_id(())
    for cl in cliques:
        for mono in _monomials_upto(list(cl), 4):
            mono_id(mono)
    coef = rng.standard_normal(len(index))
    # bounded below: each x_i^4 gets 1 + the absolute sum of the other quartic coefficients
    # whose monomial contains x_i (the random quartic would otherwise be unbounded)
    for mono, t in index.items():
        if len(mono) == 4 and len(set(mono)) == 1:
            i = mono[0]
            coef[t] = 1.0 + sum(abs(coef[u]) for mo, u in index.items()
                                if len(mo) == 4 and i in mo and len(set(mo)) > 1)
    m = len(index) - 1                        # every moment but y_0
    mats, blks, ii, jj, vv = [], [], [], [], []
    for k, cl in enumerate(cliques):
        basis = _monomials_upto(list(cl), 2)
        for a in range(len(basis)):
            for b in range(a, len(basis)):
                alpha = tuple(sorted(basis[a] + basis[b]))
                t = index[alpha]
                # F0 = -C = -B_0 at t = 0; F_t = A_t = -B_alpha otherwise
                mats.append(t)
                blks.append(k + 1)
                ii.append(a + 1)
                jj.append(b + 1)
                vv.append(-1.0)
    c = -coef[1:]
    d = _normalise(np.array(mats), np.array(blks), np.array(ii), np.array(jj), np.array(vv))
    nb = len(cliques)
    bsz = len(_monomials_upto(list(cliques[0]), 2))
    return SdpaData(np.full(nb, bsz, np.int32), c, *d, name=f"moment_chain_n{nvars}_c{clique}_seed{seed}",
                    meta=dict(kind="moment", nvars=nvars, clique=clique, seed=seed, offset=float(coef[0]), m=m))
