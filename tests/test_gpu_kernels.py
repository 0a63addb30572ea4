"""Kernel parity through the C ABI (include/bgpu.h) on a B200: each kernel against the oracle
(oracle/restate.py) or a plain FP64 reference of the same operation.  Device memory comes from
torch (allocation only); every compute call goes through libbrisk.so."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from brisk_b200 import problems, step  # noqa: E402
from oracle import restate  # noqa: E402


def dev(a, cuda, dtype=None):
    t = torch.as_tensor(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.to(cuda).contiguous()


def colmajor(A, cuda):
    """A column-major copy (the transpose's row-major buffer)."""
    return dev(np.asarray(A).T, cuda)


def from_colmajor(t, n, m=None):
    m = n if m is None else m
    return t.cpu().numpy().reshape(m, n).T


@pytest.mark.parametrize("akm,bkm", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("M,N,K", [(1, 1, 1), (130, 70, 33), (257, 200, 64), (64, 513, 129)])
def test_dgemm_layouts(cuda, akm, bkm, M, N, K):
    rng = np.random.default_rng(M * 7 + N + K)
    A = rng.standard_normal((M, K))
    B = rng.standard_normal((K, N))
    C0 = rng.standard_normal((M, N))
    # device buffers in the requested layouts
    dA = dev(A if akm else A.T, cuda)            # KMAJOR: A[i*lda+k] (row-major); MMAJOR: column-major
    dB = dev(B.T if bkm else B, cuda)            # KMAJOR: B[k+j*ldb] (column-major); NMAJOR: row-major
    dC = colmajor(C0, cuda)
    lda = K if akm else M
    ldb = K if bkm else N
    step.call("dgemm", akm, bkm, M, N, K, 1.5, dA.data_ptr(), lda, dB.data_ptr(), ldb, -0.5, dC.data_ptr(), M, 0, None)
    step.call("sync", None)
    got = from_colmajor(dC, M, N) if False else dC.cpu().numpy().reshape(N, M).T
    want = 1.5 * A @ B - 0.5 * C0
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())


def test_dgemm_lower_only(cuda):
    rng = np.random.default_rng(1)
    n, K = 150, 40
    A = rng.standard_normal((n, K))
    C0 = rng.standard_normal((n, n))
    dA = dev(A.T, cuda)                          # column-major n x K (MMAJOR), also N-major for B
    dC = colmajor(C0, cuda)
    step.call("dgemm", 0, 0, n, n, K, -1.0, dA.data_ptr(), n, dA.data_ptr(), n, 1.0, dC.data_ptr(), n, 1, None)
    step.call("sync", None)
    got = dC.cpu().numpy().reshape(n, n).T
    want = C0 - A @ A.T
    low = np.tril_indices(n)
    np.testing.assert_allclose(got[low], want[low], rtol=1e-12, atol=1e-11)
    up = np.triu_indices(n, 1)
    np.testing.assert_array_equal(got[up], C0[up])


def spd(n, seed, cond=1e3):
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    ev = np.logspace(0, np.log10(cond), n)
    return (Q * ev) @ Q.T


@pytest.mark.parametrize("n", [1, 63, 64, 65, 200, 700])
def test_potrf_trsv_trtri(cuda, n):
    A = spd(n, n)
    L_ref = np.linalg.cholesky(A)
    dA = colmajor(A, cuda)
    nb = (n + 63) // 64
    dinv = torch.zeros(nb * 4096, dtype=torch.float64, device=cuda)
    info = torch.zeros(1, dtype=torch.int32, device=cuda)
    pmin = torch.zeros(1, dtype=torch.float64, device=cuda)
    step.call("potrf", n, dA.data_ptr(), n, dinv.data_ptr(), info.data_ptr(), pmin.data_ptr(), None)
    step.call("sync", None)
    assert int(info.item()) == 0
    L = np.tril(dA.cpu().numpy().reshape(n, n).T)
    np.testing.assert_allclose(L, L_ref, rtol=1e-10, atol=1e-12 * np.abs(L_ref).max())
    # the smallest squared pivot, capped at 1 (schur_factor_'s pmin starts at 1.0, solver.c:5346)
    assert pmin.item() == pytest.approx(min(1.0, np.min(np.diag(L_ref)) ** 2), rel=1e-10)
    # triangular solves
    rng = np.random.default_rng(n + 1)
    b = rng.standard_normal(n)
    flags = torch.zeros(nb, dtype=torch.int32, device=cuda)
    err = torch.zeros(1, dtype=torch.int32, device=cuda)
    x = dev(b, cuda)
    step.call("trsv", n, dA.data_ptr(), n, dinv.data_ptr(), x.data_ptr(), 0, flags.data_ptr(), 1, err.data_ptr(), None)
    step.call("trsv", n, dA.data_ptr(), n, dinv.data_ptr(), x.data_ptr(), 1, flags.data_ptr(), 2, err.data_ptr(), None)
    step.call("sync", None)
    assert int(err.item()) == 0
    np.testing.assert_allclose(x.cpu().numpy(), np.linalg.solve(A, b), rtol=1e-8, atol=1e-10)
    # inverse of the factor
    Li = torch.zeros(n * n, dtype=torch.float64, device=cuda)
    step.call("trtri", n, dA.data_ptr(), n, dinv.data_ptr(), Li.data_ptr(), n, None)
    step.call("sync", None)
    got = Li.cpu().numpy().reshape(n, n).T
    np.testing.assert_allclose(got @ L_ref, np.eye(n), atol=1e-9)


def test_potrf_reports_first_nonpositive_pivot(cuda):
    n = 130
    A = spd(n, 3)
    A[100, 100] = -1.0           # leading minors up to 100 stay definite
    dA = colmajor(A, cuda)
    dinv = torch.zeros(3 * 4096, dtype=torch.float64, device=cuda)
    info = torch.zeros(1, dtype=torch.int32, device=cuda)
    pmin = torch.zeros(1, dtype=torch.float64, device=cuda)
    step.call("potrf", n, dA.data_ptr(), n, dinv.data_ptr(), info.data_ptr(), pmin.data_ptr(), None)
    step.call("sync", None)
    want = next(k + 1 for k in range(n) if np.linalg.eigvalsh(A[:k + 1, :k + 1])[0] <= 0)
    assert int(info.item()) == want


@pytest.mark.parametrize("n", [64, 300])
def test_potrf_f32_and_trsv_f32(cuda, n):
    A = spd(n, 11, cond=50)
    dA = colmajor(A, cuda).float()
    nb = (n + 63) // 64
    dinv = torch.zeros(nb * 4096, dtype=torch.float32, device=cuda)
    info = torch.zeros(1, dtype=torch.int32, device=cuda)
    pmin = torch.zeros(1, dtype=torch.float64, device=cuda)
    step.call("potrf_f32", n, dA.data_ptr(), n, dinv.data_ptr(), info.data_ptr(), pmin.data_ptr(), None)
    b = np.random.default_rng(2).standard_normal(n)
    x = dev(b, cuda).float()
    flags = torch.zeros(nb, dtype=torch.int32, device=cuda)
    err = torch.zeros(1, dtype=torch.int32, device=cuda)
    step.call("trsv_f32", n, dA.data_ptr(), n, dinv.data_ptr(), x.data_ptr(), 0, flags.data_ptr(), 5, err.data_ptr(), None)
    step.call("trsv_f32", n, dA.data_ptr(), n, dinv.data_ptr(), x.data_ptr(), 1, flags.data_ptr(), 6, err.data_ptr(), None)
    step.call("sync", None)
    assert int(info.item()) == 0 and int(err.item()) == 0
    np.testing.assert_allclose(x.cpu().numpy(), np.linalg.solve(A, b), rtol=1e-4, atol=1e-4)


def block_arrays(d, cuda):
    """Constraint-major device arrays of block 1 of an SdpaData, as the solver lays them out:
    scaled entries (problem_prepare), full expansion sorted by position p + q n."""
    S = restate.scale_problem(d)
    n = int(d.bs[0])
    A = S.A[0]
    con, cptr, cpos, cval = [], [0], [], []
    for t in range(d.m):
        iq = np.nonzero(A[t].T.ravel())[0]          # column-major positions
        if iq.size == 0:
            continue
        con.append(t)
        cpos.extend(iq.tolist())
        cval.extend(A[t].T.ravel()[iq].tolist())
        cptr.append(len(cpos))
    arrs = dict(con=torch.tensor(con, dtype=torch.int32, device=cuda),
                cptr=torch.tensor(cptr, dtype=torch.int64, device=cuda),
                cpos=torch.tensor(cpos, dtype=torch.int32, device=cuda),
                cval=torch.tensor(cval, dtype=torch.float64, device=cuda))
    arrs["ccol"] = torch.zeros(len(con) * (n + 1), dtype=torch.int32, device=cuda)
    step.call("schur_colptr", n, len(con), arrs["cptr"].data_ptr(), arrs["cpos"].data_ptr(), arrs["ccol"].data_ptr(),
              None)
    return S, n, arrs


@pytest.mark.parametrize("name,kw,chunk", [
    ("rand30", dict(n=30, m=60, density=0.1, seed=1), 8),
    ("rand60", dict(n=60, m=200, density=0.05, seed=2), 32),
    ("rand100", dict(n=100, m=300, density=0.02, seed=3), 64),
    ("theta50", None, 16),
])
def test_schur_fp64_matches_oracle(cuda, name, kw, chunk):
    d = problems.theta_problem() if kw is None else problems.random_sdp(**kw)
    S, n, a = block_arrays(d, cuda)
    rng = np.random.default_rng(4)
    X = spd(n, 5, cond=100)
    Zi = spd(n, 6, cond=100)
    want = restate.schur(S.A, [X], [Zi])
    M = torch.zeros(d.m * d.m, dtype=torch.float64, device=cuda)
    ws = torch.empty(step.ws_bytes(n, chunk, 0), dtype=torch.uint8, device=cuda)
    dX, dZi = colmajor(X, cuda), colmajor(Zi, cuda)
    step.call("schur_assemble", n, d.m, int(a["con"].numel()), a["con"].data_ptr(), a["cptr"].data_ptr(),
              a["ccol"].data_ptr(), a["cpos"].data_ptr(), a["cval"].data_ptr(), dX.data_ptr(), dZi.data_ptr(), M.data_ptr(), 0, chunk,
              ws.data_ptr(), ws.numel(), None)
    step.call("sync", None)
    got = M.cpu().numpy().reshape(d.m, d.m).T
    np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-12 * np.abs(want).max())


def test_first_schur_matches_oracle_at_start(cuda, golden):
    """M at the first iteration (the SDPT3 start on the scaled problem), FP64: 1e-10 relative."""
    d = problems.random_sdp(**golden["rand60"]["kwargs"])
    S, n, a = block_arrays(d, cuda)
    X, Z, y, xi, eta = restate.start_point(S)
    Zi = np.linalg.inv(Z[0])
    want = restate.schur(S.A, X, [Zi])
    M = torch.zeros(d.m * d.m, dtype=torch.float64, device=cuda)
    ws = torch.empty(step.ws_bytes(n, 0, 0), dtype=torch.uint8, device=cuda)
    dX, dZi = colmajor(X[0], cuda), colmajor(Zi, cuda)   # kept alive across the call
    step.call("schur_assemble", n, d.m, int(a["con"].numel()), a["con"].data_ptr(), a["cptr"].data_ptr(),
              a["ccol"].data_ptr(), a["cpos"].data_ptr(), a["cval"].data_ptr(), dX.data_ptr(), dZi.data_ptr(), M.data_ptr(), 0, 0,
              ws.data_ptr(), ws.numel(), None)
    step.call("sync", None)
    got = M.cpu().numpy().reshape(d.m, d.m).T
    rel = np.abs(got - want).max() / np.abs(want).max()
    assert rel <= 1e-10


def upper_arrays(a, n, cuda):
    """The upper-triangle lists of bgpu_schur_upper (count call, then fill call)."""
    ncon = int(a["con"].numel())
    counts = torch.zeros(max(ncon, 1), dtype=torch.int32, device=cuda)
    uptr = torch.zeros(ncon + 1, dtype=torch.int64, device=cuda)
    nu = ctypes.c_longlong(0)
    step.call("schur_upper", n, ncon, a["cptr"].data_ptr(), a["cpos"].data_ptr(), a["cval"].data_ptr(),
              counts.data_ptr(), uptr.data_ptr(), None, None, ctypes.addressof(nu), None)
    upos = torch.zeros(max(nu.value, 1), dtype=torch.int32, device=cuda)
    uval = torch.zeros(max(nu.value, 1), dtype=torch.float64, device=cuda)
    step.call("schur_upper", n, ncon, a["cptr"].data_ptr(), a["cpos"].data_ptr(), a["cval"].data_ptr(),
              counts.data_ptr(), uptr.data_ptr(), upos.data_ptr(), uval.data_ptr(), ctypes.addressof(nu), None)
    step.call("sync", None)
    return dict(uptr=uptr, upos=upos, uval=uval, nu=nu.value)


def test_upper_lists_match_numpy(cuda):
    """Entries p <= q of each constraint, packed index q (q+1)/2 + p ascending, same values."""
    d = problems.random_sdp(n=60, m=200, density=0.05, seed=2)
    S, n, a = block_arrays(d, cuda)
    u = upper_arrays(a, n, cuda)
    cptr, cpos, cval = (a[k].cpu().numpy() for k in ("cptr", "cpos", "cval"))
    uptr, upos, uval = u["uptr"].cpu().numpy(), u["upos"].cpu().numpy()[:u["nu"]], u["uval"].cpu().numpy()[:u["nu"]]
    want_ptr, want_pos, want_val = [0], [], []
    for t in range(len(cptr) - 1):
        pos = cpos[cptr[t]:cptr[t + 1]]
        q, p = pos // n, pos % n
        keep = p <= q
        want_pos.extend((q[keep] * (q[keep] + 1) // 2 + p[keep]).tolist())
        want_val.extend(cval[cptr[t]:cptr[t + 1]][keep].tolist())
        want_ptr.append(len(want_pos))
    np.testing.assert_array_equal(uptr, want_ptr)
    np.testing.assert_array_equal(upos, want_pos)
    np.testing.assert_array_equal(uval, want_val)
    assert all(np.all(np.diff(upos[uptr[t]:uptr[t + 1]]) > 0) for t in range(len(uptr) - 1))


@pytest.mark.parametrize("name,kw,chunk", [
    ("rand30", dict(n=30, m=60, density=0.1, seed=1), 8),
    ("rand60", dict(n=60, m=200, density=0.05, seed=2), 32),
    ("rand100", dict(n=100, m=300, density=0.02, seed=3), 64),
    ("theta50", None, 16),
])
def test_schur_sym_gather_matches_oracle(cuda, name, kw, chunk):
    """The packed symmetric gather (G + G' on the upper triangle, upper entries only): FP64 M to
    1e-10 of the oracle; the 3xTF32 one to 1e-5 of the FP64 one."""
    d = problems.theta_problem() if kw is None else problems.random_sdp(**kw)
    S, n, a = block_arrays(d, cuda)
    u = upper_arrays(a, n, cuda)
    X = spd(n, 5, cond=100)
    Zi = spd(n, 6, cond=100)
    want = restate.schur(S.A, [X], [Zi])
    dX, dZi = colmajor(X, cuda), colmajor(Zi, cuda)
    got = []
    for prec in (0, 1):
        M = torch.zeros(d.m * d.m, dtype=torch.float64, device=cuda)
        ws = torch.empty(step.ws_bytes(n, chunk, prec), dtype=torch.uint8, device=cuda)
        step.call("schur_assemble_sym", n, d.m, int(a["con"].numel()), a["con"].data_ptr(), a["cptr"].data_ptr(),
                  a["ccol"].data_ptr(), a["cpos"].data_ptr(), a["cval"].data_ptr(), u["uptr"].data_ptr(),
                  u["upos"].data_ptr(), u["uval"].data_ptr(), dX.data_ptr(), dZi.data_ptr(), M.data_ptr(), prec,
                  chunk, ws.data_ptr(), ws.numel(), None)
        step.call("sync", None)
        got.append(M.cpu().numpy().reshape(d.m, d.m).T)
    np.testing.assert_allclose(got[0], want, rtol=1e-10, atol=1e-12 * np.abs(want).max())
    assert np.abs(got[1] - got[0]).max() / np.abs(got[0]).max() <= 1e-5


def test_schur_large_block_gather_staged_by_cp_async(cuda):
    """A block of order 820: the chunk's packed sum S outgrows 32 MB at 64 constraints (86 MB in
    FP32, 172 MB in FP64), so the gather stages S rows through shared memory with cp.async; at 8
    constraints S stays small and the register gather runs.  Both give the same M (FP64: 1e-12),
    the 3xTF32 one within 1e-5, and the FP64 one matches the sparse restatement M_ab = <A_b, X A_a Zi>."""
    d = problems.random_sdp(n=820, m=96, density=0.005, seed=11)
    S, n, a = block_arrays(d, cuda)
    u = upper_arrays(a, n, cuda)
    X = spd(n, 5, cond=100)
    Zi = spd(n, 6, cond=100)
    dX, dZi = colmajor(X, cuda), colmajor(Zi, cuda)
    got = {}
    for prec, chunk in ((0, 64), (0, 8), (1, 64)):
        M = torch.zeros(d.m * d.m, dtype=torch.float64, device=cuda)
        ws = torch.empty(step.ws_bytes(n, chunk, prec), dtype=torch.uint8, device=cuda)
        step.call("schur_assemble_sym", n, d.m, int(a["con"].numel()), a["con"].data_ptr(), a["cptr"].data_ptr(),
                  a["ccol"].data_ptr(), a["cpos"].data_ptr(), a["cval"].data_ptr(), u["uptr"].data_ptr(),
                  u["upos"].data_ptr(), u["uval"].data_ptr(), dX.data_ptr(), dZi.data_ptr(), M.data_ptr(), prec,
                  chunk, ws.data_ptr(), ws.numel(), None)
        step.call("sync", None)
        got[(prec, chunk)] = M.cpu().numpy().reshape(d.m, d.m).T
    ref = got[(0, 8)]
    scale = np.abs(ref).max()
    assert np.abs(got[(0, 64)] - ref).max() <= 1e-12 * scale
    assert np.abs(got[(1, 64)] - ref).max() <= 1e-5 * scale
    A = S.A[0]
    G = np.stack([X @ A[t] @ Zi for t in range(d.m)])
    want = np.einsum("ipq,jpq->ij", A, G)
    np.testing.assert_allclose(got[(0, 64)], want, rtol=1e-10, atol=1e-12 * np.abs(want).max())


@pytest.mark.parametrize("kw", [dict(n=60, m=200, density=0.05, seed=2), dict(n=100, m=300, density=0.02, seed=3)])
def test_gram_matches_numpy(cuda, kw):
    """bgpu_schur_gram: <A_a, A_b> of the scaled constraints, to 1e-13 relative."""
    d = problems.random_sdp(**kw)
    S, n, a = block_arrays(d, cuda)
    u = upper_arrays(a, n, cuda)
    Af = np.stack([A.ravel() for A in S.A[0]])
    want = Af @ Af.T
    M = torch.zeros(d.m * d.m, dtype=torch.float64, device=cuda)
    ws = torch.empty(step.ws_bytes(n, 0, 0), dtype=torch.uint8, device=cuda)
    step.call("schur_gram", n, d.m, int(a["con"].numel()), a["con"].data_ptr(), u["uptr"].data_ptr(),
              u["upos"].data_ptr(), u["uval"].data_ptr(), M.data_ptr(), ws.data_ptr(), ws.numel(), None)
    step.call("sync", None)
    got = M.cpu().numpy().reshape(d.m, d.m).T
    np.testing.assert_allclose(got, want, rtol=1e-13, atol=1e-13 * np.abs(want).max())


def test_aop_and_symv(cuda):
    d = problems.random_sdp(n=40, m=50, density=0.1, seed=9)
    S, n, a = block_arrays(d, cuda)
    D = spd(n, 7)
    out = torch.zeros(d.m, dtype=torch.float64, device=cuda)
    dD = colmajor(D, cuda)
    step.call("aop", n, int(a["con"].numel()), a["con"].data_ptr(), a["cptr"].data_ptr(), a["cpos"].data_ptr(),
              a["cval"].data_ptr(), dD.data_ptr(), 1.0, 0.0, out.data_ptr(), None)
    step.call("sync", None)
    np.testing.assert_allclose(out.cpu().numpy(), restate.aop(S.A, [D]), rtol=1e-12, atol=1e-12)
    M = spd(300, 8)
    x = np.random.default_rng(3).standard_normal(300)
    y = torch.zeros(300, dtype=torch.float64, device=cuda)
    dM, dx = colmajor(M, cuda), dev(x, cuda)
    step.call("symv", 300, 2.0, dM.data_ptr(), 300, dx.data_ptr(), 0.0, y.data_ptr(), None)
    step.call("sync", None)
    np.testing.assert_allclose(y.cpu().numpy(), 2.0 * M @ x, rtol=1e-12, atol=1e-10)


@pytest.mark.parametrize("M,N,K", [(128, 208, 32), (300, 400, 400), (1000, 1000, 1000), (16000, 256, 100), (130, 129, 37)])
def test_gemm_tf32x3_accuracy(cuda, M, N, K):
    """3xTF32 on tcgen05 reaches FP32-level accuracy: |G - A B| <= 2e-6 |A||B| entrywise bound
    against the FP64 product of the unsplit inputs."""
    rng = np.random.default_rng(M + N + K)
    A = rng.standard_normal((M, K))
    B = rng.standard_normal((K, N))
    Kp = (K + 3) // 4 * 4                          # 16-byte row stride for the tensor maps
    dA = torch.zeros((M, Kp), dtype=torch.float64, device=cuda)
    dA[:, :K] = torch.as_tensor(A, device=cuda)
    dBt = torch.zeros((N, Kp), dtype=torch.float64, device=cuda)
    dBt[:, :K] = torch.as_tensor(B.T, device=cuda)
    Ah = torch.empty((M, Kp), dtype=torch.float32, device=cuda)
    Al = torch.empty_like(Ah)
    Bh = torch.empty((N, Kp), dtype=torch.float32, device=cuda)
    Bl = torch.empty_like(Bh)
    step.call("split_tf32", M * Kp, dA.data_ptr(), Ah.data_ptr(), Al.data_ptr(), None)
    step.call("split_tf32", N * Kp, dBt.data_ptr(), Bh.data_ptr(), Bl.data_ptr(), None)
    G = torch.zeros(M * N, dtype=torch.float32, device=cuda)
    step.call("gemm_tf32x3", M, N, K, Ah.data_ptr(), Al.data_ptr(), Kp, Bh.data_ptr(), Bl.data_ptr(), Kp,
              G.data_ptr(), M, None)
    step.call("sync", None)
    got = G.cpu().numpy().reshape(N, M).T.astype(np.float64)
    want = A @ B
    bound = np.abs(A) @ np.abs(B)
    assert np.max(np.abs(got - want) / bound) <= 2e-6


def test_schur_tf32x3_matches_fp64(cuda):
    """The mixed-precision assembly (3xTF32 GEMM, FP32 G, FP64 gather) against the FP64 one."""
    d = problems.random_sdp(n=100, m=300, density=0.02, seed=3)
    S, n, a = block_arrays(d, cuda)
    X = spd(n, 5, cond=100)
    Zi = spd(n, 6, cond=100)
    dX, dZi = colmajor(X, cuda), colmajor(Zi, cuda)
    out = []
    for prec in (0, 1):
        M = torch.zeros(d.m * d.m, dtype=torch.float64, device=cuda)
        ws = torch.empty(step.ws_bytes(n, 16, prec), dtype=torch.uint8, device=cuda)
        step.call("schur_assemble", n, d.m, int(a["con"].numel()), a["con"].data_ptr(), a["cptr"].data_ptr(),
                  a["ccol"].data_ptr(), a["cpos"].data_ptr(), a["cval"].data_ptr(), dX.data_ptr(), dZi.data_ptr(), M.data_ptr(), prec, 16,
                  ws.data_ptr(), ws.numel(), None)
        step.call("sync", None)
        out.append(M.cpu().numpy().reshape(d.m, d.m).T)
    rel = np.abs(out[1] - out[0]).max() / np.abs(out[0]).max()
    assert rel <= 1e-5


def _ptr_table(tensors, cuda):
    return torch.tensor([t.data_ptr() for t in tensors], dtype=torch.int64, device=cuda)


def test_small_batched_chol_gemm_lammin(cuda):
    """The one-CTA-per-block kernels on blocks of uneven order (1..64) against numpy FP64."""
    rng = np.random.default_rng(21)
    sizes = [1, 2, 7, 15, 15, 31, 32, 33, 63, 64]
    A = [spd(n, 100 + n) for n in sizes]
    D = []
    for n in sizes:
        R = rng.standard_normal((n, n))
        D.append(R + R.T)
    dA = [colmajor(a, cuda) for a in A]
    dL = [torch.zeros(n * n, dtype=torch.float64, device=cuda) for n in sizes]
    dLi = [torch.zeros(n * n, dtype=torch.float64, device=cuda) for n in sizes]
    dD = [colmajor(d, cuda) for d in D]
    ns = torch.tensor(sizes, dtype=torch.int32, device=cuda)
    info = torch.full((len(sizes),), -1, dtype=torch.int32, device=cuda)
    tA, tL, tLi, tD = (_ptr_table(x, cuda) for x in (dA, dL, dLi, dD))
    step.call("small_chol_inv", len(sizes), ns.data_ptr(), tA.data_ptr(), tL.data_ptr(), tLi.data_ptr(),
              info.data_ptr(), None)
    lam = torch.zeros(len(sizes), dtype=torch.float64, device=cuda)
    step.call("small_lammin", len(sizes), ns.data_ptr(), tLi.data_ptr(), tD.data_ptr(), lam.data_ptr(), None)
    C = [torch.zeros(n * n, dtype=torch.float64, device=cuda) for n in sizes]
    tC = _ptr_table(C, cuda)
    step.call("small_gemm", len(sizes), ns.data_ptr(), 1, 0, 2.0, tLi.data_ptr(), tD.data_ptr(), 0.0, tC.data_ptr(), 0,
              None)
    step.call("sync", None)
    assert info.cpu().numpy().tolist() == [0] * len(sizes)
    for k, n in enumerate(sizes):
        Lr = np.linalg.cholesky(A[k])
        L = dL[k].cpu().numpy().reshape(n, n).T
        Li = dLi[k].cpu().numpy().reshape(n, n).T
        np.testing.assert_allclose(L, Lr, rtol=1e-10, atol=1e-12 * np.abs(Lr).max())
        np.testing.assert_allclose(Li @ Lr, np.eye(n), atol=1e-9)
        Lir = np.linalg.inv(Lr)
        B = Lir @ D[k] @ Lir.T
        want = np.linalg.eigvalsh(0.5 * (B + B.T))[0]
        assert lam[k].item() <= want + 1e-10 * max(1.0, abs(want))
        assert lam[k].item() == pytest.approx(want, rel=1e-9, abs=1e-10)
        got = C[k].cpu().numpy().reshape(n, n).T
        np.testing.assert_allclose(got, 2.0 * Lir.T @ D[k], rtol=1e-10, atol=1e-10 * np.abs(got).max())


def test_small_chol_reports_failure(cuda):
    n = 20
    A = spd(n, 4)
    A[12, 12] = -5.0
    dA = colmajor(A, cuda)
    dL = torch.zeros(n * n, dtype=torch.float64, device=cuda)
    ns = torch.tensor([n], dtype=torch.int32, device=cuda)
    info = torch.zeros(1, dtype=torch.int32, device=cuda)
    tA, tL = _ptr_table([dA], cuda), _ptr_table([dL], cuda)
    step.call("small_chol_inv", 1, ns.data_ptr(), tA.data_ptr(), tL.data_ptr(), 0, info.data_ptr(), None)
    step.call("sync", None)
    want = next(k + 1 for k in range(n) if np.linalg.eigvalsh(A[:k + 1, :k + 1])[0] <= 0)
    assert int(info.item()) == want


@pytest.mark.parametrize("prec,tol", [(0, 1e-10), (1, 1e-5)])
def test_schur_dense_route_matches_oracle(cuda, prec, tol):
    """The dense route (M[:, a] = Ad vec(X A_a Zi) by GEMM) on a dense-constraint block."""
    rng = np.random.default_rng(5)
    d = problems.random_dense_instance(rng, 24, 100)
    S, n, a = block_arrays(d, cuda)
    X = spd(n, 8, cond=50)
    Zi = spd(n, 9, cond=50)
    want = restate.schur(S.A, [X], [Zi])
    ncon = int(a["con"].numel())
    Ad = torch.zeros(ncon * n * n, dtype=torch.float64, device=cuda)
    step.call("schur_densify", n, ncon, a["cptr"].data_ptr(), a["cpos"].data_ptr(), a["cval"].data_ptr(),
              Ad.data_ptr(), None)
    M = torch.zeros(d.m * d.m, dtype=torch.float64, device=cuda)
    chunk = 16
    ws = torch.empty(int(step.lib().bgpu_schur_dense_ws_bytes(n, ncon, chunk, prec)), dtype=torch.uint8, device=cuda)
    dX, dZi = colmajor(X, cuda), colmajor(Zi, cuda)
    step.call("schur_assemble_dense", n, d.m, ncon, a["con"].data_ptr(), a["cptr"].data_ptr(), a["ccol"].data_ptr(),
              a["cpos"].data_ptr(), a["cval"].data_ptr(), Ad.data_ptr(), dX.data_ptr(), dZi.data_ptr(), M.data_ptr(),
              prec, chunk, ws.data_ptr(), ws.numel(), None)
    step.call("sync", None)
    got = M.cpu().numpy().reshape(d.m, d.m).T
    assert np.abs(got - want).max() / np.abs(want).max() <= tol
