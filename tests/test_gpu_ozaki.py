"""FP64-accurate products on the INT8 tensor cores (ozaki.cu, tcgen05 kind::i8) through the C ABI:
the GEMM against numpy FP64 within the Ozaki bound, the Schur assembly in that precision against
the FP64 one, and solves with it against the reference's own runs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import brisk_b200  # noqa: E402
from brisk_b200 import problems, step  # noqa: E402
from parity import objectives_close  # noqa: E402

from test_gpu_kernels import block_arrays, colmajor, spd, upper_arrays  # noqa: E402


def ozaki(A, B, cuda, slices=8):
    """C = A B' through bgpu_gemm_ozaki (8 slices) or bgpu_gemm_ozaki_slices (A: M x K, B: N x K,
    row-major with K contiguous)."""
    M, K = A.shape
    N = B.shape[0]
    dA = torch.as_tensor(np.ascontiguousarray(A)).to(cuda)
    dB = torch.as_tensor(np.ascontiguousarray(B)).to(cuda)
    C = torch.full((N, M), np.nan, dtype=torch.float64, device=cuda)   # column-major M x N
    nws = int(step.lib().bgpu_ozaki_ws_bytes(M, N, K))
    ws = torch.empty(nws, dtype=torch.uint8, device=cuda)
    if slices == 8:
        step.call("gemm_ozaki", M, N, K, dA.data_ptr(), K, dB.data_ptr(), K, C.data_ptr(), M, ws.data_ptr(), nws, None)
    else:
        step.call("gemm_ozaki_slices", slices, M, N, K, dA.data_ptr(), K, dB.data_ptr(), K, C.data_ptr(), M,
                  ws.data_ptr(), nws, None)
    return C.cpu().numpy().T


def bound_slices(A, B, S):
    """The bound with S slices: (S + 3) 2^(-7 S) K max_k |A(i, k)| max_k |B(j, k)| (the dropped pairs
    p + q >= S + 2 and the slices' truncation), with a factor 2 of margin."""
    K = A.shape[1]
    return 2 * (S + 3) * 2.0 ** (-7 * S) * K * np.outer(np.abs(A).max(axis=1), np.abs(B).max(axis=1))


def bound(A, B):
    """The Ozaki error bound per element: about K 2^-53 max_k |A(i, k)| max_k |B(j, k)| (8 slices of 7
    bits, the products with p + q <= 9 kept), with a factor 8 of margin."""
    K = A.shape[1]
    return 8 * K * 2.0 ** -53 * np.outer(np.abs(A).max(axis=1), np.abs(B).max(axis=1))


@pytest.mark.parametrize("M,N,K", [(1, 1, 1), (128, 64, 64), (130, 70, 33), (257, 200, 1000), (1000, 129, 513)])
def test_ozaki_gemm_within_its_bound(cuda, M, N, K):
    rng = np.random.default_rng(M + 7 * N + K)
    A = rng.standard_normal((M, K))
    B = rng.standard_normal((N, K))
    C = ozaki(A, B, cuda)
    exact = A @ B.T
    assert np.all(np.abs(C - exact) <= bound(A, B) + 1e-300)
    # and close to FP64 in the usual sense
    assert np.abs(C - exact).max() <= 1e-14 * np.abs(A).max() * np.abs(B).max() * K


@pytest.mark.parametrize("S", [4, 5, 6, 7])
@pytest.mark.parametrize("M,N,K", [(130, 70, 33), (257, 200, 1000), (1000, 250, 513)])
def test_ozaki_gemm_fewer_slices_within_their_bound(cuda, S, M, N, K):
    """4-7 slices (tiles of 128, 96, 80 and 64 columns): within the bound of S slices, ragged tile
    edges included; each slice more is more accurate."""
    rng = np.random.default_rng(M + 7 * N + K + S)
    A = rng.standard_normal((M, K)) * np.exp2(rng.integers(-20, 20, size=(M, 1)))
    B = rng.standard_normal((N, K))
    C = ozaki(A, B, cuda, S)
    exact = A @ B.T
    assert np.all(np.abs(C - exact) <= bound_slices(A, B, S) + 1e-300)
    if S < 7:
        C2 = ozaki(A, B, cuda, S + 1)
        assert np.abs(C2 - exact).max() < np.abs(C - exact).max()


def test_ozaki_gemm_graded_rows(cuda):
    """Rows and columns spanning 2^-40 .. 2^40 and zero rows: the per-row exponents carry the scale."""
    rng = np.random.default_rng(5)
    M, N, K = 300, 160, 700
    A = rng.standard_normal((M, K)) * np.exp2(rng.integers(-40, 40, size=(M, 1)))
    B = rng.standard_normal((N, K)) * np.exp2(rng.integers(-40, 40, size=(N, 1)))
    A[7] = 0.0
    B[3] = 0.0
    C = ozaki(A, B, cuda)
    exact = A @ B.T
    assert np.all(np.abs(C - exact) <= bound(A, B) + 1e-300)
    assert np.all(C[7] == 0.0) and np.all(C[:, 3] == 0.0)


def test_ozaki_rejects_bad_arguments(cuda):
    z = torch.zeros(64, dtype=torch.float64, device=cuda)
    rc = step.lib().bgpu_gemm_ozaki(4, 4, 4, z.data_ptr(), 4, z.data_ptr(), 4, z.data_ptr(), 4, z.data_ptr(), 8, None)
    assert rc == -2   # workspace too small


@pytest.mark.parametrize("kw,chunk", [(dict(n=60, m=200, density=0.05, seed=2), 32),
                                      (dict(n=100, m=300, density=0.02, seed=3), 64)])
def test_schur_ozaki_matches_fp64(cuda, kw, chunk):
    """The Schur complement with the Ozaki products (precision 2) against the FP64 one, with an ill-
    conditioned Z^-1 (condition 1e8) as late in a solve."""
    d = problems.random_sdp(**kw)
    S, n, a = block_arrays(d, cuda)
    u = upper_arrays(a, n, cuda)
    X = spd(n, 5, cond=1e8)
    Zi = spd(n, 6, cond=1e8)
    dX, dZi = colmajor(X, cuda), colmajor(Zi, cuda)
    got = []
    for prec in (0, 2):
        M = torch.zeros(d.m * d.m, dtype=torch.float64, device=cuda)
        ws = torch.empty(step.ws_bytes(n, chunk, prec), dtype=torch.uint8, device=cuda)
        step.call("schur_assemble_sym", n, d.m, int(a["con"].numel()), a["con"].data_ptr(), a["cptr"].data_ptr(),
                  a["ccol"].data_ptr(), a["cpos"].data_ptr(), a["cval"].data_ptr(), u["uptr"].data_ptr(),
                  u["upos"].data_ptr(), u["uval"].data_ptr(), dX.data_ptr(), dZi.data_ptr(), M.data_ptr(), prec,
                  chunk, ws.data_ptr(), ws.numel(), None)
        step.call("sync", None)
        got.append(M.cpu().numpy().reshape(d.m, d.m).T)
    assert np.abs(got[1] - got[0]).max() <= 1e-13 * np.abs(got[0]).max()


@pytest.mark.parametrize("S,tol", [(6, 1e-9), (5, 1e-7)])
def test_schur_ozaki_fewer_slices(cuda, S, tol):
    """The assembly with S slices (precision (S << 8) | 2), the mixed path's preconditioner-grade late
    form, against the FP64 one: within tol of the largest entry, and 6 slices closer than 5."""
    d = problems.random_sdp(n=100, m=300, density=0.02, seed=3)
    S_, n, a = block_arrays(d, cuda)
    u = upper_arrays(a, n, cuda)
    X = spd(n, 5, cond=1e6)
    Zi = spd(n, 6, cond=1e6)
    dX, dZi = colmajor(X, cuda), colmajor(Zi, cuda)
    got = []
    for prec in (0, (S << 8) | 2):
        M = torch.zeros(d.m * d.m, dtype=torch.float64, device=cuda)
        ws = torch.empty(step.ws_bytes(n, 64, prec), dtype=torch.uint8, device=cuda)
        step.call("schur_assemble_sym", n, d.m, int(a["con"].numel()), a["con"].data_ptr(), a["cptr"].data_ptr(),
                  a["ccol"].data_ptr(), a["cpos"].data_ptr(), a["cval"].data_ptr(), u["uptr"].data_ptr(),
                  u["upos"].data_ptr(), u["uval"].data_ptr(), dX.data_ptr(), dZi.data_ptr(), M.data_ptr(), prec,
                  64, ws.data_ptr(), ws.numel(), None)
        step.call("sync", None)
        got.append(M.cpu().numpy().reshape(d.m, d.m).T)
    err = np.abs(got[1] - got[0]).max() / np.abs(got[0]).max()
    assert err <= tol, err
    assert np.abs(got[1] - got[1].T).max() == 0.0   # written in full, symmetric


def check(res, ref):
    assert res.status_str == ref["status"], res.log
    objectives_close(res.pobj, res.dobj, ref["pobj"], ref["dobj"], each=res.iterations == ref["iterations"])
    assert np.max(np.abs(res.dimacs)) <= 1e-7, res.dimacs


def make(entry):
    return getattr(problems, entry["generator"])(**entry["kwargs"])


@pytest.mark.parametrize("name", ["rand60", "rand100"])
def test_ozaki_solve_matches_reference(golden, name):
    e = golden[name]
    res = brisk_b200.solve_sdpa(*make(e).args(), options=["-nohsd", "-dir", "hkm", "-mixed", "0", "-tol", "1e-7",
                                                          "-asmprec", "ozaki"], verbose=False)
    check(res, e["runs"]["default"])
    assert abs(res.iterations - e["runs"]["default"]["iterations"]) <= 1


@pytest.mark.parametrize("late", ["ozaki6", "ozaki5"])
def test_mixed_path_with_preconditioner_grade_late_iterations(golden, late):
    """rand400 on the 3xTF32 path with late iterations assembled with 6 or 5 Ozaki slices (an M
    that only preconditions; PCG residuals with the FP64 operator): the reference's solution."""
    e = golden["rand400"]
    res = brisk_b200.solve_sdpa(*make(e).args(), options=["-nohsd", "-dir", "hkm", "-tol", "1e-7", "-asmprec", "tf32x3",
                                                          "-asmlate", late, "-v", "-v"], verbose=False)
    check(res, e["runs"]["default"])
    assert abs(res.iterations - e["runs"]["default"]["iterations"]) <= 1


def test_mixed_path_with_ozaki_late_iterations(golden):
    """rand400 on the 3xTF32 path: the late iterations assemble with the Ozaki products and the solve
    reaches the reference's solution."""
    e = golden["rand400"]
    res = brisk_b200.solve_sdpa(*make(e).args(), options=["-nohsd", "-dir", "hkm", "-tol", "1e-7", "-asmprec", "tf32x3",
                                                          "-asmlate", "ozaki", "-v", "-v"], verbose=False)
    check(res, e["runs"]["default"])
