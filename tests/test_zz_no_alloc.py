"""bgpu_trsv_noalloc: the triangular solve for callers that cannot allocate device memory where
they solve (between loop steps where cudaMalloc/cudaFree would synchronize the device, or under
another allocator that owns the device memory).  Its flags live in the library's static device
array; its results must equal bgpu_trsv's, which takes caller-allocated flags, on two calls in a
row (the second call reuses the array the first one left behind).

This file is collected last (tests/test_zz_*), so a run that stops at the first failure has
run every other test before it; it also passes alone in a fresh process."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from brisk_b200 import step  # noqa: E402


def spd(n, seed):
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    return (Q * np.logspace(0, 3, n)) @ Q.T


@pytest.mark.parametrize("n", [200, 777])
def test_trsv_noalloc_matches_trsv_twice(n):
    cuda = torch.device("cuda:0")
    A = spd(n, n)
    L = torch.as_tensor(np.ascontiguousarray(A.T), device=cuda).contiguous()   # column-major
    nb = (n + 63) // 64
    dinv = torch.zeros(nb * 4096, dtype=torch.float64, device=cuda)
    info = torch.zeros(1, dtype=torch.int32, device=cuda)
    pmin = torch.zeros(1, dtype=torch.float64, device=cuda)
    step.call("potrf", n, L.data_ptr(), n, dinv.data_ptr(), info.data_ptr(), pmin.data_ptr(), None)
    step.call("sync", None)
    assert int(info.item()) == 0
    flags = torch.zeros(nb, dtype=torch.int32, device=cuda)
    err = torch.zeros(1, dtype=torch.int32, device=cuda)
    rng = np.random.default_rng(n + 7)
    for call in range(2):                         # two calls in a row on the shared static array
        b = rng.standard_normal(n)
        x_ref = torch.as_tensor(b, device=cuda).clone()
        x_new = x_ref.clone()
        for trans in (0, 1):
            step.call("trsv", n, L.data_ptr(), n, dinv.data_ptr(), x_ref.data_ptr(), trans, flags.data_ptr(),
                      10 * (call + 1) + trans, err.data_ptr(), None)
            step.call("trsv_noalloc", n, L.data_ptr(), n, dinv.data_ptr(), x_new.data_ptr(), trans, None)
        step.call("sync", None)
        assert int(err.item()) == 0
        got, want = x_new.cpu().numpy(), x_ref.cpu().numpy()
        np.testing.assert_allclose(got, want, rtol=1e-13, atol=1e-13 * np.abs(want).max())
        np.testing.assert_allclose(got, np.linalg.solve(A, b), rtol=1e-8, atol=1e-10)


def test_trsv_noalloc_rejects_sizes_above_its_maximum(capfd):
    """The limit is the solve's own co-residency: one CTA of 256 threads (32 registers each) per
    block row of 64, all resident at once, 8 per SM.  One block row more is refused with
    BGPU_ERR_TOOBIG and a message that gives the limit, before anything is launched (the
    pointers below are never read)."""
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    cap = sms * 8
    for n in (64 * cap + 1, 64 * 4096 + 1):
        with pytest.raises(step.BgpuError) as e:
            step.call("trsv_noalloc", n, 1, n, 1, 1, 0, None)
        assert e.value.rc == -7
        err = capfd.readouterr().err
        assert f"n <= {64 * cap}" in err, err
