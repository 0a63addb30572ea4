"""ctypes binding of the step-level C ABI (include/bgpu.h) for callers holding device memory.

Device buffers are passed as integer addresses (``torch.Tensor.data_ptr()`` in the tests and the
benchmark; PyTorch only allocates).  Every call checks the returned status and raises
``BgpuError`` on failure; nothing falls back to the CPU.
"""
from __future__ import annotations

import ctypes

from ._core import load_library

STATUS = {0: "OK", -1: "CUDA error", -2: "bad argument", -3: "not positive definite", -4: "device wait timed out",
          -5: "out of device memory", -6: "unsupported", -7: "size above the maximum"}


class BgpuError(RuntimeError):
    def __init__(self, name, rc):
        super().__init__(f"{name} failed: {STATUS.get(rc, rc)} ({rc})")
        self.rc = rc


_sig_done = False


def lib():
    global _sig_done
    L = load_library()
    if _sig_done:
        return L
    P, I, D, I64, SZ = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int64, ctypes.c_size_t
    sigs = {
        "bgpu_sync": ([P], I),
        "bgpu_schur_ws_bytes": ([I, I, I], SZ),
        "bgpu_schur_chunk_default": ([I, I], I),
        "bgpu_schur_colptr": ([I, I, P, P, P, P], I),
        "bgpu_schur_assemble": ([I, I, I, P, P, P, P, P, P, P, P, I, I, P, SZ, P], I),
        "bgpu_schur_upper": ([I, I, P, P, P, P, P, P, P, P, P], I),
        "bgpu_schur_assemble_sym": ([I, I, I, P, P, P, P, P, P, P, P, P, P, P, I, I, P, SZ, P], I),
        "bgpu_schur_gram": ([I, I, I, P, P, P, P, P, P, SZ, P], I),
        "bgpu_schur_dense_ws_bytes": ([I, I, I, I], SZ),
        "bgpu_schol_analyze": ([I, I, P, P, P], P),
        "bgpu_schol_info": ([P, P], I),
        "bgpu_schol_perm": ([P, P], I),
        "bgpu_schol_supernodes": ([P, P, P, P, P], I),
        "bgpu_schol_factor": ([P, P, I64, P, D, P, P, P], I),
        "bgpu_schol_factor_f32": ([P, P, I64, P, D, P, P, P], I),
        "bgpu_schol_solve": ([P, P, P, P], I),
        "bgpu_schol_destroy": ([P], None),
        "bgpu_schol_set_delta": ([D], None),
        "bgpu_schur_densify": ([I, I, P, P, P, P, P], I),
        "bgpu_schur_assemble_dense": ([I, I, I, P, P, P, P, P, P, P, P, P, I, I, P, SZ, P], I),
        "bgpu_schur_lp": ([I, I, I, I64, P, P, P, P, P, P, P, P, P, P, P], I),
        "bgpu_lowrank_factor": ([I, I, P, P, P, I, P, P, P], I),
        "bgpu_schur_lowrank": ([I, I, I, P, P, P, P, P, P, P, P, P], I),
        "bgpu_potrf": ([I, P, I, P, P, P, P], I),
        "bgpu_potrf_f32": ([I, P, I, P, P, P, P], I),
        "bgpu_trsv": ([I, P, I, P, P, I, P, I, P, P], I),
        "bgpu_trsv_f32": ([I, P, I, P, P, I, P, I, P, P], I),
        "bgpu_trsv_noalloc": ([I, P, I, P, P, I, P], I),
        "bgpu_trtri": ([I, P, I, P, P, I, P], I),
        "bgpu_dgemm": ([I, I, I, I, I, D, P, I64, P, I64, D, P, I64, I, P], I),
        "bgpu_gemm_tf32x3": ([I, I, I, P, P, I64, P, P, I64, P, I64, P], I),
        "bgpu_split_tf32": ([I64, P, P, P, P], I),
        "bgpu_symv": ([I, D, P, I, P, D, P, P], I),
        "bgpu_aop": ([I, I, P, P, P, P, P, D, D, P, P], I),
        "bgpu_small_chol_inv": ([I, P, P, P, P, P, P], I),
        "bgpu_small_lammin": ([I, P, P, P, P, P], I),
        "bgpu_small_gemm": ([I, P, I, I, D, P, P, D, P, I, P], I),
        "bgpu_nt_ws_bytes": ([I], SZ),
        "bgpu_ozaki_ws_bytes": ([I, I, I], SZ),
        "bgpu_gemm_ozaki": ([I, I, I, P, I64, P, I64, P, I64, P, SZ, P], I),
        "bgpu_gemm_ozaki_slices": ([I, I, I, I, P, I64, P, I64, P, I64, P, SZ, P], I),
        "bgpu_nt_scaling": ([I, P, P, P, P, P, P, SZ, P, P], I),
    }
    for name, (args, res) in sigs.items():
        f = getattr(L, name)
        f.argtypes, f.restype = args, res
    L.bgpu_version.restype = ctypes.c_char_p
    _sig_done = True
    return L


def call(name, *args):
    """Call bgpu_<name>(*args) and raise BgpuError on a nonzero status."""
    rc = getattr(lib(), "bgpu_" + name)(*args)
    if rc != 0:
        raise BgpuError(name, rc)
    return rc


def ws_bytes(n, chunk, precision):
    return int(lib().bgpu_schur_ws_bytes(n, chunk, precision))


def chunk_default(n, precision):
    return int(lib().bgpu_schur_chunk_default(n, precision))


def nt_scaling(LX, LZ, stream=None):
    """The NT scaling of one block from the Cholesky factors of X and Z (CUDA float64 tensors, n x n,
    lower triangles read as column-major, i.e. the tensors hold the transposes row-major):
    returns (G, lam, W, sweeps) with G, W column-major in row-major tensors (transpose to read)."""
    import torch
    n = LX.shape[0]
    dev = LX.device
    G = torch.empty((n, n), dtype=torch.float64, device=dev)
    W = torch.empty((n, n), dtype=torch.float64, device=dev)
    lam = torch.empty(n, dtype=torch.float64, device=dev)
    nws = int(lib().bgpu_nt_ws_bytes(n))
    ws = torch.empty(max(nws, 8), dtype=torch.uint8, device=dev)
    sw = ctypes.c_int(0)
    call("nt_scaling", n, LX.data_ptr(), LZ.data_ptr(), G.data_ptr(), lam.data_ptr(), W.data_ptr(), ws.data_ptr(),
         nws, ctypes.byref(sw), stream)
    return G, lam, W, sw.value


class SparseCholesky:
    """Handle of bgpu_schol_analyze (the symbolic phase runs on the host, no GPU needed)."""

    def __init__(self, m, cliques):
        import numpy as np
        L = lib()
        ptr = np.zeros(len(cliques) + 1, dtype=np.int64)
        for c, cl in enumerate(cliques):
            ptr[c + 1] = ptr[c] + len(cl)
        idx = np.ascontiguousarray(np.concatenate([np.asarray(c, dtype=np.int32) for c in cliques])
                                   if cliques else np.zeros(1, np.int32), dtype=np.int32)
        rc = ctypes.c_int(0)
        self.h = L.bgpu_schol_analyze(int(m), len(cliques), ptr.ctypes.data, idx.ctypes.data, ctypes.addressof(rc))
        if not self.h:
            raise BgpuError("schol_analyze", rc.value)
        self.m = int(m)

    def info(self):
        import numpy as np
        out = np.zeros(8)
        call("schol_info", self.h, out.ctypes.data)
        keys = ("nsup", "nnz", "flops", "fmax", "levels", "pattern", "m", "bytes")
        return dict(zip(keys, out.tolist()))

    def perm(self):
        import numpy as np
        p = np.zeros(self.m, dtype=np.int32)
        call("schol_perm", self.h, p.ctypes.data)
        return p

    def supernodes(self):
        """(sfirst, parent, rptr, rows) as numpy arrays."""
        import numpy as np
        ns = int(self.info()["nsup"])
        sfirst = np.zeros(ns + 1, np.int32)
        parent = np.zeros(max(ns, 1), np.int32)
        rptr = np.zeros(ns + 1, np.int64)
        call("schol_supernodes", self.h, sfirst.ctypes.data, parent.ctypes.data, rptr.ctypes.data, None)
        rows = np.zeros(max(int(rptr[-1]), 1), np.int32)
        call("schol_supernodes", self.h, None, None, None, rows.ctypes.data)
        return sfirst, parent[:ns], rptr, rows[:int(rptr[-1])]

    def close(self):
        if self.h:
            lib().bgpu_schol_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
