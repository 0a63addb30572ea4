"""ctypes binding of libbrisk's flat C interface, B200 build (include/brisk.h).

The functions mirror the reference's Python binding (python/brisk/_core.py): the same names
(``load_library``, ``version``, ``solve_sdpa``, ``solve_file``, ``options_to_argv``), the same
argument meaning, the same ``Result`` fields and the same errors for bad input.  The library is
the in-tree ``brisk_b200/libbrisk.so`` (built by ``brisk_b200.build``); there is no fallback: if
it is missing, loading raises.

Conventions (brisk.h): the problem is the numbers of an SDPA sparse file; BRISK solves
(P) min <C,X> s.t. <A_i,X> = b_i, X >= 0 and (D) max b'y s.t. C - sum y_i A_i = Z >= 0 with
C = -F0, A_i = F_i, b = c.
"""
from __future__ import annotations

import ctypes
import os
import sys
import threading
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

STATUS = {0: "OPTIMAL", 1: "PRIMAL INFEASIBLE", 2: "DUAL INFEASIBLE", 3: "ITERATION LIMIT",
          4: "NUMERICAL DIFFICULTIES", 5: "REDUCED ACCURACY", 6: "TIME LIMIT", -1: "NOT SOLVED"}

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None
_lib_path = None
_lock = threading.Lock()           # libbrisk is not reentrant: one solve at a time per process
_PRINT = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_char_p, ctypes.c_int)


def _default_path():
    p = os.environ.get("BRISK_B200_LIBRARY", "")
    return p or os.path.join(HERE, "libbrisk.so")


def load_library(path=None):
    """Load the in-tree libbrisk.so (B200 build).  Raises OSError when it is missing."""
    global _lib, _lib_path
    if _lib is not None and (path is None or os.path.abspath(path) == _lib_path):
        return _lib
    path = os.path.abspath(path or _default_path())
    if not os.path.exists(path):
        raise OSError(f"libbrisk (B200 build) not found at {path}: run `python -m brisk_b200.build` "
                      "(or __graft_entry__.build()) first")
    L = ctypes.CDLL(path, mode=os.RTLD_LOCAL)
    P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    pd = ctypes.POINTER(ctypes.c_double)
    pi = ctypes.POINTER(ctypes.c_int)
    ppc = ctypes.POINTER(ctypes.c_char_p)
    L.brisk_version.restype = ctypes.c_char_p
    L.brisk_set_output.argtypes = [I, _PRINT]
    L.brisk_set_output.restype = None
    L.brisk_result_new.restype = P
    L.brisk_result_delete.argtypes = [P]
    L.brisk_result_delete.restype = None
    for name, rt in (("status", I), ("exit_code", I), ("iterations", I), ("m", I), ("nblk", I),
                     ("have_x", I), ("pobj", D), ("dobj", D), ("time", D)):
        f = getattr(L, "brisk_result_" + name)
        f.argtypes, f.restype = [P], rt
    L.brisk_result_status_str.argtypes, L.brisk_result_status_str.restype = [P], ctypes.c_char_p
    L.brisk_result_blocksize.argtypes, L.brisk_result_blocksize.restype = [P, I], I
    L.brisk_result_dimacs.argtypes, L.brisk_result_dimacs.restype = [P, pd], None
    L.brisk_result_y.argtypes, L.brisk_result_y.restype = [P], pd
    L.brisk_result_X.argtypes, L.brisk_result_X.restype = [P, I], pd
    L.brisk_result_Z.argtypes, L.brisk_result_Z.restype = [P, I], pd
    L.brisk_solve_data.argtypes = [I, I, pi, pd, ctypes.c_int64, pi, pi, pi, pi, pd, I, ppc, P]
    L.brisk_solve_data.restype = I
    L.brisk_solve_file.argtypes = [ctypes.c_char_p, I, ppc, P]
    L.brisk_solve_file.restype = I
    L.bgpu_batch_solve.argtypes = [I, pi, pi, pi, pd, ctypes.POINTER(ctypes.c_int64), pi, pi, pi, pi, pd, I, ppc, I,
                                   ctypes.POINTER(P), pi]
    L.bgpu_batch_solve.restype = I
    L.bgpu_sdpa_read.argtypes, L.bgpu_sdpa_read.restype = [ctypes.c_char_p, ctypes.POINTER(_SdpaArrays)], I
    L.bgpu_sdpa_free.argtypes, L.bgpu_sdpa_free.restype = [ctypes.POINTER(_SdpaArrays)], None
    L.brisk_interrupt.argtypes, L.brisk_interrupt.restype = [], None
    L.brisk_interrupted.argtypes, L.brisk_interrupted.restype = [], I
    _lib, _lib_path = L, path
    return L


def library_path():
    load_library()
    return _lib_path


def version():
    return load_library().brisk_version().decode()


@dataclass
class Result:
    """The solution of the problem as given (the reference's Result, python/brisk/_core.py:180)."""
    status: int
    status_str: str
    exit_code: int
    iterations: int
    pobj: float                      # <C,X>
    dobj: float                      # b'y
    time: float
    dimacs: np.ndarray
    blocksizes: List[int] = field(default_factory=list)
    y: Optional[np.ndarray] = None
    X: Optional[List[np.ndarray]] = None
    Z: Optional[List[np.ndarray]] = None
    log: str = ""

    @property
    def x(self):
        return None if self.y is None else -self.y


def _ints(x, what):
    a = np.atleast_1d(np.asarray(x)).ravel()
    if a.size == 0:
        return np.zeros(0, dtype=np.intc)
    if a.dtype == bool or np.iscomplexobj(a) or a.dtype == object:
        raise ValueError("%s: integers expected" % what)
    if not np.issubdtype(a.dtype, np.integer):
        a = a.astype(np.float64)
        if not np.all(np.isfinite(a)) or np.any(a != np.floor(a)):
            raise ValueError("%s: integers expected (a value is not a whole number)" % what)
    lo, hi = np.iinfo(np.intc).min, np.iinfo(np.intc).max
    if np.any(a > hi) or np.any(a < lo):
        raise ValueError("%s: a value is out of range" % what)
    return np.ascontiguousarray(a, dtype=np.intc)


def _finite(x, what):
    a = np.ascontiguousarray(x, dtype=np.float64)
    if not np.all(np.isfinite(a)):
        raise ValueError("%s: a value is not finite (NaN or infinity)" % what)
    return a


def options_to_argv(options):
    """Command-line options from a dict, a list of strings or a string (as the reference)."""
    if options is None:
        return []
    if isinstance(options, str):
        return options.split()
    if isinstance(options, dict):
        av = []
        for k, v in options.items():
            if v is None or v is False:
                continue
            k = str(k)
            av.append(k if k.startswith("-") else "-" + k.replace("_", "-"))
            if v is not True:
                av.append(repr(v) if isinstance(v, float) else str(v))
        return av
    return [str(o) for o in options]


def _collect(L, r, rc, log):
    nblk = L.brisk_result_nblk(r)
    bsz = [L.brisk_result_blocksize(r, k) for k in range(nblk)]
    err = (ctypes.c_double * 6)()
    L.brisk_result_dimacs(r, err)
    m = L.brisk_result_m(r)
    yp = L.brisk_result_y(r)
    y = np.ctypeslib.as_array(yp, shape=(m,)).copy() if yp and m > 0 else None
    X = Z = None
    if L.brisk_result_have_x(r):
        X, Z = [], []
        for k, n in enumerate(bsz):
            xp, zp = L.brisk_result_X(r, k), L.brisk_result_Z(r, k)
            if n < 0:   # an LP block: its vector of -n values
                X.append(np.ctypeslib.as_array(xp, shape=(-n,)).copy() if xp else None)
                Z.append(np.ctypeslib.as_array(zp, shape=(-n,)).copy() if zp else None)
                continue
            shape = (n, n)
            X.append(np.ctypeslib.as_array(xp, shape=shape).T.copy() if xp else None)
            Z.append(np.ctypeslib.as_array(zp, shape=shape).T.copy() if zp else None)
    return Result(status=L.brisk_result_status(r), status_str=L.brisk_result_status_str(r).decode(),
                  exit_code=rc, iterations=L.brisk_result_iterations(r), pobj=L.brisk_result_pobj(r),
                  dobj=L.brisk_result_dobj(r), time=L.brisk_result_time(r), dimacs=np.array(err[:]),
                  blocksizes=bsz, y=y, X=X, Z=Z, log=log)


def _run(call, options, verbose):
    L = load_library()
    av = options_to_argv(options)
    arr = (ctypes.c_char_p * max(len(av), 1))(*[a.encode() for a in av])
    chunks = []

    def cb(s, is_err):
        txt = s.decode(errors="replace")
        chunks.append(txt)
        if verbose or is_err:
            (sys.stderr if is_err else sys.stdout).write(txt)
        return 0

    cbf = _PRINT(cb)
    with _lock:
        L.brisk_set_output(2, cbf)
        r = L.brisk_result_new()
        try:
            rc = call(L, len(av), arr, r)
            if rc < 0:
                raise RuntimeError(f"brisk: the solve was aborted (code {rc}):\n" + "".join(chunks))
            return _collect(L, r, rc, "".join(chunks))
        finally:
            L.brisk_result_delete(r)
            L.brisk_set_output(0, _PRINT(0))


def solve_sdpa(blocksizes, c, mat, blk, i, j, v, options=None, verbose=True):
    """Solve the SDPA problem given by its numbers: blocksizes, c (m), and the entries
    mat (0..m), blk (1..nblk), i, j (1-based within the block; i > j is swapped), v."""
    bs = _ints(blocksizes, "blocksizes")
    c = _finite(c, "c")
    arrs = [_ints(a, nm) for a, nm in ((mat, "mat"), (blk, "blk"), (i, "i"), (j, "j"))]
    v = _finite(v, "v")
    nnz = v.size
    if any(a.size != nnz for a in arrs):
        raise ValueError("mat, blk, i, j and v must have the same length")
    pi = ctypes.POINTER(ctypes.c_int)
    pd = ctypes.POINTER(ctypes.c_double)
    P = lambda a, t: a.ctypes.data_as(t)   # noqa: E731
    return _run(lambda L, n, a, r: L.brisk_solve_data(
        int(c.size), int(bs.size), P(bs, pi), P(c, pd), nnz, P(arrs[0], pi), P(arrs[1], pi),
        P(arrs[2], pi), P(arrs[3], pi), P(v, pd), n, a, r), options, verbose)


class _SdpaArrays(ctypes.Structure):
    """struct bgpu_sdpa (include/bgpu.h)."""
    _fields_ = [("m", ctypes.c_int), ("nblk", ctypes.c_int), ("nnz", ctypes.c_int64),
                ("bs", ctypes.POINTER(ctypes.c_int)), ("c", ctypes.POINTER(ctypes.c_double)),
                ("mat", ctypes.POINTER(ctypes.c_int)), ("blk", ctypes.POINTER(ctypes.c_int)),
                ("i", ctypes.POINTER(ctypes.c_int)), ("j", ctypes.POINTER(ctypes.c_int)),
                ("v", ctypes.POINTER(ctypes.c_double)), ("owner", ctypes.c_void_p)]


def read_sdpa_file(path, verbose=False):
    """Read an SDPA sparse file with the library's reader (bgpu_sdpa_read, the reader of
    brisk_solve_file).  Returns (SdpaData, log); raises ValueError with the reader's message when
    the file cannot be read or is malformed."""
    from .problems import SdpaData
    L = load_library()
    chunks = []

    def cb(s, is_err):
        txt = s.decode(errors="replace")
        chunks.append(txt)
        if verbose:
            sys.stderr.write(txt)
        return 0

    cbf = _PRINT(cb)
    out = _SdpaArrays()
    with _lock:
        L.brisk_set_output(2, cbf)
        try:
            rc = L.bgpu_sdpa_read(os.fsencode(path), ctypes.byref(out))
            if rc != 0:
                raise ValueError("".join(chunks).strip() or f"bgpu_sdpa_read returned {rc}")
            try:
                def arr(ptr, n, dt):
                    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt, copy=True) if n else np.zeros(0, dt)
                nnz = int(out.nnz)
                d = SdpaData(bs=arr(out.bs, out.nblk, np.int32), c=arr(out.c, out.m, np.float64),
                             mat=arr(out.mat, nnz, np.int32), blk=arr(out.blk, nnz, np.int32),
                             i=arr(out.i, nnz, np.int32), j=arr(out.j, nnz, np.int32),
                             v=arr(out.v, nnz, np.float64), name=os.path.basename(os.fsdecode(path)))
            finally:
                L.bgpu_sdpa_free(ctypes.byref(out))
        finally:
            L.brisk_set_output(0, _PRINT(0))
    return d, "".join(chunks)


def solve_file(path, options=None, verbose=True):
    """Solve an SDPA sparse file."""
    return _run(lambda L, n, a, r: L.brisk_solve_file(os.fsencode(path), n, a, r), options, verbose)


def solve_batch_arrays(m, nblk, bs, c, nnz, mat, blk, i, j, v, options=None, workers=0):
    """Solve independent problems given as concatenated brisk_solve_data arrays (problem p: m[p]
    constraints, nblk[p] block sizes, nnz[p] entries, in problem order) with one call of
    bgpu_batch_solve.  Returns the list of Results (no log: the batch runs quiet)."""
    L = load_library()
    m, nblk, bs = _ints(m, "m"), _ints(nblk, "nblk"), _ints(bs, "bs")
    nnz = np.ascontiguousarray(nnz, dtype=np.int64)
    count = int(m.size)
    if nblk.size != count or nnz.size != count:
        raise ValueError("m, nblk and nnz must have one entry per problem")
    if int(nblk.sum()) != bs.size or int(m.sum()) != np.asarray(c).size:
        raise ValueError("bs and c must hold the block sizes and right-hand sides of every problem")
    c = _finite(c, "c")
    arrs = [np.ascontiguousarray(a, dtype=np.intc) for a in (mat, blk, i, j)]
    v = np.ascontiguousarray(v, dtype=np.float64)
    if any(a.size != int(nnz.sum()) for a in arrs) or v.size != int(nnz.sum()):
        raise ValueError("mat, blk, i, j and v must hold the entries of every problem")
    av = options_to_argv(options)
    arr = (ctypes.c_char_p * max(len(av), 1))(*[a.encode() for a in av])
    pi = ctypes.POINTER(ctypes.c_int)
    pd = ctypes.POINTER(ctypes.c_double)
    P = lambda a, t: a.ctypes.data_as(t)   # noqa: E731
    with _lock:
        L.brisk_set_output(1, _PRINT(0))
        handles = (ctypes.c_void_p * max(count, 1))(*[L.brisk_result_new() for _ in range(count)])
        rcs = np.zeros(max(count, 1), dtype=np.intc)
        try:
            rc = L.bgpu_batch_solve(count, P(m, pi), P(nblk, pi), P(bs, pi), P(c, pd),
                                    nnz.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), P(arrs[0], pi),
                                    P(arrs[1], pi), P(arrs[2], pi), P(arrs[3], pi), P(v, pd), len(av), arr,
                                    int(workers), handles, P(rcs, pi))
            if rc != 0:
                raise RuntimeError(f"brisk: bgpu_batch_solve returned {rc}")
            return [_collect(L, handles[p], int(rcs[p]), "") for p in range(count)]
        finally:
            for p in range(count):
                L.brisk_result_delete(handles[p])
            L.brisk_set_output(0, _PRINT(0))


class BatchSession:
    """A batch of one-block problems (order <= 64) kept resident in device memory
    (bgpu_batch_create / bgpu_batch_run): build once, solve many times."""

    def __init__(self, m, nblk, bs, c, nnz, mat, blk, i, j, v, options=None):
        L = load_library()
        L.bgpu_batch_create.restype = ctypes.c_void_p
        L.bgpu_batch_create.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 10 + [ctypes.c_int, ctypes.c_void_p,
                                                                                 ctypes.c_void_p]
        L.bgpu_batch_run.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.bgpu_batch_run.restype = ctypes.c_int
        L.bgpu_batch_destroy.argtypes = [ctypes.c_void_p]
        L.bgpu_batch_destroy.restype = None
        self._keep = [np.ascontiguousarray(a, dtype=t) for a, t in
                      ((m, np.intc), (nblk, np.intc), (bs, np.intc), (c, np.float64), (nnz, np.int64),
                       (mat, np.intc), (blk, np.intc), (i, np.intc), (j, np.intc), (v, np.float64))]
        self.count = int(self._keep[0].size)
        av = options_to_argv(options)
        arr = (ctypes.c_char_p * max(len(av), 1))(*[a.encode() for a in av])
        rc = ctypes.c_int(0)
        with _lock:
            L.brisk_set_output(1, _PRINT(0))
            self.h = L.bgpu_batch_create(self.count, *[a.ctypes.data for a in self._keep], len(av), arr,
                                         ctypes.addressof(rc))
            L.brisk_set_output(0, _PRINT(0))
        if not self.h:
            raise RuntimeError(f"brisk: bgpu_batch_create failed ({rc.value})")

    def run(self, collect=True):
        """Solve every problem; the list of Results (or, collect=False, the exit codes only)."""
        L = load_library()
        handles = (ctypes.c_void_p * self.count)(*[L.brisk_result_new() for _ in range(self.count)])
        rcs = np.zeros(self.count, dtype=np.intc)
        try:
            with _lock:
                L.brisk_set_output(1, _PRINT(0))
                rc = L.bgpu_batch_run(self.h, handles, rcs.ctypes.data)
                L.brisk_set_output(0, _PRINT(0))
            if rc != 0:
                raise RuntimeError(f"brisk: bgpu_batch_run returned {rc}")
            if not collect:
                return rcs.copy()
            return [_collect(L, handles[p], int(rcs[p]), "") for p in range(self.count)]
        finally:
            for p in range(self.count):
                L.brisk_result_delete(handles[p])

    def close(self):
        if getattr(self, "h", None):
            load_library().bgpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def concat_problems(problems):
    """The concatenated arrays of solve_batch_arrays for objects with the fields bs, c, mat,
    blk, i, j, v (brisk_b200.problems.SdpaData)."""
    cat = lambda k, t: np.concatenate([np.asarray(getattr(d, k), dtype=t) for d in problems])  # noqa: E731
    return dict(m=np.array([len(d.c) for d in problems], np.intc),
                nblk=np.array([len(d.bs) for d in problems], np.intc),
                bs=cat("bs", np.intc), c=cat("c", np.float64),
                nnz=np.array([len(d.v) for d in problems], np.int64),
                mat=cat("mat", np.intc), blk=cat("blk", np.intc), i=cat("i", np.intc), j=cat("j", np.intc),
                v=cat("v", np.float64))


def solve_batch(problems, options=None, workers=0):
    """Solve a list of problems (SdpaData-like objects) with one bgpu_batch_solve call."""
    return solve_batch_arrays(**concat_problems(problems), options=options, workers=workers)


def interrupt():
    load_library().brisk_interrupt()
