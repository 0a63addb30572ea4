"""The C-ABI library loads without a GPU and exports every function include/*.h declares."""
import ctypes
import os
import re

import numpy as np
import pytest
from refdir import REF_DIR

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in ("brisk.h", "bgpu.h"):
        with open(os.path.join(ROOT, "include", h)) as f:
            text = f.read()
        names |= set(re.findall(r"(?:BRISK_API|BGPU_API)[^;(]*?\b((?:brisk|bgpu)_\w+)\s*\(", text))
    return sorted(names)


def test_headers_declare_the_reference_interface():
    names = declared_symbols()
    for must in ("brisk_solve_data", "brisk_solve_file", "brisk_result_new", "brisk_result_delete",
                 "brisk_result_status", "brisk_result_dimacs", "brisk_result_y", "brisk_result_X",
                 "brisk_result_Z", "brisk_set_output", "brisk_version", "brisk_interrupt",
                 "bgpu_schur_assemble", "bgpu_potrf", "bgpu_trsv", "bgpu_dgemm", "bgpu_gemm_tf32x3"):
        assert must in names


def test_library_exports_every_declared_symbol(libpath):
    L = ctypes.CDLL(libpath, mode=os.RTLD_LOCAL)
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, missing


def test_version_and_result_handle_without_gpu(libpath):
    from brisk_b200 import _core
    L = _core.load_library(libpath)
    assert L.brisk_version().decode().startswith("1.7")
    r = L.brisk_result_new()
    assert L.brisk_result_status(r) == -1
    assert L.brisk_result_status_str(r).decode() == "NOT SOLVED"
    L.brisk_result_delete(r)


def test_bad_input_is_rejected_before_any_gpu_work(libpath):
    from brisk_b200 import _core
    with pytest.raises(ValueError):
        _core.solve_sdpa([3], [1.0], [1], [1], [1], [1], [np.nan], verbose=False)
    with pytest.raises(ValueError):
        _core.solve_sdpa([3], [1.0], [1, 1], [1], [1], [1], [1.0], verbose=False)
    # a bad option returns exit code 1 without touching the device
    res = _core.solve_sdpa([2], [1.0], [1], [1], [1], [1], [1.0], options=["-tol", "x"], verbose=False)
    assert res.exit_code == 1
    # an LP block takes diagonal entries only, and no block has size 0: input error 2
    res = _core.solve_sdpa([-2], [1.0], [1], [1], [1], [2], [1.0], verbose=False)
    assert res.exit_code == 2 and "off-diagonal entry in LP block" in res.log
    res = _core.solve_sdpa([2, 0], [1.0], [1], [1], [1], [1], [1.0], verbose=False)
    assert res.exit_code == 2


def test_options_to_argv_matches_reference_forms():
    from brisk_b200 import options_to_argv
    assert options_to_argv({"tol": 1e-7, "nohsd": True, "dir": "hkm", "x": None}) == ["-tol", "1e-07", "-nohsd", "-dir", "hkm"]
    assert options_to_argv("-tol 1e-7 -mixed 0") == ["-tol", "1e-7", "-mixed", "0"]
    assert options_to_argv(["-q"]) == ["-q"]


# The entry points the reference's ctypes loader (python/brisk/_core.py:61-102) binds without a
# hasattr guard: a drop-in must export every one of them.
REFERENCE_LOADER_SYMBOLS = [
    "brisk_version", "brisk_set_output", "brisk_result_new", "brisk_result_delete", "brisk_result_status",
    "brisk_result_exit_code", "brisk_result_iterations", "brisk_result_m", "brisk_result_nblk",
    "brisk_result_have_x", "brisk_result_pobj", "brisk_result_dobj", "brisk_result_time",
    "brisk_result_status_str", "brisk_result_blocksize", "brisk_result_dimacs", "brisk_result_y", "brisk_result_X",
    "brisk_result_Z", "brisk_solve_data", "brisk_solve_file", "brisk_result_bound", "brisk_result_resolves",
    "brisk_result_cause", "brisk_interrupt", "brisk_interrupted",
]


def test_exports_what_the_reference_loader_binds(libpath):
    L = ctypes.CDLL(libpath, mode=os.RTLD_LOCAL)
    assert [s for s in REFERENCE_LOADER_SYMBOLS if not hasattr(L, s)] == []


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF_DIR, "python", "brisk")), reason="reference tree absent")
def test_reference_python_package_loads_this_library(libpath, monkeypatch):
    """The reference's own binding loads libbrisk (B200 build) through BRISK_LIBRARY."""
    import importlib
    import sys
    monkeypatch.setenv("BRISK_LIBRARY", libpath)
    monkeypatch.syspath_prepend(os.path.join(REF_DIR, "python"))
    sys.modules.pop("brisk", None)
    sys.modules.pop("brisk._core", None)
    brisk = importlib.import_module("brisk")
    assert brisk.version().startswith("1.7")
    assert os.path.samefile(brisk.library_path(), libpath)
    sys.modules.pop("brisk", None)
    sys.modules.pop("brisk._core", None)


def test_batch_entry_checks_before_any_gpu_work(libpath):
    """bgpu_batch_solve: an empty batch returns nothing, mismatched arrays and bad options are
    rejected on the host."""
    import brisk_b200
    from brisk_b200 import problems
    assert brisk_b200.solve_batch_arrays([], [], [], [], [], [], [], [], [], []) == []
    arrs = brisk_b200.concat_problems([problems.batch_instance(5), problems.batch_instance(6)])
    bad = dict(arrs, v=arrs["v"][:-1])
    with pytest.raises(ValueError):
        brisk_b200.solve_batch_arrays(**bad)
    with pytest.raises(RuntimeError):
        brisk_b200.solve_batch_arrays(**arrs, options=["-tol", "abc"])
    assert int(arrs["nnz"].sum()) == arrs["v"].size and list(arrs["m"]) == [11, 15]


def _solve_data_raw(bs, c, mat, blk, i, j, v):
    """brisk_solve_data called straight through ctypes (no Python-side checks); returns the Result."""
    from brisk_b200 import _core
    bs = np.ascontiguousarray(bs, dtype=np.intc)
    c = np.ascontiguousarray(c, dtype=np.float64)
    arrs = [np.ascontiguousarray(a, dtype=np.intc) for a in (mat, blk, i, j)]
    v = np.ascontiguousarray(v, dtype=np.float64)
    pi, pd = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    return _core._run(lambda L, n, a, r: L.brisk_solve_data(
        int(c.size), int(bs.size), bs.ctypes.data_as(pi), c.ctypes.data_as(pd), int(v.size),
        arrs[0].ctypes.data_as(pi), arrs[1].ctypes.data_as(pi), arrs[2].ctypes.data_as(pi),
        arrs[3].ctypes.data_as(pi), v.ctypes.data_as(pd), n, a, r), None, False)


def test_solve_data_checks_entries_as_the_reference(libpath):
    """The checks of problem_from_sdpa_data (problem.c) in its order and with its messages, on the
    host before any GPU work: a value not finite (even where the indices are bad), c not finite,
    an index out of range ("bad entry" with the entry as given), an LP entry off the diagonal;
    exit code 2."""
    r = _solve_data_raw([3], [1.0], [1, 1], [1, 1], [1, 9], [1, 9], [1.0, np.nan])
    assert r.exit_code == 2 and "non-finite value in entry 1 1 9 9" in r.log
    r = _solve_data_raw([3], [np.inf], [1], [1], [1], [1], [1.0])
    assert r.exit_code == 2 and "non-finite value c[1]" in r.log
    r = _solve_data_raw([3], [1.0], [0, 1], [1, 1], [1, 4], [1, 1], [2.0, 1.0])
    assert r.exit_code == 2 and "bad entry 1 1 4 1" in r.log
    r = _solve_data_raw([3], [1.0], [2], [1], [1], [1], [1.0])
    assert r.exit_code == 2 and "bad entry 2 1 1 1" in r.log
    # zero values are no entries: not checked (the reference skips them before its range test)
    r = _solve_data_raw([3], [1.0], [7, 1], [5, 1], [0, 1], [0, 1], [0.0, np.nan])
    assert r.exit_code == 2 and "non-finite value in entry 1 1 1 1" in r.log
    r = _solve_data_raw([-2], [1.0], [1], [1], [1], [2], [1.0])
    assert r.exit_code == 2 and "off-diagonal entry in LP block" in r.log
    r = _solve_data_raw([], [1.0], [1], [1], [1], [1], [1.0])   # no block
    assert r.exit_code == 2 and "invalid problem data (m = 1, 0 blocks)" in r.log


def test_other_reference_options_take_their_values(libpath):
    """An option of the reference that this path does not use is passed over with its value (the
    next argument when it is no option: a word or a number such as -1), in one note; the options
    after it are still read (a bad -tol then stops the call with exit code 1 before any GPU work)."""
    from brisk_b200 import _core
    res = _core.solve_sdpa([2], [1.0], [1], [1], [1], [1], [1.0],
                           options=["-freeelim", "0", "-lpmethod", "-1", "-lralm", "yes", "-nosuchflag", "-tol", "x"],
                           verbose=False)
    assert res.exit_code == 1
    assert "option -freeelim 0 is not used" in res.log
    assert "option -lpmethod -1 is not used" in res.log
    assert "option -lralm yes is not used" in res.log
    assert "option -nosuchflag is not used" in res.log
    assert "option 0 " not in res.log and "option yes" not in res.log
    assert "bad -tol" in res.log


def test_options_that_change_the_method_are_noted(libpath):
    """The reference's options that ask for another method or a presolve this build does not run
    print a note naming what is not applied; the values that turn those presolves off are silent.
    -hsd (a flag, as in the reference: the option after it is still read) asks for the self-dual
    embedding, which this build has, so it prints no note."""
    from brisk_b200 import _core
    res = _core.solve_sdpa([2], [1.0], [1], [1], [1], [1], [1.0],
                           options=["-hsd", "-corr", "2", "-chordal", "1", "-sym", "auto", "-symalg", "-1",
                                    "-deprows", "1", "-mixedfrac", "0.3", "-threads", "4", "-tol", "x"],
                           verbose=False)
    assert res.exit_code == 1 and "bad -tol" in res.log
    assert "-hsd" not in res.log
    for frag in ("option -corr 2: centrality correctors are not run",
                 "option -chordal 1: no chordal decomposition",
                 "option -sym auto: no symmetry reduction",
                 "option -symalg -1: no block-algebra reduction",
                 "option -deprows 1: dependent constraints are not removed",
                 "option -mixedfrac 0.3"):
        assert frag in res.log, frag
    assert "-threads" not in res.log
    quiet = _core.solve_sdpa([2], [1.0], [1], [1], [1], [1], [1.0],
                             options=["-nohsd", "-sym", "none", "-symalg", "0", "-chordal", "0", "-deprows", "0",
                                      "-corr", "0", "-nofr", "-tol", "x"], verbose=False)
    assert quiet.exit_code == 1 and "note" not in quiet.log


@pytest.mark.parametrize("opt,val,msg", [("-lowrank", "2", "bad -lowrank"), ("-batchtune", "x", "bad -batchtune"),
                                         ("-lowrank", "abc", "bad -lowrank")])
def test_new_options_refuse_bad_values(libpath, opt, val, msg):
    """-lowrank (-1 auto, 0 off, 1 force: the reference's values) and -batchtune (0 or 1) refuse
    other values with exit code 1 and a message, before any device work."""
    from brisk_b200 import _core
    res = _core.solve_sdpa([2], [1.0], [1], [1], [1], [1], [1.0], options=[opt, val], verbose=False)
    assert res.exit_code == 1 and msg in res.log, res.log


def test_method_flags_are_accepted_silently(libpath):
    """-hsd and -nohsd choose the method (the embedding, the infeasible-start method) and print no
    note; a bad -tol after them still stops the solve at the options."""
    from brisk_b200 import _core
    for flag in ("-hsd", "-nohsd"):
        res = _core.solve_sdpa([2], [1.0], [1], [1], [1], [1], [1.0], options=[flag, "-tol", "x"], verbose=False)
        assert res.exit_code == 1 and "bad -tol" in res.log and "note" not in res.log
