"""brisk_b200: the SDP interior-point Newton step of BRISK on a B200 GPU.

The public API mirrors the reference's Python package (``brisk``): ``solve_sdpa`` and
``solve_file`` return a ``Result`` with the status, objectives, DIMACS errors and the solution;
``solve_batch`` solves many independent problems in one call (bgpu_batch_solve);
``read_sdpa_file`` reads an SDPA file with the library's parallel reader (bgpu_sdpa_read).
The work runs in the in-tree CUDA library ``libbrisk.so`` (sm_100a), which exports the same C
interface as the reference's libbrisk.
"""
from ._core import (STATUS, BatchSession, Result, concat_problems, interrupt, library_path, load_library, options_to_argv,
                    read_sdpa_file, solve_batch, solve_batch_arrays, solve_file, solve_sdpa, version)

__all__ = ["STATUS", "BatchSession", "Result", "concat_problems", "interrupt", "library_path", "load_library", "options_to_argv",
           "read_sdpa_file", "solve_batch", "solve_batch_arrays", "solve_file", "solve_sdpa", "version"]
