"""Benchmark: time to a 1e-7 DIMACS solution of a seeded random SDP on B200s.

A step is one interior-point solve of the workload to DIMACS error 1e-7 (the whole Newton-step
path: Schur assembly, factor and PCG solves, step lengths).  The default workload is `rand1000`:
one 1000 x 1000 block, m = 8000 constraints of 0.5 % density, solved by the mixed-precision path
(3xTF32 Schur assembly on the tensor cores, FP32 factor early, FP64-accurate assembly and factor
late, FP64-residual refinement throughout; `value`) and by the all-FP64 GPU path on the same
instance (`paths.fp64`, with `mixed_speedup_over_fp64`).  `--workload rand400` is the n = 400,
m = 2000, 1 % FP64 instance; the others are listed in WORKLOADS.

  value  seconds per solve with the problem resident in HBM (bgpu_session: uploaded once before
         the timed region), CUDA events on the library's stream, max over ranks
  e2e    the same solve through the reference's public C call brisk_solve_data with host arrays:
         the upload and the result download are inside the timed region

Multi-GPU: the solve does not shard (one Schur complement per solve); N GPUs run N independent
replicas (`scaling: weak`, one solve per rank per step), launched by torchrun.

`--impl reference` times the reference's own CPU solver (compiled from its sources by
oracle/Makefile into oracle/_ref/) on the same instance with every host thread (rank 0 only).
Where its full solve takes many minutes (rand1000: about 7 minutes on 16 cores), a step is one of
its interior-point iterations, timed from the time column of its own iteration table, and the
time to 1e-7 is its start plus the mean iteration times its own iteration count for the whole
solve (recorded in tests/golden/ref_runs.json).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "theta50": dict(kind="theta", gen=dict(n=50, p=0.5, seed=1),
                    desc="Lovasz theta SDP of a seeded G(50, 0.5): one 50x50 block, m=588 (tr X = 1 and one "
                         "constraint X_ij = 0 per edge), C = -J",
                    paths={"fp64": ["-mixed", "0"]}, primary="fp64"),
    "rand400": dict(kind="random", gen=dict(n=400, m=2000, density=0.01, seed=0),
                    desc="random SDP: one 400x400 block, m=2000, A_i 1% dense N(0,1), b=A(I), C=GG'/n+I, seed 0",
                    paths={"fp64": ["-mixed", "0"]}, primary="fp64"),
    "rand1000": dict(kind="random", gen=dict(n=1000, m=8000, density=0.005, seed=0),
                     desc="random SDP: one 1000x1000 block, m=8000, A_i 0.5% dense N(0,1), b=A(I), C=GG'/n+I, seed 0",
                     paths={"mixed": ["-asmprec", "tf32x3"], "fp64": ["-mixed", "0"]}, primary="mixed",
                     ref_sample_its=3),
    "mom60": dict(kind="moment", gen=dict(nvars=60, clique=4, seed=0),
                  desc="degree-2 moment relaxation of a seeded quartic in 60 variables, cliques of 4 consecutive "
                       "variables: 57 blocks of 15, m=2029, sparse Schur factor",
                  paths={"fp64": ["-mixed", "0"]}, primary="fp64"),
    "mom700": dict(kind="moment", gen=dict(nvars=700, clique=4, seed=0),
                   desc="the same moment relaxation in 700 variables: 697 blocks of 15, m=24429, sparse Schur factor",
                   paths={"fp64": ["-mixed", "0"]}, primary="fp64"),
    "batch": dict(kind="batch", gen=dict(nmin=8, nmax=64, seed=0),
                  desc="batch of independent dense random SDPs: n ~ U{8..64}, m ~ U{n..n(n+1)/4}, A_i dense N(0,1) "
                       "symmetric, b=A(I), C=GG'/n+I, seed 0",
                  paths={"fp64": ["-mixed", "0"]}, primary="fp64"),
}


def make_instance(w):
    from brisk_b200 import problems
    if w["kind"] == "moment":
        return problems.moment_relaxation(**w["gen"])
    if w["kind"] == "theta":
        return problems.theta_problem(**w["gen"])
    return problems.random_sdp(**w["gen"])


BASE_OPTS = ["-nohsd", "-dir", "hkm", "-tol", "1e-7", "-q"]
L2_NOTE = ("GPU arm: a 256 MB device buffer written between timed solves (L2 flushed); reference arm: "
           "host-resident inputs on the CPU")


def config_of(name, w):
    """The workload's description, the same dict in both arms (what is solved, not how)."""
    return {"workload": name, "desc": w["desc"], "generator": dict(w["gen"]), "tol": 1e-7, "l2": L2_NOTE}


def max_over_ranks(value, world, device="cuda"):
    """The slowest rank's value (an all-reduce MAX over the process group); the value itself on one
    rank.  device: where the reduced tensor lives ("cuda" under NCCL, "cpu" under gloo)."""
    if world <= 1:
        return value
    import torch
    t = torch.tensor([value], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def flush_l2(torch, buf):
    buf.add_(1.0)            # 256 MB written: larger than the 126 MB L2


def measure_fp64_peak(torch):
    """cuBLAS DGEMM 8192^3 (torch.matmul on float64): the FP64 tensor peak of this GPU, measured
    here (MEASURED_PEAKS.json has no FP64 entry)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) * 1e-3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


def gemm_roofline(torch, step, n, chunk, peak_tflops, launches=10):
    """The dominant kernel (the FP64 row-product GEMM of the Schur assembly, (n K) x n x n per
    launch) timed alone with CUDA events on the stream it is launched on."""
    M = n * chunk
    A = torch.randn(M * n, dtype=torch.float64, device="cuda")
    X = torch.randn(n * n, dtype=torch.float64, device="cuda")
    G = torch.empty(M * n, dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream()
    sp = ctypes.c_void_p(s.cuda_stream)
    for _ in range(3):
        step.call("dgemm", 1, 1, M, n, n, 1.0, A.data_ptr(), n, X.data_ptr(), n, 0.0, G.data_ptr(), M, 0, sp)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    for _ in range(launches):
        step.call("dgemm", 1, 1, M, n, n, 1.0, A.data_ptr(), n, X.data_ptr(), n, 0.0, G.data_ptr(), M, 0, sp)
    e1.record(s)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) * 1e-3 / launches
    flops = 2.0 * M * n * n
    ach = flops / t / 1e12
    return {"bound": "tensor", "kernel": "dgemm_kernel (FP64 DMMA m16n8k4)", "achieved": round(ach, 3),
            "peak": round(peak_tflops, 3), "unit": "TFLOP/s", "frac": round(ach / peak_tflops, 4),
            "traffic": None, "flops_per_launch": flops, "launch_ms": round(t * 1e3, 4),
            "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no FP64 entry)"}


REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libbrisk_ref.so")
REF_ROW = re.compile(r"^\s*(\d+)\s+[+-]\S+\s+[+-]\S+(?:\s+\S+){7}\s+(\S+)\s*$")
METRIC = "time_to_1e-7_dimacs_s"


def reference_solve(d, threads, opts):
    """One solve by the reference's own C API: brisk_solve_data of oracle/_ref/libbrisk_ref.so
    (the reference compiled from its sources by oracle/Makefile) on the instance's arrays, in this
    process, with -v and every given host thread (BRISK_NOBUSY=1 keeps the count exact).  Returns
    its status, iterations, its reported total time and the time column of its iteration table
    (seconds since its iterations began, one entry per row), or None when the library is absent."""
    if not os.path.exists(REF_LIB):
        return None
    os.environ["BRISK_NOBUSY"] = "1"
    L = ctypes.CDLL(REF_LIB, mode=os.RTLD_LOCAL)
    PRINT = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_char_p, ctypes.c_int)
    chunks = []

    def cb(s, is_err):
        chunks.append(s.decode(errors="replace"))
        return 0

    cbf = PRINT(cb)
    L.brisk_set_output.argtypes = [ctypes.c_int, PRINT]
    L.brisk_result_new.restype = ctypes.c_void_p
    L.brisk_result_delete.argtypes = [ctypes.c_void_p]
    L.brisk_result_status_str.argtypes, L.brisk_result_status_str.restype = [ctypes.c_void_p], ctypes.c_char_p
    L.brisk_result_iterations.argtypes, L.brisk_result_iterations.restype = [ctypes.c_void_p], ctypes.c_int
    pi, pd = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    L.brisk_solve_data.argtypes = [ctypes.c_int, ctypes.c_int, pi, pd, ctypes.c_int64, pi, pi, pi, pi, pd, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_char_p), ctypes.c_void_p]
    bs, c, mat, blk, ii, jj, v = [np.ascontiguousarray(a) for a in d.args()]
    bs, mat, blk, ii, jj = [a.astype(np.intc) for a in (bs, mat, blk, ii, jj)]
    av = list(opts) + ["-v", "-threads", str(threads)]
    arr = (ctypes.c_char_p * len(av))(*[a.encode() for a in av])
    L.brisk_set_output(2, cbf)
    res = L.brisk_result_new()
    t0 = time.perf_counter()
    rc = L.brisk_solve_data(d.m, d.nblk, bs.ctypes.data_as(pi), c.ctypes.data_as(pd), d.nnz, mat.ctypes.data_as(pi),
                            blk.ctypes.data_as(pi), ii.ctypes.data_as(pi), jj.ctypes.data_as(pi),
                            v.ctypes.data_as(pd), len(av), arr, res)
    wall = time.perf_counter() - t0
    status = L.brisk_result_status_str(res).decode()
    iters = L.brisk_result_iterations(res)
    L.brisk_result_delete(res)
    L.brisk_set_output(0, PRINT(0))
    out = "".join(chunks)
    tt = re.search(r"time: total (\S+)s \(read (\S+),", out)
    rows = [float(mm.group(2)) for mm in map(REF_ROW.match, out.splitlines()) if mm]
    if not tt:
        return {"error": f"exit {rc}: " + out[-300:]}
    return {"time": float(tt.group(1)) - float(tt.group(2)), "wall": wall, "status": status, "iterations": iters,
            "row_times": rows, "exit_code": rc}


def golden_iterations(workload, run):
    """The reference's own iteration count to 1e-7 on this instance (tests/golden/ref_runs.json)."""
    try:
        with open(os.path.join(ROOT, "tests", "golden", "ref_runs.json")) as f:
            return int(json.load(f)[workload]["runs"][run]["iterations"])
    except (OSError, KeyError, ValueError, TypeError):
        return None


def reference_options(w):
    """The reference's options on a workload: its own default precision where this build's primary
    path is the mixed one (its float Schur factor + PCG for m >= 1000), -mixed 0 where it is FP64."""
    return ["-nohsd", "-dir", "hkm", "-tol", "1e-7"] + (w["paths"]["fp64"] if w["primary"] == "fp64" else [])


def reference_measure(workload, w, d, steps, warmup, threads):
    """The reference arm's measurement.  Full solves (`steps` of them after `warmup` solves stopped
    after one iteration) where a solve is short; where `ref_sample_its` is set, one solve stopped
    after that many iterations: its iteration times are the steps, and the time to 1e-7 is its
    total time plus (the reference's own iteration count - the sampled ones) x the mean iteration."""
    opts = reference_options(w)
    S = w.get("ref_sample_its")
    if S:
        run = "mixed" if w["primary"] == "mixed" else "default"
        n_ref = golden_iterations(workload, run)
        if n_ref is None:
            return {"error": f"no recorded reference iteration count for {workload} ({run} run)"}
        if warmup > 0:
            reference_solve(d, threads, opts + ["-maxit", "0"])
        r = reference_solve(d, threads, opts + ["-maxit", str(S)])
        if r is None or "error" in r:
            return r or {"error": "oracle/_ref/libbrisk_ref.so absent"}
        rt = r["row_times"]
        its = [rt[k] - rt[k - 1] for k in range(1, len(rt))]
        if not its:
            return {"error": "no iteration rows in the reference's output"}
        per_it = statistics.mean(its)
        value = r["time"] + max(0, n_ref - len(its)) * per_it
        return {"value": value, "steps": len(its), "warmup": 1 if warmup > 0 else 0, "status": r["status"],
                "iterations": n_ref,
                "sample": f"one reference solve through its C API stopped after {len(its)} iterations ({r['time']:.1f} s "
                          f"with set-up and start; iterations {', '.join('%.2f' % t for t in its)} s); time to 1e-7 = "
                          f"that + {n_ref - len(its)} x the mean iteration ({per_it:.2f} s), {n_ref} being the "
                          f"reference's own iteration count on this instance (its recorded {run} run)"}
    for _ in range(warmup):
        reference_solve(d, threads, opts + ["-maxit", "1"])
    times, r = [], None
    for _ in range(steps):
        r = reference_solve(d, threads, opts)
        if r is None or "error" in r:
            return r or {"error": "oracle/_ref/libbrisk_ref.so absent"}
        times.append(r["time"])
    return {"value": statistics.mean(times), "steps": steps, "warmup": warmup, "status": r["status"],
            "iterations": r["iterations"],
            "sample": f"full reference solves to 1e-7 through its C API, mean of {steps} (reported time); "
                      f"{warmup} warm-up solve(s) stopped after one iteration"}


def _ref_batch_one(q):
    """One batch instance solved by the reference on one thread: (solve time, status)."""
    from brisk_b200 import problems
    from brisk_b200.problems import write_sdpa
    ref = os.path.join(ROOT, "oracle", "_ref", "brisk_ref")
    d = problems.batch_instance(q)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, f"b{q}.dat-s")
        write_sdpa(d, path)
        cmd = [ref, path, "-nohsd", "-dir", "hkm", "-tol", "1e-7", "-mixed", "0", "-v", "-threads", "1"]
        p = subprocess.run(cmd, capture_output=True, text=True, env=dict(os.environ, BRISK_NOBUSY="1"), timeout=3600)
    out = p.stdout + p.stderr
    tt = re.search(r"time: total (\S+)s \(read (\S+),", out)
    st = re.search(r"^status: (.+?)\s+iterations", out, re.M)
    if not tt:
        return None
    return float(tt.group(1)) - float(tt.group(2)), (st.group(1).strip() if st else None)


def cpu_reference_batch(count, sample):
    """The reference on a bounded sample of the batch: `sample` instances spread over the batch,
    each solved on one thread, one process per host core (the batch's natural CPU form: its
    instances are independent).  Scaled to the whole batch: sum of the sample's solve times x
    count / sample / cores."""
    import multiprocessing as mp
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "brisk_ref")):
        return None
    qs = [int(round(k * count / sample)) for k in range(sample)]
    cores = os.cpu_count() or 1
    t0 = time.time()
    with mp.get_context("spawn").Pool(cores) as pool:
        res = pool.map(_ref_batch_one, qs)
    wall = time.time() - t0
    if any(r is None for r in res):
        return {"error": "a reference solve failed"}
    tsum = sum(r[0] for r in res)
    nopt = sum(1 for r in res if r[1] == "OPTIMAL")
    return {"value": tsum * count / sample / cores, "cores": cores, "sum": tsum, "wall": wall,
            "sample": f"{sample} instances spread over the {count} (every {count // sample}-th), one thread each, "
                      f"{nopt}/{sample} OPTIMAL, sum of solve times {tsum:.1f} s; scaled: sum x {count}/{sample} / "
                      f"{cores} cores"}


def run_reference_batch(args, w):
    r = cpu_reference_batch(args.batch_count, min(args.batch_count, args.batch_sample))
    if r is None or "error" in r:
        print(json.dumps({"impl": "reference", "unavailable": (r or {}).get("error", "oracle/_ref/brisk_ref absent")}))
        return
    v = r["value"]
    print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": "s",
                      "n_gpus": args.gpus, "steps": 1, "warmup": 0, "ms_per_step": v * 1e3, "higher_is_better": False,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
                      "config": dict(config_of("batch", w), count=args.batch_count),
                      "parallelism": "one process per host core",
                      "cpu_baseline": {"value": v, "unit": "s", "cores": r["cores"], "kind": "reference",
                                       "sample": r["sample"]},
                      "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
          flush=True)


def run_ours_batch(args, w, torch):
    """The batch: `value` solves it from device-resident data (bgpu_batch_create once, then
    bgpu_batch_run per step, CUDA events around each run); `e2e` is one bgpu_batch_solve call on
    the host arrays (problem build, upload, solve, results: the call a user makes)."""
    from brisk_b200 import _core, problems, step
    rank, world, local = dist_info()
    L = _core.load_library()
    S = step.lib()
    S.bgpu_launch_count.restype = ctypes.c_longlong
    count = args.batch_count
    t0 = time.time()
    full = problems.batch_arrays(count, **w["gen"])
    gen_s = time.time() - t0
    opts = BASE_OPTS + w["paths"]["fp64"] + ["-device", str(local)]
    t0 = time.time()
    sess = _core.BatchSession(**full, options=opts)
    setup_s = time.time() - t0
    for _ in range(args.warmup):
        sess.run(collect=False)
    times = []
    l0 = S.bgpu_launch_count()
    with Clocks(local) as clk:
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            rcs = sess.run(collect=False)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) * 1e-3)
    launches = (S.bgpu_launch_count() - l0) / args.steps
    out = sess.run(collect=True)
    sess.close()
    st = {}
    for r in out:
        st[r.status_str] = st.get(r.status_str, 0) + 1
    worst = max(float(np.max(np.abs(r.dimacs))) for r in out)
    its = sum(r.iterations for r in out)
    v = max_over_ranks(statistics.mean(times), world)
    # end to end: the whole batch call on the host arrays
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = _core.solve_batch_arrays(**full, options=opts)
    e2e = time.perf_counter() - t0
    h2d = float(sum(a.nbytes for a in full.values()))
    d2h = float(sum(8.0 * (r.X[0].size + r.Z[0].size + r.y.size) for r in res))
    sizes = list(zip(full["bs"].tolist(), full["m"].tolist()))
    asm_flops = sum(m * (4.0 * n ** 3 + 2.0 * n * n * m) for n, m in sizes)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        r = cpu_reference_batch(count, min(count, args.batch_sample))
        if r and "error" not in r:
            cpu = {"value": r["value"], "unit": "s", "cores": r["cores"], "kind": "reference", "sample": r["sample"]}
        else:
            cpu = {"value": None, "error": (r or {}).get("error", "oracle/_ref/brisk_ref absent")}
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": v, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "config": dict(config_of("batch", w), count=count), "form": "lockstep (bgpu_batch_run)",
            "inputs_gb": round(8e-9 * sum(m_ * n_ * (n_ + 1) / 2 for n_, m_ in sizes), 2),
            "parallelism": f"replicas x{world}", "generation_s": round(gen_s, 1),
            "resident_setup_s": round(setup_s, 2),
            "status": st, "dimacs_max": worst, "iterations_total": int(its),
            "instances_per_s": count / v, "assembly_flops_per_iteration": asm_flops,
            "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "note": "bgpu_batch_solve on the host arrays: build, upload, solve, results"},
            "gpu_launches": int(launches), "clocks": clk.summary(), "roofline": None,
            "roofline_note": "latency-bound rounds over all instances; see DESIGN",
            "cpu_baseline": cpu}), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def run_reference(args):
    rank, world, local = dist_info()
    if rank != 0:
        return
    w = WORKLOADS[args.workload]
    if w["kind"] == "batch":
        return run_reference_batch(args, w)
    d = make_instance(w)
    threads = os.cpu_count() or 1
    r = reference_measure(args.workload, w, d, args.steps, args.warmup, threads)
    if r is None or "error" in r:
        print(json.dumps({"impl": "reference", "unavailable": "reference solve failed or absent: "
                          + (r or {}).get("error", "oracle/_ref/libbrisk_ref.so absent")[-200:]}))
        return
    v = r["value"]
    prec = "fp64 (reference -mixed 0)" if w["primary"] == "fp64" else "the reference's default (float Schur factor + PCG)"
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus,
            "steps": r["steps"], "warmup": r["warmup"], "ms_per_step": v * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "config": config_of(args.workload, w), "precision": prec, "parallelism": f"cpu threads x{threads}",
            "cpu_baseline": {"value": v, "unit": "s", "cores": threads, "kind": "reference", "sample": r["sample"]},
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_status": r["status"], "reference_iterations": r["iterations"]}
    print(json.dumps(line), flush=True)


ROW = re.compile(r"^\s*(\d+)\s+([+-]\S+)\s+([+-]\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s+\S+\s+\S+\s+\S+\s+\S+\s*$")


def table_rows(log):
    """The iteration table of a -v log: it -> (pobj, dobj, pinf, dinf, gap, mu) as printed."""
    rows = {}
    for line in log.splitlines():
        mm = ROW.match(line)
        if mm:
            rows[int(mm.group(1))] = tuple(float(x) for x in mm.groups()[1:])
    return rows


def per_iteration_errors(mixed_log, fp64_log):
    """Each iteration of the mixed solve against the FP64 solve of the same instance from the same
    start: the mixed iterate's own infeasibilities and gap, and its objectives' relative distance
    from the FP64 solve's at the same iteration (to the 9 digits the table prints)."""
    a, b = table_rows(mixed_log), table_rows(fp64_log)
    out = []
    for it in sorted(a):
        pm, dm, pinf, dinf, gap, mu = a[it]
        row = {"it": it, "pinf": pinf, "dinf": dinf, "gap": gap, "mu": mu}
        if it in b:
            pf, df = b[it][0], b[it][1]
            row["pobj_rel_vs_fp64"] = float("%.2e" % (abs(pm - pf) / (1 + abs(pf))))
            row["dobj_rel_vs_fp64"] = float("%.2e" % (abs(dm - df) / (1 + abs(df))))
        out.append(row)
    return out


def load_peaks():
    """MEASURED_PEAKS.json (driver-written: measured copy bandwidth and cuBLAS bf16 GEMM on this
    pool's B200s), else the earlier measurement on this pool."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return float(pk["bf16_tflops"]), float(pk["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 1590.0, 6650.0, "fallback"


# DRAM bytes (read + write) of one launch of the n = 1000, K = 64 chunk GEMM, from
# `ncu --set full` (profiles/tf32x3_kernel_rand1000_chunk.md): 536.1 MB + 227.5 MB
TF32X3_TRAFFIC = 763.58e6


def tf32x3_roofline(torch, step, n, chunk, launches=10):
    """The dominant kernel of the mixed path (the 3xTF32 row-product GEMM of the Schur assembly,
    (n K) x n x n per launch, three tf32 MMAs per product on tcgen05) timed alone with CUDA events
    on the stream it is launched on.  Useful flops 2 (n K) n^2 against the 3xTF32-useful peak:
    the measured dense bf16 rate / 2 (TF32 runs at half the bf16 rate) / 3 (MMAs per product)."""
    bf16, _, src = load_peaks()
    peak = bf16 / 2.0 / 3.0
    M, ld = n * chunk, (n + 3) // 4 * 4
    f32 = torch.float32
    Ah, Al = torch.randn(M * ld, dtype=f32, device="cuda"), torch.randn(M * ld, dtype=f32, device="cuda") * 1e-4
    Bh, Bl = torch.randn(n * ld, dtype=f32, device="cuda"), torch.randn(n * ld, dtype=f32, device="cuda") * 1e-4
    G = torch.empty(M * n, dtype=f32, device="cuda")
    s = torch.cuda.current_stream()
    sp = ctypes.c_void_p(s.cuda_stream)
    args = (M, n, n, Ah.data_ptr(), Al.data_ptr(), ld, Bh.data_ptr(), Bl.data_ptr(), ld, G.data_ptr(), M, sp)
    for _ in range(3):
        step.call("gemm_tf32x3", *args)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(launches):
        step.call("gemm_tf32x3", *args)
    e1.record(s)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) * 1e-3 / launches
    flops = 2.0 * M * n * n
    ach = flops / t / 1e12
    return {"bound": "tensor", "kernel": "tf32x3_kernel (3xTF32, tcgen05.mma kind::tf32, TMEM accumulator)",
            "achieved": round(ach, 2), "peak": round(peak, 2), "unit": "TFLOP/s", "frac": round(ach / peak, 4),
            "traffic": TF32X3_TRAFFIC if (n, chunk) == (1000, 64) else None,
            "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture of this launch "
                              "(profiles/tf32x3_kernel_rand1000_chunk.md); algorithmic bytes 7.76e8",
            "flops_per_launch": flops, "launch_ms": round(t * 1e3, 4),
            "peak_source": f"{src} bf16 {bf16:.1f} TF/s (burst) / 2 for TF32 / 3 MMAs per useful product "
                           f"({'of measured' if src == 'measured' else 'of fallback'})"}


def run_ours(args):
    import torch
    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    from brisk_b200 import _core, problems, step
    L = _core.load_library()
    S = step.lib()
    P, I = ctypes.c_void_p, ctypes.c_int
    S.bgpu_session_create.restype = P
    S.bgpu_session_create.argtypes = [I, I, P, P, ctypes.c_int64, P, P, P, P, P, I, P, P]
    S.bgpu_session_solve.argtypes = [P, I, P, P]
    S.bgpu_session_solve.restype = I
    S.bgpu_session_destroy.argtypes = [P]
    S.bgpu_result_measures.argtypes = [P, P]
    S.bgpu_launch_count.restype = ctypes.c_longlong
    w = WORKLOADS[args.workload]
    if w["kind"] == "batch":
        return run_ours_batch(args, w, torch)
    d = make_instance(w)
    bs, c, mat, blk, ii, jj, v = [np.ascontiguousarray(a) for a in d.args()]
    bs = bs.astype(np.intc); mat = mat.astype(np.intc); blk = blk.astype(np.intc)
    ii = ii.astype(np.intc); jj = jj.astype(np.intc)

    def argv(lst):
        arr = (ctypes.c_char_p * max(len(lst), 1))(*[a.encode() for a in lst])
        return len(lst), arr

    chunks = []
    cbf = _core._PRINT(lambda s_, e_: (chunks.append(s_.decode(errors="replace")), 0)[1])

    def logged_solve(sess, opts, res):
        """An untimed solve with -v, its output captured (the iteration table)."""
        n_v, a_v = argv([o for o in opts if o != "-q"] + ["-v"])
        chunks.clear()
        L.brisk_set_output(2, cbf)
        try:
            S.bgpu_session_solve(sess, n_v, a_v, res)
        finally:
            L.brisk_set_output(0, _core._PRINT(0))
        return "".join(chunks)

    flush_buf = torch.zeros(32 * 1024 * 1024, dtype=torch.float64, device="cuda")
    dev_opt = ["-device", str(local)]
    results, logs = {}, {}
    for pname, popts in w["paths"].items():
        opts = BASE_OPTS + popts + dev_opt
        n_o, a_o = argv(opts)
        rc = ctypes.c_int(0)
        sess = S.bgpu_session_create(d.m, d.nblk, bs.ctypes.data, c.ctypes.data, d.nnz, mat.ctypes.data,
                                     blk.ctypes.data, ii.ctypes.data, jj.ctypes.data, v.ctypes.data, n_o, a_o,
                                     ctypes.byref(rc))
        if not sess:
            raise RuntimeError(f"session create failed: exit code {rc.value}")
        res = L.brisk_result_new()
        meas = (ctypes.c_double * 8)()
        primary = pname == w["primary"]
        nsteps = args.steps if primary else max(1, min(args.steps, 2))
        nwarm = args.warmup if primary else 1
        for k in range(nwarm):
            if k == 0:
                logs[pname] = logged_solve(sess, opts, res)
            else:
                S.bgpu_session_solve(sess, n_o, a_o, res)
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        dev_times, statuses, iters, schur_t, schur_f = [], [], [], [], []
        launches0 = S.bgpu_launch_count()
        dimacs = (ctypes.c_double * 6)()
        with Clocks(local) as clk:
            for _ in range(nsteps):
                flush_l2(torch, flush_buf)
                torch.cuda.synchronize()
                S.bgpu_session_solve(sess, n_o, a_o, res)
                S.bgpu_result_measures(res, meas)
                dev_times.append(meas[0])
                schur_t.append(meas[1])
                schur_f.append(meas[2])
                iters.append(int(meas[5]))
                statuses.append(L.brisk_result_status_str(res).decode())
                L.brisk_result_dimacs(res, dimacs)
        torch.cuda.synchronize()
        launches = S.bgpu_launch_count() - launches0
        if pname not in logs:
            logs[pname] = logged_solve(sess, opts, res)
        t_step = max_over_ranks(statistics.mean(dev_times), world)
        results[pname] = dict(value=t_step, status=statuses[-1], iterations=iters[-1],
                              schur_tflops=sum(schur_f) / max(sum(schur_t), 1e-30) / 1e12,
                              schur_s_per_solve=statistics.mean(schur_t), launches_per_step=launches / nsteps,
                              clocks=clk.summary(), dimacs=[float(x) for x in dimacs], steps=nsteps,
                              pobj=float(L.brisk_result_pobj(res)), dobj=float(L.brisk_result_dobj(res)),
                              pcg_steps=int(meas[7]))
        S.bgpu_session_destroy(sess)
        # end to end through the reference's public call (host arrays, upload + download timed)
        if primary:
            e2e_times = []
            for k in range(1 + max(1, min(args.steps, 3))):   # the first call untimed (warm-up)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                L.brisk_solve_data(d.m, d.nblk, bs.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                   c.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), d.nnz,
                                   mat.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                   blk.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                   ii.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                   jj.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                   v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n_o,
                                   ctypes.cast(a_o, ctypes.POINTER(ctypes.c_char_p)), res)
                if k > 0:
                    e2e_times.append(time.perf_counter() - t0)
            S.bgpu_result_measures(res, meas)
            results[pname]["e2e"] = dict(value=statistics.mean(e2e_times), h2d=meas[3], d2h=meas[4])
        L.brisk_result_delete(res)
    prim = results[w["primary"]]
    roof, roof64, cpu = None, None, None
    if rank == 0:
        if w["kind"] == "random":
            n = w["gen"]["n"]
            peak64 = measure_fp64_peak(torch)
            roof64 = gemm_roofline(torch, step, n, step.chunk_default(n, 0), peak64)
            roof = tf32x3_roofline(torch, step, n, step.chunk_default(n, 1)) if w["primary"] == "mixed" else roof64
        if not args.no_cpu_baseline and world == 1:
            # the reference arm's own measurement, in a separate process (no CUDA or torch there)
            cmd = [sys.executable, os.path.abspath(__file__), "--impl", "reference", "--workload", args.workload,
                   "--steps", "1", "--warmup", "0"]
            p = subprocess.run(cmd, capture_output=True, text=True, timeout=3000, env=dict(os.environ, RANK="0"))
            line = next((ln for ln in p.stdout.splitlines()[::-1] if ln.startswith("{")), None)
            rj = json.loads(line) if line else {}
            if "cpu_baseline" in rj:
                cpu = dict(rj["cpu_baseline"], kind="reference")
            else:
                cpu = {"value": None, "error": (rj.get("unavailable") or p.stderr[-300:] or "no output")}
    if world > 1:
        torch.distributed.barrier()
    if rank == 0:
        line = {"metric": METRIC, "value": prim["value"], "unit": "s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": prim["value"] * 1e3,
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if w["primary"] == "fp64" else "tf32x3+f64", "data": "synthetic (seeded generator)",
                "config": config_of(args.workload, w), "precision": w["primary"], "parallelism": f"replicas x{world}",
                "status": prim["status"], "iterations": prim["iterations"], "dimacs": prim["dimacs"],
                "dimacs_max": max(abs(x) for x in prim["dimacs"]),
                "schur_tflops": round(prim["schur_tflops"], 3), "schur_s_per_solve": prim["schur_s_per_solve"],
                "e2e": {"value": prim["e2e"]["value"], "unit": "s", "h2d_bytes_per_step": int(prim["e2e"]["h2d"]),
                        "d2h_bytes_per_step": int(prim["e2e"]["d2h"])},
                "gpu_launches": int(prim["launches_per_step"] * prim["steps"]),
                "clocks": prim["clocks"], "roofline": roof, "cpu_baseline": cpu,
                "roofline_note": None if roof else "no dominant GEMM on this workload (small blocks, sparse factor)",
                "paths": {k: {kk: vv for kk, vv in r.items()
                              if kk in ("value", "status", "iterations", "schur_tflops", "schur_s_per_solve", "pobj",
                                        "dobj", "dimacs", "steps", "pcg_steps")}
                          for k, r in results.items()}}
        if "fp64" in results and w["primary"] != "fp64":
            f = results["fp64"]
            line["mixed_speedup_over_fp64"] = round(f["value"] / prim["value"], 3)
            line["mixed_vs_fp64"] = {
                "pobj_rel": abs(prim["pobj"] - f["pobj"]) / (1 + abs(f["pobj"])),
                "dobj_rel": abs(prim["dobj"] - f["dobj"]) / (1 + abs(f["dobj"])),
                "per_iteration": per_iteration_errors(logs.get(w["primary"], ""), logs.get("fp64", ""))}
            line["roofline_fp64"] = roof64
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


PROFILE_CASES = ("tf32x3", "ozaki5", "potrf_f64", "potrf_f32")


def profile_case(name, launches=3):
    """A few launches of one kernel on its rand1000 shape, for ncu captures (no timing printed):
    tf32x3 / ozaki5 the chunk GEMM of the Schur assembly ((n K) x n x n, n = 1000, K = 64: 1.3 GB
    on the device at most), potrf_f64 / potrf_f32 the factor of an m = 8000 SPD matrix (the Schur
    complement's order)."""
    import torch
    from brisk_b200 import step
    torch.cuda.set_device(0)
    cuda = torch.device("cuda:0")
    sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    torch.manual_seed(0)
    if name in ("tf32x3", "ozaki5"):
        n, K = 1000, 64
        M = n * K
        if name == "tf32x3":
            ld = (n + 3) // 4 * 4
            f32 = torch.float32
            Ah, Al = torch.randn(M * ld, dtype=f32, device=cuda), torch.randn(M * ld, dtype=f32, device=cuda) * 1e-4
            Bh, Bl = torch.randn(n * ld, dtype=f32, device=cuda), torch.randn(n * ld, dtype=f32, device=cuda) * 1e-4
            G = torch.empty(M * n, dtype=f32, device=cuda)
            for _ in range(launches):
                step.call("gemm_tf32x3", M, n, n, Ah.data_ptr(), Al.data_ptr(), ld, Bh.data_ptr(), Bl.data_ptr(), ld,
                          G.data_ptr(), M, sp)
        else:
            T = torch.randn(M * n, dtype=torch.float64, device=cuda)
            X = torch.randn(n * n, dtype=torch.float64, device=cuda)
            G = torch.empty(M * n, dtype=torch.float64, device=cuda)
            nws = int(step.lib().bgpu_ozaki_ws_bytes(M, n, n))
            ws = torch.empty(nws, dtype=torch.uint8, device=cuda)
            for _ in range(launches):
                step.call("gemm_ozaki_slices", 5, M, n, n, T.data_ptr(), n, X.data_ptr(), n, G.data_ptr(), M,
                          ws.data_ptr(), nws, sp)
    else:
        m = 8000
        dt = torch.float64 if name == "potrf_f64" else torch.float32
        R = torch.randn(m, m, dtype=torch.float64, device=cuda)
        A = (R @ R.T / m + torch.eye(m, dtype=torch.float64, device=cuda)).to(dt)
        L = torch.empty_like(A)
        nb = (m + 63) // 64
        dinv = torch.zeros(nb * 4096, dtype=dt, device=cuda)
        info = torch.zeros(1, dtype=torch.int32, device=cuda)
        pmin = torch.zeros(1, dtype=torch.float64, device=cuda)
        for _ in range(launches):
            L.copy_(A)
            step.call(name.replace("_f64", ""), m, L.data_ptr(), m, dinv.data_ptr(), info.data_ptr(),
                      pmin.data_ptr(), sp)
        torch.cuda.synchronize()
        if int(info.item()) != 0:
            raise SystemExit(f"{name}: factor failed at column {int(info.item())}")
    torch.cuda.synchronize()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="rand1000", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-count", type=int, default=4096, help="instances of the batch workload")
    ap.add_argument("--batch-sample", type=int, default=64, help="instances the reference solves for its sample")
    ap.add_argument("--profile-case", choices=PROFILE_CASES,
                    help="run three launches of one kernel on its rand1000 shape and exit (for ncu captures)")
    args = ap.parse_args()
    if args.profile_case:
        profile_case(args.profile_case)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
