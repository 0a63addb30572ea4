"""Benchmark: time to a 1e-7 DIMACS solution of the seeded random SDP on B200s.

A step is one interior-point solve of the workload to DIMACS error 1e-7 (the whole Newton-step
path: Schur assembly, factor and PCG solves, step lengths).  Default workload: one 400 x 400
block, m = 2000 constraints of 1 % density, FP64 on the GPU (`rand400`); `--workload rand1000`
is the n = 1000, m = 8000, 0.5 % instance, solved both with the 3xTF32 mixed path and in FP64.

  value  seconds per solve with the problem resident in HBM (bgpu_session: uploaded once before
         the timed region), CUDA events on the library's stream, max over ranks
  e2e    the same solve through the reference's public C call brisk_solve_data with host arrays:
         the upload and the result download are inside the timed region

Multi-GPU: the solve does not shard (one Schur complement per solve); N GPUs run N independent
replicas (`scaling: weak`, one solve per rank per step), launched by torchrun.

`--impl reference` runs the reference's own CPU solver (oracle/_ref/brisk_ref, compiled from
its sources by oracle/Makefile) on the same instance with every host thread (rank 0 only).
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
                     ref_maxit=1),
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


def cpu_reference_sample(d, workload, threads, opts_extra):
    """The reference's CPU solve (oracle/_ref/brisk_ref) of the same instance: the bounded
    sample is one full solve; value = its reported solve time without reading the file."""
    from brisk_b200.problems import write_sdpa
    ref = os.path.join(ROOT, "oracle", "_ref", "brisk_ref")
    if not os.path.exists(ref):
        return None
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, workload + ".dat-s")
        write_sdpa(d, path)
        cmd = [ref, path, "-nohsd", "-dir", "hkm", "-tol", "1e-7", "-v", "-threads", str(threads)] + opts_extra
        env = dict(os.environ, BRISK_NOBUSY="1")
        t0 = time.time()
        p = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=3600)
        wall = time.time() - t0
    out = p.stdout + p.stderr + f" [exit {p.returncode}]"
    tt = re.search(r"time: total (\S+)s \(read (\S+),", out)
    st = re.search(r"^status: (.+?)\s+iterations: (\d+)", out, re.M)
    if not tt:
        return {"error": out[-500:]}
    return {"time": float(tt.group(1)) - float(tt.group(2)), "wall": wall,
            "status": st.group(1).strip() if st else None, "iterations": int(st.group(2)) if st else None,
            "cmd": " ".join(["brisk_ref", workload + ".dat-s"] + cmd[2:])}


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
    print(json.dumps({"impl": "reference", "metric": "time_to_1e-7_dimacs_s", "value": v, "unit": "s",
                      "n_gpus": args.gpus, "steps": 1, "warmup": 0, "ms_per_step": v * 1e3, "higher_is_better": False,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
                      "config": {"workload": "batch", "count": args.batch_count, "desc": w["desc"],
                                 "parallelism": "one process per host core"},
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
            "metric": "time_to_1e-7_dimacs_s", "value": v, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "config": {"workload": "batch", "count": count, "desc": w["desc"], "form": "lockstep (bgpu_batch_run)",
                       "l2": "inputs larger than L2 (packed constraints %.1f GB)" % (8e-9 * sum(
                           m_ * n_ * (n_ + 1) / 2 for n_, m_ in sizes)),
                       "parallelism": f"replicas x{world}", "generation_s": round(gen_s, 1),
                       "resident_setup_s": round(setup_s, 2)},
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
    opts = w["paths"]["fp64"] if w["primary"] == "fp64" else []
    times = []
    for i in range(args.warmup + args.steps):
        r = cpu_reference_sample(d, args.workload, threads, opts + (["-maxit", "1"] if i < args.warmup else []))
        if r is None or "error" in r:
            print(json.dumps({"impl": "reference", "unavailable": "reference binary missing or failed: "
                              + (r or {}).get("error", "oracle/_ref/brisk_ref absent")[-200:]}))
            return
        if i >= args.warmup:
            times.append(r["time"])
    v = statistics.mean(times)
    line = {"impl": "reference", "metric": "time_to_1e-7_dimacs_s", "value": v, "unit": "s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "config": {"workload": args.workload, "desc": w["desc"], "precision": "fp64 (reference -mixed 0)" if opts else
                       "reference default mixed", "parallelism": "cpu threads"},
            "cpu_baseline": {"value": v, "unit": "s", "cores": threads, "kind": "reference",
                             "sample": f"full solve to 1e-7 of {args.workload}, mean of {args.steps}; warm-up runs -maxit 1"},
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_status": r["status"], "reference_iterations": r["iterations"]}
    print(json.dumps(line), flush=True)


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

    flush_buf = torch.zeros(32 * 1024 * 1024, dtype=torch.float64, device="cuda")
    dev_opt = ["-device", str(local)]
    results = {}
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
        nsteps = args.steps if pname == w["primary"] else max(1, min(args.steps, 2))
        for _ in range(args.warmup if pname == w["primary"] else 1):
            S.bgpu_session_solve(sess, n_o, a_o, res)
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        dev_times, statuses, iters, schur_t, schur_f = [], [], [], [], []
        launches0 = S.bgpu_launch_count()
        with Clocks(local) as clk:
            for _ in range(nsteps):
                flush_l2(torch, flush_buf)
                torch.cuda.synchronize()
                code = S.bgpu_session_solve(sess, n_o, a_o, res)
                S.bgpu_result_measures(res, meas)
                dev_times.append(meas[0])
                schur_t.append(meas[1])
                schur_f.append(meas[2])
                iters.append(int(meas[5]))
                statuses.append(L.brisk_result_status_str(res).decode())
                dimacs = (ctypes.c_double * 6)()
                L.brisk_result_dimacs(res, dimacs)
        torch.cuda.synchronize()
        launches = S.bgpu_launch_count() - launches0
        t_step = max_over_ranks(statistics.mean(dev_times), world)
        results[pname] = dict(value=t_step, status=statuses[-1], iterations=iters[-1],
                              schur_tflops=sum(schur_f) / max(sum(schur_t), 1e-30) / 1e12,
                              schur_s_per_solve=statistics.mean(schur_t), launches_per_step=launches / nsteps,
                              clocks=clk.summary(), dimacs=max(abs(x) for x in dimacs), steps=nsteps)
        S.bgpu_session_destroy(sess)
        # end to end through the reference's public call (host arrays, upload + download timed)
        if pname == w["primary"]:
            e2e_times = []
            for k in range(1 + max(1, min(args.steps, 3))):   # the first call untimed (warm-up)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                rc2 = L.brisk_solve_data(d.m, d.nblk, bs.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
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
    roof = None
    cpu = None
    if rank == 0:
        if w["kind"] == "random":
            peak64 = measure_fp64_peak(torch)
            roof = gemm_roofline(torch, step, w["gen"]["n"], step.chunk_default(w["gen"]["n"], 0), peak64)
        if not args.no_cpu_baseline and world == 1:
            threads = os.cpu_count() or 1
            opts_ref = w["paths"]["fp64"] if w["primary"] == "fp64" else []
            maxit = w.get("ref_maxit")
            r = cpu_reference_sample(d, args.workload, threads, opts_ref + (["-maxit", str(maxit)] if maxit else []))
            if r and "error" not in r and not maxit:
                cpu = {"value": r["time"], "unit": "s", "cores": threads, "kind": "reference",
                       "sample": f"one full reference solve to 1e-7 ({r['status']}, {r['iterations']} iterations)"}
            elif r and "error" not in r:
                # the full reference solve takes tens of minutes: a bounded sample of `maxit` iterations
                # (start included), scaled to the iterations this build's solve took
                per_it = r["time"] / max(1, maxit)
                cpu = {"value": per_it * prim["iterations"], "unit": "s", "cores": threads, "kind": "reference",
                       "sample": f"reference solve stopped after {maxit} iteration(s) ({r['time']:.1f} s, start "
                                 f"included), scaled to {prim['iterations']} iterations"}
            else:
                cpu = {"value": None, "error": (r or {}).get("error", "oracle/_ref/brisk_ref absent")[-300:]}
    if world > 1:
        torch.distributed.barrier()
    if rank == 0:
        line = {"metric": "time_to_1e-7_dimacs_s", "value": prim["value"], "unit": "s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": prim["value"] * 1e3,
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if w["primary"] == "fp64" else "tf32x3+f64", "data": "synthetic (seeded generator)",
                "config": {"workload": args.workload, "desc": w["desc"], "precision": w["primary"],
                           "l2": "256 MB buffer written between steps", "parallelism": f"replicas x{world}"},
                "status": prim["status"], "iterations": prim["iterations"], "dimacs_max": prim["dimacs"],
                "schur_tflops": round(prim["schur_tflops"], 3), "schur_s_per_solve": prim["schur_s_per_solve"],
                "e2e": {"value": prim["e2e"]["value"], "unit": "s", "h2d_bytes_per_step": int(prim["e2e"]["h2d"]),
                        "d2h_bytes_per_step": int(prim["e2e"]["d2h"])},
                "gpu_launches": int(prim["launches_per_step"] * prim["steps"]),
                "clocks": prim["clocks"], "roofline": roof, "cpu_baseline": cpu,
                "roofline_note": None if roof else "no dominant GEMM on this workload (small blocks, sparse factor)",
                "paths": {k: {kk: vv for kk, vv in r.items() if kk in ("value", "status", "iterations", "schur_tflops")}
                          for k, r in results.items()}}
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="rand400", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-count", type=int, default=4096, help="instances of the batch workload")
    ap.add_argument("--batch-sample", type=int, default=64, help="instances the reference solves for its sample")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
