"""Generate tests/golden/ref_runs.json: the reference BRISK solver's own results on seeded
instances of the workloads, for the parity tests.

Runs oracle/_ref/brisk_ref (the reference compiled from its sources by oracle/Makefile) on SDPA
files written by brisk_b200.problems, with the reference's presolves off so that it solves the
problem as given, and records per run: status, iterations, objectives, the six DIMACS errors,
the iteration table of -v (pobj, dobj, pinf, dinf, gap, mu per iteration) and the time.

Runs per instance: "init0" and "default" (HKM direction, SDPT3 and least-squares start), "nt"
and "nt_init0" (NT direction, least-squares and SDPT3 start), "hsd_auto" (no -nohsd: the
reference's automatic choice, the self-dual embedding first on most problems).

usage: python tests/golden/make_golden.py [--big] [--huge] [--runs r1,r2] [names]
       (--big adds rand400 and mom700; --huge adds rand1000, the n = 1000, m = 8000 instance, with
       two runs only: "default" (-mixed 0, FP64) and "mixed" (the reference's own default, an FP32
       Schur factor with PCG); --runs recomputes only those runs, keeping the others)
"""
from __future__ import annotations

import json
import os
import re
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from brisk_b200.problems import (batch_instance, dense_instance, infeasible_sdp, lowrank_sdp,  # noqa: E402
                                 moment_relaxation, random_sdp, sdp_lp_problem, theta_problem, write_sdpa)

REF = os.path.join(ROOT, "oracle", "_ref", "brisk_ref")
OUT = os.path.join(ROOT, "tests", "golden", "ref_runs.json")
AS_GIVEN = ["-sym", "none", "-symalg", "0", "-chordal", "0", "-nofr", "-deprows", "0"]

INSTANCES = {
    "theta50": (theta_problem, dict(n=50, p=0.5, seed=1)),
    "theta30": (theta_problem, dict(n=30, p=0.3, seed=7)),
    "rand30": (random_sdp, dict(n=30, m=60, density=0.1, seed=1)),
    "rand60": (random_sdp, dict(n=60, m=200, density=0.05, seed=2)),
    "rand100": (random_sdp, dict(n=100, m=300, density=0.02, seed=3)),
    "mom8": (moment_relaxation, dict(nvars=8, clique=4, seed=1)),
    "mom60": (moment_relaxation, dict(nvars=60, clique=4, seed=0)),
    "dense24": (dense_instance, dict(n=24, m=100, seed=11)),
    "dense48": (dense_instance, dict(n=48, m=500, seed=12)),
    # LP blocks (negative sizes) among SDP blocks, and an LP alone
    "lp_mixed": (sdp_lp_problem, dict(blocks=(30, -40, 6), m=50, density=0.1, lp_per_con=4, seed=3)),
    "lp_only": (sdp_lp_problem, dict(blocks=(-60,), m=30, lp_per_con=6, seed=4)),
    # an LP block of 300 variables with two rows over all of them, beside an SDP block
    # constraints of rank 1-3: dense vectors (the reference's low-rank route), and on 20 of 80 rows
    "lowrank80": (lowrank_sdp, dict(n=80, m=200, max_rank=3, support=0, seed=6)),
    "lowrank80s": (lowrank_sdp, dict(n=80, m=150, max_rank=2, support=20, seed=7)),
    # infeasible problems: no X >= 0 with trace -1 (primal), an unbounded primal (dual)
    "infeas_p": (infeasible_sdp, dict(kind="primal", n=6, m=8, seed=1)),
    "infeas_d": (infeasible_sdp, dict(kind="dual", n=6, m=5, seed=2)),
    "lp_dense": (sdp_lp_problem, dict(blocks=(20, -300), m=80, density=0.1, lp_per_con=5, seed=5, dense_rows=2)),
}
# instances of the 4096-instance uneven batch (n ~ U{8..64}, m ~ U{n..n(n+1)/4}, seed 0): the
# first twelve and the largest (q = 3339: n = 64, m = 1038)
for _q in list(range(12)) + [3339]:
    INSTANCES[f"batch_q{_q}"] = (batch_instance, dict(q=_q))
BIG = {"rand400": (random_sdp, dict(n=400, m=2000, density=0.01, seed=0)),
       "mom700": (moment_relaxation, dict(nvars=700, clique=4, seed=0))}
# about 30 CPU-minutes per run on 8 host threads: the FP64 run and the reference's default mixed run
HUGE = {"rand1000": (random_sdp, dict(n=1000, m=8000, density=0.005, seed=0))}

HKM = ["-nohsd", "-dir", "hkm", "-mixed", "0", "-tol", "1e-7"] + AS_GIVEN
NTD = ["-nohsd", "-dir", "nt", "-mixed", "0", "-tol", "1e-7"] + AS_GIVEN
# "hsd_auto": the reference's own choice of method (no -nohsd: its automatic rule runs the self-dual
# embedding first on most problems), the solve a caller gets with its default options
RUNS = {"init0": HKM + ["-init", "0"], "default": HKM, "nt": NTD, "nt_init0": NTD + ["-init", "0"],
        "hsd_auto": ["-dir", "hkm", "-mixed", "0", "-tol", "1e-7"] + AS_GIVEN}
HUGE_RUNS = {"default": HKM, "mixed": ["-nohsd", "-dir", "hkm", "-tol", "1e-7"] + AS_GIVEN}

ROW = re.compile(r"^\s*(\d+)\s+([+-]\S+)\s+([+-]\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s*$")


def run(path, opts):
    cmd = [REF, path] + opts + ["-v", "-threads", "8"]
    env = dict(os.environ, BRISK_NOBUSY="1")
    p = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=3600)
    out = p.stdout + p.stderr
    rows = []
    for line in out.splitlines():
        mm = ROW.match(line)
        if mm:
            it, po, do, pinf, dinf, gap, mu = mm.groups()[:7]
            rows.append(dict(it=int(it), pobj=float(po), dobj=float(do), pinf=float(pinf), dinf=float(dinf),
                             gap=float(gap), mu=float(mu)))
    st = re.search(r"^status: (.+?)\s+iterations: (\d+)", out, re.M)
    ob = re.search(r"primal obj <C,X> = (\S+)\s+dual obj b'y = (\S+)", out)
    de = re.search(r"^\s*DIMACS errors: (\S+) (\S+) (\S+) (\S+) (\S+) (\S+)", out, re.M)
    tt = re.search(r"^time: total (\S+)s \(read (\S+),", out, re.M)
    return dict(cmd=" ".join(["brisk_ref", os.path.basename(path)] + opts), exit_code=p.returncode,
                status=st.group(1).strip() if st else None, iterations=int(st.group(2)) if st else None,
                pobj=float(ob.group(1)) if ob else None, dobj=float(ob.group(2)) if ob else None,
                dimacs=[float(x) for x in de.groups()] if de else None,
                time_total=float(tt.group(1)) if tt else None, time_read=float(tt.group(2)) if tt else None,
                rows=rows)


def main():
    inst = dict(INSTANCES)
    if "--big" in sys.argv:
        inst.update(BIG)
    if "--huge" in sys.argv:
        inst.update(HUGE)
    res = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            res = json.load(f)
    args = sys.argv[1:]
    wanted = []
    if "--runs" in args:
        i = args.index("--runs")
        wanted = args[i + 1].split(",")
        del args[i:i + 2]
    only = [a for a in args if not a.startswith("--")]
    with tempfile.TemporaryDirectory() as td:
        for name, (fn, kw) in inst.items():
            if only and name not in only:
                continue
            d = fn(**kw)
            path = os.path.join(td, name + ".dat-s")
            write_sdpa(d, path)
            old = res.get(name, {}).get("runs", {})
            entry = dict(generator=fn.__name__, kwargs=kw, m=d.m, n=int(d.bs[0]), nblk=d.nblk, runs=dict(old))
            for rname, opts in (HUGE_RUNS if name in HUGE else RUNS).items():
                if rname in old and wanted and rname not in wanted:
                    continue
                entry["runs"][rname] = run(path, opts)
                r = entry["runs"][rname]
                print(name, rname, d.m, r["status"], r["iterations"], r["pobj"], r["dobj"], flush=True)
            res[name] = entry
    with open(OUT, "w") as f:
        json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
