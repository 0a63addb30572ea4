"""Command line: solve an SDPA file or a seeded workload on the GPU, options as for BRISK.

    python -m brisk_b200 problem.dat-s -tol 1e-7 -v
    python -m brisk_b200 --workload rand1000 -asmprec tf32x3 -v
    python -m brisk_b200 --batch 4096 -tol 1e-7 -mixed 0       (the first N instances of the
                                                                uneven batch, one bgpu_batch_solve)

The file form mirrors the reference's command line (`brisk <file> <options>`, main.c:3571); the
workload form solves one of the seeded instances of brisk_b200.problems.
"""
import sys
import time

from . import problems, solve_batch_arrays, solve_file, solve_sdpa

WORKLOADS = {
    "theta50": lambda: problems.theta_problem(n=50, p=0.5, seed=1),
    "rand400": lambda: problems.random_sdp(n=400, m=2000, density=0.01, seed=0),
    "rand1000": lambda: problems.random_sdp(n=1000, m=8000, density=0.005, seed=0),
    "mom60": lambda: problems.moment_relaxation(nvars=60, clique=4, seed=0),
    "mom700": lambda: problems.moment_relaxation(nvars=700, clique=4, seed=0),
    # an SDP block of 20 and an LP block of 300 variables, two rows over all of them (the LP route)
    "lp_dense": lambda: problems.sdp_lp_problem(blocks=(20, -300), m=80, density=0.1, lp_per_con=5, seed=5,
                                                dense_rows=2),
    # constraints of rank 1-3 with dense vectors (the low-rank route)
    "lowrank80": lambda: problems.lowrank_sdp(n=80, m=200, max_rank=3, support=0, seed=6),
}


def main(argv):
    if not argv:
        print(__doc__)
        return 1
    if argv[0] == "--batch":
        if len(argv) < 2 or not argv[1].isdigit():
            print("--batch N: the first N instances of the uneven 4096-instance batch")
            return 1
        arrs = problems.batch_arrays(int(argv[1]))
        t0 = time.time()
        out = solve_batch_arrays(**arrs, options=argv[2:])
        st = {}
        for r in out:
            st[r.status_str] = st.get(r.status_str, 0) + 1
        print(f"batch of {len(out)}: {st}, {time.time() - t0:.3f} s")
        return max((r.exit_code for r in out), default=0)
    if argv[0] == "--workload":
        if len(argv) < 2 or argv[1] not in WORKLOADS:
            print("workloads: " + ", ".join(sorted(WORKLOADS)))
            return 1
        d = WORKLOADS[argv[1]]()
        r = solve_sdpa(*d.args(), options=argv[2:], verbose=True)
    else:
        r = solve_file(argv[0], options=argv[1:], verbose=True)
    return r.exit_code


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
