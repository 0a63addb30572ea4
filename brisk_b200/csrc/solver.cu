// The infeasible-start primal-dual interior-point loop (HKM or NT direction, Mehrotra predictor-
// corrector) with every O(n^3), O(m^2 n) and O(m^3) step on the GPU.
//
// The loop follows the reference's infeasible-start method, brisk_solve_body
// (solver.c:14394-15188), step by step:
//   Z^-1 from the factor of Z, or the NT scaling W          (solver.c:14397-14421, 7898-7912)
//   residuals, objectives, stopping and infeasibility tests (solver.c:14423-14612)
//   the dual residual kept as theta R0, with a re-base      (solver.c:14317-14326, 14587-14607)
//   Schur complement M, its factor                          (solver.c:14652-14672)
//   rhs pieces a0 = A(Z^-1), h = A(Z^-1 theta R0 X)         (solver.c:14715-14735)
//   predictor, step lengths, sigma, gamma                   (solver.c:14740-14873)
//   corrector and the refinement of A(dX) = rp              (solver.c:14876-15105)
//   step lengths, catastrophe guard, try_step, y update     (solver.c:15108-15188)
// and the reference's problem scaling (problem_prepare, problem.c:1866-1910), starting point
// (start_sdpt3, solver.c:6622-6661), Schur factor rules (schur_factor_, solver.c:5296-5421),
// PCG solve (schur_solve_, solver.c:5483-5621), Lanczos step length (sdp_maxstep_lam,
// solver.c:6083-6225), try_step (solver.c:6393-6447) and DIMACS errors on the data as given
// (postsolve.c:2880-2897, main.c:2349-2362).  Vectors of length m live on the host (their
// work is O(m)); the n x n block arrays and the m x m Schur complement stay in HBM.
#include "common.cuh"
#include "elementwise.h"
#include "kernels.h"
#include "small.h"
#include "solver.h"
#include "sparse.h"
#include "lockstep.h"
#include "nt.h"
#include "tf32x3.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <atomic>
#include <map>
#include <mutex>
#include <numeric>
#include <thread>
#include <functional>
#include <tuple>

namespace bsolve {

static double wtime() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

const char *status_string(int s) {
    switch (s) {
        case 0: return "OPTIMAL";
        case 1: return "PRIMAL INFEASIBLE";
        case 2: return "DUAL INFEASIBLE";
        case 3: return "ITERATION LIMIT";
        case 4: return "NUMERICAL DIFFICULTIES";
        case 5: return "REDUCED ACCURACY";
        case 6: return "TIME LIMIT";
        default: return "NOT SOLVED";
    }
}
int exit_code_of(int s) {
    switch (s) {
        case 0: return 0;
        case 5: return 10;
        case 1: return 11;
        case 2: return 12;
        case 3: return 13;
        case 4: return 14;
        case 6: return 15;
        default: return 14;
    }
}

// ---------------------------------------------------------------------------------------------
// host problem (scaled)
// ---------------------------------------------------------------------------------------------
struct HBlock {
    int n = 0;
    std::vector<int> con;                 // global constraint ids (ascending)
    std::vector<long long> cptr;          // per local constraint, into cpos/cval (full expansion)
    std::vector<int, NoInitAlloc<int>> cpos;
    std::vector<double, NoInitAlloc<double>> cval;
    std::vector<int> Cpos;                // C, full expansion
    std::vector<double> Cval;
};

struct HProblem {
    int m = 0;
    std::vector<HBlock> blk;
    std::vector<double> b, b0;            // scaled, as given
    std::vector<double> d, du;
    double bs = 1, cs = 1, normb1 = 0, normb2 = 0, normC1 = 0, normC2 = 0;
    long long Ntot = 0;
    // the blocks as given: their sizes (negative: LP) and the first of their blocks here
    std::vector<int> in_n, in_first;
    bool lp_only = false;   // no SDP block as given
    // the lockstep batch keeps, instead of its one block's entry lists: the constraints as packed
    // upper rows (m x n(n+1)/2) and the start's scalings xi, eta
    std::vector<double, NoInitAlloc<double>> packed;
    std::vector<double> Cdense;   // C (scaled), n x n
    double xi0 = 0, eta0 = 0;
};

// The messages of brisk_solve_data's checks of an entry (problem.c, problem_from_sdpa_data), with
// the entry as given: why 1 a value not finite, 2 an index out of range, 3 an LP entry off the
// diagonal.
static std::string entry_fault(const InputView &in, long long e, int why) {
    char s[128];
    if (why == 1)
        std::snprintf(s, sizeof s, "non-finite value in entry %d %d %d %d", in.mat[e], in.blk[e], in.i[e], in.j[e]);
    else if (why == 2)
        std::snprintf(s, sizeof s, "bad entry %d %d %d %d", in.mat[e], in.blk[e], in.i[e], in.j[e]);
    else
        std::snprintf(s, sizeof s, "off-diagonal entry in LP block");
    return s;
}

// c[i] not finite (problem.c, problem_from_sdpa_data): its message, or "" when every c[i] is finite.
static std::string c_fault(const InputView &in) {
    for (int i = 0; i < in.m; i++)
        if (!std::isfinite(in.c[i])) return "non-finite value c[" + std::to_string(i + 1) + "]";
    return "";
}

// build_problem for a problem of one SDP block, straight from the caller's arrays into the packed
// rows of the lockstep batch (the same checks, duplicate sums in input order, problem_prepare
// scaling and start_sdpt3 scalings; the row norms are summed over the packed upper entries).
static int build_packed(const InputView &in, HProblem &P, std::string &err) {
    const int m = in.m, n = in.bs[0];
    if (in.nblk != 1 || n <= 0) { err = "not a one-block problem"; return 2; }
    err = c_fault(in);
    if (!err.empty()) return 2;
    const int t = n * (n + 1) / 2;
    P = HProblem();
    P.m = m;
    P.b0.assign(in.c, in.c + m);
    P.b = P.b0;
    P.blk.resize(1);
    P.blk[0].n = n;
    P.Ntot = n;
    P.packed.resize((size_t)m * t);   // each row zeroed as its matrix first appears (in cache)
    std::vector<char> zeroed(m, 0);
    std::vector<double> Cu(t, 0.0);
    for (long long e = 0; e < in.nnz; e++) {
        const double v = in.v[e];
        if (!std::isfinite(v)) { err = entry_fault(in, e, 1); return 2; }
        if (v == 0) continue;
        const int k = in.blk[e] - 1, mt = in.mat[e];
        int i = in.i[e], j = in.j[e];
        if (k != 0 || mt < 0 || mt > m || i < 1 || j < 1 || i > n || j > n) { err = entry_fault(in, e, 2); return 2; }
        if (i > j) std::swap(i, j);
        const size_t u = (size_t)(j - 1) * j / 2 + (i - 1);
        if (mt == 0) {
            Cu[u] += v;
            continue;
        }
        double *row = P.packed.data() + (size_t)(mt - 1) * t;
        if (!zeroed[mt - 1]) {
            std::fill(row, row + t, 0.0);
            zeroed[mt - 1] = 1;
        }
        row[u] += v;
    }
    for (int a = 0; a < m; a++)
        if (!zeroed[a]) std::fill(P.packed.data() + (size_t)a * t, P.packed.data() + (size_t)(a + 1) * t, 0.0);
    auto w = [](int u) {   // 2 off the diagonal: both triangles count
        int c = (int)((std::sqrt(8.0 * u + 1.0) - 1.0) * 0.5);
        while (c * (c + 1) / 2 > u) c--;
        while ((c + 1) * (c + 2) / 2 <= u) c++;
        return (u - c * (c + 1) / 2 == c) ? 1.0 : 2.0;
    };
    std::vector<double> wt(t);
    for (int u = 0; u < t; u++) wt[u] = w(u);
    // per row, while it is in cache: its squared norm, the row equilibration d = 1/norm, the row
    // scaled by d, and the scaled row's norm (for the start's scalings below)
    std::vector<double> nrm2(m, 0.0), snorm(m, 0.0);
    P.d.resize(m);
    for (int a = 0; a < m; a++) {
        double *row = P.packed.data() + (size_t)a * t;
        double s = 0;
        for (int u = 0; u < t; u++) s += wt[u] * row[u] * row[u];
        nrm2[a] = s;
        const double d = s > 0 ? 1.0 / std::sqrt(s) : 1.0;
        P.d[a] = d;
        for (int u = 0; u < t; u++) row[u] *= d;
        if (s == 0) continue;
        double s2 = 0;
        for (int u = 0; u < t; u++) s2 += wt[u] * row[u] * row[u];
        snorm[a] = std::sqrt(s2);
    }
    double c2 = 0, c1 = 0;
    for (int u = 0; u < t; u++) { c2 += wt[u] * Cu[u] * Cu[u]; c1 += wt[u] * std::fabs(Cu[u]); }
    P.normC2 = std::sqrt(c2);
    P.normC1 = c1;
    for (int i = 0; i < m; i++) { P.normb1 += std::fabs(P.b0[i]); P.normb2 += P.b0[i] * P.b0[i]; }
    P.normb2 = std::sqrt(P.normb2);
    for (int i = 0; i < m; i++)
        if (nrm2[i] == 0 && P.b[i] != 0) log_printf(1, "brisk: warning: constraint %d is empty but b != 0 (infeasible)\n", i + 1);
    double nbv = 0;
    for (int i = 0; i < m; i++) nbv += P.d[i] * P.b[i] * P.d[i] * P.b[i];
    nbv = std::sqrt(nbv);
    P.bs = nbv > 1 ? nbv : 1.0;
    for (int i = 0; i < m; i++) P.b[i] *= P.d[i];
    P.du.resize(m);
    for (int i = 0; i < m; i++) P.du[i] = P.bs / P.d[i];
    P.cs = P.normC2 > 1 ? P.normC2 : 1.0;
    for (int i = 0; i < m; i++) P.b[i] /= P.bs;
    // C = -F0 (scaled) in full, and the start's scalings (start_sdpt3, solver.c:6622-6661)
    P.Cdense.assign((size_t)n * n, 0.0);
    double nC = 0;
    for (int q = 0; q < n; q++)
        for (int p = 0; p <= q; p++) {
            const double v = -Cu[(size_t)q * (q + 1) / 2 + p] / P.cs;
            P.Cdense[p + (size_t)q * n] = v;
            P.Cdense[q + (size_t)p * n] = v;
            nC += (p == q ? 1.0 : 2.0) * v * v;
        }
    nC = std::sqrt(nC);
    double maxA = 0, ratio = 0;
    for (int a = 0; a < m; a++) {
        if (nrm2[a] == 0) continue;   // not a constraint of the block
        const double s = snorm[a];
        maxA = std::max(maxA, s);
        ratio = std::max(ratio, (1 + std::fabs(P.b[a])) / (1 + s));
    }
    P.xi0 = std::max(10.0, std::max(std::sqrt((double)n), n * ratio));
    P.eta0 = std::max(10.0, std::max(std::sqrt((double)n), std::max(maxA, nC)));
    return 0;
}

// Set in batch workers: the host problem build of one instance then runs on the calling thread
// (the batch already keeps every host core busy with other instances).
static thread_local bool tl_serial = false;

// Runs f(i) for i in [0, count) on the host's threads (contiguous chunks, joined before return).
template <typename F>
static void parallel_for(long long count, F f) {
    unsigned nt = std::thread::hardware_concurrency();
    nt = std::max(1u, std::min(nt, 32u));
    if (count < 64 || nt == 1 || tl_serial) {
        for (long long i = 0; i < count; i++) f(i);
        return;
    }
    std::vector<std::thread> th;
    const long long chunk = (count + nt - 1) / nt;
    for (unsigned t = 0; t < nt; t++) {
        const long long lo = t * chunk, hi = std::min(count, lo + chunk);
        if (lo >= hi) break;
        th.emplace_back([lo, hi, &f] { for (long long i = lo; i < hi; i++) f(i); });
    }
    for (auto &t : th) t.join();
}

// Runs f(t) for t in [0, count), each on its own host thread (on the calling thread for count 1).
template <typename F>
static void run_chunks(int count, F f) {
    if (count <= 1) {
        if (count == 1) f(0);
        return;
    }
    std::vector<std::thread> th;
    for (int t = 0; t < count; t++) th.emplace_back(f, t);
    for (auto &x : th) x.join();
}

// Host threads for a pass over `work` items: one per 64k items, up to the cores (at most 32);
// one in batch workers.
static int host_threads(long long work) {
    if (tl_serial) return 1;
    const long long hw = std::max(1u, std::min(std::thread::hardware_concurrency(), 32u));
    return (int)std::max(1LL, std::min(hw, work / 65536));
}

static int build_problem(const InputView &in, HProblem &P, std::string &err) {
    const int nbin = in.nblk, m = in.m;
    P.m = m;
    err = c_fault(in);
    if (!err.empty()) return 2;
    P.b0.assign(in.c, in.c + m);
    P.b = P.b0;
    // An LP block of size N (a negative size, brisk.h:128-140) is N semidefinite blocks of order 1:
    // x >= 0 is X = diag(x) >= 0, and an LP block's X stays diagonal on the way (its data are).
    // P.in_first[k]: the first block here of block k as given.
    P.in_n.assign(in.bs, in.bs + nbin);
    P.in_first.resize(nbin + 1);
    int nb = 0;
    for (int k = 0; k < nbin; k++) {
        if (in.bs[k] == 0) { err = "a block of size 0"; return 2; }
        P.in_first[k] = nb;
        nb += in.bs[k] > 0 ? 1 : -in.bs[k];
    }
    P.in_first[nbin] = nb;
    P.lp_only = std::all_of(in.bs, in.bs + nbin, [](int b) { return b < 0; });
    P.blk.resize(nb);
    for (int k = 0; k < nbin; k++)
        for (int q = P.in_first[k]; q < P.in_first[k + 1]; q++) {
            P.blk[q].n = in.bs[k] > 0 ? in.bs[k] : 1;
            P.Ntot += P.blk[q].n;
        }
    const int *first = P.in_first.data();
    const int *bsz = in.bs;
    auto block_here = [&](long long e) {   // entry e's block here (an LP entry: its variable's)
        const int k = in.blk[e] - 1;
        return bsz[k] > 0 ? first[k] : first[k] + in.i[e] - 1;
    };
    auto rc_here = [&](long long e, int &i, int &j) {   // its 0-based row and column there
        if (bsz[in.blk[e] - 1] > 0) {
            i = in.i[e] - 1;
            j = in.j[e] - 1;
        } else {
            i = j = 0;
        }
    };
    // The caller's entries are read in place; an entry of value 0 is no entry (neither checked nor
    // kept).  They are bucketed by block (a stable counting sort), then by matrix inside each block
    // (already so in most SDPA data; else a stable sort): input order within a (block, matrix)
    // bucket, and only the buckets that occur are kept (a dense (block, matrix) table would have
    // nb (m + 1) entries: 17 million for 697 blocks and 24k constraints).
    //
    // Pass 1, a chunk of the entries per host thread: the checks (the first failing entry in input
    // order gives the message), the entries per block, and whether they come block by block.
    const long long nnz = in.nnz;
    int T = host_threads(nnz);
    while (T > 1 && (double)T * nb * sizeof(long long) > 256e6) T--;   // the counts: at most 256 MB
    struct Chunk { std::vector<long long> cnt; long long nz = 0, bad = -1; int why = 0, k0 = -1, k1 = -1; bool sorted = true; };
    std::vector<Chunk> ch(T);
    run_chunks(T, [&](int t) {
        Chunk &c = ch[t];
        c.cnt.assign(nb, 0);
        int prev = -1;
        for (long long e = nnz * t / T, hi = nnz * (t + 1) / T; e < hi; e++) {
            // the checks in the reference's order: a finite value, then (for a nonzero one) the
            // indices, then an LP entry's place on the diagonal
            if (!std::isfinite(in.v[e])) { c.why = 1; c.bad = e; return; }
            if (in.v[e] == 0) continue;
            const int kin = in.blk[e] - 1, mt = in.mat[e];
            const int i = in.i[e], j = in.j[e];
            if (kin < 0 || kin >= nbin || mt < 0 || mt > m) { c.why = 2; c.bad = e; return; }
            const int n = std::abs(bsz[kin]);
            if (i < 1 || j < 1 || i > n || j > n) { c.why = 2; c.bad = e; return; }
            if (bsz[kin] < 0 && i != j) { c.why = 3; c.bad = e; return; }
            const int k = block_here(e);
            if (prev < 0) c.k0 = k;
            c.sorted = c.sorted && k >= prev;
            prev = k;
            c.cnt[k]++;
            c.nz++;
        }
        c.k1 = prev;
    });
    for (int t = 0; t < T; t++)
        if (ch[t].why) {
            err = entry_fault(in, ch[t].bad, ch[t].why);
            return 2;
        }
    bool by_block = true;
    long long nz = 0;
    for (int t = 0, last = -1; t < T; t++) {
        nz += ch[t].nz;
        if (ch[t].k0 < 0) continue;   // no entry in the chunk
        by_block = by_block && ch[t].sorted && ch[t].k0 >= last;
        last = ch[t].k1;
    }
    std::vector<long long> bstart(nb + 1, 0);
    for (int k = 0; k < nb; k++) {   // block starts; each chunk's count becomes its offset in the block
        long long o = bstart[k];
        for (int t = 0; t < T; t++) {
            const long long c = ch[t].cnt[k];
            ch[t].cnt[k] = o;
            o += c;
        }
        bstart[k + 1] = o;
    }
    // ord[u]: the u-th entry by block.  Not formed when the entries already come block by block
    // with no zero among them (then entry u is the u-th).
    bool ident = by_block && nz == nnz;
    std::vector<long long, NoInitAlloc<long long>> ord;
    if (!ident) {
        ord.resize(nz);
        run_chunks(T, [&](int t) {
            std::vector<long long> &fill = ch[t].cnt;
            for (long long e = nnz * t / T, hi = nnz * (t + 1) / T; e < hi; e++)
                if (in.v[e] != 0) ord[fill[block_here(e)]++] = e;
        });
    }
    ch.clear();
    auto entry = [&](long long u) { return ident ? u : ord[u]; };
    const int U = host_threads(nz);
    auto block_of = [&](long long u) {   // the block whose entries hold position u
        return (int)(std::upper_bound(bstart.begin(), bstart.end(), u) - bstart.begin()) - 1;
    };
    // the blocks whose entries are not in matrix order, which are then sorted (stably)
    std::vector<std::vector<int>> uns(U);
    run_chunks(U, [&](int t) {
        const long long lo = nz * t / U, hi = nz * (t + 1) / U;
        if (lo >= hi) return;
        int k = block_of(lo);
        for (long long u = lo; u < hi; u++) {
            while (u >= bstart[k + 1]) k++;
            if (u > bstart[k] && in.mat[entry(u)] < in.mat[entry(u - 1)] && (uns[t].empty() || uns[t].back() != k))
                uns[t].push_back(k);
        }
    });
    std::vector<int> unsorted;
    for (auto &x : uns)
        for (int k : x)
            if (unsorted.empty() || unsorted.back() != k) unsorted.push_back(k);
    if (!unsorted.empty()) {
        if (ident) {
            ord.resize(nz);
            parallel_for(nz, [&](long long u) { ord[u] = u; });
            ident = false;
        }
        parallel_for((long long)unsorted.size(), [&](long long q) {
            const int k = unsorted[q];
            std::stable_sort(ord.begin() + bstart[k], ord.begin() + bstart[k + 1],
                             [&](long long x, long long y) { return in.mat[x] < in.mat[y]; });
        });
    }
    // the (block, matrix) buckets: a run starts at each block's first entry and where the matrix
    // changes; runs in block order, then matrix order
    struct Run { int k, mt; long long s0, s1; };   // one (block, matrix) bucket: entries s0 .. s1 - 1
    std::vector<std::vector<long long>> starts(U);
    run_chunks(U, [&](int t) {
        const long long lo = nz * t / U, hi = nz * (t + 1) / U;
        if (lo >= hi) return;
        int k = block_of(lo);
        for (long long u = lo; u < hi; u++) {
            while (u >= bstart[k + 1]) k++;
            if (u == bstart[k] || in.mat[entry(u)] != in.mat[entry(u - 1)]) starts[t].push_back(u);
        }
    });
    std::vector<Run> runs;
    std::vector<size_t> rstart(nb + 1, 0);
    {
        size_t R = 0;
        for (auto &x : starts) R += x.size();
        runs.reserve(R);
        int k = 0;
        for (auto &x : starts)
            for (long long u : x) {
                while (u >= bstart[k + 1]) k++;
                if (!runs.empty()) runs.back().s1 = u;
                runs.push_back({k, in.mat[entry(u)], u, nz});
            }
        for (const Run &r : runs) rstart[r.k + 1]++;
        for (int q = 0; q < nb; q++) rstart[q + 1] += rstart[q];
    }
    starts.clear();
    // per (block, matrix): merge duplicates, expand to both triangles, sort by position p + q n
    struct Bucket { std::vector<int> pos; std::vector<double> val; double ss = 0, sa = 0; };
    std::vector<Bucket> bk(runs.size());
    parallel_for((long long)runs.size(), [&](long long key) {
        const long long s0 = runs[key].s0, s1 = runs[key].s1;
        if (s0 == s1) return;
        const int k = runs[key].k;
        const int n = P.blk[k].n;
        const long long nn = (long long)n * n;
        if (nn <= 16 * (s1 - s0) + 4096) {
            // dense enough: scatter the upper entries into a per-thread n x n scratch (duplicates
            // summed in input order), then read both triangles out in position order (no sort)
            thread_local std::vector<double> acc;
            thread_local std::vector<char> mark;
            if ((long long)acc.size() < nn) { acc.assign(nn, 0.0); mark.assign(nn, 0); }
            for (long long u = s0; u < s1; u++) {
                const long long e = entry(u);
                int i, j;
                rc_here(e, i, j);
                if (i > j) std::swap(i, j);
                const long long q = (long long)j * n + i;
                acc[q] += in.v[e];
                mark[q] = 1;
            }
            Bucket &b = bk[key];
            b.pos.reserve(2 * (s1 - s0));
            b.val.reserve(2 * (s1 - s0));
            for (int q = 0; q < n; q++)
                for (int pp = 0; pp < n; pp++) {   // position pp + q n of the full matrix
                    const long long uk = pp <= q ? (long long)q * n + pp : (long long)pp * n + q;
                    if (!mark[uk] || acc[uk] == 0.0) continue;
                    const double v = acc[uk];
                    b.pos.push_back(pp + q * n);
                    b.val.push_back(v);
                    b.ss += v * v;
                    b.sa += std::fabs(v);
                }
            for (long long u = s0; u < s1; u++) {   // clear the scratch for the next bucket
                const long long e = entry(u);
                int i, j;
                rc_here(e, i, j);
                if (i > j) std::swap(i, j);
                const long long q = (long long)j * n + i;
                acc[q] = 0.0;
                mark[q] = 0;
            }
            return;
        }
        // sparse: counting sorts by column instead of comparison sorts.  The upper entries (p, q),
        // p <= q, go to column q in input order and then by row (insertion sort: a column holds few
        // entries), duplicates summed in input order; the full expansion is then written column by
        // column, the upper part (rows <= c, from column c's list) before the mirrored part (rows > c,
        // from the entries (c, q) in order of q): position order with no sort.
        thread_local std::vector<int> cnt;
        if ((int)cnt.size() < n + 1) cnt.assign(n + 1, 0);
        const long long ne = s1 - s0;
        thread_local std::vector<int> row, col, ur, uc, lo_cnt, up_start;
        thread_local std::vector<double> val, uv;
        thread_local std::vector<long long> cstart, wpos;
        if ((long long)row.size() < ne) {
            row.resize(ne); col.resize(ne); ur.resize(ne); uc.resize(ne); val.resize(ne); uv.resize(ne);
        }
        for (long long u = 0; u < ne; u++) {
            const long long e = entry(s0 + u);
            int i, j;
            rc_here(e, i, j);
            if (i > j) std::swap(i, j);
            cnt[j + 1]++;
            row[u] = i;
            col[u] = j;
            val[u] = in.v[e];
        }
        for (int c = 0; c < n; c++) cnt[c + 1] += cnt[c];
        for (long long u = 0; u < ne; u++) {   // stable scatter by column
            const int d = cnt[col[u]]++;
            ur[d] = row[u];
            uc[d] = col[u];
            uv[d] = val[u];
        }
        for (int c = n; c > 0; c--) cnt[c] = cnt[c - 1];   // cnt[c]: the start of column c again
        cnt[0] = 0;
        long long nu = 0;   // merged upper entries, in (column, row) order, written over ur/uc/uv
        for (int c = 0; c < n; c++) {
            const int b0 = cnt[c], b1 = cnt[c + 1];
            for (int a = b0 + 1; a < b1; a++) {   // stable insertion sort by row
                const int r = ur[a];
                const double v = uv[a];
                int z = a;
                while (z > b0 && ur[z - 1] > r) {
                    ur[z] = ur[z - 1];
                    uv[z] = uv[z - 1];
                    z--;
                }
                ur[z] = r;
                uv[z] = v;
            }
            for (int a = b0; a < b1;) {
                int w = a;
                double v = 0;
                while (w < b1 && ur[w] == ur[a]) v += uv[w++];   // duplicates summed in input order
                if (v != 0.0) {
                    ur[nu] = ur[a];
                    uc[nu] = c;
                    uv[nu] = v;
                    nu++;
                }
                a = w;
            }
        }
        for (int c = 0; c <= n; c++) cnt[c] = 0;
        // per column c: its upper entries (rows <= c), then the mirrors of the row-c entries
        lo_cnt.assign(n + 1, 0);
        up_start.assign(n + 1, 0);
        cstart.assign(n + 1, 0);
        for (long long u = 0; u < nu; u++)
            if (ur[u] != uc[u]) lo_cnt[ur[u] + 1]++;
        for (long long u = 0; u < nu; u++) up_start[uc[u] + 1]++;
        for (int c = 0; c < n; c++) cstart[c + 1] = cstart[c] + up_start[c + 1] + lo_cnt[c + 1];
        Bucket &b = bk[key];
        b.pos.resize(cstart[n]);
        b.val.resize(cstart[n]);
        wpos.assign(cstart.begin(), cstart.end() - 1);
        for (long long u = 0; u < nu; u++) {   // upper parts first (their columns in order)
            const long long d = wpos[uc[u]]++;
            b.pos[d] = ur[u] + uc[u] * n;
            b.val[d] = uv[u];
        }
        for (long long u = 0; u < nu; u++) {   // then the mirrors: entry (p, q), p < q, at row q of column p
            if (ur[u] == uc[u]) continue;
            const long long d = wpos[ur[u]]++;
            b.pos[d] = uc[u] + ur[u] * n;
            b.val[d] = uv[u];
        }
        for (size_t u = 0; u < b.val.size(); u++) {
            b.ss += b.val[u] * b.val[u];
            b.sa += std::fabs(b.val[u]);
        }
    });
    std::vector<double> nrm2(P.m, 0.0);
    double c2 = 0, c1 = 0;
    struct Piece { int k, t; size_t r; };   // bucket r is local constraint t of block k
    std::vector<Piece> pieces;
    for (int k = 0; k < nb; k++) {   // a block's buckets, in matrix order
        HBlock &B = P.blk[k];
        long long total = 0;
        B.cptr.assign(1, 0);
        for (size_t r = rstart[k]; r < rstart[k + 1]; r++) {
            Bucket &b = bk[r];
            if (runs[r].mt == 0) {
                B.Cpos = std::move(b.pos);
                B.Cval = std::move(b.val);
                for (auto &v : B.Cval) v = -v;   // C = -F0
                c2 += b.ss;
                c1 += b.sa;
                continue;
            }
            if (b.pos.empty()) continue;
            B.con.push_back(runs[r].mt - 1);
            nrm2[runs[r].mt - 1] += b.ss;
            total += (long long)b.pos.size();
            B.cptr.push_back(total);
            pieces.push_back({k, (int)B.con.size() - 1, r});
        }
        B.cpos.resize(total);
        B.cval.resize(total);
    }
    // problem_prepare (problem.c:1866-1910): row equilibration, b and C scaling
    P.normC2 = std::sqrt(c2);
    P.normC1 = c1;
    P.normb1 = P.normb2 = 0;
    for (int i = 0; i < P.m; i++) { P.normb1 += std::fabs(P.b0[i]); P.normb2 += P.b0[i] * P.b0[i]; }
    P.normb2 = std::sqrt(P.normb2);
    P.d.resize(P.m);
    for (int i = 0; i < P.m; i++) {
        P.d[i] = nrm2[i] > 0 ? 1.0 / std::sqrt(nrm2[i]) : 1.0;
        if (nrm2[i] == 0 && P.b[i] != 0) log_printf(1, "brisk: warning: constraint %d is empty but b != 0 (infeasible)\n", i + 1);
    }
    double nbv = 0;
    for (int i = 0; i < P.m; i++) nbv += P.d[i] * P.b[i] * P.d[i] * P.b[i];
    nbv = std::sqrt(nbv);
    P.bs = nbv > 1 ? nbv : 1.0;
    parallel_for((long long)pieces.size(), [&](long long q) {   // every block's buckets, each row scaled by d
        const Piece &pc = pieces[q];
        HBlock &B = P.blk[pc.k];
        const Bucket &b = bk[pc.r];
        const double dq = P.d[B.con[pc.t]];
        std::copy(b.pos.begin(), b.pos.end(), B.cpos.begin() + B.cptr[pc.t]);
        double *out = B.cval.data() + B.cptr[pc.t];
        for (size_t u = 0; u < b.val.size(); u++) out[u] = b.val[u] * dq;
    });
    for (int i = 0; i < P.m; i++) P.b[i] *= P.d[i];
    P.du.resize(P.m);
    for (int i = 0; i < P.m; i++) P.du[i] = P.bs / P.d[i];
    P.cs = P.normC2 > 1 ? P.normC2 : 1.0;
    for (int i = 0; i < P.m; i++) P.b[i] /= P.bs;
    for (auto &B : P.blk)
        for (auto &v : B.Cval) v /= P.cs;
    return 0;
}


// ---------------------------------------------------------------------------------------------
// output
// ---------------------------------------------------------------------------------------------
static int (*g_print)(const char *, int) = nullptr;
void set_print_hook(int (*f)(const char *, int)) { g_print = f; }
void log_printf(int is_err, const char *fmt, ...) {
    char buf[2048];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (g_print) g_print(buf, is_err);
    else fputs(buf, is_err ? stderr : stdout);
}

// ---------------------------------------------------------------------------------------------
// the GPU solver
// ---------------------------------------------------------------------------------------------
namespace {

struct DevArrays {   // per block
    double *X, *Z, *Zi, *LX, *LZ, *LiX, *LiZ, *dX, *dZ, *F, *Fd, *R0, *G, *Q, *W, *T, *Xb, *Zb, *Bm;
    // the NT direction (allocated for it only): the scaling G (W = G G' is kept in Zi), the
    // scaled predictor directions and the scaled rhs (solver.c:7803-7810)
    double *NG, *dXt, *dZt, *Rt;
    double *dinvX, *dinvZ;
    int *flags;
};
// the n x n members, each one concatenation over the blocks
static double *DevArrays::*const kCatMembers[] = {
    &DevArrays::X,  &DevArrays::Z,  &DevArrays::Zi, &DevArrays::LX, &DevArrays::LZ, &DevArrays::LiX, &DevArrays::LiZ,
    &DevArrays::dX, &DevArrays::dZ, &DevArrays::F,  &DevArrays::Fd, &DevArrays::R0, &DevArrays::G,   &DevArrays::Q,
    &DevArrays::W,  &DevArrays::T,  &DevArrays::Xb, &DevArrays::Zb, &DevArrays::Bm};
static double *DevArrays::*const kNtMembers[] = {&DevArrays::NG, &DevArrays::dXt, &DevArrays::dZt, &DevArrays::Rt};

// Device memory of one solve.  Stand-alone solves allocate with cudaMalloc and own a stream; the
// batch workers hand in an arena (one allocation and one stream per worker, reused by every
// instance it solves) so that no cudaMalloc / cudaFree runs between instances.
struct Gpu {
    std::vector<void *> allocs;
    cudaStream_t st = nullptr;
    Arena *arena = nullptr;
    template <typename T>
    T *alloc(size_t count) {
        if (count == 0) count = 1;
        if (arena) {
            const size_t off = (arena->used + 255) & ~(size_t)255;
            if (off + count * sizeof(T) > arena->cap) {
                arena->need = std::max(arena->need, off + count * sizeof(T));
                return nullptr;
            }
            arena->used = off + count * sizeof(T);
            return (T *)(arena->base + off);
        }
        const size_t bytes = (count * sizeof(T) + 255) & ~(size_t)255;
        if (bytes > kSlabLarge) {   // large arrays: their own allocation
            void *p = nullptr;
            if (!pool_alloc(&p, bytes)) return nullptr;
            allocs.push_back(p);
            return (T *)p;
        }
        // small ones (a problem of many blocks asks for thousands) from 64 MB slabs
        if (!slab || slab_used + bytes > kSlab) {
            void *p = nullptr;
            if (!pool_alloc(&p, kSlab)) return nullptr;
            allocs.push_back(p);
            slab = (unsigned char *)p;
            slab_used = 0;
        }
        T *r = (T *)(slab + slab_used);
        slab_used += bytes;
        return r;
    }
    static constexpr size_t kSlab = (size_t)64 << 20, kSlabLarge = (size_t)4 << 20;
    // Stand-alone solves and lockstep batches allocate from the device's stream-ordered pool on
    // their own stream; the pool keeps up to 32 GB after a solve (release threshold), so the next
    // solve of a similar problem reuses that memory instead of mapping new memory (about 0.1 s per
    // rand400 solve, 1 s for the 23 GB of a 4096-instance batch).
    bool pool_alloc(void **p, size_t bytes) {
        static std::once_flag once[64];
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) return false;
        if (dev >= 0 && dev < 64)
            std::call_once(once[dev], [dev] {
                cudaMemPool_t pool;
                if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
                    uint64_t thr = (uint64_t)32 << 30;
                    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
                }
            });
        return cudaMallocAsync(p, bytes, st) == cudaSuccess;
    }
    unsigned char *slab = nullptr;
    size_t slab_used = 0;
    // Pinned host memory for the small device-to-host reads of the loop (from the arena's
    // pinned buffer in a batch worker, where it fits).
    std::vector<void *> hallocs;
    template <typename T>
    T *host_alloc(size_t count) {
        if (count == 0) count = 1;
        if (arena && arena->hbase) {
            const size_t off = (arena->hused + 63) & ~(size_t)63;
            if (off + count * sizeof(T) <= arena->hcap) {
                arena->hused = off + count * sizeof(T);
                return (T *)(arena->hbase + off);
            }
        }
        void *p = nullptr;
        if (cudaMallocHost(&p, count * sizeof(T)) != cudaSuccess) return nullptr;
        hallocs.push_back(p);
        return (T *)p;
    }
    ~Gpu() {
        if (st) cudaStreamSynchronize(st);
        for (void *p : hallocs) cudaFreeHost(p);
        for (void *p : allocs) cudaFreeAsync(p, st);
        if (st && !allocs.empty()) cudaStreamSynchronize(st);
        if (st && !arena) cudaStreamDestroy(st);
    }
};

#define RC(call)                                   \
    do {                                           \
        int rc_ = (call);                          \
        if (rc_) throw GpuFail{rc_, __LINE__};     \
    } while (0)
#define CU(call)                                                                  \
    do {                                                                          \
        cudaError_t e_ = (call);                                                  \
        if (e_ != cudaSuccess) throw GpuFail{BGPU_ERR_CUDA, __LINE__, e_};        \
    } while (0)

struct GpuFail {
    int rc;
    int line;
    cudaError_t ce = cudaSuccess;
};

class Solver {
  public:
    Solver(HProblem &P, const Options &opt, Arena *arena = nullptr) : P(P), opt(opt), m(P.m), nb((int)P.blk.size()) {
        g.arena = arena;
    }
    void setup();                 // upload the scaled problem and allocate the device state
    int run(ResultData &res);     // one solve from the resident data
    int run_hsd(ResultData &res); // the same by the self-dual embedding (HKM)
    void start_sdpt3(bool unit = false);   // unit: X = Z = I (the embedding's start)
    void set_options(const Options &o) { opt = o; }
    ~Solver() {
        schol::release(sp_f);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (evs0) cudaEventDestroy(evs0);
        if (evs1) cudaEventDestroy(evs1);
    }
    double upload_bytes = 0;

  private:
    HProblem &P;
    Options opt;
    int m, nb;
    Gpu g;
    std::vector<DevBlock> db;
    std::vector<DevArrays> da;
    std::vector<char> dense_route;   // per block: the dense Schur route (Ad resident)
    std::vector<LowRankDev> lowrank;    // per block: the low-rank route's factors (R > 0 when taken)
    void setup_lowrank(int k);
    // Schur complement
    double *M = nullptr, *Lm = nullptr, *dinvM = nullptr, *Dsc = nullptr;
    // the supernodal sparse factor of M (use_sparse): symbolic analysis and device factor
    bool use_sparse = false;
    schol::Analysis sp_an;
    schol::Factor sp_f;
    void choose_sparse();
    float *Mf = nullptr, *dinvMf = nullptr;
    int *mflags = nullptr, *d_info = nullptr, *d_err = nullptr;
    double *d_pmin = nullptr;
    double *dv_in = nullptr, *dv_out = nullptr;   // m (or n) vectors
    float *fv = nullptr;
    double *dots_out = nullptr, *dots_scratch = nullptr;
    const double **dots_a = nullptr, **dots_b = nullptr;
    double *h_dots = nullptr;
    void *ws = nullptr;
    size_t ws_bytes = 0;
    // blocks of order <= SMALL_N_MAX run through the batched one-CTA-per-block kernels (small.cu)
    std::vector<int> small_ids, big_ids;
    int *d_sns = nullptr, *d_sinfo = nullptr, *h_sinfo = nullptr;
    double *d_slam = nullptr, *h_slam = nullptr;
    // the step-length Lanczos of the blocks of order > SMALL_N_MAX: the start vector (its first n
    // entries for a block of order n), the Krylov basis and the state in device memory, and a
    // pinned copy of the state for the checkpoints
    double *lz_q0 = nullptr, *lz_Q = nullptr;
    LanczosState *lz_st = nullptr, *h_lz = nullptr;
    std::vector<std::pair<double *DevArrays::*, double **>> stab;   // device pointer tables per array kind
    double **tab(double *DevArrays::*mem);
    // C = alpha A B (column-major n x n) on every block: per-block DMMA GEMMs for the large
    // blocks, one batched launch for the small ones
    void mul_all(double alpha, double *DevArrays::*A, double *DevArrays::*B, double *DevArrays::*C);
    // the NT direction (solver.c:7803-8090; -dir auto picks it by the rule of solver.c:13585-13591)
    bool nt_mode = false;
    double *nlam = nullptr;                  // the blocks' lam, block k's from loff[k]
    std::vector<long long> loff;
    long long *d_loff = nullptr;
    int *d_ntflag = nullptr, *h_ntflag = nullptr, *d_ntinfo = nullptr, *h_ntinfo = nullptr;
    double **d_lamtab = nullptr;             // the small blocks' lam pointers
    int small_nmax = 1;
    int nt_sweeps = 0;                       // the most Jacobi sweeps of a large block this iteration
    bool nt_scaling();                       // G, lam and W (in Zi) for every block; false: a block failed
    void nt_toZ(double *DevArrays::*D, double *DevArrays::*out);     // out = sym(G' D G)
    void nt_fromS(double *DevArrays::*D, double *DevArrays::*out);   // out = sym(G D G')
    void mul_sym_all(double *DevArrays::*A, double *DevArrays::*B, double *DevArrays::*C);   // C = sym(A B)
    // the matrices the assembly and the HKM-style products take as X and Z^-1: X and Z^-1, or W and
    // W under NT (the reference's nt_view, solver.c:7813-7819)
    double *DevArrays::*xmem() const { return nt_mode ? &DevArrays::Zi : &DevArrays::X; }
    int chunk = 32, chunk64 = 32, chunk_oz = 32, asm_prec = 0;
    int chunk_fp64(int) const { return chunk64; }
    int epoch = 0;
    // factor state (Schur in solver.c:4511-4568)
    bool allow_float = false, want_double = false, is_float = false, reg_hint = false;
    // the sparse factor in FP32 while mu >= mu_switch (-mixed as for the dense factor)
    bool sparse_float = false;
    // the pattern of the sparse M (both triangles and the diagonal, rows ascending): the FP64
    // residual product reads only these entries of the dense copy
    long long *d_prow = nullptr;
    int *d_pcol = nullptr;
    double reg = 0, reg_ok = 0, min_pivot = 1;
    int nfloat = 0, nfactor = 0, pcg_iters = 0;
    double mu_now = 1e300;
    Timings tm;
    double schur_flops = 0, schur_dev_time = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evs0 = nullptr, evs1 = nullptr;

    void upload_block(int k);
    // reductions
    void dots(int nq, const double *const *a, const double *const *b, long long n, double *out);
    // operators
    // The blocks' n x n arrays are stored one after another: block k's at boff[k] of each
    // concatenation (cat.X, cat.Z, ..., Ccat, Icat = I), so element-wise work and inner products
    // over all blocks are one launch each; gall holds every constraint's entries at concatenated
    // positions (the block's own arrays when there is one block).
    std::vector<long long> boff;
    long long Ntot2 = 0;
    DevArrays cat{};
    double *Ccat = nullptr, *Icat = nullptr;
    long long *d_boff = nullptr;
    int *d_bn = nullptr, *d_bsmall = nullptr;   // block orders; 1 for the blocks of order <= SMALL_N_MAX
    double *d_bval = nullptr;                   // one value per block (scratch)
    const long long **d_ppt = nullptr;
    const int **d_pct = nullptr;
    const double **d_pvt = nullptr;
    DevBlock gall;
    void build_gall();
    // many small blocks (n <= SB_NMAX, two or more): assembled by one kernel per colour class of
    // blocks that share no constraint
    std::vector<char> in_sb;
    std::vector<int> sb_coff, sb_nmax;   // colour c: d_sb_list[sb_coff[c] .. sb_coff[c+1]), its largest n
    std::vector<int> sb_cmax;            // ... and its largest constraint count
    int *d_sb_list = nullptr, *d_sb_ncon = nullptr;
    const int **d_sb_con = nullptr, **d_sb_cpos = nullptr;
    const long long **d_sb_cptr = nullptr;
    const double **d_sb_cval = nullptr;
    // LP blocks as given: the LP route (one launch per LP block), their order-1 blocks marked in_sb
    struct LpGroup { int q0 = 0; LpGroupDev dev; };
    std::vector<LpGroup> lp_groups;
    void setup_lp_groups();
    void setup_small_schur();
    void assemble_small(const double *Xc, const double *Zc);
    void aop_cat(const double *D, std::vector<double> &out);                                    // out = A(D)
    void atop_cat(const std::vector<double> &y, double alpha, double beta, double *F);         // F = a A'y + b F
    void sym_cat(const double *G, double s, double a, const double *x, double b, const double *y, double *out);
    void dots_cat(int nq, const double *const *a, const double *const *b, double *out) { dots(nq, a, b, Ntot2, out); }
    void lincomb_cat(double a, const double *x, double b, const double *y, double c, const double *z, double *out) {
        RC(ew_lincomb(g.st, Ntot2, a, x, b, y, c, z, out));
    }
    void gemm(int akm, int bkm, int n, double alpha, const double *A, long long lda, const double *B, long long ldb,
              double beta, double *C) {
        RC(gemm_f64(g.st, akm, bkm, n, n, n, alpha, A, lda, 0, B, ldb, 0, beta, C, n, 0, 1, 0));
    }
    // C = alpha * A B with A, B column-major n x n
    void mul(int n, double alpha, const double *A, const double *B, double *C) { gemm(0, 1, n, alpha, A, n, B, n, 0.0, C); }
    void zinv(int k);
    int chol(int n, double *L, double *dinv);   // returns info
    void inv_from_chol(int n, const double *L, const double *dinv, double *Li);
    // Schur
    void assemble(std::vector<double> &dummy);
    int factor();
    void prec(const std::vector<double> &r, std::vector<double> &z);
    void schur_mv(const std::vector<double> &x, std::vector<double> &y);
    // y = A(Z^-1 A'(x) X): the Newton system's operator in FP64 without the assembled M (the
    // residual of the mixed path, whose M is FP32-accurate)
    void newton_mv(const std::vector<double> &x, std::vector<double> &y);
    void mv(const std::vector<double> &x, std::vector<double> &y) {
        if (m_exact) schur_mv(x, y);
        else newton_mv(x, y);
    }
    bool m_exact = true;      // M was assembled in FP64 (the residual may use it)
    bool asm_fp64 = false;    // the mixed path turned to its late assembly
    bool late_exact = false;  // ... and from its preconditioner-grade late form to the FP64-accurate one
    int cur_prec = 0;         // the last assembly's precision code (schur_assemble's)
    char asm_label[16] = "fp64";   // the last assembly's precision (the -vv log)
    // the precision of the next assembly: the 3xTF32 path's late form once asm_fp64 is set (with
    // fewer than 8 Ozaki slices a preconditioner-grade M, until late_exact turns it to 8 slices)
    int next_prec() const {
        if (asm_prec != 1) return asm_prec;
        if (!asm_fp64) return 1;
        const int late = opt.late_prec;
        return (late_exact && late != 0) ? 2 : late;
    }
    static bool prec_exact(int p) { return p == 0 || p == 2; }
    // the mixed path's response to a late M that no longer preconditions the FP64 operator: from
    // 3xTF32 to the late form; from a preconditioner-grade late form to the FP64-accurate one.
    // Returns false when nothing more accurate is left.
    bool raise_precision() {
        if (asm_prec != 1) return false;
        if (!asm_fp64) { asm_fp64 = true; return true; }
        if (!late_exact && !prec_exact(opt.late_prec)) { late_exact = true; return true; }
        return false;
    }
    double schur_solve(const std::vector<double> &rhs, std::vector<double> &x, double tol_rel);
    // step length
    double maxstep(int primal, int K);
    double lanczos(int n, const double *Bm, int K);
    int try_step(int primal, double *alpha, double from = 0.0);
    void least_squares_start(std::vector<double> &y);
    // final measures
    void final_measures(const std::vector<double> &y, ResultData &res);
};

void Solver::dots(int nq, const double *const *a, const double *const *b, long long n, double *out) {
    CU(cudaMemcpyAsync(dots_a, a, sizeof(double *) * nq, cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(dots_b, b, sizeof(double *) * nq, cudaMemcpyHostToDevice, g.st));
    RC(dots_f64(g.st, nq, dots_a, dots_b, n, dots_out, dots_scratch));
    CU(cudaMemcpyAsync(h_dots, dots_out, sizeof(double) * nq, cudaMemcpyDeviceToHost, g.st));
    CU(cudaStreamSynchronize(g.st));
    for (int q = 0; q < nq; q++) out[q] = h_dots[q];
}

// The low-rank route for block k (lowrank_block, problem.c:972-1075, with this build's own
// factorization and cost rule, lowrank.cu): blocks above the small-block size whose every
// constraint has low rank, where P and Q (4 n^2 R + 4 n R^2 flops) cost under half of the
// row-product route's 2 n^3 per constraint, and P and Q fit in 4 GB.
void Solver::setup_lowrank(int k) {
    const HBlock &B = P.blk[k];
    const int n = B.n, nc = (int)B.con.size();
    if (opt.lowrank == 0 || nc == 0 || n <= SMALL_N_MAX) return;
    const double nd = n, route = 2.0 * nd * nd * nd * nc;
    auto cost = [&](double R) { return 4.0 * nd * nd * R + 4.0 * nd * R * R; };
    if (opt.lowrank < 0 && cost((double)nc) >= 0.5 * route) return;   // every constraint has rank >= 1
    int max_rank = (int)std::min(16384.0, std::sqrt(4e9 / 16.0));
    std::vector<int> off;
    std::vector<double> W, sig;
    if (!lowrank_factor_block(n, nc, B.cptr.data(), B.cpos.data(), B.cval.data(), off, W, sig, max_rank)) return;
    const int R = off[nc];
    if (R == 0 || (opt.lowrank < 0 && cost((double)R) >= 0.5 * route)) return;
    LowRankDev &L = lowrank[k];
    L.n = n;
    L.ncon = nc;
    L.W = g.alloc<double>((size_t)n * R);
    L.sig = g.alloc<double>(R);
    L.off = g.alloc<int>(nc + 1);
    L.XW = g.alloc<double>((size_t)n * R);
    L.P = g.alloc<double>((size_t)R * R);
    L.Q = g.alloc<double>((size_t)R * R);
    if (!L.W || !L.sig || !L.off || !L.XW || !L.P || !L.Q) throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
    CU(cudaMemcpyAsync(L.W, W.data(), sizeof(double) * (size_t)n * R, cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(L.sig, sig.data(), sizeof(double) * R, cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(L.off, off.data(), sizeof(int) * (nc + 1), cudaMemcpyHostToDevice, g.st));
    CU(cudaStreamSynchronize(g.st));   // the host factors are freed on return
    L.R = R;
    upload_bytes += (double)n * R * 8 + (double)R * 8 + (double)(nc + 1) * 4;
    if (opt.verbose > 1)
        log_printf(0, "   [block %d: low-rank route, %d constraints of total rank %d (%.2e flops an assembly against "
                      "%.2e)]\n", k + 1, nc, R, cost((double)R), route);
}

void Solver::upload_block(int k) {
    const HBlock &B = P.blk[k];
    DevBlock &d = db[k];
    const int n = B.n;
    const long long nn = (long long)n * n;
    d.n = n;
    d.ncon = (int)B.con.size();
    d.ne = (long long)B.cpos.size();
    d.con = g.alloc<int>(d.ncon);
    d.cptr = g.alloc<long long>(d.ncon + 1);
    d.cpos = g.alloc<int>(d.ne);
    d.cval = g.alloc<double>(d.ne);
    d.ccol = g.alloc<int>((size_t)d.ncon * (n + 1));
    d.pptr = g.alloc<long long>(nn + 1);
    d.pcon = g.alloc<int>(d.ne);
    d.pval = g.alloc<double>(d.ne);
    d.C = Ccat + boff[k];
    if (!d.con || !d.cptr || !d.cpos || !d.cval || !d.ccol || !d.pptr || !d.pcon || !d.pval || !d.C)
        throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
    CU(cudaMemcpyAsync(d.con, B.con.data(), sizeof(int) * d.ncon, cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(d.cptr, B.cptr.data(), sizeof(long long) * (d.ncon + 1), cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(d.cpos, B.cpos.data(), sizeof(int) * d.ne, cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(d.cval, B.cval.data(), sizeof(double) * d.ne, cudaMemcpyHostToDevice, g.st));
    RC(schur_colptr(g.st, d));
    // upper-triangle lists for the packed symmetric gather and the Gram matrix
    if (d.ncon > 0) {
        d.uptr = g.alloc<long long>(d.ncon + 1);
        int *cnt = g.alloc<int>(d.ncon);
        if (!d.uptr || !cnt) throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
        RC(schur_upper_ptr(g.st, d, cnt));
        d.nu = 0;   // the entries p <= q (the device count, kept on the host: no read-back)
        for (long long e = 0; e < d.ne; e++) {
            const int pos = B.cpos[e], q = pos / n;
            d.nu += pos - q * n <= q;
        }
        d.upos = g.alloc<int>(d.nu);
        d.uval = g.alloc<double>(d.nu);
        if (!d.upos || !d.uval) throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
        RC(schur_upper(g.st, d));
    }
    // the dense route: constraints averaging >= 2 % of the n^2 entries (the reference's dense
    // candidates, problem.c:1299), n >= 8, and their dense copies within 8 GB
    {
        const double avg = d.ncon > 0 ? (double)d.ne / d.ncon : 0.0;
        const double bytes = (double)d.ncon * n * n * sizeof(double);
        bool dense = opt.route == 1 || (opt.route < 0 && n >= 8 && avg >= 0.02 * (double)n * n);
        if (dense && bytes > 8e9) dense = false;
        setup_lowrank(k);
        if (lowrank[k].R > 0) dense = false;
        dense_route[k] = dense;
        if (dense && d.ncon > 0) {
            d.Ad = g.alloc<double>((size_t)d.ncon * n * n);
            if (!d.Ad) throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
            RC(schur_densify(g.st, d));
        }
    }
    // position-major copy (A'(y) without atomics): entries of each position in constraint order, by
    // a stable counting sort on the host's threads.  Thread r counts the positions of a contiguous run
    // of constraints; the counts become each thread's offset inside each position, so a position's
    // entries keep the constraints' order.
    std::vector<long long, NoInitAlloc<long long>> pptr(nn + 1);
    std::vector<int, NoInitAlloc<int>> pcon(d.ne);
    std::vector<double, NoInitAlloc<double>> pval(d.ne);
    {
        int T = tl_serial || d.ne < 100000 ? 1 : (int)std::max(1u, std::min(std::thread::hardware_concurrency(), 32u));
        while (T > 1 && (double)T * nn * sizeof(int) > 256e6) T--;   // the counts: at most 256 MB
        std::vector<int> t0(T + 1, d.ncon);
        t0[0] = 0;
        for (int r = 1, t = 0; r < T; r++) {
            const long long target = d.ne * r / T;
            while (t < d.ncon && B.cptr[t] < target) t++;
            t0[r] = t;
        }
        std::vector<std::vector<int>> cnt(T);
        auto on_threads = [&](int count, const std::function<void(int)> &f) {
            if (count == 1) { f(0); return; }
            std::vector<std::thread> th;
            for (int r = 0; r < count; r++) th.emplace_back(f, r);
            for (auto &x : th) x.join();
        };
        on_threads(T, [&](int r) {
            cnt[r].assign(nn, 0);
            for (long long e = B.cptr[t0[r]]; e < B.cptr[t0[r + 1]]; e++) cnt[r][B.cpos[e]]++;
        });
        const long long pchunk = (nn + T - 1) / T;
        on_threads(T, [&](int r) {   // per position: the total, and each thread's offset in place of its count
            const long long p1 = std::min((long long)nn, (r + 1) * pchunk);
            for (long long p = r * pchunk; p < p1; p++) {
                int rel = 0;
                for (int q = 0; q < T; q++) {
                    const int c = cnt[q][p];
                    cnt[q][p] = rel;
                    rel += c;
                }
                pptr[p + 1] = rel;
            }
        });
        pptr[0] = 0;
        for (long long p = 0; p < nn; p++) pptr[p + 1] += pptr[p];
        on_threads(T, [&](int r) {
            std::vector<int> &off = cnt[r];
            for (int t = t0[r]; t < t0[r + 1]; t++)
                for (long long e = B.cptr[t]; e < B.cptr[t + 1]; e++) {
                    const int pos = B.cpos[e];
                    const long long q = pptr[pos] + off[pos]++;
                    pcon[q] = B.con[t];
                    pval[q] = B.cval[e];
                }
        });
    }
    CU(cudaMemcpyAsync(d.pptr, pptr.data(), sizeof(long long) * (nn + 1), cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(d.pcon, pcon.data(), sizeof(int) * d.ne, cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(d.pval, pval.data(), sizeof(double) * d.ne, cudaMemcpyHostToDevice, g.st));
    std::vector<double> C(nn, 0.0);
    for (size_t e = 0; e < B.Cpos.size(); e++) C[B.Cpos[e]] += B.Cval[e];
    CU(cudaMemcpyAsync(d.C, C.data(), sizeof(double) * nn, cudaMemcpyHostToDevice, g.st));
    upload_bytes += (double)sizeof(int) * d.ncon + sizeof(long long) * (d.ncon + 1) + (sizeof(int) + sizeof(double)) * 2.0 * d.ne +
                    sizeof(long long) * (nn + 1.0) + sizeof(double) * (double)nn;

    DevArrays &a = da[k];
    for (double *DevArrays::*mem : kCatMembers) a.*mem = cat.*mem + boff[k];
    if (nt_mode)
        for (double *DevArrays::*mem : kNtMembers) a.*mem = cat.*mem + boff[k];
    const int nblk64 = ceil_div(n, TRI_NB);
    a.dinvX = g.alloc<double>((size_t)nblk64 * TRI_NB * TRI_NB);
    a.dinvZ = g.alloc<double>((size_t)nblk64 * TRI_NB * TRI_NB);
    a.flags = g.alloc<int>(nblk64);
    if (!a.dinvX || !a.dinvZ || !a.flags) throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
    CU(cudaMemsetAsync(a.flags, 0, sizeof(int) * nblk64, g.st));
    // (the host vectors above may go: a copy from pageable memory has staged them when it returns)
}

void Solver::setup() {
    const double t0 = wtime();
    CU(cudaSetDevice(opt.device));
    if (g.arena) {
        g.st = (cudaStream_t)g.arena->st;
        g.arena->used = 0;
        g.arena->hused = 0;
    } else {
        CU(cudaStreamCreateWithFlags(&g.st, cudaStreamNonBlocking));
    }
    CU(cudaEventCreate(&ev0));
    CU(cudaEventCreate(&ev1));
    CU(cudaEventCreate(&evs0));
    CU(cudaEventCreate(&evs1));
    db.resize(nb);
    da.resize(nb);
    dense_route.assign(nb, 0);
    lowrank.assign(nb, LowRankDev{});
    int nmax = 1;
    const double t1 = wtime();
    boff.assign(nb + 1, 0);
    loff.assign(nb + 1, 0);
    for (int k = 0; k < nb; k++) {
        boff[k + 1] = boff[k] + (long long)P.blk[k].n * P.blk[k].n;
        loff[k + 1] = loff[k] + P.blk[k].n;
    }
    Ntot2 = boff[nb];
    {   // the direction: -dir auto takes NT when its dense work (15 sum n^3) is below a quarter of the
        // Schur work (m^3/3 + 5 sum n^3) or negligible (<= 1e8 flops), solver.c:13585-13591
        double n3 = 0;
        for (auto &B : P.blk) n3 += (double)B.n * B.n * B.n;
        const double mm = m;
        nt_mode = opt.direction == 1 ||
                  (opt.direction < 0 && (15.0 * n3 < 0.25 * (mm * mm * mm / 3.0 + 5.0 * n3) || 15.0 * n3 <= 1e8));
    }
    for (double *DevArrays::*mem : kCatMembers) {
        cat.*mem = g.alloc<double>(Ntot2);
        if (!(cat.*mem)) throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
    }
    if (nt_mode) {
        for (double *DevArrays::*mem : kNtMembers) {
            cat.*mem = g.alloc<double>(Ntot2);
            if (!(cat.*mem)) throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
        }
        nlam = g.alloc<double>(loff[nb]);
        d_loff = g.alloc<long long>(nb + 1);
        d_ntflag = g.alloc<int>(1);
        d_ntinfo = g.alloc<int>(1);
        h_ntflag = g.host_alloc<int>(1);
        h_ntinfo = g.host_alloc<int>(1);
        if (!nlam || !d_loff || !d_ntflag || !d_ntinfo || !h_ntflag || !h_ntinfo) throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
        CU(cudaMemcpyAsync(d_loff, loff.data(), sizeof(long long) * (nb + 1), cudaMemcpyHostToDevice, g.st));
    }
    Ccat = g.alloc<double>(Ntot2);
    Icat = g.alloc<double>(Ntot2);
    d_boff = g.alloc<long long>(nb + 1);
    d_bn = g.alloc<int>(nb);
    d_bval = g.alloc<double>(nb);
    d_bsmall = g.alloc<int>(nb);
    if (!Ccat || !Icat || !d_boff || !d_bn || !d_bval || !d_bsmall) throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
    {
        std::vector<int> bn(nb), bsm(nb);
        std::vector<double> ones(nb, 1.0);
        for (int k = 0; k < nb; k++) bn[k] = P.blk[k].n;
        for (int k = 0; k < nb; k++) bsm[k] = P.blk[k].n <= SMALL_N_MAX;
        CU(cudaMemcpyAsync(d_bsmall, bsm.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, g.st));
        CU(cudaMemcpyAsync(d_boff, boff.data(), sizeof(long long) * (nb + 1), cudaMemcpyHostToDevice, g.st));
        CU(cudaMemcpyAsync(d_bn, bn.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, g.st));
        CU(cudaMemcpyAsync(d_bval, ones.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, g.st));
        RC(ew_scaled_identity_blocks(g.st, nb, d_bn, d_boff, Ntot2, d_bval, nullptr, Icat));
        CU(cudaStreamSynchronize(g.st));
    }
    for (int k = 0; k < nb; k++) {
        upload_block(k);
        nmax = std::max(nmax, P.blk[k].n);
    }
    build_gall();
    if (opt.verbose > 1) log_printf(0, "   [device context %.3fs, block upload %.3fs]\n", t1 - t0, wtime() - t1);
    for (int k = 0; k < nb; k++) (P.blk[k].n <= SMALL_N_MAX ? small_ids : big_ids).push_back(k);
    setup_small_schur();
    if (!small_ids.empty()) {
        const int ns = (int)small_ids.size();
        std::vector<int> nsz(ns);
        for (int i = 0; i < ns; i++) nsz[i] = P.blk[small_ids[i]].n;
        d_sns = g.alloc<int>(ns);
        d_sinfo = g.alloc<int>(ns);
        d_slam = g.alloc<double>(ns);
        if (!d_sns || !d_sinfo || !d_slam) throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
        CU(cudaMemcpyAsync(d_sns, nsz.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, g.st));
        for (int i = 0; i < ns; i++) small_nmax = std::max(small_nmax, nsz[i]);
        if (nt_mode) {
            std::vector<double *> lp(ns);
            for (int i = 0; i < ns; i++) lp[i] = nlam + loff[small_ids[i]];
            d_lamtab = g.alloc<double *>(ns);
            if (!d_lamtab) throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
            CU(cudaMemcpyAsync(d_lamtab, lp.data(), sizeof(double *) * ns, cudaMemcpyHostToDevice, g.st));
        }
        CU(cudaStreamSynchronize(g.st));
        h_sinfo = g.host_alloc<int>(ns);
        h_slam = g.host_alloc<double>(ns);
        if (!h_sinfo || !h_slam) throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
    }
    const size_t mm = (size_t)m * m;
    M = g.alloc<double>(mm);
    if (!M) throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
    const int mb64 = ceil_div(std::max(m, 1), TRI_NB);
    dinvM = g.alloc<double>((size_t)mb64 * TRI_NB * TRI_NB);
    Dsc = g.alloc<double>(m);
    mflags = g.alloc<int>(mb64);
    d_info = g.alloc<int>(1);
    d_err = g.alloc<int>(1);
    d_pmin = g.alloc<double>(1);
    const int vlen = std::max(m, nmax);
    dv_in = g.alloc<double>(vlen);
    dv_out = g.alloc<double>(vlen);
    fv = g.alloc<float>(vlen);
    dots_out = g.alloc<double>(16);
    dots_scratch = g.alloc<double>(16 * 128);
    dots_a = (const double **)g.alloc<double *>(16);
    dots_b = (const double **)g.alloc<double *>(16);
    if (!dinvM || !Dsc || !mflags || !d_info || !d_err || !d_pmin || !dv_in || !dv_out || !fv || !dots_out ||
        !dots_scratch || !dots_a || !dots_b)
        throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
    CU(cudaMemsetAsync(mflags, 0, sizeof(int) * mb64, g.st));
    CU(cudaMemsetAsync(d_err, 0, sizeof(int), g.st));
    h_dots = g.host_alloc<double>(16);
    if (!h_dots) throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
    if (!big_ids.empty()) {
        int nbig = 1;
        for (int k : big_ids) nbig = std::max(nbig, P.blk[k].n);
        std::vector<double> q0(nbig);
        for (int i = 0; i < nbig; i++) q0[i] = 1.0 + 0.5 * std::sin(1.7 * i + 0.3);
        lz_q0 = g.alloc<double>(nbig);
        lz_Q = g.alloc<double>((size_t)31 * nbig);
        lz_st = g.alloc<LanczosState>(1);
        h_lz = g.host_alloc<LanczosState>(1);
        if (!lz_q0 || !lz_Q || !lz_st || !h_lz) throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
        CU(cudaMemcpyAsync(lz_q0, q0.data(), sizeof(double) * nbig, cudaMemcpyHostToDevice, g.st));
        CU(cudaStreamSynchronize(g.st));
    }
    choose_sparse();
    allow_float = !use_sparse && (opt.mixed > 0 || (opt.mixed < 0 && m >= 1000));
    // FP32 fronts only when asked for (-mixed 1): the fronts of these problems are small and
    // latency-bound, so FP32 saves no factor time and costs PCG steps (mom700: 0.153 s FP64,
    // 0.175 s with FP32 fronts early)
    sparse_float = use_sparse && opt.mixed > 0;
    asm_prec = opt.asm_prec < 0 ? 0 : opt.asm_prec;
    if (asm_prec == 1 && !use_sparse) allow_float = true;   // the 3xTF32 path factors in FP32 until mu_switch
    if (allow_float) {
        Mf = g.alloc<float>(mm);
        dinvMf = g.alloc<float>((size_t)mb64 * TRI_NB * TRI_NB);
        if (!Mf || !dinvMf) throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
    }
    chunk = opt.chunk > 0 ? opt.chunk : schur_chunk_default(nmax, asm_prec);
    chunk64 = opt.chunk > 0 ? opt.chunk : schur_chunk_default(nmax, 0);
    chunk_oz = opt.chunk > 0 ? opt.chunk : schur_chunk_default(nmax, 2);
    ws_bytes = std::max(schur_ws_bytes(nmax, chunk, asm_prec), schur_ws_bytes(nmax, chunk64, 0));
    if (asm_prec == 2 || (asm_prec == 1 && (opt.late_prec & 0xff) == 2))   // (8 slices: the most workspace)
        ws_bytes = std::max(ws_bytes, schur_ws_bytes(nmax, chunk_oz, 2));
    for (int k = 0; k < nb; k++)
        if (dense_route[k])
            ws_bytes = std::max(ws_bytes, std::max(schur_dense_ws_bytes(db[k].n, db[k].ncon, chunk, asm_prec),
                                                   schur_dense_ws_bytes(db[k].n, db[k].ncon, chunk64, 0)));
    ws = g.alloc<unsigned char>(ws_bytes);
    if (!ws) throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
}

// sparse_build (solver.c:4014-4100): the pattern of M is the union of the blocks' constraint
// cliques.  -sparse 1 takes the sparse factor whenever the analysis succeeds; the automatic choice
// (-sparse -1) keeps the reference's caps: m >= 200, the largest clique and the pattern within
// 0.45 m^2 (0.30 m^2 above m = 8000) of the lower triangle, and the factor's flops within
// m^3/3 x 0.75 / 1.3.
void Solver::choose_sparse() {
    use_sparse = false;
    if (opt.sparse == 0 || m <= 0 || (opt.sparse < 0 && m < 200)) return;
    const double md = m;
    const double cap = (m <= 8000 ? 0.45 : 0.30) * md * md + 1000;
    std::vector<std::vector<int>> cl;
    double cmax = 0;
    for (auto &B : P.blk) {
        cl.push_back(B.con);
        cmax = std::max(cmax, (double)B.con.size());
    }
    if (opt.sparse < 0 && 0.5 * cmax * (cmax + 1) > cap) return;
    const double t0 = wtime();
    if (schol::analyze(m, cl, sp_an)) return;
    const double fcap = md * md * md / 3.0 * 0.75 / 1.3;
    if (opt.sparse < 0 && ((double)sp_an.pattern > cap || sp_an.flops > fcap)) {
        if (opt.verbose > 1)
            log_printf(0, "   [Schur pattern: %.3g entries below the diagonal, sparse factor %.3g flops: dense factor]\n",
                       (double)sp_an.pattern, sp_an.flops);
        sp_an = schol::Analysis();
        return;
    }
    void *buf = g.alloc<unsigned char>(schol::factor_bytes(sp_an));
    if (!buf) throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
    RC(schol::factor_bind(g.st, sp_an, buf, sp_f));
    CU(cudaStreamSynchronize(g.st));
    use_sparse = true;
    {   // the pattern's rows for the residual product: row a is the union of the constraint lists
        // of the blocks that hold a (a marker per row, then each row sorted)
        std::vector<std::vector<int>> blocks_of(m);
        for (int k = 0; k < nb; k++)
            for (int c : P.blk[k].con) blocks_of[c].push_back(k);
        std::vector<long long> rp(m + 1, 0);
        std::vector<int> cols, mark(m, -1);
        for (int a = 0; a < m; a++) {
            const size_t s0 = cols.size();
            for (int k : blocks_of[a])
                for (int b : P.blk[k].con)
                    if (mark[b] != a) { mark[b] = a; cols.push_back(b); }
            std::sort(cols.begin() + s0, cols.end());
            rp[a + 1] = (long long)cols.size();
        }
        d_prow = g.alloc<long long>(m + 1);
        d_pcol = g.alloc<int>(std::max<size_t>(cols.size(), 1));
        if (!d_prow || !d_pcol) throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
        CU(cudaMemcpyAsync(d_prow, rp.data(), sizeof(long long) * (m + 1), cudaMemcpyHostToDevice, g.st));
        if (!cols.empty()) CU(cudaMemcpyAsync(d_pcol, cols.data(), sizeof(int) * cols.size(), cudaMemcpyHostToDevice, g.st));
        CU(cudaStreamSynchronize(g.st));
    }
    if (opt.verbose > 1)
        log_printf(0, "   [Schur pattern: sparse Cholesky, %.0f nonzeros in L, %.1e flops, %d supernodes, largest front %d, "
                   "%d levels (%.3fs)]\n", sp_an.nnz, sp_an.flops, sp_an.nsup, sp_an.fmax,
                   (int)sp_an.lvptr.size() - 1, wtime() - t0);
}

void Solver::build_gall() {
    if (nb == 1) {
        gall = db[0];
        return;
    }
    // every constraint's entries over all blocks (block order, then position) at concatenated
    // positions boff[k] + p + q n
    long long ne = 0;
    for (auto &B : P.blk) ne += (long long)B.cpos.size();
    std::vector<long long> cptr(m + 1, 0);
    for (auto &B : P.blk)
        for (size_t t = 0; t < B.con.size(); t++) cptr[B.con[t] + 1] += B.cptr[t + 1] - B.cptr[t];
    for (int i = 0; i < m; i++) cptr[i + 1] += cptr[i];
    std::vector<int> cpos(ne), con(m);
    std::vector<double> cval(ne);
    std::vector<long long> fill(cptr.begin(), cptr.end() - 1);
    for (int k = 0; k < nb; k++) {
        const HBlock &B = P.blk[k];
        for (size_t t = 0; t < B.con.size(); t++)
            for (long long e = B.cptr[t]; e < B.cptr[t + 1]; e++) {
                const long long q = fill[B.con[t]]++;
                cpos[q] = (int)(boff[k] + B.cpos[e]);
                cval[q] = B.cval[e];
            }
    }
    for (int i = 0; i < m; i++) con[i] = i;
    if (Ntot2 >= (1LL << 31)) throw GpuFail{BGPU_ERR_TOOBIG, __LINE__};
    gall = DevBlock();
    gall.ncon = m;
    gall.ne = ne;
    gall.con = g.alloc<int>(m);
    gall.cptr = g.alloc<long long>(m + 1);
    gall.cpos = g.alloc<int>(ne);
    gall.cval = g.alloc<double>(ne);
    d_ppt = (const long long **)g.alloc<long long *>(nb);
    d_pct = (const int **)g.alloc<int *>(nb);
    d_pvt = (const double **)g.alloc<double *>(nb);
    if (!gall.con || !gall.cptr || !gall.cpos || !gall.cval || !d_ppt || !d_pct || !d_pvt)
        throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
    std::vector<const long long *> ppt(nb);
    std::vector<const int *> pct(nb);
    std::vector<const double *> pvt(nb);
    for (int k = 0; k < nb; k++) { ppt[k] = db[k].pptr; pct[k] = db[k].pcon; pvt[k] = db[k].pval; }
    CU(cudaMemcpyAsync(gall.con, con.data(), sizeof(int) * m, cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(gall.cptr, cptr.data(), sizeof(long long) * (m + 1), cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(gall.cpos, cpos.data(), sizeof(int) * ne, cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(gall.cval, cval.data(), sizeof(double) * ne, cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(d_ppt, ppt.data(), sizeof(void *) * nb, cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(d_pct, pct.data(), sizeof(void *) * nb, cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(d_pvt, pvt.data(), sizeof(void *) * nb, cudaMemcpyHostToDevice, g.st));
    CU(cudaStreamSynchronize(g.st));
    upload_bytes += (double)ne * 12 + (double)m * 12;
}

// The LP route's lists for every LP block as given (its variables are the order-1 blocks
// in_first[k] .. in_first[k+1]): the constraints that touch it, their entries by variable, and
// each variable's entries by constraint, as schur_lp reads them (solver.c:3233, B->lp_ptr/lp_con).
void Solver::setup_lp_groups() {
    lp_groups.clear();
    const int nbin = (int)P.in_n.size();
    std::vector<int> loc(m, -1);
    for (int k = 0; k < nbin; k++) {
        if (P.in_n[k] >= 0) continue;
        const int q0 = P.in_first[k], N = P.in_first[k + 1] - q0;
        std::vector<int> gcon;
        for (int p = 0; p < N; p++)
            for (int c : P.blk[q0 + p].con) gcon.push_back(c);
        std::sort(gcon.begin(), gcon.end());
        gcon.erase(std::unique(gcon.begin(), gcon.end()), gcon.end());
        const int nc = (int)gcon.size();
        if (nc == 0) continue;
        for (int t = 0; t < nc; t++) loc[gcon[t]] = t;
        std::vector<long long> vptr(N + 1, 0), aptr(nc + 1, 0);
        std::vector<int> vcon;
        std::vector<double> vval;
        for (int p = 0; p < N; p++) {
            const HBlock &B = P.blk[q0 + p];
            for (size_t t = 0; t < B.con.size(); t++) {
                double v = 0;   // the order-1 block's one entry per constraint (summed if repeated)
                for (long long e = B.cptr[t]; e < B.cptr[t + 1]; e++) v += B.cval[e];
                if (v == 0) continue;
                vcon.push_back(loc[B.con[t]]);
                vval.push_back(v);
                aptr[loc[B.con[t]] + 1]++;
            }
            vptr[p + 1] = (long long)vcon.size();
        }
        for (int t = 0; t < nc; t++) aptr[t + 1] += aptr[t];
        const long long ne = (long long)vcon.size();
        std::vector<int> avar(ne);
        std::vector<double> aval(ne);
        std::vector<long long> fill(aptr.begin(), aptr.end() - 1);
        for (int p = 0; p < N; p++)   // by ascending variable within each constraint
            for (long long f = vptr[p]; f < vptr[p + 1]; f++) {
                const long long o = fill[vcon[f]]++;
                avar[o] = p;
                aval[o] = vval[f];
            }
        for (int t = 0; t < nc; t++) loc[gcon[t]] = -1;
        LpGroup G;
        G.q0 = q0;
        G.dev.N = N;
        G.dev.nc = nc;
        G.dev.ne = ne;
        G.dev.gcon = g.alloc<int>(nc);
        G.dev.aptr = g.alloc<long long>(nc + 1);
        G.dev.vptr = g.alloc<long long>(N + 1);
        G.dev.avar = g.alloc<int>(std::max(ne, 1LL));
        G.dev.vcon = g.alloc<int>(std::max(ne, 1LL));
        G.dev.aval = g.alloc<double>(std::max(ne, 1LL));
        G.dev.vval = g.alloc<double>(std::max(ne, 1LL));
        if (!G.dev.gcon || !G.dev.aptr || !G.dev.vptr || !G.dev.avar || !G.dev.vcon || !G.dev.aval || !G.dev.vval)
            throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
        CU(cudaMemcpyAsync(G.dev.gcon, gcon.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, g.st));
        CU(cudaMemcpyAsync(G.dev.aptr, aptr.data(), sizeof(long long) * (nc + 1), cudaMemcpyHostToDevice, g.st));
        CU(cudaMemcpyAsync(G.dev.vptr, vptr.data(), sizeof(long long) * (N + 1), cudaMemcpyHostToDevice, g.st));
        if (ne > 0) {
            CU(cudaMemcpyAsync(G.dev.avar, avar.data(), sizeof(int) * ne, cudaMemcpyHostToDevice, g.st));
            CU(cudaMemcpyAsync(G.dev.vcon, vcon.data(), sizeof(int) * ne, cudaMemcpyHostToDevice, g.st));
            CU(cudaMemcpyAsync(G.dev.aval, aval.data(), sizeof(double) * ne, cudaMemcpyHostToDevice, g.st));
            CU(cudaMemcpyAsync(G.dev.vval, vval.data(), sizeof(double) * ne, cudaMemcpyHostToDevice, g.st));
        }
        CU(cudaStreamSynchronize(g.st));   // the host lists are freed on return
        for (int p = 0; p < N; p++) in_sb[q0 + p] = 1;
        upload_bytes += (double)ne * 24 + (double)(nc + N) * 8;
        if (opt.verbose > 1)
            log_printf(0, "   [LP block %d: %d variables over %d constraints by the LP route]\n", k + 1, N, nc);
        lp_groups.push_back(std::move(G));
    }
}

void Solver::setup_small_schur() {
    in_sb.assign(nb, 0);
    setup_lp_groups();
    std::vector<int> ids;
    for (int k : small_ids)
        if (db[k].n <= SB_NMAX && db[k].ncon > 0 && !in_sb[k]) ids.push_back(k);
    if (ids.size() < 2) return;
    // greedy colouring: the first colour none of whose blocks shares a constraint with k
    std::vector<std::vector<char>> used;
    std::vector<std::vector<int>> cls;
    for (int k : ids) {
        const auto &con = P.blk[k].con;
        size_t c = 0;
        for (; c < used.size(); c++) {
            bool clash = false;
            for (int x : con)
                if (used[c][x]) { clash = true; break; }
            if (!clash) break;
        }
        if (c == used.size()) { used.emplace_back(m, 0); cls.emplace_back(); }
        for (int x : con) used[c][x] = 1;
        cls[c].push_back(k);
    }
    std::vector<int> list;
    sb_coff.assign(1, 0);
    sb_nmax.clear();
    sb_cmax.clear();
    for (auto &cl : cls) {
        int nm = 1, cm = 1;
        for (int k : cl) { list.push_back(k); nm = std::max(nm, db[k].n); cm = std::max(cm, db[k].ncon); }
        sb_coff.push_back((int)list.size());
        sb_nmax.push_back(nm);
        sb_cmax.push_back(cm);
    }
    std::vector<int> ncon(nb, 0);
    std::vector<const int *> con(nb, nullptr), cpos(nb, nullptr);
    std::vector<const long long *> cptr(nb, nullptr);
    std::vector<const double *> cval(nb, nullptr);
    for (int k = 0; k < nb; k++) {
        ncon[k] = db[k].ncon;
        con[k] = db[k].con;
        cptr[k] = db[k].cptr;
        cpos[k] = db[k].cpos;
        cval[k] = db[k].cval;
    }
    d_sb_list = g.alloc<int>(list.size());
    d_sb_ncon = g.alloc<int>(nb);
    d_sb_con = (const int **)g.alloc<int *>(nb);
    d_sb_cpos = (const int **)g.alloc<int *>(nb);
    d_sb_cptr = (const long long **)g.alloc<long long *>(nb);
    d_sb_cval = (const double **)g.alloc<double *>(nb);
    if (!d_sb_list || !d_sb_ncon || !d_sb_con || !d_sb_cpos || !d_sb_cptr || !d_sb_cval)
        throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
    CU(cudaMemcpyAsync(d_sb_list, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(d_sb_ncon, ncon.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(d_sb_con, con.data(), sizeof(void *) * nb, cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(d_sb_cpos, cpos.data(), sizeof(void *) * nb, cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(d_sb_cptr, cptr.data(), sizeof(void *) * nb, cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(d_sb_cval, cval.data(), sizeof(void *) * nb, cudaMemcpyHostToDevice, g.st));
    CU(cudaStreamSynchronize(g.st));
    for (int k : ids) in_sb[k] = 1;
    if (opt.verbose > 1)
        log_printf(0, "   [small blocks: %d assembled in %d launches of blocks sharing no constraint]\n", (int)ids.size(),
                   (int)cls.size());
}

void Solver::assemble_small(const double *Xc, const double *Zc) {
    for (const LpGroup &G : lp_groups) RC(schur_assemble_lp(g.st, G.dev, Xc + boff[G.q0], Zc + boff[G.q0], M, m));
    for (size_t c = 0; c + 1 < sb_coff.size(); c++)
        RC(schur_assemble_small(g.st, sb_coff[c + 1] - sb_coff[c], d_sb_list + sb_coff[c], sb_nmax[c], sb_cmax[c], d_bn,
                                d_sb_ncon, d_sb_con, d_sb_cptr, d_sb_cpos, d_sb_cval, d_boff, Xc, Zc, M, m));
}

void Solver::aop_cat(const double *D, std::vector<double> &out) {
    CU(cudaMemsetAsync(dv_out, 0, sizeof(double) * m, g.st));
    RC(aop_f64(g.st, gall, D, 1.0, 1.0, dv_out));
    out.resize(m);
    CU(cudaMemcpyAsync(out.data(), dv_out, sizeof(double) * m, cudaMemcpyDeviceToHost, g.st));
    CU(cudaStreamSynchronize(g.st));
}

void Solver::atop_cat(const std::vector<double> &y, double alpha, double beta, double *F) {
    CU(cudaMemcpyAsync(dv_in, y.data(), sizeof(double) * m, cudaMemcpyHostToDevice, g.st));
    if (nb == 1) RC(atop_f64(g.st, db[0], dv_in, alpha, beta, F));
    else RC(atop_blocks_f64(g.st, nb, d_boff, Ntot2, d_ppt, d_pct, d_pvt, dv_in, alpha, beta, F));
}

void Solver::sym_cat(const double *G, double s, double a, const double *x, double b, const double *y, double *out) {
    RC(ew_sym_lincomb_blocks(g.st, nb, d_bn, d_boff, Ntot2, G, s, a, x, b, y, out));
}

int Solver::chol(int n, double *L, double *dinv) {
    RC(potrf_f64(g.st, n, L, n, dinv, d_info, d_pmin));
    int info = 0;
    CU(cudaMemcpyAsync(&info, d_info, sizeof(int), cudaMemcpyDeviceToHost, g.st));
    CU(cudaStreamSynchronize(g.st));
    return info;
}

void Solver::inv_from_chol(int n, const double *L, const double *dinv, double *Li) { RC(trtri_f64(g.st, n, L, n, dinv, Li, n)); }

double **Solver::tab(double *DevArrays::*mem) {
    for (auto &e : stab)
        if (e.first == mem) return e.second;
    std::vector<double *> ptrs;
    for (int k : small_ids) ptrs.push_back(da[k].*mem);
    double **d = g.alloc<double *>(ptrs.size());
    if (!d) throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
    CU(cudaMemcpyAsync(d, ptrs.data(), sizeof(double *) * ptrs.size(), cudaMemcpyHostToDevice, g.st));
    CU(cudaStreamSynchronize(g.st));
    stab.push_back({mem, d});
    return d;
}

void Solver::mul_all(double alpha, double *DevArrays::*A, double *DevArrays::*B, double *DevArrays::*C) {
    for (int k : big_ids) mul(db[k].n, alpha, da[k].*A, da[k].*B, da[k].*C);
    if (!small_ids.empty())
        RC(small_gemm(g.st, (int)small_ids.size(), d_sns, 0, 0, alpha, (const double *const *)tab(A),
                      (const double *const *)tab(B), 0.0, tab(C), 0));
}

void Solver::zinv(int k) {
    // Zi = LZ^-T LZ^-1 (LZ and dinvZ from the last Cholesky of Z)
    const int n = db[k].n;
    DevArrays &a = da[k];
    inv_from_chol(n, a.LZ, a.dinvZ, a.LiZ);
    RC(gemm_f64(g.st, 1, 1, n, n, n, 1.0, a.LiZ, n, 0, a.LiZ, n, 0, 0.0, a.Zi, n, 0, 1, 0));
    RC(symmetrize_f64(g.st, n, a.Zi, n));
}

// nt_scaling (solver.c:7898-7912) for every block: from the Cholesky factors of X and Z to G, lam
// and W = G G' (kept in Zi, which the assembly and the products read as both X and Z^-1).  A block
// whose singular values are not all positive, or whose Jacobi iteration does not converge, fails the
// iteration (status 4, as nt_fail).
bool Solver::nt_scaling() {
    nt_sweeps = 0;
    for (int k : big_ids) {
        const int n = db[k].n;
        DevArrays &d = da[k];
        RC(nt::tril(g.st, n, d.LX, d.NG));   // rotated into L_X V
        RC(nt::tril(g.st, n, d.LZ, d.Q));
        gemm(1, 1, n, 1.0, d.Q, n, d.NG, n, 0.0, d.T);   // Mb = L_Z' L_X
        int sweeps = 0;
        RC(nt::jacobi(g.st, n, d.T, d.NG, d_ntflag, h_ntflag, &sweeps));
        nt_sweeps = std::max(nt_sweeps, sweeps);
        if (sweeps < 0) {
            if (opt.verbose > 1) log_printf(0, "   NT scaling: block %d did not converge\n", k + 1);
            return false;
        }
        CU(cudaMemsetAsync(d_ntinfo, 0, sizeof(int), g.st));
        RC(nt::finish(g.st, n, d.T, d.NG, nlam + loff[k], d_ntinfo));
        CU(cudaMemcpyAsync(h_ntinfo, d_ntinfo, sizeof(int), cudaMemcpyDeviceToHost, g.st));
        gemm(0, 0, n, 1.0, d.NG, n, d.NG, n, 0.0, d.Zi);   // W = G G'
        RC(symmetrize_f64(g.st, n, d.Zi, n));
        CU(cudaStreamSynchronize(g.st));
        if (*h_ntinfo) return false;
    }
    if (!small_ids.empty()) {
        const int ns = (int)small_ids.size();
        RC(nt::scaling_small(g.st, ns, d_sns, small_nmax, (const double *const *)tab(&DevArrays::LX),
                             (const double *const *)tab(&DevArrays::LZ), tab(&DevArrays::NG), d_lamtab,
                             tab(&DevArrays::Zi), d_sinfo));
        CU(cudaMemcpyAsync(h_sinfo, d_sinfo, sizeof(int) * ns, cudaMemcpyDeviceToHost, g.st));
        CU(cudaStreamSynchronize(g.st));
        for (int i = 0; i < ns; i++)
            if (h_sinfo[i]) return false;
    }
    return true;
}

// nt_toZ (solver.c:7990-8008): out = G' D G, symmetrized (T is the scratch)
void Solver::nt_toZ(double *DevArrays::*D, double *DevArrays::*out) {
    for (int k : big_ids) {
        const int n = db[k].n;
        DevArrays &d = da[k];
        gemm(0, 1, n, 1.0, d.*D, n, d.NG, n, 0.0, d.T);       // D G
        gemm(1, 1, n, 1.0, d.NG, n, d.T, n, 0.0, d.*out);     // G' (D G)
        RC(symmetrize_f64(g.st, n, d.*out, n));
    }
    if (!small_ids.empty()) {
        const int ns = (int)small_ids.size();
        RC(small_gemm(g.st, ns, d_sns, 0, 0, 1.0, (const double *const *)tab(D), (const double *const *)tab(&DevArrays::NG),
                      0.0, tab(&DevArrays::T), 0));
        RC(small_gemm(g.st, ns, d_sns, 1, 0, 1.0, (const double *const *)tab(&DevArrays::NG),
                      (const double *const *)tab(&DevArrays::T), 0.0, tab(out), 1));
    }
}

// nt_fromS (solver.c:8051-8068): out = G D G', symmetrized (T is the scratch)
void Solver::nt_fromS(double *DevArrays::*D, double *DevArrays::*out) {
    for (int k : big_ids) {
        const int n = db[k].n;
        DevArrays &d = da[k];
        gemm(0, 1, n, 1.0, d.NG, n, d.*D, n, 0.0, d.T);       // G D
        gemm(0, 0, n, 1.0, d.T, n, d.NG, n, 0.0, d.*out);     // (G D) G'
        RC(symmetrize_f64(g.st, n, d.*out, n));
    }
    if (!small_ids.empty()) {
        const int ns = (int)small_ids.size();
        RC(small_gemm(g.st, ns, d_sns, 0, 0, 1.0, (const double *const *)tab(&DevArrays::NG), (const double *const *)tab(D),
                      0.0, tab(&DevArrays::T), 0));
        RC(small_gemm(g.st, ns, d_sns, 0, 1, 1.0, (const double *const *)tab(&DevArrays::T),
                      (const double *const *)tab(&DevArrays::NG), 0.0, tab(out), 1));
    }
}

void Solver::mul_sym_all(double *DevArrays::*A, double *DevArrays::*B, double *DevArrays::*C) {
    for (int k : big_ids) {
        const int n = db[k].n;
        mul(n, 1.0, da[k].*A, da[k].*B, da[k].*C);
        RC(symmetrize_f64(g.st, n, da[k].*C, n));
    }
    if (!small_ids.empty())
        RC(small_gemm(g.st, (int)small_ids.size(), d_sns, 0, 0, 1.0, (const double *const *)tab(A),
                      (const double *const *)tab(B), 0.0, tab(C), 1));
}

// ---- Schur complement ----------------------------------------------------------------------
void Solver::assemble(std::vector<double> &) {
    CU(cudaMemsetAsync(M, 0, sizeof(double) * (size_t)m * m, g.st));
    CU(cudaEventRecord(ev0, g.st));
    // 3xTF32 until the mixed path turns to its late precision (FP64 or the Ozaki slices)
    const int prec = next_prec();
    const bool oz = (prec & 0xff) == 2;
    cur_prec = prec;
    m_exact = prec_exact(prec);
    const int kchunk = prec == 1 ? chunk : oz ? chunk_oz : chunk64;
    if (oz) snprintf(asm_label, sizeof asm_label, "ozaki%d", schur_ozaki_slices(prec));
    else snprintf(asm_label, sizeof asm_label, "%s", prec == 1 ? "tf32x3" : "fp64");
    assemble_small(cat.*xmem(), cat.Zi);
    for (int k = 0; k < nb; k++) {
        if (in_sb[k]) {
            schur_flops += 2.0 * db[k].n * db[k].n * db[k].n * db[k].ncon;
            continue;
        }
        const double *Xa = da[k].*xmem();
        if (lowrank[k].R > 0) {   // (FP64: the route's products are small)
            RC(schur_assemble_lowrank(g.st, lowrank[k], db[k].con, Xa, da[k].Zi, M, m));
            const double n = db[k].n, R = lowrank[k].R;
            schur_flops += 4.0 * n * n * R + 4.0 * n * R * R;
            continue;
        }
        if (dense_route[k])   // (the dense route has no Ozaki form: FP64 there)
            RC(schur_assemble_dense(g.st, db[k], Xa, da[k].Zi, M, m, oz ? 0 : prec, prec == 1 ? chunk : chunk64,
                                    ws, ws_bytes));
        else
            RC(schur_assemble(g.st, db[k], Xa, da[k].Zi, M, m, prec, kchunk, ws, ws_bytes));
        const double n = db[k].n;
        const double ncon = db[k].ncon;
        schur_flops += 2.0 * n * n * n * ncon;   // the row-product GEMMs: 2 n^2 r_a with r_a <= n
    }
    CU(cudaEventRecord(ev1, g.st));
    CU(cudaEventSynchronize(ev1));
    float ms = 0;
    CU(cudaEventElapsedTime(&ms, ev0, ev1));
    schur_dev_time += ms * 1e-3;
    if (prec == 1 || oz) {
        int bad = 0;
        RC(prec == 1 ? tf32x3_error_flag(&bad) : ozaki_error_flag(&bad));
        if (bad) throw GpuFail{BGPU_ERR_TIMEOUT, __LINE__};
    }
}

// schur_factor_ (solver.c:5296-5421), dense path
int Solver::factor() {
    nfactor++;
    const double ulp = 2.220446049250313e-16;
    const double reg_floor = opt.reg_ill > 0 ? opt.reg_ill : std::max(1e-15, (double)m * ulp);
    const double reg_first = opt.reg_ill > 0 ? 1e-13 : std::max(1e-15, (double)m * ulp);
    const bool float_now = allow_float && !want_double && !(asm_prec == 1 && mu_now < opt.mu_switch);
    if (float_now) {
        RC(schur_load_f32(g.st, m, M, m, Dsc, Mf, m));
        RC(potrf_f32(g.st, m, Mf, m, dinvMf, d_info, d_pmin));
        int info = 0;
        double pmin = 0;
        CU(cudaMemcpyAsync(&info, d_info, sizeof(int), cudaMemcpyDeviceToHost, g.st));
        CU(cudaMemcpyAsync(&pmin, d_pmin, sizeof(double), cudaMemcpyDeviceToHost, g.st));
        CU(cudaStreamSynchronize(g.st));
        if (info == 0 && pmin >= 1e-6) {
            is_float = true;
            reg = 0;
            nfloat++;
            min_pivot = pmin;
            return 0;
        }
        want_double = true;
    }
    is_float = false;
    if (use_sparse) {
        RC(schur_diag_scale(g.st, m, M, m, Dsc));
        if (sparse_float && !want_double && mu_now >= opt.mu_switch) {
            // FP32 fronts early: PCG refines against the FP64 M, and the first factor that needs a
            // shift or a PCG that struggles turns the rest of the solve to FP64 (want_double)
            RC(schol::factor(g.st, sp_f, M, m, Dsc, 0.0, true));
            int info = 0;
            double pmin = 0;
            CU(cudaMemcpyAsync(&info, sp_f.info, sizeof(int), cudaMemcpyDeviceToHost, g.st));
            CU(cudaMemcpyAsync(&pmin, sp_f.pmin, sizeof(double), cudaMemcpyDeviceToHost, g.st));
            CU(cudaStreamSynchronize(g.st));
            if (info == 0 && pmin >= 1e-6) {
                is_float = true;
                reg = 0;
                nfloat++;
                min_pivot = std::min(pmin, 1.0);
                return 0;
            }
            want_double = true;
        }
        double r = reg_hint ? std::max(reg_floor, 0.01 * reg_ok) : 0.0;
        int info = 0;
        for (int attempt = 0; attempt < 10; attempt++) {
            RC(schol::factor(g.st, sp_f, M, m, Dsc, r, false));
            double pmin = 0;
            CU(cudaMemcpyAsync(&info, sp_f.info, sizeof(int), cudaMemcpyDeviceToHost, g.st));
            CU(cudaMemcpyAsync(&pmin, sp_f.pmin, sizeof(double), cudaMemcpyDeviceToHost, g.st));
            CU(cudaStreamSynchronize(g.st));
            if (info == 0) {
                pmin = std::min(pmin, 1.0);
                if (pmin >= opt.pivtol || r >= reg_floor) {
                    reg = r;
                    min_pivot = pmin;
                    reg_hint = r > 0;
                    reg_ok = r;
                    return 0;
                }
                r = std::max(reg_floor, r * 100);
                continue;
            }
            r = (r == 0) ? reg_first : r * 100;
        }
        return info ? info : 1;
    }
    if (!Lm) {
        Lm = g.alloc<double>((size_t)m * m);
        if (!Lm) throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
    }
    double r = reg_hint ? std::max(reg_floor, 0.01 * reg_ok) : 0.0;
    int info = 0;
    for (int attempt = 0; attempt < 10; attempt++) {
        RC(schur_load_f64(g.st, m, M, m, r, Dsc, Lm, m));
        RC(potrf_f64(g.st, m, Lm, m, dinvM, d_info, d_pmin));
        double pmin = 0;
        CU(cudaMemcpyAsync(&info, d_info, sizeof(int), cudaMemcpyDeviceToHost, g.st));
        CU(cudaMemcpyAsync(&pmin, d_pmin, sizeof(double), cudaMemcpyDeviceToHost, g.st));
        CU(cudaStreamSynchronize(g.st));
        if (info == 0) {
            if (pmin >= opt.pivtol || r >= reg_floor) {
                reg = r;
                min_pivot = pmin;
                reg_hint = r > 0;
                reg_ok = r;
                return 0;
            }
            r = std::max(reg_floor, r * 100);
            continue;
        }
        r = (r == 0) ? reg_first : r * 100;
    }
    return info ? info : 1;
}

void Solver::prec(const std::vector<double> &rv, std::vector<double> &z) {
    // z = D L^-T L^-1 D r (schur_prec_, solver.c:5424-5460)
    z.resize(m);
    if (use_sparse) {   // (FP32 or FP64 fronts: the solve takes the last factor's type; D is applied on
                        // the device, and the sparse solve has no device waits to report)
        CU(cudaMemcpyAsync(dv_in, rv.data(), sizeof(double) * m, cudaMemcpyHostToDevice, g.st));
        RC(schol::solve(g.st, sp_f, Dsc, dv_in));
        CU(cudaMemcpyAsync(z.data(), dv_in, sizeof(double) * m, cudaMemcpyDeviceToHost, g.st));
        CU(cudaStreamSynchronize(g.st));
        return;
    }
    std::vector<double> h(m);
    std::vector<double> Dh(m);
    CU(cudaMemcpyAsync(Dh.data(), Dsc, sizeof(double) * m, cudaMemcpyDeviceToHost, g.st));
    CU(cudaStreamSynchronize(g.st));
    if (is_float) {
        std::vector<float> f(m);
        for (int i = 0; i < m; i++) f[i] = (float)(rv[i] * Dh[i]);
        CU(cudaMemcpyAsync(fv, f.data(), sizeof(float) * m, cudaMemcpyHostToDevice, g.st));
        RC(trsv_f32(g.st, m, Mf, m, dinvMf, fv, 0, mflags, ++epoch, d_err));
        RC(trsv_f32(g.st, m, Mf, m, dinvMf, fv, 1, mflags, ++epoch, d_err));
        CU(cudaMemcpyAsync(f.data(), fv, sizeof(float) * m, cudaMemcpyDeviceToHost, g.st));
        CU(cudaStreamSynchronize(g.st));
        for (int i = 0; i < m; i++) z[i] = (double)f[i] * Dh[i];
    } else {
        for (int i = 0; i < m; i++) h[i] = rv[i] * Dh[i];
        CU(cudaMemcpyAsync(dv_in, h.data(), sizeof(double) * m, cudaMemcpyHostToDevice, g.st));
        RC(trsv_f64(g.st, m, Lm, m, dinvM, dv_in, 0, mflags, ++epoch, d_err));
        RC(trsv_f64(g.st, m, Lm, m, dinvM, dv_in, 1, mflags, ++epoch, d_err));
        CU(cudaMemcpyAsync(h.data(), dv_in, sizeof(double) * m, cudaMemcpyDeviceToHost, g.st));
        CU(cudaStreamSynchronize(g.st));
        for (int i = 0; i < m; i++) z[i] = h[i] * Dh[i];
    }
    int err = 0;
    CU(cudaMemcpyAsync(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost, g.st));
    CU(cudaStreamSynchronize(g.st));
    if (err) throw GpuFail{BGPU_ERR_TIMEOUT, __LINE__};
}

void Solver::schur_mv(const std::vector<double> &x, std::vector<double> &y) {
    CU(cudaMemcpyAsync(dv_in, x.data(), sizeof(double) * m, cudaMemcpyHostToDevice, g.st));
    if (use_sparse && d_prow) RC(pattern_symv_f64(g.st, m, d_prow, d_pcol, M, m, dv_in, dv_out));
    else RC(symv_full_f64(g.st, m, 1.0, M, m, dv_in, 0.0, dv_out));
    y.resize(m);
    CU(cudaMemcpyAsync(y.data(), dv_out, sizeof(double) * m, cudaMemcpyDeviceToHost, g.st));
    CU(cudaStreamSynchronize(g.st));
}

void Solver::newton_mv(const std::vector<double> &x, std::vector<double> &y) {
    atop_cat(x, 1.0, 0.0, cat.W);   // A'(x)
    mul_all(1.0, &DevArrays::Zi, &DevArrays::W, &DevArrays::T);
    mul_all(1.0, &DevArrays::T, xmem(), &DevArrays::F);   // Z^-1 A'(x) X (W A'(x) W under NT)
    aop_cat(cat.F, y);
}

static double dot(const std::vector<double> &a, const std::vector<double> &b) {
    double s = 0;
    for (size_t i = 0; i < a.size(); i++) s += a[i] * b[i];
    return s;
}
static double nrm(const std::vector<double> &a) { return std::sqrt(dot(a, a)); }

// schur_solve_ (solver.c:5483-5621): PCG on M x = rhs with the factor as preconditioner
double Solver::schur_solve(const std::vector<double> &rhs, std::vector<double> &x, double tol_rel) {
    const double nb_ = nrm(rhs);
    x.assign(m, 0.0);
    if (nb_ == 0) return 0;
    prec(rhs, x);
    std::vector<double> Mx, r(m), z, p, q, xb;
    mv(x, Mx);
    for (int i = 0; i < m; i++) r[i] = rhs[i] - Mx[i];
    double nr = nrm(r);
    // a preconditioner of FP32 accuracy (the float factor, or any factor of the 3xTF32 M) is
    // refined to 1e-10 as the reference's float factor (solver.c:5547); the exact one to 1e-13
    const bool approx = is_float || !m_exact;
    const double tol = std::max(tol_rel, approx ? 1e-10 : 1e-13) * nb_;
    if (nr <= tol) return nr / nb_;
    double best = nr;
    xb = x;
    prec(r, z);
    p = z;
    double rz = dot(r, z);
    // the factor of a shifted 3xTF32 M preconditions the FP64 operator less well: more steps
    const bool shifted = !m_exact && reg > 0;
    const int maxit = shifted ? 150 : (reg > 0 || approx) ? 50 : 10;
    int stall = 0, used = 0;
    const double sgain = 0.9;
    const int smax = shifted ? 10 : 4;
    for (int k = 0; k < maxit; k++) {
        mv(p, q);
        const double pq = dot(p, q);
        if (!(pq > 0)) break;
        const double a = rz / pq;
        for (int i = 0; i < m; i++) { x[i] += a * p[i]; r[i] -= a * q[i]; }
        pcg_iters++;
        used++;
        nr = nrm(r);
        if (nr < best) {
            stall = (nr > sgain * best) ? stall + 1 : 0;
            best = nr;
            xb = x;
        } else stall++;
        if (nr <= tol || stall >= smax) break;
        prec(r, z);
        const double rz2 = dot(r, z);
        const double beta = rz2 / rz;
        rz = rz2;
        for (int i = 0; i < m; i++) p[i] = z[i] + beta * p[i];
    }
    x = xb;
    mv(x, Mx);
    for (int i = 0; i < m; i++) r[i] = rhs[i] - Mx[i];
    const double rel = nrm(r) / nb_;
    if (is_float && (used > 4 || best > tol || rel > std::max(1e-9, 10 * tol_rel))) want_double = true;
    // the mixed path: when PCG cannot reach the tolerance against the FP64 operator with the
    // factor of the approximate M, the following iterations assemble M more accurately
    if (!m_exact && (best > tol || rel > std::max(1e-9, 10 * tol_rel)) && raise_precision()) {
        if (opt.verbose > 1)
            log_printf(0, "   mixed path: PCG missed %.1e (rel %.1e): more accurate assembly from here on\n", tol / nb_, rel);
    }
    return rel;
}

// ---- step length ---------------------------------------------------------------------------
// Lanczos on the explicit Bm = L^-1 D L^-T (sdp_maxstep_lam, solver.c:6083-6225, cold start):
// returns lambda_min estimate theta - residual bound (conservative), or -1e300 on failure.  The
// steps run on the device (lanczos.cu); the host reads the state at the steps where the stop
// test runs (from the sixth, every third, and the last), once each.
double Solver::lanczos(int n, const double *Bm, int Kmax) {
    int K = std::min(n, Kmax);
    K = std::min(K, 30);
    RC(lanczos_start(g.st, n, lz_q0, lz_Q, lz_st));
    for (int j = 0; j < K; j++) {
        RC(symv_full_f64(g.st, n, 1.0, Bm, n, lz_Q + (size_t)j * n, 0.0, dv_out));
        RC(lanczos_step(g.st, n, j, K, lz_Q, dv_out, lz_st));
        const int kk = j + 1;
        if ((kk >= 6 && kk % 3 == 0) || kk == K) {
            CU(cudaMemcpyAsync(h_lz, lz_st, sizeof(LanczosState), cudaMemcpyDeviceToHost, g.st));
            CU(cudaStreamSynchronize(g.st));
            if (h_lz->done) break;
        }
    }
    return h_lz->lam;   // (done: the last step sets it)
}

// maxstep (solver.c:6300-6390): the largest alpha with V + alpha dV >= 0 over all blocks
double Solver::maxstep(int primal, int K) {
    double a = 1e30;
    for (int k : big_ids) {
        const int n = db[k].n;
        DevArrays &d = da[k];
        const double *Li = primal ? d.LiX : d.LiZ;
        const double *dV = primal ? d.dX : d.dZ;
        // Bm = Li dV Li'
        RC(gemm_f64(g.st, 0, 1, n, n, n, 1.0, Li, n, 0, dV, n, 0, 0.0, d.T, n, 0, 1, 0));
        RC(gemm_f64(g.st, 0, 0, n, n, n, 1.0, d.T, n, 0, Li, n, 0, 0.0, d.Bm, n, 0, 1, 0));
        RC(symmetrize_f64(g.st, n, d.Bm, n));
        const double lam = lanczos(n, d.Bm, K);
        double ak;
        if (lam <= -1e299) ak = 0.0;
        else ak = lam >= 0 ? 1e30 : -1.0 / lam;
        if (!std::isfinite(ak) && !(ak > 0)) ak = 0.0;
        if (ak < a) a = ak;
    }
    if (!small_ids.empty()) {   // exact lambda_min per small block, one launch (small_lammin, solver.c:5947)
        const int ns = (int)small_ids.size();
        RC(small_lammin(g.st, ns, d_sns, (const double *const *)tab(primal ? &DevArrays::LiX : &DevArrays::LiZ),
                        (const double *const *)tab(primal ? &DevArrays::dX : &DevArrays::dZ), d_slam));
        CU(cudaMemcpyAsync(h_slam, d_slam, sizeof(double) * ns, cudaMemcpyDeviceToHost, g.st));
        CU(cudaStreamSynchronize(g.st));
        for (int i = 0; i < ns; i++) {
            const double lam = h_slam[i];
            double ak = (lam <= -1e299) ? 0.0 : (lam >= 0 ? 1e30 : -1.0 / lam);
            if (!std::isfinite(ak) && !(ak > 0)) ak = 0.0;
            if (ak < a) a = ak;
        }
    }
    return a;
}

// try_step (solver.c:6393-6447): V += alpha dV with a Cholesky test, alpha *= 0.8 on failure.
// `from`: the step V already took along dV (V is moved from there to alpha).
int Solver::try_step(int primal, double *alpha, double from) {
    double a = *alpha;
    double stepped = from;   // all blocks stay at the same step
    const int ns = (int)small_ids.size();
    for (int tries = 0; tries < 40; tries++) {
        bool ok = true;
        const double inc = a - stepped;
        stepped = a;
        for (int k : big_ids) {
            const int n = db[k].n;
            DevArrays &d = da[k];
            double *V = primal ? d.X : d.Z, *dV = primal ? d.dX : d.dZ, *L = primal ? d.LX : d.LZ;
            double *dinv = primal ? d.dinvX : d.dinvZ;
            RC(ew_step_copy(g.st, (long long)n * n, inc, dV, V, L));
            if (chol(n, L, dinv) != 0) ok = false;
        }
        if (ns > 0) {
            double **V = tab(primal ? &DevArrays::X : &DevArrays::Z), **L = tab(primal ? &DevArrays::LX : &DevArrays::LZ);
            RC(small_step_copy(g.st, ns, d_sns, inc, (const double *const *)tab(primal ? &DevArrays::dX : &DevArrays::dZ),
                               V, L));
            RC(small_chol_inv(g.st, ns, d_sns, L, L, tab(primal ? &DevArrays::LiX : &DevArrays::LiZ), d_sinfo));
            CU(cudaMemcpyAsync(h_sinfo, d_sinfo, sizeof(int) * ns, cudaMemcpyDeviceToHost, g.st));
            CU(cudaStreamSynchronize(g.st));
            for (int i = 0; i < ns; i++)
                if (h_sinfo[i]) ok = false;
        }
        if (ok) {
            *alpha = a;
            return 1;
        }
        a *= 0.8;
    }
    return 0;
}

// The least-squares start (the default init = 1, solver.c:13939-14198), in its factored form:
// dy = (A A')^-1 b and y = (A A')^-1 A(C) with A A' the Schur complement at X = Zi = I, then
// X0 = A'dy and Z0 = C - A'y shifted into the cone by their smallest eigenvalues (X: 1 + |lmin|
// when not positive definite; Z: max(0, 1 - lmin)) and raised until a Cholesky test passes.
void Solver::least_squares_start(std::vector<double> &y) {
    const bool af = allow_float;
    allow_float = false;   // the start's Gram solves in FP64
    m_exact = true;        // A A' is assembled in FP64 here
    CU(cudaMemsetAsync(M, 0, sizeof(double) * (size_t)m * m, g.st));
    assemble_small(Icat, Icat);   // the Gram matrix of the small blocks: X = Zi = I
    for (int k = 0; k < nb; k++) {
        if (in_sb[k]) continue;
        RC(ew_set_scaled_identity(g.st, db[k].n, da[k].T, 1.0));
        if (lowrank[k].R > 0) RC(schur_assemble_lowrank(g.st, lowrank[k], db[k].con, da[k].T, da[k].T, M, m));
        else if (dense_route[k]) RC(schur_assemble_dense(g.st, db[k], da[k].T, da[k].T, M, m, 0, chunk_fp64(k), ws, ws_bytes));
        else RC(schur_assemble_gram(g.st, db[k], M, m, ws, ws_bytes));
    }
    const int frc = factor();
    allow_float = af;
    if (frc != 0) return;   // keep the SDPT3 start (the reference's init_ok = 0 path)
    std::vector<double> dy, AC;
    schur_solve(P.b, dy, 1e-8);
    aop_cat(Ccat, AC);
    schur_solve(AC, y, 1e-8);
    double ax = -1e300, az = -1e300;
    atop_cat(dy, 1.0, 0.0, cat.X);                               // X = A'dy
    atop_cat(y, -1.0, 0.0, cat.Z);
    lincomb_cat(1.0, cat.Z, 1.0, Ccat, 0.0, nullptr, cat.Z);     // Z = C - A'y
    for (int k : big_ids) {
        const int n = db[k].n;
        const long long nn = (long long)n * n;
        DevArrays &d = da[k];
        RC(ew_lincomb(g.st, nn, 1.0, d.X, 0.0, nullptr, 0.0, nullptr, d.Bm));
        const double lx = lanczos(n, d.Bm, opt.lanczos_k);
        RC(ew_lincomb(g.st, nn, 1.0, d.Z, 0.0, nullptr, 0.0, nullptr, d.Bm));
        const double lz = lanczos(n, d.Bm, opt.lanczos_k);
        ax = std::max(ax, -lx);
        az = std::max(az, -lz);
    }
    const int nsm = (int)small_ids.size();
    if (nsm > 0) {   // the small blocks' exact smallest eigenvalues, all at once
        CU(cudaMemcpyAsync(cat.LiX, Icat, sizeof(double) * Ntot2, cudaMemcpyDeviceToDevice, g.st));
        for (int pass = 0; pass < 2; pass++) {
            RC(small_lammin(g.st, nsm, d_sns, (const double *const *)tab(&DevArrays::LiX),
                            (const double *const *)tab(pass == 0 ? &DevArrays::X : &DevArrays::Z), d_slam));
            CU(cudaMemcpyAsync(h_slam, d_slam, sizeof(double) * nsm, cudaMemcpyDeviceToHost, g.st));
            CU(cudaStreamSynchronize(g.st));
            double &a = pass == 0 ? ax : az;
            for (int i = 0; i < nsm; i++) a = std::max(a, -h_slam[i]);
        }
    }
    const double shx = ax >= -1e-8 ? 1.0 + ax : 0.0;
    const double shz = std::max(0.0, 1.0 + az);
    lincomb_cat(1.0, cat.X, shx, Icat, 0.0, nullptr, cat.X);
    lincomb_cat(1.0, cat.Z, shz, Icat, 0.0, nullptr, cat.Z);
    if (nsm > 0) {   // Cholesky tests of the small blocks, raised where they fail
        for (int pass = 0; pass < 2; pass++) {
            double *DevArrays::*V = pass == 0 ? &DevArrays::X : &DevArrays::Z;
            double *DevArrays::*Lv = pass == 0 ? &DevArrays::LX : &DevArrays::LZ;
            double *DevArrays::*Li = pass == 0 ? &DevArrays::LiX : &DevArrays::LiZ;
            for (double extra = 1e-8;; extra *= 10) {
                RC(small_chol_inv(g.st, nsm, d_sns, tab(V), tab(Lv), tab(Li), d_sinfo));
                CU(cudaMemcpyAsync(h_sinfo, d_sinfo, sizeof(int) * nsm, cudaMemcpyDeviceToHost, g.st));
                CU(cudaStreamSynchronize(g.st));
                bool all = true;
                for (int i = 0; i < nsm; i++)
                    if (h_sinfo[i]) {
                        all = false;
                        const int k = small_ids[i];
                        RC(ew_add_diag(g.st, db[k].n, da[k].*V, db[k].n, extra));
                    }
                if (all) break;
                if (extra > 1e30) throw GpuFail{BGPU_ERR_NOTPD, __LINE__};
            }
        }
    }
    for (int k : big_ids) {
        const int n = db[k].n;
        const long long nn = (long long)n * n;
        DevArrays &d = da[k];
        for (double extra = 1e-8;; extra *= 10) {
            RC(ew_lincomb(g.st, nn, 1.0, d.X, 0.0, nullptr, 0.0, nullptr, d.LX));
            if (chol(n, d.LX, d.dinvX) == 0) break;
            RC(ew_add_diag(g.st, n, d.X, n, extra));
            if (extra > 1e30) throw GpuFail{BGPU_ERR_NOTPD, __LINE__};
        }
        for (double extra = 1e-8;; extra *= 10) {
            RC(ew_lincomb(g.st, nn, 1.0, d.Z, 0.0, nullptr, 0.0, nullptr, d.LZ));
            if (chol(n, d.LZ, d.dinvZ) == 0) break;
            RC(ew_add_diag(g.st, n, d.Z, n, extra));
            if (extra > 1e30) throw GpuFail{BGPU_ERR_NOTPD, __LINE__};
        }
        inv_from_chol(n, d.LX, d.dinvX, d.LiX);
        inv_from_chol(n, d.LZ, d.dinvZ, d.LiZ);   // the small blocks' Z^-1 comes from LiZ
    }
    // the factor state starts afresh for the loop
    want_double = is_float = reg_hint = false;
    reg = reg_ok = 0;
    nfactor = nfloat = 0;
}

// ---- the DIMACS errors of the returned point on the data as given ----------------------------
void Solver::final_measures(const std::vector<double> &y, ResultData &res) {
    // X_o = bs X, y_o = cs d y, Z_o = C - A'(y_o) = cs (C' - A'(y))   (scaled data on the device)
    const double bs = P.bs, cs = P.cs;
    res.y.resize(m);
    for (int i = 0; i < m; i++) res.y[i] = cs * P.d[i] * y[i];
    double pobj = 0, xz = 0, lamx_neg = 0, lamz_neg = 0;
    res.X.resize(nb);
    res.Z.resize(nb);
    // W = cs (C' - A'(y)) ; G = bs X
    atop_cat(y, -cs, 0.0, cat.W);
    lincomb_cat(1.0, cat.W, cs, Ccat, 0.0, nullptr, cat.W);
    lincomb_cat(bs, cat.X, 0.0, nullptr, 0.0, nullptr, cat.G);
    {
        double tmp[2];
        const double *aa[2] = {Ccat, cat.G}, *bb[2] = {cat.G, cat.W};
        dots_cat(2, aa, bb, tmp);
        pobj = cs * tmp[0];   // <C_o, X_o> = cs <C', X_o>
        xz = tmp[1];
    }
    for (int k = 0; k < nb; k++) {
        const long long nn = (long long)db[k].n * db[k].n;
        res.X[k].resize(nn);
        res.Z[k].resize(nn);
        CU(cudaMemcpyAsync(res.X[k].data(), da[k].G, sizeof(double) * nn, cudaMemcpyDeviceToHost, g.st));
        CU(cudaMemcpyAsync(res.Z[k].data(), da[k].W, sizeof(double) * nn, cudaMemcpyDeviceToHost, g.st));
    }
    const int nsm = (int)small_ids.size();
    if (nsm > 0) {   // the small blocks' cone errors: Cholesky tests, exact lambda_min where they fail
        CU(cudaMemcpyAsync(cat.LiX, Icat, sizeof(double) * Ntot2, cudaMemcpyDeviceToDevice, g.st));
        for (int pass = 0; pass < 2; pass++) {
            double *DevArrays::*V = pass == 0 ? &DevArrays::W : &DevArrays::G;
            RC(small_chol_inv(g.st, nsm, d_sns, tab(V), tab(&DevArrays::T), nullptr, d_sinfo));
            RC(small_lammin(g.st, nsm, d_sns, (const double *const *)tab(&DevArrays::LiX),
                            (const double *const *)tab(V), d_slam));
            CU(cudaMemcpyAsync(h_sinfo, d_sinfo, sizeof(int) * nsm, cudaMemcpyDeviceToHost, g.st));
            CU(cudaMemcpyAsync(h_slam, d_slam, sizeof(double) * nsm, cudaMemcpyDeviceToHost, g.st));
            CU(cudaStreamSynchronize(g.st));
            double &neg = pass == 0 ? lamz_neg : lamx_neg;
            for (int i = 0; i < nsm; i++)
                if (h_sinfo[i]) neg = std::max(neg, -h_slam[i]);
        }
    }
    // -lambda_min of V (block k) where its Cholesky test fails: the Lanczos estimate theta - res
    // (conservative: an upper bound), or the smallest shift s = 10^j 1e-16 |V|_F below it for which
    // V + s I passes a Cholesky test (also an upper bound), whichever is smaller.  The Lanczos
    // bound alone can exceed a nearly singular V's true negative part by orders of magnitude.
    auto neg_part = [&](int k, const double *V, double *dinv) {
        const int n = db[k].n;
        const long long nn = (long long)n * n;
        DevArrays &d = da[k];
        RC(ew_lincomb(g.st, nn, 1.0, V, 0.0, nullptr, 0.0, nullptr, d.Bm));
        const double est = -lanczos(n, d.Bm, 30);
        double f2 = 0;
        const double *aa[1] = {V};
        dots(1, aa, aa, nn, &f2);
        for (double sft = 1e-16 * std::sqrt(f2); sft > 0 && sft < est; sft *= 10) {
            RC(ew_lincomb(g.st, nn, 1.0, V, sft, Icat + boff[k], 0.0, nullptr, d.T));
            if (chol(n, d.T, dinv) == 0) return sft;
        }
        return est;
    };
    for (int k : big_ids) {
        const int n = db[k].n;
        const long long nn = (long long)n * n;
        DevArrays &d = da[k];
        // cone errors: a Cholesky test, then the bound of neg_part when it fails
        RC(ew_lincomb(g.st, nn, 1.0, d.W, 0.0, nullptr, 0.0, nullptr, d.T));
        if (chol(n, d.T, d.dinvZ) != 0) lamz_neg = std::max(lamz_neg, neg_part(k, d.W, d.dinvZ));
        RC(ew_lincomb(g.st, nn, 1.0, d.G, 0.0, nullptr, 0.0, nullptr, d.T));
        if (chol(n, d.T, d.dinvX) != 0) lamx_neg = std::max(lamx_neg, neg_part(k, d.G, d.dinvX));
    }
    std::vector<double> AX;
    aop_cat(cat.G, AX);   // scaled A' = d A: A_o(X_o) = AX / d
    double r2 = 0, dobj = 0;
    for (int i = 0; i < m; i++) {
        const double v = AX[i] / P.d[i] - P.b0[i];
        r2 += v * v;
        dobj += P.b0[i] * res.y[i];
    }
    const double den = 1 + std::fabs(pobj) + std::fabs(dobj);
    res.err[1] = std::sqrt(r2) / (1 + P.normb1);
    res.err[2] = std::max(0.0, lamx_neg) / (1 + P.normb1);
    res.err[3] = 0;
    res.err[4] = std::max(0.0, lamz_neg) / (1 + P.normC1);
    res.err[5] = (pobj - dobj) / den;
    res.err[6] = xz / den;
    res.pobj = pobj;
    res.dobj = dobj;
    res.have_x = 1;
    res.d2h_bytes = 0;
    for (int k = 0; k < nb; k++) res.d2h_bytes += 2.0 * sizeof(double) * (double)db[k].n * db[k].n;
    CU(cudaStreamSynchronize(g.st));
}

struct IterRes {   // Result measures of an iterate (scaled problem), as in solver.c:14470-14484
    double pobj = 0, dobj = 0, pinf = 0, dinf = 0, relgap = 0, relcomp = 0, err[7] = {0, 0, 0, 0, 0, 0, 0};
};
static double nan_inf(double v) { return v != v ? INFINITY : v; }
static double res_score(const IterRes &R) {
    return std::max(std::max(nan_inf(R.relgap), nan_inf(R.relcomp)), std::max(nan_inf(R.pinf), nan_inf(R.dinf)));
}
static double dimacs_score(const IterRes &R) {
    return std::max(std::max(std::fabs(nan_inf(R.err[1])), std::fabs(nan_inf(R.err[3]))),
                    std::max(std::fabs(nan_inf(R.err[5])), std::fabs(nan_inf(R.err[6]))));
}

// start_sdpt3 (solver.c:6622-6661): X = xi I, Z = eta I per block, their factors, the factors'
// diagonal-block inverses and the inverses of the factors.  An LP block as given takes one xi and
// one eta, from its order N and the norms over all its variables, for each of its blocks of order 1.
void Solver::start_sdpt3(bool unit) {
    std::vector<std::vector<double>> sval(6, std::vector<double>(nb, 0.0));
    std::vector<double> lp_xi(nb, 0.0), lp_eta(nb, 0.0);
    for (size_t kin = 0; kin < P.in_n.size(); kin++) {
        if (P.in_n[kin] > 0) continue;
        const int q0 = P.in_first[kin], q1 = P.in_first[kin + 1];
        double nC = 0, maxA = 0, ratio = 0;
        std::vector<double> a2(m, 0.0);
        std::vector<int> touched;
        for (int q = q0; q < q1; q++) {
            const HBlock &B = P.blk[q];
            for (double v : B.Cval) nC += v * v;
            for (size_t t = 0; t < B.con.size(); t++) {
                const int c = B.con[t];
                if (a2[c] == 0.0) touched.push_back(c);
                for (long long e = B.cptr[t]; e < B.cptr[t + 1]; e++) a2[c] += B.cval[e] * B.cval[e];
            }
        }
        nC = std::sqrt(nC);
        std::sort(touched.begin(), touched.end());
        for (int c : touched) {
            const double a = std::sqrt(a2[c]);
            maxA = std::max(maxA, a);
            ratio = std::max(ratio, (1 + std::fabs(P.b[c])) / (1 + a));
        }
        const int n = q1 - q0;
        const double xi = std::max(10.0, std::max(std::sqrt((double)n), n * ratio));
        const double eta = std::max(10.0, std::max(std::sqrt((double)n), std::max(maxA, nC)));
        for (int q = q0; q < q1; q++) {
            lp_xi[q] = xi;
            lp_eta[q] = eta;
        }
    }
    for (int k = 0; k < nb; k++) {
        const HBlock &B = P.blk[k];
        const int n = B.n;
        double nC = 0, maxA = 0, ratio = 0;
        for (double v : B.Cval) nC += v * v;
        nC = std::sqrt(nC);
        for (size_t t = 0; t < B.con.size(); t++) {
            double a = 0;
            for (long long e = B.cptr[t]; e < B.cptr[t + 1]; e++) a += B.cval[e] * B.cval[e];
            a = std::sqrt(a);
            maxA = std::max(maxA, a);
            ratio = std::max(ratio, (1 + std::fabs(P.b[B.con[t]])) / (1 + a));
        }
        const bool lp = lp_xi[k] > 0;
        double xi = lp ? lp_xi[k] : std::max(10.0, std::max(std::sqrt((double)n), n * ratio));
        double eta = lp ? lp_eta[k] : std::max(10.0, std::max(std::sqrt((double)n), std::max(maxA, nC)));
        if (unit) xi = eta = 1.0;
        DevArrays &d = da[k];
        if (n <= SMALL_N_MAX) {   // set below for all small blocks at once (closed form)
            sval[0][k] = xi;
            sval[1][k] = eta;
            sval[2][k] = std::sqrt(xi);
            sval[3][k] = std::sqrt(eta);
            sval[4][k] = 1.0 / std::sqrt(xi);
            sval[5][k] = 1.0 / std::sqrt(eta);
            continue;
        }
        RC(ew_set_scaled_identity(g.st, n, d.X, xi));
        RC(ew_set_scaled_identity(g.st, n, d.Z, eta));
        RC(ew_set_scaled_identity(g.st, n, d.LX, std::sqrt(xi)));
        RC(ew_set_scaled_identity(g.st, n, d.LZ, std::sqrt(eta)));
        // the factors' diagonal-block inverses: a Cholesky of the diagonal starts
        RC(ew_set_scaled_identity(g.st, n, d.T, xi));
        if (chol(n, d.T, d.dinvX)) throw GpuFail{BGPU_ERR_NOTPD, __LINE__};
        RC(ew_set_scaled_identity(g.st, n, d.T, eta));
        if (chol(n, d.T, d.dinvZ)) throw GpuFail{BGPU_ERR_NOTPD, __LINE__};
        inv_from_chol(n, d.LX, d.dinvX, d.LiX);
        inv_from_chol(n, d.LZ, d.dinvZ, d.LiZ);   // the small blocks' Z^-1 comes from LiZ
    }
    if (!small_ids.empty()) {   // X = xi I, Z = eta I, their factors and inverses (big blocks: kept)
        double *DevArrays::*mems[6] = {&DevArrays::X, &DevArrays::Z, &DevArrays::LX, &DevArrays::LZ, &DevArrays::LiX,
                                       &DevArrays::LiZ};
        for (int q = 0; q < 6; q++) {
            CU(cudaMemcpyAsync(d_bval, sval[q].data(), sizeof(double) * nb, cudaMemcpyHostToDevice, g.st));
            RC(ew_scaled_identity_blocks(g.st, nb, d_bn, d_boff, Ntot2, d_bval, d_bsmall, cat.*mems[q]));
            CU(cudaStreamSynchronize(g.st));   // d_bval is reused by the next member
        }
    }
}

int Solver::run(ResultData &res) {
    const double t0 = wtime();
    tm = Timings();
    want_double = is_float = reg_hint = false;
    reg = reg_ok = 0;
    min_pivot = 1;
    nfloat = nfactor = pcg_iters = 0;
    mu_now = 1e300;
    m_exact = true;
    asm_fp64 = late_exact = false;
    schur_flops = schur_dev_time = 0;
    CU(cudaEventRecord(evs0, g.st));
    std::vector<double> y(m, 0.0), ybest(m, 0.0), dy, rp(m), a0, h(m, 0.0), rhs(m), qv, ev(m), wv;
    std::vector<double> tmpv;
    start_sdpt3();
    if (opt.init >= 1 && m > 0) least_squares_start(y);
    // R0 = C - Z - A'y, theta = 1 (solver.c:14317-14326)
    double theta = 1.0, r0norm = 0;
    {
        atop_cat(y, -1.0, 0.0, cat.R0);
        lincomb_cat(1.0, Ccat, -1.0, cat.Z, 1.0, cat.R0, cat.R0);
        const double *aa[1] = {cat.R0};
        dots_cat(1, aa, aa, &r0norm);
    }
    r0norm = std::sqrt(r0norm);
    double nbs = nrm(P.b);
    int status = -1, it = 0, it_best = 0, stall = 0;
    double alp = 0, ald = 0, sigma = 0, best_score = INFINITY;
    IterRes R, best;
    const bool keep_best = true;
    const double Ntot = (double)P.Ntot;
    if (opt.verbose > 0)
        log_printf(0, " it   pobj            dobj            pinf     dinf     gap      mu       alp   ald   sigma  time\n");
    for (it = 0; it <= opt.maxit; it++) {
        double td = wtime();
        if (nt_mode) {
            // L_Z^-1 for the dual step length (zinv keeps it under HKM), then the scaling
            for (int k : big_ids) inv_from_chol(db[k].n, da[k].LZ, da[k].dinvZ, da[k].LiZ);
            if (!nt_scaling()) { status = 4; break; }
        } else {
            for (int k : big_ids) zinv(k);
            if (!small_ids.empty())   // Zi = LiZ' LiZ (symmetric part), LiZ from the last small Cholesky of Z
                RC(small_gemm(g.st, (int)small_ids.size(), d_sns, 1, 0, 1.0, (const double *const *)tab(&DevArrays::LiZ),
                              (const double *const *)tab(&DevArrays::LiZ), 0.0, tab(&DevArrays::Zi), 1));
        }
        // residuals and objectives
        std::vector<double> AX;
        aop_cat(cat.X, AX);
        for (int i = 0; i < m; i++) rp[i] = P.b[i] - AX[i];
        double pobj = 0, xz = 0, rdn2 = 0, nCR2 = 0, dev2 = 0;
        {
            atop_cat(y, 1.0, 0.0, cat.F);                                  // A'y
            lincomb_cat(1.0, cat.F, 1.0, cat.Z, 0.0, nullptr, cat.F);      // A'y + Z
            lincomb_cat(1.0, cat.F, -1.0, Ccat, 0.0, nullptr, cat.Fd);     // -Rd
            lincomb_cat(1.0, cat.Fd, theta, cat.R0, 0.0, nullptr, cat.T);  // -Rd + theta R0
            double part[5];
            const double *aa[5] = {cat.F, Ccat, cat.X, cat.Fd, cat.T}, *bb[5] = {cat.F, cat.X, cat.Z, cat.Fd, cat.T};
            dots_cat(5, aa, bb, part);
            nCR2 = part[0]; pobj = part[1]; xz = part[2]; rdn2 = part[3]; dev2 = part[4];
        }
        double dobj = dot(P.b, y);
        double mu = xz / Ntot;
        mu_now = P.bs * P.cs * mu;
        double rpo = 0;
        for (int i = 0; i < m; i++) { const double v = rp[i] * P.du[i]; rpo += v * v; }
        rpo = std::sqrt(rpo);
        const double rdo = P.cs * std::sqrt(rdn2);
        const double sc = P.bs * P.cs;
        const double po = sc * pobj, dob = sc * dobj;
        R.pobj = po; R.dobj = dob;
        R.pinf = rpo / (1 + P.normb2);
        R.dinf = rdo / (1 + P.normC2);
        const double oden = 1 + std::fabs(po) + std::fabs(dob);
        R.relgap = std::fabs(po - dob) / oden;
        R.relcomp = sc * xz / oden;
        R.err[1] = rpo / (1 + P.normb1);
        R.err[3] = rdo / (1 + P.normC1);
        R.err[5] = (po - dob) / oden;
        R.err[6] = sc * xz / oden;
        tm.dense += wtime() - td;
        if (opt.verbose > 0)
            log_printf(0, "%3d %+.8e %+.8e %.2e %.2e %.2e %.2e %.3f %.3f %.3f %6.2f\n", it, -po, -dob, R.pinf, R.dinf,
                       R.relgap, sc * mu, alp, ald, sigma, wtime() - t0);
        if (!std::isfinite(po) || !std::isfinite(dob)) { status = 4; break; }
        const double score = res_score(R);
        if (score < best_score) {
            best_score = score;
            it_best = it;
            best = R;
            ybest = y;
            if (keep_best) {
                CU(cudaMemcpyAsync(cat.Xb, cat.X, sizeof(double) * Ntot2, cudaMemcpyDeviceToDevice, g.st));
                CU(cudaMemcpyAsync(cat.Zb, cat.Z, sizeof(double) * Ntot2, cudaMemcpyDeviceToDevice, g.st));
            }
        }
        if (score < opt.tol) { status = 0; break; }
        if (keep_best && it > it_best && dimacs_score(best) <= 0.5 * opt.tol) { status = 4; break; }
        if (opt.timelimit > 0 && wtime() - t0 > opt.timelimit) { status = 6; break; }
        const double nCR = std::sqrt(nCR2);
        if (!opt.known_feasible && dobj > 0 && nCR / dobj < 1e-8 && it > 5) { status = 1; break; }
        double nAX = 0;
        for (int i = 0; i < m; i++) { const double v = P.b[i] - rp[i]; nAX += v * v; }
        nAX = std::sqrt(nAX);
        if (!opt.known_feasible && pobj < 0 && nAX / (-pobj) < 1e-8 && it > 5) { status = 2; break; }
        if (it == opt.maxit) { status = 3; break; }
        if (stall >= 3) { status = 4; break; }
        if (it - it_best >= opt.stall_win && best_score < 1e-6) { status = 4; break; }
        if (it - it_best >= 8 && best_score < 1e-4) { status = 4; break; }
        if (it - it_best >= 12) { status = 4; break; }
        // re-base the dual residual when the recurrence has drifted
        {
            const double dev = std::sqrt(dev2);
            if (dev > 1e-10 * (1.0 + theta * r0norm) && dev > 1e-12) {
                theta = 1.0;
                r0norm = std::sqrt(rdn2);
                lincomb_cat(-1.0, cat.Fd, 0.0, nullptr, 0.0, nullptr, cat.R0);
            }
            if (theta * r0norm <= 1e-13) theta = 0.0;
        }
        // ---- Schur complement ----
        const double ts_before = tm.schur, tstep_before = tm.step;
        double ts = wtime();
        assemble(tmpv);
        double tc = wtime();
        tm.schur += tc - ts;
        int frc = factor();
        if (!m_exact && frc == 0 && reg > 0 && opt.mixed_shift) {
            // the 3xTF32 M is FP32-accurate and its factor needed a shift: PCG against the FP64
            // operator with the shifted factor (schur_solve turns to FP64 assembly if it misses)
            if (opt.verbose > 1) log_printf(0, "   mixed path: the 3xTF32 M factored with shift %.1e\n", reg);
        } else if (!m_exact && (frc != 0 || reg > 0) && raise_precision()) {
            // an approximate M (3xTF32, or the preconditioner-grade late form): once its factor
            // needs a regularization it no longer preconditions the FP64 system; this and the later
            // iterations assemble more accurately
            reg_hint = false;
            reg_ok = 0;
            if (opt.verbose > 1)
                log_printf(0, "   mixed path: the %s M needed a shift: more accurate assembly from here on\n", asm_label);
            tm.chol += wtime() - tc;
            ts = wtime();
            assemble(tmpv);
            tc = wtime();
            tm.schur += tc - ts;
            frc = factor();
            if (!m_exact && (frc != 0 || reg > 0) && raise_precision()) {   // the late form needed one too
                if (opt.verbose > 1)
                    log_printf(0, "   mixed path: the %s M needed a shift: FP64-accurate assembly from here on\n", asm_label);
                reg_hint = false;
                reg_ok = 0;
                ts = wtime();
                assemble(tmpv);
                tc = wtime();
                tm.schur += tc - ts;
                frc = factor();
            }
        }
        if (frc != 0) { status = 4; tm.chol += wtime() - tc; break; }
        if (cur_prec == 1 && !asm_fp64 && !opt.mixed_shift && min_pivot < 1e-4) {
            // the FP32-accurate M is near the end of its use: its smallest scaled pivot falls by
            // 10-20x an iteration, and the factor of the next one would need a shift (rand1000: pivot
            // 7.9e-5, then a shift) — the next iterations assemble in FP64 directly
            asm_fp64 = true;
            if (opt.verbose > 1) log_printf(0, "   mixed path: smallest pivot %.1e: FP64-accurate assembly from the next iteration\n", min_pivot);
        }
        tm.chol += wtime() - tc;
        // ---- rhs pieces ----
        td = wtime();
        const bool hasH = theta > 0;
        {
            if (!nt_mode) aop_cat(cat.Zi, a0);
            if (hasH) {
                mul_all(theta, &DevArrays::Zi, &DevArrays::R0, &DevArrays::T);   // theta Zi R0
                mul_all(1.0, &DevArrays::T, xmem(), &DevArrays::G);              // theta Zi R0 X (W theta R0 W)
                aop_cat(cat.G, h);
            } else h.assign(m, 0.0);
        }
        tm.dense += wtime() - td;
        // ---- predictor ----
        for (int i = 0; i < m; i++) rhs[i] = P.b[i] + h[i];
        tc = wtime();
        schur_solve(rhs, dy, 1e-7);
        tm.chol += wtime() - tc;
        td = wtime();
        atop_cat(dy, -1.0, 0.0, cat.dZ);
        lincomb_cat(1.0, cat.dZ, theta, cat.R0, 0.0, nullptr, cat.dZ);   // dZ = -A'dy + theta R0
        if (nt_mode) {   // the scaled predictor (solver.c:14740-14792): dXt = Rt - G' dZ G, Rt = -diag(lam)
            RC(nt::rhs_scaled(g.st, nb, d_bn, d_boff, d_loff, Ntot2, nlam, 0.0, nullptr, cat.Rt));
            nt_toZ(&DevArrays::dZ, &DevArrays::dZt);
            lincomb_cat(1.0, cat.Rt, -1.0, cat.dZt, 0.0, nullptr, cat.dXt);
            nt_fromS(&DevArrays::dXt, &DevArrays::dX);                    // dX = G dXt G'
        } else {
            mul_all(1.0, &DevArrays::Zi, &DevArrays::dZ, &DevArrays::T);
            mul_all(1.0, &DevArrays::T, &DevArrays::X, &DevArrays::G);    // Zi dZ X
            sym_cat(cat.G, -1.0, -1.0, cat.X, 0.0, nullptr, cat.dX);      // dX = -sym(G) - X
        }
        tm.dense += wtime() - td;
        double tst = wtime();
        const double ap = std::min(1.0, maxstep(1, opt.lanczos_k));
        const double ad = std::min(1.0, maxstep(0, opt.lanczos_k));
        tm.step += wtime() - tst;
        double xdz = 0, dxz = 0, dxdz = 0;
        {
            double t3[3];
            const double *aa[3] = {cat.X, cat.dX, cat.dX}, *bb[3] = {cat.dZ, cat.Z, cat.dZ};
            dots_cat(3, aa, bb, t3);
            xdz = t3[0]; dxz = t3[1]; dxdz = t3[2];
        }
        const double mu_a = (xz + ap * dxz + ad * xdz + ap * ad * dxdz) / Ntot;
        const double frac = std::max(0.0, mu_a / mu);
        const double mina = std::min(ap, ad);
        // the default (solver.c:14848-14851): the adaptive rule, the cubic one when the problem
        // as given has no SDP block (LP blocks only)
        int rule = opt.sigma_rule < 0 ? (P.lp_only ? 1 : 0) : opt.sigma_rule;
        double expon;
        if (rule == 1) expon = 3.0;
        else if (rule == 2) expon = (mina < 0.1) ? 1.0 : 3.0;
        else expon = (R.relgap > 1e-6) ? std::max(1.0, 3 * mina * mina) : 3.0;
        sigma = std::min(1.0, std::pow(frac, expon));
        if (sigma < opt.sigma_min) sigma = opt.sigma_min;
        {
            const double infeas = std::max(R.pinf, R.dinf), bal = opt.balance;
            if (bal > 0 && infeas > bal * R.relcomp && R.relcomp > 0) {
                const double s_min = std::min(1.0, infeas / (bal * R.relcomp) * 0.1);
                if (sigma < s_min) sigma = s_min;
            }
        }
        const double gamma = 0.9 + (opt.gamma_max - 0.9) * mina;
        // ---- corrector ----
        const double smu = sigma * mu;
        td = wtime();
        if (nt_mode) {
            // the scaled corrector (solver.c:14876-14906, 14976-14996): Rt = L_lam^-1(smu I - lam^2 -
            // sym(dXt dZt)), rhs = b + h - A(G (Rt + lam) G'), then dX = G (Rt - G' dZ G) G'
            mul_sym_all(&DevArrays::dXt, &DevArrays::dZt, &DevArrays::W);
            RC(nt::rhs_scaled(g.st, nb, d_bn, d_boff, d_loff, Ntot2, nlam, smu, cat.W, cat.Rt));
            RC(nt::add_lam(g.st, nb, d_bn, d_boff, d_loff, Ntot2, nlam, 1.0, cat.Rt, cat.Q));
            nt_fromS(&DevArrays::Q, &DevArrays::G);
            aop_cat(cat.G, qv);
            for (int i = 0; i < m; i++) rhs[i] = P.b[i] + h[i] - qv[i];
        } else {
            mul_all(1.0, &DevArrays::Zi, &DevArrays::dZ, &DevArrays::T);
            mul_all(1.0, &DevArrays::T, &DevArrays::dX, &DevArrays::Q);   // Q = Zi dZp dXp
            aop_cat(cat.Q, qv);
            for (int i = 0; i < m; i++) rhs[i] = P.b[i] - smu * a0[i] + qv[i] + h[i];
        }
        tm.dense += wtime() - td;
        tc = wtime();
        schur_solve(rhs, dy, 0);
        tm.chol += wtime() - tc;
        td = wtime();
        atop_cat(dy, -1.0, 0.0, cat.dZ);
        lincomb_cat(1.0, cat.dZ, theta, cat.R0, 0.0, nullptr, cat.dZ);
        if (nt_mode) {
            nt_toZ(&DevArrays::dZ, &DevArrays::Q);
            lincomb_cat(1.0, cat.Rt, -1.0, cat.Q, 0.0, nullptr, cat.W);
            nt_fromS(&DevArrays::W, &DevArrays::dX);
        } else {
            mul_all(1.0, &DevArrays::Zi, &DevArrays::dZ, &DevArrays::T);
            mul_all(1.0, &DevArrays::T, &DevArrays::X, &DevArrays::G);
            lincomb_cat(1.0, cat.G, 1.0, cat.Q, 0.0, nullptr, cat.G);          // Zi dZ X + Q
            sym_cat(cat.G, -1.0, smu, cat.Zi, -1.0, cat.X, cat.dX);            // -sym(.) + smu Zi - X
        }
        tm.dense += wtime() - td;
        // ---- refinement of A(dX) = rp ----
        for (int pass = 0; pass < 3; pass++) {
            td = wtime();
            std::vector<double> AdX;
            aop_cat(cat.dX, AdX);
            for (int i = 0; i < m; i++) ev[i] = rp[i] - AdX[i];
            const double ne = nrm(ev), nrp = nrm(rp);
            tm.dense += wtime() - td;
            if (!(ne > 1e-2 * nrp && ne > 1e-3 * opt.tol * (1 + nbs))) break;
            tc = wtime();
            schur_solve(ev, wv, 0);
            tm.chol += wtime() - tc;
            td = wtime();
            atop_cat(wv, 1.0, 0.0, cat.W);                                       // A'w
            mul_all(1.0, &DevArrays::Zi, &DevArrays::W, &DevArrays::T);
            mul_all(1.0, &DevArrays::T, xmem(), &DevArrays::F);                  // Zi A'w X (W A'w W), F is free here
            sym_cat(cat.F, 1.0, 0.0, nullptr, 0.0, nullptr, cat.G);
            std::vector<double> AG;
            aop_cat(cat.G, AG);
            for (int i = 0; i < m; i++) qv[i] = ev[i] - AG[i];
            const double ne2 = nrm(qv);
            tm.dense += wtime() - td;
            if (!(ne2 < 0.5 * ne)) break;
            for (int i = 0; i < m; i++) dy[i] += wv[i];
            lincomb_cat(1.0, cat.dZ, -1.0, cat.W, 0.0, nullptr, cat.dZ);
            lincomb_cat(1.0, cat.dX, 1.0, cat.G, 0.0, nullptr, cat.dX);
        }
        tst = wtime();
        const double apr = std::min(1.0, maxstep(1, opt.lanczos_k));
        const double adr = std::min(1.0, maxstep(0, opt.lanczos_k));
        tm.step += wtime() - tst;
        double apn = std::min(1.0, gamma * apr), adn = std::min(1.0, gamma * adr);
        // catastrophe guard (solver.c:15138-15158)
        if (R.pinf < 1e-6) {
            td = wtime();
            std::vector<double> AdX;
            aop_cat(cat.dX, AdX);
            for (int i = 0; i < m; i++) ev[i] = rp[i] - AdX[i];
            const double nrp = nrm(rp), nev = nrm(ev);
            tm.dense += wtime() - td;
            const double gg = std::max(1e3, 1e-6 / std::max(R.pinf, 1e-300));
            const double lim = gg * nrp;
            if (nev > lim && nrp > 0) {
                const double cap = lim / nev;
                if (cap < apn) apn = cap;
                if (allow_float) want_double = true;
            }
        }
        tst = wtime();
        const int okp = try_step(1, &apn);
        const int okd = try_step(0, &adn);
        for (int k : big_ids) inv_from_chol(db[k].n, da[k].LX, da[k].dinvX, da[k].LiX);
        tm.step += wtime() - tst;
        if (!okp || !okd) { status = 4; break; }
        for (int i = 0; i < m; i++) y[i] += adn * dy[i];
        theta *= (1.0 - adn);
        if (opt.verbose > 1)
            log_printf(0, "     [schur %.3fs %s, factor %s reg %.0e pmin %.1e, pcg %d, step %.3fs%s]\n", tm.schur - ts_before,
                       asm_label, is_float ? "fp32" : "fp64", reg, min_pivot, pcg_iters, tm.step - tstep_before,
                       nt_mode && !big_ids.empty() ? (", NT sweeps " + std::to_string(nt_sweeps)).c_str() : "");
        alp = apn;
        ald = adn;
        stall = (apn < 1e-6 && adn < 1e-6) ? stall + 1 : 0;
    }
    res.iters = it;
    res.direction = nt_mode ? 1 : 0;
    res.embedding = 0;
    // fall back to the best iterate seen
    if (status != 0 && status != 1 && status != 2 && best_score < res_score(R)) {
        R = best;
        y = ybest;
        CU(cudaMemcpyAsync(cat.X, cat.Xb, sizeof(double) * Ntot2, cudaMemcpyDeviceToDevice, g.st));
        CU(cudaMemcpyAsync(cat.Z, cat.Zb, sizeof(double) * Ntot2, cudaMemcpyDeviceToDevice, g.st));
        if (opt.verbose > 1) log_printf(0, "   returning best iterate (iteration %d)\n", it_best);
    }
    final_measures(y, res);
    // the status of the returned point as measured on the data as given (main.c:2349-2362)
    const double acc = std::max(std::max(res.err[1], res.err[2]),
                                std::max(res.err[4], std::max(std::fabs(res.err[5]), std::fabs(res.err[6]))));
    if (status == 0 || status == 5 || status == 3 || status == 4 || status == 6) {
        if (acc <= opt.tol) status = 0;
        else if (acc <= opt.red_acc) status = 5;
        else if (status == 0 || status == 5) status = 4;
    }
    res.status = status;
    res.exit_code = exit_code_of(status);
    res.nfloat = nfloat;
    res.nfactor = nfactor;
    res.pcg_iters = pcg_iters;
    res.schur_flops = schur_flops;
    res.schur_time = schur_dev_time;
    CU(cudaEventRecord(evs1, g.st));
    CU(cudaEventSynchronize(evs1));
    float dms = 0;
    CU(cudaEventElapsedTime(&dms, evs0, evs1));
    res.device_time = dms * 1e-3;
    tm.total = wtime() - t0;
    res.t = tm;
    res.time = tm.total;
    return res.exit_code;
}

// The self-dual embedding (the reference's hsd_run, solver.c:9803, which BRISK runs first on most
// problems), as this build's own homogeneous self-dual predictor-corrector with the HKM direction
// (the reference's direction in the embedding, solver.c:13566).  With tau, kappa >= 0 the scaled
// problem is embedded as
//     A(X) - b tau = 0,   A'y + Z - C tau = 0,   b'y - <C,X> - kappa = 0,
//     X Z = mu I,  tau kappa = mu,  mu = (<X,Z> + tau kappa) / (N + 1),
// and the residuals rp = b tau - A(X), Rd = C tau - A'y - Z, rg = kappa - b'y + <C,X> fall by
// 1 - eta alpha a step (predictor: sigma 0, eta 1; corrector: Mehrotra's sigma, eta = 1 - sigma
// and the second-order terms).  The Newton system reduces to the infeasible method's Schur
// complement M:
//     dZ = C dtau - A'dy + eta Rd,  dX = sigma mu Zi - X - sym(Zi dZ X + Q),  Q = Zi dZp dXp,
//     dkappa = (sigma mu - tau kappa - dtau_p dkappa_p - kappa dtau) / tau,
//     M dy - p dtau = eta rp - sigma mu A(Zi) + A(X) + eta A(Zi Rd X) + A(Q),   p = A(Zi C X) + b,
//     (2b - p)'dy + (<C, Zi C X> + kappa / tau) dtau =
//         eta rg + sigma mu <C, Zi> - <C, X> - eta <C, Zi Rd X> - <C, Q> + (sigma mu - tau kappa - dtau_p dkappa_p) / tau,
// so dy = u + v dtau with M u = (the first right side) and M v = p; dtau's coefficient and right
// side are evaluated in a cancellation-free form (below): four Schur solves an iteration, one
// factor.  One step length for every variable keeps the
// residuals falling together.  The solution is X / tau, y / tau; kappa >> tau certifies
// infeasibility (b'y > 0: primal, <C,X> < 0: dual).  The start is X = Z = I on the equilibrated
// problem (its rows and C scaled to norm 1), tau = 1 and kappa = <X,Z> / N = 1, on the central
// path: in a dense prototype it took 1-3 iterations fewer than start_sdpt3's xi I, eta I on every
// parity instance.
int Solver::run_hsd(ResultData &res) {
    const double t0 = wtime();
    tm = Timings();
    want_double = is_float = reg_hint = false;
    reg = reg_ok = 0;
    min_pivot = 1;
    nfloat = nfactor = pcg_iters = 0;
    mu_now = 1e300;
    m_exact = true;
    asm_fp64 = late_exact = false;
    schur_flops = schur_dev_time = 0;
    CU(cudaEventRecord(evs0, g.st));
    const bool nt_saved = nt_mode;   // a session's solver keeps its own direction for run()
    nt_mode = false;
    std::vector<double> y(m, 0.0), ybest(m, 0.0), rp(m), a0, pv, hv, qv, rhs(m), u, v, dy(m), tmpv, AX;
    start_sdpt3(true);
    const double Ntot = (double)P.Ntot;
    double tau = 1.0, kap = 0.0;
    {
        const double *aa[1] = {cat.X}, *bb[1] = {cat.Z};
        dots_cat(1, aa, bb, &kap);
        kap /= Ntot;
    }
    int status = -1, it = 0, it_best = 0, stall = 0;
    double alpha = 0, sigma = 0, best_score = INFINITY, tau_best = 1.0;
    IterRes R, best;
    if (opt.verbose > 0)
        log_printf(0, " it   pobj            dobj            pinf     dinf     gap      mu       alp   ald   sigma  time\n");
    for (it = 0; it <= opt.maxit; it++) {
        double td = wtime();
        for (int k : big_ids) zinv(k);
        if (!small_ids.empty())
            RC(small_gemm(g.st, (int)small_ids.size(), d_sns, 1, 0, 1.0, (const double *const *)tab(&DevArrays::LiZ),
                          (const double *const *)tab(&DevArrays::LiZ), 0.0, tab(&DevArrays::Zi), 1));
        // residuals of the embedding
        aop_cat(cat.X, AX);
        for (int i = 0; i < m; i++) rp[i] = P.b[i] * tau - AX[i];
        atop_cat(y, 1.0, 0.0, cat.F);                                   // A'y
        lincomb_cat(tau, Ccat, -1.0, cat.F, -1.0, cat.Z, cat.Fd);       // Rd = C tau - A'y - Z
        double cx = 0, xz = 0, rd2 = 0;
        {
            double part[3];
            const double *aa[3] = {Ccat, cat.X, cat.Fd}, *bb[3] = {cat.X, cat.Z, cat.Fd};
            dots_cat(3, aa, bb, part);
            cx = part[0]; xz = part[1]; rd2 = part[2];
        }
        const double by = dot(P.b, y);
        const double rg = kap - by + cx;
        const double mu = (xz + tau * kap) / (Ntot + 1);
        // the measures of the solution X / tau, y / tau, Z / tau (as the infeasible method's)
        const double sc = P.bs * P.cs;
        mu_now = sc * xz / (tau * tau * Ntot);
        double rpo = 0;
        for (int i = 0; i < m; i++) { const double w = rp[i] * P.du[i]; rpo += w * w; }
        rpo = std::sqrt(rpo) / tau;
        const double rdo = P.cs * std::sqrt(rd2) / tau;
        const double po = sc * cx / tau, dob = sc * by / tau;
        R.pobj = po; R.dobj = dob;
        R.pinf = rpo / (1 + P.normb2);
        R.dinf = rdo / (1 + P.normC2);
        const double oden = 1 + std::fabs(po) + std::fabs(dob);
        R.relgap = std::fabs(po - dob) / oden;
        R.relcomp = sc * xz / (tau * tau) / oden;
        R.err[1] = rpo / (1 + P.normb1);
        R.err[3] = rdo / (1 + P.normC1);
        R.err[5] = (po - dob) / oden;
        R.err[6] = R.relcomp;
        tm.dense += wtime() - td;
        if (opt.verbose > 0)
            log_printf(0, "%3d %+.8e %+.8e %.2e %.2e %.2e %.2e %.3f %.3f %.3f %6.2f\n", it, -po, -dob, R.pinf, R.dinf,
                       R.relgap, mu_now, alpha, alpha, sigma, wtime() - t0);
        if (!std::isfinite(po) || !std::isfinite(dob) || !(tau > 0) || !(kap > 0)) { status = 4; break; }
        const double score = res_score(R);
        if (score < best_score) {
            best_score = score;
            it_best = it;
            best = R;
            ybest = y;
            tau_best = tau;
            CU(cudaMemcpyAsync(cat.Xb, cat.X, sizeof(double) * Ntot2, cudaMemcpyDeviceToDevice, g.st));
            CU(cudaMemcpyAsync(cat.Zb, cat.Z, sizeof(double) * Ntot2, cudaMemcpyDeviceToDevice, g.st));
        }
        if (score < opt.tol) { status = 0; break; }
        if (it > it_best && dimacs_score(best) <= 0.5 * opt.tol) { status = 4; break; }
        if (opt.timelimit > 0 && wtime() - t0 > opt.timelimit) { status = 6; break; }
        if (kap > 1e8 * tau) {   // the embedding's certificate: tau -> 0 with kappa > 0
            if (by > 0 && !opt.known_feasible) { status = 1; break; }
            if (cx < 0 && !opt.known_feasible) { status = 2; break; }
            status = 4;
            break;
        }
        if (it == opt.maxit) { status = 3; break; }
        if (stall >= 3) { status = 4; break; }
        if (it - it_best >= opt.stall_win && best_score < 1e-6) { status = 4; break; }
        if (it - it_best >= 12) { status = 4; break; }
        // ---- Schur complement (the infeasible method's, with its precision ladder) ----
        const double ts_before = tm.schur, tstep_before = tm.step;
        double ts = wtime();
        assemble(tmpv);
        double tc = wtime();
        tm.schur += tc - ts;
        int frc = factor();
        if (!m_exact && (frc != 0 || reg > 0) && raise_precision()) {
            reg_hint = false;
            reg_ok = 0;
            tm.chol += wtime() - tc;
            ts = wtime();
            assemble(tmpv);
            tc = wtime();
            tm.schur += tc - ts;
            frc = factor();
            if (!m_exact && (frc != 0 || reg > 0) && raise_precision()) {
                reg_hint = false;
                reg_ok = 0;
                ts = wtime();
                assemble(tmpv);
                tc = wtime();
                tm.schur += tc - ts;
                frc = factor();
            }
        }
        if (frc != 0) { status = 4; tm.chol += wtime() - tc; break; }
        if (cur_prec == 1 && !asm_fp64 && min_pivot < 1e-4) asm_fp64 = true;
        tm.chol += wtime() - tc;
        // ---- the pieces both directions share ----
        // dy = u + (v1 + w) dtau with M v1 = A(Zi C X), M w = b.  The third equation's coefficient
        // of dtau, (2b - p)'v + <C, Zi C X> + kappa/tau, is the difference of two terms that grow
        // like 1/mu; it equals the sum of three non-negative ones,
        //     den = b'w + <R, Zi R X> + kappa/tau,   R = C - A'v1,
        // and the right side likewise loses its 1/mu terms when written with R (below), so both
        // keep their accuracy to the end of the solve whatever the solves' residuals.
        // (scratch: the PCG's matrix-free operator, newton_mv, overwrites F, W and T, so what must
        // outlive a solve sits in R0 (C, then R) and Fd (Rd))
        td = wtime();
        CU(cudaMemcpyAsync(cat.R0, Ccat, sizeof(double) * Ntot2, cudaMemcpyDeviceToDevice, g.st));
        aop_cat(cat.Zi, a0);                                             // A(Zi)
        mul_all(1.0, &DevArrays::Zi, &DevArrays::R0, &DevArrays::T);     // Zi C
        mul_all(1.0, &DevArrays::T, &DevArrays::X, &DevArrays::G);       // Zi C X
        aop_cat(cat.G, pv);                                              // A(Zi C X)
        mul_all(1.0, &DevArrays::Zi, &DevArrays::Fd, &DevArrays::T);     // Zi Rd
        mul_all(1.0, &DevArrays::T, &DevArrays::X, &DevArrays::W);       // Zi Rd X
        aop_cat(cat.W, hv);
        tm.dense += wtime() - td;
        tc = wtime();
        schur_solve(pv, v, 0);                                           // v1
        std::vector<double> wv;
        schur_solve(P.b, wv, 0);                                         // w
        tm.chol += wtime() - tc;
        td = wtime();
        atop_cat(v, -1.0, 0.0, cat.R0);
        lincomb_cat(1.0, Ccat, 1.0, cat.R0, 0.0, nullptr, cat.R0);       // R = C - A'v1
        mul_all(1.0, &DevArrays::Zi, &DevArrays::R0, &DevArrays::T);
        mul_all(1.0, &DevArrays::T, &DevArrays::X, &DevArrays::G);       // Zi R X
        double rwr = 0, rzi = 0, rx = 0, rw = 0;
        {   // <R, Zi Rd X> as <Rd, Zi R X> (equal: tr(R Zi Rd X) = tr(Rd Zi R X))
            double part[4];
            const double *aa[4] = {cat.R0, cat.R0, cat.R0, cat.Fd}, *bb[4] = {cat.G, cat.Zi, cat.X, cat.G};
            dots_cat(4, aa, bb, part);
            rwr = part[0]; rzi = part[1]; rx = part[2]; rw = part[3];
        }
        tm.dense += wtime() - td;
        const double den = dot(P.b, wv) + rwr + kap / tau;
        if (!(den > 0) || !std::isfinite(den)) { status = 4; break; }
        const double v1rp = dot(v, rp);
        for (int i = 0; i < m; i++) v[i] += wv[i];                       // v = v1 + w
        // one direction: returns dtau, dkappa; dy, dZ, dX on the device / host.  rq = <R, Q>.
        //   dtau = (eta rg + (smu - tau kappa - dtdk)/tau - b'u + eta v1'rp + smu <R,Zi> - <R,X>
        //           - eta <R, Zi Rd X> - <R,Q>) / den
        auto direction = [&](double smu, double eta, bool corr, double dtdk, double rq, double &dt, double &dk) {
            for (int i = 0; i < m; i++)
                rhs[i] = eta * rp[i] - smu * a0[i] + AX[i] + eta * hv[i] + (corr ? qv[i] : 0.0);
            double t1 = wtime();
            schur_solve(rhs, u, corr ? 0 : 1e-7);
            tm.chol += wtime() - t1;
            t1 = wtime();
            const double num = eta * rg + (smu - tau * kap - dtdk) / tau - dot(P.b, u) + eta * v1rp + smu * rzi - rx -
                               eta * rw - rq;
            dt = num / den;
            for (int i = 0; i < m; i++) dy[i] = u[i] + v[i] * dt;
            atop_cat(dy, -1.0, 0.0, cat.dZ);
            lincomb_cat(dt, Ccat, 1.0, cat.dZ, eta, cat.Fd, cat.dZ);      // dZ = C dt - A'dy + eta Rd
            mul_all(1.0, &DevArrays::Zi, &DevArrays::dZ, &DevArrays::T);
            mul_all(1.0, &DevArrays::T, &DevArrays::X, &DevArrays::G);    // Zi dZ X
            if (corr) lincomb_cat(1.0, cat.G, 1.0, cat.Q, 0.0, nullptr, cat.G);
            sym_cat(cat.G, -1.0, smu, cat.Zi, -1.0, cat.X, cat.dX);       // -sym(.) + smu Zi - X
            dk = (smu - tau * kap - dtdk - kap * dt) / tau;
            tm.dense += wtime() - t1;
        };
        auto ratio = [](double x, double dx) { return dx < 0 ? -x / dx : 1e30; };
        // ---- predictor ----
        double dtp = 0, dkp = 0;
        direction(0.0, 1.0, false, 0.0, 0.0, dtp, dkp);
        double tst = wtime();
        const double apx = maxstep(1, opt.lanczos_k), apz = maxstep(0, opt.lanczos_k);
        tm.step += wtime() - tst;
        const double ap = std::min(1.0, std::min(std::min(apx, apz), std::min(ratio(tau, dtp), ratio(kap, dkp))));
        double xdz = 0, dxz = 0, dxdz = 0;
        {
            double t3[3];
            const double *aa[3] = {cat.X, cat.dX, cat.dX}, *bb[3] = {cat.dZ, cat.Z, cat.dZ};
            dots_cat(3, aa, bb, t3);
            xdz = t3[0]; dxz = t3[1]; dxdz = t3[2];
        }
        const double mu_a = (xz + ap * (xdz + dxz) + ap * ap * dxdz + (tau + ap * dtp) * (kap + ap * dkp)) / (Ntot + 1);
        const double expon = R.relgap > 1e-6 ? std::max(1.0, 3.0 * ap * ap) : 3.0;
        sigma = std::min(1.0, std::pow(std::max(0.0, mu_a / mu), expon));
        if (sigma < opt.sigma_min) sigma = opt.sigma_min;
        // ---- corrector ----
        td = wtime();
        mul_all(1.0, &DevArrays::Zi, &DevArrays::dZ, &DevArrays::T);
        mul_all(1.0, &DevArrays::T, &DevArrays::dX, &DevArrays::Q);       // Q = Zi dZp dXp
        aop_cat(cat.Q, qv);
        double cq = 0;   // <R, Q>
        {
            const double *aa[1] = {cat.R0}, *bb[1] = {cat.Q};
            dots_cat(1, aa, bb, &cq);
        }
        tm.dense += wtime() - td;
        double dt = 0, dk = 0;
        direction(sigma * mu, 1.0 - sigma, true, dtp * dkp, cq, dt, dk);
        tst = wtime();
        const double ax = maxstep(1, opt.lanczos_k), az = maxstep(0, opt.lanczos_k);
        tm.step += wtime() - tst;
        const double amax = std::min(std::min(ax, az), std::min(ratio(tau, dt), ratio(kap, dk)));
        const double gamma = 0.9 + (opt.gamma_max - 0.9) * std::min(1.0, amax);
        double a = std::min(1.0, gamma * amax);
        // one step for every variable: Z first, then X; Z moved back if X needed a shorter one
        tst = wtime();
        int ok = try_step(0, &a);
        const double a_z = a;
        ok = ok && try_step(1, &a);
        if (ok && a < a_z) {
            const double a_x = a;
            ok = try_step(0, &a, a_z);
            if (ok && a < a_x) ok = try_step(1, &a, a_x);
        }
        for (int k : big_ids) inv_from_chol(db[k].n, da[k].LX, da[k].dinvX, da[k].LiX);
        tm.step += wtime() - tst;
        if (!ok) { status = 4; break; }
        for (int i = 0; i < m; i++) y[i] += a * dy[i];
        tau += a * dt;
        kap += a * dk;
        if (opt.verbose > 1)
            log_printf(0, "     [schur %.3fs %s, factor %s reg %.0e pmin %.1e, pcg %d, step %.3fs, tau %.3e kappa %.3e]\n",
                       tm.schur - ts_before, asm_label, is_float ? "fp32" : "fp64", reg, min_pivot, pcg_iters,
                       tm.step - tstep_before, tau, kap);
        alpha = a;
        stall = a < 1e-6 ? stall + 1 : 0;
    }
    res.iters = it;
    res.direction = 0;
    res.embedding = 1;
    nt_mode = nt_saved;
    if (status != 0 && status != 1 && status != 2 && best_score < res_score(R)) {
        R = best;
        y = ybest;
        tau = tau_best;
        CU(cudaMemcpyAsync(cat.X, cat.Xb, sizeof(double) * Ntot2, cudaMemcpyDeviceToDevice, g.st));
        CU(cudaMemcpyAsync(cat.Z, cat.Zb, sizeof(double) * Ntot2, cudaMemcpyDeviceToDevice, g.st));
        if (opt.verbose > 1) log_printf(0, "   returning best iterate (iteration %d)\n", it_best);
    }
    // the solution of the embedding: X / tau, y / tau (final_measures takes Z as C - A'y)
    lincomb_cat(1.0 / tau, cat.X, 0.0, nullptr, 0.0, nullptr, cat.X);
    for (int i = 0; i < m; i++) y[i] /= tau;
    final_measures(y, res);
    const double acc = std::max(std::max(res.err[1], res.err[2]),
                                std::max(res.err[4], std::max(std::fabs(res.err[5]), std::fabs(res.err[6]))));
    if (status == 0 || status == 5 || status == 3 || status == 4 || status == 6) {
        if (acc <= opt.tol) status = 0;
        else if (acc <= opt.red_acc) status = 5;
        else if (status == 0 || status == 5) status = 4;
    }
    res.status = status;
    res.exit_code = exit_code_of(status);
    res.nfloat = nfloat;
    res.nfactor = nfactor;
    res.pcg_iters = pcg_iters;
    res.schur_flops = schur_flops;
    res.schur_time = schur_dev_time;
    CU(cudaEventRecord(evs1, g.st));
    CU(cudaEventSynchronize(evs1));
    float dms = 0;
    CU(cudaEventElapsedTime(&dms, evs0, evs1));
    res.device_time = dms * 1e-3;
    tm.total = wtime() - t0;
    res.t = tm;
    res.time = tm.total;
    return res.exit_code;
}

#include "lockstep_solver.cuh"

}  // namespace

// X and Z per block as given: an LP block's N blocks of order 1 become its vector of N values
// (brisk_result_X, capi.c:131-136: "n*n column-major or n for LP").
static void blocks_as_given(const HProblem &P, ResultData &res) {
    const int nbin = (int)P.in_n.size();
    if (nbin == (int)P.blk.size()) return;   // no LP block
    for (auto *V : {&res.X, &res.Z}) {
        if (V->empty()) continue;
        std::vector<std::vector<double>> out(nbin);
        for (int k = 0; k < nbin; k++) {
            const int q0 = P.in_first[k], q1 = P.in_first[k + 1];
            if (P.in_n[k] > 0) {
                out[k] = std::move((*V)[q0]);
                continue;
            }
            out[k].resize(q1 - q0);
            for (int q = q0; q < q1; q++) out[k][q - q0] = (*V)[q].empty() ? 0.0 : (*V)[q][0];
        }
        *V = std::move(out);
    }
}

static int solve_impl(const InputView &in, const Options &opt, ResultData &res, Arena *arena) {
    HProblem P;
    std::string err;
    const double t0 = wtime();
    res = ResultData();
    res.m = in.m;
    res.nblk = in.nblk;
    res.bs.assign(in.bs, in.bs + in.nblk);
    if (int rc = build_problem(in, P, err)) {
        log_printf(1, "brisk: %s\n", err.c_str());
        return rc;
    }
    if (opt.verbose > 1) log_printf(0, "   [host problem build %.3fs]\n", wtime() - t0);
    if (opt.verbose > 0) {
        int nmax = 0;
        for (auto &B : P.blk) nmax = std::max(nmax, B.n);
        log_printf(0, "BRISK-B200 %s interior-point SDP solver (Newton step on the GPU)\n", "1.7");
        log_printf(0, "problem: m = %d, %d SDP blocks (max n = %d)\n", in.m, in.nblk, nmax);
    }
    // the method (solver.c:13519-13560): the self-dual embedding with -hsd; without -hsd or
    // -nohsd the reference's rule: the embedding first when its dense work (12 sum n^3 over the
    // semidefinite blocks) is at most the Schur factor's m^3/3, or half of factor and assembly (the
    // row-product route's 2 n^3 a constraint here), or the whole is under 1e7 flops; the
    // infeasible-start method runs again from the start when the embedding stops short.  The
    // embedding takes the HKM direction (solver.c:13566).
    bool use_hsd = opt.hsd == 1;
    if (opt.hsd < 0) {
        double n3 = 0, asm_fl = 0;
        for (size_t k = 0; k < P.in_n.size(); k++)
            if (P.in_n[k] > 0) {
                const double nk = P.in_n[k];
                n3 += nk * nk * nk;
                asm_fl += 2.0 * nk * nk * nk * (double)P.blk[P.in_first[k]].con.size();
            }
        const double fac = (double)in.m * in.m * in.m / 3.0, dense = 12.0 * n3;
        use_hsd = dense <= fac || dense <= 0.5 * (fac + asm_fl) || fac + dense < 1e7;
        if (use_hsd && opt.verbose > 0)
            log_printf(0, "   self-dual embedding first (dense work %.1e, Schur factor %.1e, assembly %.1e)\n", dense, fac,
                       asm_fl);
    }
    Options sopt = opt;
    if (use_hsd) sopt.direction = 0;
    try {
        Solver S(P, sopt, arena);
        const double tsu = wtime();
        S.setup();
        const double t1 = wtime();
        if (opt.verbose > 1) log_printf(0, "   [device setup and upload %.3fs]\n", t1 - tsu);
        int rc = use_hsd ? S.run_hsd(res) : S.run(res);
        if (use_hsd && opt.hsd < 0 && res.status != 0 && res.status != 1 && res.status != 2 && res.status != 6) {
            if (opt.verbose > 0)
                log_printf(0, "   the embedding stopped short (%s): the infeasible-start method from the start\n",
                           status_string(res.status));
            const int it_hsd = res.iters;
            rc = S.run(res);
            res.iters += it_hsd;
        }
        blocks_as_given(P, res);
        res.t.setup = t1 - t0;
        res.h2d_bytes = S.upload_bytes;
        res.time = wtime() - t0;
        if (opt.verbose > 0) {
            log_printf(0, "status: %s   iterations: %d\n", status_string(res.status), res.iters);
            log_printf(0, "  Solve:             interior-point method: %s, %s direction, %d iterations\n",
                       res.embedding ? "self-dual embedding" : "infeasible start", res.direction == 1 ? "NT" : "HKM",
                       res.iters);
            log_printf(0, "  primal obj <C,X> = %.10e   dual obj b'y = %.10e\n", res.pobj, res.dobj);
            log_printf(0, "  DIMACS errors: %.1e %.1e %.1e %.1e %.1e %.1e\n", res.err[1], res.err[2], res.err[3],
                       res.err[4], res.err[5], res.err[6]);
            log_printf(0, "time: total %.3fs | schur %.3f  chol/solve %.3f  dense %.3f  step %.3f  setup %.3f\n",
                       res.t.total, res.t.schur, res.t.chol, res.t.dense, res.t.step, res.t.setup);
        }
        return rc;
    } catch (const GpuFail &f) {
        if (arena && f.rc == BGPU_ERR_NOMEM) {   // the batch worker grows its arena and retries
            res.status = 4;
            res.exit_code = BGPU_ERR_NOMEM;
            return BGPU_ERR_NOMEM;
        }
        log_printf(1, "brisk: GPU failure (code %d at solver.cu:%d%s%s)\n", f.rc, f.line,
                   f.ce != cudaSuccess ? ": " : "", f.ce != cudaSuccess ? cudaGetErrorString(f.ce) : "");
        res.status = 4;
        res.exit_code = -3;
        return -3;
    }
}

int solve_problem(const InputView &in, const Options &opt, ResultData &res) { return solve_impl(in, opt, res, nullptr); }

int solve_problem_arena(const InputView &in, const Options &opt, ResultData &res, Arena *arena) {
    tl_serial = true;
    const int rc = solve_impl(in, opt, res, arena);
    tl_serial = false;
    return rc;
}

// The lockstep form of the batch when every problem has one SDP block of order <= 64: the problems
// are built on the host threads (build_packed) and solved together (Lockstep).
struct BatchSession {
    std::vector<HProblem> good;
    std::vector<int> idx;        // problem number of each good problem
    std::vector<int> bad;        // problems rejected on input (exit code 2)
    int count = 0;
    Options opt;
    Lockstep *L = nullptr;
    double t_build = 0, t_setup = 0;
    ~BatchSession() { delete L; }
};

// Builds the session; returns nullptr when a problem does not have that shape (rc = 0: nothing
// reported), or on a GPU failure (rc < 0).
BatchSession *batch_session_create(int count, const std::function<bool(int, InputData &)> &get,
                                   const std::function<bool(int, InputView &)> &view, const Options &opt, int &rc) {
    rc = 0;
    const double t0 = wtime();
    std::vector<HProblem> Ps(count);
    std::vector<int> bad(count, 0);
    std::vector<char> shape_ok(count, 1);
    parallel_for(count, [&](long long pp) {
        const int p = (int)pp;
        tl_serial = true;
        std::string err;
        InputData inD;
        InputView in;
        if (view) {
            if (!view(p, in)) { bad[p] = 1; return; }
        } else {
            if (!get(p, inD)) { bad[p] = 1; return; }
            in.m = inD.m;
            in.nblk = inD.nblk;
            in.bs = inD.bs.data();
            in.c = inD.c.data();
            in.nnz = (long long)inD.v.size();
            in.mat = inD.mat.data();
            in.blk = inD.blk.data();
            in.i = inD.i.data();
            in.j = inD.j.data();
            in.v = inD.v.data();
        }
        if (in.nblk != 1 || !in.bs || in.bs[0] < 1 || in.bs[0] > lockstep::NMAX || in.m < 1) {
            shape_ok[p] = 0;
            return;
        }
        if (build_packed(in, Ps[p], err)) bad[p] = 1;
    });
    for (int p = 0; p < count; p++)
        if (!shape_ok[p]) return nullptr;
    BatchSession *S = new BatchSession;
    S->count = count;
    S->opt = opt;
    S->opt.verbose = 0;
    for (int p = 0; p < count; p++) {
        if (bad[p]) S->bad.push_back(p);
        else { S->idx.push_back(p); S->good.push_back(std::move(Ps[p])); }
    }
    Ps.clear();
    S->t_build = wtime() - t0;
    if (!S->good.empty()) {
        try {
            S->L = new Lockstep(S->good, S->opt);
            S->L->setup();
        } catch (const GpuFail &f) {
            log_printf(1, "brisk: GPU failure in the lockstep batch set-up (code %d at line %d)\n", f.rc, f.line);
            delete S;
            rc = -3;
            return nullptr;
        }
    }
    S->t_setup = wtime() - t0 - S->t_build;
    return S;
}

// Solves the session's problems; put(p, res, rc) receives each.  Returns 0 or -3.
int batch_session_solve(BatchSession *S, const std::function<void(int, ResultData &, int)> &put, int verbose) {
    std::vector<ResultData> res;
    int code = 0;
    if (S->L) {
        try {
            S->L->run(res);
            if (verbose > 2)   // -vv: the phases of the batch (on the error channel: the batch runs quiet)
                log_printf(1, "lockstep batch of %d: host build %.3fs, device setup %.3fs (allocations %.3fs, upload of "
                           "the packed rows %.3fs), start %.3fs, assembly %.3fs, factor %.3fs, PCG %.3fs, rest of the loop "
                           "%.3fs, final %.3fs\n", (int)S->good.size(), S->t_build, S->t_setup, S->L->t_alloc,
                           S->L->t_upload, S->L->t_start, S->L->t_asm, S->L->t_fac, S->L->t_pcg, S->L->t_loop,
                           S->L->t_final);
        } catch (const GpuFail &f) {
            log_printf(1, "brisk: GPU failure in the lockstep batch (code %d at line %d)\n", f.rc, f.line);
            code = -3;
        }
    }
    for (size_t q = 0; q < S->idx.size(); q++) {
        ResultData r = code ? ResultData() : std::move(res[q]);
        if (code) { r.status = 4; r.exit_code = code; }
        put(S->idx[q], r, code ? code : r.exit_code);
    }
    for (int p : S->bad) {
        ResultData r;
        r.exit_code = 2;
        put(p, r, 2);
    }
    return code;
}

void batch_session_destroy(BatchSession *S) { delete S; }

static bool lockstep_batch(int count, const std::function<bool(int, InputData &)> &get,
                           const std::function<bool(int, InputView &)> &view,
                           const std::function<void(int, ResultData &, int)> &put, const Options &opt) {
    int rc = 0;
    BatchSession *S = batch_session_create(count, get, view, opt, rc);
    if (!S) {
        if (rc == 0) return false;   // not the lockstep shape: the concurrent form runs
        for (int p = 0; p < count; p++) {
            ResultData r;
            r.status = 4;
            r.exit_code = rc;
            put(p, r, rc);
        }
        return true;
    }
    batch_session_solve(S, put, opt.verbose);
    batch_session_destroy(S);
    return true;
}

int solve_batch(int count, const std::vector<double> &work, const std::function<bool(int, InputData &)> &get,
                const std::function<void(int, ResultData &, int)> &put, const Options &opt, int workers,
                std::string &err, const std::function<bool(int, InputView &)> &view) {
    if (count <= 0) return 0;
    if (workers <= 0) workers = (int)std::max(2u, std::thread::hardware_concurrency());
    workers = std::min(workers, count);
    if (opt.batch_mode != 0 && lockstep_batch(count, get, view, put, opt)) return 0;
    std::vector<int> order(count);
    std::iota(order.begin(), order.end(), 0);
    if ((int)work.size() == count)
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work[a] > work[b]; });
    std::atomic<int> next{0};
    Options o = opt;
    o.verbose = 0;
    auto body = [&]() {
        cudaStream_t st = nullptr;
        Arena a;
        const bool ok = cudaSetDevice(o.device) == cudaSuccess &&
                        cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess;
        a.st = st;
        if (ok && cudaMallocHost((void **)&a.hbase, (size_t)1 << 20) == cudaSuccess) a.hcap = (size_t)1 << 20;
        else a.hbase = nullptr;
        for (;;) {
            const int q = next.fetch_add(1);
            if (q >= count) break;
            const int p = order[q];
            InputData held;   // (only when the caller gives no views)
            InputView in;
            ResultData r;
            int rc = -3;
            try {
                if (!ok) {
                    r.status = 4;
                } else if (view ? !view(p, in) : !get(p, held)) {
                    rc = 2;
                } else {
                    if (!view) in = view_of(held);
                    for (int grow = 0; grow < 8; grow++) {
                        rc = solve_problem_arena(in, o, r, &a);
                        if (rc != BGPU_ERR_NOMEM) break;
                        // The arena grows to the instance's need (with headroom); instances run
                        // largest first, so this happens a few times per worker at most.
                        const size_t want = std::max(std::max(a.cap * 2, a.need + a.need / 4), (size_t)64 << 20);
                        cudaStreamSynchronize(st);
                        if (a.base) cudaFree(a.base);
                        a.base = nullptr;
                        a.cap = a.need = 0;
                        if (cudaMalloc(&a.base, want) != cudaSuccess) {
                            a.base = nullptr;
                            rc = -3;
                            r.status = 4;
                            break;
                        }
                        a.cap = want;
                    }
                    if (rc == BGPU_ERR_NOMEM) rc = -3;
                }
            } catch (...) {
                rc = -3;
                r.status = 4;
            }
            r.exit_code = rc;
            put(p, r, rc);
        }
        if (st) cudaStreamSynchronize(st);
        if (a.base) cudaFree(a.base);
        if (a.hbase) cudaFreeHost(a.hbase);
        if (st) cudaStreamDestroy(st);
    };
    (void)err;
    std::vector<std::thread> th;
    for (int w = 0; w < workers; w++) th.emplace_back(body);
    for (auto &t : th) t.join();
    return 0;
}

}  // namespace bsolve

namespace bsolve {

struct Session {
    HProblem P;
    Solver *S = nullptr;
    int m = 0, nblk = 0;
    std::vector<int> bs;
    ~Session() { delete S; }
};

Session *session_create(const InputView &in, const Options &opt, std::string &err, int &rc) {
    Session *s = new Session;
    s->m = in.m;
    s->nblk = in.nblk;
    s->bs.assign(in.bs, in.bs + in.nblk);
    rc = build_problem(in, s->P, err);
    if (rc) { delete s; return nullptr; }
    try {
        s->S = new Solver(s->P, opt);
        s->S->setup();
    } catch (const GpuFail &f) {
        err = "GPU failure during setup (code " + std::to_string(f.rc) + ")";
        rc = -3;
        delete s;
        return nullptr;
    }
    return s;
}

int session_solve(Session *s, const Options &opt, ResultData &res) {
    res = ResultData();
    res.m = s->m;
    res.nblk = s->nblk;
    res.bs = s->bs;
    s->S->set_options(opt);
    try {
        const int rc = opt.hsd == 1 ? s->S->run_hsd(res) : s->S->run(res);   // (-hsd only: no automatic rule here)
        blocks_as_given(s->P, res);
        return rc;
    } catch (const GpuFail &f) {
        log_printf(1, "brisk: GPU failure (code %d at solver.cu:%d)\n", f.rc, f.line);
        res.status = 4;
        res.exit_code = -3;
        return -3;
    }
}

void session_destroy(Session *s) { delete s; }

}  // namespace bsolve
