// Supernodal sparse Cholesky of the Schur complement: symbolic analysis on the host, multifrontal
// numeric factorization and the triangular solves on the device (sparse.h).
//
// Symbolic phase (the reference's sparse_build + schol analysis, solver.c:4014, sparsechol.c):
// the pattern of M is the union of the blocks' constraint cliques.  A minimum-degree ordering
// runs on the quotient graph whose initial elements are those cliques: eliminating a
// (super)variable p forms the element union(E(p)) \ p, which is exactly the structure of L's
// column(s) for p; absorbed elements are dropped and variables with the same element set are
// merged into supervariables (they form the supernodes).  Degrees are exact external degrees.
// The supernodes are then put in postorder, single-child chains with nested structure are
// merged, and each front gets its rows, its children's relative indices and its storage.
//
// Numeric phase (multifrontal): the front of supernode s is F = [D M D + reg I on s's columns
// and rows] + the extend-add of its children's update matrices; its first ns columns are
// factored (the L panel) and the trailing rs x rs block becomes s's update matrix.  One CTA per
// front, the fronts of one tree level per launch, children added in a fixed order: the same
// bits on every run.
#include "common.cuh"
#include "sparse.h"

#include <algorithm>
#include <map>
#include <numeric>
#include <set>

namespace schol {

double g_mmd_delta = 1.0;

int analyze(int m, const std::vector<std::vector<int>> &cliques, Analysis &A) {
    A = Analysis();
    A.m = m;
    if (m <= 0) return m == 0 ? 0 : 1;
    // ---- quotient graph ----
    std::vector<std::vector<int>> E(m);   // elements of each variable
    std::vector<std::vector<int>> L;      // variables of each element
    std::vector<char> alive;
    long long pat = 0;
    {
        std::vector<int> mark(m, -1);
        for (size_t c = 0; c < cliques.size(); c++) {
            std::vector<int> v;
            for (int x : cliques[c]) {
                if (x < 0 || x >= m) return 1;
                if (mark[x] != (int)c) { mark[x] = (int)c; v.push_back(x); }
            }
            if (v.size() < 2) continue;
            std::sort(v.begin(), v.end());
            const int e = (int)L.size();
            for (int x : v) E[x].push_back(e);
            L.push_back(std::move(v));
            alive.push_back(1);
        }
    }
    std::vector<long long> w(m, 1);           // supervariable weight; 0: merged away or eliminated
    std::vector<std::vector<int>> mem(m);     // the constraints of each supervariable
    for (int v = 0; v < m; v++) mem[v].push_back(v);
    std::vector<char> done(m, 0);
    {   // initial supervariables: identical element sets
        std::map<std::vector<int>, int> first;
        for (int v = 0; v < m; v++) {
            if (E[v].empty()) continue;
            auto it = first.find(E[v]);
            if (it == first.end()) { first.emplace(E[v], v); continue; }
            const int f = it->second;
            w[f] += 1;
            mem[f].push_back(v);
            w[v] = 0;
            done[v] = 1;
        }
        for (auto &l : L) {
            size_t k = 0;
            for (int u : l) if (w[u] > 0) l[k++] = u;
            l.resize(k);
        }
    }
    std::vector<int> stamp(m, 0), estamp;
    int cur = 0;
    std::vector<long long> deg(m, 0);
    auto degree = [&](int u) {
        ++cur;
        stamp[u] = cur;
        long long s = 0;
        for (int e : E[u]) {
            if (!alive[e]) continue;
            auto &l = L[e];
            size_t k = 0;
            for (int x : l) {
                if (w[x] <= 0) continue;
                l[k++] = x;
                if (stamp[x] != cur) { stamp[x] = cur; s += w[x]; }
            }
            l.resize(k);
        }
        return s;
    };
    std::set<std::pair<long long, int>> pq;
    for (int v = 0; v < m; v++)
        if (w[v] > 0) { deg[v] = degree(v); pq.insert({deg[v], v}); }
    estamp.assign(L.size(), 0);
    std::vector<std::vector<int>> sup_cols, sup_off;   // constraint ids
    // Multiple elimination (rounds): every supervariable whose degree is within
    // dmin (1 + g_mmd_delta) and that is not adjacent to one already eliminated in the round goes
    // in the round; degrees are updated once per round.  Independent eliminations give a bushy
    // supernode tree (on a chain of cliques, alternate groups at each round: a tree of
    // logarithmic height, so the fronts of a level fill the GPU).
    std::vector<int> touched(m, 0), upd;
    int round = 0;
    while (!pq.empty()) {
        ++round;
        const long long dmin = pq.begin()->first;
        const long long dlim = dmin + (long long)(g_mmd_delta * (double)dmin);
        std::vector<int> cand;
        for (auto it = pq.begin(); it != pq.end() && it->first <= dlim; ++it) cand.push_back(it->second);
        upd.clear();
        for (const int p : cand) {
            if (w[p] <= 0 || touched[p] == round) continue;
            pq.erase({deg[p], p});
            ++cur;
            stamp[p] = cur;
            const int mk = cur;
            std::vector<int> Ln;
            for (int e : E[p]) {
                if (!alive[e]) continue;
                for (int u : L[e])
                    if (w[u] > 0 && stamp[u] != mk) { stamp[u] = mk; Ln.push_back(u); }
                alive[e] = 0;
            }
            std::sort(Ln.begin(), Ln.end());
            sup_cols.push_back(mem[p]);
            std::vector<int> off;
            for (int u : Ln) off.insert(off.end(), mem[u].begin(), mem[u].end());
            sup_off.push_back(std::move(off));
            w[p] = 0;
            done[p] = 1;
            E[p].clear();
            if (Ln.empty()) continue;
            const int en = (int)L.size();
            L.push_back(Ln);
            alive.push_back(1);
            estamp.push_back(0);
            // element lists of the new element's variables: the dead ones out, the new one in; an
            // element whose live variables all lie in the new one is absorbed
            for (int u : Ln) {
                auto &eu = E[u];
                size_t k = 0;
                for (int e : eu) if (alive[e]) eu[k++] = e;
                eu.resize(k);
            }
            for (int u : Ln)
                for (int e : E[u]) {
                    if (estamp[e] == mk) continue;
                    estamp[e] = mk;
                    bool sub = true;
                    for (int x : L[e])
                        if (w[x] > 0 && stamp[x] != mk) { sub = false; break; }
                    if (sub) alive[e] = 0;
                }
            for (int u : Ln) {
                auto &eu = E[u];
                size_t k = 0;
                for (int e : eu) if (alive[e]) eu[k++] = e;
                eu.resize(k);
                eu.push_back(en);
                touched[u] = round;
            }
            // indistinguishable variables of the new element merge
            {
                std::map<std::vector<int>, int> first;
                for (int u : Ln) {
                    std::vector<int> key = E[u];
                    std::sort(key.begin(), key.end());
                    auto it = first.find(key);
                    if (it == first.end()) { first.emplace(std::move(key), u); continue; }
                    const int f = it->second;
                    pq.erase({deg[u], u});
                    w[f] += w[u];
                    mem[f].insert(mem[f].end(), mem[u].begin(), mem[u].end());
                    w[u] = 0;
                    done[u] = 1;
                    E[u].clear();
                }
            }
            upd.insert(upd.end(), Ln.begin(), Ln.end());
        }
        std::sort(upd.begin(), upd.end());
        upd.erase(std::unique(upd.begin(), upd.end()), upd.end());
        for (int u : upd) {
            if (w[u] <= 0) continue;
            pq.erase({deg[u], u});
            deg[u] = degree(u);
            pq.insert({deg[u], u});
        }
    }
    // variables in no clique of size >= 2 (isolated): their own supernodes
    for (int v = 0; v < m; v++)
        if (!done[v] && w[v] > 0) { sup_cols.push_back(mem[v]); sup_off.push_back({}); }
    // ---- elimination positions and the supernode tree ----
    const int ns0 = (int)sup_cols.size();
    std::vector<int> pos_of(m, -1), sup_of_pos;
    {
        int k = 0;
        for (int s = 0; s < ns0; s++)
            for (int c : sup_cols[s]) { pos_of[c] = k++; sup_of_pos.push_back(s); }
        if (k != m) return 1;
    }
    std::vector<int> par(ns0, -1);
    for (int s = 0; s < ns0; s++) {
        int mn = m;
        for (int c : sup_off[s]) mn = std::min(mn, pos_of[c]);
        if (mn < m) par[s] = sup_of_pos[mn];
    }
    // postorder (children before parents; children in elimination order)
    std::vector<std::vector<int>> kids(ns0);
    std::vector<int> roots;
    for (int s = 0; s < ns0; s++) (par[s] < 0 ? roots : kids[par[s]]).push_back(s);
    std::vector<int> post;
    post.reserve(ns0);
    {
        std::vector<std::pair<int, size_t>> stk;
        for (int r : roots) {
            stk.push_back({r, 0});
            while (!stk.empty()) {
                auto &top = stk.back();
                if (top.second < kids[top.first].size()) {
                    const int c = kids[top.first][top.second++];
                    stk.push_back({c, 0});
                } else {
                    post.push_back(top.first);
                    stk.pop_back();
                }
            }
        }
    }
    if ((int)post.size() != ns0) return 1;
    // merge a single child into its parent when the child's off-diagonal rows are exactly the
    // parent's columns and rows (no extra entries)
    std::vector<int> grp(ns0);
    std::iota(grp.begin(), grp.end(), 0);
    std::vector<int> head(ns0);   // the group's top supernode (whose off rows the group keeps)
    std::iota(head.begin(), head.end(), 0);
    std::vector<std::vector<int>> gcols(ns0);
    for (int s = 0; s < ns0; s++) gcols[s] = sup_cols[s];
    std::vector<char> merged(ns0, 0);
    for (int s : post) {
        const int t = par[s];
        if (t < 0 || kids[t].size() != 1) continue;
        // rows_off(s) == cols(t) + rows_off(t) as sets
        if (sup_off[s].size() != sup_cols[t].size() + sup_off[t].size()) continue;
        std::vector<int> a = sup_off[s], b = sup_cols[t];
        b.insert(b.end(), sup_off[t].begin(), sup_off[t].end());
        std::sort(a.begin(), a.end());
        std::sort(b.begin(), b.end());
        if (a != b) continue;
        // s's group joins t: s's columns (and those merged into s) come first
        std::vector<int> nc = gcols[s];
        nc.insert(nc.end(), gcols[t].begin(), gcols[t].end());
        gcols[t] = std::move(nc);
        gcols[s].clear();
        merged[s] = 1;
    }
    // final supernodes in postorder of the survivors
    std::vector<int> newid(ns0, -1);
    int nsup = 0;
    for (int s : post)
        if (!merged[s]) newid[s] = nsup++;
    A.nsup = nsup;
    A.perm.assign(m, -1);
    A.iperm.assign(m, -1);
    A.sfirst.assign(nsup + 1, 0);
    std::vector<int> oldof(nsup);
    {
        int k = 0, id = 0;
        for (int s : post) {
            if (merged[s]) continue;
            oldof[id] = s;
            A.sfirst[id] = k;
            for (int c : gcols[s]) { A.perm[k] = c; A.iperm[c] = k; k++; }
            id++;
        }
        A.sfirst[nsup] = k;
        if (k != m) return 1;
    }
    // rows, parents, children, levels
    A.rptr.assign(nsup + 1, 0);
    A.parent.assign(nsup, -1);
    std::vector<std::vector<int>> srows(nsup);
    for (int s = 0; s < nsup; s++) {
        const int o = oldof[s];
        auto &r = srows[s];
        for (int k = A.sfirst[s]; k < A.sfirst[s + 1]; k++) r.push_back(k);
        std::vector<int> off;
        for (int c : sup_off[o]) off.push_back(A.iperm[c]);
        std::sort(off.begin(), off.end());
        if (!off.empty() && off.front() < A.sfirst[s + 1]) return 1;   // structure check
        r.insert(r.end(), off.begin(), off.end());
        A.rptr[s + 1] = A.rptr[s] + (long long)r.size();
    }
    std::vector<int> sup_at(m);
    for (int s = 0; s < nsup; s++)
        for (int k = A.sfirst[s]; k < A.sfirst[s + 1]; k++) sup_at[k] = s;
    for (int s = 0; s < nsup; s++) {
        const int nsc = A.sfirst[s + 1] - A.sfirst[s];
        if ((int)srows[s].size() > nsc) A.parent[s] = sup_at[srows[s][nsc]];
    }
    A.rows.reserve(A.rptr[nsup]);
    for (int s = 0; s < nsup; s++) A.rows.insert(A.rows.end(), srows[s].begin(), srows[s].end());
    A.cptr.assign(nsup + 1, 0);
    for (int s = 0; s < nsup; s++)
        if (A.parent[s] >= 0) A.cptr[A.parent[s] + 1]++;
    for (int s = 0; s < nsup; s++) A.cptr[s + 1] += A.cptr[s];
    A.child.assign(A.cptr[nsup], 0);
    {
        std::vector<int> fill(A.cptr.begin(), A.cptr.end() - 1);
        for (int s = 0; s < nsup; s++)
            if (A.parent[s] >= 0) A.child[fill[A.parent[s]]++] = s;
    }
    // relative indices of each child's off-diagonal rows in its parent's rows
    A.relptr.assign(nsup + 1, 0);
    for (int s = 0; s < nsup; s++) {
        const int nsc = A.sfirst[s + 1] - A.sfirst[s];
        const long long rs = (long long)srows[s].size() - nsc;
        A.relptr[s + 1] = A.relptr[s] + (A.parent[s] >= 0 ? rs : 0);
    }
    A.rel.assign(A.relptr[nsup], 0);
    for (int s = 0; s < nsup; s++) {
        const int t = A.parent[s];
        if (t < 0) continue;
        const int nsc = A.sfirst[s + 1] - A.sfirst[s];
        const auto &pr = srows[t];
        long long q = A.relptr[s];
        for (size_t i = nsc; i < srows[s].size(); i++) {
            auto it = std::lower_bound(pr.begin(), pr.end(), srows[s][i]);
            if (it == pr.end() || *it != srows[s][i]) return 1;   // the structure must nest
            A.rel[q++] = (int)(it - pr.begin());
        }
    }
    std::vector<int> lev(nsup, 0);
    int nlev = 0;
    for (int s = 0; s < nsup; s++) {   // children come first in postorder
        for (int c = A.cptr[s]; c < A.cptr[s + 1]; c++) lev[s] = std::max(lev[s], lev[A.child[c]] + 1);
        nlev = std::max(nlev, lev[s] + 1);
    }
    A.lvptr.assign(nlev + 1, 0);
    for (int s = 0; s < nsup; s++) A.lvptr[lev[s] + 1]++;
    for (int l = 0; l < nlev; l++) A.lvptr[l + 1] += A.lvptr[l];
    A.lvsup.assign(nsup, 0);
    {
        std::vector<int> fill(A.lvptr.begin(), A.lvptr.end() - 1);
        for (int s = 0; s < nsup; s++) A.lvsup[fill[lev[s]]++] = s;
    }
    // storage and counts
    A.lptr.assign(nsup + 1, 0);
    A.uptr.assign(nsup + 1, 0);
    for (int s = 0; s < nsup; s++) {
        const double nsc = A.sfirst[s + 1] - A.sfirst[s];
        const double f = (double)(A.rptr[s + 1] - A.rptr[s]);
        const double rs = f - nsc;
        A.lptr[s + 1] = A.lptr[s] + (long long)(f * nsc);
        A.uptr[s + 1] = A.uptr[s] + (long long)(rs * rs);
        A.flops += nsc * nsc * nsc / 3.0 + nsc * nsc * rs + nsc * rs * rs;
        A.nnz += f * nsc - nsc * (nsc - 1) / 2.0;
        A.fmax = std::max(A.fmax, (int)f);
    }
    // the pattern of M below the diagonal (pairs sharing a clique)
    {
        std::vector<int> mark(m, -1);
        std::vector<std::vector<int>> cl_of(m);
        for (size_t c = 0; c < cliques.size(); c++)
            for (int x : cliques[c]) cl_of[x].push_back((int)c);
        for (int v = 0; v < m; v++) {
            for (int c : cl_of[v])
                for (int x : cliques[c])
                    if (x > v && mark[x] != v) { mark[x] = v; pat++; }
        }
    }
    A.pattern = pat;
    return 0;
}

}  // namespace schol

// ---- numeric phase -----------------------------------------------------------------------
#include "kernels.h"

namespace schol {
namespace {
constexpr int FT = 256;        // threads per front
constexpr int FS_MAX = 160;    // fronts up to this order are factored in shared memory

__global__ void sp_init_kernel(int *info, double *pmin) {
    *info = 0;
    *pmin = 1.0;
}

// The front of supernode s (order f, ns own columns, rs = f - ns): element (i, j), i >= j, lives
// in the panel P (f x ns, ld f) when j < ns, else in the update matrix Us (rs x rs, ld rs).  In
// shared memory (SMEM) the whole lower front is held as F (ld = f | 1) and written back at the end.
template <typename T>
struct FrontRef {
    T *P, *Us, *F;
    int f, ns, rs, ldf;
    bool smem;
    __device__ __forceinline__ T &at(int i, int j) const {
        if (smem) return F[i + j * ldf];
        return j < ns ? P[i + (long long)j * f] : Us[(i - ns) + (long long)(j - ns) * rs];
    }
};

// T: the type of the front, the panel and the update matrices (double; float for the early
// iterations of the mixed path, whose PCG refines against the FP64 M).
template <bool SMEM, typename T>
__global__ void __launch_bounds__(FT) front_kernel(const int *__restrict__ sups, const int *__restrict__ fsz,
                                                   const int *__restrict__ nsz, const long long *__restrict__ rptr,
                                                   const int *__restrict__ rows, const int *__restrict__ perm,
                                                   const long long *__restrict__ lptr, const long long *__restrict__ uptr,
                                                   const int *__restrict__ cptr, const int *__restrict__ child,
                                                   const long long *__restrict__ relptr, const int *__restrict__ rel,
                                                   const double *__restrict__ M, long long ldm,
                                                   const double *__restrict__ D, double reg, T *L, T *U,
                                                   int *info, double *pmin) {
    extern __shared__ __align__(16) unsigned char fs_raw[];
    const int s = sups[blockIdx.x];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    if (*(volatile int *)info != 0) return;   // an earlier level failed
    FrontRef<T> F;
    F.f = fsz[s];
    F.ns = nsz[s];
    F.rs = F.f - F.ns;
    F.ldf = F.f | 1;
    F.P = L + lptr[s];
    F.Us = U + uptr[s];
    F.F = reinterpret_cast<T *>(fs_raw);
    F.smem = SMEM;
    const int f = F.f, ns = F.ns;
    const int *rw = rows + rptr[s];
    // 1. D M D + reg I on the own columns, zero elsewhere
    for (int j = ty; j < f; j += 16) {
        const int cj = perm[rw[j]];
        const double dj = D[cj];
        for (int i = j + tx; i < f; i += 16) {
            double v = 0.0;
            if (j < ns) {
                const int ci = perm[rw[i]];
                v = D[ci] * M[ci + (long long)cj * ldm] * dj;
                if (i == j) v += reg;
            }
            F.at(i, j) = (T)v;
        }
    }
    __syncthreads();
    // 2. extend-add of the children's update matrices, one child at a time
    for (int c = cptr[s]; c < cptr[s + 1]; c++) {
        const int k = child[c];
        const int rc = fsz[k] - nsz[k];
        const int *rl = rel + relptr[k];
        const T *Uc = U + uptr[k];
        for (int b = ty; b < rc; b += 16) {
            const int jb = rl[b];
            for (int a = b + tx; a < rc; a += 16) F.at(rl[a], jb) += Uc[a + (long long)b * rc];
        }
        __syncthreads();
    }
    // 3. partial Cholesky of the first ns columns (one barrier a column; column k-1 is scaled
    //    while column k updates the trailing front with its unscaled values / d)
    double pm = 1e300;
    int fail = 0;
    T prev_piv = 0, prev_inv = 0;
    for (int k = 0; k < ns; k++) {
        const T d = F.at(k, k);
        if (!(d > (T)0) || !isfinite((double)d)) { fail = rw[k] + 1; break; }
        pm = fmin(pm, (double)d);
        const T inv_d = (T)1 / d;
        if (k > 0)
            for (int r = k - 1 + tid; r < f; r += FT) F.at(r, k - 1) = (r == k - 1) ? prev_piv : F.at(r, k - 1) * prev_inv;
        for (int q = k + 1 + tx; q < f; q += 16) {
            const T sqc = F.at(q, k) * inv_d;
            for (int r = q + ty; r < f; r += 16) F.at(r, q) -= F.at(r, k) * sqc;
        }
        prev_piv = sqrt(d);
        prev_inv = (T)1 / prev_piv;
        __syncthreads();
    }
    if (!fail && ns > 0) {
        for (int r = ns - 1 + tid; r < f; r += FT) F.at(r, ns - 1) = (r == ns - 1) ? prev_piv : F.at(r, ns - 1) * prev_inv;
        __syncthreads();
    }
    if (fail) {
        if (tid == 0) atomicCAS(info, 0, fail);
        return;
    }
    if (tid == 0 && ns > 0) atomicMin((unsigned long long *)pmin, (unsigned long long)__double_as_longlong(pm));
    // 4. back to the panel (its strict upper part zeroed) and the update matrix
    if (SMEM) {
        for (int j = ty; j < ns; j += 16)
            for (int i = tx; i < f; i += 16) F.P[i + (long long)j * f] = i >= j ? F.F[i + j * F.ldf] : (T)0;
        const int rs = F.rs;
        for (int j = ty; j < rs; j += 16)
            for (int i = j + tx; i < rs; i += 16) F.Us[i + (long long)j * rs] = F.F[(i + ns) + (j + ns) * F.ldf];
    } else {
        for (int j = ty; j < ns; j += 16)
            for (int i = tx; i < j; i += 16) F.P[i + (long long)j * f] = (T)0;
    }
}

// Triangular solves by tree levels, one CTA per supernode (the multifrontal solve).  Forward
// (leaves first): y_s = L_ss^-1 (b_s - the children's contributions to s's columns), and s passes
// up V_s = L_off,s y_s + the children's contributions to s's off-diagonal rows (added through the
// relative indices, children in a fixed order).  Backward (root first): x_s = L_ss^-T (y_s -
// L_off,s' x_off), x_off already final.  xe holds the permuted, scaled vector.
constexpr int ST = 256;
constexpr int SX = 512;   // own columns held in shared memory (larger supernodes use the global xe)

__global__ void perm_in_kernel(int m, const int *__restrict__ perm, const double *__restrict__ D,
                               const double *__restrict__ x, double *xe) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m) { const int c = perm[k]; xe[k] = D[c] * x[c]; }
}
__global__ void perm_out_kernel(int m, const int *__restrict__ perm, const double *__restrict__ D,
                                const double *__restrict__ xe, double *x) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m) { const int c = perm[k]; x[c] = D[c] * xe[k]; }
}

template <typename T>
__global__ void __launch_bounds__(ST) fwd_kernel(const int *__restrict__ sups, const int *__restrict__ fsz,
                                                 const int *__restrict__ nsz, const long long *__restrict__ rptr,
                                                 const int *__restrict__ rows, const long long *__restrict__ lptr,
                                                 const T *__restrict__ L, const int *__restrict__ cptr,
                                                 const int *__restrict__ child, const long long *__restrict__ relptr,
                                                 const int *__restrict__ rel, double *xe, double *V) {
    __shared__ double xs[SX];
    __shared__ double yj;
    const int s = sups[blockIdx.x], tid = threadIdx.x;
    const int f = fsz[s], ns = nsz[s], rs = f - ns;
    const int k0 = rows[rptr[s]];
    const T *P = L + lptr[s];
    double *vo = V + relptr[s];   // rs values (none at a root)
    const bool sm = ns <= SX;
    double *y = sm ? xs : xe + k0;
    if (sm) for (int j = tid; j < ns; j += ST) xs[j] = xe[k0 + j];
    for (int i = tid; i < rs; i += ST) vo[i] = 0.0;
    __syncthreads();
    for (int c = cptr[s]; c < cptr[s + 1]; c++) {
        const int k = child[c];
        const int rc = fsz[k] - nsz[k];
        const int *rl = rel + relptr[k];
        const double *vc = V + relptr[k];
        for (int i = tid; i < rc; i += ST) {
            const int r = rl[i];
            if (r < ns) y[r] -= vc[i]; else vo[r - ns] += vc[i];
        }
        __syncthreads();
    }
    for (int j = 0; j < ns; j++) {
        if (tid == 0) { yj = y[j] / (double)P[j + (long long)j * f]; y[j] = yj; }
        __syncthreads();
        const double v = yj;
        for (int i = j + 1 + tid; i < ns; i += ST) y[i] -= (double)P[i + (long long)j * f] * v;
        __syncthreads();
    }
    for (int i = tid; i < rs; i += ST) {
        double a = 0.0;
        for (int j = 0; j < ns; j++) a += (double)P[(ns + i) + (long long)j * f] * y[j];
        vo[i] += a;
    }
    if (sm) for (int j = tid; j < ns; j += ST) xe[k0 + j] = xs[j];
}

template <typename T>
__global__ void __launch_bounds__(ST) bwd_kernel(const int *__restrict__ sups, const int *__restrict__ fsz,
                                                 const int *__restrict__ nsz, const long long *__restrict__ rptr,
                                                 const int *__restrict__ rows, const long long *__restrict__ lptr,
                                                 const T *__restrict__ L, double *xe) {
    __shared__ double xs[SX];
    __shared__ double xj_s;
    const int s = sups[blockIdx.x], tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int f = fsz[s], ns = nsz[s];
    const int *rw = rows + rptr[s];
    const int k0 = rw[0];
    const T *P = L + lptr[s];
    const bool sm = ns <= SX;
    double *x = sm ? xs : xe + k0;
    // x_s = y_s - L_off,s' x_off: a warp per column
    for (int j = warp; j < ns; j += ST / 32) {
        double a = 0.0;
        for (int i = ns + lane; i < f; i += 32) a += (double)P[i + (long long)j * f] * xe[rw[i]];
        a = warp_sum(a);
        if (lane == 0) x[j] = xe[k0 + j] - a;
    }
    __syncthreads();
    for (int j = ns - 1; j >= 0; j--) {
        if (tid == 0) { xj_s = x[j] / (double)P[j + (long long)j * f]; x[j] = xj_s; }
        __syncthreads();
        const double v = xj_s;
        for (int i = tid; i < j; i += ST) x[i] -= (double)P[j + (long long)i * f] * v;
        __syncthreads();
    }
    if (sm) for (int j = tid; j < ns; j += ST) xe[k0 + j] = xs[j];
}
}  // namespace

size_t factor_bytes(const Analysis &A) {
    const size_t n = A.nsup;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t b = 0;
    b += al(sizeof(int) * A.m);                   // perm
    b += 2 * al(sizeof(int) * n);                 // f, ns
    b += al(sizeof(int) * A.rows.size());         // rows
    b += al(sizeof(int) * (n + 1));               // cptr
    b += al(sizeof(int) * (A.child.size() + 1));  // child
    b += al(sizeof(int) * (A.rel.size() + 1));    // rel
    b += al(sizeof(int) * (n + 1));               // lvsup (sorted per level)
    b += 4 * al(sizeof(long long) * (n + 1));     // rptr, relptr, lptr, uptr
    b += al(sizeof(double) * (A.lptr.empty() ? 1 : A.lptr[n] + 1));
    b += al(sizeof(double) * (A.uptr.empty() ? 1 : A.uptr[n] + 1));
    b += al(sizeof(double) * (A.m + 1));          // xe
    b += al(sizeof(double) * (A.rel.size() + 1)); // V (the solve's passed-up vectors)
    b += al(sizeof(int)) + al(sizeof(double));    // info, pmin
    return b + 256;
}

int factor_bind(cudaStream_t st, const Analysis &A, void *buf, Factor &F) {
    release(F);
    F = Factor();
    F.A = &A;
    const size_t n = A.nsup;
    uintptr_t p = ((uintptr_t)buf + 255) & ~(uintptr_t)255;
    auto take = [&](size_t bytes) {
        void *r = (void *)p;
        p = (p + bytes + 255) & ~(uintptr_t)255;
        return r;
    };
    F.perm = (int *)take(sizeof(int) * A.m);
    F.f = (int *)take(sizeof(int) * n);
    F.ns = (int *)take(sizeof(int) * n);
    F.rows = (int *)take(sizeof(int) * A.rows.size());
    F.cptr = (int *)take(sizeof(int) * (n + 1));
    F.child = (int *)take(sizeof(int) * (A.child.size() + 1));
    F.rel = (int *)take(sizeof(int) * (A.rel.size() + 1));
    F.lvsup = (int *)take(sizeof(int) * (n + 1));
    F.rptr = (long long *)take(sizeof(long long) * (n + 1));
    F.relptr = (long long *)take(sizeof(long long) * (n + 1));
    F.lptr = (long long *)take(sizeof(long long) * (n + 1));
    F.uptr = (long long *)take(sizeof(long long) * (n + 1));
    F.L = (double *)take(sizeof(double) * (A.lptr[n] + 1));
    F.U = (double *)take(sizeof(double) * (A.uptr[n] + 1));
    F.x = (double *)take(sizeof(double) * (A.m + 1));
    F.V = (double *)take(sizeof(double) * (A.rel.size() + 1));
    F.info = (int *)take(sizeof(int));
    F.pmin = (double *)take(sizeof(double));
    F.bytes = factor_bytes(A);
    std::vector<int> fs(n), nss(n);
    for (size_t s = 0; s < n; s++) {
        fs[s] = (int)(A.rptr[s + 1] - A.rptr[s]);
        nss[s] = A.sfirst[s + 1] - A.sfirst[s];
    }
    // within each level the fronts that fit shared memory come first
    F.lvs.assign(A.lvsup.begin(), A.lvsup.end());
    F.lvsplit.assign(A.lvptr.size() > 0 ? A.lvptr.size() - 1 : 0, 0);
    F.lvsmem.assign(F.lvsplit.size(), 0);
    for (size_t l = 0; l + 1 < A.lvptr.size(); l++) {
        auto b = F.lvs.begin() + A.lvptr[l], e = F.lvs.begin() + A.lvptr[l + 1];
        std::stable_sort(b, e, [&](int x, int y) { return (fs[x] <= FS_MAX) > (fs[y] <= FS_MAX); });
        int cnt = 0, fm = 0;
        for (auto it = b; it != e; ++it)
            if (fs[*it] <= FS_MAX) { cnt++; fm = std::max(fm, fs[*it]); }
        F.lvsplit[l] = cnt;
        F.lvsmem[l] = fm;
    }
    F.fs = fs;
    F.nss = nss;
    auto up = [&](void *d, const void *h, size_t bytes) {
        return bytes ? cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st) : cudaSuccess;
    };
    BGPU_CHECK(up(F.perm, A.perm.data(), sizeof(int) * A.m));
    BGPU_CHECK(up(F.f, F.fs.data(), sizeof(int) * n));
    BGPU_CHECK(up(F.ns, F.nss.data(), sizeof(int) * n));
    BGPU_CHECK(up(F.rows, A.rows.data(), sizeof(int) * A.rows.size()));
    BGPU_CHECK(up(F.cptr, A.cptr.data(), sizeof(int) * (n + 1)));
    BGPU_CHECK(up(F.child, A.child.data(), sizeof(int) * A.child.size()));
    BGPU_CHECK(up(F.rel, A.rel.data(), sizeof(int) * A.rel.size()));
    BGPU_CHECK(up(F.lvsup, F.lvs.data(), sizeof(int) * n));
    BGPU_CHECK(up(F.rptr, A.rptr.data(), sizeof(long long) * (n + 1)));
    BGPU_CHECK(up(F.relptr, A.relptr.data(), sizeof(long long) * (n + 1)));
    BGPU_CHECK(up(F.lptr, A.lptr.data(), sizeof(long long) * (n + 1)));
    BGPU_CHECK(up(F.uptr, A.uptr.data(), sizeof(long long) * (n + 1)));
    return BGPU_OK;
}

namespace {
template <typename T>
int factor_t(cudaStream_t st, Factor &F, const double *M, long long ldm, const double *d_D, double reg) {
    const Analysis &A = *F.A;
    T *L = reinterpret_cast<T *>(F.L), *U = reinterpret_cast<T *>(F.U);
    sp_init_kernel<<<1, 1, 0, st>>>(F.info, F.pmin);
    BGPU_LAUNCH_CHECK();
    BGPU_ATTR_ONCE(BGPU_CHECK(cudaFuncSetAttribute(front_kernel<true, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)((FS_MAX | 1) * FS_MAX * sizeof(T)))));
    for (size_t l = 0; l + 1 < A.lvptr.size(); l++) {
        const int lo = A.lvptr[l], cnt = A.lvptr[l + 1] - lo, ns_ = F.lvsplit[l];
        if (ns_ > 0) {
            const size_t smem = (size_t)(F.lvsmem[l] | 1) * F.lvsmem[l] * sizeof(T);
            front_kernel<true, T><<<ns_, FT, smem, st>>>(F.lvsup + lo, F.f, F.ns, F.rptr, F.rows, F.perm, F.lptr,
                                                         F.uptr, F.cptr, F.child, F.relptr, F.rel, M, ldm, d_D, reg, L,
                                                         U, F.info, F.pmin);
            BGPU_LAUNCH_CHECK();
        }
        if (cnt - ns_ > 0) {
            front_kernel<false, T><<<cnt - ns_, FT, 0, st>>>(F.lvsup + lo + ns_, F.f, F.ns, F.rptr, F.rows, F.perm,
                                                             F.lptr, F.uptr, F.cptr, F.child, F.relptr, F.rel, M, ldm,
                                                             d_D, reg, L, U, F.info, F.pmin);
            BGPU_LAUNCH_CHECK();
        }
    }
    return BGPU_OK;
}

template <typename T>
int solve_t(cudaStream_t st, Factor &F, const double *d_D, double *x) {
    const Analysis &A = *F.A;
    const T *L = reinterpret_cast<const T *>(F.L);
    const int m = A.m, nlev = (int)A.lvptr.size() - 1;
    perm_in_kernel<<<ceil_div(m, 256), 256, 0, st>>>(m, F.perm, d_D, x, F.x);
    BGPU_LAUNCH_CHECK();
    for (int l = 0; l < nlev; l++) {
        const int lo = A.lvptr[l], cnt = A.lvptr[l + 1] - lo;
        fwd_kernel<T><<<cnt, ST, 0, st>>>(F.lvsup + lo, F.f, F.ns, F.rptr, F.rows, F.lptr, L, F.cptr, F.child,
                                          F.relptr, F.rel, F.x, F.V);
        BGPU_LAUNCH_CHECK();
    }
    for (int l = nlev - 1; l >= 0; l--) {
        const int lo = A.lvptr[l], cnt = A.lvptr[l + 1] - lo;
        bwd_kernel<T><<<cnt, ST, 0, st>>>(F.lvsup + lo, F.f, F.ns, F.rptr, F.rows, F.lptr, L, F.x);
        BGPU_LAUNCH_CHECK();
    }
    perm_out_kernel<<<ceil_div(m, 256), 256, 0, st>>>(m, F.perm, d_D, F.x, x);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}
}  // namespace

int factor(cudaStream_t st, Factor &F, const double *M, long long ldm, const double *d_D, double reg, bool fp32) {
    F.fp32 = fp32;
    return fp32 ? factor_t<float>(st, F, M, ldm, d_D, reg) : factor_t<double>(st, F, M, ldm, d_D, reg);
}

int solve(cudaStream_t st, Factor &F, const double *d_D, double *x) {
    auto direct = [&]() { return F.fp32 ? solve_t<float>(st, F, d_D, x) : solve_t<double>(st, F, d_D, x); };
    const int t = F.fp32 ? 1 : 0;
    if (F.solve_graph[t] && (F.graph_D[t] != d_D || F.graph_x[t] != x)) {
        cudaGraphExecDestroy(F.solve_graph[t]);
        F.solve_graph[t] = nullptr;
    }
    if (!F.solve_graph[t] && st != nullptr) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone &&
            cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            const long long before = __atomic_load_n(&g_bgpu_launches, __ATOMIC_RELAXED);
            const int rc = direct();
            cudaGraph_t graph = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(st, &graph);
            cudaGraphExec_t exec = nullptr;
            if (rc == 0 && ce == cudaSuccess && graph && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
                F.solve_graph[t] = exec;
                F.graph_D[t] = d_D;
                F.graph_x[t] = x;
                F.graph_launches = (int)(__atomic_load_n(&g_bgpu_launches, __ATOMIC_RELAXED) - before);
                __atomic_add_fetch(&g_bgpu_launches, -(long long)F.graph_launches, __ATOMIC_RELAXED);
            }
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
        }
    }
    if (F.solve_graph[t]) {
        BGPU_CHECK(cudaGraphLaunch(F.solve_graph[t], st));
        __atomic_add_fetch(&g_bgpu_launches, (long long)F.graph_launches, __ATOMIC_RELAXED);
        return BGPU_OK;
    }
    return direct();
}

void release(Factor &F) {
    for (int t = 0; t < 2; t++)
        if (F.solve_graph[t]) {
            cudaGraphExecDestroy(F.solve_graph[t]);
            F.solve_graph[t] = nullptr;
        }
}

}  // namespace schol
