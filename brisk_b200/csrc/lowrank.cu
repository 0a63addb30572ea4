// The low-rank Schur route (the reference's schur_lowrank, solver.c:1862-1934; its route choice,
// lowrank_block, problem.c:972-1075).
//
// When every constraint of a block has low rank, A_t = sum_{k in t} s_k w_k w_k' (w_k unit
// vectors), the Schur complement needs no per-constraint product:
//   M_tu = tr(A_t X A_u Zi) = sum_{k in t, l in u} s_k s_l (w_k' X w_l)(w_l' Zi w_k)
//        = sum s_k s_l P_kl Q_kl,   P = W' X W,  Q = W' Zi W   (W = [w_1 .. w_R], n x R).
// B200 form: P and Q by two DMMA GEMMs each (n x n x R, then R x n x R), then one launch that
// sums every pair of constraints' block of the Hadamard product into M.
//
// The factors are found on the host, by this file's own method (the reference uses a shared set
// of random vectors and eigendecompositions; any exact factorization gives the same M):
//   - a constraint whose support (the rows it touches) has s <= 32 rows: the s x s principal
//     matrix is diagonalised exactly by cyclic Jacobi rotations;
//   - a larger support: Y = A_t Omega with 32 Gaussian columns (fixed seed), an orthonormal Q of
//     its range by Gram-Schmidt with column pivoting, B = Q' A_t Q diagonalised by Jacobi, W = Q V;
//     accepted only if the rank is below 28 (the range was captured with margin) and A_t
//     Omega2 = W diag(s) W' Omega2 holds to 1e-12 relative on 4 further Gaussian columns.
// Eigenvalues below 1e-14 of the largest are dropped.  A block takes the route when every
// constraint factors and the route's work (P and Q: 4 n^2 R + 4 n R^2 flops) is below half of
// the row-product route's 2 n^3 per constraint (-lowrank 1 forces it, 0 turns it off).
#include "common.cuh"
#include "kernels.h"

#include <algorithm>
#include <cmath>
#include <random>
#include <thread>
#include <vector>

namespace {
constexpr int LR_SMALL = 32, LR_SKETCH = 32, LR_MAXRANK = 28, LR_CHECK = 4;

// Eigenvalues and vectors of the symmetric s x s matrix A (column-major, overwritten) by cyclic
// Jacobi rotations; V (s x s, column-major) receives the vectors, lam the values.
void jacobi_eig(int s, std::vector<double> &A, std::vector<double> &V, std::vector<double> &lam) {
    V.assign((size_t)s * s, 0.0);
    for (int i = 0; i < s; i++) V[i + (size_t)i * s] = 1.0;
    auto a = [&](int i, int j) -> double & { return A[i + (size_t)j * s]; };
    double fro = 0;
    for (double x : A) fro += x * x;
    for (int sweep = 0; sweep < 60; sweep++) {
        double off = 0;
        for (int j = 0; j < s; j++)
            for (int i = 0; i < j; i++) off += a(i, j) * a(i, j);
        if (off <= 1e-32 * fro || fro == 0) break;
        for (int p = 0; p < s - 1; p++)
            for (int q = p + 1; q < s; q++) {
                const double apq = a(p, q);
                if (apq == 0) continue;
                const double theta = (a(q, q) - a(p, p)) / (2 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
                const double c = 1 / std::sqrt(t * t + 1), sn = t * c;
                for (int k = 0; k < s; k++) {   // columns p, q
                    const double akp = a(k, p), akq = a(k, q);
                    a(k, p) = c * akp - sn * akq;
                    a(k, q) = sn * akp + c * akq;
                }
                for (int k = 0; k < s; k++) {   // rows p, q
                    const double apk = a(p, k), aqk = a(q, k);
                    a(p, k) = c * apk - sn * aqk;
                    a(q, k) = sn * apk + c * aqk;
                }
                for (int k = 0; k < s; k++) {
                    const double vkp = V[k + (size_t)p * s], vkq = V[k + (size_t)q * s];
                    V[k + (size_t)p * s] = c * vkp - sn * vkq;
                    V[k + (size_t)q * s] = sn * vkp + c * vkq;
                }
            }
    }
    lam.resize(s);
    for (int i = 0; i < s; i++) lam[i] = a(i, i);
}

struct Factor {
    std::vector<double> w;   // rank x n, each row a unit vector (dense over the block's order)
    std::vector<double> s;   // rank values
    bool ok = false;
};

// The factor of one constraint from its full-expansion entries (pos = p + q n, value).
Factor factor_one(int n, const int *pos, const double *val, long long ne, unsigned seed) {
    Factor F;
    std::vector<int> rows;
    rows.reserve(ne);
    for (long long e = 0; e < ne; e++) rows.push_back(pos[e] % n);
    std::sort(rows.begin(), rows.end());
    rows.erase(std::unique(rows.begin(), rows.end()), rows.end());
    const int s = (int)rows.size();
    if (s == 0) { F.ok = true; return F; }
    std::vector<int> loc(n, -1);
    for (int i = 0; i < s; i++) loc[rows[i]] = i;
    double amax = 0;
    for (long long e = 0; e < ne; e++) amax = std::max(amax, std::fabs(val[e]));
    std::vector<double> lam, V, Wloc;   // Wloc: s x r, column-major
    int r = 0;
    auto keep = [&](const std::vector<double> &lam_all, const std::vector<double> &Vs, int cols, const double *Q,
                    int qcols) {
        double lmax = 0;
        for (double x : lam_all) lmax = std::max(lmax, std::fabs(x));
        std::vector<int> idx;
        for (int i = 0; i < cols; i++)
            if (std::fabs(lam_all[i]) > 1e-14 * lmax) idx.push_back(i);
        r = (int)idx.size();
        Wloc.assign((size_t)s * r, 0.0);
        lam.resize(r);
        for (int c = 0; c < r; c++) {
            lam[c] = lam_all[idx[c]];
            const double *v = Vs.data() + (size_t)idx[c] * cols;
            if (!Q) {
                for (int i = 0; i < s; i++) Wloc[i + (size_t)c * s] = v[i];
            } else {
                for (int j = 0; j < qcols; j++)
                    for (int i = 0; i < s; i++) Wloc[i + (size_t)c * s] += Q[i + (size_t)j * s] * v[j];
            }
        }
    };
    if (s <= LR_SMALL) {
        std::vector<double> A((size_t)s * s, 0.0);
        for (long long e = 0; e < ne; e++) A[loc[pos[e] % n] + (size_t)loc[pos[e] / n] * s] += val[e];
        jacobi_eig(s, A, V, lam);
        std::vector<double> lam_all = lam;
        keep(lam_all, V, s, nullptr, 0);
    } else {
        // range sketch Y = A Omega (s x LR_SKETCH), then an orthonormal basis of it
        std::mt19937_64 rng(seed);
        std::normal_distribution<double> N01;
        const int kk = LR_SKETCH + LR_CHECK;
        std::vector<double> Om((size_t)s * kk);
        for (double &x : Om) x = N01(rng);
        std::vector<double> Y((size_t)s * kk, 0.0);
        for (long long e = 0; e < ne; e++) {
            const int i = loc[pos[e] % n], j = loc[pos[e] / n];
            for (int c = 0; c < kk; c++) Y[i + (size_t)c * s] += val[e] * Om[j + (size_t)c * s];
        }
        // an orthonormal basis of the sketch's range by Gram-Schmidt with column pivoting: each
        // step takes the remaining column of largest residual (a column whose residual is small
        // next to its own norm would carry cancellation into the basis), orthogonalises it once
        // more against the basis, and removes its direction from the rest
        std::vector<double> Q;   // s x q
        int q = 0;
        std::vector<double> res(Y.begin(), Y.begin() + (size_t)s * LR_SKETCH);
        std::vector<char> used(LR_SKETCH, 0);
        auto col_norm = [&](const double *y) {
            double a2 = 0;
            for (int i = 0; i < s; i++) a2 += y[i] * y[i];
            return std::sqrt(a2);
        };
        double ymax = 0;
        for (int c = 0; c < LR_SKETCH; c++) ymax = std::max(ymax, col_norm(res.data() + (size_t)c * s));
        while (q < LR_SKETCH) {
            int best = -1;
            double bn = 0;
            for (int c = 0; c < LR_SKETCH; c++) {
                if (used[c]) continue;
                const double nc = col_norm(res.data() + (size_t)c * s);
                if (nc > bn) { bn = nc; best = c; }
            }
            if (best < 0 || bn <= 1e-10 * ymax) break;   // the rest lies in the span already
            used[best] = 1;
            double *y = res.data() + (size_t)best * s;
            for (int j = 0; j < q; j++) {   // the second pass of the chosen column
                double d = 0;
                for (int i = 0; i < s; i++) d += Q[i + (size_t)j * s] * y[i];
                for (int i = 0; i < s; i++) y[i] -= d * Q[i + (size_t)j * s];
            }
            const double nrm = col_norm(y);
            if (!(nrm > 0)) break;
            Q.resize((size_t)s * (q + 1));
            for (int i = 0; i < s; i++) Q[i + (size_t)q * s] = y[i] / nrm;
            const double *qn = Q.data() + (size_t)q * s;
            for (int c = 0; c < LR_SKETCH; c++) {
                if (used[c]) continue;
                double *z = res.data() + (size_t)c * s, d = 0;
                for (int i = 0; i < s; i++) d += qn[i] * z[i];
                for (int i = 0; i < s; i++) z[i] -= d * qn[i];
            }
            q++;
        }
        if (q >= LR_MAXRANK) return F;   // not of low rank (or not captured with margin)
        // B = Q' A Q (q x q)
        std::vector<double> AQ((size_t)s * q, 0.0);
        for (long long e = 0; e < ne; e++) {
            const int i = loc[pos[e] % n], j = loc[pos[e] / n];
            for (int c = 0; c < q; c++) AQ[i + (size_t)c * s] += val[e] * Q[j + (size_t)c * s];
        }
        std::vector<double> B((size_t)q * q, 0.0);
        for (int c = 0; c < q; c++)
            for (int r2 = 0; r2 < q; r2++) {
                double d = 0;
                for (int i = 0; i < s; i++) d += Q[i + (size_t)r2 * s] * AQ[i + (size_t)c * s];
                B[r2 + (size_t)c * q] = d;
            }
        for (int c = 0; c < q; c++)   // symmetric to rounding: take its symmetric part
            for (int r2 = 0; r2 < c; r2++) B[r2 + (size_t)c * q] = B[c + (size_t)r2 * q] = 0.5 * (B[r2 + (size_t)c * q] + B[c + (size_t)r2 * q]);
        jacobi_eig(q, B, V, lam);
        std::vector<double> lam_all = lam;
        keep(lam_all, V, q, Q.data(), q);
        // the check: A Omega2 against W diag(lam) W' Omega2 on the LR_CHECK further columns
        double err = 0, ref = 0;
        for (int c = LR_SKETCH; c < kk; c++) {
            const double *om = Om.data() + (size_t)c * s;
            std::vector<double> z(s, 0.0);
            for (int k = 0; k < r; k++) {
                double d = 0;
                for (int i = 0; i < s; i++) d += Wloc[i + (size_t)k * s] * om[i];
                d *= lam[k];
                for (int i = 0; i < s; i++) z[i] += d * Wloc[i + (size_t)k * s];
            }
            for (int i = 0; i < s; i++) {
                const double y = Y[i + (size_t)c * s];
                err += (y - z[i]) * (y - z[i]);
                ref += y * y;
            }
        }
        if (!(err <= 1e-24 * std::max(ref, 1e-300))) return F;
    }
    (void)amax;
    F.w.assign((size_t)r * n, 0.0);
    F.s = lam;
    for (int k = 0; k < r; k++)
        for (int i = 0; i < s; i++) F.w[(size_t)k * n + rows[i]] = Wloc[i + (size_t)k * s];
    F.ok = true;
    return F;
}

// M[con[u], con[t]] += sum_{k in t, l in u} s_k s_l P_lk Q_lk for every pair u >= t of the
// block's constraints (and the mirror entry): one thread per pair, the terms in a fixed order.
__global__ void lowrank_agg_kernel(int nc, int R, const int *__restrict__ con, const int *__restrict__ off,
                                   const double *__restrict__ sig, const double *__restrict__ P,
                                   const double *__restrict__ Q, double *M, int m) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    for (int t = blockIdx.y; t < nc; t += gridDim.y) {
        if (u < t || u >= nc) continue;
        double sum = 0.0;
        for (int k = off[t]; k < off[t + 1]; k++) {
            double part = 0.0;
            const double *pk = P + (long long)k * R, *qk = Q + (long long)k * R;
            for (int l = off[u]; l < off[u + 1]; l++) part += sig[l] * pk[l] * qk[l];
            sum += sig[k] * part;
        }
        const long long cu = con[u], ct = con[t];
        M[cu + ct * m] += sum;
        if (u != t) M[ct + cu * m] += sum;
    }
}
}  // namespace

int lowrank_factor_block(int n, int ncon, const long long *cptr, const int *cpos, const double *cval,
                         std::vector<int> &off, std::vector<double> &W, std::vector<double> &sig, int max_rank) {
    std::vector<Factor> F(ncon);
    const int T = ncon < 64 ? 1 : (int)std::max(1u, std::min(std::thread::hardware_concurrency(), 32u));
    std::vector<char> bad(T, 0);
    auto work = [&](int r) {
        for (int t = r; t < ncon && !bad[r]; t += T) {
            F[t] = factor_one(n, cpos + cptr[t], cval + cptr[t], cptr[t + 1] - cptr[t], 0x9e3779b97f4a7c15ull + t);
            if (!F[t].ok) bad[r] = 1;
        }
    };
    if (T == 1) {
        work(0);
    } else {
        std::vector<std::thread> th;
        for (int r = 0; r < T; r++) th.emplace_back(work, r);
        for (auto &x : th) x.join();
    }
    for (char b : bad)
        if (b) return 0;
    off.assign(ncon + 1, 0);
    for (int t = 0; t < ncon; t++) off[t + 1] = off[t] + (int)F[t].s.size();
    const int R = off[ncon];
    if (R > max_rank) return 0;
    W.assign((size_t)n * std::max(R, 1), 0.0);
    sig.assign(std::max(R, 1), 0.0);
    for (int t = 0; t < ncon; t++)
        for (size_t k = 0; k < F[t].s.size(); k++) {
            std::copy(F[t].w.begin() + k * n, F[t].w.begin() + (k + 1) * n, W.begin() + (size_t)(off[t] + k) * n);
            sig[off[t] + k] = F[t].s[k];
        }
    return 1;
}

int schur_assemble_lowrank(cudaStream_t st, const LowRankDev &L, const int *con, const double *X, const double *Zi,
                           double *M, int m) {
    const int n = L.n, R = L.R, nc = L.ncon;
    if (nc <= 0 || R <= 0) return BGPU_OK;
    if (!L.W || !L.sig || !L.off || !L.XW || !L.P || !L.Q || !con || !X || !Zi || !M) return BGPU_ERR_ARG;
    int rc;
    // P = W' (X W), Q = W' (Zi W): X, Zi column-major n x n; W column-major n x R
    if ((rc = gemm_f64(st, 0, 1, n, R, n, 1.0, X, n, 0, L.W, n, 0, 0.0, L.XW, n, 0, 1, 0))) return rc;
    if ((rc = gemm_f64(st, 1, 1, R, R, n, 1.0, L.W, n, 0, L.XW, n, 0, 0.0, L.P, R, 0, 1, 0))) return rc;
    if ((rc = gemm_f64(st, 0, 1, n, R, n, 1.0, Zi, n, 0, L.W, n, 0, 0.0, L.XW, n, 0, 1, 0))) return rc;
    if ((rc = gemm_f64(st, 1, 1, R, R, n, 1.0, L.W, n, 0, L.XW, n, 0, 0.0, L.Q, R, 0, 1, 0))) return rc;
    dim3 grid(ceil_div(nc, 256), std::min(nc, 65535));
    lowrank_agg_kernel<<<grid, 256, 0, st>>>(nc, R, con, L.off, L.sig, L.P, L.Q, M, m);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}
