// Kernels of the lockstep batch (lockstep.cu): many independent single-block SDPs (block order
// n_k <= 64, m_k constraints) advanced together, each launch covering every listed instance.
//
// Concatenations, instance k at:
//   boff[k]: its n_k x n_k arrays (X, Z, ...);      coff[k]: its m_k-vectors (y, D, ...);
//   moff[k]: its m_k x m_k arrays (M, L);           poff[k]: its m_k x t_k packed rows (P, Q),
//   t_k = n_k (n_k + 1) / 2, packed index u = q (q + 1) / 2 + p for p <= q.
#pragma once
#include <cuda_runtime.h>

namespace lockstep {

constexpr int NMAX = 64;   // the largest block order of the lockstep path

struct Layout {
    int B = 0;                    // instances
    const int *n = nullptr, *m = nullptr;
    const long long *boff = nullptr, *coff = nullptr, *moff = nullptr, *poff = nullptr;
};

// P row a of instance k: the upper entries of A_a (A[p, q], p <= q) at their packed index,
// built on the host.
// Q row a = packed (G_a + G_a') off the diagonal, G_a on it, G_a = X A_a Zi, for the work items
// (instance, first constraint) in items (chunks of `item` constraints); nmax: the largest n
// listed.  The chunk size is the batch's tuned work-item shape: ITEM_CANDIDATES are the sizes the
// autotuner (lockstep_solver.cuh, Lockstep::tune_items) times on each block-order class; every
// size gives the same Q (each constraint's row is computed alone).
constexpr int ITEM = 8;   // before tuning, and with -batchtune 0
constexpr int ITEM_MIN = 2;
constexpr int ITEM_CANDIDATES[5] = {2, 4, 8, 16, 32};
int form_q(cudaStream_t st, const Layout &L, const int2 *items, int nitems, int nmax, int item, const double *P,
           const double *Xc, const double *Zc, double *Q);
// M: the lower triangle copied to the upper one, for the listed instances.
int mirror(cudaStream_t st, const Layout &L, const int *list, int cnt, double *M);
// Per listed instance: D = diag(M)^-1/2 (1 where not positive), Lf = chol(D M D + reg[k] I)
// (lower; blocked, one CTA per instance); info[k] = first failing column + 1 or 0, pmin[k] =
// the smallest pivot (squared diagonal of the scaled factor).
int chol(cudaStream_t st, const Layout &L, const int *list, int cnt, const double *M, const double *reg, double *D,
         double *Lf, int *info, double *pmin);
// x := D Lf^-T Lf^-1 D x for the listed instances (x concatenated by coff; mmax: the largest m).
int prec(cudaStream_t st, const Layout &L, const int *list, int cnt, int mmax, const double *Lf, const double *D,
         double *x);
// Work items (instance, first row / column / packed index) split the larger instances over
// several CTAs: RI rows or columns per item for aop_packed and symv, 256 packed entries for
// atop_packed.
constexpr int RI = 64;
// y = M x for the listed items (M full, both triangles).
int symv(cudaStream_t st, const Layout &L, const int2 *items, int cnt, const double *M, const double *x, double *y);
// y[coff + a] = <A_a, D_k> from the packed rows (D: the n x n concatenation), and
// F_k = alpha sum_a y_a A_a + beta F_k, for the work items (nmax: the largest n).
int aop_packed(cudaStream_t st, const Layout &L, const int2 *items, int cnt, int nmax, const double *P,
               const double *Dc, double *y);
int atop_packed(cudaStream_t st, const Layout &L, const int2 *items, int cnt, const double *P, const double *y,
                double alpha, double beta, double *Fc);
// out[k nq + q] = <a_q, b_q> over instance k's segment [off[k], off[k+1]) for all k < B (a and b
// device pointer tables of nq entries; fixed summation order).
int seg_dots(cudaStream_t st, int B, const long long *off, int nq, const double *const *a, const double *const *b,
             double *out);

}  // namespace lockstep
