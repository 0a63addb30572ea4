// Supernodal sparse Cholesky of the Schur complement (the reference's schol_* in sparsechol.c and
// sparse_build, solver.c:4014): a host symbolic phase (minimum-degree ordering on the quotient
// graph whose first elements are the blocks' constraint cliques, supernodes, the supernode tree)
// and a device numeric phase (multifrontal: one CTA per front, fronts of one tree level in one
// launch; forward and backward solves over the supernodes).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace schol {

struct Analysis {
    int m = 0;
    std::vector<int> perm, iperm;    // perm[k]: the constraint at elimination position k
    int nsup = 0;
    std::vector<int> sfirst;         // supernode s owns positions sfirst[s] .. sfirst[s+1]-1
    std::vector<long long> rptr;     // front rows of s: rows[rptr[s] .. rptr[s+1]) (positions, ascending;
    std::vector<int> rows;           //   the first ns are s's own columns)
    std::vector<int> parent;         // -1 at a root
    std::vector<int> cptr, child;    // children of s: child[cptr[s] .. cptr[s+1]) (ascending)
    std::vector<long long> relptr;   // s as a child: rel[relptr[s] ..) = indices of its off-diagonal rows
    std::vector<int> rel;            //   within its parent's front rows
    std::vector<long long> lptr;     // panel of s: f x ns column-major at L + lptr[s]
    std::vector<long long> uptr;     // update matrix of s: rs x rs column-major at U + uptr[s]
    std::vector<int> lvptr, lvsup;   // supernodes by tree level (leaves first)
    double flops = 0;                // factorization flops (ns^3/3 + ns^2 rs + ns rs^2 per front)
    double nnz = 0;                  // entries of L
    long long pattern = 0;           // entries of the pattern of M below the diagonal
    int fmax = 0;                    // the largest front
};

// Minimum-degree rounds take every supervariable of degree <= dmin (1 + g_mmd_delta) (default 1).
extern double g_mmd_delta;
// cliques: constraint index sets (each block's constraints).  Returns 0, or 1 on bad input.
int analyze(int m, const std::vector<std::vector<int>> &cliques, Analysis &A);

// The device side of a factor.
struct Factor {
    const Analysis *A = nullptr;
    // device arrays
    int *perm = nullptr, *f = nullptr, *ns = nullptr, *rows = nullptr, *cptr = nullptr, *child = nullptr,
        *rel = nullptr, *lvsup = nullptr;
    long long *rptr = nullptr, *relptr = nullptr, *lptr = nullptr, *uptr = nullptr;
    double *L = nullptr, *U = nullptr, *x = nullptr, *V = nullptr;
    int *info = nullptr;
    double *pmin = nullptr;
    size_t bytes = 0;
    bool fp32 = false;   // the last factor's type (L and U then hold floats, in the first half of their bytes)
    // the solve's launches captured as a CUDA graph, per factor type, for the (D, x) they were
    // captured with (released by release())
    cudaGraphExec_t solve_graph[2] = {nullptr, nullptr};
    const double *graph_D[2] = {nullptr, nullptr};
    double *graph_x[2] = {nullptr, nullptr};
    int graph_launches = 0;
    // host: front orders, own columns, and per level the supernodes (shared-memory fronts first),
    // how many fit shared memory and the largest of those
    std::vector<int> fs, nss, lvs, lvsplit, lvsmem;
};
// Device bytes of the factor's arrays (one allocation, carved by factor_bind).
size_t factor_bytes(const Analysis &A);
// Lays out the factor's arrays in buf (factor_bytes(A) bytes, 256-byte aligned) and uploads the
// analysis (stream-ordered; the host vectors of A must outlive the copies: call cudaStreamSynchronize).
int factor_bind(cudaStream_t st, const Analysis &A, void *buf, Factor &F);
// L L' = D M D + reg I on the pattern (M: dense m x m, column-major, both triangles; D = d_D),
// in FP64, or in FP32 (fp32: the fronts, L and the update matrices in single precision; M, D
// and the solve's vectors stay FP64).  info: first failing elimination position + 1 or 0;
// pmin: the smallest pivot (scaled).
int factor(cudaStream_t st, Factor &F, const double *M, long long ldm, const double *d_D, double reg,
           bool fp32 = false);
// x := D (L L')^-1 D x (x in constraint order, length m; D = d_D), with the last factor's type.
// The launches (two per tree level and the permutations) run as one CUDA graph, captured on
// the first solve with these (D, x) on a stream that can capture; otherwise launched directly.
int solve(cudaStream_t st, Factor &F, const double *d_D, double *x);
// Releases the factor's graphs (its device memory belongs to the caller's allocation).
void release(Factor &F);

}  // namespace schol
