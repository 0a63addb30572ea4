// Batched kernels for small blocks (n <= SMALL_N_MAX), one CTA per block (small.cu).
#pragma once
#include <cuda_runtime.h>

constexpr int SMALL_N_MAX = 64;

// L = chol(A) (lower, strict upper zeroed), Li = L^-1 (may be null); info[k]: first failing column
// (1-based) or 0.  A and L may alias.
int small_chol_inv(cudaStream_t st, int nb, const int *ns, double *const *A, double *const *L, double *const *Li,
                   int *info);
// C = alpha op(A) op(B) + beta C (ta/tb: transpose), or its symmetric part when sym (beta = 0).
int small_gemm(cudaStream_t st, int nb, const int *ns, int ta, int tb, double alpha, const double *const *A,
               const double *const *B, double beta, double *const *C, int sym);
// lam[k] = lambda_min(Li D Li'), exact (Householder tridiagonalization + bisection).
int small_lammin(cudaStream_t st, int nb, const int *ns, const double *const *Li, const double *const *D,
                 double *lam);
// V += inc dV, L = V.
int small_step_copy(cudaStream_t st, int nb, const int *ns, double inc, const double *const *dV, double *const *V,
                    double *const *L);
