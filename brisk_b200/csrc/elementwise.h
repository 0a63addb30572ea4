// Element-wise launchers over dense block arrays (elementwise.cu).
#pragma once
#include <cuda_runtime.h>

// out = a x + b y + c z (null inputs count as zero; out may alias any input)
int ew_lincomb(cudaStream_t st, long long n, double a, const double *x, double b, const double *y, double c,
               const double *z, double *out);
int ew_add_diag(cudaStream_t st, int n, double *A, long long lda, double v);
// V += inc dV and L = V (the step of try_step and the copy its Cholesky test factors)
int ew_step_copy(cudaStream_t st, long long n, double inc, const double *dV, double *V, double *L);
int ew_set_scaled_identity(cudaStream_t st, int n, double *A, double v);
// out = s sym(G) + a x + b y, sym(G) = (G + G')/2; out must not alias G
int ew_sym_lincomb(cudaStream_t st, int n, const double *G, double s, double a, const double *x, double b,
                   const double *y, double *out);
