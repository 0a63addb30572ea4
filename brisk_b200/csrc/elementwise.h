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

// Over blocks stored one after another (block k: order d_n[k], elements d_off[k] .. d_off[k+1] of
// the concatenation, column-major; d_off has nb+1 entries): the same as ew_sym_lincomb per block,
// and out_k = v_k I (only the blocks with d_only[k] != 0 when d_only is not null), in one launch each.
int ew_sym_lincomb_blocks(cudaStream_t st, int nb, const int *d_n, const long long *d_off, long long total,
                          const double *G, double s, double a, const double *x, double b, const double *y,
                          double *out);
int ew_scaled_identity_blocks(cudaStream_t st, int nb, const int *d_n, const long long *d_off, long long total,
                              const double *d_v, const int *d_only, double *out);
// Per-block coefficients (device arrays of nb values; a null array or operand counts as zero):
// out = ca x + cb y + cc z;  out = cs sym(G) + ca x + cb y;  V += inc dV, L = V;  dst = src on the
// blocks whose flag is set.
int ew_lincomb_coef(cudaStream_t st, int nb, const long long *d_off, long long total, const double *ca,
                    const double *x, const double *cb, const double *y, const double *cc, const double *z,
                    double *out);
int ew_sym_coef(cudaStream_t st, int nb, const int *d_n, const long long *d_off, long long total, const double *G,
                const double *cs, const double *ca, const double *x, const double *cb, const double *y, double *out);
int ew_step_copy_coef(cudaStream_t st, int nb, const long long *d_off, long long total, const double *inc,
                      const double *dV, double *V, double *L);
int ew_copy_masked(cudaStream_t st, int nb, const long long *d_off, long long total, const int *flag,
                   const double *src, double *dst);
