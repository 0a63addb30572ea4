// Element-wise kernels over the n x n iterate arrays of a block (X, Z, dX, dZ, R0, ...).
#include "common.cuh"
#include "kernels.h"
#include "elementwise.h"

namespace {
__global__ void lincomb_kernel(long long n, double a, const double *x, double b, const double *y, double c,
                               const double *z, double *out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = 0.0;
    if (x) v += a * x[i];
    if (y) v += b * y[i];
    if (z) v += c * z[i];
    out[i] = v;
}
__global__ void add_diag_kernel(int n, double *A, long long lda, double v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) A[i + (long long)i * lda] += v;
}
__global__ void step_copy_kernel(long long n, double inc, const double *dV, double *V, double *L) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = V[i] + inc * dV[i];
    V[i] = v;
    L[i] = v;
}
__global__ void set_diag_matrix_kernel(int n, double *A, double v) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)n * n) return;
    const int i = (int)(idx % n), j = (int)(idx / n);
    A[idx] = (i == j) ? v : 0.0;
}
// sym: out = 0.5 (G + G') + a*x + b*y  (x or y may be null)
__global__ void sym_lincomb_kernel(int n, const double *G, double s, double a, const double *x, double b,
                                   const double *y, double *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= n) return;
    const long long p = i + (long long)j * n, q = j + (long long)i * n;
    double v = s * 0.5 * (G[p] + G[q]);
    if (x) v += a * x[p];
    if (y) v += b * y[p];
    out[p] = v;
}
// the block of concatenated element g: off (nb+1 offsets) is ascending, off[0] = 0
__device__ __forceinline__ int block_of(long long g, int nb, const long long *__restrict__ off) {
    int lo = 0, hi = nb - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void sym_lincomb_blocks_kernel(int nb, const int *__restrict__ ns, const long long *__restrict__ off,
                                          long long total, const double *G, double s, double a, const double *x,
                                          double b, const double *y, double *out) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    const int k = block_of(g, nb, off), n = ns[k];
    const long long l = g - off[k];
    const int j = (int)(l / n), i = (int)(l - (long long)j * n);
    const long long q = off[k] + j + (long long)i * n;
    double v = s * 0.5 * (G[g] + G[q]);
    if (x) v += a * x[g];
    if (y) v += b * y[g];
    out[g] = v;
}

__global__ void scaled_identity_blocks_kernel(int nb, const int *__restrict__ ns, const long long *__restrict__ off,
                                              long long total, const double *__restrict__ v,
                                              const int *__restrict__ only, double *out) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    const int k = block_of(g, nb, off), n = ns[k];
    if (only && !only[k]) return;
    const long long l = g - off[k];
    out[g] = (l % (n + 1) == 0) ? v[k] : 0.0;
}
// per-block coefficients: out = ca[k] x + cb[k] y + cc[k] z on block k (a null coefficient array
// or operand counts as zero)
__global__ void lincomb_coef_kernel(int nb, const long long *__restrict__ off, long long total,
                                    const double *__restrict__ ca, const double *x, const double *__restrict__ cb,
                                    const double *y, const double *__restrict__ cc, const double *z, double *out) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    const int k = block_of(g, nb, off);
    double v = 0.0;
    if (ca && x) v += ca[k] * x[g];
    if (cb && y) v += cb[k] * y[g];
    if (cc && z) v += cc[k] * z[g];
    out[g] = v;
}

// out = cs[k] sym(G) + ca[k] x + cb[k] y on block k
__global__ void sym_coef_kernel(int nb, const int *__restrict__ ns, const long long *__restrict__ off, long long total,
                                const double *G, const double *__restrict__ cs, const double *__restrict__ ca,
                                const double *x, const double *__restrict__ cb, const double *y, double *out) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    const int k = block_of(g, nb, off), n = ns[k];
    const long long l = g - off[k];
    const int j = (int)(l / n), i = (int)(l - (long long)j * n);
    const long long q = off[k] + j + (long long)i * n;
    double v = cs[k] * 0.5 * (G[g] + G[q]);
    if (ca && x) v += ca[k] * x[g];
    if (cb && y) v += cb[k] * y[g];
    out[g] = v;
}

// V += inc[k] dV and L = V on block k
__global__ void step_copy_coef_kernel(int nb, const long long *__restrict__ off, long long total,
                                      const double *__restrict__ inc, const double *__restrict__ dV, double *V,
                                      double *L) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    const int k = block_of(g, nb, off);
    const double v = V[g] + inc[k] * dV[g];
    V[g] = v;
    L[g] = v;
}

// dst = src on the blocks with flag[k] != 0
__global__ void copy_masked_kernel(int nb, const long long *__restrict__ off, long long total, const int *__restrict__ flag,
                                   const double *__restrict__ src, double *dst) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    if (flag[block_of(g, nb, off)]) dst[g] = src[g];
}
}  // namespace

int ew_lincomb_coef(cudaStream_t st, int nb, const long long *d_off, long long total, const double *ca,
                    const double *x, const double *cb, const double *y, const double *cc, const double *z,
                    double *out) {
    if (total <= 0 || nb <= 0) return BGPU_OK;
    lincomb_coef_kernel<<<ceil_div(total, 256), 256, 0, st>>>(nb, d_off, total, ca, x, cb, y, cc, z, out);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int ew_sym_coef(cudaStream_t st, int nb, const int *d_n, const long long *d_off, long long total, const double *G,
                const double *cs, const double *ca, const double *x, const double *cb, const double *y, double *out) {
    if (total <= 0 || nb <= 0) return BGPU_OK;
    sym_coef_kernel<<<ceil_div(total, 256), 256, 0, st>>>(nb, d_n, d_off, total, G, cs, ca, x, cb, y, out);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int ew_step_copy_coef(cudaStream_t st, int nb, const long long *d_off, long long total, const double *inc,
                      const double *dV, double *V, double *L) {
    if (total <= 0 || nb <= 0) return BGPU_OK;
    step_copy_coef_kernel<<<ceil_div(total, 256), 256, 0, st>>>(nb, d_off, total, inc, dV, V, L);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int ew_copy_masked(cudaStream_t st, int nb, const long long *d_off, long long total, const int *flag,
                   const double *src, double *dst) {
    if (total <= 0 || nb <= 0) return BGPU_OK;
    copy_masked_kernel<<<ceil_div(total, 256), 256, 0, st>>>(nb, d_off, total, flag, src, dst);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int ew_sym_lincomb_blocks(cudaStream_t st, int nb, const int *d_n, const long long *d_off, long long total,
                          const double *G, double s, double a, const double *x, double b, const double *y,
                          double *out) {
    if (total <= 0 || nb <= 0) return BGPU_OK;
    sym_lincomb_blocks_kernel<<<ceil_div(total, 256), 256, 0, st>>>(nb, d_n, d_off, total, G, s, a, x, b, y, out);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int ew_scaled_identity_blocks(cudaStream_t st, int nb, const int *d_n, const long long *d_off, long long total,
                              const double *d_v, const int *d_only, double *out) {
    if (total <= 0 || nb <= 0) return BGPU_OK;
    scaled_identity_blocks_kernel<<<ceil_div(total, 256), 256, 0, st>>>(nb, d_n, d_off, total, d_v, d_only, out);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int ew_lincomb(cudaStream_t st, long long n, double a, const double *x, double b, const double *y, double c,
               const double *z, double *out) {
    if (n <= 0) return BGPU_OK;
    lincomb_kernel<<<ceil_div(n, 256), 256, 0, st>>>(n, a, x, b, y, c, z, out);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}
int ew_add_diag(cudaStream_t st, int n, double *A, long long lda, double v) {
    add_diag_kernel<<<ceil_div(n, 256), 256, 0, st>>>(n, A, lda, v);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}
int ew_step_copy(cudaStream_t st, long long n, double inc, const double *dV, double *V, double *L) {
    step_copy_kernel<<<ceil_div(n, 256), 256, 0, st>>>(n, inc, dV, V, L);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}
int ew_set_scaled_identity(cudaStream_t st, int n, double *A, double v) {
    set_diag_matrix_kernel<<<ceil_div((long long)n * n, 256), 256, 0, st>>>(n, A, v);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}
int ew_sym_lincomb(cudaStream_t st, int n, const double *G, double s, double a, const double *x, double b,
                   const double *y, double *out) {
    // out may alias x or y but not G (G is read at both (i,j) and (j,i))
    sym_lincomb_kernel<<<dim3(ceil_div(n, 128), n), 128, 0, st>>>(n, G, s, a, x, b, y, out);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}
