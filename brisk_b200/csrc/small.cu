// Batched kernels for many small SDP blocks (order n <= 64): one CTA per block, the block's
// matrices in shared memory, the blocks given by device pointer tables.  They replace, for such
// blocks, the per-block work of the reference's block-parallel loops (PBLK_FOR, solver.c:6053):
//   chol_lower (solver.c:679) with the factor's inverse,
//   small_lammin (solver.c:5947-6027): lambda_min(L^-1 D L^-T) by Householder tridiagonalization
//     and Sturm bisection, exact instead of Lanczos,
//   the n x n products of prod_pat / prod3 (solver.c:1111, 1332).
#include "common.cuh"
#include "kernels.h"
#include "small.h"

namespace {
constexpr int SN = SMALL_N_MAX;   // 64
constexpr int SL = SN + 1;        // padded smem stride

__device__ __forceinline__ void load_sq(double *S, const double *A, int n, int tid) {
    for (int idx = tid; idx < SN * SN; idx += 256) {
        const int r = idx % SN, c = idx / SN;
        S[r + c * SL] = (r < n && c < n) ? A[r + c * n] : 0.0;
    }
}

// A -> L (lower; the strict upper of the output is zeroed) and Li = L^-1 (lower); info[k] the first
// failing column (1-based) or 0.  A, L may be the same array.
__global__ void __launch_bounds__(256) chol_inv_kernel(int nb, const int *__restrict__ ns, double *const *A,
                                                       double *const *L, double *const *Li, int *info) {
    extern __shared__ __align__(16) unsigned char raw[];
    double *S = reinterpret_cast<double *>(raw);
    double *X = S + SN * SL;
    const int k = blockIdx.x, tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    if (k >= nb) return;
    const int n = ns[k];
    load_sq(S, A[k], n, tid);
    for (int idx = tid; idx < SN * SN; idx += 256) {
        const int r = idx % SN, c = idx / SN;
        X[r + c * SL] = (r == c) ? 1.0 : 0.0;
    }
    __syncthreads();
    int fail = 0;
    for (int c = 0; c < n; c++) {
        const double d = S[c + c * SL];
        if (!(d > 0.0) || !isfinite(d)) { fail = c + 1; break; }
        const double piv = sqrt(d);
        __syncthreads();
        if (tid == 0) S[c + c * SL] = piv;
        for (int r = c + 1 + tid; r < n; r += 256) S[r + c * SL] /= piv;
        __syncthreads();
        for (int q = c + 1 + tx; q < n; q += 16) {
            const double lqc = S[q + c * SL];
            for (int r = q + ty; r < n; r += 16) S[r + q * SL] -= S[r + c * SL] * lqc;
        }
        __syncthreads();
    }
    if (tid == 0) info[k] = fail;
    if (fail) return;
    for (int q = 0; q < n; q++) {
        const double lqq = S[q + q * SL];
        for (int j = tid; j <= q; j += 256) X[q + j * SL] /= lqq;
        __syncthreads();
        for (int j = tx; j <= q; j += 16) {
            const double xqj = X[q + j * SL];
            for (int r = q + 1 + ty; r < n; r += 16) X[r + j * SL] -= S[r + q * SL] * xqj;
        }
        __syncthreads();
    }
    double *Lk = L[k], *Lik = Li ? Li[k] : nullptr;
    for (int idx = tid; idx < n * n; idx += 256) {
        const int r = idx % n, c = idx / n;
        Lk[idx] = (r >= c) ? S[r + c * SL] : 0.0;
        if (Lik) Lik[idx] = (r >= c) ? X[r + c * SL] : 0.0;
    }
}

// C = alpha op(A) op(B) + beta C for n x n column-major blocks; ta/tb transpose A/B; sym writes
// the symmetric part of the product (then beta must be 0).
__global__ void __launch_bounds__(256) gemm_small_kernel(int nb, const int *__restrict__ ns, int ta, int tb,
                                                         double alpha, const double *const *A,
                                                         const double *const *B, double beta, double *const *C,
                                                         int sym) {
    extern __shared__ __align__(16) unsigned char raw[];
    double *SA = reinterpret_cast<double *>(raw);
    double *SB = SA + SN * SL;
    const int k = blockIdx.x, tid = threadIdx.x;
    if (k >= nb) return;
    const int n = ns[k];
    const double *a = A[k], *b = B[k];
    for (int idx = tid; idx < n * n; idx += 256) {
        const int r = idx % n, c = idx / n;
        SA[(ta ? c : r) + (ta ? r : c) * SL] = a[idx];   // SA holds op(A)
        SB[(tb ? c : r) + (tb ? r : c) * SL] = b[idx];   // SB holds op(B)
    }
    __syncthreads();
    double *ck = C[k];
    if (!sym) {
        for (int idx = tid; idx < n * n; idx += 256) {
            const int r = idx % n, c = idx / n;
            double s = 0.0;
            for (int q = 0; q < n; q++) s += SA[r + q * SL] * SB[q + c * SL];
            ck[idx] = (beta == 0.0) ? alpha * s : alpha * s + beta * ck[idx];
        }
    } else {
        for (int idx = tid; idx < n * n; idx += 256) {
            const int r = idx % n, c = idx / n;
            if (r < c) continue;
            double s1 = 0.0, s2 = 0.0;
            for (int q = 0; q < n; q++) {
                s1 += SA[r + q * SL] * SB[q + c * SL];
                s2 += SA[c + q * SL] * SB[q + r * SL];
            }
            const double v = alpha * 0.5 * (s1 + s2);
            ck[r + c * n] = v;
            ck[c + r * n] = v;
        }
    }
}

// lambda_min(Li D Li') per block: B formed in shared memory, reduced to tridiagonal form by
// Householder reflections, smallest eigenvalue by Sturm-count bisection to full precision.
__global__ void __launch_bounds__(256) lammin_kernel(int nb, const int *__restrict__ ns, const double *const *Li,
                                                     const double *const *D, double *lam) {
    extern __shared__ __align__(16) unsigned char raw[];
    double *SB = reinterpret_cast<double *>(raw);   // B
    double *SL_ = SB + SN * SL;                      // Li, then scratch
    double *W = SL_ + SN * SL;                       // Li D
    __shared__ double v[SN], p[SN], dg[SN], off[SN], red[8];
    const int k = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (k >= nb) return;
    const int n = ns[k];
    load_sq(SL_, Li[k], n, tid);
    load_sq(SB, D[k], n, tid);   // D temporarily in SB
    __syncthreads();
    for (int idx = tid; idx < n * n; idx += 256) {   // W = Li D
        const int r = idx % n, c = idx / n;
        double s = 0.0;
        for (int q = 0; q <= r; q++) s += SL_[r + q * SL] * SB[q + c * SL];
        W[r + c * SL] = s;
    }
    __syncthreads();
    for (int idx = tid; idx < n * n; idx += 256) {   // B = W Li'
        const int r = idx % n, c = idx / n;
        double s = 0.0;
        for (int q = 0; q <= c; q++) s += W[r + q * SL] * SL_[c + q * SL];
        SB[r + c * SL] = s;
    }
    __syncthreads();
    for (int idx = tid; idx < n * n; idx += 256) {   // exact symmetry
        const int r = idx % n, c = idx / n;
        if (r > c) {
            const double s = 0.5 * (SB[r + c * SL] + SB[c + r * SL]);
            SB[r + c * SL] = s;
            SB[c + r * SL] = s;
        }
    }
    __syncthreads();
    // Householder: column j, reflect rows j+1..n-1
    for (int j = 0; j + 2 < n; j++) {
        const int m0 = j + 1, len = n - m0;
        double part = 0.0;
        for (int i = tid; i < len; i += 256) { const double x = SB[m0 + i + j * SL]; part += x * x; }
        part = warp_sum(part);
        if (lane == 0) red[warp] = part;
        __syncthreads();
        double nx2 = 0.0;
        for (int w = 0; w < 8; w++) nx2 += red[w];
        const double x0 = SB[m0 + j * SL];
        const double alpha = (x0 >= 0.0) ? -sqrt(nx2) : sqrt(nx2);
        const double vtv = nx2 - 2.0 * alpha * x0 + alpha * alpha;   // |x - alpha e1|^2
        __syncthreads();
        if (tid == 0) { dg[j] = SB[j + j * SL]; off[j] = alpha; }
        if (!(vtv > 0.0)) {   // the column is already reduced
            if (tid == 0) off[j] = x0;
            __syncthreads();
            continue;
        }
        for (int i = tid; i < len; i += 256) v[i] = SB[m0 + i + j * SL] - (i == 0 ? alpha : 0.0);
        __syncthreads();
        const double tau = 2.0 / vtv;
        for (int i = tid; i < len; i += 256) {   // p = tau B22 v
            double s = 0.0;
            for (int q = 0; q < len; q++) s += SB[m0 + i + (m0 + q) * SL] * v[q];
            p[i] = tau * s;
        }
        __syncthreads();
        part = 0.0;
        for (int i = tid; i < len; i += 256) part += v[i] * p[i];
        part = warp_sum(part);
        if (lane == 0) red[warp] = part;
        __syncthreads();
        double vtp = 0.0;
        for (int w = 0; w < 8; w++) vtp += red[w];
        const double Kc = 0.5 * tau * vtp;
        __syncthreads();
        for (int i = tid; i < len; i += 256) p[i] -= Kc * v[i];   // w = p - K v
        __syncthreads();
        for (int idx = tid; idx < len * len; idx += 256) {         // B22 -= v w' + w v'
            const int r = idx % len, c = idx / len;
            SB[m0 + r + (m0 + c) * SL] -= v[r] * p[c] + p[r] * v[c];
        }
        __syncthreads();
    }
    if (tid == 0) {
        if (n >= 2) {
            dg[n - 2] = SB[(n - 2) + (n - 2) * SL];
            dg[n - 1] = SB[(n - 1) + (n - 1) * SL];
            off[n - 2] = SB[(n - 1) + (n - 2) * SL];
        } else {
            dg[0] = SB[0];
        }
        double lo = 1e300, hi = -1e300;
        for (int i = 0; i < n; i++) {
            const double r = (i > 0 ? fabs(off[i - 1]) : 0.0) + (i + 1 < n ? fabs(off[i]) : 0.0);
            lo = fmin(lo, dg[i] - r);
            hi = fmax(hi, dg[i] + r);
        }
        for (int it = 0; it < 200; it++) {
            const double mid = 0.5 * (lo + hi);
            if (!(mid > lo && mid < hi)) break;
            int cnt = 0;
            double q = dg[0] - mid;
            if (q < 0) cnt++;
            for (int i = 1; i < n; i++) {
                if (q == 0.0) q = 1e-300;
                q = (dg[i] - mid) - off[i - 1] * off[i - 1] / q;
                if (q < 0) cnt++;
            }
            if (cnt >= 1) hi = mid; else lo = mid;
        }
        lam[k] = (isfinite(lo) && isfinite(hi)) ? lo : -1e300;   // the lower end: conservative
    }
}

// V += inc dV and L = V for every block (try_step's step and the copy its Cholesky factors)
__global__ void step_copy_small_kernel(int nb, const int *__restrict__ ns, double inc, const double *const *dV,
                                       double *const *V, double *const *L) {
    const int k = blockIdx.x;
    if (k >= nb) return;
    const int n = ns[k];
    const double *d = dV[k];
    double *v = V[k], *l = L[k];
    for (int i = threadIdx.x; i < n * n; i += blockDim.x) {
        const double x = v[i] + inc * d[i];
        v[i] = x;
        l[i] = x;
    }
}

size_t smem2() { return 2 * (size_t)SN * SL * sizeof(double); }
size_t smem3() { return 3 * (size_t)SN * SL * sizeof(double); }

template <typename F>
int set_smem(F f, size_t bytes) {
    BGPU_CHECK(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    return BGPU_OK;
}
std::atomic<unsigned long long> g_attr_done{0};   // one bit per device
int attrs() {
    return once_per_device(g_attr_done, [] {
        int rc;
        if ((rc = set_smem(chol_inv_kernel, smem2()))) return rc;
        if ((rc = set_smem(gemm_small_kernel, smem2()))) return rc;
        return set_smem(lammin_kernel, smem3());
    });
}
}  // namespace

int small_chol_inv(cudaStream_t st, int nb, const int *ns, double *const *A, double *const *L, double *const *Li,
                   int *info) {
    if (nb <= 0) return BGPU_OK;
    if (int rc = attrs()) return rc;
    chol_inv_kernel<<<nb, 256, smem2(), st>>>(nb, ns, A, L, Li, info);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int small_gemm(cudaStream_t st, int nb, const int *ns, int ta, int tb, double alpha, const double *const *A,
               const double *const *B, double beta, double *const *C, int sym) {
    if (nb <= 0) return BGPU_OK;
    if (int rc = attrs()) return rc;
    gemm_small_kernel<<<nb, 256, smem2(), st>>>(nb, ns, ta, tb, alpha, A, B, beta, C, sym);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int small_lammin(cudaStream_t st, int nb, const int *ns, const double *const *Li, const double *const *D,
                 double *lam) {
    if (nb <= 0) return BGPU_OK;
    if (int rc = attrs()) return rc;
    lammin_kernel<<<nb, 256, smem3(), st>>>(nb, ns, Li, D, lam);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int small_step_copy(cudaStream_t st, int nb, const int *ns, double inc, const double *const *dV, double *const *V,
                    double *const *L) {
    if (nb <= 0) return BGPU_OK;
    step_copy_small_kernel<<<nb, 256, 0, st>>>(nb, ns, inc, dV, V, L);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}
