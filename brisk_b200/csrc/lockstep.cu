// Kernels of the lockstep batch (lockstep.h).  Every kernel covers all listed instances in one
// launch, one CTA per instance (or per work item), and sums in a fixed order.
#include "common.cuh"
#include "lockstep.h"

#include <algorithm>

namespace lockstep {
namespace {

__device__ __forceinline__ long long upk(int p, int q) { return (long long)q * (q + 1) / 2 + p; }
// the (p, q), p <= q, of packed index u
__device__ __forceinline__ void unpk(int u, int &p, int &q) {
    int c = (int)((sqrt(8.0 * (double)u + 1.0) - 1.0) * 0.5);
    while (c * (c + 1) / 2 > u) c--;
    while ((c + 1) * (c + 2) / 2 <= u) c++;
    q = c;
    p = u - c * (c + 1) / 2;
}

// C = A B for n x n matrices in shared memory (column-major), thread (tx, ty) of a 16 x 16 grid
// owning the RT x RT outputs (tx + 16 r, ty + 16 c): consecutive tx read consecutive A rows.
template <int RT>
__device__ __forceinline__ void smem_gemm(int n, const double *__restrict__ A, const double *__restrict__ Bm,
                                          double *__restrict__ C) {
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    double acc[RT][RT];
#pragma unroll
    for (int r = 0; r < RT; r++)
#pragma unroll
        for (int c = 0; c < RT; c++) acc[r][c] = 0.0;
    for (int q = 0; q < n; q++) {
        double a[RT], b[RT];
#pragma unroll
        for (int r = 0; r < RT; r++) { const int i = tx + 16 * r; a[r] = i < n ? A[i + q * n] : 0.0; }
#pragma unroll
        for (int c = 0; c < RT; c++) { const int j = ty + 16 * c; b[c] = j < n ? Bm[q + j * n] : 0.0; }
#pragma unroll
        for (int r = 0; r < RT; r++)
#pragma unroll
            for (int c = 0; c < RT; c++) acc[r][c] += a[r] * b[c];
    }
#pragma unroll
    for (int r = 0; r < RT; r++)
#pragma unroll
        for (int c = 0; c < RT; c++) {
            const int i = tx + 16 * r, j = ty + 16 * c;
            if (i < n && j < n) C[i + j * n] = acc[r][c];
        }
}

__device__ __forceinline__ void smem_gemm_n(int n, const double *A, const double *Bm, double *C) {
    if (n <= 16) smem_gemm<1>(n, A, Bm, C);
    else if (n <= 32) smem_gemm<2>(n, A, Bm, C);
    else if (n <= 48) smem_gemm<3>(n, A, Bm, C);
    else smem_gemm<4>(n, A, Bm, C);
}

// one work item: `item` constraints of one instance; shared: X, Z, A, W (n x n each); 256 threads
__global__ void __launch_bounds__(256) form_q_kernel(int item, const int2 *__restrict__ items, const int *__restrict__ nv,
                                                     const int *__restrict__ mv, const long long *__restrict__ boff,
                                                     const long long *__restrict__ poff, const double *__restrict__ P,
                                                     const double *__restrict__ Xc, const double *__restrict__ Zc,
                                                     double *Q) {
    extern __shared__ __align__(16) double fq[];
    const int2 it = items[blockIdx.x];
    const int k = it.x, a0 = it.y;
    const int n = nv[k], m = mv[k], nn = n * n, t = n * (n + 1) / 2;
    double *Xs = fq, *Zs = fq + nn, *As = fq + 2 * nn, *Ws = fq + 3 * nn;
    const double *X = Xc + boff[k], *Z = Zc + boff[k];
    for (int i = threadIdx.x; i < nn; i += blockDim.x) { Xs[i] = X[i]; Zs[i] = Z[i]; }
    const double *Pk = P + poff[k];
    double *Qk = Q + poff[k];
    const int a1 = min(m, a0 + item);
    for (int a = a0; a < a1; a++) {
        const double *prow = Pk + (long long)a * t;
        __syncthreads();   // the previous constraint's A (G) is no longer read
        for (int u = threadIdx.x; u < t; u += blockDim.x) {   // A from its packed upper entries
            int i, j;
            unpk(u, i, j);
            const double v = prow[u];
            As[i + j * n] = v;
            As[j + i * n] = v;
        }
        __syncthreads();
        smem_gemm_n(n, As, Zs, Ws);   // W = A Zi
        __syncthreads();
        smem_gemm_n(n, Xs, Ws, As);   // G = X W, into A's buffer
        __syncthreads();
        double *qrow = Qk + (long long)a * t;
        for (int u = threadIdx.x; u < t; u += blockDim.x) {   // Q = packed (G + G')
            int i, j;
            unpk(u, i, j);
            qrow[u] = (i < j) ? As[i + j * n] + As[j + i * n] : As[i + i * n];
        }
    }
}

__global__ void mirror_kernel(const int *__restrict__ list, const int *__restrict__ mv, const long long *__restrict__ moff,
                              double *M) {
    const int k = list[blockIdx.x], m = mv[k];
    double *Mk = M + moff[k];
    for (long long idx = threadIdx.x; idx < (long long)m * m; idx += blockDim.x) {
        const int i = (int)(idx % m), j = (int)(idx / m);
        if (i < j) Mk[idx] = Mk[j + (long long)i * m];
    }
}

constexpr int CB = 32;   // panel width of the batched Cholesky
constexpr int CT = 64;   // tile of its trailing update

__global__ void __launch_bounds__(256) chol_kernel(const int *__restrict__ list, const int *__restrict__ mv,
                                                   const long long *__restrict__ moff, const long long *__restrict__ coff,
                                                   const double *__restrict__ M, const double *__restrict__ reg,
                                                   double *D, double *Lf, int *info, double *pmin) {
    __shared__ double S[CB][CB + 1];
    __shared__ double PI[CT][CB + 1], PJ[CT][CB + 1];
    __shared__ int fail_s;
    __shared__ double pm_s;
    const int k = list[blockIdx.x], m = mv[k];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const double *Mk = M + moff[k];
    double *Lk = Lf + moff[k];
    double *Dk = D + coff[k];
    const double r = reg[k];
    for (int i = tid; i < m; i += 256) {
        const double d = Mk[i + (long long)i * m];
        Dk[i] = d > 0 ? 1.0 / sqrt(d) : 1.0;
    }
    if (tid == 0) { fail_s = 0; pm_s = 1e300; }
    __syncthreads();
    for (long long idx = tid; idx < (long long)m * m; idx += 256) {
        const int i = (int)(idx % m), j = (int)(idx / m);
        Lk[idx] = (i >= j) ? Dk[i] * Mk[idx] * Dk[j] + (i == j ? r : 0.0) : 0.0;
    }
    __syncthreads();
    for (int k0 = 0; k0 < m; k0 += CB) {
        const int nb = min(CB, m - k0);
        for (int idx = tid; idx < CB * CB; idx += 256) {
            const int i = idx % CB, j = idx / CB;
            S[i][j] = (i < nb && j < nb && i >= j) ? Lk[(k0 + i) + (long long)(k0 + j) * m] : 0.0;
        }
        __syncthreads();
        if (warp == 0) {   // the diagonal block, one warp (lane r owns row r)
            for (int c = 0; c < nb; c++) {
                __syncwarp();
                const double d = S[c][c];
                if (!(d > 0.0) || !isfinite(d)) {
                    if (lane == 0) fail_s = k0 + c + 1;
                    break;
                }
                if (lane == 0) pm_s = fmin(pm_s, d);
                const double sd = sqrt(d);
                __syncwarp();
                if (lane > c && lane < nb) S[lane][c] /= sd;
                __syncwarp();
                if (lane == c) S[c][c] = sd;
                if (lane > c && lane < nb)
                    for (int q = c + 1; q <= lane; q++) S[lane][q] -= S[lane][c] * S[q][c];
            }
        }
        __syncthreads();
        if (fail_s) break;
        for (int idx = tid; idx < CB * CB; idx += 256) {
            const int i = idx % CB, j = idx / CB;
            if (i < nb && j < nb && i >= j) Lk[(k0 + i) + (long long)(k0 + j) * m] = S[i][j];
        }
        // the panel below: L(i, k0..k0+nb) = A(i, .) L_kk^-T
        for (int i = k0 + nb + tid; i < m; i += 256) {
            for (int c = 0; c < nb; c++) {
                double v = Lk[i + (long long)(k0 + c) * m];
                for (int q = 0; q < c; q++) v -= Lk[i + (long long)(k0 + q) * m] * S[c][q];
                Lk[i + (long long)(k0 + c) * m] = v / S[c][c];
            }
        }
        __syncthreads();
        // the trailing lower triangle: L(i, j) -= L(i, panel) L(j, panel)', i >= j >= k0 + nb
        const int base = k0 + nb, rem = m - base, T = (rem + CT - 1) / CT;
        for (int ti = 0; ti < T; ti++) {
            for (int idx = tid; idx < CT * CB; idx += 256) {
                const int ii = idx % CT, c = idx / CT;
                const int i = base + ti * CT + ii;
                PI[ii][c] = (i < m && c < nb) ? Lk[i + (long long)(k0 + c) * m] : 0.0;
            }
            for (int tj = 0; tj <= ti; tj++) {
                for (int idx = tid; idx < CT * CB; idx += 256) {
                    const int jj = idx % CT, c = idx / CT;
                    const int j = base + tj * CT + jj;
                    PJ[jj][c] = (j < m && c < nb) ? Lk[j + (long long)(k0 + c) * m] : 0.0;
                }
                __syncthreads();
                for (int e = tid; e < CT * CT; e += 256) {
                    const int ii = e % CT, jj = e / CT;
                    const int i = base + ti * CT + ii, j = base + tj * CT + jj;
                    if (i < m && j < m && i >= j) {
                        double s = 0.0;
                        for (int c = 0; c < nb; c++) s += PI[ii][c] * PJ[jj][c];
                        Lk[i + (long long)j * m] -= s;
                    }
                }
                __syncthreads();
            }
        }
    }
    if (tid == 0) {
        info[k] = fail_s;
        pmin[k] = fail_s ? 0.0 : pm_s;
    }
}

__global__ void __launch_bounds__(256) prec_kernel(const int *__restrict__ list, const int *__restrict__ mv,
                                                   const long long *__restrict__ moff, const long long *__restrict__ coff,
                                                   const double *__restrict__ Lf, const double *__restrict__ D,
                                                   double *x) {
    extern __shared__ __align__(16) double xs[];
    const int k = list[blockIdx.x], m = mv[k];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const double *Lk = Lf + moff[k];
    const double *Dk = D + coff[k];
    double *xk = x + coff[k];
    for (int i = tid; i < m; i += 256) xs[i] = Dk[i] * xk[i];
    __syncthreads();
    for (int k0 = 0; k0 < m; k0 += 32) {   // forward: L y = x
        const int nb = min(32, m - k0);
        if (warp == 0) {
            double v = lane < nb ? xs[k0 + lane] : 0.0;
            for (int c = 0; c < nb; c++) {
                const double xc = __shfl_sync(0xffffffffu, v, c) / Lk[(k0 + c) + (long long)(k0 + c) * m];
                if (lane == c) v = xc;
                else if (lane > c && lane < nb) v -= Lk[(k0 + lane) + (long long)(k0 + c) * m] * xc;
            }
            if (lane < nb) xs[k0 + lane] = v;
        }
        __syncthreads();
        for (int i = k0 + nb + tid; i < m; i += 256) {
            double s = 0.0;
            for (int c = 0; c < nb; c++) s += Lk[i + (long long)(k0 + c) * m] * xs[k0 + c];
            xs[i] -= s;
        }
        __syncthreads();
    }
    for (int k0 = ((m - 1) / 32) * 32; k0 >= 0; k0 -= 32) {   // backward: L' z = y
        const int nb = min(32, m - k0);
        for (int c = warp; c < nb; c += 8) {
            double s = 0.0;
            for (int i = k0 + nb + lane; i < m; i += 32) s += Lk[i + (long long)(k0 + c) * m] * xs[i];
            s = warp_sum(s);
            if (lane == 0) xs[k0 + c] -= s;
        }
        __syncthreads();
        if (warp == 0) {
            double v = lane < nb ? xs[k0 + lane] : 0.0;
            for (int c = nb - 1; c >= 0; c--) {
                const double xc = __shfl_sync(0xffffffffu, v, c) / Lk[(k0 + c) + (long long)(k0 + c) * m];
                if (lane == c) v = xc;
                else if (lane < c) v -= Lk[(k0 + c) + (long long)(k0 + lane) * m] * xc;
            }
            if (lane < nb) xs[k0 + lane] = v;
        }
        __syncthreads();
    }
    for (int i = tid; i < m; i += 256) xk[i] = Dk[i] * xs[i];
}

__global__ void __launch_bounds__(256) symv_kernel(const int2 *__restrict__ items, const int *__restrict__ mv,
                                                   const long long *__restrict__ moff, const long long *__restrict__ coff,
                                                   const double *__restrict__ M, const double *__restrict__ x, double *y) {
    const int2 it = items[blockIdx.x];
    const int k = it.x, m = mv[k];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double *Mk = M + moff[k];
    const double *xk = x + coff[k];
    double *yk = y + coff[k];
    const int i1 = min(m, it.y + RI);
    for (int i = it.y + warp; i < i1; i += 8) {   // column i of the symmetric M
        double s = 0.0;
        for (int j = lane; j < m; j += 32) s += Mk[j + (long long)i * m] * xk[j];
        s = warp_sum(s);
        if (lane == 0) yk[i] = s;
    }
}

// y[a] = <A_a, D> = sum_u P[a, u] Dp[u], Dp = packed (D + D') off the diagonal, D on it; a work
// item is (instance, first row) with RI rows
__global__ void __launch_bounds__(256) aop_packed_kernel(const int2 *__restrict__ items, const int *__restrict__ nv,
                                                         const int *__restrict__ mv, const long long *__restrict__ boff,
                                                         const long long *__restrict__ coff,
                                                         const long long *__restrict__ poff, const double *__restrict__ P,
                                                         const double *__restrict__ Dc, double *y) {
    extern __shared__ __align__(16) double dp[];
    const int2 it = items[blockIdx.x];
    const int k = it.x, r0 = it.y, n = nv[k], m = mv[k], t = n * (n + 1) / 2;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double *D = Dc + boff[k];
    for (int u = threadIdx.x; u < t; u += blockDim.x) {
        int i, j;
        unpk(u, i, j);
        dp[u] = (i < j) ? D[i + j * n] + D[j + i * n] : D[i + i * n];
    }
    __syncthreads();
    const double *Pk = P + poff[k];
    double *yk = y + coff[k];
    const int r1 = min(m, r0 + RI);
    for (int a = r0 + warp; a < r1; a += 8) {
        const double *row = Pk + (long long)a * t;
        double s = 0.0;
        for (int u = lane; u < t; u += 32) s += row[u] * dp[u];
        s = warp_sum(s);
        if (lane == 0) yk[a] = s;
    }
}

// F = alpha unpack(P' y) + beta F; a work item is (instance, first packed index) with 256 of them
__global__ void __launch_bounds__(256) atop_packed_kernel(const int2 *__restrict__ items, const int *__restrict__ nv,
                                                          const int *__restrict__ mv, const long long *__restrict__ boff,
                                                          const long long *__restrict__ coff,
                                                          const long long *__restrict__ poff,
                                                          const double *__restrict__ P, const double *__restrict__ y,
                                                          double alpha, double beta, double *Fc) {
    const int2 it = items[blockIdx.x];
    const int k = it.x, n = nv[k], m = mv[k], t = n * (n + 1) / 2;
    const int u = it.y + threadIdx.x;
    if (u >= t) return;
    const double *Pk = P + poff[k];
    const double *yk = y + coff[k];
    double s = 0.0;
    for (int a = 0; a < m; a++) s += Pk[(long long)a * t + u] * yk[a];
    int i, j;
    unpk(u, i, j);
    double *F = Fc + boff[k];
    const double v = alpha * s;
    F[i + j * n] = beta == 0.0 ? v : v + beta * F[i + j * n];
    if (i != j) F[j + i * n] = beta == 0.0 ? v : v + beta * F[j + i * n];
}

constexpr int DQ = 8;
__global__ void __launch_bounds__(256) seg_dots_kernel(const long long *__restrict__ off, int nq,
                                                       const double *const *__restrict__ a,
                                                       const double *const *__restrict__ b, double *out) {
    __shared__ double part[DQ][8];
    const int k = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double acc[DQ];
#pragma unroll
    for (int q = 0; q < DQ; q++) acc[q] = 0.0;
    for (long long i = off[k] + tid; i < off[k + 1]; i += 256)
#pragma unroll
        for (int q = 0; q < DQ; q++)
            if (q < nq) acc[q] += a[q][i] * b[q][i];
#pragma unroll
    for (int q = 0; q < DQ; q++) {
        const double v = warp_sum(acc[q]);
        if (lane == 0) part[q][warp] = v;
    }
    __syncthreads();
    if (tid < nq) {
        double s = 0.0;
        for (int w = 0; w < 8; w++) s += part[tid][w];
        out[(long long)k * nq + tid] = s;
    }
}
}  // namespace

size_t form_q_smem(int nmax) { return 4 * (size_t)nmax * nmax * sizeof(double); }

int form_q(cudaStream_t st, const Layout &L, const int2 *items, int nitems, int nmax, int item, const double *P,
           const double *Xc, const double *Zc, double *Q) {
    if (nitems <= 0) return BGPU_OK;
    if (nmax <= 0 || nmax > NMAX || item <= 0) return BGPU_ERR_ARG;
    BGPU_ATTR_ONCE(BGPU_CHECK(cudaFuncSetAttribute(form_q_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)form_q_smem(NMAX))));
    form_q_kernel<<<nitems, 256, form_q_smem(nmax), st>>>(item, items, L.n, L.m, L.boff, L.poff, P, Xc, Zc, Q);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int mirror(cudaStream_t st, const Layout &L, const int *list, int cnt, double *M) {
    if (cnt <= 0) return BGPU_OK;
    mirror_kernel<<<cnt, 256, 0, st>>>(list, L.m, L.moff, M);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int chol(cudaStream_t st, const Layout &L, const int *list, int cnt, const double *M, const double *reg, double *D,
         double *Lf, int *info, double *pmin) {
    if (cnt <= 0) return BGPU_OK;
    chol_kernel<<<cnt, 256, 0, st>>>(list, L.m, L.moff, L.coff, M, reg, D, Lf, info, pmin);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int prec(cudaStream_t st, const Layout &L, const int *list, int cnt, int mmax, const double *Lf, const double *D,
         double *x) {
    if (cnt <= 0) return BGPU_OK;
    const size_t smem = (size_t)std::max(mmax, 1) * sizeof(double);
    if (smem > 200 * 1024) return BGPU_ERR_TOOBIG;
    BGPU_ATTR_ONCE(BGPU_CHECK(cudaFuncSetAttribute(prec_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   200 * 1024)));
    prec_kernel<<<cnt, 256, smem, st>>>(list, L.m, L.moff, L.coff, Lf, D, x);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int symv(cudaStream_t st, const Layout &L, const int2 *items, int cnt, const double *M, const double *x, double *y) {
    if (cnt <= 0) return BGPU_OK;
    symv_kernel<<<cnt, 256, 0, st>>>(items, L.m, L.moff, L.coff, M, x, y);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int aop_packed(cudaStream_t st, const Layout &L, const int2 *items, int cnt, int nmax, const double *P,
               const double *Dc, double *y) {
    if (cnt <= 0) return BGPU_OK;
    aop_packed_kernel<<<cnt, 256, (size_t)nmax * (nmax + 1) / 2 * sizeof(double), st>>>(items, L.n, L.m, L.boff, L.coff,
                                                                                       L.poff, P, Dc, y);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int atop_packed(cudaStream_t st, const Layout &L, const int2 *items, int cnt, const double *P, const double *y,
                double alpha, double beta, double *Fc) {
    if (cnt <= 0) return BGPU_OK;
    atop_packed_kernel<<<cnt, 256, 0, st>>>(items, L.n, L.m, L.boff, L.coff, L.poff, P, y, alpha, beta, Fc);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int seg_dots(cudaStream_t st, int B, const long long *off, int nq, const double *const *a, const double *const *b,
             double *out) {
    if (B <= 0) return BGPU_OK;
    if (nq <= 0 || nq > DQ) return BGPU_ERR_ARG;
    seg_dots_kernel<<<B, 256, 0, st>>>(off, nq, a, b, out);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

}  // namespace lockstep
