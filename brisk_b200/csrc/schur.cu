// Schur complement assembly and the constraint operators A(.) and A'(.).
//
// Row-product route (the reference's route 1, schur_sdp_id, solver.c:2416-2625 / 2670-2960):
// for each constraint a of a block, G_a = X A_a Z^-1 and M_ba = <A_b, G_a> for every b >= a.
// B200 form, per chunk of K consecutive constraints a0..a0+K-1:
//   1. tprod:  T[(q*K + t), k] = (Zi A_a)[q, k]          (a = a0 + t; sparse A_a, dense Zi)
//   2. GEMM:   G[(q*K + t), p] = sum_k T[(q*K+t), k] X[k, p]  = G_a[p, q]
//              one DMMA GEMM of (n K) x n x n, X shared by the whole chunk (L2-resident)
//   3. gather: M[a, b] = sum_{(p,q) in A_b} A_b[p,q] G_a[p,q] for the K constraints of the chunk
//              at once: G is stored (p, q, t) with t fastest, so an entry of A_b reads K
//              contiguous values (one coalesced line for the warp) instead of K scattered ones.
// Because every A_b is symmetric, sum A_b[p,q] G_a[p,q] = sum A_b[p,q] G_a[q,p]; the gather
// indexes G by the entry's column-major position pos = p + q n directly.
// M is written in full (both triangles): the symmetric product of the FP64 residual, the
// equilibration and the factor copies read it without a transpose.
#include "common.cuh"
#include "kernels.h"
#include "tf32x3.h"

namespace {
constexpr int TP_Q = 128, TP_K = 32, TP_LD = TP_K + 1;   // CTA tile: 128 rows q x 32 columns k

// T[(q K + t) ldt + k] = sum_{p'} Zi[q, p'] A_a[p', k]  (a = a0 + t): column k of Zi A_a is the
// combination of the Zi columns p' that column k of A_a holds (Zi is symmetric: Zi[q, p'] =
// Zi[q + p' n]).  Warp w owns columns k0 + w, k0 + w + 8, ...; a lane owns rows q0 + lane + 32 u.
// The column's entries come from the per-constraint column pointers ccol, so no entry is read
// by a warp that does not use it and the sums stay in registers in a fixed order.
template <typename OutT>
__global__ void __launch_bounds__(256) tprod_kernel(int n, int ldt, int K, int a0, int ncon,
                                                   const long long *__restrict__ cptr, const int *__restrict__ ccol,
                                                   const int *__restrict__ cpos, const double *__restrict__ cval,
                                                   const double *__restrict__ Zi, OutT *__restrict__ T,
                                                   OutT *__restrict__ Tlo) {
    __shared__ double tile[TP_Q * TP_LD];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int q0 = blockIdx.x * TP_Q, k0 = blockIdx.y * TP_K, t = blockIdx.z;
    const int a = a0 + t;
    for (int kk = warp; kk < TP_K; kk += 8) {
        const int k = k0 + kk;
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        if (a < ncon && k < n) {
            const long long base = cptr[a];
            const int *cc = ccol + (long long)a * (n + 1);
            const long long e0 = base + cc[k], e1 = base + cc[k + 1];
            for (long long e = e0; e < e1; e++) {
                const int pp = cpos[e] - k * n;   // the row p' of the entry (p', k)
                const double v = cval[e];
                const double *z = Zi + (long long)pp * n + q0 + lane;
#pragma unroll
                for (int u = 0; u < 4; u++)
                    if (q0 + lane + 32 * u < n) acc[u] += v * z[32 * u];
            }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) tile[(lane + 32 * u) * TP_LD + kk] = acc[u];
    }
    __syncthreads();
    // rows (q, t) of T, k contiguous: a warp writes one row of 32 values per step
    const int kw = min(TP_K, n - k0);
    for (int r = warp; r < TP_Q; r += 8) {
        const int q = q0 + r;
        if (q >= n || lane >= kw) continue;
        const double v = tile[r * TP_LD + lane];
        const long long o = ((long long)q * K + t) * ldt + k0 + lane;
        if (sizeof(OutT) == 8) {
            T[o] = (OutT)v;
        } else {
            const float hi_ = tf32_round((float)v);
            T[o] = (OutT)hi_;
            Tlo[o] = (OutT)tf32_round((float)(v - (double)hi_));
        }
    }
}

// One CTA of GW warps per constraint b (b >= a0): warp w sums a fixed slice of b's entries
// with LPG lanes per entry group, each lane holding K / LPG of the chunk's K columns; the slices
// are added in warp order (a fixed order: the same bits on every run).
constexpr int GW = 8;
template <int K, typename GT>
__global__ void __launch_bounds__(GW * 32) gather_kernel(int a0, int ncon, int m, const int *__restrict__ con,
                                                        const long long *__restrict__ cptr, const int *__restrict__ cpos,
                                                        const double *__restrict__ cval, const GT *__restrict__ G,
                                                        double *M) {
    constexpr int LPG = K < 32 ? K : 32;       // lanes per entry group
    constexpr int GPW = 32 / LPG;              // entry groups per warp
    constexpr int PER = K / LPG;               // columns per lane
    __shared__ double part[GW][K];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int b = a0 + blockIdx.x;
    if (b >= ncon) return;
    const int sub = lane / LPG, l = lane % LPG;
    double acc[PER], acc2[PER];
#pragma unroll
    for (int u = 0; u < PER; u++) acc[u] = acc2[u] = 0.0;
    const long long s0 = cptr[b], e0 = cptr[b + 1];
    const long long len = e0 - s0, per_w = (len + GW - 1) / GW;
    const long long s = s0 + warp * per_w, e = min(e0, s + per_w);
    long long base = s;
    for (; base + 32 <= e; base += 32) {
        const int pos = cpos[base + lane];
        const double v = cval[base + lane];
        const GT *gp = G + l;
#pragma unroll
        for (int j = 0; j < 32; j += GPW) {
            const int pj = __shfl_sync(0xffffffffu, pos, j + sub);
            const double vj = __shfl_sync(0xffffffffu, v, j + sub);
            const GT *g = gp + (long long)pj * K;
            if ((j / GPW) & 1) {
#pragma unroll
                for (int u = 0; u < PER; u++) acc2[u] += vj * (double)g[u * LPG];
            } else {
#pragma unroll
                for (int u = 0; u < PER; u++) acc[u] += vj * (double)g[u * LPG];
            }
        }
    }
    if (base < e) {   // the ragged last group of the slice
        const long long my = base + lane;
        int pos = 0;
        double v = 0.0;
        if (my < e) { pos = cpos[my]; v = cval[my]; }
        const int cnt = (int)(e - base);
        for (int j = 0; j < cnt; j += GPW) {   // uniform trip count: every lane shuffles together
            const int jj = j + sub;
            const int src = jj < cnt ? jj : 0;
            const int pj = __shfl_sync(0xffffffffu, pos, src);
            const double vj = __shfl_sync(0xffffffffu, v, src);
            if (jj < cnt) {
                const GT *g = G + (long long)pj * K + l;
#pragma unroll
                for (int u = 0; u < PER; u++) acc[u] += vj * (double)g[u * LPG];
            }
        }
    }
#pragma unroll
    for (int u = 0; u < PER; u++) {
        acc[u] += acc2[u];
#pragma unroll
        for (int o = LPG; o < 32; o <<= 1) acc[u] += __shfl_xor_sync(0xffffffffu, acc[u], o);
    }
    if (sub == 0)
#pragma unroll
        for (int u = 0; u < PER; u++) part[warp][l + u * LPG] = acc[u];
    __syncthreads();
    if (threadIdx.x < K) {
        const int t = threadIdx.x;
        double v = 0.0;
#pragma unroll
        for (int w = 0; w < GW; w++) v += part[w][t];
        const int a = a0 + t;
        if (a < ncon && a <= b) {
            const int ca = con[a], cb = con[b];
            M[(long long)ca + (long long)cb * m] += v;
            if (ca != cb) M[(long long)cb + (long long)ca * m] += v;
        }
    }
}

template <typename GT>
int gather_launch(cudaStream_t st, int K, int a0, int ncon, int m, const DevBlock &B, const GT *G, double *M) {
    const int nb = ncon - a0;
    if (nb <= 0) return BGPU_OK;
    dim3 grid(nb);
    switch (K) {
        case 8: gather_kernel<8, GT><<<grid, GW * 32, 0, st>>>(a0, ncon, m, B.con, B.cptr, B.cpos, B.cval, G, M); break;
        case 16: gather_kernel<16, GT><<<grid, GW * 32, 0, st>>>(a0, ncon, m, B.con, B.cptr, B.cpos, B.cval, G, M); break;
        case 32: gather_kernel<32, GT><<<grid, GW * 32, 0, st>>>(a0, ncon, m, B.con, B.cptr, B.cpos, B.cval, G, M); break;
        case 64: gather_kernel<64, GT><<<grid, GW * 32, 0, st>>>(a0, ncon, m, B.con, B.cptr, B.cpos, B.cval, G, M); break;
        default: return BGPU_ERR_ARG;
    }
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

// hi/lo tf32 parts of a column-major n x n double matrix into rows of stride ld (ld >= n)
__global__ void split2d_kernel(int n, const double *__restrict__ X, int ld, float *__restrict__ hi, float *__restrict__ lo) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= ld) return;
    const double v = i < n ? X[i + (long long)j * n] : 0.0;
    const float h = tf32_round((float)v);
    hi[i + (long long)j * ld] = h;
    lo[i + (long long)j * ld] = tf32_round((float)(v - (double)h));
}

__global__ void aop_kernel(int ncon, const int *__restrict__ con, const long long *__restrict__ cptr,
                           const int *__restrict__ cpos, const double *__restrict__ cval, const double *__restrict__ D,
                           double alpha, double beta, double *out) {
    const int t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (t >= ncon) return;
    double s = 0.0;
    for (long long e = cptr[t] + lane; e < cptr[t + 1]; e += 32) s += cval[e] * D[cpos[e]];
    s = warp_sum(s);
    if (lane == 0) {
        const int c = con[t];
        out[c] = (beta == 0.0) ? alpha * s : alpha * s + beta * out[c];
    }
}

__global__ void atop_kernel(long long npos, const long long *__restrict__ pptr, const int *__restrict__ pcon,
                            const double *__restrict__ pval, const double *__restrict__ y, double alpha, double beta,
                            double *F) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npos) return;
    double s = 0.0;
    for (long long e = pptr[p]; e < pptr[p + 1]; e++) s += pval[e] * y[pcon[e]];
    F[p] = (beta == 0.0) ? alpha * s : alpha * s + beta * F[p];
}
}  // namespace

namespace {
__global__ void colptr_kernel(int n, int ncon, const long long *__restrict__ cptr, const int *__restrict__ cpos,
                              int *__restrict__ ccol) {
    const int t = blockIdx.x;
    if (t >= ncon) return;
    const long long s = cptr[t], e = cptr[t + 1];
    for (int k = threadIdx.x; k <= n; k += blockDim.x) {
        const long long key = (long long)k * n;   // first position of column k
        long long L = s, R = e;
        while (L < R) {
            const long long mid = (L + R) >> 1;
            if ((long long)cpos[mid] < key) L = mid + 1; else R = mid;
        }
        ccol[(long long)t * (n + 1) + k] = (int)(L - s);
    }
}
}  // namespace

int schur_colptr(cudaStream_t st, const DevBlock &B) {
    if (B.ncon <= 0) return BGPU_OK;
    colptr_kernel<<<B.ncon, 128, 0, st>>>(B.n, B.ncon, B.cptr, B.cpos, B.ccol);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int aop_f64(cudaStream_t st, const DevBlock &B, const double *D, double alpha, double beta, double *out) {
    if (B.ncon <= 0) return BGPU_OK;
    aop_kernel<<<ceil_div(B.ncon, 8), 256, 0, st>>>(B.ncon, B.con, B.cptr, B.cpos, B.cval, D, alpha, beta, out);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int atop_f64(cudaStream_t st, const DevBlock &B, const double *y, double alpha, double beta, double *F) {
    const long long npos = (long long)B.n * B.n;
    atop_kernel<<<ceil_div(npos, 256), 256, 0, st>>>(npos, B.pptr, B.pcon, B.pval, y, alpha, beta, F);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int schur_chunk_default(int n, int precision) {
    // the chunk's G (n^2 K values) should stay L2-resident during the gather (<= 64 MB of the
    // 126 MB L2); a wider chunk reads each constraint's entry list fewer times
    const double gbytes = (double)n * n * (precision == 0 ? 8.0 : 4.0);
    int K = 64;
    while (K > 8 && gbytes * K > 64e6) K >>= 1;
    return K;
}

// tf32 operand rows padded to a multiple of 4 floats: the tensor maps need 16-byte strides
static inline int tf32_ld(int n) { return (n + 3) / 4 * 4; }

size_t schur_ws_bytes(int n, int chunk, int precision) {
    const size_t nn = (size_t)n * n * chunk;
    if (precision == 0) return 2 * nn * sizeof(double);            // T, G
    const size_t ld = tf32_ld(n);
    // T hi/lo (n K rows of ld), G (float, n K x n), X hi/lo (n rows of ld), plus 256 B alignment slack each
    return (2 * (size_t)n * chunk * ld + nn + 2 * (size_t)n * ld) * sizeof(float) + 5 * 256;
}

int schur_assemble(cudaStream_t st, const DevBlock &B, const double *X, const double *Zi, double *M, int m,
                   int precision, int chunk, void *ws, size_t ws_bytes) {
    const int n = B.n, K = chunk;
    if (B.ncon <= 0) return BGPU_OK;
    if (K != 8 && K != 16 && K != 32 && K != 64) return BGPU_ERR_ARG;
    if (!B.ccol) return BGPU_ERR_ARG;
    if (ws_bytes < schur_ws_bytes(n, K, precision)) return BGPU_ERR_ARG;
    const size_t nnK = (size_t)n * n * K;
    dim3 tgrid(ceil_div(n, TP_Q), ceil_div(n, TP_K), K);
    if (precision == 0) {
        double *T = (double *)ws, *G = T + nnK;
        for (int a0 = 0; a0 < B.ncon; a0 += K) {
            tprod_kernel<double><<<tgrid, 256, 0, st>>>(n, n, K, a0, B.ncon, B.cptr, B.ccol, B.cpos, B.cval, Zi, T, nullptr);
            BGPU_LAUNCH_CHECK();
            int rc = gemm_f64(st, 1, 1, n * K, n, n, 1.0, T, n, 0, X, n, 0, 0.0, G, (long long)n * K, 0, 1, 0);
            if (rc) return rc;
            rc = gather_launch<double>(st, K, a0, B.ncon, m, B, G, M);
            if (rc) return rc;
        }
        return BGPU_OK;
    }
    // 3xTF32: T and X split into tf32 hi + lo parts; G accumulated in FP32 on the tensor cores
    const int ld = tf32_ld(n);
    auto carve = [&](size_t count) {   // 256-byte aligned sub-buffers of the workspace
        static_assert(sizeof(float) == 4, "");
        uintptr_t p = ((uintptr_t)ws + 255) & ~(uintptr_t)255;
        float *r = (float *)p;
        ws = (void *)(p + count * sizeof(float));
        return r;
    };
    float *Th = carve((size_t)n * K * ld), *Tl = carve((size_t)n * K * ld), *G = carve(nnK);
    float *Xh = carve((size_t)n * ld), *Xl = carve((size_t)n * ld);
    split2d_kernel<<<dim3(ceil_div(ld, 256), n), 256, 0, st>>>(n, X, ld, Xh, Xl);
    BGPU_LAUNCH_CHECK();
    for (int a0 = 0; a0 < B.ncon; a0 += K) {
        tprod_kernel<float><<<tgrid, 256, 0, st>>>(n, ld, K, a0, B.ncon, B.cptr, B.ccol, B.cpos, B.cval, Zi, Th, Tl);
        BGPU_LAUNCH_CHECK();
        int rc = gemm_tf32x3(st, n * K, n, n, Th, Tl, ld, Xh, Xl, ld, G, (long long)n * K);
        if (rc) return rc;
        rc = gather_launch<float>(st, K, a0, B.ncon, m, B, G, M);
        if (rc) return rc;
    }
    return BGPU_OK;
}

// ---- the dense route -------------------------------------------------------------------------
namespace {
__global__ void densify_kernel(int n, int ncon, const long long *__restrict__ cptr, const int *__restrict__ cpos,
                               const double *__restrict__ cval, double *__restrict__ Ad) {
    const int t = blockIdx.x;
    if (t >= ncon) return;
    double *row = Ad + (long long)t * n * n;
    for (long long e = cptr[t] + threadIdx.x; e < cptr[t + 1]; e += blockDim.x) row[cpos[e]] = cval[e];
}
__global__ void f2d_kernel(long long count, const float *__restrict__ src, double *__restrict__ dst) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) dst[i] = (double)src[i];
}
// M[con[b], con[a0 + j]] += Mloc[b + j ncon] for every local b and the chunk's columns j
__global__ void scatter_cols_kernel(int ncon, int a0, int kw, int m, const int *__restrict__ con,
                                    const double *__restrict__ Mloc, double *M) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (b >= ncon || j >= kw) return;
    M[(long long)con[b] + (long long)con[a0 + j] * m] += Mloc[b + (long long)j * ncon];
}
}  // namespace

size_t schur_dense_ws_bytes(int n, int ncon, int chunk, int precision) {
    size_t b = schur_ws_bytes(n, chunk, precision) + (size_t)ncon * chunk * sizeof(double) + 256;
    if (precision == 1) b += (size_t)n * n * chunk * sizeof(double) + 256;
    return b;
}

int schur_densify(cudaStream_t st, const DevBlock &B) {
    if (B.ncon <= 0) return BGPU_OK;
    BGPU_CHECK(cudaMemsetAsync(B.Ad, 0, sizeof(double) * (size_t)B.ncon * B.n * B.n, st));
    densify_kernel<<<B.ncon, 256, 0, st>>>(B.n, B.ncon, B.cptr, B.cpos, B.cval, B.Ad);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int schur_assemble_dense(cudaStream_t st, const DevBlock &B, const double *X, const double *Zi, double *M, int m,
                         int precision, int chunk, void *ws, size_t ws_bytes) {
    const int n = B.n, K = chunk, ncon = B.ncon;
    if (ncon <= 0) return BGPU_OK;
    if (!B.Ad || !B.ccol) return BGPU_ERR_ARG;
    if (ws_bytes < schur_dense_ws_bytes(n, ncon, K, precision)) return BGPU_ERR_ARG;
    const size_t nnK = (size_t)n * n * K;
    const size_t base_bytes = schur_ws_bytes(n, K, precision);
    uintptr_t tail = ((uintptr_t)ws + base_bytes + 255) & ~(uintptr_t)255;
    double *Mloc = (double *)tail;
    double *G64 = nullptr;
    if (precision == 1) G64 = (double *)((((uintptr_t)(Mloc + (size_t)ncon * K)) + 255) & ~(uintptr_t)255);
    dim3 tgrid(ceil_div(n, TP_Q), ceil_div(n, TP_K), K);
    double *T64 = (double *)ws, *Gd = T64 + nnK;   // FP64 layout of the workspace
    float *Th = nullptr, *Tl = nullptr, *Gf = nullptr, *Xh = nullptr, *Xl = nullptr;
    const int ld = tf32_ld(n);
    if (precision == 1) {
        void *w = ws;
        auto carve = [&](size_t count) {
            uintptr_t p = ((uintptr_t)w + 255) & ~(uintptr_t)255;
            w = (void *)(p + count * sizeof(float));
            return (float *)p;
        };
        Th = carve((size_t)n * K * ld);
        Tl = carve((size_t)n * K * ld);
        Gf = carve(nnK);
        Xh = carve((size_t)n * ld);
        Xl = carve((size_t)n * ld);
        split2d_kernel<<<dim3(ceil_div(ld, 256), n), 256, 0, st>>>(n, X, ld, Xh, Xl);
        BGPU_LAUNCH_CHECK();
    }
    for (int a0 = 0; a0 < ncon; a0 += K) {
        const int kw = min(K, ncon - a0);
        const double *G = nullptr;
        if (precision == 0) {
            tprod_kernel<double><<<tgrid, 256, 0, st>>>(n, n, K, a0, ncon, B.cptr, B.ccol, B.cpos, B.cval, Zi, T64, nullptr);
            BGPU_LAUNCH_CHECK();
            int rc = gemm_f64(st, 1, 1, n * K, n, n, 1.0, T64, n, 0, X, n, 0, 0.0, Gd, (long long)n * K, 0, 1, 0);
            if (rc) return rc;
            G = Gd;
        } else {
            tprod_kernel<float><<<tgrid, 256, 0, st>>>(n, ld, K, a0, ncon, B.cptr, B.ccol, B.cpos, B.cval, Zi, Th, Tl);
            BGPU_LAUNCH_CHECK();
            int rc = gemm_tf32x3(st, n * K, n, n, Th, Tl, ld, Xh, Xl, ld, Gf, (long long)n * K);
            if (rc) return rc;
            f2d_kernel<<<ceil_div((long long)nnK, 256), 256, 0, st>>>((long long)nnK, Gf, G64);
            BGPU_LAUNCH_CHECK();
            G = G64;
        }
        // Mloc (ncon x K) = Ad (ncon x n^2, K-major rows) * G (n^2 x K, column index fastest)
        int rc = gemm_f64(st, 1, 0, ncon, kw, n * n, 1.0, B.Ad, (long long)n * n, 0, G, K, 0, 0.0, Mloc, ncon, 0, 1, 0);
        if (rc) return rc;
        scatter_cols_kernel<<<dim3(ceil_div(ncon, 256), kw), 256, 0, st>>>(ncon, a0, kw, m, B.con, Mloc, M);
        BGPU_LAUNCH_CHECK();
    }
    return BGPU_OK;
}
