// The step-level C ABI (include/bgpu.h): thin wrappers over the kernel launchers.
#include "../../include/bgpu.h"
#include "common.cuh"
#include "kernels.h"
#include "tf32x3.h"
#include "small.h"
#include "sparse.h"
#include "nt.h"

long long g_bgpu_launches = 0;
static cudaStream_t S(void *s) { return (cudaStream_t)s; }
// the assembly's precision codes: 0 FP64, 1 3xTF32, 2 Ozaki (8 slices), (S << 8) | 2 Ozaki with S
static bool valid_precision(int p) {
    if (p == 0 || p == 1 || p == 2) return true;
    const int sl = (p >> 8) & 0xf;
    return (p & 0xff) == 2 && (p >> 12) == 0 && sl >= 4 && sl <= 8;
}

static std::atomic<unsigned> g_wait_limit{BGPU_SPIN_LIMIT};
static std::atomic<int> g_trsv_hold{-1};
unsigned wait_limit() { return g_wait_limit.load(std::memory_order_relaxed); }
int trsv_hold_row() { return g_trsv_hold.load(std::memory_order_relaxed); }

extern "C" {

BGPU_API int bgpu_sync(void *stream) {
    BGPU_CHECK(cudaStreamSynchronize(S(stream)));
    return BGPU_OK;
}
BGPU_API const char *bgpu_version(void) { return "brisk_b200 1.7-b200 sm_100a"; }
BGPU_API long long bgpu_launch_count(void) { return __atomic_load_n(&g_bgpu_launches, __ATOMIC_RELAXED); }
BGPU_API void bgpu_set_wait_limit(unsigned polls) { g_wait_limit.store(polls ? polls : BGPU_SPIN_LIMIT); }
BGPU_API void bgpu_test_hold_trsv_row(int r) { g_trsv_hold.store(r < 0 ? -1 : r); }

BGPU_API size_t bgpu_schur_ws_bytes(int n, int chunk, int precision) {
    if (chunk <= 0) chunk = schur_chunk_default(n, precision);
    return schur_ws_bytes(n, chunk, precision);
}
BGPU_API int bgpu_schur_chunk_default(int n, int precision) { return schur_chunk_default(n, precision); }

BGPU_API size_t bgpu_nt_ws_bytes(int n) {
    if (n <= 0) return 0;
    if (n <= nt::SMALL_NMAX) return 256;
    return 2 * (size_t)n * n * sizeof(double) + 256;
}

BGPU_API int bgpu_nt_scaling(int n, const double *d_LX, const double *d_LZ, double *d_G, double *d_lam,
                             double *d_W, void *d_ws, size_t ws_bytes, int *sweeps, void *stream) {
    if (sweeps) *sweeps = 0;
    if (n <= 0 || !d_LX || !d_LZ || !d_G || !d_lam || !d_W || !d_ws || ws_bytes < bgpu_nt_ws_bytes(n))
        return BGPU_ERR_ARG;
    cudaStream_t st = S(stream);
    int info = 0;
    if (n <= nt::SMALL_NMAX) {
        // the one-CTA form over a table of one block: 5 pointers, then n and info
        struct Tab {
            const double *LX, *LZ;
            double *G, *lam, *W;
            int n, info;
        } h{d_LX, d_LZ, d_G, d_lam, d_W, n, 0};
        Tab *t = (Tab *)d_ws;
        BGPU_CHECK(cudaMemcpyAsync(t, &h, sizeof(Tab), cudaMemcpyHostToDevice, st));
        int rc = nt::scaling_small(st, 1, &t->n, n, &t->LX, &t->LZ, &t->G, &t->lam, &t->W, &t->info);
        if (rc) return rc;
        BGPU_CHECK(cudaMemcpyAsync(&info, &t->info, sizeof(int), cudaMemcpyDeviceToHost, st));
        BGPU_CHECK(cudaStreamSynchronize(st));
        return info == 0 ? BGPU_OK : (info == 2 ? BGPU_ERR_TIMEOUT : BGPU_ERR_NOTPD);
    }
    double *Mb = (double *)d_ws, *Lz = Mb + (size_t)n * n;
    int *flag = (int *)(Lz + (size_t)n * n), *dinfo = flag + 1;
    int rc = nt::tril(st, n, d_LX, d_G);
    if (!rc) rc = nt::tril(st, n, d_LZ, Lz);
    if (!rc) rc = gemm_f64(st, 1, 1, n, n, n, 1.0, Lz, n, 0, d_G, n, 0, 0.0, Mb, n, 0, 1, 0);   // L_Z' L_X
    if (rc) return rc;
    int hflag = 0, sw = 0;
    rc = nt::jacobi(st, n, Mb, d_G, flag, &hflag, &sw);
    if (rc) return rc;
    if (sweeps) *sweeps = sw;
    if (sw < 0) return BGPU_ERR_TIMEOUT;
    BGPU_CHECK(cudaMemsetAsync(dinfo, 0, sizeof(int), st));
    rc = nt::finish(st, n, Mb, d_G, d_lam, dinfo);
    if (!rc) rc = gemm_f64(st, 0, 0, n, n, n, 1.0, d_G, n, 0, d_G, n, 0, 0.0, d_W, n, 0, 1, 0);   // G G'
    if (!rc) rc = symmetrize_f64(st, n, d_W, n);
    if (rc) return rc;
    BGPU_CHECK(cudaMemcpyAsync(&info, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st));
    BGPU_CHECK(cudaStreamSynchronize(st));
    return info ? BGPU_ERR_NOTPD : BGPU_OK;
}

BGPU_API size_t bgpu_ozaki_ws_bytes(int M, int N, int K) {
    if (M <= 0 || N <= 0 || K <= 0) return 0;
    return ozaki_operand_bytes(M, K, 8) + ozaki_operand_bytes(N, K, 8);
}

BGPU_API int bgpu_gemm_ozaki(int M, int N, int K, const double *d_A, int64_t lda, const double *d_B, int64_t ldb,
                             double *d_C, int64_t ldc, void *d_ws, size_t ws_bytes, void *stream) {
    return bgpu_gemm_ozaki_slices(8, M, N, K, d_A, lda, d_B, ldb, d_C, ldc, d_ws, ws_bytes, stream);
}

BGPU_API int bgpu_gemm_ozaki_slices(int slices, int M, int N, int K, const double *d_A, int64_t lda, const double *d_B,
                                    int64_t ldb, double *d_C, int64_t ldc, void *d_ws, size_t ws_bytes, void *stream) {
    if (slices < 4 || slices > 8) return BGPU_ERR_ARG;
    if (M <= 0 || N <= 0 || K <= 0 || lda < K || ldb < K || ldc < M || !d_A || !d_B || !d_C || !d_ws ||
        ws_bytes < bgpu_ozaki_ws_bytes(M, N, K))
        return BGPU_ERR_ARG;
    cudaStream_t st = S(stream);
    OzakiOperand a, b;
    uint8_t *wa = (uint8_t *)d_ws, *wb = wa + ozaki_operand_bytes(M, K, slices);
    int rc = ozaki_slice(st, M, K, d_A, lda, wa, &a, slices);
    if (!rc) rc = ozaki_slice(st, N, K, d_B, ldb, wb, &b, slices);
    if (!rc) rc = ozaki_gemm(st, a, b, d_C, ldc);
    if (rc) return rc;
    BGPU_CHECK(cudaStreamSynchronize(st));
    int bad = 0;
    if ((rc = ozaki_error_flag(&bad))) return rc;
    return bad ? BGPU_ERR_TIMEOUT : BGPU_OK;
}

BGPU_API int bgpu_schur_colptr(int n, int ncon, const long long *d_cptr, const int *d_cpos, int *d_ccol, void *stream) {
    DevBlock B;
    B.n = n;
    B.ncon = ncon;
    B.cptr = (long long *)d_cptr;
    B.cpos = (int *)d_cpos;
    B.ccol = d_ccol;
    return schur_colptr(S(stream), B);
}

BGPU_API int bgpu_schur_assemble(int n, int m, int ncon, const int *d_con, const long long *d_cptr,
                                 const int *d_ccol, const int *d_cpos, const double *d_cval, const double *d_X,
                                 const double *d_Zi, double *d_M, int precision, int chunk, void *d_ws,
                                 size_t ws_bytes, void *stream) {
    if (n <= 0 || m <= 0 || ncon < 0 || !valid_precision(precision)) return BGPU_ERR_ARG;
    if (chunk <= 0) chunk = schur_chunk_default(n, precision);
    DevBlock B;
    B.n = n;
    B.ncon = ncon;
    B.con = (int *)d_con;
    B.cptr = (long long *)d_cptr;
    B.ccol = (int *)d_ccol;
    B.cpos = (int *)d_cpos;
    B.cval = (double *)d_cval;
    return schur_assemble(S(stream), B, d_X, d_Zi, d_M, m, precision, chunk, d_ws, ws_bytes);
}

BGPU_API int bgpu_schur_upper(int n, int ncon, const long long *d_cptr, const int *d_cpos, const double *d_cval,
                              int *d_counts, long long *d_uptr, int *d_upos, double *d_uval, long long *nu,
                              void *stream) {
    if (n <= 0 || ncon < 0 || !d_uptr || !d_counts || !nu) return BGPU_ERR_ARG;
    DevBlock B;
    B.n = n;
    B.ncon = ncon;
    B.cptr = (long long *)d_cptr;
    B.cpos = (int *)d_cpos;
    B.cval = (double *)d_cval;
    B.uptr = d_uptr;
    B.upos = d_upos;
    B.uval = d_uval;
    *nu = 0;
    if (ncon == 0) return BGPU_OK;
    int rc = schur_upper_ptr(S(stream), B, d_counts);
    if (rc) return rc;
    BGPU_CHECK(cudaMemcpyAsync(nu, d_uptr + ncon, sizeof(long long), cudaMemcpyDeviceToHost, S(stream)));
    BGPU_CHECK(cudaStreamSynchronize(S(stream)));
    if (!d_upos || !d_uval) return BGPU_OK;
    return schur_upper(S(stream), B);
}

BGPU_API int bgpu_schur_assemble_sym(int n, int m, int ncon, const int *d_con, const long long *d_cptr,
                                     const int *d_ccol, const int *d_cpos, const double *d_cval,
                                     const long long *d_uptr, const int *d_upos, const double *d_uval,
                                     const double *d_X, const double *d_Zi, double *d_M, int precision, int chunk,
                                     void *d_ws, size_t ws_bytes, void *stream) {
    if (n <= 0 || m <= 0 || ncon < 0 || !valid_precision(precision)) return BGPU_ERR_ARG;
    if (ncon > 0 && (!d_uptr || !d_upos || !d_uval)) return BGPU_ERR_ARG;
    if (chunk <= 0) chunk = schur_chunk_default(n, precision);
    DevBlock B;
    B.n = n;
    B.ncon = ncon;
    B.con = (int *)d_con;
    B.cptr = (long long *)d_cptr;
    B.ccol = (int *)d_ccol;
    B.cpos = (int *)d_cpos;
    B.cval = (double *)d_cval;
    B.uptr = (long long *)d_uptr;
    B.upos = (int *)d_upos;
    B.uval = (double *)d_uval;
    return schur_assemble(S(stream), B, d_X, d_Zi, d_M, m, precision, chunk, d_ws, ws_bytes);
}

BGPU_API int bgpu_schur_gram(int n, int m, int ncon, const int *d_con, const long long *d_uptr, const int *d_upos,
                             const double *d_uval, double *d_M, void *d_ws, size_t ws_bytes, void *stream) {
    if (n <= 0 || m <= 0 || ncon < 0) return BGPU_ERR_ARG;
    DevBlock B;
    B.n = n;
    B.ncon = ncon;
    B.con = (int *)d_con;
    B.uptr = (long long *)d_uptr;
    B.upos = (int *)d_upos;
    B.uval = (double *)d_uval;
    return schur_assemble_gram(S(stream), B, d_M, m, d_ws, ws_bytes);
}

BGPU_API size_t bgpu_schur_dense_ws_bytes(int n, int ncon, int chunk, int precision) {
    if (chunk <= 0) chunk = schur_chunk_default(n, precision);
    return schur_dense_ws_bytes(n, ncon, chunk, precision);
}
BGPU_API int bgpu_schur_densify(int n, int ncon, const long long *d_cptr, const int *d_cpos, const double *d_cval,
                                double *d_Ad, void *stream) {
    DevBlock B;
    B.n = n;
    B.ncon = ncon;
    B.cptr = (long long *)d_cptr;
    B.cpos = (int *)d_cpos;
    B.cval = (double *)d_cval;
    B.Ad = d_Ad;
    return schur_densify(S(stream), B);
}
BGPU_API int bgpu_schur_assemble_dense(int n, int m, int ncon, const int *d_con, const long long *d_cptr,
                                       const int *d_ccol, const int *d_cpos, const double *d_cval, const double *d_Ad,
                                       const double *d_X, const double *d_Zi, double *d_M, int precision, int chunk,
                                       void *d_ws, size_t ws_bytes, void *stream) {
    if (n <= 0 || m <= 0 || ncon < 0 || (precision != 0 && precision != 1)) return BGPU_ERR_ARG;
    if (chunk <= 0) chunk = schur_chunk_default(n, precision);
    DevBlock B;
    B.n = n;
    B.ncon = ncon;
    B.con = (int *)d_con;
    B.cptr = (long long *)d_cptr;
    B.ccol = (int *)d_ccol;
    B.cpos = (int *)d_cpos;
    B.cval = (double *)d_cval;
    B.Ad = (double *)d_Ad;
    return schur_assemble_dense(S(stream), B, d_X, d_Zi, d_M, m, precision, chunk, d_ws, ws_bytes);
}

BGPU_API int bgpu_schur_lp(int m, int N, int nc, int64_t ne, const int *d_gcon, const int64_t *d_aptr,
                           const int *d_avar, const double *d_aval, const int64_t *d_vptr, const int *d_vcon,
                           const double *d_vval, const double *d_x, const double *d_zi, double *d_M, void *stream) {
    if (m <= 0 || N < 0 || nc < 0 || nc > m || ne < 0) return BGPU_ERR_ARG;
    LpGroupDev G;
    G.N = N;
    G.nc = nc;
    G.ne = ne;
    G.gcon = (int *)d_gcon;
    G.aptr = (long long *)d_aptr;
    G.avar = (int *)d_avar;
    G.aval = (double *)d_aval;
    G.vptr = (long long *)d_vptr;
    G.vcon = (int *)d_vcon;
    G.vval = (double *)d_vval;
    return schur_assemble_lp(S(stream), G, d_x, d_zi, d_M, m);
}

BGPU_API int bgpu_lowrank_factor(int n, int ncon, const int64_t *h_cptr, const int *h_cpos, const double *h_cval,
                                 int max_rank, int *off, double *W, double *sig) {
    if (n <= 0 || ncon < 0 || max_rank < 0 || !h_cptr || !h_cpos || !h_cval || !off) return BGPU_ERR_ARG;
    std::vector<int> o;
    std::vector<double> w, s;
    if (!lowrank_factor_block(n, ncon, (const long long *)h_cptr, h_cpos, h_cval, o, w, s, max_rank))
        return BGPU_ERR_UNSUPPORTED;
    const int R = o[ncon];
    std::copy(o.begin(), o.end(), off);
    if (W) std::copy(w.begin(), w.begin() + (size_t)n * R, W);
    if (sig) std::copy(s.begin(), s.begin() + R, sig);
    return R;
}

BGPU_API int bgpu_schur_lowrank(int n, int m, int ncon, const int *d_con, const int64_t *h_cptr, const int *h_cpos,
                                const double *h_cval, const double *d_X, const double *d_Zi, double *d_M, int *rank,
                                void *stream) {
    if (n <= 0 || m <= 0 || ncon < 0 || ncon > m || !h_cptr || !h_cpos || !h_cval || !rank) return BGPU_ERR_ARG;
    *rank = 0;
    std::vector<int> off;
    std::vector<double> W, sig;
    if (!lowrank_factor_block(n, ncon, (const long long *)h_cptr, h_cpos, h_cval, off, W, sig, 1 << 15))
        return BGPU_ERR_UNSUPPORTED;
    const int R = ncon > 0 ? off[ncon] : 0;
    *rank = R;
    if (R == 0) return BGPU_OK;
    cudaStream_t st = S(stream);
    LowRankDev L;
    L.n = n;
    L.ncon = ncon;
    L.R = R;
    const size_t bytes = sizeof(double) * ((size_t)2 * n * R + (size_t)2 * R * R + R) + sizeof(int) * (ncon + 1);
    unsigned char *buf = nullptr;
    BGPU_CHECK(cudaMalloc(&buf, bytes + 256));
    double *p = (double *)buf;
    L.W = p; p += (size_t)n * R;
    L.XW = p; p += (size_t)n * R;
    L.P = p; p += (size_t)R * R;
    L.Q = p; p += (size_t)R * R;
    L.sig = p; p += R;
    L.off = (int *)p;
    int rc = BGPU_OK;
    if (cudaMemcpyAsync(L.W, W.data(), sizeof(double) * (size_t)n * R, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(L.sig, sig.data(), sizeof(double) * R, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(L.off, off.data(), sizeof(int) * (ncon + 1), cudaMemcpyHostToDevice, st) != cudaSuccess)
        rc = BGPU_ERR_CUDA;
    if (!rc) rc = schur_assemble_lowrank(st, L, d_con, d_X, d_Zi, d_M, m);
    if (cudaStreamSynchronize(st) != cudaSuccess && !rc) rc = BGPU_ERR_CUDA;
    cudaFree(buf);
    return rc;
}

BGPU_API int bgpu_potrf(int n, double *d_A, int lda, double *d_dinv, int *d_info, double *d_pmin, void *stream) {
    if (n <= 0 || lda < n) return BGPU_ERR_ARG;
    return potrf_f64(S(stream), n, d_A, lda, d_dinv, d_info, d_pmin);
}
BGPU_API int bgpu_potrf_f32(int n, float *d_A, int lda, float *d_dinv, int *d_info, double *d_pmin, void *stream) {
    if (n <= 0 || lda < n) return BGPU_ERR_ARG;
    return potrf_f32(S(stream), n, d_A, lda, d_dinv, d_info, d_pmin);
}
BGPU_API int bgpu_trsv(int n, const double *d_L, int lda, const double *d_dinv, double *d_x, int trans,
                       int *d_flags, int epoch, int *d_err, void *stream) {
    if (n <= 0 || lda < n) return BGPU_ERR_ARG;
    return trsv_f64(S(stream), n, d_L, lda, d_dinv, d_x, trans, d_flags, epoch, d_err);
}
BGPU_API int bgpu_trsv_f32(int n, const float *d_L, int lda, const float *d_dinv, float *d_x, int trans,
                           int *d_flags, int epoch, int *d_err, void *stream) {
    if (n <= 0 || lda < n) return BGPU_ERR_ARG;
    return trsv_f32(S(stream), n, d_L, lda, d_dinv, d_x, trans, d_flags, epoch, d_err);
}
BGPU_API int bgpu_trtri(int n, const double *d_L, int lda, const double *d_dinv, double *d_Linv, int ldi,
                        void *stream) {
    if (n <= 0 || lda < n || ldi < n) return BGPU_ERR_ARG;
    return trtri_f64(S(stream), n, d_L, lda, d_dinv, d_Linv, ldi);
}
BGPU_API int bgpu_dgemm(int a_kmajor, int b_kmajor, int M, int N, int K, double alpha, const double *d_A,
                        int64_t lda, const double *d_B, int64_t ldb, double beta, double *d_C, int64_t ldc,
                        int lower, void *stream) {
    if (M < 0 || N < 0 || K < 0) return BGPU_ERR_ARG;
    return gemm_f64(S(stream), a_kmajor, b_kmajor, M, N, K, alpha, d_A, lda, 0, d_B, ldb, 0, beta, d_C, ldc, 0, 1,
                    lower);
}
BGPU_API int bgpu_gemm_tf32x3(int M, int N, int K, const float *d_Ah, const float *d_Al, int64_t lda,
                              const float *d_Bh, const float *d_Bl, int64_t ldb, float *d_G, int64_t ldg,
                              void *stream) {
    if (M < 0 || N < 0 || K < 0) return BGPU_ERR_ARG;
    return gemm_tf32x3(S(stream), M, N, K, d_Ah, d_Al, lda, d_Bh, d_Bl, ldb, d_G, ldg);
}
BGPU_API int bgpu_split_tf32(int64_t n, const double *d_x, float *d_hi, float *d_lo, void *stream) {
    return split_tf32(S(stream), n, d_x, d_hi, d_lo);
}
BGPU_API int bgpu_symv(int n, double alpha, const double *d_M, int ldm, const double *d_x, double beta,
                       double *d_y, void *stream) {
    if (n <= 0 || ldm < n) return BGPU_ERR_ARG;
    return symv_full_f64(S(stream), n, alpha, d_M, ldm, d_x, beta, d_y);
}
BGPU_API int bgpu_aop(int n, int ncon, const int *d_con, const long long *d_cptr, const int *d_cpos,
                      const double *d_cval, const double *d_D, double alpha, double beta, double *d_out,
                      void *stream) {
    DevBlock B;
    B.n = n;
    B.ncon = ncon;
    B.con = (int *)d_con;
    B.cptr = (long long *)d_cptr;
    B.cpos = (int *)d_cpos;
    B.cval = (double *)d_cval;
    return aop_f64(S(stream), B, d_D, alpha, beta, d_out);
}

BGPU_API int bgpu_small_chol_inv(int nb, const int *d_n, double *const *d_A, double *const *d_L,
                                 double *const *d_Li, int *d_info, void *stream) {
    if (nb < 0) return BGPU_ERR_ARG;
    return small_chol_inv(S(stream), nb, d_n, d_A, d_L, d_Li, d_info);
}
BGPU_API int bgpu_small_lammin(int nb, const int *d_n, const double *const *d_Li, const double *const *d_D,
                               double *d_lam, void *stream) {
    if (nb < 0) return BGPU_ERR_ARG;
    return small_lammin(S(stream), nb, d_n, d_Li, d_D, d_lam);
}
BGPU_API int bgpu_small_gemm(int nb, const int *d_n, int ta, int tb, double alpha, const double *const *d_A,
                             const double *const *d_B, double beta, double *const *d_C, int sym, void *stream) {
    if (nb < 0) return BGPU_ERR_ARG;
    return small_gemm(S(stream), nb, d_n, ta, tb, alpha, d_A, d_B, beta, d_C, sym);
}

struct bgpu_schol {
    schol::Analysis A;
    schol::Factor F;
    void *buf = nullptr;
    bool bound = false;
};

BGPU_API bgpu_schol *bgpu_schol_analyze(int m, int ncliques, const int64_t *clq_ptr, const int *clq_idx, int *rc) {
    int code = BGPU_OK;
    bgpu_schol *h = nullptr;
    if (m < 0 || ncliques < 0 || (ncliques > 0 && (!clq_ptr || !clq_idx))) code = BGPU_ERR_ARG;
    if (!code) {
        std::vector<std::vector<int>> cl(ncliques);
        for (int c = 0; c < ncliques; c++) {
            if (clq_ptr[c + 1] < clq_ptr[c]) { code = BGPU_ERR_ARG; break; }
            cl[c].assign(clq_idx + clq_ptr[c], clq_idx + clq_ptr[c + 1]);
        }
        if (!code) {
            h = new (std::nothrow) bgpu_schol;
            if (!h) code = BGPU_ERR_NOMEM;
            else if (schol::analyze(m, cl, h->A)) { delete h; h = nullptr; code = BGPU_ERR_ARG; }
        }
    }
    if (rc) *rc = code;
    return h;
}

BGPU_API void bgpu_schol_set_delta(double delta) { schol::g_mmd_delta = delta < 0 ? 0 : delta; }

BGPU_API int bgpu_schol_info(const bgpu_schol *h, double *out8) {
    if (!h || !out8) return BGPU_ERR_ARG;
    out8[0] = h->A.nsup;
    out8[1] = h->A.nnz;
    out8[2] = h->A.flops;
    out8[3] = h->A.fmax;
    out8[4] = h->A.lvptr.empty() ? 0 : (double)(h->A.lvptr.size() - 1);
    out8[5] = (double)h->A.pattern;
    out8[6] = h->A.m;
    out8[7] = (double)schol::factor_bytes(h->A);
    return BGPU_OK;
}

BGPU_API int bgpu_schol_perm(const bgpu_schol *h, int *perm) {
    if (!h || !perm) return BGPU_ERR_ARG;
    std::copy(h->A.perm.begin(), h->A.perm.end(), perm);
    return BGPU_OK;
}

BGPU_API int bgpu_schol_supernodes(const bgpu_schol *h, int *sfirst, int *parent, int64_t *rptr, int *rows) {
    if (!h) return BGPU_ERR_ARG;
    const auto &A = h->A;
    if (sfirst) std::copy(A.sfirst.begin(), A.sfirst.end(), sfirst);
    if (parent) std::copy(A.parent.begin(), A.parent.end(), parent);
    if (rptr) for (size_t s = 0; s < A.rptr.size(); s++) rptr[s] = A.rptr[s];
    if (rows) std::copy(A.rows.begin(), A.rows.end(), rows);
    return BGPU_OK;
}

static int schol_factor_any(bgpu_schol *h, const double *d_M, int64_t ldm, const double *d_D, double reg, int *info,
                            double *pmin, void *stream, bool fp32) {
    if (!h || !d_M || !d_D || ldm < h->A.m) return BGPU_ERR_ARG;
    if (!h->bound) {
        const size_t b = schol::factor_bytes(h->A);
        if (cudaMalloc(&h->buf, b) != cudaSuccess) { h->buf = nullptr; return BGPU_ERR_NOMEM; }
        int rc = schol::factor_bind(S(stream), h->A, h->buf, h->F);
        if (rc) return rc;
        h->bound = true;
    }
    int rc = schol::factor(S(stream), h->F, d_M, ldm, d_D, reg, fp32);
    if (rc) return rc;
    if (info || pmin) {
        int i = 0;
        double p = 0;
        BGPU_CHECK(cudaMemcpyAsync(&i, h->F.info, sizeof(int), cudaMemcpyDeviceToHost, S(stream)));
        BGPU_CHECK(cudaMemcpyAsync(&p, h->F.pmin, sizeof(double), cudaMemcpyDeviceToHost, S(stream)));
        BGPU_CHECK(cudaStreamSynchronize(S(stream)));
        if (info) *info = i;
        if (pmin) *pmin = p;
    }
    return BGPU_OK;
}

BGPU_API int bgpu_schol_factor(bgpu_schol *h, const double *d_M, int64_t ldm, const double *d_D, double reg,
                               int *info, double *pmin, void *stream) {
    return schol_factor_any(h, d_M, ldm, d_D, reg, info, pmin, stream, false);
}

BGPU_API int bgpu_schol_factor_f32(bgpu_schol *h, const double *d_M, int64_t ldm, const double *d_D, double reg,
                                   int *info, double *pmin, void *stream) {
    return schol_factor_any(h, d_M, ldm, d_D, reg, info, pmin, stream, true);
}

BGPU_API int bgpu_schol_solve(bgpu_schol *h, const double *d_D, double *d_x, void *stream) {
    if (!h || !h->bound || !d_D || !d_x) return BGPU_ERR_ARG;
    return schol::solve(S(stream), h->F, d_D, d_x);
}

BGPU_API void bgpu_schol_destroy(bgpu_schol *h) {
    if (!h) return;
    if (h->buf) {
        cudaDeviceSynchronize();
        cudaFree(h->buf);
    }
    delete h;
}

}  // extern "C"
