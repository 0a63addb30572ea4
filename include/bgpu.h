/*
 * bgpu.h - step-level C ABI of the B200 Newton-step kernels.
 *
 * The reference's hot functions are static inside solver.c and sparsechol.c, so this
 * interface is the framework's own; each entry mirrors the contract of the reference
 * function it replaces (cited per entry).  Every pointer argument named d_* is device memory
 * (allocated by the caller: cudaMalloc, or torch tensors in the tests); stream is a
 * cudaStream_t (NULL for the default stream).  Every call returns a status: 0 on success,
 * BGPU_ERR_* (< 0) otherwise; no exception crosses the ABI.  Calls are asynchronous on the
 * stream unless stated; bgpu_sync waits for it.
 */
#ifndef BGPU_H
#define BGPU_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define BGPU_API __attribute__((visibility("default")))
#else
#define BGPU_API
#endif

#define BGPU_OK 0
#define BGPU_ERR_CUDA (-1)
#define BGPU_ERR_ARG (-2)
#define BGPU_ERR_NOTPD (-3)
#define BGPU_ERR_TIMEOUT (-4)
#define BGPU_ERR_NOMEM (-5)
#define BGPU_ERR_UNSUPPORTED (-6)
#define BGPU_ERR_TOOBIG (-7)

BGPU_API int bgpu_sync(void *stream);
BGPU_API const char *bgpu_version(void);
/* Number of kernels this library has launched since it was loaded (all entry points). */
BGPU_API long long bgpu_launch_count(void);
/* The bound of the triangular solves' device-side waits (bgpu_trsv, bgpu_trsv_f32,
 * bgpu_trsv_noalloc and the solves inside brisk_solve_*): the number of polls of an awaited flag,
 * each followed by a 64 ns sleep, after which the waiting block row gives up, the solve sets its
 * error flag and every CTA returns.  0 restores the default, 2^22 polls (about a second).  The
 * tensor-core GEMMs' barrier waits keep their fixed bound of 2^22 polls.  No counterpart in the
 * reference (its CPU solves do not wait on other threads' flags). */
BGPU_API void bgpu_set_wait_limit(unsigned polls);
/* Failure-path testing of the bounded waits: from now on, the CTA of block row r (64 rows each)
 * of every triangular solve computes its rows but does not publish its flag, so the block rows
 * that depend on it wait until the bound of bgpu_set_wait_limit runs out and the solve reports
 * BGPU_ERR_TIMEOUT; r < 0 restores normal solves (the default).  A test hook with no
 * counterpart in the reference: no GPU fault, hang or trap is involved. */
BGPU_API void bgpu_test_hold_trsv_row(int r);

/* An SDPA sparse file read into host arrays that the library owns: the reader of brisk_solve_file
 * (the reference's read_sdpa, problem.c:426, and its tokenizers, problem.c:58-91: comment lines,
 * the separators ",{}()=", Fortran exponents, text after the last entry, the same checks and
 * messages), on all host threads.  The arrays hold the numbers brisk_solve_data (capi.c:175)
 * takes: 1-based indices as written (a lower-triangle entry is not swapped), F0 as mat 0, entries
 * with value 0 left out.  Returns 0 and fills *out, whose arrays stay valid until
 * bgpu_sdpa_free(out); 2 when the file cannot be read or is malformed (the message goes to the
 * output set by brisk_set_output); BGPU_ERR_ARG for a NULL argument. */
typedef struct bgpu_sdpa {
    int m, nblk;
    int64_t nnz;
    const int *bs;
    const double *c;
    const int *mat, *blk, *i, *j;
    const double *v;
    void *owner;
} bgpu_sdpa;
BGPU_API int bgpu_sdpa_read(const char *path, bgpu_sdpa *out);
BGPU_API void bgpu_sdpa_free(bgpu_sdpa *s);

/* A problem kept resident in device memory between solves: bgpu_session_create takes the
 * numbers of brisk_solve_data (capi.c:175) and the options, uploads the scaled problem and
 * returns a handle (NULL on failure, *rc the exit code: 1 bad options, 2 bad problem, < 0 GPU
 * failure); bgpu_session_solve runs one interior-point solve from the resident data into res
 * (a brisk_result_new handle) and returns the exit code as brisk_solve_data.  Extension of
 * this build: the reference re-reads the problem on every call. */
struct BriskResult;
typedef struct bgpu_session bgpu_session;
BGPU_API bgpu_session *bgpu_session_create(int m, int nblk, const int *bs, const double *c, int64_t nnz,
                                           const int *mat, const int *blk, const int *i, const int *j,
                                           const double *v, int nopt, const char *const *opts, int *rc);
BGPU_API int bgpu_session_solve(bgpu_session *s, int nopt, const char *const *opts, struct BriskResult *res);
BGPU_API void bgpu_session_destroy(bgpu_session *s);
/* Solves `count` independent problems in one call: the arrays of brisk_solve_data (capi.c:175)
 * for every problem, concatenated in problem order.  Problem p has m[p] constraints, nblk[p]
 * blocks (its sizes follow those of problems 0..p-1 in bs), m[p] right-hand sides in c and
 * nnz[p] entries in mat/blk/i/j/v.  Every problem takes the same options; res[p] (a
 * brisk_result_new handle each) receives its result and rc[p] its exit code as brisk_solve_data
 * returns it.  The problems run concurrently on `workers` host threads (0: one per host core),
 * each with its own CUDA stream and one device arena reused from problem to problem, so no
 * device allocation or device-wide synchronisation runs between problems; each problem's result
 * is the result of brisk_solve_data on it.  Returns 0, 1 on bad options, -1 on bad arguments.
 * Replaces a loop of brisk_solve_data calls (capi.c:175), which is not reentrant. */
BGPU_API int bgpu_batch_solve(int count, const int *m, const int *nblk, const int *bs, const double *c,
                              const int64_t *nnz, const int *mat, const int *blk, const int *i, const int *j,
                              const double *v, int nopt, const char *const *opts, int workers,
                              struct BriskResult *const *res, int *rc);
/* A batch kept resident in device memory between solves: bgpu_batch_create takes the arrays of
 * bgpu_batch_solve for problems of one SDP block of order <= 64 each (the lockstep form), builds
 * and uploads them, and returns a handle (NULL on failure; *rc: 1 bad options, -1 bad arguments,
 * -6 a problem not of that shape, < 0 a GPU failure).  bgpu_batch_run solves every problem from
 * the resident data into res[p] (brisk_result_new handles), rc[p] its exit code (2 for a problem
 * rejected on input), and returns 0 or a negative GPU failure code.  Extension of this build: the
 * reference re-reads every problem on every call. */
typedef struct bgpu_batch bgpu_batch;
BGPU_API bgpu_batch *bgpu_batch_create(int count, const int *m, const int *nblk, const int *bs, const double *c,
                                       const int64_t *nnz, const int *mat, const int *blk, const int *i, const int *j,
                                       const double *v, int nopt, const char *const *opts, int *rc);
BGPU_API int bgpu_batch_run(bgpu_batch *h, struct BriskResult *const *res, int *rc);
BGPU_API void bgpu_batch_destroy(bgpu_batch *h);

/* Measures of the last solve of res: [0] device time (s, CUDA events on the library's
 * stream), [1] assembly device time (s), [2] assembly algorithmic flops, [3] host-to-device
 * bytes, [4] device-to-host bytes, [5] iterations, [6] float factorizations, [7] PCG steps. */
BGPU_API int bgpu_result_measures(const struct BriskResult *res, double *out8);

/* Workspace bytes of bgpu_schur_assemble for a block of order n, chunk constraints per GEMM
 * (8, 16, 32 or 64; 0 picks the default) and precision (0 FP64, 1 3xTF32, 2 the Ozaki products
 * with 8 slices, (S << 8) | 2 with S = 4..8 slices, as bgpu_gemm_ozaki_slices). */
BGPU_API size_t bgpu_schur_ws_bytes(int n, int chunk, int precision);
BGPU_API int bgpu_schur_chunk_default(int n, int precision);

/* Schur complement of one SDP block, accumulated into the full symmetric d_M (m x m,
 * column-major): M[con_a, con_b] += <A_b, X A_a Zi> for all constraint pairs of the block.
 * Constraints are given constraint-major: local constraint t has global index d_con[t] and
 * entries d_cpos/d_cval[d_cptr[t] .. d_cptr[t+1]) of the full (both triangles) expansion, with
 * positions p + q n ascending.  d_ccol (ncon*(n+1) ints) receives/holds the per-constraint
 * column pointers: bgpu_schur_colptr fills it once per problem.  Replaces schur_sdp /
 * schur_sdp_id (solver.c:1969, 2339-3021) for the row-product route. */
BGPU_API int bgpu_schur_colptr(int n, int ncon, const long long *d_cptr, const int *d_cpos, int *d_ccol, void *stream);
BGPU_API int bgpu_schur_assemble(int n, int m, int ncon, const int *d_con, const long long *d_cptr,
                                 const int *d_ccol, const int *d_cpos, const double *d_cval, const double *d_X,
                                 const double *d_Zi, double *d_M, int precision, int chunk, void *d_ws,
                                 size_t ws_bytes, void *stream);

/* Upper-triangle entry lists of the block's constraints for the packed symmetric gather:
 * entries p <= q of each constraint's full list, packed index u = q (q+1)/2 + p (ascending),
 * value A[p, q].  Fills d_uptr (ncon+1 offsets; d_counts is ncon ints of scratch) and *nu (the
 * total; the call synchronises on the stream); with d_upos and d_uval (nu each) non-NULL it
 * also fills them.  The reference keeps both triangles of each constraint (problem.c:1570-1610);
 * these lists are this build's own layout. */
BGPU_API int bgpu_schur_upper(int n, int ncon, const long long *d_cptr, const int *d_cpos, const double *d_cval,
                              int *d_counts, long long *d_uptr, int *d_upos, double *d_uval, long long *nu,
                              void *stream);
/* bgpu_schur_assemble with the packed symmetric gather: each chunk's G is folded into
 * G + G' on the upper triangle and every constraint's upper entries are read once (half the
 * entries and G values of the full gather; the same M up to rounding). */
BGPU_API int bgpu_schur_assemble_sym(int n, int m, int ncon, const int *d_con, const long long *d_cptr,
                                     const int *d_ccol, const int *d_cpos, const double *d_cval,
                                     const long long *d_uptr, const int *d_upos, const double *d_uval,
                                     const double *d_X, const double *d_Zi, double *d_M, int precision, int chunk,
                                     void *d_ws, size_t ws_bytes, void *stream);
/* M[con_a, con_b] += <A_a, A_b> for the block's constraints (the Gram matrix A A' of the
 * least-squares start, solver.c:13939-14198, which the reference assembles as the Schur
 * complement at X = Z = I): no products, the constraints' entries are scattered and gathered.
 * d_ws holds the packed chunk (n(n+1)/2 x K doubles, K the widest of 64..8 that fits). */
BGPU_API int bgpu_schur_gram(int n, int m, int ncon, const int *d_con, const long long *d_uptr, const int *d_upos,
                             const double *d_uval, double *d_M, void *d_ws, size_t ws_bytes, void *stream);

/* The dense route (the reference's route 2, solver.c:2972-3021) for blocks of dense constraints:
 * bgpu_schur_densify writes the constraints as dense matrices (d_Ad: ncon * n*n doubles, row t
 * the column-major A_t); bgpu_schur_assemble_dense then forms G_a = X A_a Zi per chunk of
 * constraints and M[:, a] = Ad vec(G_a) by one DMMA GEMM per chunk (full columns of M).  The
 * workspace is bgpu_schur_dense_ws_bytes. */
BGPU_API size_t bgpu_schur_dense_ws_bytes(int n, int ncon, int chunk, int precision);
BGPU_API int bgpu_schur_densify(int n, int ncon, const long long *d_cptr, const int *d_cpos, const double *d_cval,
                                double *d_Ad, void *stream);
BGPU_API int bgpu_schur_assemble_dense(int n, int m, int ncon, const int *d_con, const long long *d_cptr,
                                       const int *d_ccol, const int *d_cpos, const double *d_cval, const double *d_Ad,
                                       const double *d_X, const double *d_Zi, double *d_M, int precision, int chunk,
                                       void *d_ws, size_t ws_bytes, void *stream);

/* The LP route (schur_lp, solver.c:3233): M += A diag(x_p zi_p) A' over the N variables of one LP
 * block, A its nc x N constraint matrix, both triangles of M (column-major, m x m).  d_gcon[t]
 * is local constraint t's row of M; per constraint, its entries (variable, value) by ascending
 * variable in d_aptr (nc+1) / d_avar / d_aval; per variable, its entries (local constraint,
 * value) by ascending constraint in d_vptr (N+1) / d_vcon / d_vval (ne entries each); d_x and
 * d_zi the variables' x and 1/z.  Each entry of M sums its terms by ascending variable, as the
 * reference does; no atomics. */
BGPU_API int bgpu_schur_lp(int m, int N, int nc, int64_t ne, const int *d_gcon, const int64_t *d_aptr,
                           const int *d_avar, const double *d_aval, const int64_t *d_vptr, const int *d_vcon,
                           const double *d_vval, const double *d_x, const double *d_zi, double *d_M, void *stream);

/* The low-rank route (schur_lowrank, solver.c:1862-1934) for one block of order n: every
 * constraint's factor A_t = sum_k sig_k w_k w_k' is found on the host from the block's
 * full-expansion lists (host memory, as bgpu_schur_assemble takes them on the device: h_cptr
 * ncon+1 offsets, h_cpos positions p + q n, h_cval values), then M += the block's Schur
 * complement from P = W' X W and Q = W' Zi W (DMMA) and one launch over the pairs of
 * constraints; d_con[t] is constraint t's row of M (m x m, both triangles).  *rank receives the
 * total rank R.  Returns BGPU_ERR_UNSUPPORTED, leaving M alone, when some constraint has no
 * factor of rank below 28.  The device workspace (2 n R + 2 R^2 + 2 R doubles) is allocated and
 * freed inside the call, which waits for the stream. */
/* The host half of the low-rank route alone (no GPU): the factors of a block's constraints,
 * off[t] .. off[t+1] the columns of constraint t (off: ncon+1 ints), W (n x max_rank, column-major,
 * unit columns) and sig (max_rank) written when not NULL.  Returns R, or BGPU_ERR_UNSUPPORTED
 * when a constraint has no factor of rank below 28 or R > max_rank. */
BGPU_API int bgpu_lowrank_factor(int n, int ncon, const int64_t *h_cptr, const int *h_cpos, const double *h_cval,
                                 int max_rank, int *off, double *W, double *sig);
BGPU_API int bgpu_schur_lowrank(int n, int m, int ncon, const int *d_con, const int64_t *h_cptr, const int *h_cpos,
                                const double *h_cval, const double *d_X, const double *d_Zi, double *d_M, int *rank,
                                void *stream);

/* In-place Cholesky L L' = A of the lower triangle (column-major, lda); d_dinv receives the
 * inverses of the 64 x 64 diagonal blocks (ceil(n/64)*4096 entries), *d_info the first failing
 * column (1-based) or 0, *d_pmin the smallest squared pivot.  Replaces brisk_dpotrf
 * (sparsechol.c:3822) / chol_lower (solver.c:679); the float form replaces brisk_spotrf
 * (sparsechol.c:3841). */
BGPU_API int bgpu_potrf(int n, double *d_A, int lda, double *d_dinv, int *d_info, double *d_pmin, void *stream);
BGPU_API int bgpu_potrf_f32(int n, float *d_A, int lda, float *d_dinv, int *d_info, double *d_pmin, void *stream);

/* x <- L^-1 x (trans 0) or L^-T x (trans 1) with the factor of bgpu_potrf.  d_flags holds
 * ceil(n/64) ints; epoch must differ from the value of every earlier call on the same flags;
 * *d_err is set to 1 when a bounded device wait gives up.  Replaces brisk_dpotrs1 /
 * brisk_spotrs1 (sparsechol.c:4060-4180). */
BGPU_API int bgpu_trsv(int n, const double *d_L, int lda, const double *d_dinv, double *d_x, int trans,
                       int *d_flags, int epoch, int *d_err, void *stream);
BGPU_API int bgpu_trsv_f32(int n, const float *d_L, int lda, const float *d_dinv, float *d_x, int trans,
                           int *d_flags, int epoch, int *d_err, void *stream);

/* bgpu_trsv without caller-provided scratch, for callers that cannot allocate device memory
 * where they solve (between loop steps where cudaMalloc/cudaFree would synchronize the device,
 * or under another allocator that owns the device memory).  It has no counterpart in the
 * reference.  The block-row flags and the wait-error flag live in a static 8 KB device array of
 * the library.  The limit on n is the solve's own: one CTA per block row of 64 rows, all resident
 * at once, so n <= 64 x (SMs x resident CTAs per SM) -- on a B200 148 x 8 block rows, n <= 75776;
 * a larger n returns BGPU_ERR_TOOBIG with a message that gives the limit.  The first call on each
 * device looks up the array's device address.  Every call waits for the stream (it reads the
 * error flag back), so a call cannot be made while the stream is being captured into a CUDA
 * graph; it returns BGPU_ERR_TIMEOUT when a bounded device wait gave up.  Every call on a device
 * shares the array: calls that overlap on the GPU (other streams, other threads) race. */
BGPU_API int bgpu_trsv_noalloc(int n, const double *d_L, int lda, const double *d_dinv, double *d_x, int trans,
                               void *stream);

/* Linv = L^-1 from the factor of bgpu_potrf (the first half of brisk_dpotri_full,
 * sparsechol.c:4190). */
BGPU_API int bgpu_trtri(int n, const double *d_L, int lda, const double *d_dinv, double *d_Linv, int ldi,
                        void *stream);

/* C = alpha op(A) op(B) + beta C in FP64 on the DMMA tensor path (a_kmajor: A(i,k) =
 * A[i*lda+k], else A[i+k*lda]; b_kmajor: B(k,j) = B[k+j*ldb], else B[k*ldb+j]; C column-
 * major; lower: only i >= j).  The BLAS dgemm/dsyrk calls of the reference's dense routes. */
BGPU_API int bgpu_dgemm(int a_kmajor, int b_kmajor, int M, int N, int K, double alpha, const double *d_A,
                        int64_t lda, const double *d_B, int64_t ldb, double beta, double *d_C, int64_t ldc,
                        int lower, void *stream);

/* G = (Ah+Al)(Bh+Bl) by 3xTF32 on tcgen05 (A K-major rows, B K-major columns, G column-major). */
BGPU_API int bgpu_gemm_tf32x3(int M, int N, int K, const float *d_Ah, const float *d_Al, int64_t lda,
                              const float *d_Bh, const float *d_Bl, int64_t ldb, float *d_G, int64_t ldg,
                              void *stream);
BGPU_API int bgpu_split_tf32(int64_t n, const double *d_x, float *d_hi, float *d_lo, void *stream);

/* Batched small blocks (order n[k] <= 64, one CTA each; d_* arrays of nb device pointers to
 * n x n column-major matrices).  bgpu_small_chol_inv: L = chol(A), Li = L^-1 (lower), info[k]
 * the first failing column or 0 (chol_lower, solver.c:679).  bgpu_small_lammin: lam[k] =
 * lambda_min(Li D Li') by Householder tridiagonalization and Sturm bisection (small_lammin,
 * solver.c:5947-6027).  bgpu_small_gemm: C = alpha op(A) op(B) + beta C, or its symmetric part. */
BGPU_API int bgpu_small_chol_inv(int nb, const int *d_n, double *const *d_A, double *const *d_L,
                                 double *const *d_Li, int *d_info, void *stream);
BGPU_API int bgpu_small_lammin(int nb, const int *d_n, const double *const *d_Li, const double *const *d_D,
                               double *d_lam, void *stream);
BGPU_API int bgpu_small_gemm(int nb, const int *d_n, int ta, int tb, double alpha, const double *const *d_A,
                             const double *const *d_B, double beta, double *const *d_C, int sym, void *stream);

/* C = A B' (C(i, j) = sum_k A[i lda + k] B[j ldb + k], C column-major) with FP64-accurate
 * products on the INT8 tensor cores (tcgen05 kind::i8): each row of A and of B is cut exactly
 * into 8 signed 7-bit slices under a power-of-two exponent, the slice products with p + q <= 9
 * accumulate exactly in int32 and are summed in FP64 (the Ozaki scheme; K <= 16000).  The error
 * is below about 2^-53 K max_k |A(i, k)| max_k |B(j, k)|.  d_ws: bgpu_ozaki_ws_bytes(M, N, K) bytes.
 * Returns BGPU_ERR_TIMEOUT when a bounded wait of the kernel ran out; synchronizes the stream.
 * Replaces the pdgemm of the Schur assembly's row products (solver.c:2571-2590) where FP32
 * accuracy no longer suffices. */
BGPU_API size_t bgpu_ozaki_ws_bytes(int M, int N, int K);
BGPU_API int bgpu_gemm_ozaki(int M, int N, int K, const double *d_A, int64_t lda, const double *d_B, int64_t ldb,
                             double *d_C, int64_t ldc, void *d_ws, size_t ws_bytes, void *stream);
/* bgpu_gemm_ozaki with `slices` = 4..8 slices per operand: the pairs p + q <= slices + 1 are kept,
 * so the error is below about (slices + 3) 2^(-7 slices) K max_k |A(i, k)| max_k |B(j, k)|
 * (slices 6: 2^-39 K, slices 5: 2^-32 K), for 21 (6) or 15 (5) int8 products instead of 36, on
 * tiles of 80 (6) or 96 (5) columns instead of 64.  The workspace of bgpu_ozaki_ws_bytes serves
 * every slice count.  The mixed path's late Schur complements, a preconditioner whose residuals
 * are taken in FP64, need no more. */
BGPU_API int bgpu_gemm_ozaki_slices(int slices, int M, int N, int K, const double *d_A, int64_t lda, const double *d_B,
                                    int64_t ldb, double *d_C, int64_t ldc, void *d_ws, size_t ws_bytes, void *stream);

/* The NT scaling of one SDP block (nt_scaling, solver.c:7898-7912; nt_prep/nt_eig/nt_post,
 * solver.c:7824-7896): from the Cholesky factors L_X, L_Z of X and Z (lower triangles, n x n
 * column-major; the strict upper triangles are ignored) to G (n x n), lam (n) and W = G G'
 * (n x n), with G' Z G = G^-1 X G^-T = diag(lam) and W Z W = X.  V (G = L_X V diag(lam)^-1/2)
 * comes from one-sided Jacobi on L_Z' L_X: one CTA for n <= 64, block Jacobi above (d_ws of
 * bgpu_nt_ws_bytes(n) bytes).  Returns BGPU_OK, BGPU_ERR_NOTPD when a singular value is not
 * positive (nt_post's failure), BGPU_ERR_TIMEOUT when Jacobi did not converge in 40 sweeps;
 * *sweeps (may be null): the sweeps of the block form, 0 for n <= 64.  Synchronizes the stream. */
BGPU_API size_t bgpu_nt_ws_bytes(int n);
BGPU_API int bgpu_nt_scaling(int n, const double *d_LX, const double *d_LZ, double *d_G, double *d_lam,
                             double *d_W, void *d_ws, size_t ws_bytes, int *sweeps, void *stream);

/* y = alpha M x + beta y for a full symmetric M (schur_mv_, solver.c:4815). */
BGPU_API int bgpu_symv(int n, double alpha, const double *d_M, int ldm, const double *d_x, double beta,
                       double *d_y, void *stream);

/* out[con[t]] = beta out[con[t]] + alpha <A_t, D> (blk_Aop, solver.c:884-994). */
BGPU_API int bgpu_aop(int n, int ncon, const int *d_con, const long long *d_cptr, const int *d_cpos,
                      const double *d_cval, const double *d_D, double alpha, double beta, double *d_out,
                      void *stream);

/* Supernodal sparse Cholesky of the Schur complement (replaces sparse_build, solver.c:4014, and
 * schol_analyze / schol_factor / schol_solve, sparsechol.c).  The pattern of M is the union of
 * the cliques (the constraint sets of the blocks, clique c = clq_idx[clq_ptr[c] .. clq_ptr[c+1])).
 * bgpu_schol_analyze orders it (minimum degree on the clique quotient graph) and finds the
 * supernodes on the host (no GPU needed); *rc is 0 or a BGPU_ERR_ code.  bgpu_schol_info gives
 * [0] supernodes [1] entries of L [2] factor flops [3] largest front [4] tree levels [5] pattern
 * entries below the diagonal [6] m [7] device bytes of the factor.  bgpu_schol_perm gives the
 * elimination order (perm[k] = constraint eliminated k-th); bgpu_schol_supernodes gives the
 * supernodes' first positions (nsup+1), parents (-1 at a root), and the front rows (rptr nsup+1,
 * rows: elimination positions), any of them NULL to skip.
 * bgpu_schol_factor computes L L' = D M D + reg I on the pattern from the dense device M
 * (m x m, both triangles, leading dimension ldm) and the scaling d_D (m), on the device; the
 * first call allocates the factor's memory.  *info: 0 or the failing elimination position + 1;
 * *pmin: the smallest pivot (either pointer may be NULL; the call then does not synchronise).
 * bgpu_schol_factor_f32: the same factor with the fronts, L and the update matrices in FP32
 * (M, D and the solve's vectors stay FP64): the early iterations' factor, refined by PCG against
 * the FP64 M.  bgpu_schol_solve: d_x := D (L L')^-1 D d_x with the last factor's type. */
typedef struct bgpu_schol bgpu_schol;
BGPU_API bgpu_schol *bgpu_schol_analyze(int m, int ncliques, const int64_t *clq_ptr, const int *clq_idx, int *rc);
BGPU_API int bgpu_schol_info(const bgpu_schol *h, double *out8);
BGPU_API int bgpu_schol_perm(const bgpu_schol *h, int *perm);
BGPU_API int bgpu_schol_supernodes(const bgpu_schol *h, int *sfirst, int *parent, int64_t *rptr, int *rows);
BGPU_API int bgpu_schol_factor(bgpu_schol *h, const double *d_M, int64_t ldm, const double *d_D, double reg,
                               int *info, double *pmin, void *stream);
BGPU_API int bgpu_schol_factor_f32(bgpu_schol *h, const double *d_M, int64_t ldm, const double *d_D, double reg,
                                   int *info, double *pmin, void *stream);
BGPU_API int bgpu_schol_solve(bgpu_schol *h, const double *d_D, double *d_x, void *stream);
BGPU_API void bgpu_schol_destroy(bgpu_schol *h);
/* The ordering's tolerance for later analyses: each minimum-degree round eliminates the
 * independent supervariables of degree <= dmin (1 + delta) (default 1; 0: strict minimum degree,
 * the least fill, a taller tree).  No counterpart in the reference (its AMD has none). */
BGPU_API void bgpu_schol_set_delta(double delta);

#ifdef __cplusplus
}
#endif
#endif
