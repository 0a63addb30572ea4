// Internal host-side launchers of the Newton-step kernels (not exported; include/bgpu.h is
// the C ABI).  All device pointers; every launcher returns a BGPU_* status.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <vector>

// ---- GEMM (gemm_f64.cu) ----------------------------------------------------------------
int gemm_f64(cudaStream_t st, int a_kmajor, int b_kmajor, int M, int N, int K, double alpha, const double *A,
             long long lda, long long sA, const double *B, long long ldb, long long sB, double beta, double *C,
             long long ldc, long long sC, int batch, int lower);
// Grouped lower-triangle GEMMs: C_g(i, j) = alpha sum_k A_g(i, k) B_g(k, j) + beta C_g(i, j) for
// i >= j, A_g K-major (A(i,k) = A[i lda + k]), B_g K-major (B(k,j) = B[k + j ldb]); CTA t computes
// the 128 x 64 tile (tiles[t].y, tiles[t].z) of group tiles[t].x.
struct GemmGroup {
    const double *A, *B;
    double *C;
    int M, N, K;
    long long lda, ldb, ldc;
};
int gemm_f64_grouped(cudaStream_t st, int ntiles, const int4 *d_tiles, const GemmGroup *d_groups, double alpha,
                     double beta);
int gemm_grouped_tile_rows();   // 128 (the tile is 128 x 64)
int scale_matrix_f64(cudaStream_t st, int M, int N, double beta, double *C, long long ldc, long long sC, int batch,
                     int lower);

// ---- FP64-accurate GEMM on the INT8 tensor cores (ozaki.cu) ---------------------------------
// An operand cut into `slices` int8 slices (stacked, srows rows each, row stride ldk bytes) with
// one power-of-two exponent per row.
struct OzakiOperand {
    long long rows = 0, srows = 0, ldk = 0;
    int K = 0, slices = 8;
    int8_t *q = nullptr;
    int *e = nullptr;
};
int ozaki_max_slices();   // 8: FP64-like products
size_t ozaki_operand_bytes(long long rows, int K, int S);
// the slice layout of a rows x K operand in buf (ozaki_operand_bytes)
int ozaki_layout(long long rows, int K, void *buf, OzakiOperand *op, int S);
// S (4..8) slices of the rows x K operand src (row r at src + r lds) into buf (ozaki_operand_bytes)
int ozaki_slice(cudaStream_t st, long long rows, int K, const double *src, long long lds, void *buf, OzakiOperand *op,
                int S);
// C(i, j) = sum_k A(i, k) B(j, k), C column-major (ldc); A and B cut into the same number of slices
int ozaki_gemm(cudaStream_t st, const OzakiOperand &A, const OzakiOperand &B, double *C, long long ldc);
int ozaki_error_flag(int *host_value);

// ---- dense factor / solves (dense.cu) -----------------------------------------------------
constexpr int TRI_NB = 64;   // diagonal block order of the blocked factor and solves

// Blocked right-looking Cholesky of the lower triangle of A (n x n, column-major, lda), in
// place.  Writes the inverses of the 64 x 64 diagonal blocks of L to dinv (ceil(n/64) blocks of
// 64*64, column-major), the first failing column (1-based, 0 when none) to *d_info and the
// smallest squared pivot to *d_pmin (both device scalars, reset here).
int potrf_f64(cudaStream_t st, int n, double *A, long long lda, double *dinv, int *d_info, double *d_pmin);
int potrf_f32(cudaStream_t st, int n, float *A, long long lda, float *dinv, int *d_info, double *d_pmin);

// Persistent flag-chained triangular solves with the factor of potrf_*: x <- L^{-1} x (trans=0)
// or x <- L^{-T} x (trans=1), one right-hand side.  flags: ceil(n/64) ints, epoch: a value not
// used by an earlier call on the same flags; d_err is set to 1 when a wait gives up.
int trsv_f64(cudaStream_t st, int n, const double *L, long long lda, const double *dinv, double *x, int trans,
             int *flags, int epoch, int *d_err);
int trsv_f32(cudaStream_t st, int n, const float *L, long long lda, const float *dinv, float *x, int trans,
             int *flags, int epoch, int *d_err);

// Lower triangular inverse: Linv <- L^{-1} (n x n, column-major), using the diagonal-block
// inverses of potrf_f64.  The strict upper triangle of Linv is set to zero.
int trtri_f64(cudaStream_t st, int n, const double *L, long long lda, const double *dinv, double *Linv,
              long long ldi);

// y = alpha M x + beta y, M symmetric and stored in full (column-major, ldm).
int symv_full_f64(cudaStream_t st, int n, double alpha, const double *M, long long ldm, const double *x, double beta,
                  double *y);
// The step-length Lanczos on the device (lanczos.cu).  lanczos_start: Q[0] = q0 / |q0| (first n
// entries of q0) and the state reset; lanczos_step j (0 <= j < K <= 30), after w = B Q[j]:
// alpha_j, w orthogonalised twice against Q[0..j], beta_j, the stop test, Q[j+1] = w / beta_j;
// once done, lam = theta - res of the last T (or -1e300 when no bound exists) and the later steps
// are no-ops.  Q holds (K + 1) n doubles.
struct LanczosState {
    double alpha[32], beta[32];
    double scale, lam;
    int kk, done;
};
int lanczos_start(cudaStream_t st, int n, const double *q0, double *Q, LanczosState *s);
int lanczos_step(cudaStream_t st, int n, int j, int K, double *Q, double *w, LanczosState *s);

// y = M x reading only the pattern's entries (rowptr/cols: each row's columns, both triangles and
// the diagonal, ascending; entries of M off the pattern must be zero)
int pattern_symv_f64(cudaStream_t st, int n, const long long *rowptr, const int *cols, const double *M, long long ldm,
                     const double *x, double *y);

// Equilibrated copy for the factor: L = D M D + reg I (lower triangle; D = diag(M)^{-1/2},
// computed here into d_D), and the float variant writing Mf.
// d_D = diag(M)^-1/2 (1 where the diagonal is not positive).
int schur_diag_scale(cudaStream_t st, int m, const double *M, long long ldm, double *d_D);
int schur_load_f64(cudaStream_t st, int m, const double *M, long long ldm, double reg, double *d_D, double *L,
                   long long ldl);
int schur_load_f32(cudaStream_t st, int m, const double *M, long long ldm, double *d_D, float *Mf, long long ldf);

// ---- vector and matrix element-wise helpers (dense.cu) -----------------------------------
// Deterministic sums: out[q] = sum_i a_q[i] * b_q[i] for `nq` pairs of length n (one launch),
// written to the device array out.
int dots_f64(cudaStream_t st, int nq, const double *const *a, const double *const *b, long long n, double *out,
             double *scratch);
int symmetrize_f64(cudaStream_t st, int n, double *A, long long lda);
int copy_lower_to_upper_f64(cudaStream_t st, int n, double *A, long long lda);

// ---- Schur complement assembly (schur.cu) -------------------------------------------------
struct DevBlock {
    int n = 0;              // block order
    int ncon = 0;           // constraints that touch the block
    long long ne = 0;       // entries of the full (both triangles) expansion
    int *con = nullptr;     // [ncon] global constraint index
    long long *cptr = nullptr;  // [ncon+1] constraint-major offsets
    int *cpos = nullptr;    // [ne] position p + q*n, ascending within a constraint
    int *ccol = nullptr;    // [ncon*(n+1)] first entry of each column k, relative to cptr[t]
    double *cval = nullptr; // [ne]
    long long *pptr = nullptr;  // [n*n+1] position-major offsets
    int *pcon = nullptr;    // [ne] global constraint index of each position-major entry
    double *pval = nullptr; // [ne]
    double *C = nullptr;    // dense n x n (scaled)
    double *Ad = nullptr;   // [ncon * n*n] the constraints as dense matrices (dense route only)
    // upper-triangle lists (optional): entries p <= q of each constraint, packed index
    // u = q (q + 1) / 2 + p (ascending), value A[p, q]; the assembly then gathers from the packed
    // symmetric sum G_a + G_a' and reads half the entries and half the G values
    long long nu = 0;            // upper entries in all
    long long *uptr = nullptr;   // [ncon+1]
    int *upos = nullptr;         // [nu]
    double *uval = nullptr;      // [nu]
};

// out[con[t]] = beta*out[con[t]] + alpha * <A_t, D>  for every constraint of the block.
int aop_f64(cudaStream_t st, const DevBlock &B, const double *D, double alpha, double beta, double *out);
// F = alpha * sum_i y_i A_i + beta * F (full n x n).
int atop_f64(cudaStream_t st, const DevBlock &B, const double *y, double alpha, double beta, double *F);
// The same for nb blocks stored one after another in F (block k at d_off[k], d_off has nb+1
// entries, total = d_off[nb]); the blocks' position-major lists as device pointer tables.
int atop_blocks_f64(cudaStream_t st, int nb, const long long *d_off, long long total, const long long *const *pptr,
                    const int *const *pcon, const double *const *pval, const double *y, double alpha, double beta,
                    double *F);

// Workspace of the row-product assembly, sized by schur_ws_bytes.
struct SchurWs {
    void *buf = nullptr;
    size_t bytes = 0;
};
size_t schur_ws_bytes(int n, int chunk, int precision);
// Workspace of the dense route: schur_ws_bytes plus the chunk's output columns (and an FP64 copy
// of G in the mixed path).
size_t schur_dense_ws_bytes(int n, int ncon, int chunk, int precision);
// Fills B.Ad (device, ncon * n*n doubles) from the constraint-major entries.
int schur_densify(cudaStream_t st, const DevBlock &B);
// The dense route (the reference's route 2, solver.c:2972-3021): G_a = X A_a Zi as in the
// row-product route, then M[:, a] = Ad vec(G_a) for the chunk's constraints as one DMMA GEMM
// (ncon x K x n^2) instead of the entry gather.
int schur_assemble_dense(cudaStream_t st, const DevBlock &B, const double *X, const double *Zi, double *M, int m,
                         int precision, int chunk, void *ws, size_t ws_bytes);
// Many small blocks (n <= SB_NMAX) at once: M += each listed block's contribution (FP64), one CTA
// per block.  The listed blocks must share no constraint.  Per-block data by block id: order d_n,
// constraint count d_ncon, and device pointer tables of con / cptr / cpos / cval (the full
// expansion); X and Zi are the concatenations (block k at d_boff[k]); nmax = the largest listed n,
// ncon_max = the largest listed constraint count (it sets how many CTAs share a block).
constexpr int SB_NMAX = 32;
size_t schur_small_smem(int nmax);
int schur_assemble_small(cudaStream_t st, int count, const int *d_blocks, int nmax, int ncon_max, const int *d_n,
                         const int *d_ncon, const int *const *con_tab, const long long *const *cptr_tab,
                         const int *const *cpos_tab, const double *const *cval_tab, const long long *d_boff,
                         const double *Xcat, const double *Zicat, double *M, int m);
// The LP route (schur_lp, solver.c:3233): M += A diag(x_p zi_p) A' for the N variables of one LP
// block, A the block's nc x N constraint matrix.  Per local constraint t (global id gcon[t]): its
// entries (variable, value) by ascending variable in aptr/avar/aval; per variable p: its entries
// (local constraint, value) by ascending constraint in vptr/vcon/vval.  Xv[p], Zv[p] are the
// variables' X and Z^-1 (their order-1 blocks, one after another).  One warp per constraint a
// writes column gcon[a] (rows b >= a) and its mirror; each entry sums over ascending p, as the
// reference does.
struct LpGroupDev {
    int N = 0, nc = 0;
    long long ne = 0;
    int *gcon = nullptr;
    long long *aptr = nullptr;   // [nc+1]
    int *avar = nullptr;         // [ne]
    double *aval = nullptr;      // [ne]
    long long *vptr = nullptr;   // [N+1]
    int *vcon = nullptr;         // [ne]
    double *vval = nullptr;      // [ne]
};
int schur_assemble_lp(cudaStream_t st, const LpGroupDev &G, const double *Xv, const double *Zv, double *M, int m);
// The low-rank route (schur_lowrank, solver.c:1862-1934; lowrank.cu): a block whose every
// constraint is A_t = sum_{k in t} sig_k w_k w_k' (columns off[t] .. off[t+1] of W, n x R,
// column-major, unit columns).  XW (n x R), P and Q (R x R) are the route's workspace.
struct LowRankDev {
    int n = 0, ncon = 0, R = 0;
    double *W = nullptr, *sig = nullptr, *XW = nullptr, *P = nullptr, *Q = nullptr;
    int *off = nullptr;   // [ncon+1]
};
// Host: the factors of every constraint of a block from its full-expansion lists (cptr, cpos,
// cval as in DevBlock, host memory); 1 when every constraint factors and R <= max_rank, else 0.
int lowrank_factor_block(int n, int ncon, const long long *cptr, const int *cpos, const double *cval,
                         std::vector<int> &off, std::vector<double> &W, std::vector<double> &sig, int max_rank);
// M += the block's Schur complement: P = W' X W, Q = W' Zi W (DMMA), then M[con[u], con[t]] (and
// its mirror) += sum_{k in t, l in u} sig_k sig_l P_lk Q_lk over the pairs u >= t.
int schur_assemble_lowrank(cudaStream_t st, const LowRankDev &L, const int *con, const double *X, const double *Zi,
                           double *M, int m);
// Fills B.ccol (device, ncon*(n+1) ints) from cptr/cpos: the column pointers of each constraint.
int schur_colptr(cudaStream_t st, const DevBlock &B);
// Upper-triangle lists from the full ones: schur_upper_ptr fills B.uptr (ncon+1; uptr[ncon] is
// the total) using counts (device scratch, ncon ints); schur_upper then fills B.upos / B.uval.
int schur_upper_ptr(cudaStream_t st, const DevBlock &B, int *counts);
int schur_upper(cudaStream_t st, const DevBlock &B);
// M += the Gram matrix <A_b, A_a> of the block's constraints (the assembly at X = Zi = I, with no
// products): needs the upper lists.
int schur_assemble_gram(cudaStream_t st, const DevBlock &B, double *M, int m, void *ws, size_t ws_bytes);
int schur_chunk_default(int n, int precision);
int schur_ozaki_slices(int precision);   // the slices of an Ozaki precision code (8 when unset)
// M (m x m, column-major, full symmetric) += the block's contribution sum over its constraints
// of M_ab = <A_b, X A_a Zi>.  precision 0: FP64 (DMMA), 1: 3xTF32 (tcgen05), 2: products on the
// INT8 tensor cores (ozaki.cu) with 8 slices (FP64-accurate), (S << 8) | 2 with S = 4..8 slices.
int schur_assemble(cudaStream_t st, const DevBlock &B, const double *X, const double *Zi, double *M, int m,
                   int precision, int chunk, void *ws, size_t ws_bytes);
