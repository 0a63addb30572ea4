// Dense factor and solve kernels for the Schur complement M and the per-block X, Z.
//
// Cholesky: blocked right-looking, 64-column panels.  The diagonal block is factored in one
// CTA, which also writes the inverse of its 64 x 64 triangle; the panel below is then solved
// as a GEMM with that inverse and the trailing lower triangle updated by a DMMA rank-64 update
// (gemm_f64 with lower = 1).  This is the GPU counterpart of the reference's tiled dense
// Cholesky brisk_dpotrf / brisk_spotrf (sparsechol.c:3822-3860) and of chol_lower
// (solver.c:679): the same factor L L' = A and the same failure report (the first
// non-positive pivot), with the smallest squared pivot recorded for the acceptance test of
// schur_factor_ (solver.c:5344-5353, 5400-5410).
//
// Triangular solves: one persistent, cooperatively launched kernel per solve.  CTA r owns block
// row r; it subtracts L(r, c) x_c as soon as block c is published (a release/acquire flag with
// a bounded wait) and finishes with the diagonal-block inverse.  Replaces brisk_dpotrs1 /
// brisk_spotrs1 (sparsechol.c:4060-4180) and the dtrsv calls of the Lanczos step length.
#include "common.cuh"
#include "kernels.h"
#include <cooperative_groups.h>
#include <algorithm>

namespace {
constexpr int NB = TRI_NB;      // 64
constexpr int LDS = NB + 1;     // padded smem stride

// ---- diagonal-block factor + inverse ----------------------------------------------------
// One CTA of 256 threads on the 64 x 64 diagonal block in shared memory, in four steps of 16
// columns.  Step k: one warp factors the 16 x 16 diagonal sub-block L_kk and inverts it in its
// registers (lane r holds row r; the pivots and rows travel by shuffles, no barrier), the rows
// below are solved against it (L_ik = A_ik L_kk^-T: one thread a row), and the trailing lower
// triangle takes the rank-16 update.  The inverse X = L^-1 of the whole block then follows by
// its block diagonals: X_kk from the steps, X_ij = -X_ii sum_{k=j}^{i-1} L_ik X_kj for i - j =
// 1, 2, 3.  About twenty barriers instead of two a column.  Rows and columns past the block's
// order are the identity, so a partial last block factors and inverts as a whole one.
constexpr int DB = 16;   // sub-block order (16 lanes of a warp)

// Cholesky of the 16 x 16 block held by lanes 0-15 (a[j], j <= lane; lanes 16-31 hold zeros)
// and its inverse (x[j], j <= lane).  `real` columns count for the smallest pivot; returns the
// first failing column (0-based) or -1.
template <typename T>
__device__ __forceinline__ int chol_inv16(T (&a)[DB], T (&x)[DB], int lane, int real, double &pm) {
    int fail = -1;   // (the loops run on past a failure, on values the caller then discards: no early
                     // exit, so they unroll whole and the rows stay in registers)
#pragma unroll
    for (int c = 0; c < DB; c++) {
        const T d = __shfl_sync(0xffffffffu, a[c], c);
        if (fail < 0 && (!(d > (T)0) || !isfinite((double)d))) fail = c;   // uniform over the warp
        if (c < real && (double)d < pm) pm = (double)d;
        const T sd = sqrt(d), isd = (T)1 / sd;
        if (lane == c) a[c] = sd;
        else if (lane > c) a[c] *= isd;
#pragma unroll
        for (int j = 0; j < DB; j++) {   // (fixed bounds: both loops unroll and a[] stays in registers)
            const T ljc = __shfl_sync(0xffffffffu, a[c], j);
            if (j > c && lane >= j) a[j] -= a[c] * ljc;
        }
    }
    T diag = (T)1;
#pragma unroll
    for (int j = 0; j < DB; j++)
        if (lane == j) diag = a[j];
    const T rd = (T)1 / diag;
    // X = L^-1 row by row: row k is final once the rows above have been subtracted (acc), so step
    // k finishes it in lane k and broadcasts it; the 16 shuffles of a step are independent, and
    // the chain is 16 steps long: X[r][j] = -(sum_{k<r} L[r][k] X[k][j]) / L[r][r], X[r][r] = 1/L[r][r]
    T acc[DB];
#pragma unroll
    for (int j = 0; j < DB; j++) acc[j] = (T)0;
#pragma unroll
    for (int k = 0; k < DB; k++) {
        if (lane == k) {
#pragma unroll
            for (int j = 0; j < DB; j++) x[j] = (j < k) ? -acc[j] * rd : (j == k ? rd : (T)0);
        }
        const T lrk = a[k];   // L[r][k] of this lane's row r
#pragma unroll
        for (int j = 0; j < DB; j++) {
            if (j > k) continue;
            const T xkj = __shfl_sync(0xffffffffu, x[j], k);
            if (lane > k) acc[j] += lrk * xkj;
        }
    }
    return fail;
}

template <typename T>
__global__ void __launch_bounds__(256, 1) potrf_diag_kernel(int n, T *A, long long lda, int j0, T *dinv, int *info,
                                                         double *pmin) {
    extern __shared__ __align__(16) unsigned char dsm_raw[];
    T *S = reinterpret_cast<T *>(dsm_raw);   // S[r + c*LDS]: the block, then L
    T *X = S + NB * LDS;                      // the inverse of L
    __shared__ T P[3][DB][DB + 1];            // the sums of the off-diagonal inverse blocks
    __shared__ int s_fail;
    __shared__ double s_pm;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nb = min(NB, n - j0);
    if (*(volatile int *)info != 0) return;   // an earlier panel failed: nothing to do
    T *Ad = A + (long long)j0 + (long long)j0 * lda;
    for (int idx = tid; idx < NB * NB; idx += 256) {
        const int r = idx & (NB - 1), c = idx >> 6;   // column c: rows coalesced
        T v = (r == c) ? (T)1 : (T)0;                 // the identity past the block's order
        if (r < nb && c < nb && r >= c) v = Ad[r + (long long)c * lda];
        S[r + c * LDS] = v;
        X[r + c * LDS] = (T)0;
    }
    if (tid == 0) { s_fail = -1; s_pm = 1e300; }
    __syncthreads();
    for (int kb = 0; kb < NB / DB; kb++) {
        const int k0 = kb * DB;
        if (warp == 0) {
            T a[DB], x[DB];
#pragma unroll
            for (int j = 0; j < DB; j++) a[j] = (lane < DB && j <= lane) ? S[(k0 + lane) + (k0 + j) * LDS] : (T)0;
            double pm = 1e300;
            const int f = chol_inv16<T>(a, x, lane, nb - k0, pm);
            if (f >= 0) {
                if (lane == 0) s_fail = k0 + f;
            } else if (lane < DB) {
#pragma unroll
                for (int j = 0; j < DB; j++)
                    if (j <= lane) {
                        S[(k0 + lane) + (k0 + j) * LDS] = a[j];
                        X[(k0 + lane) + (k0 + j) * LDS] = x[j];
                    }
            }
            if (lane == 0 && pm < s_pm) s_pm = pm;
        }
        __syncthreads();
        if (s_fail >= 0) break;
        // rows below: L_ik = A_ik L_kk^-T, one thread a row (its 16 values first, then written)
        const int rows = NB - k0 - DB;
        if (tid < rows) {
            const int r = k0 + DB + tid;
            T v[DB];
#pragma unroll
            for (int k = 0; k < DB; k++) v[k] = S[r + (k0 + k) * LDS];
#pragma unroll
            for (int j = 0; j < DB; j++) {   // L_rj = sum_{k <= j} v_k X_kk[j][k] (v read whole first)
                T s = (T)0;
#pragma unroll
                for (int k = 0; k <= j; k++) s += v[k] * X[(k0 + j) + (k0 + k) * LDS];
                S[r + (k0 + j) * LDS] = s;
            }
        }
        __syncthreads();
        // the trailing lower triangle: S[i][j] -= sum_k L[i][k] L[j][k], i >= j > k0 + 15
        const int t0 = k0 + DB, tn = NB - t0;
        for (int idx = tid; idx < tn * tn; idx += 256) {
            const int i = t0 + idx % tn, jj = t0 + idx / tn;
            if (i < jj) continue;
            T s = (T)0;
#pragma unroll
            for (int k = 0; k < DB; k++) s += S[i + (k0 + k) * LDS] * S[jj + (k0 + k) * LDS];
            S[i + jj * LDS] -= s;
        }
        __syncthreads();
    }
    if (s_fail >= 0) {
        if (tid == 0 && s_fail < nb) atomicCAS(info, 0, j0 + s_fail + 1);
        return;
    }
    if (tid == 0) atomicMin((unsigned long long *)pmin, (unsigned long long)__double_as_longlong(s_pm));
    // the off-diagonal blocks of X, one block diagonal at a time
    for (int d = 1; d < NB / DB; d++) {
        const int nblk = NB / DB - d;
        for (int idx = tid; idx < nblk * DB * DB; idx += 256) {   // P = sum_{k=j}^{i-1} L_ik X_kj
            const int bj = idx / (DB * DB), e = idx % (DB * DB), r = e % DB, c = e / DB, bi = bj + d;
            T s = (T)0;
            for (int k = bj * DB; k < bi * DB; k++) s += S[(bi * DB + r) + k * LDS] * X[k + (bj * DB + c) * LDS];
            P[bj][r][c] = s;
        }
        __syncthreads();
        for (int idx = tid; idx < nblk * DB * DB; idx += 256) {   // X_ij = -X_ii P
            const int bj = idx / (DB * DB), e = idx % (DB * DB), r = e % DB, c = e / DB, bi = bj + d;
            T s = (T)0;
#pragma unroll
            for (int k = 0; k < DB; k++) s += X[(bi * DB + r) + (bi * DB + k) * LDS] * P[bj][k][c];
            X[(bi * DB + r) + (bj * DB + c) * LDS] = -s;
        }
        __syncthreads();
    }
    for (int idx = tid; idx < NB * NB; idx += 256) {
        const int r = idx & (NB - 1), c = idx >> 6;
        if (r < nb && c < nb && r >= c) Ad[r + (long long)c * lda] = S[r + c * LDS];
        dinv[r + c * NB] = (r >= c) ? X[r + c * LDS] : (T)0;   // identity past the block's order
    }
}

__global__ void init_info_kernel(int *info, double *pmin) {
    *info = 0;
    *pmin = 1.0;
}

// ---- float panel solve and trailing update (SIMT FFMA; the mixed path's factor) --------------
// A21 <- A21 * Dinv^T  (rows below the panel), in place: a CTA reads a full row block first.
__global__ void __launch_bounds__(256) trsm_panel_f32(int rows, int nb, float *A21, long long lda, const float *dinv) {
    __shared__ float Di[NB * NB];
    __shared__ float R[64 * LDS];
    const int tid = threadIdx.x;
    const int r0 = blockIdx.x * 64;
    for (int idx = tid; idx < NB * NB; idx += 256) Di[idx] = dinv[idx];
    for (int idx = tid; idx < 64 * NB; idx += 256) {
        const int r = idx % 64, c = idx / 64;
        R[r + c * LDS] = (r0 + r < rows && c < nb) ? A21[(r0 + r) + (long long)c * lda] : 0.f;
    }
    __syncthreads();
    // out(r, j) = sum_k R(r, k) Di(j, k)
    for (int idx = tid; idx < 64 * nb; idx += 256) {
        const int r = idx % 64, j = idx / 64;
        float s = 0.f;
        for (int k = 0; k <= j; k++) s += R[r + k * LDS] * Di[j + k * NB];
        if (r0 + r < rows) A21[(r0 + r) + (long long)j * lda] = s;
    }
}

// C(i, j) -= sum_k A(i, k) A(j, k) for i >= j, i < M, j < N (the lower part of an M x N block whose
// diagonal starts at its top left, N <= M): 128 x 128 output tiles (tiles wholly above the
// diagonal return at once), 8 x 8 outputs a thread, K in steps of 16 through shared memory (a
// quarter of a shared-memory load per FMA).
constexpr int SY_T = 128, SY_K = 16;
__global__ void __launch_bounds__(256) syrk_f32(int M, int N, int K, const float *A, long long lda, float *C,
                                                long long ldc) {
    const int bi = blockIdx.x, bj = blockIdx.y;
    if (bi < bj) return;
    __shared__ __align__(16) float As[SY_K][SY_T + 4], Bs[SY_K][SY_T + 4];
    const int tid = threadIdx.x;
    // rows tr*4 .. +3 and 64 + tr*4 .. +3, columns likewise from tc: a quarter-warp's float4 reads
    // of a shared-memory row are 128 contiguous bytes (no bank conflict)
    const int tr = tid % 16, tc = tid / 16;
    float acc[8][8];
#pragma unroll
    for (int u = 0; u < 8; u++)
#pragma unroll
        for (int v = 0; v < 8; v++) acc[u][v] = 0.f;
    const long long ri0 = (long long)bi * SY_T, rj0 = (long long)bj * SY_T;
    for (int k0 = 0; k0 < K; k0 += SY_K) {
        __syncthreads();   // the previous step's tiles are consumed
        for (int idx = tid; idx < SY_T * SY_K; idx += 256) {
            const int r = idx % SY_T, k = idx / SY_T;   // rows contiguous in A (column-major)
            const bool kin = k0 + k < K;
            As[k][r] = (ri0 + r < M && kin) ? A[(ri0 + r) + (long long)(k0 + k) * lda] : 0.f;
            Bs[k][r] = (rj0 + r < N && kin) ? A[(rj0 + r) + (long long)(k0 + k) * lda] : 0.f;
        }
        __syncthreads();
#pragma unroll 4
        for (int k = 0; k < SY_K; k++) {
            const float4 a0 = *reinterpret_cast<const float4 *>(&As[k][tr * 4]);
            const float4 a1 = *reinterpret_cast<const float4 *>(&As[k][SY_T / 2 + tr * 4]);
            const float4 b0 = *reinterpret_cast<const float4 *>(&Bs[k][tc * 4]);
            const float4 b1 = *reinterpret_cast<const float4 *>(&Bs[k][SY_T / 2 + tc * 4]);
            const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float b[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int u = 0; u < 8; u++)
#pragma unroll
                for (int v = 0; v < 8; v++) acc[u][v] += a[u] * b[v];
        }
    }
#pragma unroll
    for (int u = 0; u < 8; u++)
#pragma unroll
        for (int v = 0; v < 8; v++) {
            const long long i = ri0 + (u < 4 ? tr * 4 + u : SY_T / 2 + tr * 4 + u - 4);
            const long long j = rj0 + (v < 4 ? tc * 4 + v : SY_T / 2 + tc * 4 + v - 4);
            if (i < M && j < N && i >= j) C[i + j * ldc] -= acc[u][v];
        }
}

// ---- persistent triangular solve -----------------------------------------------------------
// trans = 0: solve L x = b (block rows top-down); trans = 1: solve L' x = b (bottom-up).
// One CTA per block row (all co-resident: a cooperative launch).  Thread (row, q) of the CTA of
// block row r keeps, in a register, the sum over the blocks c that row r depends on of
// L(r, c)[row, 16 q .. 16 q + 15] x_c; each warp waits by itself (its lane 0, at most `limit`
// polls) for block c's flag before it reads x_c, so the waits cost no CTA barrier.  Once every
// dependency is in, x_r = Dinv_r (b_r - sum) and the flag of r is published.  The critical path
// is the chain of these last steps: with PRE, the block of the last dependency (c = r - 1, or
// r + 1 for trans = 1) and Dinv_r are loaded into shared memory while the earlier rows solve, so
// that step reads nothing but x_c from global memory.
// hold >= 0 (failure-path tests only): the CTA of that block row computes its rows but does
// not publish its flag, so the rows after it give up waiting and report through *err.
template <typename T, bool PRE>
__global__ void __launch_bounds__(256, PRE ? 1 : 8) trsv_kernel(int n, const T *L, long long lda, const T *dinv, T *x,
                                                                int trans, int *flags, int epoch, int *err,
                                                                unsigned limit, int hold) {
    extern __shared__ __align__(16) unsigned char tsm_raw[];   // PRE: Bs[NB * NB], Ds[NB * NB]
    __shared__ T part[4][NB];
    __shared__ T acc[NB];
    __shared__ int bad;
    const int tid = threadIdx.x, lane = tid & 31;
    const int nblk = (n + NB - 1) / NB;
    const int r = trans ? (nblk - 1 - blockIdx.x) : blockIdx.x;   // the block row this CTA owns
    const int r0 = r * NB, nr = min(NB, n - r0);
    const int row = tid & 63, q = tid >> 6;   // 4 threads per row, 16 columns each
    const int ndep = trans ? (nblk - 1 - r) : r;
    const T *D = dinv + (size_t)r * NB * NB;
    T *Bs = reinterpret_cast<T *>(tsm_raw), *Ds = Bs + NB * NB;
    if (tid < NB) acc[tid] = (tid < nr) ? x[r0 + tid] : (T)0;
    if (tid == 0) bad = 0;
    if (PRE) {
        // Ds[i + k NB] = the (i, k) coefficient of x_r = Ds acc; Bs[i + k NB] the one of the last
        // dependency's block (0 past the order)
        for (int idx = tid; idx < NB * NB; idx += 256) {
            const int a = idx & 63, b = idx >> 6;   // a: the index that is contiguous in memory
            if (!trans) Ds[a + b * NB] = D[a + b * NB];
            else Ds[b + a * NB] = D[a + b * NB];
        }
        if (ndep > 0) {
            const int c = trans ? r + 1 : r - 1, c0 = c * NB, nc = min(NB, n - c0);
            for (int idx = tid; idx < NB * NB; idx += 256) {
                const int a = idx & 63, b = idx >> 6;
                if (!trans)   // L(r0 + a, c0 + b): rows a contiguous
                    Bs[a + b * NB] = (a < nr && b < nc) ? L[(r0 + a) + (long long)(c0 + b) * lda] : (T)0;
                else          // L(c0 + a, r0 + b), the coefficient of row b, column a
                    Bs[b + a * NB] = (b < nr && a < nc) ? L[(c0 + a) + (long long)(r0 + b) * lda] : (T)0;
            }
        }
    }
    __syncthreads();
    T s = (T)0;
    bool ok = true;
    for (int d = 0; d < ndep; d++) {
        const int c = trans ? (nblk - 1 - d) : d;   // dependencies in the order they finish
        if (lane == 0) {
            unsigned spins = 0;
            while (ld_acquire(&flags[c]) != epoch) {
                if (++spins > limit) { ok = false; break; }
                __nanosleep(64);
            }
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) break;
        const int c0 = c * NB, nc = min(NB, n - c0);
        const bool last = PRE && d == ndep - 1;
        if (row < nr) {
#pragma unroll 4
            for (int k = q * 16; k < q * 16 + 16; k++) {
                if (k >= nc) break;
                const T xv = ((volatile T *)x)[c0 + k];
                const T lv = last ? Bs[row + k * NB]
                                  : (trans ? L[(c0 + k) + (long long)(r0 + row) * lda] : L[(r0 + row) + (long long)(c0 + k) * lda]);
                s += lv * xv;
            }
        }
    }
    if (!ok) bad = 1;
    part[q][row] = s;
    __syncthreads();
    if (bad) {
        if (tid == 0) atomicExch(err, 1);
        return;
    }
    if (tid < NB) acc[tid] -= (part[0][tid] + part[1][tid]) + (part[2][tid] + part[3][tid]);
    __syncthreads();
    // x_r = Dinv_r acc (trans = 0) or Dinv_r' acc (trans = 1)
    T t = (T)0;
    if (PRE) { for (int k = q * 16; k < q * 16 + 16; k++) t += Ds[row + k * NB] * acc[k]; }
    else if (!trans) { for (int k = q * 16; k < q * 16 + 16; k++) t += D[row + k * NB] * acc[k]; }
    else             { for (int k = q * 16; k < q * 16 + 16; k++) t += D[k + row * NB] * acc[k]; }
    part[q][row] = t;
    __syncthreads();
    if (tid < nr) x[r0 + tid] = (part[0][tid] + part[1][tid]) + (part[2][tid] + part[3][tid]);
    __threadfence();
    __syncthreads();
    if (tid == 0 && r != hold) st_release(&flags[r], epoch);
}

template <typename T> constexpr size_t trsv_pre_smem() { return 2 * (size_t)NB * NB * sizeof(T); }

// The largest number of block rows one solve can take on the current device: every CTA of the
// cooperative launch must be resident at once (SMs x resident CTAs per SM), for the kernel
// without (PRE = false) or with the shared-memory preload.
std::atomic<int> g_trsv_cap[2][2][64];
template <typename T, bool PRE = false>
int trsv_max_blocks(int *cap) {
    int dev = 0;
    BGPU_CHECK(cudaGetDevice(&dev));
    std::atomic<int> *slot = (dev >= 0 && dev < 64) ? &g_trsv_cap[sizeof(T) == 8][PRE][dev] : nullptr;
    if (slot && slot->load(std::memory_order_relaxed) > 0) {
        *cap = slot->load(std::memory_order_relaxed);
        return BGPU_OK;
    }
    int nsm = 0, per = 0;
    BGPU_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    if (PRE)
        BGPU_CHECK(cudaFuncSetAttribute(trsv_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)trsv_pre_smem<T>()));
    BGPU_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, trsv_kernel<T, PRE>, 256,
                                                             PRE ? trsv_pre_smem<T>() : 0));
    *cap = nsm * per;
    if (slot) slot->store(*cap, std::memory_order_relaxed);
    return BGPU_OK;
}

template <typename T>
int trsv_launch(cudaStream_t st, int n, const T *L, long long lda, const T *dinv, T *x, int trans, int *flags,
                int epoch, int *d_err) {
    if (n <= 0) return BGPU_OK;
    const int nblk = (n + NB - 1) / NB;
    int cap = 0, cap_pre = 0;
    if (int rc = trsv_max_blocks<T>(&cap)) return rc;
    if (nblk > cap) return BGPU_ERR_TOOBIG;
    if (int rc = trsv_max_blocks<T, true>(&cap_pre)) return rc;
    unsigned limit = wait_limit();
    int hold = trsv_hold_row();
    void *args[] = {(void *)&n, (void *)&L, (void *)&lda, (void *)&dinv, (void *)&x, (void *)&trans,
                    (void *)&flags, (void *)&epoch, (void *)&d_err, (void *)&limit, (void *)&hold};
    if (nblk <= cap_pre)
        BGPU_CHECK(cudaLaunchCooperativeKernel((void *)trsv_kernel<T, true>, dim3(nblk), dim3(256), args,
                                               trsv_pre_smem<T>(), st));
    else
        BGPU_CHECK(cudaLaunchCooperativeKernel((void *)trsv_kernel<T, false>, dim3(nblk), dim3(256), args, 0, st));
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

// ---- element-wise helpers ---------------------------------------------------------------
__global__ void set_identity_lower_kernel(int n, double *A, long long lda) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)n * n) return;
    const int i = (int)(idx % n), j = (int)(idx / n);
    A[i + (long long)j * lda] = (i == j) ? 1.0 : 0.0;
}

__global__ void symv_full_kernel(int n, double alpha, const double *M, long long ldm, const double *x, double beta,
                                 double *y) {
    const int warps = blockDim.x >> 5;
    const int col = blockIdx.x * warps + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (col >= n) return;
    const double *c = M + (long long)col * ldm;
    double s = 0.0;
    for (int i = lane; i < n; i += 32) s += c[i] * x[i];
    s = warp_sum(s);
    if (lane == 0) y[col] = (beta == 0.0) ? alpha * s : alpha * s + beta * y[col];
}

// y = M x over a known pattern: row a holds the columns cols[rowptr[a] .. rowptr[a+1]) (ascending),
// read from column a of the symmetric dense M (contiguous in memory); one warp a row, lanes
// strided over the row's entries and summed by a fixed reduction.  Entries off the pattern are
// zero in M, so this is M x with a fraction of the reads.
__global__ void pattern_symv_kernel(int n, const long long *__restrict__ rowptr, const int *__restrict__ cols,
                                    const double *__restrict__ M, long long ldm, const double *__restrict__ x,
                                    double *y) {
    const int warps = blockDim.x >> 5;
    const int a = blockIdx.x * warps + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (a >= n) return;
    const double *c = M + (long long)a * ldm;
    double s = 0.0;
    for (long long t = rowptr[a] + lane; t < rowptr[a + 1]; t += 32) {
        const int b = cols[t];
        s += c[b] * x[b];
    }
    s = warp_sum(s);
    if (lane == 0) y[a] = s;
}

__global__ void diag_scale_kernel(int m, const double *M, long long ldm, double *D) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const double d = M[i + (long long)i * ldm];
    D[i] = d > 0 ? 1.0 / sqrt(d) : 1.0;
}

__global__ void load_scaled_f64_kernel(int m, const double *M, long long ldm, const double *D, double reg, double *L,
                                       long long ldl) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= m || i < j) return;
    double v = M[i + (long long)j * ldm] * D[i] * D[j];
    if (i == j) v += reg;
    L[i + (long long)j * ldl] = v;
}

__global__ void load_scaled_f32_kernel(int m, const double *M, long long ldm, const double *D, float *F,
                                       long long ldf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= m || i < j) return;
    const double v = M[i + (long long)j * ldm] * D[i] * D[j];
    F[i + (long long)j * ldf] = (fabs(v) < 1e-30) ? 0.0f : (float)v;   // no subnormals in the float factor
}

__global__ void symmetrize_kernel(int n, double *A, long long lda) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= n || i <= j) return;
    double *a = A + i + (long long)j * lda, *b = A + j + (long long)i * lda;
    const double v = 0.5 * (*a + *b);
    *a = v;
    *b = v;
}

__global__ void lower_to_upper_kernel(int n, double *A, long long lda) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= n || i <= j) return;
    A[j + (long long)i * lda] = A[i + (long long)j * lda];
}

// Deterministic two-level dot products: a fixed number of partial sums per pair.
constexpr int DOT_PARTS = 128;
__global__ void dots_partial_kernel(const double *const *a, const double *const *b, long long n, double *scratch) {
    const int q = blockIdx.y, part = blockIdx.x;
    const double *x = a[q], *y = b[q];
    const long long chunk = (n + DOT_PARTS - 1) / DOT_PARTS;
    const long long lo = part * chunk, hi = min(n, lo + chunk);
    double s = 0.0;
    for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) s += x[i] * y[i];
    __shared__ double red[8];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
        scratch[(long long)q * DOT_PARTS + part] = t;
    }
}
__global__ void dots_final_kernel(const double *scratch, double *out) {
    const int q = blockIdx.x;
    double s = 0.0;
    for (int i = threadIdx.x; i < DOT_PARTS; i += 32) s += scratch[(long long)q * DOT_PARTS + i];
    s = warp_sum(s);
    if (threadIdx.x == 0) out[q] = s;
}
}  // namespace

// ---- host launchers -------------------------------------------------------------------------
template <typename T>
int diag_smem_attr() {
    BGPU_ATTR_ONCE(BGPU_CHECK(cudaFuncSetAttribute(potrf_diag_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)(2 * NB * LDS * sizeof(T)))));
    return BGPU_OK;
}

// The blocked factor in outer panels of PANEL columns.  Within a panel, each 64-column block is
// factored (potrf_diag_kernel), the whole column below it solved against its inverse, and the
// panel's later columns updated (rank 64).  The columns right of the panel then take one
// rank-PANEL update, which reads and writes the trailing triangle once per panel (not once per 64
// columns) and gives the tensor-core GEMM a depth of PANEL.
constexpr int PANEL = 256;

namespace {
// factor the panel of columns [J0, J0 + JB) (all its updates from earlier panels applied)
template <typename T>
int factor_panel(cudaStream_t st, int n, T *A, long long lda, T *dinv, int J0, int JB, int *d_info, double *d_pmin);

template <>
int factor_panel<double>(cudaStream_t st, int n, double *A, long long lda, double *dinv, int J0, int JB, int *d_info,
                         double *d_pmin) {
    for (int j0 = J0; j0 < J0 + JB; j0 += NB) {
        const int nb = std::min(NB, n - j0);
        double *Di = dinv + (size_t)(j0 / NB) * NB * NB;
        potrf_diag_kernel<double><<<1, 256, 2 * NB * LDS * sizeof(double), st>>>(n, A, lda, j0, Di, d_info, d_pmin);
        BGPU_LAUNCH_CHECK();
        const int rest = n - j0 - nb;
        if (rest <= 0) break;
        double *A21 = A + (j0 + nb) + (long long)j0 * lda;
        // A21 <- A21 Di'  (B(k, j) = Di(j, k) = Di[j + k*NB]: N-major); in place, N = nb <= 64
        int rc = gemm_f64(st, 0, 0, rest, nb, nb, 1.0, A21, lda, 0, Di, NB, 0, 0.0, A21, lda, 0, 1, 0);
        if (rc) return rc;
        // the panel's later columns: A[j0+nb.., j0+nb .. J0+JB) -= A21 A21(top pc rows)', lower
        const int pc = J0 + JB - (j0 + nb);
        if (pc > 0) {
            rc = gemm_f64(st, 0, 0, rest, pc, nb, -1.0, A21, lda, 0, A21, lda, 0, 1.0,
                          A + (j0 + nb) + (long long)(j0 + nb) * lda, lda, 0, 1, 1);
            if (rc) return rc;
        }
    }
    return BGPU_OK;
}

template <>
int factor_panel<float>(cudaStream_t st, int n, float *A, long long lda, float *dinv, int J0, int JB, int *d_info,
                        double *d_pmin) {
    for (int j0 = J0; j0 < J0 + JB; j0 += NB) {
        const int nb = std::min(NB, n - j0);
        float *Di = dinv + (size_t)(j0 / NB) * NB * NB;
        potrf_diag_kernel<float><<<1, 256, 2 * NB * LDS * sizeof(float), st>>>(n, A, lda, j0, Di, d_info, d_pmin);
        BGPU_LAUNCH_CHECK();
        const int rest = n - j0 - nb;
        if (rest <= 0) break;
        float *A21 = A + (j0 + nb) + (long long)j0 * lda;
        trsm_panel_f32<<<ceil_div(rest, 64), 256, 0, st>>>(rest, nb, A21, lda, Di);
        BGPU_LAUNCH_CHECK();
        const int pc = J0 + JB - (j0 + nb);
        if (pc > 0) {
            syrk_f32<<<dim3(ceil_div(rest, SY_T), ceil_div(pc, SY_T)), 256, 0, st>>>(
                rest, pc, nb, A21, lda, A + (j0 + nb) + (long long)(j0 + nb) * lda, lda);
            BGPU_LAUNCH_CHECK();
        }
    }
    return BGPU_OK;
}

// A[C0.., C0 .. C0 + cols) -= P P' (lower part), P = A[C0.., P0 .. P0 + PB): the update of the
// columns from C0 on by the factored panel at P0
template <typename T>
int update_lower(cudaStream_t st, int n, T *A, long long lda, int C0, int cols, int P0, int PB);

template <>
int update_lower<double>(cudaStream_t st, int n, double *A, long long lda, int C0, int cols, int P0, int PB) {
    const double *P = A + C0 + (long long)P0 * lda;
    return gemm_f64(st, 0, 0, n - C0, cols, PB, -1.0, P, lda, 0, P, lda, 0, 1.0, A + C0 + (long long)C0 * lda, lda,
                    0, 1, 1);
}

template <>
int update_lower<float>(cudaStream_t st, int n, float *A, long long lda, int C0, int cols, int P0, int PB) {
    const float *P = A + C0 + (long long)P0 * lda;
    syrk_f32<<<dim3(ceil_div(n - C0, SY_T), ceil_div(cols, SY_T)), 256, 0, st>>>(n - C0, cols, PB, P, lda,
                                                                                 A + C0 + (long long)C0 * lda, lda);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

// Two streams of this host thread on this device for the look-ahead factor: `crit` (the highest
// priority: its CTAs go ahead of the waiting CTAs of the trailing update as SMs free up) and
// `bulk`, with the events that order them.  Created once per thread and device, kept for the
// life of the thread.
struct FactorStreams {
    cudaStream_t crit = nullptr, bulk = nullptr;
    cudaEvent_t fork = nullptr, panel = nullptr, trail = nullptr, done = nullptr;
    ~FactorStreams() {
        for (cudaEvent_t e : {fork, panel, trail, done})
            if (e) cudaEventDestroy(e);
        if (crit) cudaStreamDestroy(crit);
        if (bulk) cudaStreamDestroy(bulk);
    }
};

int factor_streams(FactorStreams **out) {
    int dev = 0;
    BGPU_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return BGPU_ERR_ARG;
    thread_local FactorStreams fs[64];
    FactorStreams &f = fs[dev];
    if (!f.crit) {
        int lo = 0, hi = 0;
        BGPU_CHECK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        BGPU_CHECK(cudaStreamCreateWithPriority(&f.crit, cudaStreamNonBlocking, hi));
        BGPU_CHECK(cudaStreamCreateWithPriority(&f.bulk, cudaStreamNonBlocking, lo));
        for (cudaEvent_t *e : {&f.fork, &f.panel, &f.trail, &f.done})
            BGPU_CHECK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    *out = &f;
    return BGPU_OK;
}

// The factor with a look-ahead of one panel.  On `crit`: factor panel k, update panel k+1's
// columns by it (U_next), factor panel k+1, ...; on `bulk`: update the columns from panel k+2 on
// by panel k (U_rest, the big rank-PANEL GEMM), while `crit` factors panel k+1.  Order: U_rest(k)
// waits for panel k's factor; U_next(k+1) writes panel k+2's columns, as U_rest(k) does, so it
// waits for U_rest(k).  The chain of diagonal-block factors then runs under the trailing updates
// instead of between them.  Small orders (three panels or fewer) run the plain order on `st`.
template <typename T>
int potrf_blocked(cudaStream_t st, int n, T *A, long long lda, T *dinv, int *d_info, double *d_pmin) {
    if (int rc = diag_smem_attr<T>()) return rc;
    init_info_kernel<<<1, 1, 0, st>>>(d_info, d_pmin);
    BGPU_LAUNCH_CHECK();
    const int np = ceil_div(n, PANEL);
    if (np <= 3) {
        for (int J0 = 0; J0 < n; J0 += PANEL) {
            const int JB = std::min(PANEL, n - J0);
            if (int rc = factor_panel<T>(st, n, A, lda, dinv, J0, JB, d_info, d_pmin)) return rc;
            if (J0 + JB < n)
                if (int rc = update_lower<T>(st, n, A, lda, J0 + JB, n - J0 - JB, J0, JB)) return rc;
        }
        return BGPU_OK;
    }
    FactorStreams *f = nullptr;
    if (int rc = factor_streams(&f)) return rc;
    BGPU_CHECK(cudaEventRecord(f->fork, st));
    BGPU_CHECK(cudaStreamWaitEvent(f->crit, f->fork, 0));
    BGPU_CHECK(cudaStreamWaitEvent(f->bulk, f->fork, 0));
    int rc = factor_panel<T>(f->crit, n, A, lda, dinv, 0, std::min(PANEL, n), d_info, d_pmin);
    for (int k = 0; rc == 0 && k + 1 < np; k++) {
        const int J0 = k * PANEL, JB = PANEL;            // panel k (not the last: full width)
        const int J1 = J0 + JB, JB1 = std::min(PANEL, n - J1);
        const int J2 = J1 + JB1;
        BGPU_CHECK(cudaEventRecord(f->panel, f->crit));
        if (J2 < n) {   // U_rest(k) on bulk, after panel k's factor
            BGPU_CHECK(cudaStreamWaitEvent(f->bulk, f->panel, 0));
            if ((rc = update_lower<T>(f->bulk, n, A, lda, J2, n - J2, J0, JB))) break;
            BGPU_CHECK(cudaEventRecord(f->trail, f->bulk));
        }
        // U_next(k) (panel k+1's columns by panel k), then panel k+1's factor, on crit.  Panel
        // k+1's columns took U_rest(k-1) before: crit waited for it ahead of U_next(k) below.
        if ((rc = update_lower<T>(f->crit, n, A, lda, J1, JB1, J0, JB))) break;
        if ((rc = factor_panel<T>(f->crit, n, A, lda, dinv, J1, JB1, d_info, d_pmin))) break;
        if (J2 < n) BGPU_CHECK(cudaStreamWaitEvent(f->crit, f->trail, 0));   // before U_next(k+1)
    }
    // join (also on an error: nothing is left running ahead of st)
    BGPU_CHECK(cudaEventRecord(f->done, f->bulk));
    BGPU_CHECK(cudaStreamWaitEvent(st, f->done, 0));
    BGPU_CHECK(cudaEventRecord(f->done, f->crit));
    BGPU_CHECK(cudaStreamWaitEvent(st, f->done, 0));
    return rc;
}
}  // namespace

int potrf_f64(cudaStream_t st, int n, double *A, long long lda, double *dinv, int *d_info, double *d_pmin) {
    return potrf_blocked<double>(st, n, A, lda, dinv, d_info, d_pmin);
}

int potrf_f32(cudaStream_t st, int n, float *A, long long lda, float *dinv, int *d_info, double *d_pmin) {
    return potrf_blocked<float>(st, n, A, lda, dinv, d_info, d_pmin);
}

int trsv_f64(cudaStream_t st, int n, const double *L, long long lda, const double *dinv, double *x, int trans,
             int *flags, int epoch, int *d_err) {
    return trsv_launch<double>(st, n, L, lda, dinv, x, trans, flags, epoch, d_err);
}
int trsv_f32(cudaStream_t st, int n, const float *L, long long lda, const float *dinv, float *x, int trans,
             int *flags, int epoch, int *d_err) {
    return trsv_launch<float>(st, n, L, lda, dinv, x, trans, flags, epoch, d_err);
}

int trtri_f64(cudaStream_t st, int n, const double *L, long long lda, const double *dinv, double *Linv,
              long long ldi) {
    // Solve L X = I by block rows: X_i = Dinv_i B_i, then B_below -= L(below, i) X_i.
    set_identity_lower_kernel<<<ceil_div((long long)n * n, 256), 256, 0, st>>>(n, Linv, ldi);
    BGPU_LAUNCH_CHECK();
    for (int i0 = 0; i0 < n; i0 += NB) {
        const int nb = (n - i0 < NB) ? n - i0 : NB;
        const int ncols = i0 + nb;   // columns 0..i0+nb-1 can be nonzero in block row i
        double *Xi = Linv + i0;      // rows i0.., all columns (ld ldi)
        // X_i <- Dinv_i X_i  (A = Dinv: A(r, k) = Dinv[r + k*NB], M-major; B = X_i K-major rows) in place, M <= 128
        int rc = gemm_f64(st, 0, 1, nb, ncols, nb, 1.0, dinv + (size_t)(i0 / NB) * NB * NB, NB, 0, Xi, ldi, 0, 0.0,
                          Xi, ldi, 0, 1, 0);
        if (rc) return rc;
        const int below = n - i0 - nb;
        if (below <= 0) break;
        // X_below -= L(below, i) X_i : A = L(i0+nb.., i0..) M-major, B(k, j) = X_i[k + j*ldi] K-major
        rc = gemm_f64(st, 0, 1, below, ncols, nb, -1.0, L + (i0 + nb) + (long long)i0 * lda, lda, 0, Xi, ldi, 0, 1.0,
                      Linv + (i0 + nb), ldi, 0, 1, 0);
        if (rc) return rc;
    }
    return BGPU_OK;
}

int symv_full_f64(cudaStream_t st, int n, double alpha, const double *M, long long ldm, const double *x, double beta,
                  double *y) {
    symv_full_kernel<<<ceil_div(n, 8), 256, 0, st>>>(n, alpha, M, ldm, x, beta, y);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int pattern_symv_f64(cudaStream_t st, int n, const long long *rowptr, const int *cols, const double *M, long long ldm,
                     const double *x, double *y) {
    if (n <= 0) return BGPU_OK;
    pattern_symv_kernel<<<ceil_div(n, 8), 256, 0, st>>>(n, rowptr, cols, M, ldm, x, y);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int schur_load_f64(cudaStream_t st, int m, const double *M, long long ldm, double reg, double *d_D, double *L,
                   long long ldl) {
    diag_scale_kernel<<<ceil_div(m, 256), 256, 0, st>>>(m, M, ldm, d_D);
    BGPU_LAUNCH_CHECK();
    load_scaled_f64_kernel<<<dim3(ceil_div(m, 256), m), 256, 0, st>>>(m, M, ldm, d_D, reg, L, ldl);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int schur_diag_scale(cudaStream_t st, int m, const double *M, long long ldm, double *d_D) {
    diag_scale_kernel<<<ceil_div(m, 256), 256, 0, st>>>(m, M, ldm, d_D);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int schur_load_f32(cudaStream_t st, int m, const double *M, long long ldm, double *d_D, float *Mf, long long ldf) {
    diag_scale_kernel<<<ceil_div(m, 256), 256, 0, st>>>(m, M, ldm, d_D);
    BGPU_LAUNCH_CHECK();
    load_scaled_f32_kernel<<<dim3(ceil_div(m, 256), m), 256, 0, st>>>(m, M, ldm, d_D, Mf, ldf);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int symmetrize_f64(cudaStream_t st, int n, double *A, long long lda) {
    symmetrize_kernel<<<dim3(ceil_div(n, 128), n), 128, 0, st>>>(n, A, lda);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int copy_lower_to_upper_f64(cudaStream_t st, int n, double *A, long long lda) {
    lower_to_upper_kernel<<<dim3(ceil_div(n, 128), n), 128, 0, st>>>(n, A, lda);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int dots_f64(cudaStream_t st, int nq, const double *const *a, const double *const *b, long long n, double *out,
             double *scratch) {
    if (nq <= 0) return BGPU_OK;
    dots_partial_kernel<<<dim3(DOT_PARTS, nq), 256, 0, st>>>(a, b, n, scratch);
    BGPU_LAUNCH_CHECK();
    dots_final_kernel<<<nq, 32, 0, st>>>(scratch, out);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

// ---- the triangular solve without caller-provided scratch ----------------------------------
// Some callers cannot allocate device memory where they solve: code between the steps of a loop
// where cudaMalloc / cudaFree would synchronize the device, or a process whose device memory is
// owned by another allocator (a framework's caching pool, a fixed budget).  For them,
// bgpu_trsv_noalloc keeps the block-row flags and the wait-error flag of the solve in this
// file-scope array instead of buffers the caller passes.  Every GPU that loads the library holds
// the array (8 KB) until the process exits.
//
// Its size limit is the solve's own: one CTA per block row of 64, all resident at once (a
// cooperative launch), so n <= 64 x (SMs x resident CTAs of trsv_kernel per SM); on a B200,
// 148 x 8 = 1184 block rows, n <= 75776.  The array holds 2048 block rows, more than any device
// of up to 256 SMs can keep resident.
#include <mutex>
#define BGPU_NOALLOC_TRSV_MAXBLK 2048
static __device__ __align__(256) int g_trsv_noalloc_scratch[BGPU_NOALLOC_TRSV_MAXBLK + 1];

namespace {
struct NoallocDev {
    int *ptr = nullptr;   // device address of g_trsv_noalloc_scratch on this device
    int epoch = 0;
};
constexpr int NOALLOC_MAXDEV = 64;
NoallocDev g_noalloc[NOALLOC_MAXDEV];
std::mutex g_noalloc_mu;
}  // namespace

extern "C" BGPU_API int bgpu_trsv_noalloc(int n, const double *d_L, int lda, const double *d_dinv, double *d_x,
                                          int trans, void *stream) {
    if (n <= 0 || lda < n || !d_L || !d_dinv || !d_x) return BGPU_ERR_ARG;
    const int nblk = (n + NB - 1) / NB;
    int cap = 0;
    if (int rc = trsv_max_blocks<double>(&cap)) return rc;
    cap = std::min(cap, BGPU_NOALLOC_TRSV_MAXBLK);
    if (nblk > cap) {
        fprintf(stderr,
                "bgpu_trsv_noalloc: n = %d needs %d block rows of %d; this device keeps at most %d resident at once "
                "(n <= %d)\n", n, nblk, NB, cap, cap * NB);
        return BGPU_ERR_TOOBIG;
    }
    int dev = 0;
    BGPU_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NOALLOC_MAXDEV) return BGPU_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    int *scratch = nullptr, epoch = 0;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        NoallocDev &d = g_noalloc[dev];
        if (!d.ptr) {
            // set-up on the first call on this device: the array's device address (the host-side
            // symbol is only a stand-in).  The array is zero when the module loads (static
            // device storage), and every epoch below is > 0, so no flag needs clearing here.
            void *p = nullptr;
            BGPU_CHECK(cudaGetSymbolAddress(&p, g_trsv_noalloc_scratch));
            d.ptr = (int *)p;
        }
        if (d.epoch == 0x7fffffff) {   // epochs exhausted: start over from cleared flags
            BGPU_CHECK(cudaMemsetAsync(d.ptr, 0, sizeof(int) * BGPU_NOALLOC_TRSV_MAXBLK, st));
            d.epoch = 0;
        }
        epoch = ++d.epoch;
        scratch = d.ptr;
    }
    int *err = scratch + BGPU_NOALLOC_TRSV_MAXBLK;
    BGPU_CHECK(cudaMemsetAsync(err, 0, sizeof(int), st));   // the error flag starts each call at 0
    int rc = trsv_launch<double>(st, n, d_L, lda, d_dinv, d_x, trans, scratch, epoch, err);
    if (rc) return rc;
    int h_err = 0;
    BGPU_CHECK(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    BGPU_CHECK(cudaStreamSynchronize(st));
    return h_err ? BGPU_ERR_TIMEOUT : BGPU_OK;
}
