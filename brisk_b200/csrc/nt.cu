// The Nesterov-Todd scaling point of SDP blocks (nt.h), after the reference's nt_scaling
// (solver.c:7803-7912): the same G, lam and W = G G' from the Cholesky factors of X and Z.
//
// The reference takes V, the right singular vectors of Mb = L_Z' L_X, from the eigenvectors of
// Mb' Mb (LAPACK dsyevd; dgesdd when that fails).  Here V comes from one-sided (Hestenes) Jacobi on
// Mb itself: plane rotations of column pairs until every pair is orthogonal to working precision
// (|a_p' a_q| <= sqrt(n) eps |a_p| |a_q|), the same rotations applied to L_X, so that the rotated L_X
// is L_X V and the rotated Mb's column norms are the singular values lam (no squared eigenvalues).
// The rotation of a pair is the classical one: zeta = (|a_q|^2 - |a_p|^2) / (2 a_p' a_q),
// t = sign(zeta) / (|zeta| + sqrt(1 + zeta^2)), c = 1 / sqrt(1 + t^2), s = c t,
// (a_p, a_q) <- (c a_p - s a_q, s a_p + c a_q).
//
// Small blocks (n <= 64): one CTA per block, Mb and L_X in shared memory, the n/2 disjoint pairs of
// a round (round-robin order) rotated at once by groups of lanes.  Large blocks: the columns in
// groups of b, the groups paired round-robin, one CTA per pair of groups: the 2b x 2b Gram matrix
// of its columns, diagonalised by cyclic Jacobi in shared memory, then both matrices' columns
// multiplied by its eigenvectors (block one-sided Jacobi); the host checks convergence once a sweep.
#include <cfloat>
#include <mutex>
#include <vector>
#include "common.cuh"
#include "nt.h"

namespace nt {
namespace {

// Pair i of round r in the round-robin order of np (even) players: every pair meets once in np - 1
// rounds, and the pairs of a round are disjoint.
__device__ __forceinline__ void rr_pair(int np, int r, int i, int &p, int &q) {
    const int K = np - 1;
    if (i == 0) {
        p = r;
        q = K;
    } else {
        p = (r + i) % K;
        q = (r - i + K) % K;
    }
}

// the rotation that makes columns with squared norms a, b and inner product c orthogonal
__device__ __forceinline__ void rotation(double a, double b, double c, double &cs, double &sn) {
    const double zeta = (b - a) / (2.0 * c);
    const double az = fabs(zeta);
    const double t = az > 1e150 ? 0.5 / zeta : (zeta >= 0 ? 1.0 : -1.0) / (az + sqrt(1.0 + zeta * zeta));
    cs = 1.0 / sqrt(1.0 + t * t);
    sn = cs * t;
}

__device__ __forceinline__ double jacobi_tol(int n) { return sqrt((double)n) * DBL_EPSILON; }

// ---- small blocks ----------------------------------------------------------------------------
constexpr int SM_THREADS = 256;
__host__ __device__ __forceinline__ int small_ld(int n) { return n | 1; }   // odd: fewer bank conflicts

__global__ void __launch_bounds__(SM_THREADS) scaling_small_kernel(const int *__restrict__ ns,
                                                                   const double *const *LXt, const double *const *LZt,
                                                                   double *const *Gt, double *const *lamt,
                                                                   double *const *Wt, int *info) {
    extern __shared__ double sm[];
    __shared__ double slam[SMALL_NMAX];
    __shared__ int rotated, bad;
    const int k = blockIdx.x, n = ns[k], ld = small_ld(n), tid = threadIdx.x;
    double *A = sm;                          // Mb = L_Z' L_X
    double *U = sm + (size_t)ld * n;         // L_X, rotated into L_X V, then G
    double *Zt = U + (size_t)ld * n;         // L_Z transposed: Zt[i + kk ld] = L_Z(kk, i)
    const double *LX = LXt[k], *LZ = LZt[k];
    for (int e = tid; e < n * n; e += SM_THREADS) {
        const int i = e % n, j = e / n;
        U[i + j * ld] = i >= j ? LX[e] : 0.0;
        Zt[j + i * ld] = i >= j ? LZ[e] : 0.0;   // L_Z(i, j) at (j, i)
    }
    __syncthreads();
    for (int e = tid; e < n * n; e += SM_THREADS) {
        const int i = e % n, j = e / n;
        double s = 0.0;   // sum over kk >= max(i, j) of L_Z(kk, i) L_X(kk, j)
        for (int kk = i > j ? i : j; kk < n; kk++) s += Zt[i + kk * ld] * U[kk + j * ld];
        A[i + j * ld] = s;
    }
    __syncthreads();
    const int np = n + (n & 1), npairs = np / 2;
    int g = 32;   // lanes per pair: a power of two, so a group lies within one warp
    while (g > 1 && g * npairs > SM_THREADS) g >>= 1;
    const int pi = tid / g, l = tid % g;
    const double tol = jacobi_tol(n);
    bool conv = false;
    for (int sweep = 0; sweep < MAX_SWEEPS; sweep++) {
        if (tid == 0) rotated = 0;
        __syncthreads();
        for (int r = 0; r < np - 1; r++) {
            int p = 0, q = 0;
            bool act = pi < npairs;
            if (act) {
                rr_pair(np, r, pi, p, q);
                act = p < n && q < n;   // the extra player of odd n sits out
            }
            double a = 0.0, b = 0.0, c = 0.0;
            if (act)
                for (int i = l; i < n; i += g) {
                    const double x = A[i + p * ld], y = A[i + q * ld];
                    a += x * x;
                    b += y * y;
                    c += x * y;
                }
            for (int o = g >> 1; o > 0; o >>= 1) {   // every lane of the group ends with the same sums
                a += __shfl_xor_sync(0xffffffffu, a, o);
                b += __shfl_xor_sync(0xffffffffu, b, o);
                c += __shfl_xor_sync(0xffffffffu, c, o);
            }
            if (act && fabs(c) > tol * sqrt(a * b)) {
                double cs, sn;
                rotation(a, b, c, cs, sn);
                for (int i = l; i < n; i += g) {
                    const double x = A[i + p * ld], y = A[i + q * ld];
                    A[i + p * ld] = cs * x - sn * y;
                    A[i + q * ld] = sn * x + cs * y;
                    const double u = U[i + p * ld], v = U[i + q * ld];
                    U[i + p * ld] = cs * u - sn * v;
                    U[i + q * ld] = sn * u + cs * v;
                }
                if (l == 0) rotated = 1;
            }
            __syncthreads();
        }
        const int rot = rotated;
        __syncthreads();
        if (!rot) {
            conv = true;
            break;
        }
    }
    if (tid == 0) bad = conv ? 0 : 2;
    __syncthreads();
    const int warp = tid / 32, lane = tid % 32;
    for (int j = warp; j < n; j += SM_THREADS / 32) {
        double s = 0.0;
        for (int i = lane; i < n; i += 32) s += A[i + j * ld] * A[i + j * ld];
        s = warp_sum(s);
        const double lam = sqrt(s);
        if (lane == 0) {
            slam[j] = lam;
            if (!(lam > 0.0) || !isfinite(lam)) bad = 1;
        }
    }
    __syncthreads();
    double *G = Gt[k], *lamk = lamt[k], *W = Wt[k];
    for (int e = tid; e < n * n; e += SM_THREADS) {
        const int i = e % n, j = e / n;
        const double v = U[i + j * ld] / sqrt(slam[j]);
        U[i + j * ld] = v;
        G[e] = v;
    }
    for (int i = tid; i < n; i += SM_THREADS) lamk[i] = slam[i];
    __syncthreads();
    for (int e = tid; e < n * n; e += SM_THREADS) {   // W = G G', the lower triangle mirrored
        const int i = e % n, j = e / n;
        if (i < j) continue;
        double s = 0.0;
        for (int kk = 0; kk < n; kk++) s += U[i + kk * ld] * U[j + kk * ld];
        W[i + j * n] = s;
        W[j + i * n] = s;
    }
    if (tid == 0) info[k] = bad;
}

// ---- large blocks ----------------------------------------------------------------------------
constexpr int BS_THREADS = 256;
constexpr int BS_ROWS = 64;          // rows per shared-memory tile
// Sweeps of cyclic Jacobi on a pair's Gram matrix: one is enough (the outer iteration converges in
// as many sweeps as with the Gram matrix fully diagonalised, measured on graded matrices of order
// 100 and condition 1e12 for groups of 1 to 16 columns)
constexpr int INNER_SWEEPS = 1;

// Cyclic Jacobi on the P x P Gram matrix C by one warp: C <- Q' C Q (Q accumulated from the
// identity) until every off-diagonal pair passes the test, at most INNER_SWEEPS sweeps.
template <int P>
__device__ void gram_jacobi(double (*C)[P + 1], double (*Q)[P + 1], double *rcs, double *rsn, int *rfl, double tol) {
    constexpr int E = P * P;
    const int lane = threadIdx.x % 32;
    for (int x = lane; x < E; x += 32) Q[x / P][x % P] = (x / P == x % P) ? 1.0 : 0.0;
    __syncwarp();
    for (int sw = 0; sw < INNER_SWEEPS; sw++) {
        bool any = false;
        for (int rr = 0; rr < P - 1; rr++) {
            int f = 0;
            if (lane < P / 2) {
                int p, q;
                rr_pair(P, rr, lane, p, q);
                const double a = C[p][p], b = C[q][q], c = C[p][q];
                double cs = 1.0, sn = 0.0;
                if (fabs(c) > tol * sqrt(a * b)) {
                    rotation(a, b, c, cs, sn);
                    f = 1;
                }
                rcs[lane] = cs;
                rsn[lane] = sn;
                rfl[lane] = f;
            }
            const bool rot = __any_sync(0xffffffffu, f) != 0;
            __syncwarp();
            if (!rot) continue;
            any = true;
            for (int x = lane; x < (P / 2) * P; x += 32) {   // columns p, q of C and Q
                const int pr = x / P, kk = x % P;
                if (!rfl[pr]) continue;
                int p, q;
                rr_pair(P, rr, pr, p, q);
                const double cs = rcs[pr], sn = rsn[pr];
                const double u = C[kk][p], v = C[kk][q];
                C[kk][p] = cs * u - sn * v;
                C[kk][q] = sn * u + cs * v;
                const double qu = Q[kk][p], qv = Q[kk][q];
                Q[kk][p] = cs * qu - sn * qv;
                Q[kk][q] = sn * qu + cs * qv;
            }
            __syncwarp();
            for (int x = lane; x < (P / 2) * P; x += 32) {   // rows p, q of C
                const int pr = x / P, kk = x % P;
                if (!rfl[pr]) continue;
                int p, q;
                rr_pair(P, rr, pr, p, q);
                const double cs = rcs[pr], sn = rsn[pr];
                const double u = C[p][kk], v = C[q][kk];
                C[p][kk] = cs * u - sn * v;
                C[q][kk] = sn * u + cs * v;
            }
            __syncwarp();
            if (lane < P / 2 && rfl[lane]) {
                int p, q;
                rr_pair(P, rr, lane, p, q);
                C[p][q] = 0.0;
                C[q][p] = 0.0;
            }
            __syncwarp();
        }
        if (!any) break;
    }
}

// One round of a sweep: CTA c takes the column groups (I, J) of pair c of round r (groups of P/2
// columns; nblk groups, nbe = nblk rounded up to even; a group >= nblk is empty).
template <int P>
__global__ void __launch_bounds__(BS_THREADS) block_step_kernel(int n, double *__restrict__ Mb, double *__restrict__ U,
                                                                int r, int nblk, int nbe, double tol, int *notconv) {
    constexpr int B = P / 2, E = P * P, PARTS = BS_THREADS / E, RPART = BS_ROWS / PARTS, TL = P + 1;
    static_assert(BS_THREADS % E == 0 && BS_ROWS % PARTS == 0, "tile shape");
    __shared__ double tile[BS_ROWS * TL];
    __shared__ double C[P][P + 1], Q[P][P + 1];
    __shared__ double part[BS_THREADS];
    __shared__ double rcs[P / 2], rsn[P / 2];
    __shared__ int rfl[P / 2];
    __shared__ int cols[P];
    __shared__ int need;
    const int tid = threadIdx.x;
    int I, J;
    rr_pair(nbe, r, blockIdx.x, I, J);
    if (tid < P) {
        const int gI = tid < B ? I : J, c = gI * B + tid % B;
        cols[tid] = (gI < nblk && c < n) ? c : -1;
    }
    __syncthreads();
    // the Gram matrix of the 2b columns: thread (e, part) sums its rows of every tile
    const int e = tid % E, pid = tid / E, gp = e / P, gq = e % P;
    double acc = 0.0;
    for (int i0 = 0; i0 < n; i0 += BS_ROWS) {
        for (int x = tid; x < BS_ROWS * P; x += BS_THREADS) {
            const int i = x % BS_ROWS, p = x / BS_ROWS, c = cols[p];
            tile[i * TL + p] = (c >= 0 && i0 + i < n) ? Mb[(i0 + i) + (long long)c * n] : 0.0;
        }
        __syncthreads();
        for (int i = pid * RPART; i < (pid + 1) * RPART; i++) acc += tile[i * TL + gp] * tile[i * TL + gq];
        __syncthreads();
    }
    part[tid] = acc;
    __syncthreads();
    if (tid < E) {
        double s = 0.0;
        for (int t = 0; t < PARTS; t++) s += part[t * E + tid];
        C[tid / P][tid % P] = s;
    }
    __syncthreads();
    if (tid < 32) {   // any pair of the 2b columns not yet orthogonal
        int nd = 0;
        for (int x = tid; x < E; x += 32) {
            const int p = x / P, q = x % P;
            if (p < q && fabs(C[p][q]) > tol * sqrt(C[p][p] * C[q][q])) nd = 1;
        }
        nd = __any_sync(0xffffffffu, nd);
        if (tid == 0) {
            need = nd;
            if (nd) atomicExch(notconv, 1);
        }
    }
    __syncthreads();
    if (!need) return;
    if (tid < 32) gram_jacobi<P>(C, Q, rcs, rsn, rfl, tol);   // warp 0: C <- Q' C Q
    __syncthreads();
    // the columns of Mb and U times Q
    for (int mat = 0; mat < 2; mat++) {
        double *Xm = mat ? U : Mb;
        for (int i0 = 0; i0 < n; i0 += BS_ROWS) {
            for (int x = tid; x < BS_ROWS * P; x += BS_THREADS) {
                const int i = x % BS_ROWS, p = x / BS_ROWS, c = cols[p];
                tile[i * TL + p] = (c >= 0 && i0 + i < n) ? Xm[(i0 + i) + (long long)c * n] : 0.0;
            }
            __syncthreads();
            for (int x = tid; x < BS_ROWS * P; x += BS_THREADS) {
                const int i = x % BS_ROWS, q = x / BS_ROWS, c = cols[q];
                if (c < 0 || i0 + i >= n) continue;
                double s = 0.0;
#pragma unroll
                for (int p = 0; p < P; p++) s += tile[i * TL + p] * Q[p][q];
                Xm[(i0 + i) + (long long)c * n] = s;
            }
            __syncthreads();
        }
    }
}

// The same round with the pair's columns of Mb staged in shared memory (ldm = n rounded up to
// odd: the Gram reads of different columns fall in different banks): one load, the Gram matrix,
// the Jacobi of C, then each thread rotates whole rows of Mb (from shared memory) and of U.
template <int P>
__global__ void __launch_bounds__(BS_THREADS) block_step_smem_kernel(int n, double *__restrict__ Mb,
                                                                     double *__restrict__ U, int r, int nblk, int nbe,
                                                                     double tol, int *notconv, int stage_u) {
    constexpr int B = P / 2, E = P * P, PARTS = BS_THREADS / E;
    static_assert(BS_THREADS % E == 0, "tile shape");
    extern __shared__ double Ms[];   // column p of the pair at Ms + p ldm; U's columns after (stage_u)
    __shared__ double C[P][P + 1], Q[P][P + 1];
    __shared__ double part[BS_THREADS];
    __shared__ double rcs[P / 2], rsn[P / 2];
    __shared__ int rfl[P / 2];
    __shared__ int cols[P];
    __shared__ int need;
    const int tid = threadIdx.x, ldm = n | 1;
    int I, J;
    rr_pair(nbe, r, blockIdx.x, I, J);
    if (tid < P) {
        const int gI = tid < B ? I : J, c = gI * B + tid % B;
        cols[tid] = (gI < nblk && c < n) ? c : -1;
    }
    __syncthreads();
    double *Us = Ms + (size_t)P * ldm;
    // every load in flight at once (asynchronous copies): Mb's columns, then U's (used at the end)
    for (int p = 0; p < P; p++) {
        const int c = cols[p];
        for (int i = tid; i < n; i += BS_THREADS) cp_async8(&Ms[i + p * ldm], Mb + i + (long long)(c < 0 ? 0 : c) * n, c >= 0);
    }
    cp_async_commit();
    if (stage_u) {
        for (int p = 0; p < P; p++) {
            const int c = cols[p];
            for (int i = tid; i < n; i += BS_THREADS) cp_async8(&Us[i + p * ldm], U + i + (long long)(c < 0 ? 0 : c) * n, c >= 0);
        }
    }
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    {   // the Gram matrix: thread (e, part) sums rows part, part + PARTS, ...
        const int e = tid % E, pid = tid / E, gp = e / P, gq = e % P;
        double acc = 0.0;
        for (int i = pid; i < n; i += PARTS) acc += Ms[i + gp * ldm] * Ms[i + gq * ldm];
        part[tid] = acc;
    }
    __syncthreads();
    if (tid < E) {
        double s = 0.0;
        for (int t = 0; t < PARTS; t++) s += part[t * E + tid];
        C[tid / P][tid % P] = s;
    }
    __syncthreads();
    if (tid < 32) {   // any pair of the 2b columns not yet orthogonal
        int nd = 0;
        for (int x = tid; x < E; x += 32) {
            const int p = x / P, q = x % P;
            if (p < q && fabs(C[p][q]) > tol * sqrt(C[p][p] * C[q][q])) nd = 1;
        }
        nd = __any_sync(0xffffffffu, nd);
        if (tid == 0) {
            need = nd;
            if (nd) atomicExch(notconv, 1);
        }
    }
    __syncthreads();
    if (!need) {
        cp_async_wait<0>();   // no copy may still write shared memory when the CTA ends
        return;
    }
    if (tid < 32) gram_jacobi<P>(C, Q, rcs, rsn, rfl, tol);   // warp 0: C <- Q' C Q
    cp_async_wait<0>();
    __syncthreads();
    for (int i = tid; i < n; i += BS_THREADS) {   // rows of Mb and U times Q
        double a[P], u[P];
#pragma unroll
        for (int p = 0; p < P; p++) {
            a[p] = Ms[i + p * ldm];
            u[p] = stage_u ? Us[i + p * ldm] : (cols[p] >= 0 ? U[i + (long long)cols[p] * n] : 0.0);
        }
#pragma unroll
        for (int q = 0; q < P; q++) {
            if (cols[q] < 0) continue;
            double sa = 0.0, su = 0.0;
#pragma unroll
            for (int p = 0; p < P; p++) {
                sa += a[p] * Q[p][q];
                su += u[p] * Q[p][q];
            }
            Mb[i + (long long)cols[q] * n] = sa;
            U[i + (long long)cols[q] * n] = su;
        }
    }
}

__global__ void finish_kernel(int n, const double *__restrict__ Mb, double *__restrict__ U, double *__restrict__ lam,
                              int *info) {
    const int j = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32), lane = threadIdx.x % 32;
    if (j >= n) return;
    double s = 0.0;
    for (int i = lane; i < n; i += 32) {
        const double v = Mb[i + (long long)j * n];
        s += v * v;
    }
    s = warp_sum(s);
    const double l = sqrt(s);
    const bool ok = l > 0.0 && isfinite(l);
    if (lane == 0) {
        lam[j] = l;
        if (!ok) atomicExch(info, 1);
    }
    if (!ok) return;
    const double f = 1.0 / sqrt(l);
    for (int i = lane; i < n; i += 32) U[i + (long long)j * n] *= f;
}

__global__ void tril_kernel(int n, const double *__restrict__ L, double *__restrict__ out) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)n * n) return;
    const int i = (int)(e % n), j = (int)(e / n);
    out[e] = i >= j ? L[e] : 0.0;
}

// ---- element-wise pieces over the concatenation ----------------------------------------------
__device__ __forceinline__ int block_of(long long g, int nb, const long long *__restrict__ off) {
    int lo = 0, hi = nb - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void rhs_scaled_kernel(int nb, const int *__restrict__ ns, const long long *__restrict__ off,
                                  const long long *__restrict__ loff, long long total, const double *__restrict__ lam,
                                  double smu, const double *__restrict__ H, double *__restrict__ Rt,
                                  const double *__restrict__ smu_blk) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    const int k = block_of(g, nb, off), n = ns[k];
    const long long l = g - off[k];
    const int j = (int)(l / n), i = (int)(l - (long long)j * n);
    const double li = lam[loff[k] + i], lj = lam[loff[k] + j];
    double v = -2.0 * (H ? H[g] : 0.0) / (li + lj);
    if (i == j) v += (smu_blk ? smu_blk[k] : smu) / li - li;
    Rt[g] = v;
}

__global__ void add_lam_kernel(int nb, const int *__restrict__ ns, const long long *__restrict__ off,
                               const long long *__restrict__ loff, long long total, const double *__restrict__ lam,
                               double alpha, const double *src, double *out) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    const int k = block_of(g, nb, off), n = ns[k];
    const long long l = g - off[k];
    const int j = (int)(l / n), i = (int)(l - (long long)j * n);
    double v = src[g];
    if (i == j) v += alpha * lam[loff[k] + i];
    out[g] = v;
}

}  // namespace

int scaling_small(cudaStream_t st, int nb, const int *d_n, int nmax, const double *const *LX, const double *const *LZ,
                  double *const *G, double *const *lam, double *const *W, int *info) {
    if (nb <= 0) return BGPU_OK;
    if (nmax < 1 || nmax > SMALL_NMAX) return BGPU_ERR_ARG;
    const size_t smem = sizeof(double) * 3 * (size_t)small_ld(nmax) * nmax;
    BGPU_ATTR_ONCE(BGPU_CHECK(cudaFuncSetAttribute(scaling_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)(sizeof(double) * 3 * small_ld(SMALL_NMAX) * SMALL_NMAX))));
    scaling_small_kernel<<<nb, SM_THREADS, smem, st>>>(d_n, LX, LZ, G, lam, W, info);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int tril(cudaStream_t st, int n, const double *L, double *out) {
    if (n <= 0) return BGPU_OK;
    const long long nn = (long long)n * n;
    tril_kernel<<<ceil_div(nn, 256), 256, 0, st>>>(n, L, out);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

namespace {
// One sweep's launches (the flag's reset and every round) as a CUDA graph, instantiated once per
// (n, Mb, U, flag) and replayed each sweep: the rounds then follow one another without a host
// launch between them.  At most 32 graphs are kept (the oldest is dropped).
struct SweepGraph {
    int n;
    const double *Mb, *U;
    const int *flag;
    cudaGraphExec_t exec;
};
std::mutex g_graph_mu;
std::vector<SweepGraph> g_graphs;

struct SweepShape {
    bool staged, stage_u;
    size_t smem;
    int P, nblk, nbe;
    double tol;
    explicit SweepShape(int n) {
        // groups of 4 columns (8-column pairs) with the pair's columns of Mb in shared memory while
        // they fit (n <= 3500; U's columns as well below n = 1750); above, groups of 8 streamed
        // through shared-memory tiles
        const size_t col8 = sizeof(double) * 8 * (size_t)(n | 1);
        staged = col8 <= 224 * 1024;
        stage_u = 2 * col8 <= 224 * 1024;
        smem = stage_u ? 2 * col8 : col8;
        P = staged ? 8 : 16;
        nblk = ceil_div(n, P / 2);
        nbe = nblk + (nblk & 1);
        tol = std::sqrt((double)n) * DBL_EPSILON;
    }
};

int launch_sweep(cudaStream_t st, int n, const SweepShape &sh, double *Mb, double *U, int *d_flag) {
    BGPU_CHECK(cudaMemsetAsync(d_flag, 0, sizeof(int), st));
    for (int r = 0; r < sh.nbe - 1; r++) {
        if (sh.staged)
            block_step_smem_kernel<8><<<sh.nbe / 2, BS_THREADS, sh.smem, st>>>(n, Mb, U, r, sh.nblk, sh.nbe, sh.tol,
                                                                               d_flag, sh.stage_u);
        else block_step_kernel<16><<<sh.nbe / 2, BS_THREADS, 0, st>>>(n, Mb, U, r, sh.nblk, sh.nbe, sh.tol, d_flag);
        BGPU_LAUNCH_CHECK();
    }
    return BGPU_OK;
}

// the cached graph of a sweep, or nullptr where the stream cannot be captured (the legacy
// default stream) or the capture failed
cudaGraphExec_t sweep_graph(cudaStream_t st, int n, const SweepShape &sh, double *Mb, double *U, int *d_flag) {
    if (st == nullptr) return nullptr;
    std::lock_guard<std::mutex> lk(g_graph_mu);
    for (auto &e : g_graphs)
        if (e.n == n && e.Mb == Mb && e.U == U && e.flag == d_flag) return e.exec;
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    const int rc = launch_sweep(st, n, sh, Mb, U, d_flag);
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(st, &graph);
    cudaGraphExec_t exec = nullptr;
    if (rc || ce != cudaSuccess || !graph || cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) exec = nullptr;
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    if (!exec) return nullptr;
    if (g_graphs.size() >= 32) {
        cudaGraphExecDestroy(g_graphs.front().exec);
        g_graphs.erase(g_graphs.begin());
    }
    g_graphs.push_back({n, Mb, U, d_flag, exec});
    return exec;
}
}  // namespace

int jacobi(cudaStream_t st, int n, double *Mb, double *U, int *d_flag, int *h_flag, int *sweeps) {
    *sweeps = -1;
    if (n <= 0) {
        *sweeps = 0;
        return BGPU_OK;
    }
    const SweepShape sh(n);
    if (sh.staged)
        BGPU_CHECK(cudaFuncSetAttribute(block_step_smem_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)sh.smem));
    cudaGraphExec_t exec = sweep_graph(st, n, sh, Mb, U, d_flag);
    for (int s = 0; s < MAX_SWEEPS; s++) {
        if (exec) {
            BGPU_CHECK(cudaGraphLaunch(exec, st));
            __atomic_add_fetch(&g_bgpu_launches, sh.nbe - 1, __ATOMIC_RELAXED);
        } else if (int rc = launch_sweep(st, n, sh, Mb, U, d_flag)) {
            return rc;
        }
        BGPU_CHECK(cudaMemcpyAsync(h_flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, st));
        BGPU_CHECK(cudaStreamSynchronize(st));
        if (!*h_flag) {
            *sweeps = s + 1;
            return BGPU_OK;
        }
    }
    return BGPU_OK;
}

int finish(cudaStream_t st, int n, const double *Mb, double *U, double *lam, int *d_info) {
    if (n <= 0) return BGPU_OK;
    finish_kernel<<<ceil_div((long long)n * 32, 256), 256, 0, st>>>(n, Mb, U, lam, d_info);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int rhs_scaled(cudaStream_t st, int nb, const int *d_n, const long long *d_off, const long long *d_loff,
               long long total, const double *lam, double smu, const double *H, double *Rt, const double *d_smu) {
    if (total <= 0) return BGPU_OK;
    rhs_scaled_kernel<<<ceil_div(total, 256), 256, 0, st>>>(nb, d_n, d_off, d_loff, total, lam, smu, H, Rt, d_smu);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int add_lam(cudaStream_t st, int nb, const int *d_n, const long long *d_off, const long long *d_loff,
            long long total, const double *lam, double alpha, const double *src, double *out) {
    if (total <= 0) return BGPU_OK;
    add_lam_kernel<<<ceil_div(total, 256), 256, 0, st>>>(nb, d_n, d_off, d_loff, total, lam, alpha, src, out);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

}  // namespace nt
