// FP64 tensor-core GEMM for sm_100a (DMMA: mma.sync m16n8k4 .f64), cp.async 3-stage pipeline.
//
// C(i,j) = alpha * sum_k A(i,k) B(k,j) + beta * C(i,j), C column-major (C[i + j*ldc]).
//   A layout MMAJOR: A(i,k) = A[i + k*lda]   KMAJOR: A(i,k) = A[i*lda + k]
//   B layout KMAJOR: B(k,j) = B[k + j*ldb]   NMAJOR: B(k,j) = B[k*ldb + j]
// `lower` restricts the update to i >= j (a symmetric rank-k update of a lower triangle).
// Batched over blockIdx.z with element strides sA, sB, sC.  C may alias A or B when every
// CTA reads only the rows it writes (N <= 64 with A == C, or M <= 128 with B == C): all loads of
// a tile complete before its epilogue stores.  Tiles are 128 x BN with BN in {64, 80, 112, 128},
// chosen per call to pad N least (N = 400 -> 80, N = 1000 -> 112).
//
// Used for: the row-product Schur GEMM G = X (A_a Z^-1) (FP64 mode), the trailing updates
// of the blocked Cholesky of M and of X/Z, the HKM products Z^-1 dZ X, and the blocked
// triangular inverses.  FP64 on B200 has no tcgen05 kind, so DMMA is the tensor path.
#include "common.cuh"
#include "kernels.h"

namespace {
constexpr int BM = 128, BK = 16, NT = 256;
constexpr int LDA_M = BM + 8;   // smem stride for an MMAJOR A tile  [BK][BM+8]
constexpr int LDA_K = BK + 4;   // smem stride for a  KMAJOR A tile  [BM][BK+4]
constexpr int LDB_K = BK + 4;   // smem stride for a  KMAJOR B tile  [BN][BK+4]
constexpr int A_STAGE = (BK * LDA_M > BM * LDA_K) ? BK * LDA_M : BM * LDA_K;
// the N tile (64, 80, 112 or 128 columns): the launcher picks the one that pads N least
template <int BN>
struct TileN {
    // 3 stages keep two 64-wide CTAs per SM; the wider tiles (one CTA per SM) pipeline 4 deep
    static constexpr int STAGES = BN <= 64 ? 3 : 4;
    static constexpr int LDB_N = BN + 8;   // smem stride for an NMAJOR B tile  [BK][BN+8]
    static constexpr int B_STAGE = (BN * LDB_K > BK * LDB_N) ? BN * LDB_K : BK * LDB_N;
    static constexpr int NT8 = BN / 16;     // n8 tiles per warp (warps are 4 x 2)
    static constexpr size_t SMEM = (size_t)STAGES * (A_STAGE + B_STAGE) * sizeof(double);
};

__device__ __forceinline__ void dmma16(double (&c)[4], double a0, double a1, double b0) {
    asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
                 : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                 : "d"(a0), "d"(a1), "d"(b0));
}

// One BM x BN tile of C at (i0, j0).
template <bool A_KM, bool B_KM, int BN>
__device__ __forceinline__ void gemm_tile(int i0, int j0, int M, int N, int K, double alpha, const double *A,
                                          long long lda, const double *B, long long ldb, double beta, double *C,
                                          long long ldc, int lower, double *smem) {
    constexpr int LDB_N = TileN<BN>::LDB_N, B_STAGE = TileN<BN>::B_STAGE, NT8 = TileN<BN>::NT8;
    constexpr int STAGES = TileN<BN>::STAGES;
    double *As = smem;
    double *Bs = smem + STAGES * A_STAGE;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 3, wn = warp >> 2;          // 4 x 2 warps, 32 x BN/2 each
    const int g = lane >> 2, tig = lane & 3;
    const int nk = (K + BK - 1) / BK;

    auto load_stage = [&](int stage, int kt) {
        const int k0 = kt * BK;
        double *as = As + stage * A_STAGE;
        double *bs = Bs + stage * B_STAGE;
#pragma unroll
        for (int e = 0; e < (BM * BK) / NT; e++) {
            const int idx = tid + e * NT;
            if (A_KM) {
                const int i = idx / BK, k = idx % BK;
                const bool v = (i0 + i < M) && (k0 + k < K);
                const double *src = v ? A + (long long)(i0 + i) * lda + (k0 + k) : A;
                cp_async8(as + i * LDA_K + k, src, v);
            } else {
                const int k = idx / BM, i = idx % BM;
                const bool v = (i0 + i < M) && (k0 + k < K);
                const double *src = v ? A + (long long)(i0 + i) + (long long)(k0 + k) * lda : A;
                cp_async8(as + k * LDA_M + i, src, v);
            }
        }
#pragma unroll
        for (int e = 0; e < (BN * BK) / NT; e++) {
            const int idx = tid + e * NT;
            if (B_KM) {
                const int j = idx / BK, k = idx % BK;
                const bool v = (j0 + j < N) && (k0 + k < K);
                const double *src = v ? B + (long long)(k0 + k) + (long long)(j0 + j) * ldb : B;
                cp_async8(bs + j * LDB_K + k, src, v);
            } else {
                const int k = idx / BN, j = idx % BN;
                const bool v = (j0 + j < N) && (k0 + k < K);
                const double *src = v ? B + (long long)(k0 + k) * ldb + (j0 + j) : B;
                cp_async8(bs + k * LDB_N + j, src, v);
            }
        }
    };

    double acc[2][NT8][4];
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < NT8; b++)
#pragma unroll
            for (int c = 0; c < 4; c++) acc[a][b][c] = 0.0;

#pragma unroll
    for (int s = 0; s < STAGES - 1; s++) {
        if (s < nk) load_stage(s, s);
        cp_async_commit();
    }
    for (int kt = 0; kt < nk; kt++) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        {   // prefetch the stage STAGES-1 ahead (its buffer was consumed at kt-1)
            const int kn = kt + STAGES - 1;
            if (kn < nk) load_stage(kn % STAGES, kn);
            cp_async_commit();
        }
        const double *as = As + (kt % STAGES) * A_STAGE;
        const double *bs = Bs + (kt % STAGES) * B_STAGE;
#pragma unroll
        for (int kk = 0; kk < BK / 4; kk++) {
            const int k = kk * 4 + tig;
            double af[2][2], bf[NT8];
#pragma unroll
            for (int mt = 0; mt < 2; mt++) {
                const int r = wm * 32 + mt * 16 + g;
                if (A_KM) { af[mt][0] = as[r * LDA_K + k]; af[mt][1] = as[(r + 8) * LDA_K + k]; }
                else      { af[mt][0] = as[k * LDA_M + r]; af[mt][1] = as[k * LDA_M + r + 8]; }
            }
#pragma unroll
            for (int nt = 0; nt < NT8; nt++) {
                const int c = wn * (BN / 2) + nt * 8 + g;
                bf[nt] = B_KM ? bs[c * LDB_K + k] : bs[k * LDB_N + c];
            }
#pragma unroll
            for (int mt = 0; mt < 2; mt++)
#pragma unroll
                for (int nt = 0; nt < NT8; nt++) dmma16(acc[mt][nt], af[mt][0], af[mt][1], bf[nt]);
        }
    }
    cp_async_wait<0>();
    // epilogue: c0 (g, 2tig), c1 (g, 2tig+1), c2 (g+8, 2tig), c3 (g+8, 2tig+1)
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int nt = 0; nt < NT8; nt++)
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int i = i0 + wm * 32 + mt * 16 + g + (q >> 1) * 8;
                const int j = j0 + wn * (BN / 2) + nt * 8 + 2 * tig + (q & 1);
                if (i < M && j < N && (!lower || i >= j)) {
                    double *p = C + (long long)i + (long long)j * ldc;
                    const double v = alpha * acc[mt][nt][q];
                    *p = (beta == 0.0) ? v : v + beta * *p;
                }
            }
}

template <bool A_KM, bool B_KM, int BN>
__global__ void __launch_bounds__(NT, (BN <= 64) ? 2 : 1) dgemm_kernel(int M, int N, int K, double alpha,
                                                   const double *A, long long lda, long long sA,
                                                   const double *B, long long ldb, long long sB,
                                                   double beta, double *C, long long ldc, long long sC,
                                                   int lower) {
    extern __shared__ __align__(16) double smem[];
    // N tiles vary fastest: the CTAs that share an A row panel run together and reuse it from L2
    const int i0 = blockIdx.y * BM, j0 = blockIdx.x * BN;
    if (lower && i0 + BM - 1 < j0) return;   // tile entirely above the diagonal
    gemm_tile<A_KM, B_KM, BN>(i0, j0, M, N, K, alpha, A + (long long)blockIdx.z * sA, lda,
                              B + (long long)blockIdx.z * sB, ldb, beta, C + (long long)blockIdx.z * sC, ldc, lower,
                              smem);
}

// Grouped: CTA t computes tile (tiles[t].y, tiles[t].z) (row, column tile index) of group
// tiles[t].x, each group with its own sizes and operands (A K-major, B K-major, C lower).
__global__ void __launch_bounds__(NT, 2) dgemm_grouped_kernel(const int4 *__restrict__ tiles,
                                                              const GemmGroup *__restrict__ groups, double alpha,
                                                              double beta) {
    extern __shared__ __align__(16) double smem[];
    const int4 t = tiles[blockIdx.x];
    const GemmGroup gr = groups[t.x];
    gemm_tile<true, true, 64>(t.y * BM, t.z * 64, gr.M, gr.N, gr.K, alpha, gr.A, gr.lda, gr.B, gr.ldb, beta, gr.C,
                              gr.ldc, 1, smem);
}

template <bool A_KM, bool B_KM, int BN>
int launch(cudaStream_t st, int M, int N, int K, double alpha, const double *A, long long lda, long long sA,
           const double *B, long long ldb, long long sB, double beta, double *C, long long ldc, long long sC,
           int batch, int lower) {
    BGPU_ATTR_ONCE(BGPU_CHECK(cudaFuncSetAttribute(dgemm_kernel<A_KM, B_KM, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)TileN<BN>::SMEM)));
    if (ceil_div(M, BM) > 65535) return BGPU_ERR_TOOBIG;
    dim3 grid(ceil_div(N, BN), ceil_div(M, BM), batch);
    dgemm_kernel<A_KM, B_KM, BN><<<grid, NT, TileN<BN>::SMEM, st>>>(M, N, K, alpha, A, lda, sA, B, ldb, sB, beta, C,
                                                                    ldc, sC, lower);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

template <bool A_KM, bool B_KM>
int launch_bn(cudaStream_t st, int M, int N, int K, double alpha, const double *A, long long lda, long long sA,
              const double *B, long long ldb, long long sB, double beta, double *C, long long ldc, long long sC,
              int batch, int lower) {
    // the N tile that pads N least (ties to the wider); N <= 64 always takes 64
    const int cand[4] = {128, 112, 80, 64};
    int best = 64;
    long long pad = 1LL << 60;
    for (int c : cand) {
        const long long p = (long long)ceil_div(N, c) * c;
        if (p < pad) { pad = p; best = c; }
    }
    switch (best) {
        case 128: return launch<A_KM, B_KM, 128>(st, M, N, K, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC, batch, lower);
        case 112: return launch<A_KM, B_KM, 112>(st, M, N, K, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC, batch, lower);
        case 80: return launch<A_KM, B_KM, 80>(st, M, N, K, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC, batch, lower);
        default: return launch<A_KM, B_KM, 64>(st, M, N, K, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC, batch, lower);
    }
}
}  // namespace

int gemm_f64(cudaStream_t st, int a_kmajor, int b_kmajor, int M, int N, int K, double alpha, const double *A,
             long long lda, long long sA, const double *B, long long ldb, long long sB, double beta, double *C,
             long long ldc, long long sC, int batch, int lower) {
    if (M <= 0 || N <= 0 || batch <= 0) return BGPU_OK;
    if (K <= 0) {   // C = beta C
        if (beta == 1.0) return BGPU_OK;
        return scale_matrix_f64(st, M, N, beta, C, ldc, sC, batch, lower);
    }
    if (a_kmajor) {
        if (b_kmajor) return launch_bn<true, true>(st, M, N, K, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC, batch, lower);
        return launch_bn<true, false>(st, M, N, K, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC, batch, lower);
    }
    if (b_kmajor) return launch_bn<false, true>(st, M, N, K, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC, batch, lower);
    return launch_bn<false, false>(st, M, N, K, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC, batch, lower);
}

namespace {
__global__ void scale_kernel(int M, int N, double beta, double *C, long long ldc, long long sC, int lower) {
    C += (long long)blockIdx.z * sC;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i < M && j < N && (!lower || i >= j)) C[i + (long long)j * ldc] *= beta;
}
}  // namespace

int gemm_f64_grouped(cudaStream_t st, int ntiles, const int4 *d_tiles, const GemmGroup *d_groups, double alpha,
                     double beta) {
    if (ntiles <= 0) return BGPU_OK;
    BGPU_ATTR_ONCE(BGPU_CHECK(cudaFuncSetAttribute(dgemm_grouped_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)TileN<64>::SMEM)));
    dgemm_grouped_kernel<<<ntiles, NT, TileN<64>::SMEM, st>>>(d_tiles, d_groups, alpha, beta);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int gemm_grouped_tile_rows() { return BM; }

int scale_matrix_f64(cudaStream_t st, int M, int N, double beta, double *C, long long ldc, long long sC, int batch,
                     int lower) {
    dim3 grid(ceil_div(M, 256), N, batch);
    scale_kernel<<<grid, 256, 0, st>>>(M, N, beta, C, ldc, sC, lower);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}
