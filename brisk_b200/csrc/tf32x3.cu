// 3xTF32 split-product GEMM on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// G = A B with A = Ah + Al and B = Bh + Bl, each part tf32-rounded, computed as
// Ah Bh + Ah Bl + Al Bh with FP32 accumulation in tensor memory: FP32-level accuracy at
// three tf32 MMAs per product (the dropped Al Bl term is below FP32 rounding).
//
// One CTA per 128 x BN output tile (cta_group::1):
//   warp 0 / lane 0  TMA producer: 4 operand tiles (Ah, Al, Bh, Bl: 32 fp32 of K x 128 or BN
//                    rows, 128-byte swizzle) per k-block into a STAGES-deep ring, one mbarrier
//                    with the transaction count per stage
//   warp 1 / lane 0  MMA issuer: 4 K-steps of 8 x 3 products per k-block (tcgen05.mma kind::tf32,
//                    M = 128, N = BN), tcgen05.commit releases the stage, a last commit the tile
//   all 4 warps      epilogue: tcgen05.ld 32x32b (warp w reads TMEM lanes 32w..32w+31 = rows),
//                    column-major stores (consecutive lanes = consecutive rows: coalesced)
// Every mbarrier wait is bounded; a wait that runs out sets *err and the CTA winds down.
// No cluster, no multicast: each CTA loads its own tiles from this GPU's memory.
#include "common.cuh"
#include "kernels.h"
#include "tf32x3.h"
#include "tcgen05.cuh"

#include <cuda.h>
#include <mutex>
#include <unordered_map>

namespace {
using namespace tc;
constexpr int BM = 128, BK = 32, STAGES = 2, NTHREADS = 128;
constexpr int A_BYTES = BM * BK * 4;   // 16 KB

// tcgen05 shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);        // start address
    d |= (uint64_t)(16u >> 4) << 16;                  // leading byte offset (unused with this swizzle)
    d |= (uint64_t)(1024u >> 4) << 32;                // stride byte offset: 8 rows x 128 B
    d |= (uint64_t)1 << 46;                           // descriptor version
    d |= (uint64_t)2 << 61;                           // swizzle: 128 B
    return d;
}
// instruction descriptor: D f32, A/B tf32, both K-major, N and M
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
    return (1u << 4)                       // D format f32
           | (2u << 7) | (2u << 10)        // A, B format tf32
           | ((uint32_t)(N >> 3) << 17)    // N / 8
           | ((uint32_t)(M >> 4) << 24);   // M / 16
}
__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
template <int BN>
struct Cfg {
    static constexpr int B_BYTES = BN * BK * 4;
    static constexpr int STAGE = 2 * A_BYTES + 2 * B_BYTES;
    static constexpr int TMEM_COLS = BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;
    static constexpr size_t SMEM = (size_t)STAGES * STAGE + 1024 /*align*/ + 256 /*barriers*/;
};

template <int BN>
__global__ void __launch_bounds__(NTHREADS, 1)
    tf32x3_kernel(const __grid_constant__ CUtensorMap tAh, const __grid_constant__ CUtensorMap tAl,
                  const __grid_constant__ CUtensorMap tBh, const __grid_constant__ CUtensorMap tBl, float *G,
                  long long ldg, int M, int N, int K, int *err) {
    using C = Cfg<BN>;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t *full = (uint64_t *)(smem + STAGES * C::STAGE);
    uint64_t *empty = full + STAGES;
    uint64_t *done = empty + STAGES;
    uint32_t *tslot = (uint32_t *)(done + 1);
    int *bad = (int *)(tslot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // N tiles vary fastest: the CTAs that share an A row panel run together and reuse it from L2
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int nkb = (K + BK - 1) / BK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        *bad = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(C::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    if (warp == 0 && lane == 0) {
        // ---- TMA producer ----
        int issued = 0;
        for (int kb = 0; kb < nkb; kb++) {
            const int s = kb % STAGES, use = kb / STAGES;
            if (use > 0 && !mbar_wait(&empty[s], (use - 1) & 1)) { atomicExch(bad, 1); break; }
            uint8_t *st = smem + s * C::STAGE;
            mbar_expect_tx(&full[s], C::STAGE);
            const int x = kb * BK;
            tma_load_2d(st, &tAh, &full[s], x, m0);
            tma_load_2d(st + A_BYTES, &tAl, &full[s], x, m0);
            tma_load_2d(st + 2 * A_BYTES, &tBh, &full[s], x, n0);
            tma_load_2d(st + 2 * A_BYTES + C::B_BYTES, &tBl, &full[s], x, n0);
            issued++;
        }
        // copies still in flight are waited for before the CTA ends (bounded)
        for (int kb = (issued > STAGES ? issued - STAGES : 0); kb < issued; kb++)
            mbar_wait(&full[kb % STAGES], (kb / STAGES) & 1);
    } else if (warp == 1 && lane == 0) {
        // ---- MMA issuer ----
        constexpr uint32_t idesc = idesc_tf32(BM, BN);
        for (int kb = 0; kb < nkb; kb++) {
            const int s = kb % STAGES;
            if (!mbar_wait(&full[s], (kb / STAGES) & 1)) { atomicExch(bad, 1); break; }
            tc_fence_after();
            const uint32_t base = smem_u32(smem + s * C::STAGE);
#pragma unroll
            for (int ks = 0; ks < BK / 8; ks++) {   // K-step of 8 tf32 = 32 bytes inside the swizzle atom
                const uint32_t off = ks * 32;
                const uint64_t ah = smem_desc(base + off), al = smem_desc(base + A_BYTES + off);
                const uint64_t bh = smem_desc(base + 2 * A_BYTES + off);
                const uint64_t bl = smem_desc(base + 2 * A_BYTES + C::B_BYTES + off);
                umma_tf32(tmem, al, bh, idesc, (kb | ks) != 0);   // small terms first
                umma_tf32(tmem, ah, bl, idesc, 1);
                umma_tf32(tmem, ah, bh, idesc, 1);
            }
            umma_commit(&empty[s]);   // the stage is free once these MMAs have read it
        }
        umma_commit(done);
    }
    __syncwarp();
    // ---- epilogue: TMEM -> registers -> global (column-major) ----
    const bool ok = mbar_wait(done, 0);
    tc_fence_after();
    // tcgen05.ld is warp-collective: the decision must be uniform across the warp
    const bool good = __all_sync(0xffffffffu, ok && !*(volatile int *)bad);
    if (good) {
        const int row = m0 + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 16) {
            uint32_t r[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, r);
            if (row < M) {
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    const int col = n0 + c0 + j;
                    if (col < N) G[(long long)row + (long long)col * ldg] = __uint_as_float(r[j]);
                }
            }
        }
    } else if (threadIdx.x == 0) {
        atomicExch(err, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(C::TMEM_COLS)
                     : "memory");
    }
}

__global__ void split_kernel(long long n, const double *x, float *hi, float *lo) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = x[i];
    const float h = tf32_round((float)v);
    hi[i] = h;
    lo[i] = tf32_round((float)(v - (double)h));
}

// rows x K fp32, row stride ld elements, box 32 (K) x box_rows, 128-byte swizzle
int make_map(CUtensorMap *map, const float *ptr, long long rows, long long K, long long ld, int box_rows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return BGPU_ERR_CUDA;
    if (((uintptr_t)ptr & 15) || ((ld * 4) & 15)) return BGPU_ERR_ARG;   // TMA: 16-byte base and stride
    cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)(ld * 4)};
    cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void *)ptr, dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? BGPU_OK : BGPU_ERR_ARG;
}

// The sticky error flag of the bounded mbarrier waits: a device variable (one per device, zero at
// module load), so the first use needs no allocation and no lock.
__device__ int g_tf32x3_err = 0;

int *err_flag() {
    void *d = nullptr;
    if (cudaGetSymbolAddress(&d, g_tf32x3_err) != cudaSuccess) return nullptr;
    return (int *)d;
}

template <int BN>
int launch(cudaStream_t st, int M, int N, int K, const float *Ah, const float *Al, long long lda, const float *Bh,
           const float *Bl, long long ldb, float *G, long long ldg) {
    CUtensorMap mAh, mAl, mBh, mBl;
    int rc;
    if ((rc = make_map(&mAh, Ah, M, K, lda, BM)) || (rc = make_map(&mAl, Al, M, K, lda, BM)) ||
        (rc = make_map(&mBh, Bh, N, K, ldb, BN)) || (rc = make_map(&mBl, Bl, N, K, ldb, BN)))
        return rc;
    BGPU_ATTR_ONCE(BGPU_CHECK(cudaFuncSetAttribute(tf32x3_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)Cfg<BN>::SMEM)));
    int *err = err_flag();
    if (!err) return BGPU_ERR_NOMEM;
    dim3 grid(ceil_div(N, BN), ceil_div(M, BM));
    tf32x3_kernel<BN><<<grid, NTHREADS, Cfg<BN>::SMEM, st>>>(mAh, mAl, mBh, mBl, G, ldg, M, N, K, err);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}
}  // namespace

int split_tf32(cudaStream_t st, long long n, const double *x, float *hi, float *lo) {
    if (n <= 0) return BGPU_OK;
    split_kernel<<<ceil_div(n, 256), 256, 0, st>>>(n, x, hi, lo);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int tf32x3_error_flag(int *host_value) {
    int *d = err_flag();
    if (!d) return BGPU_ERR_NOMEM;
    BGPU_CHECK(cudaMemcpy(host_value, d, sizeof(int), cudaMemcpyDeviceToHost));
    return BGPU_OK;
}

int gemm_tf32x3(cudaStream_t st, int M, int N, int K, const float *Ah, const float *Al, long long lda,
                const float *Bh, const float *Bl, long long ldb, float *G, long long ldg) {
    if (M <= 0 || N <= 0 || K <= 0) return BGPU_OK;
    // the tile width (128, 208 or 256 columns) that pads N (the block order) least; ties to the wider
    const int cand[3] = {256, 208, 128};
    int best = 256;
    long long pad = 1LL << 60;
    for (int c : cand) {
        const long long p = (long long)ceil_div(N, c) * c;
        if (p < pad) { pad = p; best = c; }
    }
    if (best == 256) return launch<256>(st, M, N, K, Ah, Al, lda, Bh, Bl, ldb, G, ldg);
    if (best == 208) return launch<208>(st, M, N, K, Ah, Al, lda, Bh, Bl, ldb, G, ldg);
    return launch<128>(st, M, N, K, Ah, Al, lda, Bh, Bl, ldb, G, ldg);
}
