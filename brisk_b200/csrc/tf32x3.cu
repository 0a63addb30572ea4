// 3xTF32 split-product GEMM on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// G = A B with A = Ah + Al and B = Bh + Bl, each part tf32-rounded, computed as
// Ah Bh + Ah Bl + Al Bh with FP32 accumulation in tensor memory: FP32-level accuracy at
// three tf32 MMAs per product (the dropped Al Bl term is below FP32 rounding).
//
// Persistent and warp-specialised: one CTA per SM walks the 128 x BN output tiles t = blockIdx.x,
// blockIdx.x + gridDim.x, ... (N tiles fastest, so the CTAs that share an A row panel run
// together and reuse it from L2).
//   warp 0 / lane 0  TMA producer: the 4 operand tiles of a 16-column k-block (Ah, Al: 128 rows;
//                    Bh, Bl: BN rows; 64-byte rows, 64-byte swizzle) into a STAGES-deep ring that
//                    runs on across tile boundaries, one mbarrier with the transaction count a stage
//   warp 1 / lane 0  MMA issuer: 2 K-steps of 3 products a k-block (tcgen05.mma kind::tf32,
//                    M = 128, N = BN) into one of two TMEM accumulators (2 x BN <= 512 columns);
//                    tcgen05.commit frees a stage, and at a tile's end hands its accumulator over
//   warps 2-5        epilogue: tcgen05.ld 32x32b (warp w reads TMEM lanes 32 (w % 4) .. +31 =
//                    rows), column-major stores (consecutive lanes = consecutive rows: coalesced),
//                    then the accumulator goes back to the MMA warp
// So one tile's epilogue runs under the next tile's MMAs, and the next tile's loads under both.
// Every mbarrier wait is bounded; a role that gives up sets a flag that stops the others, the
// producer waits (bounded) for its copies in flight, the MMA warp for its last MMAs, and *err
// records the failure.  No cluster, no multicast: each CTA loads its own tiles from this GPU's
// memory.
#include "common.cuh"
#include "kernels.h"
#include "tf32x3.h"
#include "tcgen05.cuh"

#include <cuda.h>
#include <algorithm>
#include <mutex>
#include <unordered_map>

namespace {
using namespace tc;
constexpr int BM = 128, BK = 16, STAGES = 4, NTHREADS = 192;
constexpr int A_BYTES = BM * BK * 4;   // 8 KB

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
    static constexpr int ACC_COLS = BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;   // one accumulator
    static constexpr int TMEM_COLS = 2 * ACC_COLS;
    static constexpr size_t SMEM = (size_t)STAGES * STAGE + 1024 /*align*/ + 256 /*barriers*/;
    static_assert(TMEM_COLS <= 512, "two accumulators in TMEM");
    static_assert(STAGE % 1024 == 0, "stages keep the alignment of the swizzled tiles");
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
    uint64_t *tfull = empty + STAGES;     // [2] accumulator ready for the epilogue
    uint64_t *tempty = tfull + 2;         // [2] accumulator drained (4 epilogue warps arrive)
    uint64_t *mdone = tempty + 2;         // the MMA warp's last MMAs
    uint32_t *tslot = (uint32_t *)(mdone + 1);
    volatile int *bad = (volatile int *)(tslot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntn = (N + BN - 1) / BN, ntm = (M + BM - 1) / BM, ntiles = ntn * ntm;
    const int nkb = (K + BK - 1) / BK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; a++) {
            mbar_init(&tfull[a], 1);
            mbar_init(&tempty[a], 4);
        }
        mbar_init(mdone, 1);
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

    if (warp == 0) {
        if (lane == 0) {
            // ---- TMA producer ----
            long long it = 0;
            for (int t = blockIdx.x; t < ntiles && !*bad; t += gridDim.x) {
                const int m0 = (t / ntn) * BM, n0 = (t % ntn) * BN;
                for (int kb = 0; kb < nkb; kb++, it++) {
                    const int s = (int)(it % STAGES);
                    const long long use = it / STAGES;
                    if (use > 0 && !mbar_wait_or_stop(&empty[s], (uint32_t)((use - 1) & 1), bad)) { *bad = 1; break; }
                    uint8_t *st = smem + s * C::STAGE;
                    mbar_expect_tx(&full[s], C::STAGE);
                    const int x = kb * BK;
                    tma_load_2d(st, &tAh, &full[s], x, m0);
                    tma_load_2d(st + A_BYTES, &tAl, &full[s], x, m0);
                    tma_load_2d(st + 2 * A_BYTES, &tBh, &full[s], x, n0);
                    tma_load_2d(st + 2 * A_BYTES + C::B_BYTES, &tBl, &full[s], x, n0);
                }
            }
            // copies still in flight are waited for before the CTA ends (bounded)
            for (long long k = (it > STAGES ? it - STAGES : 0); k < it; k++)
                mbar_wait(&full[k % STAGES], (uint32_t)((k / STAGES) & 1));
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---- MMA issuer ----
            constexpr uint32_t idesc = idesc_tf32(BM, BN);
            long long it = 0;
            int lt = 0;
            for (int t = blockIdx.x; t < ntiles && !*bad; t += gridDim.x, lt++) {
                const int a = lt & 1, use = lt >> 1;
                if (use > 0 && !mbar_wait_or_stop(&tempty[a], (uint32_t)((use - 1) & 1), bad)) { *bad = 1; break; }
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(a * C::ACC_COLS);
                bool ok = true;
                for (int kb = 0; kb < nkb; kb++, it++) {
                    const int s = (int)(it % STAGES);
                    if (!mbar_wait_or_stop(&full[s], (uint32_t)((it / STAGES) & 1), bad)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t base = smem_u32(smem + s * C::STAGE);
#pragma unroll
                    for (int ks = 0; ks < BK / 8; ks++) {   // K-step of 8 tf32 = 32 bytes inside the swizzle atom
                        const uint32_t off = ks * 32;
                        const uint64_t ah = smem_desc_sw64(base + off), al = smem_desc_sw64(base + A_BYTES + off);
                        const uint64_t bh = smem_desc_sw64(base + 2 * A_BYTES + off);
                        const uint64_t bl = smem_desc_sw64(base + 2 * A_BYTES + C::B_BYTES + off);
                        umma_tf32(d, al, bh, idesc, (kb | ks) != 0);   // small terms first
                        umma_tf32(d, ah, bl, idesc, 1);
                        umma_tf32(d, ah, bh, idesc, 1);
                    }
                    umma_commit(&empty[s]);   // the stage is free once these MMAs have read it
                }
                if (!ok) { *bad = 1; break; }
                umma_commit(&tfull[a]);       // the accumulator is complete once these MMAs are
            }
            umma_commit(mdone);
            mbar_wait(mdone, 0);              // every MMA of this CTA has completed (bounded)
        }
    } else {
        // ---- epilogue: TMEM -> registers -> global (column-major) ----
        const int q = warp & 3;               // the TMEM lane quarter this warp may read
        int lt = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, lt++) {
            const int a = lt & 1, use = lt >> 1;
            const bool ok = mbar_wait_or_stop(&tfull[a], (uint32_t)(use & 1), bad);
            // tcgen05.ld is warp-collective: the decision must be uniform across the warp
            if (!__all_sync(0xffffffffu, ok)) { if (lane == 0) *bad = 1; break; }
            tc_fence_after();
            const int m0 = (t / ntn) * BM, n0 = (t % ntn) * BN;
            const int row = m0 + q * 32 + lane;
#pragma unroll 1
            for (int c0 = 0; c0 < BN; c0 += 16) {
                uint32_t r[16];
                tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(a * C::ACC_COLS + c0), r);
                if (row < M) {
#pragma unroll
                    for (int j = 0; j < 16; j++) {
                        const int col = n0 + c0 + j;
                        if (col < N) G[(long long)row + (long long)col * ldg] = __uint_as_float(r[j]);
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[a]);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && *bad) atomicExch(err, 1);
    tc_fence_after();
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

// rows x K fp32, row stride ld elements, box BK = 16 (K: 64 bytes) x box_rows, 64-byte swizzle
int make_map(CUtensorMap *map, const float *ptr, long long rows, long long K, long long ld, int box_rows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return BGPU_ERR_CUDA;
    if (((uintptr_t)ptr & 15) || ((ld * 4) & 15)) return BGPU_ERR_ARG;   // TMA: 16-byte base and stride
    cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)(ld * 4)};
    cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void *)ptr, dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
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
    int dev = 0, nsm = 0;
    BGPU_CHECK(cudaGetDevice(&dev));
    BGPU_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const long long ntiles = (long long)ceil_div(N, BN) * ceil_div(M, BM);
    if (ntiles > 0x7fffffffLL) return BGPU_ERR_TOOBIG;
    const int grid = (int)std::min<long long>(ntiles, nsm);   // persistent: one CTA per SM
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
