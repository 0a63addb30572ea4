// FP64-accurate GEMM on the INT8 tensor cores (tcgen05 kind::i8, sm_100a): the Ozaki scheme of
// exact splitting into integer slices (Ozaki, Ogita, Oishi, Rump 2012; its integer form, Ootomo,
// Ozaki, Yokota 2024), for the Schur assembly's G = T X where FP32 accuracy no longer suffices.
//
// C(i, j) = sum_k A(i, k) B(j, k), A and B row-major with K contiguous (A(i, k) = A[i lda + k],
// B(j, k) = B[j ldb + k]), C column-major.
//
// Slicing (slice_kernel): each row r of A (of B) gets the exponent e_r with max_k |A(r, k)| < 2^e_r;
// a = A(r, k) 2^-e_r lies in (-1, 1) and is cut exactly into S signed 7-bit digits:
//   a = sum_{p=1..S} s_p 2^(-7p) + rest,  s_p = trunc(128 (rest of the previous digits)) in [-127, 127]
// (multiplications by powers of two and subtractions of integers: no rounding).
//
// Products (ozaki_kernel): A B' = 2^(e_i + f_j) sum_{p,q} 2^(-7(p+q)) (S_p^A S_q^B') with the pairs
// p + q <= S + 1 kept.  The dropped pairs (p + q >= S + 2: at most 127^2 2^(-7(p+q)) each) and the
// slices' truncation (below 2^(-7S) per entry) leave an error below about (S + 3) 2^(-7S) K
// 2^(e_i + f_j): with S = 8, about 2^-53 K relative to the largest entries of row i of A and of
// row j of B (FP64-like); with S = 6, 2^-39 K; with S = 5, 2^-32 K.  Each product of int8 slices
// accumulates exactly in int32 (|sum| <= S 127^2 K < 2^31 for K <= 16000), and all pairs of one
// diagonal d = p + q share one TMEM accumulator: S accumulators of BN columns side by side in the
// 512 TMEM columns for the whole K loop.  The epilogue drains them once, smallest diagonal terms
// first, into FP64: C = 2^(e_i + f_j) sum_d 2^(-7d) ACC_d.
//
// Tiles (S accumulators of BN columns must fit the 512 TMEM columns): S = 8 and 7 take BN = 64,
// S = 6 BN = 80, S = 5 BN = 96, S = 4 BN = 128.  With fewer slices the tile is wider, so each
// MMA reads less shared memory per multiply-add (a 128 x 64 x 32 int8 MMA reads 6 KB for 262 k
// multiply-adds; 128 x 96 x 32 reads 7 KB for 393 k) as well as issuing fewer MMAs: S = 5 issues
// 15 per 32-deep k-step and 96 columns, S = 8 36 per 64 columns.
//
// Persistent and warp-specialised, as tf32x3.cu: one CTA per SM walks the 128 x BN tiles (N tiles
// fastest).  Warp 0 / lane 0 is the TMA producer (the S slices of A and of B for a 64-byte
// k-block, 64-byte swizzle, a 2- or 3-deep ring that runs on across tiles), warp 1 / lane 0 the
// MMA issuer (kind::i8, M = 128, N = BN, K = 32 per instruction), warps 2-5 the epilogue (16
// columns at a time over all S accumulators, the tile's column exponents staged in shared
// memory, the scale 2^(e_i + f_j) built exactly as a power of two).  The S accumulators fill
// TMEM, so the MMAs of the next tile wait for this tile's epilogue; the next tile's loads do not.
// Every mbarrier wait is bounded; a role that gives up stops the others, the producer waits
// (bounded) for its copies in flight, the MMA warp for its last MMAs, and *err records the
// failure.  No cluster, no multicast.
#include "common.cuh"
#include "kernels.h"
#include "tcgen05.cuh"

namespace {
using namespace tc;
constexpr int OZ_SMAX = 8;               // most slices per operand (56 bits)
constexpr int BM = 128, BK = 64, NTHREADS = 192;
constexpr int A_TILE = BM * BK;          // bytes of one slice's A tile
constexpr int TMEM_COLS = 512;           // S accumulators of BN columns

template <int S> struct OzCfg;           // tile width and ring depth per slice count
template <> struct OzCfg<8> { static constexpr int BN = 64, STAGES = 2; };
template <> struct OzCfg<7> { static constexpr int BN = 64, STAGES = 2; };
template <> struct OzCfg<6> { static constexpr int BN = 80, STAGES = 2; };
template <> struct OzCfg<5> { static constexpr int BN = 96, STAGES = 3; };
template <> struct OzCfg<4> { static constexpr int BN = 128, STAGES = 3; };
template <int S> struct OzShape {
    static constexpr int BN = OzCfg<S>::BN, STAGES = OzCfg<S>::STAGES;
    static constexpr int B_TILE = BN * BK;
    static constexpr int STAGE = S * (A_TILE + B_TILE);
    static constexpr size_t SMEM = (size_t)STAGES * STAGE + 1024 /*align*/ + 256 /*barriers*/ + BN * sizeof(int);
    static_assert(S * BN <= TMEM_COLS, "accumulators must fit in TMEM");
    static_assert(STAGE % 1024 == 0, "stages keep the 1024-byte alignment of the swizzled tiles");
    static_assert(SMEM <= 232448, "shared memory of one CTA");
};

// tcgen05 shared-memory matrix descriptor: K-major, 64-byte swizzle, 8-row groups 512 B apart
__device__ __forceinline__ uint64_t smem_desc64(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);        // start address
    d |= (uint64_t)(16u >> 4) << 16;                  // leading byte offset (unused with this swizzle)
    d |= (uint64_t)(512u >> 4) << 32;                 // stride byte offset: 8 rows x 64 B
    d |= (uint64_t)1 << 46;                           // descriptor version
    d |= (uint64_t)4 << 61;                           // swizzle: 64 B
    return d;
}
// instruction descriptor: D s32, A and B signed 8-bit, both K-major, N and M
__host__ __device__ constexpr uint32_t idesc_i8(int M, int N) {
    return (2u << 4)                       // D format s32
           | (1u << 7) | (1u << 10)        // A, B format s8
           | ((uint32_t)(N >> 3) << 17)    // N / 8
           | ((uint32_t)(M >> 4) << 24);   // M / 16
}
__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

// 2^e as a double, exactly, for e in the normal range (ldexp otherwise)
__device__ __forceinline__ double pow2(int e) {
    if (e >= -1022 && e <= 1023) return __longlong_as_double((long long)(e + 1023) << 52);
    return ldexp(1.0, e);
}

template <int S>
__global__ void __launch_bounds__(NTHREADS, 1)
    ozaki_kernel(const __grid_constant__ CUtensorMap tA, const __grid_constant__ CUtensorMap tB, long long a_slice_rows,
                 long long b_slice_rows, const int *__restrict__ ea, const int *__restrict__ eb, double *C, long long ldc,
                 int M, int N, int K, int *err) {
    using Sh = OzShape<S>;
    constexpr int BN = Sh::BN, STAGES = Sh::STAGES, B_TILE = Sh::B_TILE, STAGE = Sh::STAGE;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t *full = (uint64_t *)(smem + STAGES * STAGE);
    uint64_t *empty = full + STAGES;
    uint64_t *tfull = empty + STAGES;     // the accumulators are ready for the epilogue
    uint64_t *tempty = tfull + 1;         // ... drained (4 epilogue warps arrive)
    uint64_t *mdone = tempty + 1;         // the MMA warp's last MMAs
    uint32_t *tslot = (uint32_t *)(mdone + 1);
    volatile int *bad = (volatile int *)(tslot + 1);
    int *ebs = (int *)(smem + STAGES * STAGE + 256);   // the tile's column exponents
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntn = (N + BN - 1) / BN, ntm = (M + BM - 1) / BM, ntiles = ntn * ntm;
    const int nkb = (K + BK - 1) / BK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(tfull, 1);
        mbar_init(tempty, 4);
        mbar_init(mdone, 1);
        *bad = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    if (warp == 0) {
        if (lane == 0) {
            // ---- TMA producer: the S slices of A (rows m0..) and of B (rows n0..) of a k-block ----
            long long it = 0;
            for (int t = blockIdx.x; t < ntiles && !*bad; t += gridDim.x) {
                const int m0 = (t / ntn) * BM, n0 = (t % ntn) * BN;
                for (int kb = 0; kb < nkb; kb++, it++) {
                    const int s = (int)(it % STAGES);
                    const long long use = it / STAGES;
                    if (use > 0 && !mbar_wait_or_stop(&empty[s], (uint32_t)((use - 1) & 1), bad)) { *bad = 1; break; }
                    uint8_t *st = smem + s * STAGE;
                    mbar_expect_tx(&full[s], STAGE);
                    const int x = kb * BK;
                    for (int p = 0; p < S; p++) {
                        tma_load_2d(st + p * A_TILE, &tA, &full[s], x, (int)(p * a_slice_rows + m0));
                        tma_load_2d(st + S * A_TILE + p * B_TILE, &tB, &full[s], x, (int)(p * b_slice_rows + n0));
                    }
                }
            }
            for (long long k = (it > STAGES ? it - STAGES : 0); k < it; k++)
                mbar_wait(&full[k % STAGES], (uint32_t)((k / STAGES) & 1));
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---- MMA issuer: every slice pair p + q <= S + 1 into the accumulator of its diagonal ----
            constexpr uint32_t idesc = idesc_i8(BM, BN);
            long long it = 0;
            int lt = 0;
            for (int t = blockIdx.x; t < ntiles && !*bad; t += gridDim.x, lt++) {
                if (lt > 0 && !mbar_wait_or_stop(tempty, (uint32_t)((lt - 1) & 1), bad)) { *bad = 1; break; }
                tc_fence_after();
                bool ok = true;
                for (int kb = 0; kb < nkb; kb++, it++) {
                    const int s = (int)(it % STAGES);
                    if (!mbar_wait_or_stop(&full[s], (uint32_t)((it / STAGES) & 1), bad)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t base = smem_u32(smem + s * STAGE);
#pragma unroll
                    for (int ks = 0; ks < BK / 32; ks++) {   // K-step of 32 int8 = 32 bytes inside the swizzle atom
                        const uint32_t off = ks * 32;
#pragma unroll
                        for (int d = 0; d < S; d++) {          // diagonal p + q = d + 2 (0-based slices: p + q = d)
#pragma unroll
                            for (int p = 0; p <= d; p++) {
                                const int q = d - p;
                                const uint64_t a = smem_desc64(base + p * A_TILE + off);
                                const uint64_t b = smem_desc64(base + S * A_TILE + q * B_TILE + off);
                                umma_i8(tmem + (uint32_t)(d * BN), a, b, idesc, (kb | ks | p) != 0);
                            }
                        }
                    }
                    umma_commit(&empty[s]);
                }
                if (!ok) { *bad = 1; break; }
                umma_commit(tfull);
            }
            umma_commit(mdone);
            mbar_wait(mdone, 0);
        }
    } else {
        // ---- epilogue: the S accumulators -> FP64, smallest terms first, scaled by 2^(e_i + f_j) ----
        const int q = warp & 3;               // the TMEM lane quarter this warp may read
        const int et = threadIdx.x - 64;      // 0..127 over the 4 epilogue warps
        int lt = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, lt++) {
            const int m0 = (t / ntn) * BM, n0 = (t % ntn) * BN;
            // the tile's column exponents (the previous tile's have been read: every epilogue
            // thread passed the barrier below after its last read of them)
            asm volatile("bar.sync 1, 128;" ::: "memory");
            for (int c = et; c < BN; c += 128) ebs[c] = n0 + c < N ? eb[n0 + c] : 0;
            const bool ok = mbar_wait_or_stop(tfull, (uint32_t)(lt & 1), bad);
            // one decision for the 4 warps (a barrier reduction: the next iteration's barrier must
            // see all 128 threads or none), which also publishes ebs
            unsigned stop;
            asm volatile("{\n .reg .pred p, r;\n setp.ne.u32 p, %1, 0;\n bar.red.or.pred r, 1, 128, p;\n selp.u32 %0, 1, 0, r;\n}\n"
                         : "=r"(stop) : "r"((unsigned)(!ok)) : "memory");
            if (stop) { if (et == 0) *bad = 1; break; }
            tc_fence_after();
            const int row = m0 + q * 32 + lane;
            const int e = row < M ? ea[row] : 0;
#pragma unroll 1
            for (int c0 = 0; c0 < BN; c0 += 16) {
                double acc[16];
#pragma unroll
                for (int j = 0; j < 16; j++) acc[j] = 0.0;
#pragma unroll
                for (int d = S - 1; d >= 0; d--) {
                    const double w = pow2(-7 * (d + 2));
                    uint32_t r[16];
                    tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(d * BN + c0), r);
#pragma unroll
                    for (int j = 0; j < 16; j++) acc[j] += w * (double)(int)r[j];
                }
                if (row < M) {
#pragma unroll
                    for (int j = 0; j < 16; j++) {
                        const int col = n0 + c0 + j;
                        if (col < N) C[(long long)row + (long long)col * ldc] = acc[j] * pow2(e + ebs[c0 + j]);
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(tempty);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && *bad) atomicExch(err, 1);
    tc_fence_after();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// One warp per row: the row's exponent and its S digits (row stride ldk bytes, slice p at
// dst + p * slice_bytes; the K..ldk padding is zero).
__global__ void slice_kernel(int rows, int K, int S, const double *__restrict__ src, long long lds, int8_t *dst,
                             long long ldk, long long slice_bytes, int *exps) {
    const int r = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (r >= rows) return;
    const double *x = src + (long long)r * lds;
    double mx = 0.0;
    for (int k = lane; k < K; k += 32) mx = fmax(mx, fabs(x[k]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    const int e = mx > 0.0 ? ilogb(mx) + 1 : 0;   // max |x| 2^-e < 1
    if (lane == 0) exps[r] = e;
    // 8 consecutive columns a lane (ldk is a multiple of 64): each slice's 8 digits go out as
    // one 8-byte store
    int8_t *out = dst + (long long)r * ldk;
    for (long long k8 = lane; k8 < ldk / 8; k8 += 32) {
        double a[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const long long k = k8 * 8 + i;
            a[i] = k < K ? ldexp(x[k], -e) : 0.0;
        }
#pragma unroll
        for (int p = 0; p < OZ_SMAX; p++) {
            if (p >= S) break;
            unsigned long long w = 0;
#pragma unroll
            for (int i = 0; i < 8; i++) {
                a[i] *= 128.0;
                const double t = trunc(a[i]);
                a[i] -= t;
                w |= (unsigned long long)(uint8_t)(int8_t)(int)t << (8 * i);
            }
            *reinterpret_cast<unsigned long long *>(out + p * slice_bytes + k8 * 8) = w;
        }
    }
}

// the slices of rows x K bytes each, stacked (slice p at rows p * slice_rows), row stride ldk
// bytes, box 64 (K) x box_rows, 64-byte swizzle
int make_map_i8(CUtensorMap *map, const int8_t *ptr, long long total_rows, long long K, long long ldk, int box_rows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return BGPU_ERR_CUDA;
    if (((uintptr_t)ptr & 15) || (ldk & 15)) return BGPU_ERR_ARG;   // TMA: 16-byte base and stride
    cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)total_rows};
    cuuint64_t strides[1] = {(cuuint64_t)ldk};
    cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void *)ptr, dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? BGPU_OK : BGPU_ERR_ARG;
}

__device__ int g_ozaki_err = 0;   // sticky flag of the bounded waits (zero at module load)

inline long long round_up(long long x, long long a) { return (x + a - 1) / a * a; }
}  // namespace

int ozaki_max_slices() { return OZ_SMAX; }

// bytes of the S slices (and exponents) of a rows x K operand
size_t ozaki_operand_bytes(long long rows, int K, int S) {
    const long long ldk = round_up(K, 64), srows = round_up(rows, 128);
    return (size_t)S * srows * ldk + sizeof(int) * srows + 1024;
}

// The layout of a rows x K operand's S slices in buf (ozaki_operand_bytes): row stride ldk = K
// rounded up to 64 bytes, srows = rows rounded up to 128, slice p at q + p srows ldk.
int ozaki_layout(long long rows, int K, void *buf, OzakiOperand *op, int S) {
    if (S < 4 || S > OZ_SMAX) return BGPU_ERR_ARG;
    const long long ldk = round_up(K, 64), srows = round_up(rows, 128);
    op->rows = rows;
    op->srows = srows;
    op->K = K;
    op->ldk = ldk;
    op->slices = S;
    op->q = (int8_t *)(((uintptr_t)buf + 255) & ~(uintptr_t)255);
    op->e = (int *)(op->q + (size_t)S * srows * ldk);
    return BGPU_OK;
}

// The operand's S slices into buf (ozaki_operand_bytes): returns the slice layout in *op.
int ozaki_slice(cudaStream_t st, long long rows, int K, const double *src, long long lds, void *buf, OzakiOperand *op,
                int S) {
    if (int rc = ozaki_layout(rows, K, buf, op, S)) return rc;
    const long long ldk = op->ldk, srows = op->srows;
    if (rows <= 0) return BGPU_OK;
    if ((rows + 7) / 8 > (1LL << 31) - 1) return BGPU_ERR_TOOBIG;
    slice_kernel<<<ceil_div(rows * 32, 256), 256, 0, st>>>((int)rows, K, S, src, lds, op->q, ldk, srows * ldk, op->e);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

namespace {
template <int S>
int ozaki_launch(cudaStream_t st, const OzakiOperand &A, const OzakiOperand &B, double *C, long long ldc) {
    using Sh = OzShape<S>;
    const int M = (int)A.rows, N = (int)B.rows, K = A.K;
    CUtensorMap mA, mB;
    int rc;
    if ((rc = make_map_i8(&mA, A.q, S * A.srows, K, A.ldk, BM)) || (rc = make_map_i8(&mB, B.q, S * B.srows, K, B.ldk, Sh::BN)))
        return rc;
    BGPU_ATTR_ONCE(BGPU_CHECK(cudaFuncSetAttribute(ozaki_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)Sh::SMEM)));
    void *d = nullptr;
    BGPU_CHECK(cudaGetSymbolAddress(&d, g_ozaki_err));
    int dev = 0, nsm = 0;
    BGPU_CHECK(cudaGetDevice(&dev));
    BGPU_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const long long ntiles = (long long)ceil_div(N, Sh::BN) * ceil_div(M, BM);
    if (ntiles > 0x7fffffffLL) return BGPU_ERR_TOOBIG;
    const int grid = (int)(ntiles < nsm ? ntiles : nsm);   // persistent: one CTA per SM
    ozaki_kernel<S><<<grid, NTHREADS, Sh::SMEM, st>>>(mA, mB, A.srows, B.srows, A.e, B.e, C, ldc, M, N, K, (int *)d);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}
}  // namespace

// C (column-major, ldc) = A B' from the sliced operands (A: M rows, B: N rows, both K, the same
// number of slices)
int ozaki_gemm(cudaStream_t st, const OzakiOperand &A, const OzakiOperand &B, double *C, long long ldc) {
    const int M = (int)A.rows, N = (int)B.rows, K = A.K;
    if (M <= 0 || N <= 0 || K <= 0) return BGPU_OK;
    const int S = A.slices;
    if (B.K != K || B.slices != S || K > 16000 || (long long)S * A.srows > (1LL << 31) - 1 ||
        (long long)S * B.srows > (1LL << 31) - 1)
        return BGPU_ERR_ARG;
    switch (S) {
        case 8: return ozaki_launch<8>(st, A, B, C, ldc);
        case 7: return ozaki_launch<7>(st, A, B, C, ldc);
        case 6: return ozaki_launch<6>(st, A, B, C, ldc);
        case 5: return ozaki_launch<5>(st, A, B, C, ldc);
        case 4: return ozaki_launch<4>(st, A, B, C, ldc);
        default: return BGPU_ERR_ARG;
    }
}

int ozaki_error_flag(int *host_value) {
    void *d = nullptr;
    BGPU_CHECK(cudaGetSymbolAddress(&d, g_ozaki_err));
    BGPU_CHECK(cudaMemcpy(host_value, d, sizeof(int), cudaMemcpyDeviceToHost));
    return BGPU_OK;
}
