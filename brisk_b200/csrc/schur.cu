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
// ZT: the type Zi is read in, and the type of the sums.  The 3xTF32 form reads an FP32 copy of
// Zi and sums in FP32: half the L2 traffic of this L2-bound kernel (each entry reads a 128-value
// segment of a Zi column), no conversions, half the tile, and T keeps the accuracy its tf32
// hi + lo split can carry (2^-24 relative per term against the split's 2^-22).
template <typename OutT, typename ZT = double>
__global__ void __launch_bounds__(256) tprod_kernel(int n, int ldt, int K, int a0, int ncon,
                                                   const long long *__restrict__ cptr, const int *__restrict__ ccol,
                                                   const int *__restrict__ cpos, const double *__restrict__ cval,
                                                   const ZT *__restrict__ Zi, OutT *__restrict__ T,
                                                   OutT *__restrict__ Tlo) {
    using AccT = ZT;
    __shared__ AccT tile[TP_Q * TP_LD];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int q0 = blockIdx.x * TP_Q, k0 = blockIdx.y * TP_K, t = blockIdx.z;
    const int a = a0 + t;
    for (int kk = warp; kk < TP_K; kk += 8) {
        const int k = k0 + kk;
        AccT acc[4] = {(AccT)0, (AccT)0, (AccT)0, (AccT)0};
        if (a < ncon && k < n) {
            const long long base = cptr[a];
            const int *cc = ccol + (long long)a * (n + 1);
            const long long e0 = base + cc[k], e1 = base + cc[k + 1];
            for (long long e = e0; e < e1; e++) {
                const int pp = cpos[e] - k * n;   // the row p' of the entry (p', k)
                const AccT v = (AccT)cval[e];
                const ZT *z = Zi + (long long)pp * n + q0 + lane;
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
        const AccT v = tile[r * TP_LD + lane];
        const long long o = ((long long)q * K + t) * ldt + k0 + lane;
        if (sizeof(OutT) == 8) {
            T[o] = (OutT)v;
        } else {
            const float hi_ = tf32_round((float)v);
            T[o] = (OutT)hi_;
            Tlo[o] = (OutT)tf32_round((float)((double)v - (double)hi_));
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

// ---- the packed symmetric gather ---------------------------------------------------------
// Every A_b is symmetric, so <A_b, G_a> = sum_{p<=q} A_b[p,q] S_a[p,q] with S_a = G_a + G_a' off
// the diagonal and S_a[p,p] = G_a[p,p]: sym_pack_kernel folds the chunk's G into S (packed upper,
// index u = q (q+1)/2 + p, K values per position, t fastest) and gather_sym_kernel reads each
// constraint's upper entries only: half the entries and half the G values of the full gather.
__device__ __forceinline__ long long upk(int p, int q) { return (long long)q * (q + 1) / 2 + p; }

template <typename GT> struct Vec16;
template <> struct Vec16<float> { using T = float4; static constexpr int N = 4; };
template <> struct Vec16<double> { using T = double2; static constexpr int N = 2; };
__device__ __forceinline__ void vget(const float4 &v, double *o) { o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w; }
__device__ __forceinline__ void vget(const double2 &v, double *o) { o[0] = v.x; o[1] = v.y; }
__device__ __forceinline__ float4 vadd(const float4 &a, const float4 &b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
__device__ __forceinline__ double2 vadd(const double2 &a, const double2 &b) { return make_double2(a.x + b.x, a.y + b.y); }

// S[(upk(i, j)) K + t] = G_a[i, j] + G_a[j, i] (i < j) or G_a[i, i]; G holds G_a[p, q] at
// ((p n + q) K + t).  Column j = blockIdx.y; a thread owns 16 bytes of one position.
template <typename GT, int K>
__global__ void sym_pack_kernel(int n, const GT *__restrict__ G, GT *__restrict__ S) {
    using V = typename Vec16<GT>::T;
    constexpr int NV = K / Vec16<GT>::N;
    const int j = blockIdx.y;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (int)(idx / NV), v = (int)(idx % NV);
    if (i > j) return;
    const V a = reinterpret_cast<const V *>(G + ((long long)i * n + j) * K)[v];
    V r = a;
    if (i < j) r = vadd(a, reinterpret_cast<const V *>(G + ((long long)j * n + i) * K)[v]);
    reinterpret_cast<V *>(S + upk(i, j) * K)[v] = r;
}

// One CTA of GW warps per constraint b >= a0 over b's upper entries; LPG lanes per entry, each
// loading 16 contiguous bytes of S (VEC columns); fixed summation order as gather_kernel.
template <int K, typename GT>
__global__ void __launch_bounds__(GW * 32) gather_sym_kernel(int a0, int ncon, int m, const int *__restrict__ con,
                                                            const long long *__restrict__ uptr,
                                                            const int *__restrict__ upos,
                                                            const double *__restrict__ uval,
                                                            const GT *__restrict__ S, double *M) {
    using V = typename Vec16<GT>::T;
    constexpr int VEC = Vec16<GT>::N;
    constexpr int LPG = K / VEC;               // lanes per entry
    constexpr int GPW = 32 / LPG;              // entries per warp step
    __shared__ double part[GW][K];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int b = a0 + blockIdx.x;
    if (b >= ncon) return;
    const int sub = lane / LPG, l = lane % LPG;
    double acc[VEC], acc2[VEC], g[VEC];
#pragma unroll
    for (int u = 0; u < VEC; u++) acc[u] = acc2[u] = 0.0;
    const long long s0 = uptr[b], e0 = uptr[b + 1];
    const long long len = e0 - s0, per_w = (len + GW - 1) / GW;
    const long long s = s0 + warp * per_w, e = min(e0, s + per_w);
    long long base = s;
    // S rows are K sizeof(GT) bytes at random positions of an S as large as L2: the loads below
    // wait on memory.  With FP32 rows (the 3xTF32 assembly), each lane asks L2 ahead of time for
    // the row of its entry in the next group of 32 (prefetch.global.L2: no register is held while
    // it is in flight), so that group's loads find their rows in L2 (measured on B200, rand1000:
    // the assembly 175 -> 164 ms; with the FP64 rows, twice as long, the prefetches cost more than
    // they save: 669 -> 709 ms, so they are left out there).
    constexpr int RB = K * (int)sizeof(GT);
    auto prefetch_row = [&](long long at) {
        if (sizeof(GT) == 4 && at < e) {
            const char *row = reinterpret_cast<const char *>(S + (long long)upos[at] * K);
#pragma unroll
            for (int o = 0; o < RB; o += 128) asm volatile("prefetch.global.L2 [%0];" ::"l"(row + o));
        }
    };
    prefetch_row(base + lane);
    for (; base + 32 <= e; base += 32) {
        const int pos = upos[base + lane];
        const double v = uval[base + lane];
        prefetch_row(base + 32 + lane);
#pragma unroll
        for (int j = 0; j < 32; j += GPW) {
            const int pj = __shfl_sync(0xffffffffu, pos, j + sub);
            const double vj = __shfl_sync(0xffffffffu, v, j + sub);
            vget(__ldg(reinterpret_cast<const V *>(S + (long long)pj * K) + l), g);
            if ((j / GPW) & 1) {
#pragma unroll
                for (int u = 0; u < VEC; u++) acc2[u] += vj * g[u];
            } else {
#pragma unroll
                for (int u = 0; u < VEC; u++) acc[u] += vj * g[u];
            }
        }
    }
    if (base < e) {   // the ragged last group of the slice
        const long long my = base + lane;
        int pos = 0;
        double v = 0.0;
        if (my < e) { pos = upos[my]; v = uval[my]; }
        const int cnt = (int)(e - base);
        for (int j = 0; j < cnt; j += GPW) {   // uniform trip count: every lane shuffles together
            const int jj = j + sub;
            const int src = jj < cnt ? jj : 0;
            const int pj = __shfl_sync(0xffffffffu, pos, src);
            const double vj = __shfl_sync(0xffffffffu, v, src);
            if (jj < cnt) {
                vget(__ldg(reinterpret_cast<const V *>(S + (long long)pj * K) + l), g);
#pragma unroll
                for (int u = 0; u < VEC; u++) acc[u] += vj * g[u];
            }
        }
    }
#pragma unroll
    for (int u = 0; u < VEC; u++) {
        acc[u] += acc2[u];
#pragma unroll
        for (int o = LPG; o < 32; o <<= 1) acc[u] += __shfl_xor_sync(0xffffffffu, acc[u], o);
    }
    if (sub == 0)
#pragma unroll
        for (int u = 0; u < VEC; u++) part[warp][l * VEC + u] = acc[u];
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

// S[(u K) + t] = A_a[p, q] + A_a[q, p] for the upper entries of constraint a = a0 + t (the Gram
// matrix's "G_a" is A_a itself)
__global__ void gram_scatter_kernel(int K, int a0, int ncon, const long long *__restrict__ uptr,
                                    const int *__restrict__ upos, const double *__restrict__ uval, double *S) {
    const int t = blockIdx.y, a = a0 + t;
    if (a >= ncon) return;
    for (long long e = uptr[a] + (long long)blockIdx.x * blockDim.x + threadIdx.x; e < uptr[a + 1];
         e += (long long)gridDim.x * blockDim.x) {
        const long long u = upos[e];
        long long q = (long long)((sqrt(8.0 * (double)u + 1.0) - 1.0) * 0.5);
        while (q * (q + 1) / 2 > u) q--;
        while ((q + 1) * (q + 2) / 2 <= u) q++;
        const long long p = u - q * (q + 1) / 2;
        S[u * K + t] = (p == q) ? uval[e] : 2.0 * uval[e];
    }
}

__global__ void upper_count_kernel(int n, int ncon, const long long *__restrict__ cptr, const int *__restrict__ cpos,
                                   int *counts) {
    __shared__ int wsum[8];
    const int t = blockIdx.x;
    if (t >= ncon) return;
    int c = 0;
    for (long long e = cptr[t] + threadIdx.x; e < cptr[t + 1]; e += blockDim.x) {
        const int pos = cpos[e], q = pos / n, p = pos - q * n;
        c += p <= q;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int tot = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) tot += wsum[w];
        counts[t] = tot;
    }
}

// uptr = exclusive scan of counts (one CTA of 1024 threads, each a contiguous range)
__global__ void __launch_bounds__(1024) upper_scan_kernel(int ncon, const int *__restrict__ counts, long long *uptr) {
    __shared__ long long part[1024];
    const int tid = threadIdx.x;
    const int per = (ncon + 1023) / 1024;
    const int lo = min(ncon, tid * per), hi = min(ncon, lo + per);
    long long s = 0;
    for (int i = lo; i < hi; i++) s += counts[i];
    part[tid] = s;
    __syncthreads();
    if (tid == 0) {
        long long run = 0;
        for (int w = 0; w < 1024; w++) { const long long v = part[w]; part[w] = run; run += v; }
        uptr[ncon] = run;
    }
    __syncthreads();
    long long run = part[tid];
    for (int i = lo; i < hi; i++) { uptr[i] = run; run += counts[i]; }
}

// order-preserving compaction of each constraint's entries p <= q (one CTA of 256 per constraint)
__global__ void __launch_bounds__(256) upper_fill_kernel(int n, int ncon, const long long *__restrict__ cptr,
                                                         const int *__restrict__ cpos,
                                                         const double *__restrict__ cval,
                                                         const long long *__restrict__ uptr, int *upos, double *uval) {
    __shared__ int wcount[8];
    __shared__ long long base_s;
    const int t = blockIdx.x;
    if (t >= ncon) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) base_s = uptr[t];
    __syncthreads();
    for (long long e0 = cptr[t]; e0 < cptr[t + 1]; e0 += 256) {
        const long long e = e0 + threadIdx.x;
        int p = 1, q = 0, pos = 0;
        if (e < cptr[t + 1]) { pos = cpos[e]; q = pos / n; p = pos - q * n; }
        const bool keep = e < cptr[t + 1] && p <= q;
        const unsigned mask = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) wcount[warp] = __popc(mask);
        __syncthreads();
        long long off = base_s;
        for (int w = 0; w < warp; w++) off += wcount[w];
        off += __popc(mask & ((1u << lane) - 1u));
        if (keep) {
            upos[off] = (int)upk(p, q);
            uval[off] = cval[e];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            long long tot = 0;
            for (int w = 0; w < 8; w++) tot += wcount[w];
            base_s += tot;
        }
        __syncthreads();
    }
}

template <typename GT>
int sym_pack_launch(cudaStream_t st, int K, int n, const GT *G, GT *S) {
    const int NV = K / Vec16<GT>::N;
    dim3 grid(ceil_div((long long)n * NV, 256), n);
    switch (K) {
        case 8: sym_pack_kernel<GT, 8><<<grid, 256, 0, st>>>(n, G, S); break;
        case 16: sym_pack_kernel<GT, 16><<<grid, 256, 0, st>>>(n, G, S); break;
        case 32: sym_pack_kernel<GT, 32><<<grid, 256, 0, st>>>(n, G, S); break;
        case 64: sym_pack_kernel<GT, 64><<<grid, 256, 0, st>>>(n, G, S); break;
        default: return BGPU_ERR_ARG;
    }
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

template <typename GT>
int gather_sym_launch(cudaStream_t st, int K, int a0, int ncon, int m, const DevBlock &B, const GT *S, double *M) {
    const int nb = ncon - a0;
    if (nb <= 0) return BGPU_OK;
    dim3 grid(nb);
    switch (K) {
        case 8: gather_sym_kernel<8, GT><<<grid, GW * 32, 0, st>>>(a0, ncon, m, B.con, B.uptr, B.upos, B.uval, S, M); break;
        case 16: gather_sym_kernel<16, GT><<<grid, GW * 32, 0, st>>>(a0, ncon, m, B.con, B.uptr, B.upos, B.uval, S, M); break;
        case 32: gather_sym_kernel<32, GT><<<grid, GW * 32, 0, st>>>(a0, ncon, m, B.con, B.uptr, B.upos, B.uval, S, M); break;
        case 64: gather_sym_kernel<64, GT><<<grid, GW * 32, 0, st>>>(a0, ncon, m, B.con, B.uptr, B.upos, B.uval, S, M); break;
        default: return BGPU_ERR_ARG;
    }
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
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

__global__ void to_f32_kernel(long long count, const double *__restrict__ src, float *__restrict__ dst) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) dst[i] = (float)src[i];
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
// A'(y) for blocks stored one after another: position g of the concatenation lies in block k
// (off ascending); the block's position-major lists come from pointer tables.
__global__ void atop_blocks_kernel(int nb, const long long *__restrict__ off, long long total,
                                   const long long *const *__restrict__ pptr, const int *const *__restrict__ pcon,
                                   const double *const *__restrict__ pval, const double *__restrict__ y, double alpha,
                                   double beta, double *F) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    int lo = 0, hi = nb - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= g) lo = mid; else hi = mid - 1;
    }
    const long long p = g - off[lo];
    const long long *pp = pptr[lo];
    const int *pc = pcon[lo];
    const double *pv = pval[lo];
    double s = 0.0;
    for (long long e = pp[p]; e < pp[p + 1]; e++) s += pv[e] * y[pc[e]];
    F[g] = (beta == 0.0) ? alpha * s : alpha * s + beta * F[g];
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

int atop_blocks_f64(cudaStream_t st, int nb, const long long *d_off, long long total, const long long *const *pptr,
                    const int *const *pcon, const double *const *pval, const double *y, double alpha, double beta,
                    double *F) {
    if (total <= 0 || nb <= 0) return BGPU_OK;
    atop_blocks_kernel<<<ceil_div(total, 256), 256, 0, st>>>(nb, d_off, total, pptr, pcon, pval, y, alpha, beta, F);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int atop_f64(cudaStream_t st, const DevBlock &B, const double *y, double alpha, double beta, double *F) {
    const long long npos = (long long)B.n * B.n;
    atop_kernel<<<ceil_div(npos, 256), 256, 0, st>>>(npos, B.pptr, B.pcon, B.pval, y, alpha, beta, F);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

// tf32 operand rows padded to a multiple of 4 floats: the tensor maps need 16-byte strides
static inline int tf32_ld(int n) { return (n + 3) / 4 * 4; }

int schur_ozaki_slices(int precision) {
    const int S = (precision >> 8) & 0xf;
    return S == 0 ? 8 : S;
}

int schur_chunk_default(int n, int precision) {
    // the widest chunk whose workspace stays within 4 GB: a wider chunk reads each constraint's
    // entry list fewer times in the gather.  Measured on B200 (rand400 FP64, rand1000 FP64 and
    // 3xTF32): K = 64 assembles 10-15 % faster than 16 or 32, although the chunk's G then no longer
    // fits in L2.
    int K = 64;
    while (K > 8 && schur_ws_bytes(n, K, precision) > ((size_t)4 << 30)) K >>= 1;
    return K;
}

size_t schur_ws_bytes(int n, int chunk, int precision) {
    const size_t nn = (size_t)n * n * chunk;
    if (precision == 0) return 2 * nn * sizeof(double);            // T, G
    if ((precision & 0xff) == 2) {                                 // T, G, the slices of T and of X
        const int S = schur_ozaki_slices(precision);
        return 2 * nn * sizeof(double) + ozaki_operand_bytes((long long)n * chunk, n, S) + ozaki_operand_bytes(n, n, S);
    }
    const size_t ld = tf32_ld(n);
    // T hi/lo (n K rows of ld), G (float, n K x n), X hi/lo (n rows of ld), Zi in FP32 (n x n), plus
    // 256 B alignment slack each
    return (2 * (size_t)n * chunk * ld + nn + 2 * (size_t)n * ld + (size_t)n * n) * sizeof(float) + 6 * 256;
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
    const bool oz = (precision & 0xff) == 2;
    if (precision == 0 || oz) {
        double *T = (double *)ws, *G = T + nnK;
        // products on the INT8 tensor cores: X's slices once, T's per chunk
        const int S = oz ? schur_ozaki_slices(precision) : 0;
        uint8_t *sa = (uint8_t *)(G + nnK), *sb = oz ? sa + ozaki_operand_bytes((long long)n * K, n, S) : nullptr;
        OzakiOperand opA, opB;
        if (oz)
            if (int rc = ozaki_slice(st, n, n, X, n, sb, &opB, S)) return rc;
        for (int a0 = 0; a0 < B.ncon; a0 += K) {
            tprod_kernel<double><<<tgrid, 256, 0, st>>>(n, n, K, a0, B.ncon, B.cptr, B.ccol, B.cpos, B.cval, Zi, T, nullptr);
            BGPU_LAUNCH_CHECK();
            int rc;
            if (oz) {
                if ((rc = ozaki_slice(st, (long long)n * K, n, T, n, sa, &opA, S))) return rc;
                rc = ozaki_gemm(st, opA, opB, G, (long long)n * K);
            } else {
                rc = gemm_f64(st, 1, 1, n * K, n, n, 1.0, T, n, 0, X, n, 0, 0.0, G, (long long)n * K, 0, 1, 0);
            }
            if (rc) return rc;
            if (B.upos) {   // T is free again: it takes the packed symmetric sum
                if ((rc = sym_pack_launch<double>(st, K, n, G, T))) return rc;
                rc = gather_sym_launch<double>(st, K, a0, B.ncon, m, B, T, M);
            } else {
                rc = gather_launch<double>(st, K, a0, B.ncon, m, B, G, M);
            }
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
    float *Xh = carve((size_t)n * ld), *Xl = carve((size_t)n * ld), *Zf = carve((size_t)n * n);
    split2d_kernel<<<dim3(ceil_div(ld, 256), n), 256, 0, st>>>(n, X, ld, Xh, Xl);
    BGPU_LAUNCH_CHECK();
    to_f32_kernel<<<ceil_div((long long)n * n, 256), 256, 0, st>>>((long long)n * n, Zi, Zf);
    BGPU_LAUNCH_CHECK();
    for (int a0 = 0; a0 < B.ncon; a0 += K) {
        tprod_kernel<float, float><<<tgrid, 256, 0, st>>>(n, ld, K, a0, B.ncon, B.cptr, B.ccol, B.cpos, B.cval, Zf, Th, Tl);
        BGPU_LAUNCH_CHECK();
        int rc = gemm_tf32x3(st, n * K, n, n, Th, Tl, ld, Xh, Xl, ld, G, (long long)n * K);
        if (rc) return rc;
        if (B.upos) {
            if ((rc = sym_pack_launch<float>(st, K, n, G, Th))) return rc;
            rc = gather_sym_launch<float>(st, K, a0, B.ncon, m, B, Th, M);
        } else {
            rc = gather_launch<float>(st, K, a0, B.ncon, m, B, G, M);
        }
        if (rc) return rc;
    }
    return BGPU_OK;
}

int schur_upper_ptr(cudaStream_t st, const DevBlock &B, int *counts) {
    if (B.ncon <= 0) return BGPU_OK;
    if (!B.uptr || !counts) return BGPU_ERR_ARG;
    upper_count_kernel<<<B.ncon, 256, 0, st>>>(B.n, B.ncon, B.cptr, B.cpos, counts);
    BGPU_LAUNCH_CHECK();
    upper_scan_kernel<<<1, 1024, 0, st>>>(B.ncon, counts, B.uptr);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int schur_upper(cudaStream_t st, const DevBlock &B) {
    if (B.ncon <= 0) return BGPU_OK;
    if (!B.uptr || !B.upos || !B.uval) return BGPU_ERR_ARG;
    upper_fill_kernel<<<B.ncon, 256, 0, st>>>(B.n, B.ncon, B.cptr, B.cpos, B.cval, B.uptr, B.upos, B.uval);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int schur_assemble_gram(cudaStream_t st, const DevBlock &B, double *M, int m, void *ws, size_t ws_bytes) {
    const int n = B.n, ncon = B.ncon;
    if (ncon <= 0) return BGPU_OK;
    if (!B.upos || !B.uptr || !B.uval) return BGPU_ERR_ARG;
    if (((uintptr_t)ws & 15) != 0) return BGPU_ERR_ARG;
    const size_t npk = (size_t)n * (n + 1) / 2;
    int K = 64;   // the widest chunk whose packed S fits the workspace and stays L2-resident (64 MB)
    while (K > 8 && (npk * K * sizeof(double) > ws_bytes || npk * K * sizeof(double) > 64e6)) K >>= 1;
    if (npk * K * sizeof(double) > ws_bytes) return BGPU_ERR_ARG;
    double *S = (double *)ws;
    for (int a0 = 0; a0 < ncon; a0 += K) {
        BGPU_CHECK(cudaMemsetAsync(S, 0, npk * K * sizeof(double), st));
        gram_scatter_kernel<<<dim3(16, K), 256, 0, st>>>(K, a0, ncon, B.uptr, B.upos, B.uval, S);
        BGPU_LAUNCH_CHECK();
        int rc = gather_sym_launch<double>(st, K, a0, ncon, m, B, S, M);
        if (rc) return rc;
    }
    return BGPU_OK;
}

// ---- many small blocks at once ----------------------------------------------------------------
// gridDim.y CTAs per block (n <= SB_NMAX), one warp per constraint a of the block (the block's
// constraints dealt round-robin to the CTAs' warps): W = A_a Zi row by row from a's entries
// (W[p, :] += v Zi[q, :]), G = X W over the rows A_a touches, then M[a, b] = <A_b, G> for the
// block's b >= a, a warp sum per b.  The blocks of one launch share no constraint (the caller
// colours them), so every M entry has one writer per launch and the launches add in a fixed
// order; how many CTAs share a block changes no sum.
namespace {
constexpr int SB_W = 8;   // warps per CTA
__global__ void __launch_bounds__(SB_W * 32) small_schur_kernel(
    const int *__restrict__ blocks, const int *__restrict__ bn, const int *__restrict__ bncon,
    const int *const *__restrict__ con_tab, const long long *const *__restrict__ cptr_tab,
    const int *const *__restrict__ cpos_tab, const double *const *__restrict__ cval_tab,
    const long long *__restrict__ boff, const double *__restrict__ Xcat, const double *__restrict__ Zcat, double *M,
    int m) {
    extern __shared__ __align__(16) double sb_sm[];
    const int k = blocks[blockIdx.x];
    const int n = bn[k], ncon = bncon[k], nn = n * n;
    if ((int)blockIdx.y * SB_W >= ncon) return;   // no constraint of this block for this CTA
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *Xs = sb_sm, *Zs = sb_sm + nn;
    double *W = sb_sm + 2 * nn + (size_t)warp * 2 * nn, *G = W + nn;
    const double *X = Xcat + boff[k], *Zi = Zcat + boff[k];
    for (int i = threadIdx.x; i < nn; i += SB_W * 32) { Xs[i] = X[i]; Zs[i] = Zi[i]; }
    __syncthreads();
    const int *con = con_tab[k];
    const long long *cptr = cptr_tab[k];
    const int *cpos = cpos_tab[k];
    const double *cval = cval_tab[k];
    for (int a = (int)blockIdx.y * SB_W + warp; a < ncon; a += SB_W * (int)gridDim.y) {
        for (int i = lane; i < nn; i += 32) W[i] = 0.0;
        __syncwarp();
        unsigned long long rows = 0;
        for (long long e = cptr[a]; e < cptr[a + 1]; e++) {   // every lane walks the entries in order
            const int pos = cpos[e], q = pos / n, p = pos - q * n;
            const double v = cval[e];
            rows |= 1ull << p;
            for (int j = lane; j < n; j += 32) W[p + j * n] += v * Zs[q + j * n];   // Zi symmetric
            __syncwarp();
        }
        for (int i = lane; i < nn; i += 32) {   // G = X W over the touched rows
            const int r = i % n, c = i / n;
            double acc = 0.0;
            for (unsigned long long b = rows; b; b &= b - 1) {
                const int p = __ffsll((long long)b) - 1;
                acc += Xs[r + p * n] * W[p + c * n];
            }
            G[i] = acc;
        }
        __syncwarp();
        const int ca = con[a];
        for (int b = a; b < ncon; b++) {
            double sum = 0.0;
            for (long long e = cptr[b] + lane; e < cptr[b + 1]; e += 32) sum += cval[e] * G[cpos[e]];
            sum = warp_sum(sum);
            if (lane == 0) {
                const int cb = con[b];
                M[(long long)ca + (long long)cb * m] += sum;
                if (ca != cb) M[(long long)cb + (long long)ca * m] += sum;
            }
        }
        __syncwarp();
    }
}
}  // namespace

size_t schur_small_smem(int nmax) { return (size_t)(2 + 2 * SB_W) * nmax * nmax * sizeof(double); }

int schur_assemble_small(cudaStream_t st, int count, const int *d_blocks, int nmax, int ncon_max, const int *d_n,
                         const int *d_ncon, const int *const *con_tab, const long long *const *cptr_tab,
                         const int *const *cpos_tab, const double *const *cval_tab, const long long *d_boff,
                         const double *Xcat, const double *Zicat, double *M, int m) {
    if (count <= 0) return BGPU_OK;
    if (nmax <= 0 || nmax > SB_NMAX) return BGPU_ERR_ARG;
    BGPU_ATTR_ONCE(BGPU_CHECK(cudaFuncSetAttribute(small_schur_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)schur_small_smem(SB_NMAX))));
    // enough CTAs per block that the launch fills the SMs twice over, one warp per constraint at most
    int dev = 0, nsm = 0;
    BGPU_CHECK(cudaGetDevice(&dev));
    BGPU_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int per_block = std::max(1, std::min(ceil_div(std::max(ncon_max, 1), SB_W), ceil_div(2 * nsm, count)));
    small_schur_kernel<<<dim3(count, per_block), SB_W * 32, schur_small_smem(nmax), st>>>(
        d_blocks, d_n, d_ncon, con_tab, cptr_tab, cpos_tab, cval_tab, d_boff, Xcat, Zicat, M, m);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

// ---- the LP route ----------------------------------------------------------------------------
namespace {
constexpr int LP_WARPS = 8;
// One warp per local constraint a: for each variable p of a (ascending), w = A[a,p] d_p, and the
// lanes add w A[b,p] to M[b, a] and M[a, b] for the constraints b >= a of p.  Within one p every
// b is distinct, and __syncwarp orders one p after the next, so each entry of column gcon[a] sums
// its terms by ascending p with no atomics; no other warp writes that column or its mirror row.
__global__ void __launch_bounds__(LP_WARPS * 32) lp_schur_kernel(
    int nc, const int *__restrict__ gcon, const long long *__restrict__ aptr, const int *__restrict__ avar,
    const double *__restrict__ aval, const long long *__restrict__ vptr, const int *__restrict__ vcon,
    const double *__restrict__ vval, const double *__restrict__ Xv, const double *__restrict__ Zv, double *M,
    int m) {
    const int lane = threadIdx.x & 31;
    const int ta = blockIdx.x * LP_WARPS + (threadIdx.x >> 5);
    if (ta >= nc) return;
    const long long ga = gcon[ta];
    for (long long e = aptr[ta]; e < aptr[ta + 1]; e++) {
        const int p = avar[e];
        const double w = aval[e] * (Xv[p] * Zv[p]);
        // the entries of p below a: p's list is sorted by constraint, so start at a's own entry
        long long lo = vptr[p], hi = vptr[p + 1];
        while (lo < hi) {
            const long long mid = (lo + hi) >> 1;
            if (vcon[mid] < ta) lo = mid + 1; else hi = mid;
        }
        for (long long f = lo + lane; f < vptr[p + 1]; f += 32) {
            const int tb = vcon[f];
            const long long gb = gcon[tb];
            const double v = w * vval[f];
            M[gb + ga * m] += v;
            if (tb != ta) M[ga + gb * m] += v;
        }
        __syncwarp();
    }
}
}  // namespace

int schur_assemble_lp(cudaStream_t st, const LpGroupDev &G, const double *Xv, const double *Zv, double *M, int m) {
    if (G.nc <= 0 || G.ne <= 0) return BGPU_OK;
    if (!G.gcon || !G.aptr || !G.avar || !G.aval || !G.vptr || !G.vcon || !G.vval || !Xv || !Zv || !M)
        return BGPU_ERR_ARG;
    lp_schur_kernel<<<ceil_div(G.nc, LP_WARPS), LP_WARPS * 32, 0, st>>>(G.nc, G.gcon, G.aptr, G.avar, G.aval, G.vptr,
                                                                         G.vcon, G.vval, Xv, Zv, M, m);
    BGPU_LAUNCH_CHECK();
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
