// 3xTF32 split-product GEMM on the tcgen05 tensor cores (tf32x3.cu).
#pragma once
#include <cuda_runtime.h>

// tf32 rounding (round to nearest, ties away) of a float, returned as a float whose low 13
// mantissa bits are zero.
__device__ __forceinline__ float tf32_round(float x) {
    unsigned r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// hi = tf32(x), lo = tf32(x - hi) for n doubles x (x is rounded to float first).
int split_tf32(cudaStream_t st, long long n, const double *x, float *hi, float *lo);

// G(i, j) = sum_k A(i, k) B(k, j) with A = Ah + Al (K-major rows: A[i*lda + k]) and
// B = Bh + Bl (K-major columns: B[k + j*ldb]), computed as Ah Bh + Ah Bl + Al Bh in FP32
// accumulation; G column-major (G[i + j*ldg]).
int gemm_tf32x3(cudaStream_t st, int M, int N, int K, const float *Ah, const float *Al, long long lda,
                const float *Bh, const float *Bl, long long ldb, float *G, long long ldg);

// The sticky device flag of the tcgen05 GEMM: 1 once a bounded wait ran out (read, not reset).
int tf32x3_error_flag(int *host_value);
