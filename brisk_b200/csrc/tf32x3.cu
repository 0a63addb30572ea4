// 3xTF32 split-product GEMM (tcgen05).  The split kernel is here; the tensor-core GEMM is
// added with the mixed-precision path.
#include "common.cuh"
#include "kernels.h"
#include "tf32x3.h"

namespace {
__global__ void split_kernel(long long n, const double *x, float *hi, float *lo) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = x[i];
    const float h = tf32_round((float)v);
    hi[i] = h;
    lo[i] = tf32_round((float)(v - (double)h));
}
}  // namespace

int split_tf32(cudaStream_t st, long long n, const double *x, float *hi, float *lo) {
    if (n <= 0) return BGPU_OK;
    split_kernel<<<ceil_div(n, 256), 256, 0, st>>>(n, x, hi, lo);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int gemm_tf32x3(cudaStream_t, int, int, int, const float *, const float *, long long, const float *, const float *,
                long long, float *, long long) {
    return BGPU_ERR_UNSUPPORTED;
}
