// The step-length Lanczos on the device (sdp_maxstep_lam, solver.c:6083-6225): lambda_min of the
// explicit B = L^-1 dV L^-T of one block, estimated as theta - res from at most K <= 30 steps
// from the fixed start vector.
//
// The host issues, per step j, the matrix-vector product w = B q_j (symv_full_f64, all SMs) and
// lanczos_step_kernel (one CTA): alpha_j = q_j'w, w orthogonalised twice against q_0 .. q_j
// (classical Gram-Schmidt, each pass all j + 1 products at once, where the reference takes them
// one after the other: the same projection, rounded differently), beta_j = |w|, and from the
// sixth step every third step the Ritz bound of the tridiagonal T decides the stop (warp 0).
// The state (alpha, beta, the step count, the stop flag, the estimate) stays in device memory:
// the host reads it at those checkpoints only, instead of a round trip a step.  A step after the
// stop is a no-op.
#include "common.cuh"
#include "kernels.h"

#include <cmath>

namespace {
constexpr int LZ_T = 1024;   // threads of the step kernel

__device__ int sturm_below_d(int k, const double *a, const double *b, double x) {
    int cnt = 0;
    double q = a[0] - x;
    if (q < 0) cnt++;
    for (int i = 1; i < k; i++) {
        if (q == 0) q = 1e-300;
        q = (a[i] - x) - b[i - 1] * b[i - 1] / q;
        if (q < 0) cnt++;
    }
    return cnt;
}

// theta = lambda_min(T_k) (alpha[0..k-1], beta[0..k-2]) and the residual bound |beta[k-1] z[k-1]|
// of its unit eigenvector z (ritz_bound, solver.c:6030-6039), called by all 32 lanes of a warp,
// which return the same values.  theta by multisection of the Gershgorin interval: each round
// the lanes take the Sturm count at 32 interior points, and the interval shrinks to the cell
// that holds the smallest eigenvalue (the count is monotone in x), until no interior point is
// left (lo and hi adjacent doubles, as bisection ends).  z by three passes of inverse iteration
// on T - (theta - 1e-10 scale) I, Gaussian elimination with partial pivoting on the band (two
// rows and three columns a step: the other entries are zeros).
__device__ double ritz_bound_w(int k, const double *alpha, const double *beta, double *theta) {
    const int lane = threadIdx.x & 31;
    double lo = 1e300, hi = -1e300;
    for (int i = 0; i < k; i++) {
        const double r = (i > 0 ? fabs(beta[i - 1]) : 0) + (i + 1 < k ? fabs(beta[i]) : 0);
        lo = fmin(lo, alpha[i] - r);
        hi = fmax(hi, alpha[i] + r);
    }
    if (!isfinite(lo) || !isfinite(hi)) { *theta = 0; return 1e300; }
    for (int it = 0; it < 64; it++) {
        const double x = lo + (hi - lo) * ((lane + 1) / 33.0);
        const bool in = x > lo && x < hi;
        const unsigned valid = __ballot_sync(0xffffffffu, in);
        if (!valid) break;
        const unsigned below = __ballot_sync(0xffffffffu, in && sturm_below_d(k, alpha, beta, x) >= 1);
        double nhi = hi, nlo = lo;
        unsigned under = valid & ~below;
        if (below) {
            const int f = __ffs(below) - 1;
            nhi = __shfl_sync(0xffffffffu, x, f);
            under &= (1u << f) - 1;
        }
        if (under) nlo = __shfl_sync(0xffffffffu, x, 31 - __clz(under));
        lo = nlo;
        hi = nhi;
    }
    const double th = 0.5 * (lo + hi);
    *theta = th;
    const double scale = fmax(fabs(lo), fabs(hi));
    if (!(scale > 1e-280)) return fabs(beta[k - 1]);   // a zero operator: theta = 0, |z_k| <= 1
    const double sh = th - 1e-10 * scale;
    // row r of the band: sub (column r - 1), d0 (r), d1 (r + 1), d2 (r + 2, fill from a swap)
    double z[32], sub[32], d0[32], d1[32], d2[32], w[32];
    for (int i = 0; i < k; i++) z[i] = 1.0 / sqrt((double)k) * (1.0 + 0.01 * i);
    for (int pass = 0; pass < 3; pass++) {
        for (int i = 0; i < k; i++) {
            d0[i] = alpha[i] - sh;
            d1[i] = i + 1 < k ? beta[i] : 0.0;
            d2[i] = 0.0;
            sub[i] = i > 0 ? beta[i - 1] : 0.0;
            w[i] = z[i];
        }
        for (int c = 0; c < k; c++) {
            if (c + 1 < k && fabs(sub[c + 1]) > fabs(d0[c])) {   // swap rows c and c + 1
                const double t0 = d0[c], t1 = d1[c], t2 = d2[c];
                d0[c] = sub[c + 1];
                d1[c] = d0[c + 1];
                d2[c] = d1[c + 1];
                sub[c + 1] = t0;
                d0[c + 1] = t1;
                d1[c + 1] = t2;
                const double tw = w[c];
                w[c] = w[c + 1];
                w[c + 1] = tw;
            }
            if (d0[c] == 0) d0[c] = 1e-300;
            if (c + 1 < k) {
                const double f = sub[c + 1] / d0[c];
                if (f != 0) {
                    sub[c + 1] = 0.0;
                    d0[c + 1] -= f * d1[c];
                    d1[c + 1] -= f * d2[c];
                    w[c + 1] -= f * w[c];
                }
            }
        }
        for (int c = k - 1; c >= 0; c--) {
            double s = w[c];
            if (c + 1 < k) s -= d1[c] * z[c + 1];
            if (c + 2 < k) s -= d2[c] * z[c + 2];
            z[c] = s / d0[c];
        }
        double zmax = 0;
        for (int i = 0; i < k; i++) zmax = fmax(zmax, fabs(z[i]));
        if (!(zmax > 0) || !isfinite(zmax)) return fabs(beta[k - 1]);   // the trivial bound |z_k| <= 1
        double nz = 0;
        for (int i = 0; i < k; i++) {
            z[i] /= zmax;
            nz += z[i] * z[i];
        }
        nz = sqrt(nz);
        for (int i = 0; i < k; i++) z[i] /= nz;
    }
    return fabs(beta[k - 1] * z[k - 1]);
}

__device__ double block_sum(double v, double *red) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();   // red is free (its last reader passed this barrier)
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double s = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
        s = warp_sum(s);
        if (lane == 0) red[32] = s;
    }
    __syncthreads();
    return red[32];
}

__global__ void __launch_bounds__(LZ_T) lanczos_start_kernel(int n, const double *__restrict__ q0, double *Q,
                                                             LanczosState *st) {
    __shared__ double red[33];
    double s = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += q0[i] * q0[i];
    const double inv = 1.0 / sqrt(block_sum(s, red));
    for (int i = threadIdx.x; i < n; i += blockDim.x) Q[i] = q0[i] * inv;
    if (threadIdx.x == 0) {
        st->kk = 0;
        st->done = 0;
        st->scale = 0;
        st->lam = -1e300;
    }
}

__global__ void __launch_bounds__(LZ_T) lanczos_step_kernel(int n, int j, int K, double *Q, double *w,
                                                            LanczosState *st) {
    __shared__ double red[33];
    __shared__ double c[32], sa[32], sb[32];
    __shared__ int stop;
    if (st->done) return;   // (the same value in every thread: one block)
    const double *qj = Q + (long long)j * n;
    double s = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += qj[i] * w[i];
    const double a = block_sum(s, red);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int pass = 0; pass < 2; pass++) {
        for (int i = warp; i <= j; i += nw) {   // c_i = q_i'w, a warp a product
            const double *qi = Q + (long long)i * n;
            double t = 0;
            for (int r = lane; r < n; r += 32) t += qi[r] * w[r];
            t = warp_sum(t);
            if (lane == 0) c[i] = t;
        }
        __syncthreads();
        for (int r = threadIdx.x; r < n; r += blockDim.x) {
            double v = w[r];
            for (int i = 0; i <= j; i++) v -= c[i] * Q[(long long)i * n + r];
            w[r] = v;
        }
        __syncthreads();
    }
    s = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += w[i] * w[i];
    const double b = sqrt(block_sum(s, red));
    if (warp == 0) {
        const int kk = j + 1;
        const double scale = fmax(st->scale, fabs(a));
        for (int i = lane; i < j; i += 32) {
            sa[i] = st->alpha[i];
            sb[i] = st->beta[i];
        }
        int done = 0;
        if (lane == 0) {
            sa[j] = a;
            sb[j] = b;
        }
        if (b <= 1e-12 * (scale + 1e-300)) {
            if (lane == 0) sb[j] = 0;
            done = 1;
        }
        __syncwarp();
        double theta = 0, res = 0;
        bool have = false;
        if (!done && kk >= 6 && kk % 3 == 0) {
            res = ritz_bound_w(kk, sa, sb, &theta);
            have = true;
            if (res <= 0.02 * fabs(theta) + 1e-14 * scale) done = 1;
        }
        if (kk >= K) done = 1;
        if (done && !have) res = ritz_bound_w(kk, sa, sb, &theta);
        if (lane == 0) {
            st->alpha[j] = a;
            st->beta[j] = sb[j];
            st->scale = scale;
            st->kk = kk;
            if (done) st->lam = res > 1e299 ? -1e300 : theta - res;
            st->done = done;
            stop = done;
        }
    }
    __syncthreads();
    if (!stop) {
        const double inv = 1.0 / b;
        double *qn = Q + (long long)(j + 1) * n;
        for (int i = threadIdx.x; i < n; i += blockDim.x) qn[i] = w[i] * inv;
    }
}
}  // namespace

int lanczos_start(cudaStream_t s, int n, const double *q0, double *Q, LanczosState *st) {
    if (n < 1) return BGPU_ERR_ARG;
    lanczos_start_kernel<<<1, LZ_T, 0, s>>>(n, q0, Q, st);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}

int lanczos_step(cudaStream_t s, int n, int j, int K, double *Q, double *w, LanczosState *st) {
    if (n < 1 || j < 0 || j >= K || K > 30) return BGPU_ERR_ARG;
    lanczos_step_kernel<<<1, LZ_T, 0, s>>>(n, j, K, Q, w, st);
    BGPU_LAUNCH_CHECK();
    return BGPU_OK;
}
