// The Nesterov-Todd scaling of SDP blocks and the element-wise pieces of the NT direction in the
// scaled space (nt.cu; the reference's nt_scaling / nt_rhs_scaled, solver.c:7803-7912, 8071-8090).
//
//   X = L_X L_X',  Z = L_Z L_Z',  L_Z' L_X = U diag(lam) V'
//   G = L_X V diag(lam)^-1/2,  W = G G'  (W Z W = X),  G' Z G = G^-1 X G^-T = diag(lam).
#pragma once
#include <cuda_runtime.h>

namespace nt {

constexpr int SMALL_NMAX = 64;   // the one-CTA-per-block form
constexpr int MAX_SWEEPS = 40;   // Jacobi sweeps before a block counts as failed

// Blocks of order <= SMALL_NMAX, one CTA each: from the factors LX, LZ (lower; the strict upper
// triangle is ignored) to G (n x n), lam (n) and W = G G' (n x n, exactly symmetric).  info[k]:
// 0, 1 a singular value not positive or not finite, 2 Jacobi did not converge in MAX_SWEEPS.
// nmax: the largest listed order.
int scaling_small(cudaStream_t st, int nb, const int *d_n, int nmax, const double *const *LX,
                  const double *const *LZ, double *const *G, double *const *lam, double *const *W, int *info);

// A large block in steps: out = tril(L);  Mb = L_Z' L_X is formed by the caller (a GEMM of the
// two triangles);  jacobi() rotates the columns of Mb and U (= tril(L_X) on entry) until Mb's
// columns are orthogonal (then U = L_X V), one host synchronisation per sweep (d_flag: a device
// int, h_flag: pinned host int); *sweeps = the sweeps taken, -1 when MAX_SWEEPS did not suffice.
// finish(): lam_j = |Mb(:, j)|, U(:, j) /= sqrt(lam_j) (U becomes G); *d_info = 1 (device) when a
// lam_j is not positive or not finite.
int tril(cudaStream_t st, int n, const double *L, double *out);
int jacobi(cudaStream_t st, int n, double *Mb, double *U, int *d_flag, int *h_flag, int *sweeps);
int finish(cudaStream_t st, int n, const double *Mb, double *U, double *lam, int *d_info);

// Over blocks stored one after another (block k: order d_n[k], n x n entries from d_off[k], its
// lam from d_loff[k]; total = d_off[nb]):
// Rt = L_lam^-1 (smu I - diag(lam)^2 - H), L_lam^-1(M)_ij = 2 M_ij / (lam_i + lam_j) (H may be null;
// d_smu, when not null, holds one smu per block instead)
int rhs_scaled(cudaStream_t st, int nb, const int *d_n, const long long *d_off, const long long *d_loff,
               long long total, const double *lam, double smu, const double *H, double *Rt,
               const double *d_smu = nullptr);
// out = src + alpha diag(lam) (out may alias src)
int add_lam(cudaStream_t st, int nb, const int *d_n, const long long *d_off, const long long *d_loff,
            long long total, const double *lam, double alpha, const double *src, double *out);

}  // namespace nt
