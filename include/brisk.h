/*
 * brisk.h - the C interface of libbrisk (B200 build).
 *
 * Drop-in for the reference's flat C interface (capi.c) on the semidefinite interior-point
 * path: the same exported names, argument meaning, return codes and accessors, so a caller
 * that links or dlopens libbrisk (ctypes in python/brisk/_core.py, Julia's ccall, a C program
 * like tools/capi_test.c) works unchanged.  The Newton step of every solve runs on the GPU.
 *
 *   (P) min <C,X> s.t. <A_i,X> = b_i, X >= 0      (D) max b'y s.t. C - sum y_i A_i = Z >= 0
 *   with C = -F0, A_i = F_i, b = c in SDPA numbering.
 *
 * The result is an opaque handle read through the accessors.  Not reentrant: callers
 * serialize solves (as the reference, capi.c:19-20).
 */
#ifndef BRISK_B200_H
#define BRISK_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define BRISK_API __attribute__((visibility("default")))
#else
#define BRISK_API
#endif

typedef struct BriskResult BriskResult;

/* Output: mode 0 stdout/stderr, 1 errors only, 2 every piece to cb(s, is_err).
 * Replaces capi.c:60 brisk_set_output. */
BRISK_API void brisk_set_output(int mode, int (*cb)(const char *s, int is_err));
/* Replaces capi.c:65 brisk_version ("1.7-b200"). */
BRISK_API const char *brisk_version(void);

/* Result handle and accessors.  Replace capi.c:68-138 (brisk_result_new ... brisk_result_Z). */
BRISK_API BriskResult *brisk_result_new(void);
BRISK_API void brisk_result_delete(BriskResult *r);
BRISK_API int brisk_result_status(const BriskResult *r);          /* 0 optimal .. 6 time limit, -1 not solved */
BRISK_API const char *brisk_result_status_str(const BriskResult *r);
BRISK_API int brisk_result_exit_code(const BriskResult *r);
BRISK_API int brisk_result_iterations(const BriskResult *r);
BRISK_API int brisk_result_m(const BriskResult *r);
BRISK_API int brisk_result_nblk(const BriskResult *r);
BRISK_API int brisk_result_blocksize(const BriskResult *r, int k);
BRISK_API double brisk_result_pobj(const BriskResult *r);         /* <C,X> on the data as given */
BRISK_API double brisk_result_dobj(const BriskResult *r);         /* b'y */
BRISK_API double brisk_result_time(const BriskResult *r);
BRISK_API int brisk_result_have_x(const BriskResult *r);
BRISK_API void brisk_result_dimacs(const BriskResult *r, double *err);   /* 6 DIMACS errors */
BRISK_API const double *brisk_result_y(const BriskResult *r);
BRISK_API const double *brisk_result_X(const BriskResult *r, int k);     /* n x n column-major */
BRISK_API const double *brisk_result_Z(const BriskResult *r, int k);
/* Bound mode, re-solves and causes are not part of this path: the reference's accessors
 * (capi.c:100-121, 123-126) answer "none" here. */
BRISK_API int brisk_result_bound(const BriskResult *r, double *out);
BRISK_API int brisk_result_resolves(const BriskResult *r, double *t);
BRISK_API const char *brisk_result_cause(const BriskResult *r);

/* Interrupts (capi.c:165-168). */
BRISK_API void brisk_interrupt(void);
BRISK_API int brisk_interrupted(void);
BRISK_API void brisk_clear_interrupt(void);
BRISK_API void brisk_set_interrupt_owner(int caller);

/* Solve the SDPA problem given by its numbers: block sizes bs (an LP block is a negative size:
 * its variables are solved as blocks of order 1, and brisk_result_X / brisk_result_Z return it
 * as its vector of values, as the reference does), c (m), entries (mat, blk, i, j, v), 1-based as
 * in the file, mat 0 = F0.  Options are command-line strings.  Returns the exit code: 0 optimal, 10
 * reduced accuracy, 11/12 primal/dual infeasible, 13 iteration limit, 14 numerical
 * difficulties, 15 time limit, 1 bad options, 2 unreadable problem, < 0 abort.
 * Replaces capi.c:175 brisk_solve_data. */
BRISK_API int brisk_solve_data(int m, int nblk, const int *bs, const double *c, int64_t nnz, const int *mat,
                               const int *blk, const int *i, const int *j, const double *v, int nopt,
                               const char *const *opts, BriskResult *res);
/* Solve an SDPA sparse file.  Replaces capi.c:520 brisk_solve_file. */
BRISK_API int brisk_solve_file(const char *fname, int nopt, const char *const *opts, BriskResult *res);

#ifdef __cplusplus
}
#endif
#endif
