/* oracle.h -- TEST INFRASTRUCTURE ONLY.  A CPU restatement of the FPLUS numeric path (fplus_factor / fplus_solve with
 * partial pivoting and drop_tol 0) used by the tests, smoke() and the benchmark's CPU baseline as the checker of the CUDA
 * path.  Nothing in the product links or calls it.
 *
 * Pinned against the reference itself (oracle/_ref/libfplusref.so, built from the reference sources by oracle/Makefile)
 * and against the committed golden fixtures (tests/golden/).
 */
#ifndef FPLUS_ORACLE_H
#define FPLUS_ORACLE_H
#include <stddef.h>
#include <stdint.h>

typedef struct orc_numeric orc_numeric;

/* B = A[row_perm, :][:, col_perm] in canonical CSC (FPLUS src/pipeline.c:14-82); Bp (n+1), Bi, Bx (nnz) caller-allocated */
int orc_permute_csc(int64_t n, const int64_t *Ap, const int64_t *Ai, const void *Ax, int is_complex,
                    const int64_t *row_perm, const int64_t *col_perm, int64_t *Bp, int64_t *Bi, void *Bx);

/* Ruiz L-inf equilibration of a CSC matrix in place (FPLUS src/equil.c:60-183, 186-441): the same operations in the same
 * order, so Dr, Dc and the scaled values are bit-identical.  Returns 0, -2 (a zero line) or -3 (range beyond double). */
int orc_ruiz(int64_t n, const int64_t *Bp, const int64_t *Bi, void *Bx, int is_complex, int max_iter, double tol,
             double *Dr, double *Dc, int *iters, char *err, size_t errlen);

/* fplus_factor with partial pivoting (FPLUS src/numeric.c:39-83, src/pipeline.c:84-111, src/factor_sn.c): permute,
 * Ruiz (when equilibrate), left-looking LU with partial pivoting, then p, q, Dr, Dc composed into original coordinates. */
int orc_factor(int64_t n, const int64_t *Ap, const int64_t *Ai, const void *Ax, int is_complex,
               const int64_t *row_perm, const int64_t *col_perm, int equilibrate, int ruiz_max_iter, double ruiz_tol,
               double pivot_rel, orc_numeric **out, char *err, size_t errlen);

/* fplus_solve (FPLUS src/numeric.c:88-131): trans 0 A x = b, 1 A^T x = b, 2 A^H x = b, in place, column-major b */
int orc_solve(const orc_numeric *num, void *b, int64_t nrhs, int64_t ldb, int trans);

void orc_free(orc_numeric *num);

/* the factors of the scaled permuted matrix: L unit lower (diagonal first, pivot-order rows), U upper (diagonal last) */
int64_t orc_n(const orc_numeric *num);
const int64_t *orc_Lp(const orc_numeric *num);
const int64_t *orc_Li(const orc_numeric *num);
const void *orc_Lx(const orc_numeric *num);
const int64_t *orc_Up(const orc_numeric *num);
const int64_t *orc_Ui(const orc_numeric *num);
const void *orc_Ux(const orc_numeric *num);
const int64_t *orc_p_lu(const orc_numeric *num);      /* pivot step k -> row of the permuted matrix */
const int64_t *orc_p(const orc_numeric *num);         /* composed: original row of pivot step k */
const int64_t *orc_q(const orc_numeric *num);
const double *orc_Dr(const orc_numeric *num);         /* original coordinates */
const double *orc_Dc(const orc_numeric *num);
const double *orc_Drp(const orc_numeric *num);        /* permuted coordinates (as Ruiz produced them) */
const double *orc_Dcp(const orc_numeric *num);
int orc_ruiz_iters(const orc_numeric *num);
/* the scaled permuted matrix the LU factored (CSC) */
const int64_t *orc_Bp(const orc_numeric *num);
const int64_t *orc_Bi(const orc_numeric *num);
const void *orc_Bx(const orc_numeric *num);

#endif
