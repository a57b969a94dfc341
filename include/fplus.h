/* fplus.h -- the FPLUS C interface, served by the B200 build (libfplus.so).
 *
 * The declarations, struct layouts, enum values and macro values below are the FPLUS C interface (FPLUS include/fplus.h);
 * they are kept identical so that a program or binding written against FPLUS links against this library unchanged.  Each
 * entry point names the FPLUS declaration it replaces.
 *
 * Conventions (FPLUS include/fplus.h:3-5): int64 indices; values double or C99 double complex (interleaved re, im),
 * chosen by is_complex; every entry point returns FPLUS_OK or a negative FPLUS_ERR_* code with a message in err (when err
 * is not NULL).  Handles are independent: separate handles may be used from separate host threads.  In this build every
 * numeric step (permutation, Ruiz equilibration, the supernodal LU and the triangular solves) runs on the GPU; the
 * symbolic analysis runs on the host.  CUDA failures are reported as FPLUS_ERR_GPU.
 */
#ifndef FPLUS_H
#define FPLUS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* return codes (FPLUS include/fplus.h:17-24) */
enum {
    FPLUS_OK = 0,
    FPLUS_ERR_NOMEM = -1,      /* host or device allocation failed */
    FPLUS_ERR_SINGULAR = -2,   /* no admissible pivot, an all-zero row or column, or a zero diagonal in a solve */
    FPLUS_ERR_BADARG = -3,     /* invalid argument */
    FPLUS_ERR_GPU = -4,        /* a CUDA call failed, or a device-side wait gave up */
    FPLUS_ERR_INTERNAL = -5
};

/* pivot strategies (FPLUS include/fplus.h:27-29); this build factors with partial pivoting */
#define FPLUS_PIVOT_FULL    0
#define FPLUS_PIVOT_PARTIAL 1
#define FPLUS_PIVOT_ROOK    2

/* sqrt(DBL_EPSILON) (FPLUS include/fplus.h:32) */
#define FPLUS_PIVOT_REL_DEFAULT 1.4901161193847656e-08

/* Host copies of L and U (FPLUS include/fplus.h:37-46): P A Q = L U in the scaled, statically ordered coordinates,
 * column-compressed (csc = 1); L unit lower with its unit diagonal stored first in every column, U upper with its
 * diagonal stored. */
typedef struct {
    int64_t n;
    int is_complex;
    int csc;
    int64_t *Lp, *Li; void *Lx;
    int64_t *Up, *Ui; void *Ux;
    int64_t *p, *q;
    int64_t nsupernodes;
    int64_t n_pivots_replaced;
} fplus_factors;

/* FPLUS include/fplus.h:48.  Also releases the device copy of factors returned by fplus_factor_sn_perm / _sym. */
void fplus_factors_free(fplus_factors *f);

/* ---- the low-level interface (what FPLUS's Python extension calls: _sparse_lu_c.c:360, 526) ---- */

/* FPLUS include/fplus.h:54-56: the LU with partial pivoting of the matrix as given (no permutation, no equilibration; q
 * the identity).  The CSC input is checked but need not be sorted: repeated entries of a column are summed.
 * relax_rows, panel, use_gpu and gpu_min_flops are accepted; the work runs on the GPU as fplus_factor_sn_perm's with
 * identity orders. */
int fplus_factor_sn(int64_t n, const int64_t *Ap, const int64_t *Ai, const void *Ax, int is_complex, int verbose,
                    int64_t relax_rows, int64_t panel, int use_gpu, double gpu_min_flops, double pivot_rel,
                    fplus_factors *out, char *err, size_t errlen);

/* FPLUS include/fplus.h:60-62, 139-147: the row kernel (full, partial or rook pivoting on CSR input, incomplete LU).  Not
 * built in this library: every call returns FPLUS_ERR_BADARG with a message (partial pivoting is fplus_factor_sn*). */
int fplus_factor_row(int64_t n, const int64_t *indptr, const int64_t *indices, const void *data, double drop_tol,
                     int is_complex, int verbose, int pivot_strategy, double pivot_rel,
                     fplus_factors *out, char *err, size_t errlen);
int fplus_factor_row_perm(int64_t n, const int64_t *Ap, const int64_t *Ai, const void *Ax, int is_complex,
                          const int64_t *row_perm, const int64_t *col_perm,
                          int equilibrate, int ruiz_max_iter, double ruiz_tol, int verbose,
                          double drop_tol, int pivot_strategy, double pivot_rel,
                          fplus_factors *out, double *Dr, double *Dc, char *err, size_t errlen);

/* FPLUS include/fplus.h:64-67: Ruiz L-inf equilibration in place: data (CSR, or CSC when is_csc) becomes
 * diag(Dr) A diag(Dc); Dr, Dc (length n) are filled.  Both routes give the same scalings.  On the GPU. */
int fplus_ruiz(int64_t n, const int64_t *indptr, const int64_t *indices, void *data, int is_complex, int is_csc,
               int max_iter, double tol, int verbose, double *Dr, double *Dc, char *err, size_t errlen);

/* FPLUS include/fplus.h:73-74: triangular solve in place on x (one right-hand side): trans 0 solves L U x = b, 1
 * (L U)^T x = b, 2 (L U)^H x = b.  L unit lower (an explicit unit diagonal is skipped), U upper with its diagonal stored.
 * FPLUS_ERR_SINGULAR for a zero or missing diagonal in U.  On the GPU, through a plan made for the call. */
int fplus_tri_solve(int64_t n, const int64_t *Lp, const int64_t *Li, const void *Lx, const int64_t *Up, const int64_t *Ui,
                    const void *Ux, void *x, int trans, int is_complex);

/* FPLUS include/fplus.h:81-88: solve plans.  A plan is made once per factorization from the CSC patterns; then
 * fplus_tri_solve_plan solves for nrhs right-hand sides stored column-major in x (leading dimension ldx >= n), in place,
 * with the same factor arrays.  A zero or missing diagonal in U fails (FPLUS_ERR_SINGULAR) before x is touched.  In this
 * build the solves run on the GPU: for the arrays fplus_factor_sn_perm / _sym returned (the same pointers, the values
 * unchanged) with the factorization's device copy; for any other CSC factors with level-scheduled sweeps over the arrays
 * given.  nsupernodes: the fronts of the factorization for the former, -1 for the latter. */
typedef struct fplus_solve_plan fplus_solve_plan;
int fplus_solve_plan_create(int64_t n, const int64_t *Lp, const int64_t *Li, const int64_t *Up, const int64_t *Ui,
                            fplus_solve_plan **plan, char *err, size_t errlen);
int fplus_tri_solve_plan(const fplus_solve_plan *plan, int64_t n, const int64_t *Lp, const int64_t *Li, const void *Lx,
                         const int64_t *Up, const int64_t *Ui, const void *Ux, void *x, int64_t nrhs, int64_t ldx,
                         int trans, int is_complex);
int64_t fplus_solve_plan_nsupernodes(const fplus_solve_plan *plan);
void fplus_solve_plan_free(fplus_solve_plan *plan);

/* ---- symbolic analysis (FPLUS include/fplus.h:94-120) ---- */
typedef struct fplus_symbolic fplus_symbolic;

#define FPLUS_ORDER_COLAMD  0
#define FPLUS_ORDER_AMD_ATA 1
#define FPLUS_ORDER_AUTO    2

/* FPLUS include/fplus.h:101-103: dense-line pinning, a fill-reducing column order on the remaining pattern, and (postorder)
 * the column-etree postorder.  Dense rows go last in the row order, dense columns last in the column order. */
int fplus_analyze(int64_t n, const int64_t *Ap, const int64_t *Ai, int pin_dense, double tau_density, int64_t tau_min_nnz,
                  const unsigned char *tau_row_mask, const unsigned char *tau_col_mask, int postorder,
                  fplus_symbolic **sym, char *err, size_t errlen);
/* FPLUS include/fplus.h:111-113 */
int fplus_analyze_ord(int64_t n, const int64_t *Ap, const int64_t *Ai, int pin_dense, double tau_density, int64_t tau_min_nnz,
                      const unsigned char *tau_row_mask, const unsigned char *tau_col_mask, int postorder, int ordering,
                      fplus_symbolic **sym, char *err, size_t errlen);
void fplus_symbolic_free(fplus_symbolic *sym);
int64_t fplus_symbolic_n(const fplus_symbolic *sym);
int64_t fplus_symbolic_nnz(const fplus_symbolic *sym);
const int64_t *fplus_symbolic_row_perm(const fplus_symbolic *sym);   /* A[row_perm, :][:, col_perm] is factored */
const int64_t *fplus_symbolic_col_perm(const fplus_symbolic *sym);
int64_t fplus_symbolic_n_dense_rows(const fplus_symbolic *sym);
int64_t fplus_symbolic_n_dense_cols(const fplus_symbolic *sym);

/* FPLUS include/fplus.h:125-129: the factorization of A[row_perm, :][:, col_perm] (A canonical CSC): the permuted
 * matrix, Ruiz (when equilibrate; Dr, Dc of length n filled, in the permuted order), then the LU with partial pivoting.
 * The host factors in *out and p (q the identity) refer to the permuted matrix; free them with fplus_factors_free.
 * relax_rows, panel, use_gpu and gpu_min_flops are accepted; the work runs on the GPU as in fplus_factor.  The device
 * factors are kept with the returned arrays, so that a plan made on those arrays solves with them. */
int fplus_factor_sn_perm(int64_t n, const int64_t *Ap, const int64_t *Ai, const void *Ax, int is_complex,
                         const int64_t *row_perm, const int64_t *col_perm,
                         int equilibrate, int ruiz_max_iter, double ruiz_tol, int verbose,
                         int64_t relax_rows, int64_t panel, int use_gpu, double gpu_min_flops, double pivot_rel,
                         fplus_factors *out, double *Dr, double *Dc, char *err, size_t errlen);
/* FPLUS include/fplus.h:130-134: the same with the orders of a symbolic analysis (the pattern must be the analysed one) */
int fplus_factor_sn_sym(const fplus_symbolic *sym, const int64_t *Ap, const int64_t *Ai, const void *Ax, int is_complex,
                        int equilibrate, int ruiz_max_iter, double ruiz_tol, int verbose,
                        int64_t relax_rows, int64_t panel, int use_gpu, double gpu_min_flops, double pivot_rel,
                        fplus_factors *out, double *Dr, double *Dc, char *err, size_t errlen);

/* FPLUS include/fplus.h:144-147: the row kernel on a symbolic analysis's orders; not built (FPLUS_ERR_BADARG) */
int fplus_factor_row_sym(const fplus_symbolic *sym, const int64_t *Ap, const int64_t *Ai, const void *Ax, int is_complex,
                         int equilibrate, int ruiz_max_iter, double ruiz_tol, int verbose,
                         double drop_tol, int pivot_strategy, double pivot_rel,
                         fplus_factors *out, double *Dr, double *Dc, char *err, size_t errlen);

/* FPLUS include/fplus.h:92: postorder of the column elimination tree of the m x n CSC pattern; post[k] = the column placed
 * k-th. */
int fplus_coletree_postorder(int64_t m, int64_t n, const int64_t *Ap, const int64_t *Ai, int64_t *post);

/* ---- the high-level interface (FPLUS include/fplus.h:150-200) ---- */
typedef struct {
    int     pin_dense;          /* dense rows / columns last (1) */
    double  tau_density;        /* a line is dense with more than max(tau_density n, tau_min_nnz) entries (0.5) */
    int64_t tau_min_nnz;        /* (10) */
    int     postorder;          /* column-etree postorder after the fill-reducing order (1) */
    int     equilibrate;        /* Ruiz (1) */
    int     ruiz_max_iter;      /* (20) */
    double  ruiz_tol;           /* (1e-2) */
    double  pivot_rel;          /* singular when the best pivot < pivot_rel * the column's max (FPLUS_PIVOT_REL_DEFAULT) */
    int     pivot_strategy;     /* FPLUS_PIVOT_PARTIAL (the only strategy of this build) */
    double  drop_tol;           /* 0: exact LU (the only mode of this build) */
    int64_t relax_rows;         /* accepted; the supernode partition of this build is static (symbolic analysis) */
    int64_t panel;              /* accepted; caps the width of a supernode of the static partition (512) */
    int     use_gpu;            /* accepted and ignored: the numeric phase always runs on the GPU */
    double  gpu_min_flops;      /* accepted and ignored */
    int     verbose;            /* (0) */
} fplus_options;

/* FPLUS include/fplus.h:168 (defaults: FPLUS src/numeric.c:15-22) */
void fplus_default_options(fplus_options *opt);

/* FPLUS include/fplus.h:171-172 */
int fplus_analyze_opts(int64_t n, const int64_t *Ap, const int64_t *Ai, const fplus_options *opt,
                       fplus_symbolic **sym, char *err, size_t errlen);

/* FPLUS include/fplus.h:187-189: diag(Dr) A[p,:][:,q] diag(Dc) = L U with p, q, Dr, Dc in original coordinates.  The
 * factors stay in device memory; the host copies behind fplus_numeric_factors are made on first use. */
typedef struct fplus_numeric fplus_numeric;
int fplus_factor(const fplus_symbolic *sym, const int64_t *Ap, const int64_t *Ai, const void *Ax, int is_complex,
                 const fplus_options *opt, fplus_numeric **num, char *err, size_t errlen);

/* FPLUS include/fplus.h:193: solve in place for nrhs right-hand sides stored column-major in host memory b (leading
 * dimension ldb >= n): trans 0: A x = b, 1: A^T x = b, 2: A^H x = b. */
int fplus_solve(const fplus_numeric *num, void *b, int64_t nrhs, int64_t ldb, int trans, char *err, size_t errlen);

/* FPLUS include/fplus.h:195-200 */
const fplus_factors *fplus_numeric_factors(const fplus_numeric *num);
const int64_t *fplus_numeric_p(const fplus_numeric *num);
const int64_t *fplus_numeric_q(const fplus_numeric *num);
const double *fplus_numeric_Dr(const fplus_numeric *num);
const double *fplus_numeric_Dc(const fplus_numeric *num);
void fplus_numeric_free(fplus_numeric *num);

#ifdef __cplusplus
}
#endif
#endif /* FPLUS_H */
