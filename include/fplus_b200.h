/* fplus_b200.h -- additions of the B200 build of FPLUS to the fplus.h interface (libfplus.so).
 *
 * fplus.h stays ABI-identical to FPLUS; what this build adds lives here, as new functions: device-resident inputs and
 * right-hand sides (no host copies in the way), the CUDA stream to run on, factorization statistics, and the pieces of
 * the symbolic analysis the tests inspect.  None of these has a counterpart in FPLUS unless its comment names one.
 */
#ifndef FPLUS_B200_H
#define FPLUS_B200_H

#include "fplus.h"

#ifdef __cplusplus
extern "C" {
#endif

/* A symbolic object for static orders the caller chose, for fplus_factor (whose factors stay in device memory).  FPLUS
 * takes such orders in fplus_factor_sn_perm only, which returns host factors; this is the same analysis for the
 * device-resident path (FPLUS's SparseLU without colamd factors in the identity order).  The trailing rows and columns
 * of A[row_perm, :][:, col_perm] with more than max(n / 2, 10) entries become its dense lines.  Free with
 * fplus_symbolic_free. */
int fplus_b200_symbolic_from_orders(int64_t n, const int64_t *Ap, const int64_t *Ai, const int64_t *row_perm,
                                    const int64_t *col_perm, fplus_symbolic **sym, char *err, size_t errlen);

/* Statistics of one factorization. */
typedef struct {
    int64_t n;
    int64_t nfronts;            /* fronts of the multifrontal structure used */
    int64_t f_dense;            /* first column of the dense chain (n when there is none) */
    int     attempts;           /* 1, or 2 when a dense row was chosen as a pivot before the chain and the LU was redone */
    int     ruiz_iters;         /* Ruiz iterations run */
    int64_t nnz_L, nnz_U;       /* stored entries (explicit zeros of the front structure included) */
    double  front_flops;        /* real floating-point operations of the front factorizations (complex: x4) */
    double  ms_equil;           /* device time: permutation + Ruiz */
    double  ms_fronts;          /* device time: the fronts (last attempt) */
    int64_t device_bytes;       /* device memory held by the factorization */
    int     precision;          /* FPLUS_B200_PREC_* of the Schur-complement updates (fplus_b200_factor_prec) */
    int     reserved;
    int64_t tc_updates;         /* Schur updates that ran on the tcgen05 tensor cores in reduced precision */
    double  tc_flops;           /* their real floating-point operations (complex: x4) */
} fplus_b200_info;

int fplus_b200_numeric_info(const fplus_numeric *num, fplus_b200_info *info);

/* Run this host thread's subsequent fplus_factor / fplus_solve / fplus_b200_* calls on the given CUDA stream
 * (a cudaStream_t; NULL: each factorization's own stream). */
void fplus_b200_use_stream(void *stream);

/* fplus_factor with the values already in device memory (Ax_dev: nnz doubles or nnz interleaved complex pairs, the
 * analysed pattern Ap / Ai on the host).  The values are checked for finiteness on the device. */
int fplus_b200_factor_dev(const fplus_symbolic *sym, const int64_t *Ap, const int64_t *Ai, const void *Ax_dev, int is_complex,
                          const fplus_options *opt, fplus_numeric **num, char *err, size_t errlen);

/* The precision form (no counterpart in FPLUS, which factors in FP64 only): fplus_factor (ax_on_device = 0) or
 * fplus_b200_factor_dev (1) with the Schur-complement updates of the large fronts (at least 128 x 256 contribution
 * blocks) on the tcgen05 tensor cores in reduced precision, FP32 accumulation:
 *   FPLUS_B200_PREC_FP32    operands split into two TF32 parts, three products: FP32-level accuracy
 *   FPLUS_B200_PREC_BF16X3  operands split into two BF16 parts, three products
 *   FPLUS_B200_PREC_TF32    one TF32 part, one product
 * FPLUS_B200_PREC_FP64 is fplus_factor itself.  Ruiz scaling, the pivot search and pivot-block factorization, the
 * triangular solves for U12 and every smaller update stay FP64, as do the stored factors.  The pivots are those of the
 * reduced-precision elimination (they can differ from FP64's where candidates are close); solve with
 * fplus_b200_solve_refine to bring the solution back to FP64 accuracy.  The operands of the reduced-precision products
 * must lie within FP32's range (Ruiz scaling, the default, ensures that for the matrices FPLUS targets). */
#define FPLUS_B200_PREC_FP64   0
#define FPLUS_B200_PREC_FP32   1
#define FPLUS_B200_PREC_BF16X3 2
#define FPLUS_B200_PREC_TF32   3
int fplus_b200_factor_prec(const fplus_symbolic *sym, const int64_t *Ap, const int64_t *Ai, const void *Ax, int is_complex,
                           const fplus_options *opt, int precision, int ax_on_device, fplus_numeric **num, char *err,
                           size_t errlen);

/* The precision form's Schur-complement update on device buffers, as the factorization runs it on a large front:
 * Cout[i, j] = Cin[rmap[i], j] - sum_k A[i, k] B[k, j] (rmap NULL: Cin[i, j]) for i < M, j < N, with A (M x K, lda), B
 * (K x N, ldb), Cin (ldci), Cout (ldco) FP64 column-major device arrays (is_complex: interleaved double pairs) and the
 * product in precision FPLUS_B200_PREC_FP32, _BF16X3 or _TF32 on the tcgen05 tensor cores.  M >= 128 and N >= 256
 * (N >= 128 complex).  Runs on `stream` (a cudaStream_t, NULL: the default stream) and waits for it; the workspace is
 * allocated and freed on the stream.  No counterpart in FPLUS. */
int fplus_b200_schur_update(int precision, int is_complex, int64_t M, int64_t N, int64_t K, const void *A, int64_t lda,
                            const void *B, int64_t ldb, const void *Cin, int64_t ldci, const int *rmap, void *Cout, int64_t ldco,
                            void *stream, char *err, size_t errlen);

/* fplus_solve with the right-hand sides in device memory (column-major, leading dimension ldb >= n), solved in place. */
int fplus_b200_solve_dev(const fplus_numeric *num, void *b_dev, int64_t nrhs, int64_t ldb, int trans, char *err, size_t errlen);

/* The fill-reducing column order of the interior pattern (the dense rows' entries and the dense columns, given by the
 * 0/1 masks, left out; empty columns last).  The order fplus_analyze uses before the column-etree postorder. */
int fplus_b200_interior_order(int64_t n, const int64_t *Ap, const int64_t *Ai, const unsigned char *tau_row_mask,
                              const unsigned char *tau_col_mask, int64_t *perm);

/* The multifrontal structure of an analysed pattern (host only, no GPU): with a dense chain from column `tail`
 * (-1: none).  plan_size returns the number of fronts and the total length of the column lists; plan_export fills
 * col_front[n] (the front of each column), parent[nf], col_ptr[nf + 1] / cols[] (each front's columns: pivot columns
 * first), nrows[nf] and nbord[nf] (its rows, the border rows among them). */
int fplus_b200_plan_size(const fplus_symbolic *sym, int64_t tail, int64_t *nfronts, int64_t *ncols_total, int64_t *f_dense);
int fplus_b200_plan_export(const fplus_symbolic *sym, int64_t tail, int64_t *col_front, int64_t *parent, int64_t *col_ptr,
                           int64_t *cols, int64_t *nrows, int64_t *nbord);

/* Batches of independent factorizations and solves.  No counterpart in FPLUS (one of the forms the B200 build adds): many
 * pencils of one problem, or many shifts A - sigma_k B refactored on one analysed pattern.  Matrix k is analysed by
 * syms[k] (the same object may appear several times), given by Ap[k], Ai[k], Ax[k] (host memory; all real or all
 * complex); the factorizations run concurrently on `nworkers` host threads (<= 0: 8), each numeric object on its own
 * CUDA stream, so that the GPU overlaps them.  nums[k] receives the k-th numeric object (NULL if it failed) and rcs[k]
 * (when rcs is not NULL) its return code; the function returns FPLUS_OK, or the first failing code with its message.
 * The results are those of fplus_factor / fplus_solve called one by one.  solve_batch solves nums[k] x = b[k] in place
 * (host buffers, nrhs[k] right-hand sides, leading dimension ldb[k]). */
int fplus_b200_factor_batch(int64_t count, const fplus_symbolic *const *syms, const int64_t *const *Ap, const int64_t *const *Ai,
                            const void *const *Ax, int is_complex, const fplus_options *opt, int nworkers, fplus_numeric **nums,
                            int *rcs, char *err, size_t errlen);
int fplus_b200_solve_batch(int64_t count, fplus_numeric *const *nums, void *const *b, const int64_t *nrhs, const int64_t *ldb,
                           int trans, int nworkers, int *rcs, char *err, size_t errlen);

/* The Frobenius norms of the factors, L (unit diagonal included) and U, computed on the GPU from the device factors
 * (the sums are scaled by each factor's largest modulus, so they neither overflow nor underflow).  No counterpart in
 * FPLUS; it lets a caller check factors too large to read back to the host (for instance against a stored oracle). */
int fplus_b200_factor_norms(const fplus_numeric *num, double *L_fro, double *U_fro, char *err, size_t errlen);

/* The batch form as one CUDA graph (no counterpart in FPLUS).  fplus_b200_graph_create captures, for every matrix k,
 * the refactorization of new values on its pattern (the permutation, Ruiz, the fronts) and the solve of nrhs[k]
 * right-hand sides with op = trans, each matrix on its own stream as an independent branch of one graph; nums[k] must
 * be a factorization (fplus_factor / _dev / _prec) on the current device, and stays owned by the caller (free the graph
 * first).  Capture needs no host decision: every Ruiz iteration is launched (they stop on the device once converged).
 * Between launches, write matrix k's values (nnz entries, in A's order, as for fplus_factor) into
 * fplus_b200_graph_values(g, k) and its right-hand sides (n x nrhs[k], column-major, ld n) into
 * fplus_b200_graph_rhs(g, k), both device memory; fplus_b200_graph_launch replays the graph on `stream` (NULL: the
 * graph's own stream); fplus_b200_graph_status waits for it and gives each matrix's code in rcs (FPLUS_OK,
 * FPLUS_ERR_SINGULAR, or FPLUS_ERR_BADARG for values that need the uncaptured path: a dense row chosen as a pivot where
 * the pattern's last factorization had none, or entries beyond 2^+-500 that the Ruiz range guard would rescale).  The
 * solutions are then in the right-hand-side buffers.  After a replay the numeric objects' host-side accessors
 * (fplus_numeric_p, _Dr, _factors, ...) still describe the factorization made before the capture. */
typedef struct fplus_b200_graph fplus_b200_graph;
int fplus_b200_graph_create(int64_t count, fplus_numeric *const *nums, const int64_t *nrhs, int trans, fplus_b200_graph **graph,
                            char *err, size_t errlen);
void *fplus_b200_graph_values(fplus_b200_graph *graph, int64_t k);
void *fplus_b200_graph_rhs(fplus_b200_graph *graph, int64_t k);
/* Host-memory conveniences: copy matrix k's values and / or right-hand sides (either may be NULL) into the graph's buffers
 * on the graph's stream (launch orders after them); copy matrix k's solutions out after fplus_b200_graph_status. */
int fplus_b200_graph_upload(fplus_b200_graph *graph, int64_t k, const void *Ax, const void *b, char *err, size_t errlen);
int fplus_b200_graph_download(fplus_b200_graph *graph, int64_t k, void *x, char *err, size_t errlen);
int fplus_b200_graph_launch(fplus_b200_graph *graph, void *stream, char *err, size_t errlen);
int fplus_b200_graph_status(fplus_b200_graph *graph, int *rcs, char *err, size_t errlen);
void fplus_b200_graph_free(fplus_b200_graph *graph);

/* The front-shape autotuner (no counterpart in FPLUS): factors the given values once per candidate shape of the
 * multifrontal structure (at most 128, 256 or 512 pivot columns per front, the panel width of the large fronts' Schur
 * updates; for a pattern with a dense chain also 32 or 64 pivots per chain front), then the best shape with the blocked
 * pivot-block LU, each timed on the device twice (permutation, Ruiz and the fronts), in the given precision
 * (FPLUS_B200_PREC_*), and keeps the fastest in sym for every later factorization on it.  The pivots do not depend on the shape.  best_width, best_nb, best_ms may be NULL. */
int fplus_b200_autotune(fplus_symbolic *sym, const int64_t *Ap, const int64_t *Ai, const void *Ax, int is_complex,
                        const fplus_options *opt, int precision, int64_t *best_width, int64_t *best_nb, int *best_lu,
                        double *best_ms, char *err, size_t errlen);

/* The front shape of every later factorization on sym, chosen by the caller instead of the autotuner: at most max_width
 * pivot columns per front (16 .. 4096), nb_chain pivots per dense-chain front (8 .. 64), and the pivot-block LU of the
 * small fronts (2: the block in shared memory, one barrier per pivot step, the default; 1: 8-column panels with the
 * later columns' rank-8 updates on the FP64 tensor cores; 3: blocked 8-column panels in FP64 lanes), plus 4 to pivot the pivot blocks too large for one CTA by one CTA per 32-column panel
 * instead of all SMs in one launch, plus 8 to factor every front on its own instead of the small fronts at the bottom of
 * the tree level by level (variant 3 also turns that off), plus 16 to form the small fronts' U12 and contribution blocks
 * by 16-row forward-substitution steps instead of products with the inverted diagonal blocks, plus 32 to pass the
 * pipelined fronts' contribution blocks through the stack instead of writing them into the parent's working block.  The
 * pivots do not depend on these.  No counterpart in FPLUS. */
int fplus_b200_set_front_shape(fplus_symbolic *sym, int64_t max_width, int64_t nb_chain, int lu_variant);

/* The device time of a batch: from the earliest start of the factorizations nums[0 .. count) (their first operation) to
 * the latest end of their last solves, from CUDA events on their own streams (no host timing).  No counterpart in FPLUS. */
int fplus_b200_batch_span_ms(int64_t count, fplus_numeric *const *nums, double *ms, char *err, size_t errlen);

/* fplus_b200_solve_dev for callers that cannot allocate device memory.  No counterpart in the reference (FPLUS has no GPU
 * solve).  Some callers may not call cudaMalloc at solve time: code running inside another runtime that owns the device
 * memory (a framework's custom operator given only its input and output buffers), latency-critical loops in which an
 * allocation's implicit device synchronization is not acceptable, and processes run under a fixed device-memory budget.
 * This entry point allocates nothing: it solves in place on b_dev (nrhs right-hand sides, column-major, leading
 * dimension ldb >= n), m = min(nrhs, 32) of them per pass, with its scratch vectors taken from one fixed array of
 * 16 MiB that the library declares in device memory; every GPU that loads the library holds that array until the
 * process exits.  One pass needs two n x m vectors plus the partial sums of the widest U12 product (a few npiv x m),
 * each rounded up to 256 bytes: about n <= 32,000 real or 16,000 complex at m = 32, proportionally more with fewer
 * right-hand sides.  A call that needs more than 16 MiB is rejected, before any work, with FPLUS_ERR_BADARG and a
 * message giving the size needed.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress): make that first call before any stream capture.  The array is shared by every call on the
 * device and keeps the last call's contents (every scratch value is written before it is read); calls that overlap on
 * the GPU (from other streams or host threads) race on it: serialize them.  It runs the unfused sweep kernels, whose
 * scratch is smallest, so its solutions agree with fplus_b200_solve_dev's to rounding, not bit for bit. */
int fplus_b200_solve_dev_noalloc(const fplus_numeric *num, void *b_dev, int64_t nrhs, int64_t ldb, int trans, char *err, size_t errlen);

/* fplus_solve with iterative refinement in FP64.  No counterpart in FPLUS: the refinement driver of the precision form.
 * It solves in place on b (host memory, nrhs right-hand sides, column-major, leading dimension ldb >= n), then corrects
 * x += solve(b - op(A) x) while a right-hand side's componentwise backward error max_i |r_i| / (|op(A)| |x| + |b|)_i is
 * above tol and at least halves from one correction to the next, at most max_iter times (LAPACK's xGERFS rule).  The
 * residual is formed on the GPU in FP64 from the factorization's own device copy of A, with a fixed summation order.
 * A right-hand side whose refinement stalls above tol (a factorization from fplus_b200_factor_prec on an ill-conditioned
 * matrix) continues with GMRES-IR: restarted GMRES (30 vectors, classical Gram-Schmidt applied twice, all in FP64) on
 * the correction equation preconditioned by the factorization, M^-1 op(A) d = M^-1 r, until tol is met, a cycle does
 * not lower the error, or max(max_iter, 62) applications of the factors in all.  berr[k] receives the final backward
 * error and iters[k] the applications of the factors after the first solve for right-hand side k (either may be NULL).
 * max_iter 0 gives fplus_solve's result with its backward error. */
int fplus_b200_solve_refine(const fplus_numeric *num, void *b, int64_t nrhs, int64_t ldb, int trans, int max_iter, double tol,
                            double *berr, int *iters, char *err, size_t errlen);

/* Kernel launches made by this library since it was loaded (all threads). */
long long fplus_b200_launch_count(void);

/* Device timing of the factorization's kernels by class, for measurement: when on, every launch of a class is bracketed
 * by CUDA events (a small perturbation; off by default).  Turning it on clears the totals.  Classes: 0 the Schur-
 * complement GEMM into the contribution block, 1 the pivot-block LU of the fronts one CTA holds, 2 U12 (gather + TRSM),
 * 3 assembly and extend-add, 4 the pivot-block LU of the taller fronts (all SMs in one launch).  profile_read returns the class's total device milliseconds, launches, and the algorithmic flops and bytes of those
 * launches. */
void fplus_b200_profile(int on);
int fplus_b200_profile_read(int cls, double *ms, long long *count, double *flops, double *bytes);

#ifdef __cplusplus
}
#endif
#endif /* FPLUS_B200_H */
