// numeric.hpp -- the device state of the numeric phase and the launch sequences (numeric.cu).
#pragma once
#include <cstdint>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>
#include "internal.hpp"
#include "plan.hpp"

namespace fpl {

struct DevStatus;

// per-class device timing (fplus_b200_profile): 0 Schur GEMM into the CB, 1 pivot-block LU, 2 U12 (gather + TRSM),
// 3 assembly and extend-add
enum { PROF_SCHUR = 0, PROF_LU = 1, PROF_U12 = 2, PROF_ASM = 3, PROF_LU_TALL = 4, PROF_NCLASS = 5 };
struct ProfClass { double ms = 0, flops = 0, bytes = 0; long long count = 0; };
void prof_enable(int on);
ProfClass prof_read(int cls);
long long launch_count();
void add_launches(long long k);          // kernel launches made outside numeric.cu

inline double bitsd_h(unsigned long long b) { double d; std::memcpy(&d, &b, 8); return d; }

// device copies of a plan and of the symbolic object's permutation (read-only, shared by every factorization)
struct DevPlan {
    int device = -1;
    int64_t *cols = nullptr, *relcol = nullptr, *rowinit = nullptr, *asm_src = nullptr, *asm_dst = nullptr;
    int64_t *Bp = nullptr, *Bi = nullptr, *Bsrc = nullptr, *row_perm = nullptr, *col_perm = nullptr;
    // B's columns cut into segments of at most 1024 entries (column, first entry, end), for the column passes
    int64_t *seg = nullptr;
    int64_t nseg = 0;
    // the dense chain as the column-oriented backward sweep sees it: fronts [chain_begin, nfronts), chain_nb pivots each
    // (the last one at most), first column chain_f0, their U offsets; chain_begin < 0 when the fronts do not qualify
    int64_t chain_begin = -1, chain_nb = 0, chain_f0 = 0;
    int64_t *chain_uoff = nullptr;
    // the level-scheduled solve: every front's descriptor; per level (ascending height) the fronts the one-CTA kernels
    // take, as device lists (sv_rows: the L and L^T sweeps; sv_cols: the U and U^T sweeps) with host ranges and the
    // level's largest sizes, and the others as host lists; the lists of the children's contribution entries landing on
    // each plan row (rsp/rsi) and plan column (csp/csi); 0 .. max_nrows - 1
    SvFront *sv = nullptr;
    int *sv_rows = nullptr, *sv_cols = nullptr;
    std::vector<int64_t> sv_rows_ptr, sv_cols_ptr;
    std::vector<int64_t> sv_rows_maxnr, sv_rows_maxnp, sv_cols_maxnc, sv_cols_maxnp;
    std::vector<std::vector<int64_t>> big_rows, big_cols;
    // the trans-0 sweeps' larger fronts as device lists by level (brows: the L sweep; bcols: the U sweep below the dense
    // chain), with host ranges and the level's largest sizes; the partial sums a level's U sweep needs (per right-hand side)
    int *sv_brows = nullptr, *sv_bcols = nullptr;
    std::vector<int> sv_brows_host;
    std::vector<int64_t> sv_brows_ptr, sv_bcols_ptr;
    std::vector<int64_t> brows_maxnr, brows_maxnp, brows_maxm, bcols_maxnp, bcols_maxnch, bcols_maxchunk;
    int64_t part_need = 0;
    // the batched fronts of the factorization: every interior front whose whole subtree fits the one-CTA pivot-block LU
    // and the fused tail (at most 128 rows and 64 pivots).  They run first, level by level, three launches per level
    // (assembly, LU, tail), each front with its own working block (wofs, within the level's workspace) and its
    // contribution block in a separate arena (cbofs); the other fronts follow front by front.  Device descriptors and
    // children, lists by level with host ranges and the level's largest sizes and algorithmic counts; host flags and
    // contribution-block offsets
    FcFront *fc = nullptr;
    int64_t *children = nullptr;
    int *bs_list = nullptr;
    std::vector<int64_t> bs_ptr, bs_maxnr, bs_maxnp, bs_maxtiles, bs_wsz;
    std::vector<double> bs_lu_flops, bs_tail_flops, bs_asm_bytes, bs_lu_bytes, bs_tail_bytes;
    std::vector<char> is_bs;
    std::vector<int64_t> bs_cbofs;
    int64_t bs_ws = 0, bs_cb = 0;
    int64_t *rsp = nullptr, *rsi = nullptr, *csp = nullptr, *csi = nullptr, *iota = nullptr;
    int64_t vrow = 0, vcol = 0;              // the plan's total front rows, total front columns
    ~DevPlan();
};

// the device buffers of one factorization (and of its solves)
struct DevNum {
    int device = -1;
    int64_t n = 0, nnz = 0;
    int cplx = 0;
    int64_t vs = 8;
    cudaStream_t stream = nullptr;
    bool stream_owned = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t ev_begin = nullptr, ev_done = nullptr;   // the first operation of the factorization, the end of the last solve
    void *Ax = nullptr, *Bx = nullptr;
    double *Drp = nullptr, *Dcp = nullptr, *colmax = nullptr;
    void *Larena = nullptr, *Uarena = nullptr, *cbstack = nullptr, *work = nullptr;
    size_t cap_L = 0, cap_U = 0, cap_cb = 0, cap_work = 0, cap_rowid = 0, cap_ipiv = 0;
    int64_t *rowid = nullptr, *p_lu = nullptr, *pinv = nullptr;
    int *ipiv = nullptr, *perm = nullptr;
    size_t cap_perm = 0;
    int *permall = nullptr;        // every front's final row order (position -> initial local row), kept for the solves
    size_t cap_permall = 0;
    void *vbuf = nullptr;          // the level-scheduled solve's contribution vectors
    size_t cap_vb = 0;
    void *bsw = nullptr, *bscb = nullptr;   // the batched fronts' working blocks (one level) and contribution blocks
    size_t cap_bsw = 0, cap_bscb = 0;
    // the look-ahead over chain fronts: a second working block and row order, the critical stream and its events
    void *work2 = nullptr;
    int *perm2 = nullptr;
    size_t cap_work2 = 0, cap_perm2 = 0;
    cudaStream_t crit = nullptr;
    cudaEvent_t ev_lu = nullptr, ev_head = nullptr;
    DevStatus *st = nullptr;
    void *scratch = nullptr;
    void *scratch_norm = nullptr;
    size_t cap_norm = 0;
    // the precision form: the arithmetic of the large fronts' Schur updates (schur_tc.hpp), their operand workspace, and
    // the updates that ran on the tensor cores in the last factorization
    int prec = 0;
    void *coopbuf = nullptr;       // the multi-CTA pivot-block LU: the CTAs' posts, the ticket, the choices, U12, row scratch
    size_t cap_coop = 0;
    int lu_variant = 2;            // the small fronts' pivot-block LU (2: k_front_lu2, 1: k_front_lu5, 3: k_front_lu3); + 4: the tall
                                   // blocks by one CTA per 32-column panel instead of k_block_lu_mc; + 8: no batched
                                   // fronts (every front on its own); + 16: the small fronts' tails by forward
                                   // substitution (k_front_tail) instead of the block-inverse products (k_front_tail2);
                                   // + 32: the pipelined chain's contribution blocks through the stack and the
                                   // extend-add instead of straight into the parent's working block
    int capture = 0;               // the launches are being captured into a CUDA graph: no host copies, waits or decisions
    void *gm_buf = nullptr;        // GMRES-IR: the Krylov basis and its vectors
    size_t cap_gm = 0;
    void *tcws = nullptr;
    size_t cap_tcws = 0;
    long long tc_updates = 0;
    double tc_flops = 0;
    void *rbuf = nullptr, *sbuf = nullptr, *xbuf = nullptr, *part = nullptr;
    size_t cap_r = 0, cap_s = 0, cap_x = 0, cap_part = 0;
    int ruiz_iters = 0;
    // iterative refinement: B's rows (CSR; entry -> position in Ax), built on the first refined solve, and its buffers
    int64_t *rr_p = nullptr, *rr_l = nullptr, *rr_s = nullptr;
    void *ir_b = nullptr, *ir_x = nullptr, *ir_r = nullptr, *ir_d = nullptr;
    unsigned long long *ir_bits = nullptr;
    size_t cap_rrp = 0, cap_rrl = 0, cap_rrs = 0, cap_irb = 0, cap_irx = 0, cap_irr = 0, cap_ird = 0, cap_bits = 0;
    ~DevNum();
};

int dev_upload_plan(const fplus_symbolic *S, const FrontPlan &P, DevPlan &D, char *err, size_t errlen);
int dev_num_init(DevNum &N, int64_t n, int64_t nnz, int cplx, char *err, size_t errlen);
int dev_equilibrate(const DevPlan &D, DevNum &N, int equilibrate, int max_iter, double tol, char *err, size_t errlen);
// Ruiz equilibration of a caller's matrix (the public fplus_ruiz): its CSC pattern Cp, Ci and gather map src (CSC entry k
// holds input value src[k]); x_in host values in the caller's order, x_out the scaled values in CSC order (host)
int dev_ruiz_matrix(int64_t n, const std::vector<int64_t> &Cp, const std::vector<int64_t> &Ci, const std::vector<int64_t> &src,
                    const void *x_in, void *x_out, int cplx, int max_iter, double tol, double *Dr, double *Dc, int *iters,
                    cudaStream_t stream, char *err, size_t errlen);
int dev_factor_fronts(const FrontPlan &P, const DevPlan &D, DevNum &N, double pivot_rel, int64_t *border_front,
                      char *err, size_t errlen);
// raw: b and x are in the coordinates of the factors of the permuted matrix (trans 0: b in pivot order, x in column
// order; trans 1/2 the other way round), without the scalings (the low-level fplus_tri_solve_plan)
int dev_solve(const FrontPlan &P, const DevPlan &D, DevNum &N, void *x_dev, int64_t nrhs, int trans, char *err, size_t errlen,
              int raw = 0);
int dev_status(DevNum &N, int *code, int64_t *idx, char *err, size_t errlen);
// A solve with iterative refinement in FP64 (b in host memory, ld ldb, nrhs right-hand sides, solved in place): the
// solve, then corrections x += solve(b - op(A) x) with the residual formed on the device from the factorization's own
// copy of A, while a right-hand side's componentwise backward error is above tol and at least halves (at most max_iter
// corrections).  A correction that raised the error is undone.  berr[c] is the final backward error, iters[c] the
// corrections kept.
int dev_solve_refine(const FrontPlan &P, const DevPlan &D, DevNum &N, void *b, int64_t ldb, int64_t nrhs, int trans,
                     int max_iter, double tol, double *berr, int *iters, char *err, size_t errlen);
int dev_solve_noalloc(const FrontPlan &P, const DevPlan &D, DevNum &N, void *b_dev, int64_t ldb, int64_t nrhs, int trans,
                      cudaStream_t s, char *err, size_t errlen);
int dev_clear_status(DevNum &N, char *err, size_t errlen);
// after a captured factorization and solve: *rc = FPLUS_OK, FPLUS_ERR_SINGULAR (no admissible pivot, a zero line or a
// zero diagonal), FPLUS_ERR_GPU (a tensor-core wait ran out) or FPLUS_ERR_BADARG (a dense-row pivot where the plan had
// none, or the range guard); waits for the status word
int dev_status_rc(DevNum &N, int *rc, char *err, size_t errlen);
// ||L||_F and ||U||_F of the device factors (L with its unit diagonal), from the arenas
int dev_factor_norms(const FrontPlan &P, DevNum &N, double *lfro, double *ufro, char *err, size_t errlen);
int dev_check_finite(DevNum &N, char *err, size_t errlen);
int dev_ensure_x(DevNum &N, size_t bytes, char *err, size_t errlen);
int ensure_async(DevNum &N, void **p, size_t *cap, size_t bytes, char *err, size_t errlen);

}  // namespace fpl
