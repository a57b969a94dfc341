// api.cpp -- the fplus.h entry points of the numeric phase (FPLUS src/numeric.c, src/pipeline.c:84-127) and the
// fplus_b200.h additions.  The numeric work runs on the GPU (numeric.cu); this file validates, composes the orders and
// scalings (FPLUS src/numeric.c:71-77), moves data, and materializes host copies of the factors on request.
#include "internal.hpp"
#include "numeric.hpp"
#include "fplus_b200.h"
#include <algorithm>
#include <cstring>
#include <new>
#include <thread>
#include <string>
#include <functional>
#include <atomic>
#include <memory>
#include <vector>
#include "trisolve.hpp"
#include "schur_tc.hpp"

using namespace fpl;

static thread_local cudaStream_t tl_stream = nullptr;

extern "C" void fplus_b200_use_stream(void *stream) { tl_stream = (cudaStream_t)stream; }

struct fplus_numeric {
    int64_t n = 0;
    int is_complex = 0;
    std::shared_ptr<FrontPlan> plan;
    std::shared_ptr<DevPlan> dplan;
    std::unique_ptr<DevNum> dev;
    std::vector<int64_t> p, q, p_lu;
    std::vector<double> Dr, Dc, Drp, Dcp;
    fplus_b200_info info{};
    int equilibrate = 1, ruiz_max_iter = 20;   // the options the factorization ran with (a captured refactorization reuses them)
    double ruiz_tol = 1e-2, pivot_rel = 0.0;
    mutable std::mutex mu;               // solves and the lazy host factors share the device buffers
    mutable bool have_host = false;
    mutable fplus_factors f{};
};

#define CKH(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) { errf(err, errlen, "CUDA: %s", cudaGetErrorString(e_)); return FPLUS_ERR_GPU; } } while (0)

// the plan for the symbolic object's current dense-chain hint, and its device copy (built on first use)
static int get_plan(const fplus_symbolic *sym, int64_t tail, std::shared_ptr<FrontPlan> *plan, std::shared_ptr<DevPlan> *dplan,
                    char *err, size_t errlen)
{
    std::lock_guard<std::mutex> lk(sym->mu);
    int dev = 0;
    CKH(cudaGetDevice(&dev));
    if (tail < sym->tail_hint || sym->tail_hint < 0) { if (tail >= 0) sym->tail_hint = tail; }
    const int64_t want = sym->tail_hint;
    if (!sym->plan || sym->plan->f_dense != (want >= 0 && want < sym->n - sym->n_tau_cols ? want : sym->n - sym->n_tau_cols) ||
        sym->plan->max_width != sym->max_width || sym->plan->nb_chain != sym->nb_chain) {
        auto P = std::make_shared<FrontPlan>();
        fplus_symbolic_view v{sym->n, sym->n_tau_rows, sym->n_tau_cols, sym->Bp.data(), sym->Bi.data()};
        if (build_plan(v, want, sym->nb_chain, sym->max_width, *P)) { errf(err, errlen, "out of memory (symbolic structure)"); return FPLUS_ERR_NOMEM; }
        sym->plan = P;
        sym->dplan.reset();
    }
    if (!sym->dplan || sym->dplan->device != dev) {
        auto D = std::make_shared<DevPlan>();
        int rc = dev_upload_plan(sym, *sym->plan, *D, err, errlen);
        if (rc) return rc;
        sym->dplan = D;
    }
    *plan = sym->plan;
    *dplan = sym->dplan;
    return FPLUS_OK;
}

static int factor_common(const fplus_symbolic *sym, const int64_t *Ap, const int64_t *Ai, const void *Ax, int ax_on_device,
                         int is_complex, const fplus_options *opt, fplus_numeric **out, char *err, size_t errlen,
                         int prec = FPLUS_B200_PREC_FP64)
{
    if (!out) { errf(err, errlen, "num is NULL"); return FPLUS_ERR_BADARG; }
    *out = nullptr;
    if (prec < FPLUS_B200_PREC_FP64 || prec > FPLUS_B200_PREC_TF32) { errf(err, errlen, "unknown precision %d", prec); return FPLUS_ERR_BADARG; }
    if (!sym) { errf(err, errlen, "sym is NULL"); return FPLUS_ERR_BADARG; }
    fplus_options d;
    if (!opt) { fplus_default_options(&d); opt = &d; }
    // options (FPLUS src/numeric.c:51-57)
    if (opt->pivot_strategy != FPLUS_PIVOT_PARTIAL && opt->pivot_strategy != FPLUS_PIVOT_ROOK && opt->pivot_strategy != FPLUS_PIVOT_FULL) {
        errf(err, errlen, "pivot_strategy must be FPLUS_PIVOT_PARTIAL, _ROOK or _FULL (got %d)", opt->pivot_strategy);
        return FPLUS_ERR_BADARG;
    }
    if (!(opt->drop_tol >= 0.0)) { errf(err, errlen, "drop_tol must be >= 0 (got %g)", opt->drop_tol); return FPLUS_ERR_BADARG; }
    if (opt->pivot_strategy != FPLUS_PIVOT_PARTIAL || opt->drop_tol != 0.0) {
        errf(err, errlen, "this build factors with partial pivoting and drop_tol 0 only (rook / full pivoting and incomplete LU "
                          "are not built)");
        return FPLUS_ERR_BADARG;
    }
    if (!(opt->pivot_rel >= 0.0)) { errf(err, errlen, "pivot_rel must be >= 0"); return FPLUS_ERR_BADARG; }
    const int64_t n = sym->n;
    // the analysed pattern (FPLUS src/pipeline.c:91-99, 118-123)
    if (!Ap || (n > 0 && !Ai && Ap[n] > 0)) { errf(err, errlen, "NULL index array"); return FPLUS_ERR_BADARG; }
    if (Ap[n] != sym->nnz) {
        errf(err, errlen, "the matrix has %ld nonzeros, the symbolic analysis %ld", (long)Ap[n], (long)sym->nnz);
        return FPLUS_ERR_BADARG;
    }
    int rc = FPLUS_OK;
    // The pattern must be the analysed one (which was checked canonical when analysed).  The column pointers are
    // compared here; the row indices below, on a host thread while the GPU permutes and equilibrates the values (which
    // it reads only through the analysed pattern's maps, so a different pattern cannot make it read out of bounds).
    if (std::memcmp(Ap, sym->Ap0.data(), (size_t)(n + 1) * sizeof(int64_t)) != 0) {
        rc = check_compressed(n, Ap, Ai, 1, err, errlen);
        if (rc) return rc;
        errf(err, errlen, "the pattern differs from the analysed one (column pointers)");
        return FPLUS_ERR_BADARG;
    }

    // the row indices: compared on another host thread while the values are checked, uploaded, permuted and
    // equilibrated; a difference takes precedence over any other error
    int prc = FPLUS_OK;
    char perr[256] = {0};
    std::thread checker([&]() {
        if (sym->nnz > 0 && std::memcmp(Ai, sym->Ai0.data(), (size_t)sym->nnz * sizeof(int64_t)) != 0) {
            prc = check_compressed(n, Ap, Ai, 1, perr, sizeof perr);
            if (prc == FPLUS_OK) { errf(perr, sizeof perr, "the pattern differs from the analysed one (row indices)"); prc = FPLUS_ERR_BADARG; }
        }
    });
    auto body = [&]() -> int {
    int rc = FPLUS_OK;
    if (!ax_on_device) { rc = check_finite(Ap[n], Ax, is_complex, err, errlen); if (rc) return rc; }
    fplus_numeric *num = new (std::nothrow) fplus_numeric;
    if (!num) { errf(err, errlen, "out of memory"); return FPLUS_ERR_NOMEM; }
    std::unique_ptr<fplus_numeric> guard(num);
    try {
        num->n = n; num->is_complex = is_complex ? 1 : 0;
        num->equilibrate = opt->equilibrate; num->ruiz_max_iter = opt->ruiz_max_iter; num->ruiz_tol = opt->ruiz_tol;
        num->pivot_rel = opt->pivot_rel;
        num->dev.reset(new DevNum);
        DevNum &N = *num->dev;
        if (tl_stream) N.stream = tl_stream;
        N.prec = prec;
        {
            std::lock_guard<std::mutex> lk(sym->mu);
            N.lu_variant = sym->lu_variant;
        }
        rc = dev_num_init(N, n, sym->nnz, num->is_complex, err, errlen);
        if (rc) return rc;
        CKH(cudaEventRecord(N.ev_begin, N.stream));
        const size_t bytes = (size_t)sym->nnz * (size_t)N.vs;
        if (bytes) CKH(cudaMemcpyAsync(N.Ax, Ax, bytes, ax_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, N.stream));
        std::shared_ptr<FrontPlan> P;
        std::shared_ptr<DevPlan> D;
        rc = get_plan(sym, -1, &P, &D, err, errlen);
        if (rc) return rc;
        if (ax_on_device) { rc = dev_check_finite(N, err, errlen); if (rc) return rc; }
        CKH(cudaEventRecord(N.ev0, N.stream));
        rc = dev_equilibrate(*D, N, opt->equilibrate, opt->ruiz_max_iter, opt->ruiz_tol, err, errlen);
        if (rc) return rc;
        checker.join();
        if (prc) return prc;
        CKH(cudaEventRecord(N.ev1, N.stream));
        CKH(cudaEventSynchronize(N.ev1));
        float ms = 0;
        CKH(cudaEventElapsedTime(&ms, N.ev0, N.ev1));
        num->info.ms_equil = ms;
        int attempts = 0;
        for (;;) {
            attempts++;
            int64_t border = -1;
            CKH(cudaEventRecord(N.ev0, N.stream));
            rc = dev_factor_fronts(*P, *D, N, opt->pivot_rel, &border, err, errlen);
            if (rc) return rc;
            CKH(cudaEventRecord(N.ev1, N.stream));
            CKH(cudaEventSynchronize(N.ev1));
            CKH(cudaEventElapsedTime(&ms, N.ev0, N.ev1));
            num->info.ms_fronts = ms;
            if (border < 0) break;
            if (attempts >= 3) { errf(err, errlen, "dense-row pivot reported again after the restart (front %ld)", (long)border); return FPLUS_ERR_INTERNAL; }
            // a dense row was chosen as pivot in front `border`: the dense chain starts at that front
            rc = get_plan(sym, P->fronts[border].f, &P, &D, err, errlen);
            if (rc) return rc;
        }
        num->plan = P;
        num->dplan = D;
        // compose the orders and scalings (FPLUS src/numeric.c:71-77)
        num->p_lu.resize((size_t)n); num->Drp.resize((size_t)n); num->Dcp.resize((size_t)n);
        if (n > 0) {
            CKH(cudaMemcpyAsync(num->p_lu.data(), N.p_lu, (size_t)n * 8, cudaMemcpyDeviceToHost, N.stream));
            CKH(cudaMemcpyAsync(num->Drp.data(), N.Drp, (size_t)n * 8, cudaMemcpyDeviceToHost, N.stream));
            CKH(cudaMemcpyAsync(num->Dcp.data(), N.Dcp, (size_t)n * 8, cudaMemcpyDeviceToHost, N.stream));
            CKH(cudaStreamSynchronize(N.stream));
        }
        num->p.resize((size_t)n); num->q.resize((size_t)n); num->Dr.resize((size_t)n); num->Dc.resize((size_t)n);
        const int64_t *rp = sym->row_perm.data(), *cp = sym->col_perm.data();
        for (int64_t k = 0; k < n; k++) {
            num->p[k] = rp[num->p_lu[k]];
            num->q[k] = cp[k];
            num->Dr[rp[k]] = num->Drp[k];
            num->Dc[cp[k]] = num->Dcp[k];
        }
        fplus_b200_info &I = num->info;
        I.n = n; I.nfronts = (int64_t)P->fronts.size(); I.f_dense = P->f_dense; I.attempts = attempts;
        I.ruiz_iters = N.ruiz_iters;
        int64_t nl = 0, nu = 0;
        for (auto &F : P->fronts) {
            for (int64_t i = 0; i < F.npiv && i < F.nrows; i++) { nl += F.nrows - i; nu += F.ncols - i; }
        }
        I.nnz_L = nl; I.nnz_U = nu;
        I.front_flops = 2.0 * P->flops_real * (is_complex ? 4.0 : 1.0);
        I.device_bytes = (int64_t)(N.cap_L + N.cap_U + N.cap_cb + N.cap_work + N.cap_work2 + N.cap_tcws + 2 * bytes);
        I.precision = prec;
        I.tc_updates = N.tc_updates;
        I.tc_flops = N.tc_flops;
    } catch (const std::bad_alloc &) {
        errf(err, errlen, "out of memory");
        return FPLUS_ERR_NOMEM;
    }
    *out = guard.release();
    return FPLUS_OK;
    };
    rc = body();
    if (checker.joinable()) checker.join();
    if (prc) {
        if (*out) { delete *out; *out = nullptr; }
        errf(err, errlen, "%s", perr);
        return prc;
    }
    return rc;
}

extern "C" int fplus_factor(const fplus_symbolic *sym, const int64_t *Ap, const int64_t *Ai, const void *Ax, int is_complex,
                            const fplus_options *opt, fplus_numeric **num, char *err, size_t errlen)
{
    return factor_common(sym, Ap, Ai, Ax, 0, is_complex, opt, num, err, errlen);
}

extern "C" int fplus_b200_factor_dev(const fplus_symbolic *sym, const int64_t *Ap, const int64_t *Ai, const void *Ax_dev,
                                     int is_complex, const fplus_options *opt, fplus_numeric **num, char *err, size_t errlen)
{
    return factor_common(sym, Ap, Ai, Ax_dev, 1, is_complex, opt, num, err, errlen);
}

extern "C" int fplus_b200_factor_prec(const fplus_symbolic *sym, const int64_t *Ap, const int64_t *Ai, const void *Ax,
                                      int is_complex, const fplus_options *opt, int precision, int ax_on_device,
                                      fplus_numeric **num, char *err, size_t errlen)
{
    return factor_common(sym, Ap, Ai, Ax, ax_on_device ? 1 : 0, is_complex, opt, num, err, errlen, precision);
}

extern "C" int fplus_b200_schur_update(int precision, int is_complex, int64_t M, int64_t N, int64_t K, const void *A, int64_t lda,
                                       const void *B, int64_t ldb, const void *Cin, int64_t ldci, const int *rmap, void *Cout,
                                       int64_t ldco, void *stream, char *err, size_t errlen)
{
    if (precision < FPLUS_B200_PREC_FP32 || precision > FPLUS_B200_PREC_TF32) { errf(err, errlen, "precision must be FP32, BF16X3 or TF32"); return FPLUS_ERR_BADARG; }
    if (!A || !B || !Cin || !Cout || lda < M || ldb < K || ldci < 1 || ldco < M || !schur_tc_supported(M, N, K, is_complex ? 1 : 0)) {
        errf(err, errlen, "fplus_b200_schur_update: bad arguments or a shape below one 128 x 256 tile");
        return FPLUS_ERR_BADARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const size_t wsb = schur_tc_workspace(precision, M, N, K, is_complex ? 1 : 0);
    void *ws = nullptr;
    unsigned *derr = nullptr;
    CKH(cudaMallocAsync(&ws, wsb, s));
    cudaError_t e = cudaMallocAsync((void **)&derr, sizeof(unsigned), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(derr, 0, sizeof(unsigned), s);
    int rc = FPLUS_OK;
    if (e != cudaSuccess) { errf(err, errlen, "CUDA: %s", cudaGetErrorString(e)); rc = FPLUS_ERR_GPU; }
    else {
        const int trc = schur_tc(precision, is_complex ? 1 : 0, M, N, K, (const double *)A, lda, (const double *)B, ldb,
                                 (const double *)Cin, ldci, rmap, (double *)Cout, ldco, ws, wsb, derr, s);
        unsigned herr = 0;
        if (trc != 0) { errf(err, errlen, "fplus_b200_schur_update: launch failed (%d)", trc); rc = FPLUS_ERR_GPU; }
        else {
            add_launches(3);
            e = cudaMemcpyAsync(&herr, derr, sizeof herr, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) { errf(err, errlen, "CUDA: %s", cudaGetErrorString(e)); rc = FPLUS_ERR_GPU; }
            else if (herr) { errf(err, errlen, "fplus_b200_schur_update: a wait timed out (status %u)", herr); rc = FPLUS_ERR_GPU; }
        }
    }
    cudaFreeAsync(ws, s);
    if (derr) cudaFreeAsync(derr, s);
    cudaStreamSynchronize(s);
    return rc;
}

// the front shape chosen by the caller (what fplus_b200_autotune sets), for every later factorization on sym
extern "C" int fplus_b200_set_front_shape(fplus_symbolic *sym, int64_t max_width, int64_t nb_chain, int lu_variant)
{
    if (!sym || max_width < 16 || max_width > 4096 || nb_chain < 8 || nb_chain > 64 ||
        (lu_variant & 3) == 0 || (lu_variant & ~63) != 0)
        return FPLUS_ERR_BADARG;
    std::lock_guard<std::mutex> lk(sym->mu);
    sym->max_width = max_width;
    sym->nb_chain = nb_chain;
    sym->lu_variant = lu_variant;
    return FPLUS_OK;
}

// The front-shape autotuner: factor the given values with each candidate shape (at most 128, 256 or 512 pivot columns per
// front; for a pattern with a dense chain also 32 or 64 pivots per chain front), timed on the device (permutation,
// Ruiz and the fronts, CUDA events), and keep the fastest in the symbolic object for every later factorization of the
// pattern.  Each candidate is timed twice, the better time kept.  The pivots do not depend on the shape.
extern "C" int fplus_b200_autotune(fplus_symbolic *sym, const int64_t *Ap, const int64_t *Ai, const void *Ax, int is_complex,
                                   const fplus_options *opt, int precision, int64_t *best_width, int64_t *best_nb,
                                   int *best_lu, double *best_ms, char *err, size_t errlen)
{
    if (!sym) { errf(err, errlen, "sym is NULL"); return FPLUS_ERR_BADARG; }
    const int64_t widths[3] = {128, 256, 512}, nbs[2] = {32, 64};
    const int64_t w0 = sym->max_width, b0 = sym->nb_chain;
    const int l0 = sym->lu_variant;
    int64_t bw = w0, bb = b0;
    int bl = l0;
    double bms = -1.0;
    bool chain = false;
    // the front shapes with the shared-memory pivot-block LU, then the best shape with the panel LU (tensor-core updates)
    for (int ci = 0; ci < 7; ci++) {
        const int wi = ci < 6 ? ci / 2 : -1, bi = ci < 6 ? ci % 2 : -1;
        if (ci < 6 && bi == 0 && !chain && wi > 0) continue;      // the chain size matters only with a dense chain
        {
            std::lock_guard<std::mutex> lk(sym->mu);
            sym->max_width = ci < 6 ? widths[wi] : bw;
            sym->nb_chain = ci < 6 ? nbs[bi] : bb;
            sym->lu_variant = ci < 6 ? 2 : 1;
        }
        {
            double t = -1.0;
            for (int rep = 0; rep < 2; rep++) {
                fplus_numeric *num = nullptr;
                const int rc = factor_common(sym, Ap, Ai, Ax, 0, is_complex, opt, &num, err, errlen, precision);
                if (rc != FPLUS_OK) {
                    std::lock_guard<std::mutex> lk(sym->mu);
                    sym->max_width = w0; sym->nb_chain = b0; sym->lu_variant = l0;
                    return rc;
                }
                const double ms = num->info.ms_equil + num->info.ms_fronts;
                chain = chain || num->info.f_dense < num->n;
                fplus_numeric_free(num);
                if (t < 0 || ms < t) t = ms;
            }
            if (bms < 0 || t < bms) {
                bms = t;
                if (ci < 6) { bw = widths[wi]; bb = nbs[bi]; bl = 2; } else bl = 1;
            }
        }
    }
    {
        std::lock_guard<std::mutex> lk(sym->mu);
        sym->max_width = bw;
        sym->nb_chain = bb;
        sym->lu_variant = bl;
    }
    if (best_width) *best_width = bw;
    if (best_nb) *best_nb = bb;
    if (best_lu) *best_lu = bl;
    if (best_ms) *best_ms = bms;
    return FPLUS_OK;
}

#define SOLVE_GROUP 32

static int solve_common(const fplus_numeric *num, void *b, int64_t nrhs, int64_t ldb, int trans, int on_device, char *err,
                        size_t errlen, int raw = 0)
{
    if (!num) { errf(err, errlen, "fplus_solve: num is NULL"); return FPLUS_ERR_BADARG; }
    const int64_t n = num->n;
    if (trans < 0 || trans > 2 || nrhs < 0 || ldb < n) { errf(err, errlen, "fplus_solve: bad trans, nrhs or ldb"); return FPLUS_ERR_BADARG; }
    if (nrhs == 0 || n == 0) return FPLUS_OK;
    if (!b) { errf(err, errlen, "fplus_solve: b is NULL"); return FPLUS_ERR_BADARG; }
    std::lock_guard<std::mutex> lk(num->mu);
    DevNum &N = *num->dev;
    CKH(cudaSetDevice(N.device));
    cudaStream_t saved = N.stream;
    if (tl_stream) N.stream = tl_stream;
    const size_t vs = (size_t)N.vs;
    const int64_t g = nrhs < SOLVE_GROUP ? nrhs : SOLVE_GROUP;
    int rc = FPLUS_OK;
    if ((rc = dev_ensure_x(N, (size_t)n * (size_t)g * vs, err, errlen))) { N.stream = saved; return rc; }
    dev_clear_status(N, err, errlen);
    for (int64_t r0 = 0; r0 < nrhs && rc == FPLUS_OK; r0 += g) {
        const int64_t m = nrhs - r0 < g ? nrhs - r0 : g;
        char *bb = (char *)b + (size_t)r0 * (size_t)ldb * vs;
        cudaError_t e = cudaMemcpy2DAsync(N.xbuf, (size_t)n * vs, bb, (size_t)ldb * vs, (size_t)n * vs, (size_t)m,
                                          on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, N.stream);
        if (e != cudaSuccess) { errf(err, errlen, "CUDA: %s", cudaGetErrorString(e)); rc = FPLUS_ERR_GPU; break; }
        rc = dev_solve(*num->plan, *num->dplan, N, N.xbuf, m, trans, err, errlen, raw);
        if (rc) break;
        e = cudaMemcpy2DAsync(bb, (size_t)ldb * vs, N.xbuf, (size_t)n * vs, (size_t)n * vs, (size_t)m,
                              on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, N.stream);
        if (e != cudaSuccess) { errf(err, errlen, "CUDA: %s", cudaGetErrorString(e)); rc = FPLUS_ERR_GPU; break; }
    }
    if (rc == FPLUS_OK) {
        cudaEventRecord(N.ev_done, N.stream);
        int code = 0; int64_t idx = 0;
        rc = dev_status(N, &code, &idx, err, errlen);
        if (rc == FPLUS_OK && code != 0) { errf(err, errlen, "fplus_solve: zero or missing diagonal in U"); rc = FPLUS_ERR_SINGULAR; }
    }
    N.stream = saved;
    return rc;
}

// ---------------------------------------------------------------------------------------------------------------------
// The batch form as one CUDA graph: the refactorization (new values on the same patterns) and solve of many matrices,
// captured once from their own launch sequences and replayed.  Each matrix's work is captured on its own stream, forked
// from and joined to a capture stream, so the graph's branches are independent and run concurrently.
struct fplus_b200_graph {
    std::vector<fplus_numeric *> nums;
    std::vector<int64_t> nrhs;
    std::vector<void *> rhs;                 // n x nrhs[k] device buffers
    int trans = 0;
    int device = 0;
    cudaStream_t s0 = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> joins;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t launched = nullptr;
    ~fplus_b200_graph()
    {
        cudaSetDevice(device);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (auto e : joins) if (e) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        for (void *p : rhs) if (p) cudaFree(p);
        if (s0) cudaStreamDestroy(s0);
    }
};

extern "C" int fplus_b200_graph_create(int64_t count, fplus_numeric *const *nums, const int64_t *nrhs, int trans,
                                       fplus_b200_graph **out, char *err, size_t errlen)
{
    if (!out) { errf(err, errlen, "graph is NULL"); return FPLUS_ERR_BADARG; }
    *out = nullptr;
    if (count < 1 || !nums || !nrhs || trans < 0 || trans > 2) { errf(err, errlen, "bad arguments"); return FPLUS_ERR_BADARG; }
    std::unique_ptr<fplus_b200_graph> g(new (std::nothrow) fplus_b200_graph);
    if (!g) { errf(err, errlen, "out of memory"); return FPLUS_ERR_NOMEM; }
    g->trans = trans;
    for (int64_t k = 0; k < count; k++) {
        if (!nums[k] || !nums[k]->dev || nrhs[k] < 1) { errf(err, errlen, "matrix %ld: no factorization or nrhs < 1", (long)k); return FPLUS_ERR_BADARG; }
        if (k > 0 && nums[k]->dev->device != nums[0]->dev->device) { errf(err, errlen, "the matrices are on different devices"); return FPLUS_ERR_BADARG; }
        for (int64_t j = 0; j < k; j++) if (nums[j] == nums[k]) { errf(err, errlen, "matrix %ld appears twice", (long)k); return FPLUS_ERR_BADARG; }
    }
    g->device = nums[0]->dev->device;
    CKH(cudaSetDevice(g->device));
    CKH(cudaStreamCreateWithFlags(&g->s0, cudaStreamNonBlocking));
    CKH(cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming));
    int rc = FPLUS_OK;
    // every buffer sized beforehand: one uncaptured solve per matrix with its right-hand side count
    for (int64_t k = 0; k < count && rc == FPLUS_OK; k++) {
        fplus_numeric *num = nums[k];
        DevNum &N = *num->dev;
        g->nums.push_back(num);
        g->nrhs.push_back(nrhs[k]);
        void *b = nullptr;
        const size_t bytes = (size_t)num->n * (size_t)nrhs[k] * (size_t)N.vs;
        CKH(cudaMalloc(&b, bytes > 0 ? bytes : 16));
        g->rhs.push_back(b);
        CKH(cudaMemsetAsync(b, 0, bytes, N.stream));
        rc = dev_solve(*num->plan, *num->dplan, N, b, nrhs[k], trans, err, errlen);
        if (rc == FPLUS_OK) CKH(cudaStreamSynchronize(N.stream));
        cudaEvent_t e = nullptr;
        CKH(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        g->joins.push_back(e);
    }
    if (rc) return rc;
    CKH(cudaStreamBeginCapture(g->s0, cudaStreamCaptureModeThreadLocal));
    cudaError_t ce = cudaEventRecord(g->fork, g->s0);
    for (int64_t k = 0; k < count && rc == FPLUS_OK && ce == cudaSuccess; k++) {
        fplus_numeric *num = nums[k];
        DevNum &N = *num->dev;
        if ((ce = cudaStreamWaitEvent(N.stream, g->fork, 0)) != cudaSuccess) break;
        N.capture = 1;
        rc = dev_equilibrate(*num->dplan, N, num->equilibrate, num->ruiz_max_iter, num->ruiz_tol, err, errlen);
        int64_t border = -1;
        if (rc == FPLUS_OK) rc = dev_factor_fronts(*num->plan, *num->dplan, N, num->pivot_rel, &border, err, errlen);
        if (rc == FPLUS_OK) rc = dev_solve(*num->plan, *num->dplan, N, g->rhs[(size_t)k], nrhs[k], trans, err, errlen);
        N.capture = 0;
        if (rc == FPLUS_OK && (ce = cudaEventRecord(g->joins[(size_t)k], N.stream)) == cudaSuccess)
            ce = cudaStreamWaitEvent(g->s0, g->joins[(size_t)k], 0);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(g->s0, &graph);
    g->graph = graph;
    if (rc) return rc;
    if (ce != cudaSuccess || ee != cudaSuccess) {
        errf(err, errlen, "CUDA graph capture: %s", cudaGetErrorString(ce != cudaSuccess ? ce : ee));
        return FPLUS_ERR_GPU;
    }
    CKH(cudaGraphInstantiate(&g->exec, g->graph, 0));
    *out = g.release();
    return FPLUS_OK;
}

extern "C" void *fplus_b200_graph_values(fplus_b200_graph *g, int64_t k)
{
    return g && k >= 0 && k < (int64_t)g->nums.size() ? g->nums[(size_t)k]->dev->Ax : nullptr;
}

extern "C" void *fplus_b200_graph_rhs(fplus_b200_graph *g, int64_t k)
{
    return g && k >= 0 && k < (int64_t)g->rhs.size() ? g->rhs[(size_t)k] : nullptr;
}

extern "C" int fplus_b200_graph_upload(fplus_b200_graph *g, int64_t k, const void *Ax, const void *b, char *err, size_t errlen)
{
    if (!g || k < 0 || k >= (int64_t)g->nums.size()) { errf(err, errlen, "bad graph or index"); return FPLUS_ERR_BADARG; }
    CKH(cudaSetDevice(g->device));
    const fplus_numeric *num = g->nums[(size_t)k];
    const DevNum &N = *num->dev;
    if (Ax) CKH(cudaMemcpyAsync(N.Ax, Ax, (size_t)N.nnz * (size_t)N.vs, cudaMemcpyHostToDevice, g->s0));
    if (b) CKH(cudaMemcpyAsync(g->rhs[(size_t)k], b, (size_t)num->n * (size_t)g->nrhs[(size_t)k] * (size_t)N.vs,
                               cudaMemcpyHostToDevice, g->s0));
    return FPLUS_OK;
}

extern "C" int fplus_b200_graph_download(fplus_b200_graph *g, int64_t k, void *x, char *err, size_t errlen)
{
    if (!g || !x || k < 0 || k >= (int64_t)g->nums.size()) { errf(err, errlen, "bad graph, index or buffer"); return FPLUS_ERR_BADARG; }
    CKH(cudaSetDevice(g->device));
    const fplus_numeric *num = g->nums[(size_t)k];
    CKH(cudaMemcpyAsync(x, g->rhs[(size_t)k], (size_t)num->n * (size_t)g->nrhs[(size_t)k] * (size_t)num->dev->vs,
                        cudaMemcpyDeviceToHost, g->launched ? g->launched : g->s0));
    CKH(cudaStreamSynchronize(g->launched ? g->launched : g->s0));
    return FPLUS_OK;
}

extern "C" int fplus_b200_graph_launch(fplus_b200_graph *g, void *stream, char *err, size_t errlen)
{
    if (!g || !g->exec) { errf(err, errlen, "graph is NULL"); return FPLUS_ERR_BADARG; }
    CKH(cudaSetDevice(g->device));
    g->launched = stream ? (cudaStream_t)stream : g->s0;
    if (g->launched != g->s0) {           // after the uploads made on the graph's stream
        CKH(cudaEventRecord(g->fork, g->s0));
        CKH(cudaStreamWaitEvent(g->launched, g->fork, 0));
    }
    CKH(cudaGraphLaunch(g->exec, g->launched));
    return FPLUS_OK;
}

extern "C" int fplus_b200_graph_status(fplus_b200_graph *g, int *rcs, char *err, size_t errlen)
{
    if (!g) { errf(err, errlen, "graph is NULL"); return FPLUS_ERR_BADARG; }
    CKH(cudaSetDevice(g->device));
    CKH(cudaStreamSynchronize(g->launched ? g->launched : g->s0));
    int rc = FPLUS_OK;
    for (size_t k = 0; k < g->nums.size(); k++) {
        int r = FPLUS_OK;
        const int qrc = dev_status_rc(*g->nums[k]->dev, &r, err, errlen);
        if (qrc) return qrc;
        if (rcs) rcs[k] = r;
        if (rc == FPLUS_OK && r != FPLUS_OK) {
            rc = r;
            errf(err, errlen, "matrix %ld: %s", (long)k, r == FPLUS_ERR_SINGULAR ? "singular" :
                 r == FPLUS_ERR_GPU ? "a tensor-core update timed out" :
                 "needs the uncaptured path (a dense-row pivot at a new place, or values beyond the range guard)");
        }
    }
    return rc;
}

extern "C" void fplus_b200_graph_free(fplus_b200_graph *g) { delete g; }

// the device time from the earliest factorization start to the latest solve end over a batch (events on the jobs' own
// streams, read after they have completed)
extern "C" int fplus_b200_batch_span_ms(int64_t count, fplus_numeric *const *nums, double *ms, char *err, size_t errlen)
{
    if (!nums || !ms || count < 1) { errf(err, errlen, "bad arguments"); return FPLUS_ERR_BADARG; }
    cudaEvent_t ref = nullptr;
    double lo = 0, hi = 0;
    for (int64_t k = 0; k < count; k++) {
        if (!nums[k] || !nums[k]->dev) { errf(err, errlen, "matrix %ld: no factorization", (long)k); return FPLUS_ERR_BADARG; }
        DevNum &N = *nums[k]->dev;
        CKH(cudaEventSynchronize(N.ev_begin));
        CKH(cudaEventSynchronize(N.ev_done));
        if (!ref) ref = N.ev_begin;
        float a = 0, b = 0;
        CKH(cudaEventElapsedTime(&a, ref, N.ev_begin));
        CKH(cudaEventElapsedTime(&b, ref, N.ev_done));
        if (k == 0 || a < lo) lo = a;
        if (k == 0 || b > hi) hi = b;
    }
    *ms = hi - lo;
    return FPLUS_OK;
}

// ---------------------------------------------------------------------------------------------------------------------
// Batches: independent factorizations / solves run concurrently.  Each numeric object has its own CUDA stream (the
// worker threads leave fplus_b200_use_stream unset), so the pivot-block chains of different matrices, each on one SM,
// overlap on the GPU, as do their bulk kernels.  The work itself is the single-matrix path: the results are those of
// fplus_factor / fplus_solve called one by one.
// The workers take the jobs largest first (cost[k], when given: longest processing time first), so that the large
// matrices of an uneven batch start early and the small ones fill in around them.  The order changes no result.
static int run_batch(int64_t count, int nworkers, const std::function<int(int64_t, char *, size_t)> &job, int *rcs, char *err,
                     size_t errlen, const std::vector<double> *cost = nullptr)
{
    if (count < 0) { errf(err, errlen, "count must be >= 0"); return FPLUS_ERR_BADARG; }
    if (nworkers <= 0) nworkers = 8;
    if (nworkers > count) nworkers = (int)count;
    std::vector<int64_t> order((size_t)count);
    for (int64_t k = 0; k < count; k++) order[(size_t)k] = k;
    if (cost) std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return (*cost)[a] > (*cost)[b]; });
    std::atomic<int64_t> next{0};
    std::vector<int> rc_local((size_t)count, FPLUS_OK);
    std::vector<std::string> msg((size_t)count);
    auto worker = [&]() {
        char e[512];
        for (;;) {
            const int64_t t = next.fetch_add(1);
            if (t >= count) break;
            const int64_t k = order[(size_t)t];
            e[0] = 0;
            rc_local[(size_t)k] = job(k, e, sizeof e);
            if (rc_local[(size_t)k]) msg[(size_t)k] = e;
        }
    };
    std::vector<std::thread> pool;
    try {
        for (int w = 0; w < nworkers; w++) pool.emplace_back(worker);
    } catch (...) {
        for (auto &t : pool) t.join();
        errf(err, errlen, "could not start the worker threads");
        return FPLUS_ERR_NOMEM;
    }
    for (auto &t : pool) t.join();
    int rc = FPLUS_OK;
    for (int64_t k = 0; k < count; k++) {
        if (rcs) rcs[k] = rc_local[(size_t)k];
        if (rc == FPLUS_OK && rc_local[(size_t)k]) { rc = rc_local[(size_t)k]; errf(err, errlen, "matrix %ld: %s", (long)k, msg[(size_t)k].c_str()); }
    }
    return rc;
}

extern "C" int fplus_b200_factor_batch(int64_t count, const fplus_symbolic *const *syms, const int64_t *const *Ap,
                                       const int64_t *const *Ai, const void *const *Ax, int is_complex,
                                       const fplus_options *opt, int nworkers, fplus_numeric **nums, int *rcs, char *err,
                                       size_t errlen)
{
    if (count > 0 && (!syms || !Ap || !Ai || !Ax || !nums)) { errf(err, errlen, "NULL array"); return FPLUS_ERR_BADARG; }
    for (int64_t k = 0; k < count; k++) nums[k] = nullptr;
    // predicted cost, in one unit for the whole batch: the front structures' multiply-adds when every pattern has been
    // factored before, else n * nnz for every matrix
    std::vector<double> flops(count > 0 ? (size_t)count : 0, 0.0), nz(flops.size(), 0.0);
    bool all_planned = true;
    for (int64_t k = 0; k < count; k++) {
        const fplus_symbolic *S = syms[k];
        if (!S) continue;
        std::lock_guard<std::mutex> lk(S->mu);
        nz[(size_t)k] = (double)S->n * (double)S->nnz;
        if (S->plan) flops[(size_t)k] = S->plan->flops_real;
        else all_planned = false;
    }
    const std::vector<double> &cost = all_planned ? flops : nz;
    return run_batch(count, nworkers, [&](int64_t k, char *e, size_t el) {
        return factor_common(syms[k], Ap[k], Ai[k], Ax[k], 0, is_complex, opt, &nums[k], e, el);
    }, rcs, err, errlen, &cost);
}

extern "C" int fplus_b200_solve_batch(int64_t count, fplus_numeric *const *nums, void *const *b, const int64_t *nrhs,
                                      const int64_t *ldb, int trans, int nworkers, int *rcs, char *err, size_t errlen)
{
    if (count > 0 && (!nums || !b || !nrhs || !ldb)) { errf(err, errlen, "NULL array"); return FPLUS_ERR_BADARG; }
    // predicted cost: the factor entries read by the sweeps, times the right-hand sides
    std::vector<double> cost(count > 0 ? (size_t)count : 0, 0.0);
    for (int64_t k = 0; k < count; k++)
        if (nums[k]) cost[(size_t)k] = (double)(nums[k]->info.nnz_L + nums[k]->info.nnz_U) * (double)(nrhs[k] > 0 ? nrhs[k] : 0);
    return run_batch(count, nworkers, [&](int64_t k, char *e, size_t el) {
        return solve_common(nums[k], b[k], nrhs[k], ldb[k], trans, 0, e, el);
    }, rcs, err, errlen, &cost);
}

extern "C" int fplus_solve(const fplus_numeric *num, void *b, int64_t nrhs, int64_t ldb, int trans, char *err, size_t errlen)
{
    return solve_common(num, b, nrhs, ldb, trans, 0, err, errlen);
}

extern "C" int fplus_b200_solve_dev(const fplus_numeric *num, void *b_dev, int64_t nrhs, int64_t ldb, int trans, char *err,
                                    size_t errlen)
{
    return solve_common(num, b_dev, nrhs, ldb, trans, 1, err, errlen);
}

static void low_unregister(const void *Lx);

extern "C" void fplus_factors_free(fplus_factors *f)
{
    if (!f) return;
    if (f->Lx) low_unregister(f->Lx);
    free(f->Lp); free(f->Li); free(f->Lx); free(f->Up); free(f->Ui); free(f->Ux); free(f->p); free(f->q);
    f->Lp = f->Li = f->Up = f->Ui = f->p = f->q = nullptr; f->Lx = f->Ux = nullptr;
}

extern "C" void fplus_numeric_free(fplus_numeric *num)
{
    if (!num) return;
    fplus_factors_free(&num->f);
    delete num;
}

// Host copies of L and U (FPLUS src/factor_sn.c:741-808 layout): L in pivot order with the unit diagonal first and the
// rows below ascending, U with rows ascending (the diagonal last); the front structure's explicit zeros included.
static int materialize(const fplus_numeric *num)
{
    const FrontPlan &P = *num->plan;
    DevNum &N = *num->dev;
    const int64_t n = num->n;
    const size_t vs = (size_t)N.vs;
    std::vector<char> La((size_t)P.L_size * vs), Ua((size_t)P.U_size * vs);
    std::vector<int64_t> rowid((size_t)P.rows_total);
    if (cudaSetDevice(N.device) != cudaSuccess) return FPLUS_ERR_GPU;
    if (P.L_size && cudaMemcpy(La.data(), N.Larena, La.size(), cudaMemcpyDeviceToHost) != cudaSuccess) return FPLUS_ERR_GPU;
    if (P.U_size && cudaMemcpy(Ua.data(), N.Uarena, Ua.size(), cudaMemcpyDeviceToHost) != cudaSuccess) return FPLUS_ERR_GPU;
    if (P.rows_total && cudaMemcpy(rowid.data(), N.rowid, rowid.size() * 8, cudaMemcpyDeviceToHost) != cudaSuccess) return FPLUS_ERR_GPU;
    std::vector<int64_t> pinv((size_t)(n > 0 ? n : 1));
    for (int64_t k = 0; k < n; k++) pinv[num->p_lu[k]] = k;
    fplus_factors &f = num->f;
    std::memset(&f, 0, sizeof(f));
    f.n = n; f.is_complex = num->is_complex; f.csc = 1; f.nsupernodes = (int64_t)P.fronts.size();
    // L
    int64_t nl = 0;
    for (auto &F : P.fronts) for (int64_t i = 0; i < F.npiv && i < F.nrows; i++) nl += F.nrows - i;
    f.Lp = (int64_t *)malloc((size_t)(n + 1) * 8);
    f.Li = (int64_t *)malloc((size_t)(nl > 0 ? nl : 1) * 8);
    f.Lx = malloc((size_t)(nl > 0 ? nl : 1) * vs);
    f.p = (int64_t *)malloc((size_t)(n > 0 ? n : 1) * 8);
    f.q = (int64_t *)malloc((size_t)(n > 0 ? n : 1) * 8);
    if (!f.Lp || !f.Li || !f.Lx || !f.p || !f.q) { fplus_factors_free(&f); return FPLUS_ERR_NOMEM; }
    std::vector<std::pair<int64_t, int64_t>> ord;
    int64_t o = 0;
    const double one[2] = {1.0, 0.0};
    for (auto &F : P.fronts) {
        for (int64_t i = 0; i < F.npiv && i < F.nrows; i++) {
            const int64_t k = F.f + i;
            f.Lp[k] = o;
            f.Li[o] = k;
            std::memcpy((char *)f.Lx + (size_t)o * vs, one, vs);
            o++;
            ord.clear();
            for (int64_t r = i + 1; r < F.nrows; r++) ord.emplace_back(pinv[rowid[F.row_off + r]], r);
            std::sort(ord.begin(), ord.end());
            for (auto &t : ord) {
                f.Li[o] = t.first;
                std::memcpy((char *)f.Lx + (size_t)o * vs, La.data() + (size_t)(F.L_off + t.second + i * F.nrows) * vs, vs);
                o++;
            }
        }
    }
    f.Lp[n] = o;
    // U: per column, the rows of the fronts that hold it, ascending
    std::vector<int64_t> cnt((size_t)n + 1, 0);
    for (auto &F : P.fronts)
        for (int64_t i = 0; i < F.npiv && i < F.nrows; i++)
            for (int64_t t = i; t < F.ncols; t++) cnt[P.cols[F.col_off + t] + 1]++;
    for (int64_t j = 0; j < n; j++) cnt[j + 1] += cnt[j];
    const int64_t nu = cnt[n];
    f.Up = (int64_t *)malloc((size_t)(n + 1) * 8);
    f.Ui = (int64_t *)malloc((size_t)(nu > 0 ? nu : 1) * 8);
    f.Ux = malloc((size_t)(nu > 0 ? nu : 1) * vs);
    if (!f.Up || !f.Ui || !f.Ux) { fplus_factors_free(&f); return FPLUS_ERR_NOMEM; }
    std::memcpy(f.Up, cnt.data(), (size_t)(n + 1) * 8);
    std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
    for (auto &F : P.fronts)      // fronts in increasing pivot order: each column fills in ascending row order
        for (int64_t i = 0; i < F.npiv && i < F.nrows; i++) {
            const int64_t k = F.f + i;
            for (int64_t t = i; t < F.ncols; t++) {
                const int64_t c = P.cols[F.col_off + t];
                const int64_t w = fill[c]++;
                f.Ui[w] = k;
                const char *src = t < F.npiv ? La.data() + (size_t)(F.L_off + i + t * F.nrows) * vs
                                             : Ua.data() + (size_t)(F.U_off + i + (t - F.npiv) * F.npiv) * vs;
                std::memcpy((char *)f.Ux + (size_t)w * vs, src, vs);
            }
        }
    for (int64_t k = 0; k < n; k++) { f.p[k] = num->p_lu[k]; f.q[k] = k; }
    return FPLUS_OK;
}

extern "C" const fplus_factors *fplus_numeric_factors(const fplus_numeric *num)
{
    std::lock_guard<std::mutex> lk(num->mu);
    if (!num->have_host) {
        if (materialize(num) != FPLUS_OK) return nullptr;
        num->have_host = true;
    }
    return &num->f;
}

extern "C" const int64_t *fplus_numeric_p(const fplus_numeric *num) { return num->p.data(); }
extern "C" const int64_t *fplus_numeric_q(const fplus_numeric *num) { return num->q.data(); }
extern "C" const double *fplus_numeric_Dr(const fplus_numeric *num) { return num->Dr.data(); }
extern "C" const double *fplus_numeric_Dc(const fplus_numeric *num) { return num->Dc.data(); }

extern "C" int fplus_b200_numeric_info(const fplus_numeric *num, fplus_b200_info *info)
{
    if (!num || !info) return FPLUS_ERR_BADARG;
    *info = num->info;
    return FPLUS_OK;
}

extern "C" int fplus_b200_factor_norms(const fplus_numeric *num, double *L_fro, double *U_fro, char *err, size_t errlen)
{
    if (!num || !L_fro || !U_fro) { errf(err, errlen, "NULL argument"); return FPLUS_ERR_BADARG; }
    std::lock_guard<std::mutex> lk(num->mu);
    DevNum &N = *num->dev;
    CKH(cudaSetDevice(N.device));
    cudaStream_t saved = N.stream;
    if (tl_stream) N.stream = tl_stream;
    const int rc = dev_factor_norms(*num->plan, N, L_fro, U_fro, err, errlen);
    N.stream = saved;
    return rc;
}

// ---- host-only views of the multifrontal structure (tests)
static int plan_for(const fplus_symbolic *sym, int64_t tail, FrontPlan &P)
{
    fplus_symbolic_view v{sym->n, sym->n_tau_rows, sym->n_tau_cols, sym->Bp.data(), sym->Bi.data()};
    return build_plan(v, tail, 64, 256, P) ? FPLUS_ERR_NOMEM : FPLUS_OK;
}

extern "C" int fplus_b200_plan_size(const fplus_symbolic *sym, int64_t tail, int64_t *nfronts, int64_t *ncols_total, int64_t *f_dense)
{
    if (!sym) return FPLUS_ERR_BADARG;
    FrontPlan P;
    int rc = plan_for(sym, tail, P);
    if (rc) return rc;
    if (nfronts) *nfronts = (int64_t)P.fronts.size();
    if (ncols_total) *ncols_total = (int64_t)P.cols.size();
    if (f_dense) *f_dense = P.f_dense;
    return FPLUS_OK;
}

extern "C" int fplus_b200_plan_export(const fplus_symbolic *sym, int64_t tail, int64_t *col_front, int64_t *parent,
                                      int64_t *col_ptr, int64_t *cols, int64_t *nrows, int64_t *nbord)
{
    if (!sym) return FPLUS_ERR_BADARG;
    FrontPlan P;
    int rc = plan_for(sym, tail, P);
    if (rc) return rc;
    const int64_t nf = (int64_t)P.fronts.size();
    if (col_front) std::memcpy(col_front, P.col_front.data(), (size_t)sym->n * 8);
    for (int64_t s = 0; s < nf; s++) {
        const Front &F = P.fronts[s];
        if (parent) parent[s] = F.parent;
        if (col_ptr) col_ptr[s] = F.col_off;
        if (nrows) nrows[s] = F.nrows;
        if (nbord) nbord[s] = F.nbord;
    }
    if (col_ptr) col_ptr[nf] = (int64_t)P.cols.size();
    if (cols) std::memcpy(cols, P.cols.data(), P.cols.size() * 8);
    return FPLUS_OK;
}

extern "C" long long fplus_b200_launch_count(void) { return launch_count(); }

extern "C" void fplus_b200_profile(int on) { prof_enable(on); }

extern "C" int fplus_b200_profile_read(int cls, double *ms, long long *count, double *flops, double *bytes)
{
    if (cls < 0 || cls >= PROF_NCLASS) return FPLUS_ERR_BADARG;
    ProfClass c = prof_read(cls);
    if (ms) *ms = c.ms;
    if (count) *count = c.count;
    if (flops) *flops = c.flops;
    if (bytes) *bytes = c.bytes;
    return FPLUS_OK;
}

// The allocation-free solve: see include/fplus_b200.h.  The status word read afterwards belongs to the factorization.
extern "C" int fplus_b200_solve_dev_noalloc(const fplus_numeric *num, void *b_dev, int64_t nrhs, int64_t ldb, int trans,
                                            char *err, size_t errlen)
{
    if (!num) { errf(err, errlen, "fplus_b200_solve_dev_noalloc: num is NULL"); return FPLUS_ERR_BADARG; }
    const int64_t n = num->n;
    if (trans < 0 || trans > 2 || nrhs < 0 || ldb < n) { errf(err, errlen, "fplus_b200_solve_dev_noalloc: bad trans, nrhs or ldb"); return FPLUS_ERR_BADARG; }
    if (nrhs == 0 || n == 0) return FPLUS_OK;
    if (!b_dev) { errf(err, errlen, "fplus_b200_solve_dev_noalloc: b is NULL"); return FPLUS_ERR_BADARG; }
    std::lock_guard<std::mutex> lk(num->mu);
    DevNum &N = *num->dev;
    CKH(cudaSetDevice(N.device));
    cudaStream_t s = tl_stream ? tl_stream : N.stream;
    cudaStream_t saved = N.stream;
    N.stream = s;
    int rc = dev_clear_status(N, err, errlen);
    if (rc == FPLUS_OK) rc = dev_solve_noalloc(*num->plan, *num->dplan, N, b_dev, ldb, nrhs, trans, s, err, errlen);
    if (rc == FPLUS_OK) {
        int code = 0; int64_t idx = 0;
        rc = dev_status(N, &code, &idx, err, errlen);
        if (rc == FPLUS_OK && code != 0) { errf(err, errlen, "fplus_b200_solve_dev_noalloc: zero or missing diagonal in U"); rc = FPLUS_ERR_SINGULAR; }
    }
    N.stream = saved;
    return rc;
}

// ---------------------------------------------------------------------------------------------------------------------
// The low-level interface that FPLUS's Python extension calls (FPLUS include/fplus.h:73-88, 125-134;
// _sparse_lu_c.c:360, 526): the factorization of A[row_perm, :][:, col_perm] with orders the caller chose, returned as
// host CSC factors, and triangular solves on CSC factors with a plan.
//
// The factorization is fplus_factor's GPU path on a symbolic object made from the given orders (kept in a small cache,
// so that refactoring with the same orders and pattern reuses its front structure and dense-chain start).  Its device
// factors stay alive beside the host arrays it returns, in a registry of the most recent DEV_KEEP factorizations: a
// plan made on those very arrays (the same pointers) solves on the GPU with them, in the coordinates of the permuted
// matrix.  A solve checks that the arrays are still the ones returned (pointers, sizes and a digest of every byte);
// anything else (factors from elsewhere, copies, modified values, an entry dropped from the registry) takes the
// level-scheduled GPU sweeps over the arrays passed (trisolve.cu).  fplus_factors_free on the returned struct drops
// the registry entry; the Python extension frees the arrays itself, so its entries go when the registry is full.

namespace {

constexpr size_t SYM_KEEP = 4, DEV_KEEP = 4;

std::mutex g_sym_mu;
std::vector<std::shared_ptr<fplus_symbolic>> g_syms;        // most recently used last

// A 128-bit digest of the factor arrays (Lp, Li, Lx, Up, Ui, Ux: every byte), so that a solve can tell whether the
// arrays still hold what the factorization returned.  Each array is hashed in 4 MiB chunks (four interleaved
// multiply-rotate lanes over 8-byte words, finished by a 64-bit avalanche), on up to 16 host threads for large arrays;
// the chunk hashes are folded in order, so the digest does not depend on the thread count.
struct Digest {
    uint64_t a = 0, b = 0;
    bool operator==(const Digest &o) const { return a == o.a && b == o.b; }
};
inline uint64_t rotl64(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }
inline uint64_t fmix64(uint64_t k)
{
    k ^= k >> 33; k *= 0xff51afd7ed558ccdULL;
    k ^= k >> 33; k *= 0xc4ceb9fe1a85ec53ULL;
    k ^= k >> 33;
    return k;
}
uint64_t hash_words(const uint64_t *w, size_t nw, uint64_t seed)
{
    const uint64_t K1 = 0x87c37b91114253d5ULL, K2 = 0x4cf5ad432745937fULL;
    uint64_t h[4] = {seed, seed ^ K1, seed ^ K2, seed ^ (K1 + K2)};
    size_t i = 0;
    for (; i + 4 <= nw; i += 4)
        for (int l = 0; l < 4; l++) h[l] = rotl64(h[l] + w[i + l] * K1, 31) * K2;
    for (; i < nw; i++) h[0] = rotl64(h[0] + w[i] * K1, 31) * K2;
    return fmix64(h[0] ^ rotl64(h[1], 17) ^ rotl64(h[2], 29) ^ rotl64(h[3], 43) ^ (uint64_t)nw);
}
void digest_bytes(const void *p, size_t bytes, Digest &d)
{
    const size_t nw = bytes / 8, CH = (size_t)1 << 19;       // 4 MiB chunks of 8-byte words (sizes are multiples of 8)
    const size_t nch = (nw + CH - 1) / CH;
    std::vector<uint64_t> hc(nch, 0);
    const uint64_t *w = (const uint64_t *)p;
    auto run = [&](size_t c0, size_t c1) {
        for (size_t c = c0; c < c1; c++) hc[c] = hash_words(w + c * CH, std::min(CH, nw - c * CH), 0x9e3779b97f4a7c15ULL + c);
    };
    const unsigned hw = std::thread::hardware_concurrency();
    const size_t nt = std::min<size_t>(std::min<size_t>(hw ? hw : 1, 16), nch >= 8 ? nch / 4 : 1);
    if (nt <= 1) run(0, nch);
    else {
        std::vector<std::thread> th;
        const size_t per = (nch + nt - 1) / nt;
        try {
            for (size_t t = 0; t < nt; t++) th.emplace_back(run, std::min(nch, t * per), std::min(nch, (t + 1) * per));
        } catch (...) {
            for (auto &x : th) x.join();
            th.clear();
            run(0, nch);
        }
        for (auto &x : th) x.join();
    }
    for (size_t c = 0; c < nch; c++) {
        d.a = fmix64(d.a ^ hc[c]) + (uint64_t)c;
        d.b = rotl64(d.b, 23) ^ fmix64(hc[c] + d.b * 0x9e3779b97f4a7c15ULL);
    }
    d.a = fmix64(d.a ^ (uint64_t)bytes);
    d.b = fmix64(d.b + (uint64_t)bytes);
}

struct DevFactors {
    fplus_numeric *num = nullptr;
    int64_t n = 0, nnzL = 0, nnzU = 0;
    int is_complex = 0;
    const int64_t *Lp = nullptr, *Li = nullptr, *Up = nullptr, *Ui = nullptr;
    const void *Lx = nullptr, *Ux = nullptr;
    Digest fp;                                               // digest of the six arrays as returned
    ~DevFactors() { fplus_numeric_free(num); }
};
std::mutex g_dev_mu;
std::vector<std::shared_ptr<DevFactors>> g_dev;             // most recent last

Digest fingerprint(int64_t n, const int64_t *Lp, const int64_t *Li, const void *Lx, const int64_t *Up, const int64_t *Ui,
                   const void *Ux, size_t vs)
{
    Digest d;
    const int64_t nnzL = Lp[n], nnzU = Up[n];
    digest_bytes(Lp, (size_t)(n + 1) * 8, d);
    digest_bytes(Li, (size_t)nnzL * 8, d);
    digest_bytes(Lx, (size_t)nnzL * vs, d);
    digest_bytes(Up, (size_t)(n + 1) * 8, d);
    digest_bytes(Ui, (size_t)nnzU * 8, d);
    digest_bytes(Ux, (size_t)nnzU * vs, d);
    return d;
}

// the cached symbolic object for these orders and this pattern, or a new one
int sym_for_orders(int64_t n, const int64_t *Ap, const int64_t *Ai, const int64_t *rp, const int64_t *cp,
                   std::shared_ptr<fplus_symbolic> *out, char *err, size_t errlen)
{
    const int64_t nnz = Ap[n];
    {
        std::lock_guard<std::mutex> lk(g_sym_mu);
        for (size_t k = 0; k < g_syms.size(); k++) {
            const fplus_symbolic &S = *g_syms[k];
            if (S.n != n || S.nnz != nnz) continue;
            if (std::memcmp(S.row_perm.data(), rp, (size_t)n * 8) || std::memcmp(S.col_perm.data(), cp, (size_t)n * 8)) continue;
            if (std::memcmp(S.Ap0.data(), Ap, (size_t)(n + 1) * 8) || (nnz && std::memcmp(S.Ai0.data(), Ai, (size_t)nnz * 8))) continue;
            *out = g_syms[k];
            g_syms.erase(g_syms.begin() + (long)k);
            g_syms.push_back(*out);
            return FPLUS_OK;
        }
    }
    fplus_symbolic *s = nullptr;
    int rc = symbolic_from_orders(n, Ap, Ai, rp, cp, &s, err, errlen);
    if (rc != FPLUS_OK) return rc;
    out->reset(s, fplus_symbolic_free);
    std::lock_guard<std::mutex> lk(g_sym_mu);
    g_syms.push_back(*out);
    if (g_syms.size() > SYM_KEEP) g_syms.erase(g_syms.begin());
    return FPLUS_OK;
}

// fplus_factor on sym with the low-level arguments; the host factors (FPLUS src/factor_sn.c:741-808 layout, p and q of
// the permuted matrix) into *out, the scalings in the permuted order into Dr, Dc; the device factors registered
int low_factor(const fplus_symbolic *sym, const int64_t *Ap, const int64_t *Ai, const void *Ax, int is_complex, int equilibrate,
               int ruiz_max_iter, double ruiz_tol, int verbose, int64_t relax_rows, int64_t panel, int use_gpu,
               double gpu_min_flops, double pivot_rel, fplus_factors *out, double *Dr, double *Dc, char *err, size_t errlen)
{
    fplus_options opt;
    fplus_default_options(&opt);
    opt.equilibrate = equilibrate; opt.ruiz_max_iter = ruiz_max_iter; opt.ruiz_tol = ruiz_tol; opt.verbose = verbose;
    opt.relax_rows = relax_rows; opt.panel = panel; opt.use_gpu = use_gpu; opt.gpu_min_flops = gpu_min_flops;
    opt.pivot_rel = pivot_rel;
    fplus_numeric *num = nullptr;
    int rc = fplus_factor(sym, Ap, Ai, Ax, is_complex, &opt, &num, err, errlen);
    if (rc != FPLUS_OK) return rc;
    {
        std::lock_guard<std::mutex> lk(num->mu);
        rc = materialize(num);
        if (rc == FPLUS_OK) { *out = num->f; std::memset(&num->f, 0, sizeof(num->f)); num->have_host = false; }
    }
    if (rc != FPLUS_OK) {
        fplus_numeric_free(num);
        errf(err, errlen, rc == FPLUS_ERR_NOMEM ? "out of memory" : "reading the factors back failed");
        return rc;
    }
    const int64_t n = num->n;
    for (int64_t k = 0; k < n; k++) { Dr[k] = num->Drp[k]; Dc[k] = num->Dcp[k]; }
    auto d = std::make_shared<DevFactors>();
    d->num = num; d->n = n; d->is_complex = is_complex;
    d->nnzL = out->Lp[n]; d->nnzU = out->Up[n];
    d->Lp = out->Lp; d->Li = out->Li; d->Up = out->Up; d->Ui = out->Ui; d->Lx = out->Lx; d->Ux = out->Ux;
    d->fp = fingerprint(n, d->Lp, d->Li, d->Lx, d->Up, d->Ui, d->Ux, is_complex ? 16 : 8);
    std::shared_ptr<DevFactors> dropped;
    {
        std::lock_guard<std::mutex> lk(g_dev_mu);
        g_dev.push_back(d);
        if (g_dev.size() > DEV_KEEP) { dropped = g_dev.front(); g_dev.erase(g_dev.begin()); }
    }
    return FPLUS_OK;
}

}  // namespace

static void low_unregister(const void *Lx)
{
    std::shared_ptr<DevFactors> dropped;      // released after the lock (its numeric frees device memory)
    std::lock_guard<std::mutex> lk(g_dev_mu);
    for (size_t k = 0; k < g_dev.size(); k++)
        if (g_dev[k]->Lx == Lx) { dropped = g_dev[k]; g_dev.erase(g_dev.begin() + (long)k); break; }
}

// FPLUS include/fplus.h:125-129, src/pipeline.c:84-111
extern "C" int fplus_factor_sn_perm(int64_t n, const int64_t *Ap, const int64_t *Ai, const void *Ax, int is_complex,
                                    const int64_t *row_perm, const int64_t *col_perm, int equilibrate, int ruiz_max_iter,
                                    double ruiz_tol, int verbose, int64_t relax_rows, int64_t panel, int use_gpu,
                                    double gpu_min_flops, double pivot_rel, fplus_factors *out, double *Dr, double *Dc,
                                    char *err, size_t errlen)
{
    if (!out) { errf(err, errlen, "out is NULL"); return FPLUS_ERR_BADARG; }
    std::memset(out, 0, sizeof(*out));
    int rc = check_compressed(n, Ap, Ai, 1, err, errlen);
    if (rc == FPLUS_OK && (!row_perm || !col_perm || !Dr || !Dc || (!Ax && Ap[n] > 0))) {
        errf(err, errlen, "NULL argument");
        rc = FPLUS_ERR_BADARG;
    }
    if (rc == FPLUS_OK) rc = check_perm(n, row_perm, "row_perm", err, errlen);
    if (rc == FPLUS_OK) rc = check_perm(n, col_perm, "col_perm", err, errlen);
    if (rc != FPLUS_OK) return rc;
    std::shared_ptr<fplus_symbolic> sym;
    if ((rc = sym_for_orders(n, Ap, Ai, row_perm, col_perm, &sym, err, errlen))) return rc;
    return low_factor(sym.get(), Ap, Ai, Ax, is_complex, equilibrate, ruiz_max_iter, ruiz_tol, verbose, relax_rows, panel,
                      use_gpu, gpu_min_flops, pivot_rel, out, Dr, Dc, err, errlen);
}

// FPLUS include/fplus.h:54-56, src/factor_sn.c:609-660: partial-pivot LU of the matrix as given (no permutation, no
// equilibration), q the identity.  The input need not be canonical (the reference checks it with canonical = 0): rows are
// sorted within each column and repeated entries summed (the reference accumulates them when it scatters a column), then
// the factorization is fplus_factor_sn_perm's on identity orders, so its device factors serve plans on the returned arrays.
extern "C" int fplus_factor_sn(int64_t n, const int64_t *Ap, const int64_t *Ai, const void *Ax, int is_complex, int verbose,
                               int64_t relax_rows, int64_t panel, int use_gpu, double gpu_min_flops, double pivot_rel,
                               fplus_factors *out, char *err, size_t errlen)
{
    if (!out) { errf(err, errlen, "out is NULL"); return FPLUS_ERR_BADARG; }
    std::memset(out, 0, sizeof(*out));
    if (!(pivot_rel >= 0.0)) { errf(err, errlen, "pivot_rel must be >= 0"); return FPLUS_ERR_BADARG; }
    int rc = check_compressed(n, Ap, Ai, 0, err, errlen);
    if (rc != FPLUS_OK) return rc;
    if (!Ax && Ap[n] > 0) { errf(err, errlen, "NULL argument"); return FPLUS_ERR_BADARG; }
    if ((rc = check_finite(Ap[n], Ax, is_complex, err, errlen))) return rc;
    const size_t vs = is_complex ? 16 : 8;
    try {
        std::vector<int64_t> Cp((size_t)n + 1, 0), Ci, ord;
        std::vector<unsigned char> Cx;
        Ci.reserve((size_t)Ap[n]);
        Cx.reserve((size_t)Ap[n] * vs);
        for (int64_t j = 0; j < n; j++) {
            ord.clear();
            for (int64_t q = Ap[j]; q < Ap[j + 1]; q++) ord.push_back(q);
            std::stable_sort(ord.begin(), ord.end(), [&](int64_t a, int64_t b) { return Ai[a] < Ai[b]; });
            for (size_t t = 0; t < ord.size(); t++) {
                const double *v = (const double *)((const char *)Ax + (size_t)ord[t] * vs);
                if (t > 0 && Ai[ord[t]] == Ai[ord[t - 1]]) {           // a repeated entry: summed into the previous one
                    double *w = (double *)(Cx.data() + Cx.size() - vs);
                    w[0] += v[0];
                    if (is_complex) w[1] += v[1];
                    continue;
                }
                Ci.push_back(Ai[ord[t]]);
                Cx.insert(Cx.end(), (const unsigned char *)v, (const unsigned char *)v + vs);
            }
            Cp[(size_t)j + 1] = (int64_t)Ci.size();
        }
        std::vector<int64_t> id((size_t)(n > 0 ? n : 1));
        for (int64_t k = 0; k < n; k++) id[(size_t)k] = k;
        std::vector<double> Dr((size_t)(n > 0 ? n : 1)), Dc((size_t)(n > 0 ? n : 1));
        return fplus_factor_sn_perm(n, Cp.data(), Ci.data(), Cx.data(), is_complex, id.data(), id.data(), 0, 20, 1e-2, verbose,
                                    relax_rows, panel, use_gpu, gpu_min_flops, pivot_rel, out, Dr.data(), Dc.data(), err, errlen);
    } catch (const std::bad_alloc &) {
        errf(err, errlen, "out of memory");
        return FPLUS_ERR_NOMEM;
    }
}

// FPLUS include/fplus.h:60-62, 139-147: the row kernel (rook / full pivoting, incomplete LU) is not built in this
// library; these entry points exist so that programs linked against FPLUS resolve, and refuse every call.
static int row_kernel_absent(fplus_factors *out, char *err, size_t errlen)
{
    if (out) std::memset(out, 0, sizeof(*out));
    errf(err, errlen, "the row kernel (rook / full pivoting, incomplete LU) is not built in this library: use partial "
                      "pivoting (fplus_factor_sn*, fplus_factor)");
    return FPLUS_ERR_BADARG;
}
extern "C" int fplus_factor_row(int64_t, const int64_t *, const int64_t *, const void *, double, int, int, int, double,
                                fplus_factors *out, char *err, size_t errlen)
{
    return row_kernel_absent(out, err, errlen);
}
extern "C" int fplus_factor_row_perm(int64_t, const int64_t *, const int64_t *, const void *, int, const int64_t *,
                                     const int64_t *, int, int, double, int, double, int, double, fplus_factors *out, double *,
                                     double *, char *err, size_t errlen)
{
    return row_kernel_absent(out, err, errlen);
}
extern "C" int fplus_factor_row_sym(const fplus_symbolic *, const int64_t *, const int64_t *, const void *, int, int, int,
                                    double, int, double, int, double, fplus_factors *out, double *, double *, char *err,
                                    size_t errlen)
{
    return row_kernel_absent(out, err, errlen);
}

// FPLUS include/fplus.h:130-134, src/pipeline.c:113-127
extern "C" int fplus_factor_sn_sym(const fplus_symbolic *sym, const int64_t *Ap, const int64_t *Ai, const void *Ax, int is_complex,
                                   int equilibrate, int ruiz_max_iter, double ruiz_tol, int verbose, int64_t relax_rows,
                                   int64_t panel, int use_gpu, double gpu_min_flops, double pivot_rel, fplus_factors *out,
                                   double *Dr, double *Dc, char *err, size_t errlen)
{
    if (!out) { errf(err, errlen, "out is NULL"); return FPLUS_ERR_BADARG; }
    std::memset(out, 0, sizeof(*out));
    if (!sym || !Ap || !Dr || !Dc) { errf(err, errlen, "NULL argument"); return FPLUS_ERR_BADARG; }
    if (Ap[sym->n] != sym->nnz) {
        errf(err, errlen, "the matrix has %ld nonzeros, the symbolic analysis %ld", (long)Ap[sym->n], (long)sym->nnz);
        return FPLUS_ERR_BADARG;
    }
    return low_factor(sym, Ap, Ai, Ax, is_complex, equilibrate, ruiz_max_iter, ruiz_tol, verbose, relax_rows, panel, use_gpu,
                      gpu_min_flops, pivot_rel, out, Dr, Dc, err, errlen);
}

struct fplus_solve_plan {
    int64_t n = 0, nnzL = 0, nnzU = 0, nsn = -1;
    std::shared_ptr<DevFactors> dev;                 // the registered factorization these arrays came with, if any
    std::vector<int64_t> udiag;                      // position of U(j, j), -1 when missing
    std::mutex mu;
    std::unique_ptr<TriPlan> gen;                    // the level-scheduled sweeps, built when first needed
};

// FPLUS include/fplus.h:81-83, src/solve_plan.c:81-207
extern "C" int fplus_solve_plan_create(int64_t n, const int64_t *Lp, const int64_t *Li, const int64_t *Up, const int64_t *Ui,
                                       fplus_solve_plan **plan, char *err, size_t errlen)
{
    if (!plan) { errf(err, errlen, "plan is NULL"); return FPLUS_ERR_BADARG; }
    *plan = nullptr;
    int rc = check_compressed(n, Lp, Li, 0, err, errlen);
    if (rc == FPLUS_OK) rc = check_compressed(n, Up, Ui, 0, err, errlen);
    if (rc != FPLUS_OK) return rc;
    fplus_solve_plan *pl = new (std::nothrow) fplus_solve_plan;
    if (!pl) { errf(err, errlen, "out of memory"); return FPLUS_ERR_NOMEM; }
    try {
        pl->n = n; pl->nnzL = Lp[n]; pl->nnzU = Up[n];
        {
            std::lock_guard<std::mutex> lk(g_dev_mu);
            for (auto &d : g_dev)
                if (d->n == n && d->Lp == Lp && d->Li == Li && d->Up == Up && d->Ui == Ui && d->nnzL == pl->nnzL && d->nnzU == pl->nnzU)
                    pl->dev = d;
        }
        pl->udiag.assign((size_t)(n > 0 ? n : 1), -1);
        if (pl->dev) {
            // this library's U: rows ascending in every column, the diagonal last
            for (int64_t j = 0; j < n; j++) if (Up[j + 1] > Up[j] && Ui[Up[j + 1] - 1] == j) pl->udiag[j] = Up[j + 1] - 1;
            pl->nsn = (int64_t)pl->dev->num->plan->fronts.size();
        } else {
            pl->gen.reset(new TriPlan);
            tri_plan_build(*pl->gen, n, Lp, Li, Up, Ui);
            pl->udiag = pl->gen->udiag;
        }
    } catch (const std::bad_alloc &) {
        delete pl;
        errf(err, errlen, "out of memory");
        return FPLUS_ERR_NOMEM;
    }
    *plan = pl;
    return FPLUS_OK;
}

// FPLUS include/fplus.h:84-86, src/solve_plan.c:661-719
extern "C" int fplus_tri_solve_plan(const fplus_solve_plan *pl, int64_t n, const int64_t *Lp, const int64_t *Li, const void *Lx,
                                    const int64_t *Up, const int64_t *Ui, const void *Ux, void *x, int64_t nrhs, int64_t ldx,
                                    int trans, int is_complex)
{
    if (!pl || !Lp || !Up || trans < 0 || trans > 2 || n < 0 || nrhs < 0 || ldx < n || n != pl->n || Lp[n] != pl->nnzL ||
        Up[n] != pl->nnzU)
        return FPLUS_ERR_BADARG;
    const size_t vs = is_complex ? 16 : 8;
    if (n > 0 && !Ux) return FPLUS_ERR_BADARG;
    for (int64_t j = 0; j < n; j++) {      // a zero or missing pivot fails before x is touched
        const int64_t q = pl->udiag[j];
        if (q < 0) return FPLUS_ERR_SINGULAR;
        const double *u = (const double *)((const char *)Ux + (size_t)q * vs);
        if (u[0] == 0.0 && (!is_complex || u[1] == 0.0)) return FPLUS_ERR_SINGULAR;
    }
    if (nrhs == 0 || n == 0) return FPLUS_OK;
    if (!x || !Lx || !Ux) return FPLUS_ERR_BADARG;
    char err[256] = {0};
    const DevFactors *d = pl->dev.get();
    if (d && d->Lp == Lp && d->Li == Li && d->Up == Up && d->Ui == Ui && d->Lx == Lx && d->Ux == Ux && d->is_complex == is_complex) {
        if (fingerprint(n, Lp, Li, Lx, Up, Ui, Ux, vs) == d->fp) return solve_common(d->num, x, nrhs, ldx, trans, 0, err, sizeof(err), 1);
    }
    fplus_solve_plan *mp = const_cast<fplus_solve_plan *>(pl);      // the sweeps are built once, under the plan's lock
    TriPlan *g = nullptr;
    {
        std::lock_guard<std::mutex> lk(mp->mu);
        if (!mp->gen) {
            try {
                mp->gen.reset(new TriPlan);
                tri_plan_build(*mp->gen, n, Lp, Li, Up, Ui);
            } catch (const std::bad_alloc &) {
                mp->gen.reset();
                return FPLUS_ERR_NOMEM;
            }
        }
        g = mp->gen.get();
    }
    return tri_plan_solve(*g, Lx, Ux, x, nrhs, ldx, trans, is_complex, tl_stream, err, sizeof(err));
}

// FPLUS include/fplus.h:87
extern "C" int64_t fplus_solve_plan_nsupernodes(const fplus_solve_plan *plan) { return plan ? plan->nsn : -1; }

// FPLUS include/fplus.h:88
extern "C" void fplus_solve_plan_free(fplus_solve_plan *plan) { delete plan; }

// FPLUS include/fplus.h:73-74, src/solve.c:62-74: one right-hand side, through a plan made for the call
extern "C" int fplus_tri_solve(int64_t n, const int64_t *Lp, const int64_t *Li, const void *Lx, const int64_t *Up,
                               const int64_t *Ui, const void *Ux, void *x, int trans, int is_complex)
{
    if (trans < 0 || trans > 2 || n < 0) return FPLUS_ERR_BADARG;
    fplus_solve_plan *pl = nullptr;
    char err[256] = {0};
    int rc = fplus_solve_plan_create(n, Lp, Li, Up, Ui, &pl, err, sizeof(err));
    if (rc != FPLUS_OK) return rc;
    rc = fplus_tri_solve_plan(pl, n, Lp, Li, Lx, Up, Ui, Ux, x, 1, n, trans, is_complex);
    fplus_solve_plan_free(pl);
    return rc;
}

// FPLUS include/fplus.h:66-67, src/equil.c:186-441: Ruiz equilibration in place on a CSC (is_csc) or CSR matrix, on the
// GPU.  FPLUS computes the same scalings by either route; here a CSR matrix is equilibrated as its CSC form (the device
// gathers the values into column order and the scaled values are scattered back).
extern "C" int fplus_ruiz(int64_t n, const int64_t *indptr, const int64_t *indices, void *data, int is_complex, int is_csc,
                          int max_iter, double tol, int verbose, double *Dr, double *Dc, char *err, size_t errlen)
{
    int rc = check_compressed(n, indptr, indices, 0, err, errlen);
    if (rc == FPLUS_OK && ((!data && indptr[n] > 0) || (n > 0 && (!Dr || !Dc)))) { errf(err, errlen, "NULL argument"); rc = FPLUS_ERR_BADARG; }
    if (rc == FPLUS_OK) rc = check_finite(indptr[n], data, is_complex, err, errlen);
    if (rc != FPLUS_OK) return rc;
    if (n == 0) return FPLUS_OK;
    const int64_t nnz = indptr[n];
    const size_t vs = is_complex ? 16 : 8;
    std::vector<int64_t> Cp((size_t)n + 1, 0), Ci((size_t)(nnz > 0 ? nnz : 1)), src((size_t)(nnz > 0 ? nnz : 1));
    if (is_csc) {
        Cp.assign(indptr, indptr + n + 1);
        for (int64_t k = 0; k < nnz; k++) { Ci[k] = indices[k]; src[k] = k; }
    } else {
        for (int64_t k = 0; k < nnz; k++) Cp[indices[k] + 1]++;
        for (int64_t j = 0; j < n; j++) Cp[j + 1] += Cp[j];
        std::vector<int64_t> fill(Cp.begin(), Cp.end() - 1);
        for (int64_t i = 0; i < n; i++)
            for (int64_t k = indptr[i]; k < indptr[i + 1]; k++) { const int64_t o = fill[indices[k]]++; Ci[o] = i; src[o] = k; }
    }
    std::vector<unsigned char> out((size_t)(nnz > 0 ? nnz : 1) * vs);
    int iters = 0;
    rc = dev_ruiz_matrix(n, Cp, Ci, src, data, out.data(), is_complex ? 1 : 0, max_iter, tol, Dr, Dc, &iters, tl_stream, err,
                         errlen);
    if (rc != FPLUS_OK) return rc;
    for (int64_t k = 0; k < nnz; k++) std::memcpy((unsigned char *)data + (size_t)src[k] * vs, out.data() + (size_t)k * vs, vs);
    if (verbose >= 1) { std::printf("[FPLUS] Ruiz: %d iterations (GPU)\n", iters); std::fflush(stdout); }
    return FPLUS_OK;
}

// Solve with iterative refinement (include/fplus_b200.h).
extern "C" int fplus_b200_solve_refine(const fplus_numeric *num, void *b, int64_t nrhs, int64_t ldb, int trans, int max_iter,
                                       double tol, double *berr, int *iters, char *err, size_t errlen)
{
    if (!num) { errf(err, errlen, "fplus_b200_solve_refine: num is NULL"); return FPLUS_ERR_BADARG; }
    const int64_t n = num->n;
    if (trans < 0 || trans > 2 || nrhs < 0 || ldb < n || max_iter < 0 || !(tol >= 0.0)) {
        errf(err, errlen, "fplus_b200_solve_refine: bad trans, nrhs, ldb, max_iter or tol");
        return FPLUS_ERR_BADARG;
    }
    if (nrhs == 0 || n == 0) return FPLUS_OK;
    if (!b) { errf(err, errlen, "fplus_b200_solve_refine: b is NULL"); return FPLUS_ERR_BADARG; }
    std::vector<double> be((size_t)nrhs);
    std::vector<int> it((size_t)nrhs);
    std::lock_guard<std::mutex> lk(num->mu);
    DevNum &N = *num->dev;
    CKH(cudaSetDevice(N.device));
    cudaStream_t saved = N.stream;
    if (tl_stream) N.stream = tl_stream;
    dev_clear_status(N, err, errlen);
    int rc = dev_solve_refine(*num->plan, *num->dplan, N, b, ldb, nrhs, trans, max_iter, tol, be.data(), it.data(), err, errlen);
    if (rc == FPLUS_OK) {
        int code = 0; int64_t idx = 0;
        rc = dev_status(N, &code, &idx, err, errlen);
        if (rc == FPLUS_OK && code != 0) { errf(err, errlen, "fplus_b200_solve_refine: zero or missing diagonal in U"); rc = FPLUS_ERR_SINGULAR; }
    }
    N.stream = saved;
    if (rc == FPLUS_OK) {
        if (berr) std::memcpy(berr, be.data(), (size_t)nrhs * sizeof(double));
        if (iters) std::memcpy(iters, it.data(), (size_t)nrhs * sizeof(int));
    }
    return rc;
}

// A symbolic object for static orders the caller chose (include/fplus_b200.h).
extern "C" int fplus_b200_symbolic_from_orders(int64_t n, const int64_t *Ap, const int64_t *Ai, const int64_t *row_perm,
                                               const int64_t *col_perm, fplus_symbolic **sym, char *err, size_t errlen)
{
    if (!sym) { errf(err, errlen, "sym is NULL"); return FPLUS_ERR_BADARG; }
    *sym = nullptr;
    int rc = check_compressed(n, Ap, Ai, 1, err, errlen);
    if (rc == FPLUS_OK && (!row_perm || !col_perm)) { errf(err, errlen, "NULL permutation"); rc = FPLUS_ERR_BADARG; }
    if (rc == FPLUS_OK) rc = check_perm(n, row_perm, "row_perm", err, errlen);
    if (rc == FPLUS_OK) rc = check_perm(n, col_perm, "col_perm", err, errlen);
    if (rc != FPLUS_OK) return rc;
    return symbolic_from_orders(n, Ap, Ai, row_perm, col_perm, sym, err, errlen);
}
