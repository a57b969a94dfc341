// trisolve.hpp -- triangular solves on caller-supplied CSC factors (the low-level fplus_tri_solve_plan / fplus_tri_solve
// of FPLUS include/fplus.h:73-88) for factors that this library's device factorization does not hold: a level-scheduled
// sweep on the GPU.  The plan is built on the host from the patterns; its device copy is made on the first solve.
#pragma once
#include <cstdint>
#include <cstddef>
#include <mutex>
#include <vector>
#include <cuda_runtime.h>

namespace fpl {

// One sweep: x[r] = (x[r] - sum_e v(e) x[idx[e]]) / d(r) for the rows r in level order, where the entries of row r are
// ptr[r] .. ptr[r + 1], v(e) = val[src[e]] (conjugated for trans 2) and d(r) = val[diag[r]] (1 when diag[r] < 0).  Every
// row reads only rows of earlier levels.  Consecutive levels of at most TRI_THIN rows run in one CTA, separated by
// block barriers; a wider level is one launch with a warp per row.
struct TriSweep {
    std::vector<int64_t> ptr, idx, src, diag;
    std::vector<int64_t> order, lev_ptr;
    struct Run { int64_t l0, l1; bool cta; };
    std::vector<Run> runs;
    int64_t *d_ptr = nullptr, *d_idx = nullptr, *d_src = nullptr, *d_diag = nullptr, *d_order = nullptr, *d_lev = nullptr;
};

struct TriPlan {
    int64_t n = 0, nnzL = 0, nnzU = 0;
    std::vector<int64_t> udiag;              // position of U(j, j) in Ux, -1 when missing
    TriSweep lf, ub, utf, ltb;               // trans 0: L forward, U backward; trans 1/2: U^T forward, L^T backward
    // device state, made on the first solve and reused; solves on one plan are serialised
    std::mutex mu;
    int device = -1;
    bool uploaded = false;
    cudaStream_t stream = nullptr;
    void *d_Lx = nullptr, *d_Ux = nullptr, *d_x = nullptr;
    size_t cap_Lx = 0, cap_Ux = 0, cap_x = 0;
    ~TriPlan();
};

constexpr int64_t TRI_THIN = 512;

// Builds the four sweeps from the CSC patterns (L unit lower: its diagonal entries are skipped, so are entries above
// it; U upper with its diagonal: entries below the diagonal are skipped).  Host only.
void tri_plan_build(TriPlan &P, int64_t n, const int64_t *Lp, const int64_t *Li, const int64_t *Up, const int64_t *Ui);

// Solves in place on the host array x (nrhs columns, leading dimension ldx) with the values Lx, Ux (host memory), on the
// GPU.  The caller has checked the arguments and that every U(j, j) is present and non-zero.
int tri_plan_solve(TriPlan &P, const void *Lx, const void *Ux, void *x, int64_t nrhs, int64_t ldx, int trans,
                   int is_complex, cudaStream_t user_stream, char *err, size_t errlen);

}  // namespace fpl
