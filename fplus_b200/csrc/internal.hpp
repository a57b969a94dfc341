// internal.hpp -- shared declarations of the host side of libfplus (not installed).
#pragma once
#include <cstdint>
#include <cstddef>
#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <vector>
#include <memory>
#include "fplus.h"

namespace fpl {

void errf(char *err, size_t errlen, const char *fmt, ...);

// Canonical-CSC check (FPLUS src/fplus_internal.h:147-162): n >= 0, ptr[0] == 0, non-decreasing pointers, indices in
// [0, n), strictly increasing inside a line when `canonical`.
int check_compressed(int64_t n, const int64_t *ptr, const int64_t *idx, int canonical, char *err, size_t errlen);
// every value finite (FPLUS src/fplus_internal.h:165-172)
int check_finite(int64_t nnz, const void *x, int is_complex, char *err, size_t errlen);
// p is a permutation of 0..n-1 (FPLUS src/fplus_internal.h:175-182)
int check_perm(int64_t n, const int64_t *p, const char *name, char *err, size_t errlen);

// Minimum-degree column order of the n_col columns of the m x n_col CSC pattern (Cp, Ci), on the column intersection
// graph (the graph of C^T C) held implicitly as a quotient graph whose initial elements are the rows of C.  Empty columns
// go last, in their natural order.  perm[k] = the column placed k-th.
void colamd_order(int64_t m, int64_t n_col, const int64_t *Cp, const int64_t *Ci, int64_t *perm);

// Column elimination tree of the m x n CSC pattern: parent[j] (-1 for a root), and its postorder with children in
// increasing order (post[k] = the column placed k-th).
void coletree(int64_t m, int64_t n, const int64_t *Cp, const int64_t *Ci, int64_t *parent);
void tree_postorder(int64_t n, const int64_t *parent, int64_t *post);

// A symbolic object for the caller's own static orders (the low-level fplus_factor_sn_perm), order.cpp.
int symbolic_from_orders(int64_t n, const int64_t *Ap, const int64_t *Ai, const int64_t *row_perm, const int64_t *col_perm,
                         fplus_symbolic **out, char *err, size_t errlen);

struct FrontPlan;     // the multifrontal structure (symbolic.cpp)
struct DevPlan;       // its device copy (device.cu)

}  // namespace fpl

// The symbolic object: the static orders (FPLUS src/order.c:240-244), the permuted pattern, and the cached multifrontal
// structure for the numeric phase.
struct fplus_symbolic {
    int64_t n = 0, nnz = 0;
    std::vector<int64_t> row_perm, col_perm;
    int64_t n_tau_rows = 0, n_tau_cols = 0;
    // the permuted pattern B = A[row_perm,:][:,col_perm] (canonical CSC) and, per entry of B, its position in A
    std::vector<int64_t> Bp, Bi, Bsrc;
    // the analysed pattern itself (A's Ap, Ai): a factorization's pattern is compared with it
    std::vector<int64_t> Ap0, Ai0;
    // the multifrontal structure, built on first use; rebuilt with a dense tail when a dense row is chosen as a pivot
    // before the tail (the pivot order is value dependent); guarded by mu
    mutable std::mutex mu;
    mutable int64_t tail_hint = -1;       // first column of the dense tail last needed (-1: none)
    // the front structure's shape: at most max_width pivot columns per front, nb_chain per dense-chain front (the
    // autotuner, fplus_b200_autotune, may change them)
    mutable int64_t max_width = 256, nb_chain = 64;
    // the pivot-block LU kernel of the small fronts: 2 (the block in shared memory, a barrier per pivot step), 1 (8-column
    // panels, the later columns' updates on the FP64 tensor cores) or 3 (blocked panels); autotuned
    mutable int lu_variant = 2;
    mutable std::shared_ptr<fpl::FrontPlan> plan;
    mutable std::shared_ptr<fpl::DevPlan> dplan;
};
