// plan.hpp -- the multifrontal structure of the numeric factorization (built on the host from the pattern alone).
//
// The factorization of B = A[row_perm,:][:,col_perm] (its interior: rows [0, mi), columns [0, ni); its dense rows
// [mi, n) and dense columns [ni, n) come last) runs as a sequence of fronts, each a dense column-major block of nrows
// x ncols: the pivot columns [f, f + npiv) first, then the columns its Schur complement (the contribution block, CB)
// reaches.  Partial pivoting may take any row of the front: every row that can hold a nonzero in a pivot column is in
// the front (the row-merge structure of George and Ng, the Cholesky structure of B^T B), so the pivots are those of
// left-looking partial pivoting on B.
//
//   interior fronts   supernodes of the column elimination tree of the interior (fundamental, then relaxed, width-
//                     capped), for the columns [0, f_dense).  Their rows: the interior rows whose first column is a
//                     pivot column, the children's CB rows, and the dense rows as `border` rows at the bottom.  A dense
//                     row is dense in every column, so it is never part of the column structure; a front assembles its
//                     entries in the front's own pivot columns and carries the updates of its other columns upward.  A
//                     border row chosen as a pivot would need columns outside the structure: the factorization reports
//                     it and is redone with the dense chain starting at that front.
//   dense chain       the columns [f_dense, n) in blocks of at most nb columns, each front's columns all of [f, n).
//                     Without a reported border pivot f_dense = ni (the dense columns only).  The first chain front
//                     takes every pending CB and the dense rows (as ordinary rows); each chain front's CB is the next
//                     one's child.
#pragma once
#include <cstdint>
#include <vector>

namespace fpl {

struct Front {
    int64_t f = 0, npiv = 0;       // pivot columns [f, f + npiv)
    int64_t ncols = 0, nrows = 0;  // front size; CB = rows [npiv, nrows) x cols [npiv, ncols) after pivoting
    int64_t nbord = 0;             // border rows at the bottom (never pivots)
    int64_t nri = 0;               // rows above the border (nrows - nbord)
    int64_t tau_base = 0;          // local row of the first dense row (border or ordinary); children's CB border rows go here
    int64_t parent = -1;
    int64_t slot = 0;              // first local row in the parent for this front's interior CB rows
    int64_t col_off = 0;           // cols[col_off .. + ncols): B column of each local column
    int64_t row_off = 0;           // rowinit / device rowid [row_off .. + nrows)
    int64_t relcol_off = 0;        // relcol[relcol_off .. + ncols - npiv): parent local column of each CB column
    int64_t asm_begin = 0, asm_end = 0;
    int64_t asm_mid = 0;           // [asm_begin, asm_mid): entries in the pivot columns; [asm_mid, asm_end): the others
    int64_t child_begin = 0, child_end = 0;
    int64_t L_off = 0, U_off = 0;  // factor arena (elements): nrows x npiv, npiv x (ncols - npiv)
    int64_t cb_off = 0;            // CB stack (elements): (nrows - npiv) x (ncols - npiv), column-major
    int dense = 0;                 // a chain front: columns [f, n)
    int level = 0;                 // height above the leaves (0 = leaf)
};

struct FrontPlan {
    int64_t n = 0, mi = 0, ni = 0, ntr = 0, ntc = 0;
    int64_t f_dense = 0;           // first column of the dense chain
    int64_t nb_chain = 64, max_width = 256;
    std::vector<Front> fronts;     // in processing order: children before parents, subtrees contiguous
    std::vector<int64_t> cols, relcol, children, rowinit;
    std::vector<int64_t> asm_src, asm_dst;     // B entry -> offset in the front's working block
    std::vector<int64_t> col_front;            // B column -> front
    std::vector<int64_t> head_cols;            // per front: how many of its CB columns lie in its parent's pivot columns,
                                               // which come first (-1: they do not come first; 0 without a parent)
    int64_t L_size = 0, U_size = 0, cb_size = 0, work_size = 0, rows_total = 0;
    int64_t max_nrows = 0, max_ncols = 0, max_npiv = 0;
    double flops_real = 0;         // multiply-adds of the dense fronts (partial factorization), real count
    int nlevels = 0;
};

// Where a Schur update's output element (i, j) goes: identity when col is null, else row i < nslot -> slot + i, row
// i >= nslot -> tau + (i - nslot), column j -> col[j] (a child's contribution block written straight into its parent's
// working block, through the extend-add maps)
struct OutMap {
    const int64_t *col;
    int64_t nslot, slot, tau;
};

// a front as the level-scheduled solve kernels read it (pivot columns [f, f + np), nr rows of which nri above the border,
// nc columns; its L block, its U12 block, its first entry in the plan's row and column arrays)
struct SvFront {
    long long f, np, nr, nri, nc, L_off, U_off, row_off, col_off;
    long long nch, poff;           // the U sweep of a larger front: CB-column chunks, first partial sum (per right-hand side)
};

// a front as the batched factorization kernels read it: its shape, arenas and row / column entries, its assembly entries
// and children, its working block (wofs, within its level's workspace) and contribution block (cbofs, in the batched
// fronts' contribution-block arena)
struct FcFront {
    long long f, np, nr, nri, nc, L_off, U_off, row_off, relcol_off, asm_begin, asm_end, child_begin, child_end, slot,
        tau_base, wofs, cbofs;
};

struct fplus_symbolic_view {
    int64_t n, ntr, ntc;
    const int64_t *Bp, *Bi;
};

// Build the plan for the given dense-chain start (-1: none, the dense columns only).  Returns 0, or -1 (out of memory).
int build_plan(const fplus_symbolic_view &S, int64_t f_tail, int64_t nb_chain, int64_t max_width, FrontPlan &P);

}  // namespace fpl
