// kernels.cuh -- the CUDA kernels of the numeric phase (sm_100a): permutation, Ruiz equilibration, the front kernels
// of the multifrontal LU (assembly, extend-add, panel with partial pivoting, row swaps, unit-lower TRSM, FP64 tensor-core
// GEMM, copy-out) and the supernodal triangular sweeps.  Included once, by numeric.cu.
#pragma once
#include <climits>
#include <cooperative_groups.h>
#include "dev_common.cuh"
#include "plan.hpp"

namespace fpl {

// =====================================================================================================================
// permutation and Ruiz equilibration (FPLUS src/pipeline.c:14-82, src/equil.c:60-183, 186-441)
// =====================================================================================================================

// Bx[p] = Ax[src[p]]: the values of B = A[row_perm,:][:,col_perm] (the pattern and src come from the analysis)
template <typename T>
__global__ void k_gather(T *__restrict__ Bx, const T *__restrict__ Ax, const int64_t *__restrict__ src, int64_t nnz)
{
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < nnz; p += (int64_t)gridDim.x * blockDim.x)
        Bx[p] = Ax[src[p]];
}

// the largest |d| and the smallest positive |d| over the raw doubles (range guard, FPLUS src/equil.c:197-206)
__global__ void k_abs_range(const double *__restrict__ d, int64_t m, DevStatus *st)
{
    double amax = 0.0, amin = INFINITY;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < m; q += (int64_t)gridDim.x * blockDim.x) {
        double a = fabs(d[q]);
        amax = fmax(amax, a);
        if (a > 0.0) amin = fmin(amin, a);
    }
    for (int o = 16; o > 0; o >>= 1) {
        amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
        amin = fmin(amin, __shfl_xor_sync(0xffffffffu, amin, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&st->amax_bits, dbits(amax));
        atomicMin(&st->amin_bits, dbits(amin));
    }
}

// line maxima of max(|re|, |im|) for the wide-range guard (FPLUS src/equil.c:215-227); lmax: 2n zeroed bit patterns
template <bool CPLX>
__global__ void k_line_max(const int64_t *__restrict__ Bp, const int64_t *__restrict__ Bi, const double *__restrict__ d,
                           int64_t n, unsigned long long *lmax)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
        for (int64_t p = Bp[j]; p < Bp[j + 1]; p++) {
            double a = CPLX ? fmax(fabs(d[2 * p]), fabs(d[2 * p + 1])) : fabs(d[p]);
            atomicMax(&lmax[Bi[p]], dbits(a));
            atomicMax(&lmax[n + j], dbits(a));
        }
}

__global__ void k_min_pos(const unsigned long long *__restrict__ v, int64_t m, DevStatus *st)
{
    double amin = INFINITY;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < m; q += (int64_t)gridDim.x * blockDim.x) {
        double a = bitsd(v[q]);
        if (a > 0.0) amin = fmin(amin, a);
    }
    for (int o = 16; o > 0; o >>= 1) amin = fmin(amin, __shfl_xor_sync(0xffffffffu, amin, o));
    if ((threadIdx.x & 31) == 0) atomicMin(&st->amin_bits, dbits(amin));
}

__global__ void k_scale_raw(double *d, int64_t m, double sc)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < m; q += (int64_t)gridDim.x * blockDim.x) d[q] *= sc;
}

// squared modulus exactly as the reference rounds it: re*re + im*im, two products and a sum, no contraction
__device__ __forceinline__ double sqmod(double a) { return __dmul_rn(a, a); }
__device__ __forceinline__ double sqmod(cplx a) { return __dadd_rn(__dmul_rn(a.x, a.x), __dmul_rn(a.y, a.y)); }

// row maxima of |b|^2 (order independent: the maximum of non-negative doubles is their integer maximum)
template <typename T>
__global__ void k_ruiz_rowmax(const int64_t *__restrict__ Bi, const T *__restrict__ Bx, int64_t nnz,
                              unsigned long long *__restrict__ rmax, const DevStatus *st)
{
    if (st->done || st->code) return;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < nnz; p += (int64_t)gridDim.x * blockDim.x)
        atomicMax(&rmax[Bi[p]], dbits(sqmod(Bx[p])));
}

// zero-row check, residual, row scale 1/sqrt(sqrt(max)), Dr *= scale (FPLUS src/equil.c:80-92); the column maxima of
// the coming column pass start at zero
__global__ void k_ruiz_rowscale(int64_t n, unsigned long long *__restrict__ rmax, double *__restrict__ Dr,
                                unsigned long long *__restrict__ cmax, DevStatus *st)
{
    if (st->done || st->code) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        cmax[i] = 0ull;
        double m = bitsd(rmax[i]);
        if (m == 0.0) {           // the smallest zero row wins (the reference reports the first)
            atomicCAS(&((DevStatus *)st)->code, 0, ST_ZERO_ROW);
            continue;
        }
        double v = 0.5 * fabs(log(m));
        atomicMax(&st->res_bits, dbits(v));
        double dr = 1.0 / sqrt(sqrt(m));
        Dr[i] = __dmul_rn(Dr[i], dr);
        rmax[i] = dbits(dr);
    }
}

// zero-row index: the smallest (second pass so the index is deterministic)
__global__ void k_first_zero(int64_t n, const unsigned long long *__restrict__ v, DevStatus *st, int code)
{
    if (st->code != code || st->done) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (bitsd(v[i]) == 0.0) atomicMin((unsigned long long *)&st->idx, (unsigned long long)i);
}

// Column passes run over column segments of at most COL_SEG entries (seg: column, first entry, end; a warp each), so a
// dense column is spread over many warps; a segment's maximum joins its column's by an integer atomicMax (the maximum
// of non-negative doubles is their integer maximum, so the result does not depend on the order).
constexpr int64_t COL_SEG = 1024;

// scale by the row scales, then the column maximum of |b|^2 (FPLUS src/equil.c:93-147); cmax starts at zero
template <typename T>
__global__ void k_ruiz_colpass(const int64_t *__restrict__ seg, int64_t nseg, const int64_t *__restrict__ Bi, T *__restrict__ Bx,
                               const unsigned long long *__restrict__ rscale, unsigned long long *__restrict__ cmax,
                               const DevStatus *st)
{
    if (st->done || st->code) return;
    const int lane = threadIdx.x & 31;
    for (int64_t g = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; g < nseg; g += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int64_t j = seg[3 * g], p1 = seg[3 * g + 2];
        double cm = 0.0;
        for (int64_t p = seg[3 * g + 1] + lane; p < p1; p += 32) {
            T v = scal(Bx[p], bitsd(rscale[Bi[p]]));
            Bx[p] = v;
            cm = fmax(cm, sqmod(v));
        }
        for (int o = 16; o > 0; o >>= 1) cm = fmax(cm, __shfl_xor_sync(0xffffffffu, cm, o));
        if (lane == 0) atomicMax(&cmax[j], dbits(cm));
    }
}

// the zero-column check, residual, column scale, Dc *= scale (FPLUS src/equil.c:148-155)
__global__ void k_ruiz_colscale(int64_t n, unsigned long long *__restrict__ cmax, double *__restrict__ Dc, DevStatus *st)
{
    if (st->done || st->code) return;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        double m = bitsd(cmax[j]);
        if (m == 0.0) { atomicCAS(&st->code, 0, ST_ZERO_COL); continue; }
        double v = 0.5 * fabs(log(m));
        atomicMax(&st->res_bits, dbits(v));
        double c = 1.0 / sqrt(sqrt(m));
        Dc[j] = __dmul_rn(Dc[j], c);
        cmax[j] = dbits(c);
    }
}

template <typename T>
__global__ void k_ruiz_colapply(const int64_t *__restrict__ seg, int64_t nseg, T *__restrict__ Bx,
                                const unsigned long long *__restrict__ cscale, const DevStatus *st)
{
    if (st->done || st->code) return;
    const int lane = threadIdx.x & 31;
    for (int64_t g = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; g < nseg; g += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const double c = bitsd(cscale[seg[3 * g]]);
        const int64_t p1 = seg[3 * g + 2];
        for (int64_t p = seg[3 * g + 1] + lane; p < p1; p += 32) Bx[p] = scal(Bx[p], c);
    }
}

// end of an iteration: count it, stop when the residual is below tol (FPLUS src/equil.c:405-411)
__global__ void k_ruiz_check(DevStatus *st, double tol)
{
    if (st->done) return;
    if (st->code) { st->done = 1; return; }      // an error: later iterations change nothing (the index stays)
    st->iters++;
    if (bitsd(st->res_bits) < tol) st->done = 1;
    st->res_bits = 0ull;
}

__global__ void k_fold(double *Dr, double *Dc, int64_t n, double h)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        Dr[i] *= h; Dc[i] *= h;
    }
}

// the largest modulus of each column of the scaled B (the singular-pivot threshold, FPLUS src/factor_sn_panel.inc:50)
// (over column segments; cm, the bits of non-negative doubles, starts at zero)
template <typename T>
__global__ void k_colmax(const int64_t *__restrict__ seg, int64_t nseg, const T *__restrict__ Bx, unsigned long long *__restrict__ cm)
{
    const int lane = threadIdx.x & 31;
    for (int64_t g = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; g < nseg; g += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        double m = 0.0;
        const int64_t p1 = seg[3 * g + 2];
        for (int64_t p = seg[3 * g + 1] + lane; p < p1; p += 32) m = fmax(m, vabs(Bx[p]));
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0) atomicMax(&cm[seg[3 * g]], dbits(m));
    }
}

// =====================================================================================================================
// fronts
// =====================================================================================================================

// original entries into the front's working block; static row ids
template <typename T>
__global__ void k_assemble(T *__restrict__ W, const T *__restrict__ Bx, const int64_t *__restrict__ src,
                           const int64_t *__restrict__ dst, int64_t cnt, int64_t *__restrict__ rowid,
                           const int64_t *__restrict__ rowinit, int64_t nrows, const DevStatus *st, int addto = 0)
{
    // addto: the block already holds the child's contribution block (written by its Schur update), the entries add to it
    if (st->code) return;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
    if (addto) for (int64_t e = tid; e < cnt; e += stride) W[dst[e]] = add(W[dst[e]], Bx[src[e]]);
    else for (int64_t e = tid; e < cnt; e += stride) W[dst[e]] = Bx[src[e]];
    for (int64_t i = tid; i < nrows; i += stride) if (rowinit[i] >= 0) rowid[i] = rowinit[i];
}

// W += the child's contribution block (rows: the child's interior CB rows into its slots, its border rows onto the
// parent's dense rows; columns through relcol); the child's CB row ids fill the slots
// (columns [c0, c1) of the CB; the row ids when `rowids`)
template <typename T>
__global__ void k_extend_add(T *__restrict__ W, int64_t ldw, const T *__restrict__ cb, int64_t cbr, int64_t c0, int64_t c1,
                             int64_t nslot, int64_t slot, int64_t tau_base, const int64_t *__restrict__ relcol,
                             int64_t *__restrict__ rowid_parent, const int64_t *__restrict__ rowid_child_cb, int rowids,
                             const DevStatus *st)
{
    if (st->code) return;
    const int64_t total = cbr * (c1 - c0);
    if (total < INT_MAX && (int64_t)gridDim.x * blockDim.x < INT_MAX - total) {
        // 32-bit index arithmetic (a 64-bit division per entry costs more than the entry's memory traffic)
        const int cb32 = (int)cbr, tot32 = (int)total;
        for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < tot32; e += gridDim.x * blockDim.x) {
            const int cl = e / cb32, t = e - cl * cb32;
            const int64_t c = c0 + cl;
            const int64_t pr = t < nslot ? slot + t : tau_base + (t - nslot);
            const int64_t pc = relcol[c];
            T v = cb[t + c * cbr];
            T *w = W + pr + pc * ldw;
            *w = add(*w, v);
        }
    } else {
        for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
            const int64_t t = e % cbr, c = c0 + e / cbr;
            const int64_t pr = t < nslot ? slot + t : tau_base + (t - nslot);
            const int64_t pc = relcol[c];
            T v = cb[t + c * cbr];
            T *w = W + pr + pc * ldw;
            *w = add(*w, v);
        }
    }
    if (rowids)
        for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nslot; t += (int64_t)gridDim.x * blockDim.x)
            rowid_parent[slot + t] = rowid_child_cb[t];
}

// Partial pivoting on columns [k0, k0 + w) of the working block (rows [k0, nrows)), one CTA: per column, the argmax of
// the moduli (warp shuffles, then across warps; ties to the smaller row of B), the singular test against pivot_rel *
// max |B(:, j)|, the border test, the row swap inside the panel (and of the row ids), the division by the pivot and the
// rank-1 update of the panel's remaining columns.  Swaps are recorded in ipiv for the other columns.
template <typename T>
__global__ void __launch_bounds__(512) k_panel(T *__restrict__ W, int64_t ld, int64_t nrows, int64_t nri, int k0, int w,
                                              int64_t fcol, const double *__restrict__ colmax, double pivot_rel,
                                              int64_t *__restrict__ rowid, int *__restrict__ ipiv, DevStatus *st,
                                              int64_t front)
{
    __shared__ double s_val[32];
    __shared__ int64_t s_idx[32], s_rid[32];
    __shared__ int64_t s_piv;
    __shared__ T s_row[32];
    __shared__ int s_stop;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    if (tid == 0) s_stop = st->code != 0;
    __syncthreads();
    if (s_stop) return;
    for (int kk = 0; kk < w; kk++) {
        const int64_t j = k0 + kk;
        // argmax over rows [j, nrows)
        double bv = -1.0; int64_t bi = -1, br = INT64_MAX;
        for (int64_t i = j + tid; i < nrows; i += blockDim.x) {
            double a = vabs(W[i + j * ld]);
            int64_t r = rowid[i];
            if (a > bv || (a == bv && r < br)) { bv = a; bi = i; br = r; }
        }
        for (int o = 16; o > 0; o >>= 1) {
            double ov = __shfl_xor_sync(0xffffffffu, bv, o);
            int64_t oi = __shfl_xor_sync(0xffffffffu, bi, o), orr = __shfl_xor_sync(0xffffffffu, br, o);
            if (ov > bv || (ov == bv && orr < br)) { bv = ov; bi = oi; br = orr; }
        }
        if (lane == 0) { s_val[warp] = bv; s_idx[warp] = bi; s_rid[warp] = br; }
        __syncthreads();
        if (tid == 0) {
            double v = s_val[0]; int64_t ix = s_idx[0], rr = s_rid[0];
            for (int q = 1; q < nw; q++)
                if (s_val[q] > v || (s_val[q] == v && s_rid[q] < rr)) { v = s_val[q]; ix = s_idx[q]; rr = s_rid[q]; }
            const double thr = pivot_rel * colmax[fcol + j];
            if (ix < 0 || v <= 0.0 || v < thr) { set_status(st, ST_SINGULAR, fcol + j, v > 0 ? v : 0.0, thr); s_stop = 1; }
            else if (ix >= nri) { set_status(st, ST_BORDER, front, v, thr); s_stop = 1; }
            s_piv = ix;
            if (!s_stop) {
                ipiv[j] = (int)ix;
                if (ix != j) { int64_t t = rowid[j]; rowid[j] = rowid[ix]; rowid[ix] = t; }
            }
        }
        __syncthreads();
        if (s_stop) return;
        const int64_t p = s_piv;
        // swap rows j and p inside the panel; keep the pivot row's panel entries in shared memory
        if (tid < w) {
            const int64_t c = k0 + tid;
            T a = W[j + c * ld], b = W[p + c * ld];
            if (p != j) { W[j + c * ld] = b; W[p + c * ld] = a; }
            s_row[tid] = p != j ? b : a;
        }
        __syncthreads();
        const T piv = s_row[kk];
        for (int64_t i = j + 1 + tid; i < nrows; i += blockDim.x) {
            T l = divv(W[i + j * ld], piv);
            W[i + j * ld] = l;
            for (int c = kk + 1; c < w; c++) {
                T *x = W + i + (k0 + c) * ld;
                *x = sub(*x, mul(l, s_row[c]));
            }
        }
        __syncthreads();
    }
}

// The partial-pivot LU of a tall front's pivot block (nrows x npiv, too large for one CTA's shared memory) in one launch
// over G CTAs resident at once: one thread-block cluster (G <= MC_CMAX: the CTAs exchange their candidates through
// distributed shared memory and the cluster barrier), or a cooperative launch (G up to one CTA per SM: the candidates go
// through global memory and a counter that every CTA increments).  CTA b owns the rows [b * per, b * per + per) and
// keeps its rows' values of the current 32-column panel in shared memory.  Per pivot column j:
//   1. each CTA finds the best of its live rows (the largest pivot key, ties to the smaller row of B) and posts it: the
//      key, the row of B, the position and the row's panel values (cluster: into every CTA's shared memory; grid: into
//      its global slot, then a release increment of the counter);
//   2. after the barrier (the cluster barrier; grid: the counter reaching G (j + 1), a bounded wait) every CTA takes the
//      same winner, applies the same singular / border decision (a stop ends every CTA at the same column), keeps the
//      winner's panel values (row j of L11\U11) and updates its live rows: the multiplier, then the rank-1 update of the
//      panel's later columns.
// After a panel every CTA forms U12 = L11^-1 A12 for the panel's pivot rows (read from W: their owners wrote them before
// posting the panel's first column), by column chunks and redundantly, and applies A22 -= L21 U12 to its own live rows;
// one CTA per chunk keeps U12 in Ub for the final block.  Rows never move: the pivot rows are marked, and k_mc_order /
// k_mc_lout turn the choices (chosen[j] = the position of step j's pivot row) into the final row order (the pivot rows
// in step order, then the others in their order) and the block in that order.  The operations on every value are those
// of the swapping form (the same multipliers, the same forward substitution order), so the factors agree with it.
// The posts alternate by the column's parity.  Grid form: sync[0] is the exit ticket, sync[1] the counter; the last CTA
// to finish resets both, so they start at zero at the next launch (a CUDA graph replay included).
constexpr int MC_THREADS = 512, MC_PW = 32, MC_LB = MC_PW + 1, MC_CMAX = 16;
constexpr unsigned MC_SPIN = 1u << 22;         // polls of the counter before the wait gives up (about a second)
template <typename T> struct __align__(16) McSlot {
    long long key, rid, pos, pad;
    T v[MC_PW];
};
template <typename T> __host__ __device__ constexpr int mc_cw() { return VT<T>::cplx_ ? 64 : 128; }
// shared memory of k_block_lu_mc for `per` rows per CTA (cl: the cluster form's posts too)
template <typename T> __host__ __device__ constexpr size_t mc_smem(int per, bool cl)
{
    return (size_t)(MC_PW * per + MC_PW * MC_LB + MC_PW * mc_cw<T>()) * sizeof(T) +
           (cl ? (size_t)2 * MC_CMAX * sizeof(McSlot<T>) : 0) + (size_t)per * 8 + (size_t)((per + 15) & ~15);
}

template <typename T, bool CL>
__global__ void __launch_bounds__(MC_THREADS) k_block_lu_mc(T *W, int64_t ld, int nrows, int npiv, int nri, int per,
                                                          int64_t fcol, const double *__restrict__ colmax, double pivot_rel,
                                                          const int64_t *__restrict__ rowid, int64_t *__restrict__ chosen,
                                                          T *__restrict__ Ub, McSlot<T> *gslots, unsigned int *sync,
                                                          DevStatus *st, int64_t front)
{
    namespace cg = cooperative_groups;
    constexpr int CW = mc_cw<T>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *S = reinterpret_cast<T *>(smem_raw);              // the panel: S[c * per + r], own row r, panel column c
    T *Lb = S + MC_PW * per;                             // the panel's pivot rows: Lb[k * MC_LB + c] (L11 \ U11)
    T *Uc = Lb + MC_PW * MC_LB;                          // a chunk of U12: Uc[k * CW + c]
    McSlot<T> *cs = reinterpret_cast<McSlot<T> *>(Uc + MC_PW * CW);    // cluster form: the posts, [parity][CTA]
    long long *rid_s = reinterpret_cast<long long *>(reinterpret_cast<unsigned char *>(cs) +
                                                     (CL ? (size_t)2 * MC_CMAX * sizeof(McSlot<T>) : 0));
    unsigned char *live = reinterpret_cast<unsigned char *>(rid_s + per);
    __shared__ long long s_k[16], s_r[16], s_p[16];
    __shared__ int s_q[16];
    __shared__ int s_piv[MC_PW];
    __shared__ T s_wc[16 * MC_PW];                      // cluster form: each warp's candidate row, fully updated
    __shared__ double s_thr[MC_PW];
    __shared__ int s_stop, s_wait;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = MC_THREADS / 32;
    const int G = gridDim.x, b = blockIdx.x;
    const int r_lo = b * per, r_hi = r_lo + per < nrows ? r_lo + per : nrows, nmine = r_hi > r_lo ? r_hi - r_lo : 0;
    const int npr = npiv < nrows ? npiv : nrows;
    if (tid == 0) { s_stop = st->code != 0; s_wait = 0; }
    for (int r = tid; r < per; r += MC_THREADS) {
        live[r] = r < nmine;
        rid_s[r] = r < nmine ? rowid[r_lo + r] : LLONG_MAX;
    }
    if constexpr (CL) {
        // every CTA of the cluster starts from CTA 0's reading of the status word (the barrier counts must agree)
        cg::this_cluster().sync();
        if (tid == 0) s_stop = *cg::this_cluster().map_shared_rank(&s_stop, 0);
    }
    __syncthreads();
    bool stopped = s_stop != 0;                          // the same in every thread (every decision below is)
    for (int p0 = 0; p0 < npr && !stopped; p0 += MC_PW) {
        const int w = npr - p0 < MC_PW ? npr - p0 : MC_PW;
        if (tid < w) s_thr[tid] = pivot_rel * colmax[fcol + p0 + tid];
        for (int e = tid; e < w * nmine; e += MC_THREADS) {
            const int c = e / nmine, r = e - c * nmine;
            S[c * per + r] = W[(r_lo + r) + (int64_t)(p0 + c) * ld];
        }
        __syncthreads();
        // every thread owns row tid of this CTA's rows for the whole panel (per <= MC_THREADS): its key, its multiplier
        // and its update need no block barrier
        bool mine = tid < nmine && live[tid];
        for (int kk = 0; kk < w; kk++) {
            const int j = p0 + kk, par = j & 1;
            // 1. the best of this CTA's live rows in column j, posted
            long long bk = mine ? (long long)pivkey(S[kk * per + tid]) : -1, brid = mine ? rid_s[tid] : LLONG_MAX;
            long long brow = mine ? tid : -1;
            {
                const int src = warp_argbest(bk, brid);
                bk = src >= 0 ? __shfl_sync(0xffffffffu, bk, src) : -1;
                brid = src >= 0 ? __shfl_sync(0xffffffffu, brid, src) : LLONG_MAX;
                brow = src >= 0 ? __shfl_sync(0xffffffffu, brow, src) : -1;
            }
            if constexpr (CL) {
                // the warp's candidate row in full: its later columns still lack the previous pivot's update (applied
                // to every row during the cluster barrier below), so it is applied here, with the same arithmetic
                __syncwarp();
                if (lane < w) {
                    T v = brow >= 0 ? S[lane * per + brow] : VT<T>::zero();
                    if (brow >= 0 && kk >= 1 && lane > kk)
                        v = sub(v, mul(S[(kk - 1) * per + brow], Lb[(kk - 1) * MC_LB + lane]));
                    s_wc[warp * MC_PW + lane] = v;
                }
            }
            if (lane == 0) { s_k[warp] = bk; s_r[warp] = brid; s_p[warp] = brow; }
            __syncthreads();
            if (CL ? warp < G : warp == 0) {
                // the CTA's best (cluster form: every pushing warp takes it; warp d pushes it into CTA d)
                bk = lane < nw ? s_k[lane] : -1; brid = lane < nw ? s_r[lane] : LLONG_MAX; brow = lane < nw ? s_p[lane] : -1;
                const int src = warp_argbest(bk, brid);
                bk = src >= 0 ? __shfl_sync(0xffffffffu, bk, src) : -1;
                brid = src >= 0 ? __shfl_sync(0xffffffffu, brid, src) : LLONG_MAX;
                brow = src >= 0 ? __shfl_sync(0xffffffffu, brow, src) : -1;
                const T v = (lane < w && brow >= 0) ? (CL ? s_wc[src * MC_PW + lane] : S[lane * per + brow]) : VT<T>::zero();
                const long long pos = brow >= 0 ? r_lo + brow : -1;
                if constexpr (CL) {
                    McSlot<T> *dst = cg::this_cluster().map_shared_rank(cs + par * MC_CMAX + b, warp);
                    if (lane < w) dst->v[lane] = v;
                    if (lane == 0) { dst->key = bk; dst->rid = brid; dst->pos = pos; }
                } else {
                    McSlot<T> *my = gslots + (size_t)par * G + b;
                    if (lane < w) my->v[lane] = v;
                    if (lane == 0) { my->key = bk; my->rid = brid; my->pos = pos; }
                    __syncwarp();
                    if (lane == 0) {
                        red_release_add_u32(sync + 1, 1u);
                        const unsigned target = (unsigned)G * (unsigned)(j + 1);
                        unsigned it = 0;
                        while (ld_acquire_u32(sync + 1) < target && ++it < MC_SPIN) {}
                        if (it >= MC_SPIN) s_wait = 1;
                    }
                }
            }
            // 2. the barrier, then the same winner in every warp
            long long gk = -1, gr = LLONG_MAX, gp = -1;
            int gq = -1;
            const T *wv;                                 // the winner's panel values
            if constexpr (CL) {
                asm volatile("barrier.cluster.arrive.release;" ::: "memory");
                // while the other CTAs arrive: the previous pivot's update of this row's later columns
                if (mine && kk >= 1) {
                    const T l = S[(kk - 1) * per + tid];
                    for (int c = kk + 1; c < w; c++) S[c * per + tid] = sub(S[c * per + tid], mul(l, Lb[(kk - 1) * MC_LB + c]));
                }
                asm volatile("barrier.cluster.wait.acquire;" ::: "memory");
                if (lane < G) {
                    const McSlot<T> *c = cs + par * MC_CMAX + lane;
                    gk = c->key; gr = c->rid; gp = c->pos; gq = lane;
                }
                const int src = warp_argbest(gk, gr);
                gp = src >= 0 ? __shfl_sync(0xffffffffu, gp, src) : -1;
                gq = src >= 0 ? __shfl_sync(0xffffffffu, gq, src) : -1;
                gk = src >= 0 ? __shfl_sync(0xffffffffu, gk, src) : -1;
                wv = gq >= 0 ? cs[par * MC_CMAX + gq].v : Lb + kk * MC_LB;
            } else {
                __syncthreads();
                if (tid < G && !s_wait) {
                    const McSlot<T> *c = gslots + (size_t)par * G + tid;
                    gk = __ldcg(&c->key); gr = __ldcg(&c->rid); gp = __ldcg(&c->pos); gq = tid;
                }
                {
                    const int src = warp_argbest(gk, gr);
                    gk = src >= 0 ? __shfl_sync(0xffffffffu, gk, src) : -1;
                    gr = src >= 0 ? __shfl_sync(0xffffffffu, gr, src) : LLONG_MAX;
                    gp = src >= 0 ? __shfl_sync(0xffffffffu, gp, src) : -1;
                    gq = src >= 0 ? __shfl_sync(0xffffffffu, gq, src) : -1;
                }
                if (lane == 0) { s_k[warp] = gk; s_r[warp] = gr; s_p[warp] = gp; s_q[warp] = gq; }
                __syncthreads();
                gk = lane < nw ? s_k[lane] : -1; gr = lane < nw ? s_r[lane] : LLONG_MAX;
                gp = lane < nw ? s_p[lane] : -1; gq = lane < nw ? s_q[lane] : -1;
                const int src = warp_argbest(gk, gr);
                gp = src >= 0 ? __shfl_sync(0xffffffffu, gp, src) : -1;
                gq = src >= 0 ? __shfl_sync(0xffffffffu, gq, src) : -1;
                gk = src >= 0 ? __shfl_sync(0xffffffffu, gk, src) : -1;
                // warp 0 brings the winner's values into Lb for every warp
                if (warp == 0 && lane < w)
                    Lb[kk * MC_LB + lane] = gq >= 0 ? ldcg_v(&gslots[(size_t)par * G + gq].v[lane]) : VT<T>::zero();
                __syncthreads();
                wv = Lb + kk * MC_LB;
            }
            const T pv = gq >= 0 ? wv[kk] : VT<T>::zero();
            // the decision, the same in every thread
            const double t = s_thr[kk];
            int stop = 0;
            if (!CL && s_wait) stop = 2;
            else if (gp < 0 || gk <= 0 || ((unsigned long long)gk < pivkey_of_modulus<T>(2.0 * t) && vabs(pv) < t)) stop = 1;
            else if (gp >= nri) stop = 3;
            if (tid == 0) {
                if (stop == 2) set_status(st, ST_WAIT, front, 0.0, 0.0);
                else if (stop == 1 && b == 0) set_status(st, ST_SINGULAR, fcol + j, gp >= 0 ? vabs(pv) : 0.0, t);
                else if (stop == 3 && b == 0) set_status(st, ST_BORDER, front, vabs(pv), t);
                if (!stop) { if (b == 0) chosen[j] = gp; s_piv[kk] = (int)gp; }
            }
            if (stop) { stopped = true; break; }
            if constexpr (CL) {             // every warp keeps the winner's row (the same values) for its deferred update
                if (lane < w) Lb[kk * MC_LB + lane] = wv[lane];
                __syncwarp();
            }
            // 3. this thread's row: the pivot row leaves the search; a live row takes its multiplier and the update of
            // the panel's later columns
            if (mine) {
                if (r_lo + tid == gp) mine = false;
                else {
                    const T inv = recip(pv);
                    const T l = mul(S[kk * per + tid], inv);
                    S[kk * per + tid] = l;
                    if constexpr (CL) {         // the next column now; the others during the next column's barrier
                        if (kk + 1 < w) S[(kk + 1) * per + tid] = sub(S[(kk + 1) * per + tid], mul(l, wv[kk + 1]));
                    } else {
#pragma unroll 4
                        for (int c = kk + 1; c < w; c++) S[c * per + tid] = sub(S[c * per + tid], mul(l, wv[c]));
                    }
                }
            }
        }
        if (tid < per) live[tid] = mine ? 1 : 0;
        if (stopped) break;
        __syncthreads();
        for (int e = tid; e < w * nmine; e += MC_THREADS) {
            const int c = e / nmine, r = e - c * nmine;
            W[(r_lo + r) + (int64_t)(p0 + c) * ld] = S[c * per + r];
        }
        // the trailing columns [p0 + w, npiv) by chunks
        for (int c0 = p0 + w; c0 < npiv; c0 += CW) {
            const int cw = npiv - c0 < CW ? npiv - c0 : CW;
            for (int e0 = tid; e0 < w * cw; e0 += 8 * MC_THREADS) {        // eight loads in flight per thread
                T u[8];
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    const int e = e0 + q * MC_THREADS;
                    u[q] = e < w * cw ? ldcg_v(W + s_piv[e % w] + (int64_t)(c0 + e / w) * ld) : VT<T>::zero();
                }
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    const int e = e0 + q * MC_THREADS;
                    if (e < w * cw) Uc[(e % w) * CW + e / w] = u[q];
                }
            }
            __syncthreads();
            // U12 = L11^-1 A12: a thread per column, 8-row blocks in registers (the order of a forward substitution)
            for (int c = tid; c < cw; c += MC_THREADS) {
                for (int r0 = 0; r0 < w; r0 += 8) {
                    T y[8];
#pragma unroll
                    for (int q = 0; q < 8; q++) y[q] = r0 + q < w ? Uc[(r0 + q) * CW + c] : VT<T>::zero();
                    for (int i = 0; i < r0; i++) {
                        const T xi = Uc[i * CW + c];
#pragma unroll
                        for (int q = 0; q < 8; q++) y[q] = sub(y[q], mul(Lb[(r0 + q) * MC_LB + i], xi));
                    }
#pragma unroll
                    for (int q = 1; q < 8; q++)
#pragma unroll
                        for (int qq = 0; qq < q; qq++) y[q] = sub(y[q], mul(Lb[(r0 + q) * MC_LB + r0 + qq], y[qq]));
#pragma unroll
                    for (int q = 0; q < 8; q++) if (r0 + q < w) Uc[(r0 + q) * CW + c] = y[q];
                }
            }
            __syncthreads();
            if (b == (c0 / CW) % G)
                for (int e = tid; e < w * cw; e += MC_THREADS) {
                    const int k = e % w, c = e / w;
                    Ub[(p0 + k) + (int64_t)(c0 + c) * npiv] = Uc[k * CW + c];
                }
            // A22 -= L21 U12 on this CTA's live rows: 4 x 4 tiles per thread
            const int tr = (nmine + 3) >> 2, tc = (cw + 3) >> 2;
            for (int t = tid; t < tr * tc; t += MC_THREADS) {
                const int rb = (t % tr) * 4, cb = (t / tr) * 4;
                T acc[4][4];
#pragma unroll
                for (int a = 0; a < 4; a++)
#pragma unroll
                    for (int q = 0; q < 4; q++) acc[a][q] = VT<T>::zero();
                for (int k = 0; k < w; k++) {
                    T lv[4], uv[4];
#pragma unroll
                    for (int a = 0; a < 4; a++) lv[a] = rb + a < nmine ? S[k * per + rb + a] : VT<T>::zero();
#pragma unroll
                    for (int q = 0; q < 4; q++) uv[q] = cb + q < cw ? Uc[k * CW + cb + q] : VT<T>::zero();
#pragma unroll
                    for (int a = 0; a < 4; a++)
#pragma unroll
                        for (int q = 0; q < 4; q++) acc[a][q] = add(acc[a][q], mul(lv[a], uv[q]));
                }
#pragma unroll
                for (int a = 0; a < 4; a++) {
                    const int r = rb + a;
                    if (r >= nmine || !live[r]) continue;
#pragma unroll
                    for (int q = 0; q < 4; q++)
                        if (cb + q < cw) {
                            T *x = W + (r_lo + r) + (int64_t)(c0 + cb + q) * ld;
                            *x = sub(*x, acc[a][q]);
                        }
                }
            }
            __syncthreads();
        }
    }
    __syncthreads();
    if constexpr (CL) {
        cg::this_cluster().sync();            // no CTA leaves while another may still write its shared memory
    } else if (tid == 0) {
        __threadfence();
        if (atomicAdd(sync, 1u) == (unsigned)(G - 1)) {   // the last CTA out resets the counter and the ticket
            sync[1] = 0u;
            __threadfence();
            sync[0] = 0u;
        }
    }
}

// After k_block_lu_mc (one CTA of 1024 threads): the final row order of the front (the pivot rows in step order, then
// the other rows in their order) into perm, the front's row ids in that order, and the pivot rows' rows of B into p_lu.
// mark / rid_tmp: scratch of nrows entries.
template <typename T>
__global__ void __launch_bounds__(1024) k_mc_order(int nrows, int npr, const int64_t *__restrict__ chosen,
                                                   int64_t *__restrict__ rowid, int *__restrict__ perm, int64_t f,
                                                   int64_t *__restrict__ p_lu, int *__restrict__ mark,
                                                   int64_t *__restrict__ rid_tmp, const DevStatus *st)
{
    __shared__ int s_cnt[1024];
    if (st->code) return;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int i = tid; i < nrows; i += nt) mark[i] = -1;
    __syncthreads();
    for (int k = tid; k < npr; k += nt) mark[chosen[k]] = k;
    __syncthreads();
    const int seg = (nrows + nt - 1) / nt, lo = tid * seg < nrows ? tid * seg : nrows, hi = lo + seg < nrows ? lo + seg : nrows;
    int cnt = 0;
    for (int i = lo; i < hi; i++) cnt += mark[i] < 0;
    s_cnt[tid] = cnt;
    __syncthreads();
    for (int o = 1; o < nt; o <<= 1) {              // inclusive scan of the counts
        const int v = tid >= o ? s_cnt[tid - o] : 0;
        __syncthreads();
        s_cnt[tid] += v;
        __syncthreads();
    }
    int pos = npr + s_cnt[tid] - cnt;
    for (int i = lo; i < hi; i++) {
        const int k = mark[i] < 0 ? pos++ : mark[i];
        perm[k] = i;
        rid_tmp[k] = rowid[i];
    }
    __syncthreads();
    for (int k = tid; k < nrows; k += nt) {
        rowid[k] = rid_tmp[k];
        if (k < npr) p_lu[f + k] = rid_tmp[k];
    }
}

// the pivot block in the final row order into the arena: row k of L \ U takes W's row perm[k], except the pivot rows'
// entries right of their own panel, which are U12 (Ub)
template <typename T>
__global__ void k_mc_lout(const T *__restrict__ W, int64_t ld, int64_t nrows, int64_t npiv, int64_t npr,
                          const int *__restrict__ perm, const T *__restrict__ Ub, T *__restrict__ Lout, const DevStatus *st)
{
    if (st->code) return;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nrows * npiv; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = e % nrows, c = e / nrows;
        const int64_t pend = k < npr ? ((k / MC_PW + 1) * MC_PW < npr ? (k / MC_PW + 1) * MC_PW : npr) : 0;
        Lout[e] = (k < npr && c >= pend) ? Ub[k + c * npiv] : W[perm[k] + c * ld];
    }
}

// apply the recorded swaps ipiv[k0 .. k0 + cnt) in order to the columns [c0, c1)
template <typename T>
__global__ void k_laswp(T *__restrict__ W, int64_t ld, const int *__restrict__ ipiv, int k0, int cnt, int64_t c0, int64_t c1,
                        const DevStatus *st)
{
    if (st->code) return;
    for (int64_t c = c0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < c1; c += (int64_t)gridDim.x * blockDim.x) {
        T *col = W + c * ld;
        for (int k = 0; k < cnt; k++) {
            const int64_t j = k0 + k, p = ipiv[j];
            if (p < 0 || p >= ld) continue;       // never written by a panel that stopped: skip
            if (p != j) { T t = col[j]; col[j] = col[p]; col[p] = t; }
        }
    }
}

// X <- L^-1 X for the unit lower w x w block L = W[k0.., k0..] and X = rows [k0, k0 + w) of columns [c0, c1)
template <typename T>
__global__ void __launch_bounds__(128) k_trsm_unit(T *__restrict__ W, int64_t ld, int k0, int w, int64_t c0, int64_t c1,
                                                   const DevStatus *st)
{
    __shared__ T sL[32][33];
    if (st->code) return;
    for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
        int r = e % w, c = e / w;
        sL[r][c] = W[(k0 + r) + (int64_t)(k0 + c) * ld];
    }
    __syncthreads();
    for (int64_t c = c0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < c1; c += (int64_t)gridDim.x * blockDim.x) {
        T x[32];
        T *col = W + k0 + c * ld;
#pragma unroll
        for (int i = 0; i < 32; i++) if (i < w) x[i] = col[i];
#pragma unroll
        for (int i = 0; i < 32; i++) {
            if (i >= w) break;
#pragma unroll
            for (int r = i + 1; r < 32; r++) if (r < w) x[r] = sub(x[r], mul(sL[r][i], x[i]));
        }
#pragma unroll
        for (int i = 0; i < 32; i++) if (i < w) col[i] = x[i];
    }
}

// ---------------------------------------------------------------------------------------------------------------------
// Cout <- Cin - A B (column-major; M x K times K x N; Cin's rows optionally gathered through rmap) on the FP64 tensor cores: mma.sync m8n8k4 f64 (DMMA).  64 x 64 block
// tiles, 16-deep K slices staged in shared memory, 8 warps of 32 x 16.  Complex: four real products per complex one
// (Cr += Ar Br - Ai Bi, Ci += Ar Bi + Ai Br), the minus folded into a negated copy of Bi.
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}

constexpr int GBM = 64, GBN = 64, GBK = 16, GPAD = 68, GBP = 20;   // A staged [k][m] (row 68), B staged [n][k] (row 20)

template <typename T>
__global__ void __launch_bounds__(256) k_gemm_sub(int64_t M, int64_t N, int64_t K, const T *__restrict__ A, int64_t lda,
                                                 const T *__restrict__ B, int64_t ldb, const T *Cin, int64_t ldci,
                                                 const int *__restrict__ rmap, T *Cout, int64_t ldco, const DevStatus *st,
                                                 OutMap om)
{
    constexpr bool CP = VT<T>::cplx_;
    __shared__ double As[CP ? 2 : 1][GBK][GPAD];
    __shared__ double Bs[CP ? 3 : 1][GBN][GBP];
    if (st->code) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 1, wn = warp >> 1;
    const int64_t m0 = (int64_t)blockIdx.x * GBM, n0 = (int64_t)blockIdx.y * GBN;
    double acc[CP ? 2 : 1][4][2][2];
#pragma unroll
    for (int z = 0; z < (CP ? 2 : 1); z++)
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
            for (int b = 0; b < 2; b++) { acc[z][a][b][0] = 0.0; acc[z][a][b][1] = 0.0; }
    // the next K slice is loaded into registers while the current one is multiplied
    T pa[4], pb[4];
    auto load_slice = [&](int64_t k0) {
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int m = tid & 63, k = (tid >> 6) + 4 * i;
            const int64_t gm = m0 + m, gk = k0 + k;
            pa[i] = (gm < M && gk < K) ? A[gm + gk * lda] : VT<T>::zero();
        }
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int k = tid & 15, nn = (tid >> 4) + 16 * i;
            const int64_t gk = k0 + k, gn = n0 + nn;
            pb[i] = (gk < K && gn < N) ? B[gk + gn * ldb] : VT<T>::zero();
        }
    };
    load_slice(0);
    for (int64_t k0 = 0; k0 < K; k0 += GBK) {
        // stage A (64 x 16) and B (16 x 64) from the registers, then load the next slice
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int m = tid & 63, k = (tid >> 6) + 4 * i;
            const T v = pa[i];
            if constexpr (CP) { As[0][k][m] = v.x; As[1][k][m] = v.y; } else As[0][k][m] = v;
        }
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int k = tid & 15, nn = (tid >> 4) + 16 * i;
            const T v = pb[i];
            if constexpr (CP) { Bs[0][nn][k] = v.x; Bs[1][nn][k] = v.y; Bs[2][nn][k] = -v.y; } else Bs[0][nn][k] = v;
        }
        __syncthreads();
        if (k0 + GBK < K) load_slice(k0 + GBK);
#pragma unroll
        for (int ks = 0; ks < GBK; ks += 4) {
            const int kr = ks + (lane & 3);
            double ar[4], ai[4], br[2], bi[2], bn[2];
#pragma unroll
            for (int a = 0; a < 4; a++) {
                const int m = wm * 32 + a * 8 + (lane >> 2);
                ar[a] = As[0][kr][m];
                if constexpr (CP) ai[a] = As[1][kr][m];
            }
#pragma unroll
            for (int b = 0; b < 2; b++) {
                const int nn = wn * 16 + b * 8 + (lane >> 2);
                br[b] = Bs[0][nn][kr];
                if constexpr (CP) { bi[b] = Bs[1][nn][kr]; bn[b] = Bs[2][nn][kr]; }
            }
#pragma unroll
            for (int a = 0; a < 4; a++)
#pragma unroll
                for (int b = 0; b < 2; b++) {
                    dmma(acc[0][a][b][0], acc[0][a][b][1], ar[a], br[b]);
                    if constexpr (CP) {
                        dmma(acc[0][a][b][0], acc[0][a][b][1], ai[a], bn[b]);
                        dmma(acc[1][a][b][0], acc[1][a][b][1], ar[a], bi[b]);
                        dmma(acc[1][a][b][0], acc[1][a][b][1], ai[a], br[b]);
                    }
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 2; b++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int64_t gm = m0 + wm * 32 + a * 8 + (lane >> 2);
                const int64_t gn = n0 + wn * 16 + b * 8 + 2 * (lane & 3) + h;
                if (gm < M && gn < N) {
                    const int64_t gi = rmap ? (int64_t)rmap[gm] : gm;
                    T v = Cin[gi + gn * ldci];
                    if constexpr (CP) { v.x -= acc[0][a][b][h]; v.y -= acc[1][a][b][h]; }
                    else v -= acc[0][a][b][h];
                    if (om.col) Cout[(gm < om.nslot ? om.slot + gm : om.tau + (gm - om.nslot)) + om.col[gn] * ldco] = v;
                    else Cout[gm + gn * ldco] = v;
                }
            }
}



// asynchronous global -> shared copies of one element (cp.async: all of a thread's copies in flight at once; completed
// by cp_async_wait_all, then a barrier).  Both addresses aligned to the element size.
template <typename T> __device__ __forceinline__ void cp_async_el(T *dst, const T *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if constexpr (sizeof(T) == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Programmatic dependent launch: a kernel launched with programmatic stream serialization may start before the kernel
// ahead of it in the stream has finished; pdl_wait() blocks until that kernel has completed and its writes are visible
// (a no-op for a normally launched kernel); pdl_trigger() lets the next such kernel start its own launch.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }


template <typename T> __device__ __forceinline__ T shfl_xor_v(T v, int m);
template <> __device__ __forceinline__ double shfl_xor_v<double>(double v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }
template <> __device__ __forceinline__ cplx shfl_xor_v<cplx>(cplx v, int m)
{
    return cplx{__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m)};
}

template <typename T> __device__ __forceinline__ T shfl_v(T v, int src);
template <> __device__ __forceinline__ double shfl_v<double>(double v, int src) { return __shfl_sync(0xffffffffu, v, src); }
template <> __device__ __forceinline__ cplx shfl_v<cplx>(cplx v, int src)
{
    return cplx{__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src)};
}


// Partial-pivot LU of a front's pivot block in shared memory, with a pivot warp and one-column look-ahead (one CTA of
// up to 1024 threads).  Warp 0 owns the critical path: at step j it updates column j + 1 for every row with the step-j
// multipliers and, in the same pass, finds the pivot of column j + 1 (the largest pivot key, i.e. modulus, ties to the
// smaller row of B), then publishes the row and 1 / pivot (double-buffered slots).  The other warps update columns
// j + 2 .. with the step-j pivot meanwhile, keep the multipliers (double-buffered) and store those of step j - 1 into
// column j - 1 (no longer read by anyone).  One barrier per step.  No row swaps: the pivot row of step j is tagged j.
// The singular test uses the column thresholds staged in shared memory (keys; the modulus itself near the threshold).
// a named barrier for `count` threads (a multiple of 32); the non-aligned form, so that a warp need not be converged
__device__ __forceinline__ void named_bar(int id, int count) { asm volatile("barrier.sync %0, %1;" ::"r"(id), "r"(count) : "memory"); }

// The sources of a front's pivot block when the LU kernel assembles it itself (instead of reading it from the working
// block): the original entries of the pivot columns and the pivot-column part of at most one child's contribution block.
struct PivotAsm {
    int on;                                  // assemble from these sources
    const void *cb;                          // the child's CB (cbr x cbc, column-major), or null
    int64_t cbr, h, nslot, slot, tau_base;   // its rows, its CB columns in the pivot columns (a prefix), row placement
    const int64_t *relcol, *child_rowid;     // the child's CB columns -> local columns; its CB rows' ids
    const int64_t *asrc, *adst;              // original entries: B entry -> offset in the block (column-major, ld nrows)
    int64_t acnt;
    const void *Bx;
    const int64_t *rowinit;                  // the entering rows' ids (-1 for rows from children)
};

// A front's pivot block into shared memory (A: npiv x nrows, column-major, A[c * nrows + i]) with its row ids (rid): read
// from the working block, or (pa.on) assembled here from the original entries and at most one child's contribution
// block.  Every thread of the CTA takes part; the caller synchronises before reading A.
template <typename T>
__device__ __forceinline__ void stage_pivot_block(T *__restrict__ A, int64_t *__restrict__ rid, const T *__restrict__ W, int64_t ld,
                                                  int nrows, int npiv, const int64_t *__restrict__ rowid, const PivotAsm &pa,
                                                  int tid, int nt)
{
    const int ne = npiv * nrows;
    if (!pa.on) {
        pdl_wait();
        // the block from the working block, 8 loads in flight per thread
        for (int e0 = tid; e0 < ne; e0 += 8 * nt) {
            T v[8];
#pragma unroll
            for (int q = 0; q < 8; q++) { const int e = e0 + q * nt; v[q] = e < ne ? W[e % nrows + (int64_t)(e / nrows) * ld] : VT<T>::zero(); }
#pragma unroll
            for (int q = 0; q < 8; q++) { const int e = e0 + q * nt; if (e < ne) A[e] = v[q]; }
        }
        for (int i = tid; i < nrows; i += nt) rid[i] = rowid[i];
    } else {
        // assembled here: zero, the original entries, then the child's CB columns added; the row ids
        for (int e = tid; e < ne; e += nt) A[e] = VT<T>::zero();
        for (int i = tid; i < nrows; i += nt) rid[i] = pa.rowinit[i];
        __syncthreads();
        const T *Bx = reinterpret_cast<const T *>(pa.Bx);
#pragma unroll 4
        for (int64_t e = tid; e < pa.acnt; e += nt) A[pa.adst[e]] = Bx[pa.asrc[e]];
        pdl_wait();                                   // the child's CB columns (the launch before) are written
        for (int64_t t = tid; t < pa.nslot; t += nt) rid[pa.slot + t] = pa.child_rowid[t];
        __syncthreads();
        const T *cb = reinterpret_cast<const T *>(pa.cb);
        // the CB's pivot-column part is at most nrows x npiv entries: 32-bit index arithmetic
        const int cbr = (int)pa.cbr, tot = (int)(pa.cbr * pa.h), nsl = (int)pa.nslot, sl = (int)pa.slot, tb = (int)pa.tau_base;
#pragma unroll 4
        for (int e = tid; e < tot; e += nt) {
            const int c = e / cbr, t = e - c * cbr;
            const int pr = t < nsl ? sl + t : tb + (t - nsl);
            T *a = A + (int)pa.relcol[c] * nrows + pr;
            *a = add(*a, cb[t + (int64_t)c * cbr]);
        }
    }
}

template <typename T>
__device__ __forceinline__ void front_lu2_body(const T *__restrict__ W, int64_t ld, int nrows, int npiv, int nri,
                                               int64_t fcol, const double *__restrict__ colmax, double pivot_rel,
                                               int64_t *__restrict__ rowid, T *__restrict__ Lout, int *__restrict__ perm,
                                               int64_t *__restrict__ p_lu, DevStatus *st, int64_t front, const PivotAsm &pa)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *A = reinterpret_cast<T *>(smem_raw);                        // npiv x nrows, column-major: A[c * nrows + i]
    T *lcol = A + (size_t)npiv * nrows;                            // 2 x nrows: multipliers of steps j (j & 1)
    int64_t *rid = reinterpret_cast<int64_t *>(lcol + 2 * nrows);
    double *thr = reinterpret_cast<double *>(rid + nrows);         // npiv: pivot_rel * max |B(:, column)|
    unsigned long long *thk = reinterpret_cast<unsigned long long *>(thr + npiv);   // npiv: the pivot key of 2 thr
    int *tag = reinterpret_cast<int *>(thk + npiv);
    int *pos = tag + nrows;
    __shared__ int s_bi[2], s_stv[2], s_stop;                      // s_stv: the stop decision of steps j (j & 1)
    __shared__ T s_inv[2];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nt = blockDim.x;
    const int ne = npiv * nrows;
    stage_pivot_block<T>(A, rid, W, ld, nrows, npiv, rowid, pa, tid, nt);
    for (int i = tid; i < nrows; i += nt) tag[i] = INT_MAX;
    for (int c = tid; c < npiv; c += nt) { thr[c] = pivot_rel * colmax[fcol + c]; thk[c] = pivkey_of_modulus<T>(2.0 * thr[c]); }
    if (tid == 0) s_stop = st->code != 0 ? 3 : 0;
    __syncthreads();
    if (s_stop) return;
    // The SM sub-partition of warp w is w % 4: sub-partition 0 is left to the pivot warp (warps 4, 8, ... leave here),
    // the update warps run on the other three.  The steps synchronise the remaining warps with a named barrier.
    if ((warp & 3) == 0 && warp != 0) return;
    const int nwarp = nt >> 5, nuw = (nwarp - 1) - (nwarp - 1) / 4;
    const int nact = 32 * (1 + nuw);                                // the pivot warp and the update warps
    const int uw = warp == 0 ? -1 : (warp >> 2) * 3 + (warp & 3) - 1;
    const int at = (uw + 1) * 32 + lane;                            // index among the remaining threads
    const int nu = 32 * nuw, ut = warp == 0 ? -1 : uw * 32 + lane;  // update threads
    const int R = (nrows + 31) & ~31;
    const int G = nu >= R ? nu / R : 1, rstep = nu >= R ? R : nu;
    const int my_i = ut >= 0 ? (nu >= R ? ut % R : ut) : 0, my_g = ut >= 0 ? (nu >= R ? ut / R : 0) : G;
    const bool upd = ut >= 0 && my_g < G;
    // The singular test of the reference (FPLUS src/factor_sn_panel.inc:232-233): no candidate, a zero modulus, or a
    // modulus below t = pivot_rel * max |B(:, column)|.  A key at or above the key of 2t (tk, staged) is clear of the
    // threshold; below it the modulus itself is compared.
    auto singular = [&](int bi, unsigned long long key, double t, unsigned long long tk, T pv) -> bool {
        if (bi < 0 || key == 0ull) return true;
        return key < tk && vabs(pv) < t;
    };
    // warp 0: decide on the winner (bi, pivot key) of column j, publish into slot
    auto decide = [&](int j, int bi, unsigned long long key, int slot) {
        if (lane != 0) return;
        const double t = thr[j];
        int stop = 0;
        const T pv = bi >= 0 ? A[(size_t)j * nrows + bi] : VT<T>::zero();
        if (singular(bi, key, t, thk[j], pv)) { set_status(st, ST_SINGULAR, fcol + j, bi >= 0 ? vabs(pv) : 0.0, t); stop = 1; }
        else if (bi >= nri) { set_status(st, ST_BORDER, front, vabs(pv), t); stop = 1; }
        s_bi[slot] = bi;
        s_stv[slot] = stop;
        if (!stop) { s_inv[slot] = recip(pv); tag[bi] = j; }
        else s_stop = 1;
    };
    // the warp's winner: the largest key, ties to the smaller row of B
    auto reduce = [&](unsigned long long bk, int bi, int64_t br, unsigned long long *key_out) -> int {
        const unsigned long long key = bi >= 0 ? bk : 0ull;
        const unsigned long long m = warp_max_key(key);
        unsigned cand = __ballot_sync(0xffffffffu, bi >= 0 && key == m);
        *key_out = m;
        if (cand == 0) return -1;
        if ((cand & (cand - 1)) != 0) {
            int64_t rr = (cand >> lane) & 1u ? br : INT64_MAX;
            for (int o = 16; o > 0; o >>= 1) { int64_t t = __shfl_xor_sync(0xffffffffu, rr, o); rr = t < rr ? t : rr; }
            cand = __ballot_sync(0xffffffffu, ((cand >> lane) & 1u) && br == rr);
        }
        return __shfl_sync(0xffffffffu, bi, __ffs(cand) - 1);
    };
    if (warp == 0 && nrows <= 128) {
        // the pivot warp with its rows' state in registers (4 row slots per lane): row ids, not-yet-pivoted flags, and
        // its own copy of the running column (it computes column j + 1 at step j and uses it as column j at step j + 1)
        T xc[4];
        int64_t rr[4];
        bool al[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int i = lane + 32 * q;
            al[q] = i < nrows;
            rr[q] = al[q] ? rid[i] : INT64_MAX;
            xc[q] = al[q] ? A[i] : VT<T>::zero();
        }
        // the warp's winner among the live slots; every lane also forms 1 / its own candidate while the reduction runs,
        // and the winner's reciprocal comes back with its value
        auto pick = [&](const T *xv, unsigned long long *m, T *pv, T *pinv) -> int {
            long long bk = -1; int wi = -1; int64_t br = INT64_MAX; T bx = VT<T>::zero();
#pragma unroll
            for (int q = 0; q < 4; q++) {
                if (!al[q]) continue;
                const long long a = (long long)pivkey(xv[q]);       // keys are below 2^63
                if (a > bk || (a == bk && rr[q] < br)) { bk = a; wi = lane + 32 * q; br = rr[q]; bx = xv[q]; }
            }
            const T binv = wi >= 0 && bk > 0 ? recip(bx) : VT<T>::zero();
            const unsigned long long key = wi >= 0 ? (unsigned long long)bk : 0ull;
            const unsigned long long mk = warp_max_key(key);
            unsigned cand = __ballot_sync(0xffffffffu, wi >= 0 && key == mk);
            *m = mk;
            if (cand == 0) { *pv = VT<T>::zero(); *pinv = VT<T>::zero(); return -1; }
            if ((cand & (cand - 1)) != 0) {
                int64_t r2 = (cand >> lane) & 1u ? br : INT64_MAX;
                for (int o = 16; o > 0; o >>= 1) { int64_t t = __shfl_xor_sync(0xffffffffu, r2, o); r2 = t < r2 ? t : r2; }
                cand = __ballot_sync(0xffffffffu, ((cand >> lane) & 1u) && br == r2);
            }
            const int wl = __ffs(cand) - 1;
            *pv = shfl_v<T>(bx, wl);
            *pinv = shfl_v<T>(binv, wl);
            return __shfl_sync(0xffffffffu, wi, wl);
        };
        // lane 0 decides with the winner's value pv and its reciprocal pinv (held by every lane)
        auto decide_v = [&](int j, int bi, unsigned long long key, int slot, T pv, T pinv) -> T {
            if (lane == 0) {
                const double t = thr[j];
                int stop = 0;
                if (singular(bi, key, t, thk[j], pv)) { set_status(st, ST_SINGULAR, fcol + j, bi >= 0 ? vabs(pv) : 0.0, t); stop = 1; }
                else if (bi >= nri) { set_status(st, ST_BORDER, front, vabs(pv), t); stop = 1; }
                s_bi[slot] = bi;
                s_stv[slot] = stop;
                if (!stop) { s_inv[slot] = pinv; tag[bi] = j; }
            }
            return pinv;
        };
        unsigned long long m;
        T pv, pinv;
        int bi = pick(xc, &m, &pv, &pinv);
        T inv = decide_v(0, bi, m, 0, pv, pinv);
#pragma unroll
        for (int q = 0; q < 4; q++) al[q] = al[q] && lane + 32 * q != bi;
        __syncwarp();
        named_bar(1, nact);
        for (int j = 0; j < npiv; j++) {
            if (s_stv[j & 1]) return;                               // decided before the last barrier, seen by all
            if (j + 1 < npiv) {
                T *cn = A + (size_t)(j + 1) * nrows;
                const T pr = cn[bi];
                T xb[4];
#pragma unroll
                for (int q = 0; q < 4; q++) xb[q] = al[q] ? cn[lane + 32 * q] : VT<T>::zero();
#pragma unroll
                for (int q = 0; q < 4; q++) xb[q] = sub(xb[q], mul(mul(xc[q], inv), pr));
#pragma unroll
                for (int q = 0; q < 4; q++) if (al[q]) cn[lane + 32 * q] = xb[q];
                const int w = pick(xb, &m, &pv, &pinv);
                inv = decide_v(j + 1, w, m, (j + 1) & 1, pv, pinv);
#pragma unroll
                for (int q = 0; q < 4; q++) { xc[q] = xb[q]; al[q] = al[q] && lane + 32 * q != w; }
                bi = w;
                __syncwarp();
            }
            named_bar(1, nact);
        }
    } else if (warp == 0) {
        {
            long long bk = -1; int bi = -1; int64_t br = INT64_MAX;
            for (int i = lane; i < nrows; i += 32) {
                const long long a = (long long)pivkey(A[i]);
                const int64_t r = rid[i];
                if (a > bk || (a == bk && r < br)) { bk = a; bi = i; br = r; }
            }
            unsigned long long m;
            const int w = reduce((unsigned long long)bk, bi, br, &m);
            decide(0, w, m, 0);
            __syncwarp();
        }
        named_bar(1, nact);
        for (int j = 0; j < npiv; j++) {
            if (s_stv[j & 1]) return;
            const int bi = s_bi[j & 1];
            const T inv = s_inv[j & 1];
            if (j + 1 < npiv) {
                // column j + 1 for every row not yet pivoted, and its pivot, in one pass: the row slots of a lane are
                // independent (loads first, then the arithmetic), 4 slots per round
                const T pr = A[(size_t)(j + 1) * nrows + bi];
                const T *cj = A + (size_t)j * nrows;
                T *cn = A + (size_t)(j + 1) * nrows;
                long long bk = -1; int wi = -1; int64_t br = INT64_MAX;
                for (int i0 = lane; i0 < nrows; i0 += 128) {
                    T xa[4], xb[4];
                    bool ok[4];
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const int i = i0 + 32 * q;
                        ok[q] = i < nrows && tag[i] > j;
                        xa[q] = ok[q] ? cj[i] : VT<T>::zero();
                        xb[q] = ok[q] ? cn[i] : VT<T>::zero();
                    }
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const T x = sub(xb[q], mul(mul(xa[q], inv), pr));
                        xb[q] = x;
                    }
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const int i = i0 + 32 * q;
                        if (ok[q]) {
                            cn[i] = xb[q];
                            const long long a = (long long)pivkey(xb[q]);
                            const int64_t r = rid[i];
                            if (a > bk || (a == bk && r < br)) { bk = a; wi = i; br = r; }
                        }
                    }
                }
                unsigned long long m;
                const int w = reduce((unsigned long long)bk, wi, br, &m);
                decide(j + 1, w, m, (j + 1) & 1);
                __syncwarp();
            }
            named_bar(1, nact);
        }
    } else {
        named_bar(1, nact);
        for (int j = 0; j < npiv; j++) {
            if (s_stv[j & 1]) return;
            const int bi = s_bi[j & 1];
            const T inv = s_inv[j & 1];
            if (upd) {
                T *lc = lcol + (j & 1) * nrows;
                const T *lp = lcol + ((j + 1) & 1) * nrows;
                // (32-bit offsets, one per column for the row and the pivot row; a - l p in fused multiply-adds)
                const int gs = G * nrows;                             // from one of this thread's columns to the next
                for (int i = my_i; i < nrows; i += rstep) {
                    if (my_g == 0 && j > 0 && tag[i] >= j) A[(j - 1) * nrows + i] = lp[i];   // step j - 1's multiplier
                    if (tag[i] <= j) continue;
                    const T l = mul(A[j * nrows + i], inv);
                    if (my_g == 0) lc[i] = l;
                    int c = j + 2 + my_g;
                    T *xa = A + c * nrows + i;
                    const T *pa_ = A + c * nrows + bi;
                    for (; c + 3 * G < npiv; c += 4 * G, xa += 4 * gs, pa_ += 4 * gs) {   // 4 independent columns, loads first
                        T xv[4], pv[4];
#pragma unroll
                        for (int q = 0; q < 4; q++) { xv[q] = xa[q * gs]; pv[q] = pa_[q * gs]; }
#pragma unroll
                        for (int q = 0; q < 4; q++) xa[q * gs] = msub(xv[q], l, pv[q]);
                    }
                    for (; c < npiv; c += G, xa += gs, pa_ += gs) *xa = msub(*xa, l, *pa_);
                }
            }
            named_bar(1, nact);
        }
    }
    // the last step's multipliers
    if (upd && my_g == 0 && npiv > 0) {
        const T *lp = lcol + ((npiv - 1) & 1) * nrows;
        for (int i = my_i; i < nrows; i += rstep) if (tag[i] >= npiv) A[(size_t)(npiv - 1) * nrows + i] = lp[i];
    }
    const int steps = npiv;
    if (warp == 0) {
        int base = steps;
        for (int i0 = 0; i0 < nrows; i0 += 32) {
            const int i = i0 + lane;
            const bool un = i < nrows && tag[i] >= steps;
            const unsigned m = __ballot_sync(0xffffffffu, un);
            if (i < nrows) pos[i] = un ? base + __popc(m & ((1u << lane) - 1u)) : tag[i];
            base += __popc(m);
        }
    }
    named_bar(1, nact);
    for (int i = at; i < nrows; i += nact) {
        const int k = pos[i];
        perm[k] = i;
        rowid[k] = rid[i];
        if (k < steps) p_lu[fcol + k] = rid[i];
    }
    for (int e = at; e < ne; e += nact) { const int i = e % nrows; Lout[pos[i] + (int64_t)(e / nrows) * nrows] = A[e]; }
}

template <typename T>
__global__ void __launch_bounds__(640) k_front_lu2(const T *__restrict__ W, int64_t ld, int nrows, int npiv, int nri,
                                                    int64_t fcol, const double *__restrict__ colmax, double pivot_rel,
                                                    int64_t *__restrict__ rowid, T *__restrict__ Lout, int *__restrict__ perm,
                                                    int64_t *__restrict__ p_lu, DevStatus *st, int64_t front, PivotAsm pa)
{
    front_lu2_body<T>(W, ld, nrows, npiv, nri, fcol, colmax, pivot_rel, rowid, Lout, perm, p_lu, st, front, pa);
}

// Blocked partial-pivot LU of a front's pivot block (nrows <= 128, npiv <= 64; one CTA of 256 threads): 8-column panels
// pivoted by warps 0-3 (thread i < 128 holds row i's eight panel entries in registers; per pivot step every warp posts its
// candidate with the candidate row's panel entries, one 128-thread barrier, and every thread makes the same decision),
// then the panel's pivot rows' U for the later columns by an 8-step forward substitution (a thread per column), then
// the rank-8 update of every later column as FP64 tensor-core products (mma m8n8k4) of the masked multipliers (rows
// already pivoted read zero) and the pivot rows' U.  Rows never move: a row pivoted at step j is tagged j, and the block
// goes out in the final order at the end.  The pivots are those of the step-by-step elimination (the update of a later
// column sums the panel's eight products in another order, so the values agree to rounding).
constexpr int LU5_THREADS = 256, LU5_PB = 8, LU5_LMLD = 132;

template <typename T> struct Lu5Cand {
    unsigned long long key;
    long long rid;
    int row, pad;
    T val, inv;
    T u[LU5_PB];
};

// dynamic shared memory: the block, row ids, thresholds and their keys, the masked multipliers (two planes for complex),
// the final order
static inline size_t front_lu5_smem(int64_t nrows, int64_t npiv, int64_t vs)
{
    return (size_t)(nrows * npiv * vs + nrows * 8 + npiv * 16 + (vs / 8) * LU5_PB * LU5_LMLD * 8 + nrows * 4);
}

template <typename T>
__device__ __forceinline__ void front_lu5_body(const T *__restrict__ W, int64_t ld, int nrows, int npiv, int nri,
                                               int64_t fcol, const double *__restrict__ colmax, double pivot_rel,
                                               int64_t *__restrict__ rowid, T *__restrict__ Lout, int *__restrict__ perm,
                                               int64_t *__restrict__ p_lu, DevStatus *st, int64_t front, const PivotAsm &pa)
{
    constexpr bool CP = VT<T>::cplx_;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *A = reinterpret_cast<T *>(smem_raw);                        // npiv x nrows, column-major: A[c * nrows + i]
    int64_t *rid = reinterpret_cast<int64_t *>(A + (size_t)npiv * nrows);
    double *thr = reinterpret_cast<double *>(rid + nrows);
    unsigned long long *thk = reinterpret_cast<unsigned long long *>(thr + npiv);
    double *Lmr = reinterpret_cast<double *>(thk + npiv);         // masked multipliers: Lm[k][row] at k * LU5_LMLD + row
    double *Lmi = Lmr + (CP ? LU5_PB * LU5_LMLD : 0);
    int *sperm = reinterpret_cast<int *>(Lmr + (CP ? 2 : 1) * LU5_PB * LU5_LMLD);
    __shared__ Lu5Cand<T> cand[2][4];
    __shared__ int prow[LU5_PB], s_stop, wcnt[4];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_stop = st->code != 0;
    stage_pivot_block<T>(A, rid, W, ld, nrows, npiv, rowid, pa, tid, LU5_THREADS);
    for (int c = tid; c < npiv; c += LU5_THREADS) {
        thr[c] = pivot_rel * colmax[fcol + c];
        thk[c] = pivkey_of_modulus<T>(2.0 * thr[c]);
    }
    __syncthreads();
    if (s_stop) return;
    const bool pg = tid < 128;                                     // the panel group: thread i holds row i
    const int i = tid;
    const long long myrid = pg && i < nrows ? (long long)rid[i] : LLONG_MAX;
    bool live = pg && i < nrows;
    int mytag = INT_MAX;
    for (int c0 = 0; c0 < npiv; c0 += LU5_PB) {
        const int w = npiv - c0 < LU5_PB ? npiv - c0 : LU5_PB;   // pivot steps of this panel
        if (pg) {
            T pv[LU5_PB];
#pragma unroll
            for (int s = 0; s < LU5_PB; s++) pv[s] = i < nrows && s < w ? A[(c0 + s) * nrows + i] : VT<T>::zero();
#pragma unroll
            for (int s = 0; s < LU5_PB; s++) {
                if (s >= w) break;
                const int par = s & 1, j = c0 + s;
                // this warp's candidate for column j, posted with its row's panel entries
                const unsigned long long key = live ? pivkey(pv[s]) : 0ull;
                const T xinv = key != 0ull ? recip(pv[s]) : VT<T>::zero();
                const unsigned long long mk = warp_max_key(key);
                unsigned cnd = __ballot_sync(0xffffffffu, key != 0ull && key == mk);
                if (cnd != 0u && (cnd & (cnd - 1u)) != 0u) {
                    long long r2 = (cnd >> lane) & 1u ? myrid : LLONG_MAX;
                    for (int o = 16; o > 0; o >>= 1) { const long long t = __shfl_xor_sync(0xffffffffu, r2, o); r2 = t < r2 ? t : r2; }
                    cnd = __ballot_sync(0xffffffffu, ((cnd >> lane) & 1u) && myrid == r2);
                }
                const int wl = cnd != 0u ? __ffs(cnd) - 1 : 0;
                if (lane == wl) {
                    Lu5Cand<T> &cd = cand[par][warp];
                    cd.key = cnd != 0u ? mk : 0ull; cd.rid = cnd != 0u ? myrid : LLONG_MAX; cd.row = cnd != 0u ? i : -1;
                    cd.val = pv[s]; cd.inv = xinv;
#pragma unroll
                    for (int q = 0; q < LU5_PB; q++) cd.u[q] = pv[q];
                }
                named_bar(1, 128);
                // the winner (every thread of the group the same): the largest key, ties to the smaller row of B
                int bs = 0;
                unsigned long long bk = cand[par][0].key;
                long long br = cand[par][0].rid;
#pragma unroll
                for (int q = 1; q < 4; q++) {
                    const unsigned long long k = cand[par][q].key;
                    const long long r = cand[par][q].rid;
                    if (k > bk || (k == bk && r < br)) { bk = k; br = r; bs = q; }
                }
                const int bi = cand[par][bs].row;
                const T pvw = cand[par][bs].val, inv = cand[par][bs].inv;
                int stop = 0;
                if (bi < 0 || bk == 0ull || (bk < thk[j] && vabs(pvw) < thr[j])) stop = 1;
                else if (bi >= nri) stop = 2;
                if (stop) {
                    if (tid == 0) {
                        if (stop == 1) set_status(st, ST_SINGULAR, fcol + j, bi >= 0 ? vabs(pvw) : 0.0, thr[j]);
                        else set_status(st, ST_BORDER, front, vabs(pvw), thr[j]);
                        s_stop = 1;
                    }
                    break;                                         // (every thread of the group the same)
                }
                if (i == bi) { mytag = j; live = false; prow[s] = i; }
                if (live) {
                    const T l = mul(pv[s], inv);
                    pv[s] = l;
#pragma unroll
                    for (int q = s + 1; q < LU5_PB; q++) pv[q] = sub(pv[q], mul(l, cand[par][bs].u[q]));
                }
            }
            // the panel back into the block; the masked multipliers (zero for every row pivoted so far)
#pragma unroll
            for (int s = 0; s < LU5_PB; s++) {
                if (i < nrows && s < w) A[(c0 + s) * nrows + i] = pv[s];
                const T lm = live && s < w ? pv[s] : VT<T>::zero();
                if constexpr (CP) { Lmr[s * LU5_LMLD + i] = lm.x; Lmi[s * LU5_LMLD + i] = lm.y; } else Lmr[s * LU5_LMLD + i] = lm;
            }
        }
        __syncthreads();
        if (s_stop) return;
        const int t0 = c0 + w, T_ = npiv - t0;                     // the later columns
        if (T_ <= 0) continue;
        // the pivot rows' U for the later columns: forward substitution with the panel's unit-lower L (a thread per column)
        for (int c = t0 + tid; c < npiv; c += LU5_THREADS) {
            T u[LU5_PB];
#pragma unroll
            for (int k = 0; k < LU5_PB; k++) u[k] = k < w ? A[c * nrows + prow[k]] : VT<T>::zero();
#pragma unroll
            for (int k = 1; k < LU5_PB; k++) {
                if (k >= w) break;
                T acc = u[k];
#pragma unroll
                for (int q = 0; q < k; q++) acc = sub(acc, mul(A[(c0 + q) * nrows + prow[k]], u[q]));
                u[k] = acc;
                A[c * nrows + prow[k]] = acc;
            }
        }
        __syncthreads();
        // the rank-w update of every later column on the FP64 tensor cores: A[r, c] -= sum_k Lm[k][r] U[k, c]
        // (item = an 8-row x 8-column fragment; rows already pivoted have zero multipliers and stay as they are)
        {
            const int rf = (nrows + 7) >> 3, cf = (T_ + 7) >> 3;
            for (int p = warp; p < rf * cf; p += LU5_THREADS / 32) {
                const int r0 = 8 * (p % rf), cb = t0 + 8 * (p / rf);
                double a0 = 0.0, a1 = 0.0, b0 = 0.0, b1 = 0.0;
                const int am = r0 + (lane >> 2), bn = cb + (lane >> 2);
#pragma unroll
                for (int ks = 0; ks < LU5_PB; ks += 4) {
                    const int k = ks + (lane & 3);
                    const bool kin = k < w;
                    const double ar = kin && am < nrows ? Lmr[k * LU5_LMLD + am] : 0.0;
                    const double ai = CP && kin && am < nrows ? Lmi[k * LU5_LMLD + am] : 0.0;
                    T bv = kin && bn < npiv ? A[bn * nrows + prow[k < w ? k : 0]] : VT<T>::zero();
                    double brr, bii;
                    if constexpr (CP) { brr = bv.x; bii = bv.y; } else { brr = bv; bii = 0.0; }
                    dmma(a0, a1, ar, brr);
                    if constexpr (CP) {
                        dmma(b0, b1, ar, bii);
                        dmma(a0, a1, ai, -bii);
                        dmma(b0, b1, ai, brr);
                    }
                }
                const int cr = r0 + (lane >> 2), cc = cb + 2 * (lane & 3);
                if (cr < nrows) {
                    if (cc < npiv) {
                        T *x = A + cc * nrows + cr;
                        if constexpr (CP) *x = cplx{x->x - a0, x->y - b0}; else *x = *x - a0;
                    }
                    if (cc + 1 < npiv) {
                        T *x = A + (cc + 1) * nrows + cr;
                        if constexpr (CP) *x = cplx{x->x - a1, x->y - b1}; else *x = *x - a1;
                    }
                }
            }
        }
        __syncthreads();
    }
    // the final order: pivot rows at their step, the others after them in block order (warps 0-3, a row each)
    if (pg) {
        const bool un = i < nrows && mytag == INT_MAX;
        const unsigned bal = __ballot_sync(0xffffffffu, un);
        if (lane == 0) wcnt[warp] = __popc(bal);
        named_bar(1, 128);
        int k0 = npiv;
        for (int q = 0; q < warp; q++) k0 += wcnt[q];
        const int k = un ? k0 + __popc(bal & ((1u << lane) - 1u)) : mytag;
        if (i < nrows) {
            sperm[k] = i;
            perm[k] = i;
            rowid[k] = myrid;
            if (k < npiv) p_lu[fcol + k] = myrid;
        }
    }
    __syncthreads();
    const int ne = npiv * nrows;
    for (int e = tid; e < ne; e += LU5_THREADS) { const int kk = e % nrows, c = e / nrows; Lout[e] = A[c * nrows + sperm[kk]]; }
}

template <typename T>
__global__ void __launch_bounds__(LU5_THREADS) k_front_lu5(const T *__restrict__ W, int64_t ld, int nrows, int npiv, int nri,
                                                            int64_t fcol, const double *__restrict__ colmax, double pivot_rel,
                                                            int64_t *__restrict__ rowid, T *__restrict__ Lout,
                                                            int *__restrict__ perm, int64_t *__restrict__ p_lu, DevStatus *st,
                                                            int64_t front, PivotAsm pa)
{
    front_lu5_body<T>(W, ld, nrows, npiv, nri, fcol, colmax, pivot_rel, rowid, Lout, perm, p_lu, st, front, pa);
}

// Blocked partial-pivot LU of a front's pivot block in shared memory (nrows <= 128, npiv <= 64; one CTA of LU3_THREADS):
// the same elimination as k_front_lu2 in panels of LU3_PB columns with a one-panel look-ahead.
//   warp 0 (the panel warp)  factors panel p = columns [c0, c1) with its rows in registers (row i in lane i % 32, slot
//                            i / 32): per column, the pivot (largest key, ties to the smaller row of B), the singular and
//                            border tests, the multipliers, and the update of the panel's later columns; no block barrier
//                            inside a panel.  Then the panel goes back to shared memory, with a copy of its multipliers
//                            in which every row already pivoted reads zero (Lm, double-buffered by panel parity).
//   warps 1.. (the workers)  for the columns after the panel, first the next panel's, then the rest: the pivot rows' U
//                            values by forward substitution with the panel's unit-lower L11 (a thread per column), then
//                            every row's update A[c][i] -= sum_k Lm[k][i] U[k][c].  As soon as the next panel's columns
//                            are done, warp 0 moves on to it while the workers finish the rest.
// Rows are never swapped: the pivot row of step j is tagged j, as in k_front_lu2, and the final order is formed at the end.
// Decisions to stop (singular column, dense-row pivot) are made by warp 0 before a panel's barrier and read by every warp
// after it.  Named barriers: 1 (all, a panel is factored), 2 (all, the next panel's columns are updated), 3 (workers).
constexpr int LU3_PB = 8, LU3_THREADS = 256;

template <typename T>
__global__ void __launch_bounds__(LU3_THREADS) k_front_lu3(const T *__restrict__ W, int64_t ld, int nrows, int npiv, int nri,
                                                           int64_t fcol, const double *__restrict__ colmax, double pivot_rel,
                                                           int64_t *__restrict__ rowid, T *__restrict__ Lout, int *__restrict__ perm,
                                                           int64_t *__restrict__ p_lu, DevStatus *st, int64_t front, PivotAsm pa)
{
    constexpr int PB = LU3_PB;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *A = reinterpret_cast<T *>(smem_raw);                        // npiv x nrows, column-major: A[c * nrows + i]
    T *Lm = A + (size_t)npiv * nrows;                              // 2 x PB x nrows: masked multipliers of a panel
    int64_t *rid = reinterpret_cast<int64_t *>(Lm + 2 * PB * nrows);
    double *thr = reinterpret_cast<double *>(rid + nrows);         // npiv: pivot_rel * max |B(:, column)|
    int *tag = reinterpret_cast<int *>(thr + npiv);
    int *pos = tag + nrows;
    int *piv = pos + nrows;                                        // npiv: the pivot row (local) of each step
    __shared__ int s_stop;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nt = blockDim.x;
    const int ne = npiv * nrows;
    if (!pa.on) {
        pdl_wait();
        for (int e0 = tid; e0 < ne; e0 += 8 * nt) {
            T v[8];
#pragma unroll
            for (int q = 0; q < 8; q++) { const int e = e0 + q * nt; v[q] = e < ne ? W[e % nrows + (int64_t)(e / nrows) * ld] : VT<T>::zero(); }
#pragma unroll
            for (int q = 0; q < 8; q++) { const int e = e0 + q * nt; if (e < ne) A[e] = v[q]; }
        }
        for (int i = tid; i < nrows; i += nt) rid[i] = rowid[i];
    } else {
        for (int e = tid; e < ne; e += nt) A[e] = VT<T>::zero();
        for (int i = tid; i < nrows; i += nt) rid[i] = pa.rowinit[i];
        __syncthreads();
        const T *Bx = reinterpret_cast<const T *>(pa.Bx);
#pragma unroll 4
        for (int64_t e = tid; e < pa.acnt; e += nt) A[pa.adst[e]] = Bx[pa.asrc[e]];
        pdl_wait();
        for (int64_t t = tid; t < pa.nslot; t += nt) rid[pa.slot + t] = pa.child_rowid[t];
        __syncthreads();
        const T *cb = reinterpret_cast<const T *>(pa.cb);
        const int cbr = (int)pa.cbr, tot = (int)(pa.cbr * pa.h), nsl = (int)pa.nslot, sl = (int)pa.slot, tb = (int)pa.tau_base;
#pragma unroll 4
        for (int e = tid; e < tot; e += nt) {
            const int c = e / cbr, t = e - c * cbr;
            const int pr = t < nsl ? sl + t : tb + (t - nsl);
            T *a = A + (int)pa.relcol[c] * nrows + pr;
            *a = add(*a, cb[t + (int64_t)c * cbr]);
        }
    }
    for (int i = tid; i < nrows; i += nt) tag[i] = INT_MAX;
    for (int c = tid; c < npiv; c += nt) thr[c] = pivot_rel * colmax[fcol + c];
    if (tid == 0) s_stop = st->code != 0 ? 3 : 0;
    __syncthreads();
    if (s_stop) return;
    const int npan = (npiv + PB - 1) / PB;
    if (warp == 0) {
        int64_t rr[4];
        bool al[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int i = lane + 32 * q;
            al[q] = i < nrows;
            rr[q] = al[q] ? rid[i] : INT64_MAX;
        }
        for (int p = 0; p < npan; p++) {
            const int c0 = p * PB, w = npiv - c0 < PB ? npiv - c0 : PB;
            T x[4][PB];
#pragma unroll
            for (int q = 0; q < 4; q++)
#pragma unroll
                for (int k = 0; k < PB; k++) {
                    const int i = lane + 32 * q;
                    x[q][k] = (i < nrows && k < w) ? A[(size_t)(c0 + k) * nrows + i] : VT<T>::zero();
                }
            int stop = 0;
#pragma unroll
            for (int k = 0; k < PB; k++) {
                if (k >= w) break;
                const int j = c0 + k;
                // the pivot: each lane's best live slot, then the warp's largest key (ties: the smaller row of B)
                long long bk = -1; int wi = -1; int64_t br = INT64_MAX;
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    if (!al[q]) continue;
                    const long long a = (long long)pivkey(x[q][k]);
                    if (a > bk || (a == bk && rr[q] < br)) { bk = a; wi = lane + 32 * q; br = rr[q]; }
                }
                const unsigned long long key = wi >= 0 ? (unsigned long long)bk : 0ull;
                const unsigned long long mk = warp_max_key(key);
                unsigned cand = __ballot_sync(0xffffffffu, wi >= 0 && key == mk);
                int bi = -1;
                if (cand != 0) {
                    if ((cand & (cand - 1)) != 0) {
                        int64_t r2 = (cand >> lane) & 1u ? br : INT64_MAX;
                        for (int o = 16; o > 0; o >>= 1) { const int64_t t = __shfl_xor_sync(0xffffffffu, r2, o); r2 = t < r2 ? t : r2; }
                        cand = __ballot_sync(0xffffffffu, ((cand >> lane) & 1u) && br == r2);
                    }
                    bi = __shfl_sync(0xffffffffu, wi, __ffs(cand) - 1);
                }
                // the pivot row's values in this panel's columns, from the lane that holds it
                const int ql = bi >= 0 ? bi >> 5 : 0, ol = bi >= 0 ? bi & 31 : 0;
                T prow[PB];
#pragma unroll
                for (int k2 = 0; k2 < PB; k2++) {
                    T mine = x[0][k2];
#pragma unroll
                    for (int q = 1; q < 4; q++) if (q == ql) mine = x[q][k2];
                    prow[k2] = shfl_v<T>(mine, ol);
                }
                const T pv = prow[k];
                if (lane == 0) {
                    const double t = thr[j];
                    const bool sing = bi < 0 || mk == 0ull || (mk < pivkey_of_modulus<T>(2.0 * t) && vabs(pv) < t);
                    if (sing) { set_status(st, ST_SINGULAR, fcol + j, bi >= 0 ? vabs(pv) : 0.0, t); stop = 1; }
                    else if (bi >= nri) { set_status(st, ST_BORDER, front, vabs(pv), t); stop = 1; }
                    if (!stop) { tag[bi] = j; piv[j] = bi; }
                }
                stop = __shfl_sync(0xffffffffu, stop, 0);
                if (stop) break;
                const T inv = recip(pv);
                if (lane == ol) {
#pragma unroll
                    for (int q = 0; q < 4; q++) if (q == ql) al[q] = false;
                }
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    if (!al[q]) continue;
                    const T l = mul(x[q][k], inv);
                    x[q][k] = l;
#pragma unroll
                    for (int k2 = k + 1; k2 < PB; k2++) if (k2 < w) x[q][k2] = sub(x[q][k2], mul(l, prow[k2]));
                }
            }
            // the panel back to shared memory; the multipliers of the rows still live (zero for every pivoted row)
            T *Lb = Lm + (size_t)(p & 1) * PB * nrows;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int i = lane + 32 * q;
                if (i >= nrows) continue;
#pragma unroll
                for (int k = 0; k < PB; k++) {
                    if (k >= w) break;
                    A[(size_t)(c0 + k) * nrows + i] = x[q][k];
                    Lb[(size_t)k * nrows + i] = al[q] ? x[q][k] : VT<T>::zero();
                }
            }
            if (lane == 0 && stop) s_stop = 1;
            __syncwarp();
            named_bar(1, nt);
            if (s_stop) return;
            if (p + 1 < npan) named_bar(2, nt);
        }
    } else {
        const int wt = tid - 32, nwt = nt - 32;
        for (int p = 0; p < npan; p++) {
            named_bar(1, nt);
            if (s_stop) return;
            const int c0 = p * PB, w = npiv - c0 < PB ? npiv - c0 : PB, c1 = c0 + w;
            const int c2 = c1 + PB < npiv ? c1 + PB : npiv;
            const T *Lb = Lm + (size_t)(p & 1) * PB * nrows;
            for (int part = 0; part < 2; part++) {
                const int ca = part ? c2 : c1, cb = part ? npiv : c2;
                if (ca < cb) {
                    // U rows of the panel's pivots in columns [ca, cb): forward substitution with L11 (a thread per column)
                    for (int c = ca + wt; c < cb; c += nwt) {
                        T u[PB];
#pragma unroll
                        for (int k = 0; k < PB; k++) {
                            if (k >= w) break;
                            const int pr = piv[c0 + k];
                            T v = A[(size_t)c * nrows + pr];
#pragma unroll
                            for (int m = 0; m < PB; m++) if (m < k) v = sub(v, mul(A[(size_t)(c0 + m) * nrows + pr], u[m]));
                            u[k] = v;
                            A[(size_t)c * nrows + pr] = v;
                        }
                    }
                    named_bar(3, nwt);
                    // every row: A[c][i] -= sum_k Lm[k][i] U[k][c] (the pivoted rows' Lm is zero: they are left alone)
                    const int tot = (cb - ca) * nrows;
                    for (int e = wt; e < tot; e += nwt) {
                        const int c = ca + e / nrows, i = e - (e / nrows) * nrows;
                        T acc = VT<T>::zero();
#pragma unroll
                        for (int k = 0; k < PB; k++) {
                            if (k >= w) break;
                            acc = add(acc, mul(Lb[(size_t)k * nrows + i], A[(size_t)c * nrows + piv[c0 + k]]));
                        }
                        if (!is_zero(acc)) A[(size_t)c * nrows + i] = sub(A[(size_t)c * nrows + i], acc);
                    }
                }
                if (part == 0 && p + 1 < npan) named_bar(2, nt);
            }
        }
    }
    __syncthreads();
    const int steps = npiv;
    if (warp == 0) {
        int base = steps;
        for (int i0 = 0; i0 < nrows; i0 += 32) {
            const int i = i0 + lane;
            const bool un = i < nrows && tag[i] >= steps;
            const unsigned m = __ballot_sync(0xffffffffu, un);
            if (i < nrows) pos[i] = un ? base + __popc(m & ((1u << lane) - 1u)) : tag[i];
            base += __popc(m);
        }
    }
    __syncthreads();
    for (int i = tid; i < nrows; i += nt) {
        const int k = pos[i];
        perm[k] = i;
        rowid[k] = rid[i];
        if (k < steps) p_lu[fcol + k] = rid[i];
    }
    for (int e = tid; e < ne; e += nt) { const int i = e % nrows; Lout[pos[i] + (int64_t)(e / nrows) * nrows] = A[e]; }
}

// After the blocked (global-memory) pivoting of a large front's pivot block: the final row order from the swaps, the
// pivot rows (the swaps already moved the row ids), and the block into the arena
template <typename T>
__global__ void k_left_finish(const T *__restrict__ W, int64_t ld, int64_t nrows, int64_t npiv, const int *__restrict__ ipiv,
                              int *__restrict__ perm, const int64_t *__restrict__ rowid, int64_t f, int64_t *__restrict__ p_lu,
                              T *__restrict__ Lout, const DevStatus *st)
{
    if (st->code) return;
    if (blockIdx.x == 0) {          // the identity by the whole first CTA, then the interchanges in order by one thread
        for (int64_t i = threadIdx.x; i < nrows; i += blockDim.x) perm[i] = (int)i;
        __syncthreads();
        if (threadIdx.x == 0)
            for (int64_t j = 0; j < npiv && j < nrows; j++) { int p = ipiv[j]; int t = perm[j]; perm[j] = perm[p]; perm[p] = t; }
    }
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = tid; e < nrows * npiv; e += stride) Lout[e] = W[e % nrows + (e / nrows) * ld];
    for (int64_t i = tid; i < npiv && i < nrows; i += stride) p_lu[f + i] = rowid[i];
}

// U12 rows in pivot order: U[i + c * npiv] = W[perm[i] + (npiv + c) * ld]
template <typename T>
__global__ void k_u12_gather(const T *__restrict__ W, int64_t ld, int64_t npiv, int64_t ncb, const int *__restrict__ perm,
                             T *__restrict__ U, const DevStatus *st)
{
    if (st->code) return;
    const int64_t total = npiv * ncb;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e % npiv, c = e / npiv;
        U[e] = W[perm[i] + (npiv + c) * ld];
    }
}


// U12 = L11^-1 A12[perm] for npiv <= 64, by column tiles of 32 in shared memory (persistent CTAs: L11 staged once per
// CTA): the tile's pivot rows are gathered through perm; then per 16-row block, the diagonal 16 x 16 solve by half-warps
// (one column each, 16 shuffle steps) and the update of the rows below from shared memory by the whole CTA; the tile
// leaves for the arena.  The same operations as a blocked forward substitution.
constexpr int U12_TN = 32, U12_NP = 64, U12_BK = 16;
template <typename T>
__global__ void __launch_bounds__(256) k_u12_blk(const T *__restrict__ W, int64_t ld, const int *__restrict__ perm, int npiv,
                                                 int64_t ncb, const T *__restrict__ Lb, int64_t ldl, T *__restrict__ U,
                                                 const DevStatus *st)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *sL = reinterpret_cast<T *>(smem_raw);                 // U12_NP x U12_NP, column-major (ld U12_NP)
    T *X = sL + U12_NP * U12_NP;                             // U12_NP x U12_TN, column-major (ld U12_NP)
    __shared__ int sperm[U12_NP];
    if (st->code) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int e = tid; e < U12_NP * U12_NP; e += blockDim.x) {
        const int r = e % U12_NP, c = e / U12_NP;
        sL[e] = (r < npiv && c < npiv) ? Lb[r + (int64_t)c * ldl] : VT<T>::zero();
    }
    for (int i = tid; i < U12_NP; i += blockDim.x) sperm[i] = i < npiv ? perm[i] : 0;
    __syncthreads();
    const int64_t ntile = (ncb + U12_TN - 1) / U12_TN;
    const int nb = (npiv + U12_BK - 1) / U12_BK;
    const int half = lane >> 4, hl = lane & 15;
    for (int64_t t = blockIdx.x; t < ntile; t += gridDim.x) {
        const int64_t c0 = t * U12_TN;
        const int tn = (int)(ncb - c0 < U12_TN ? ncb - c0 : U12_TN);
        for (int e = tid; e < U12_NP * U12_TN; e += blockDim.x) {
            const int r = e % U12_NP, c = e / U12_NP;
            X[e] = (r < npiv && c < tn) ? W[sperm[r] + (npiv + c0 + c) * ld] : VT<T>::zero();
        }
        __syncthreads();
        for (int b = 0; b < nb; b++) {
            const int r0 = b * U12_BK, w = npiv - r0 < U12_BK ? npiv - r0 : U12_BK;
            // the diagonal block: a half-warp per column (both halves of a warp step through the column pairs together,
            // so every shuffle has the full warp), lane hl holds row r0 + hl
            for (int cp = warp; 2 * cp < tn; cp += blockDim.x >> 5) {
                const int c = 2 * cp + half;
                const bool act = c < tn;
                T x = act ? X[r0 + hl + c * U12_NP] : VT<T>::zero();
                for (int i = 0; i < w; i++) {
                    T xi;
                    if constexpr (VT<T>::cplx_) xi = T{__shfl_sync(0xffffffffu, x.x, i, 16), __shfl_sync(0xffffffffu, x.y, i, 16)};
                    else xi = __shfl_sync(0xffffffffu, x, i, 16);
                    if (hl > i && hl < w) x = sub(x, mul(sL[r0 + hl + (r0 + i) * U12_NP], xi));
                }
                if (act && hl < w) X[r0 + hl + c * U12_NP] = x;
            }
            __syncthreads();
            // the rows below: X[r, c] -= sum_k L[r, r0 + k] X[r0 + k, c]
            const int rb = r0 + w;
            if (rb < npiv) {
                const int mrows = npiv - rb;
                for (int e = tid; e < mrows * tn; e += blockDim.x) {
                    const int r = rb + e % mrows, c = e / mrows;
                    T acc = VT<T>::zero();
#pragma unroll 4
                    for (int kk = 0; kk < w; kk++) acc = add(acc, mul(sL[r + (r0 + kk) * U12_NP], X[r0 + kk + c * U12_NP]));
                    X[r + c * U12_NP] = sub(X[r + c * U12_NP], acc);
                }
            }
            __syncthreads();
        }
        for (int e = tid; e < npiv * tn; e += blockDim.x) {
            const int r = e % npiv, c = e / npiv;
            U[r + (c0 + c) * (int64_t)npiv] = X[r + c * U12_NP];
        }
        __syncthreads();
    }
}

// The tail of a front with npiv <= 64 and nrows <= 128, in one pass over its contribution-block columns: for each tile of
// TN columns (32; 8 for the few columns the next pivot block waits for), the tile's rows are gathered in pivot order (perm; the next tile's values are loaded into registers while
// this one is computed), then per 16-row block of the pivot rows, the diagonal 16 x 16 unit-lower solve by half-warps
// (one column each, 16 shuffle steps) and the update of every row below, pivot rows and contribution-block rows alike,
// X[r, c] -= sum_k L[r, k] X[k, c], on the FP64 tensor cores (mma m8n8k4; complex as four real products).  Rows [0, npiv)
// leave as U12 (into the arena), rows [npiv, nrows) as the contribution block A22[perm] - L21 U12 (into the stack): the
// blocked forward substitution with [L11; L21] of the front's columns.  L (real and imaginary planes) and the tile live
// in shared memory with a leading dimension of 132 doubles (4 mod 16: the mma fragments of a half-warp hit 16 banks).
constexpr int FT_TN = 32, FT_LD = 132, FT_NP = 64, FT_NR = 128, FT_THREADS = 512;
template <typename T, int TN>
__device__ __forceinline__ void front_tail_body(const T *__restrict__ W, int64_t ld, const int *__restrict__ perm, int npiv,
                                                int nrows, int64_t ncb, int64_t cb0, int64_t cb1, const T *__restrict__ Lb,
                                                T *__restrict__ U, T *__restrict__ CB, const DevStatus *st, int bid, int nbk)
{
    constexpr bool CP = VT<T>::cplx_;
    constexpr int PER = FT_NR * TN / FT_THREADS;                   // tile values per thread
    extern __shared__ __align__(16) double ft_smem[];
    double *sLr = ft_smem;                                          // L[m, k] at k * FT_LD + m
    double *sLi = sLr + (CP ? FT_NP * FT_LD : 0);
    double *sXr = sLr + (CP ? 2 : 1) * FT_NP * FT_LD;               // X[r, c] at c * FT_LD + r
    double *sXi = sXr + (CP ? TN * FT_LD : 0);
    __shared__ int sperm[FT_NR];
    pdl_trigger();                                   // the next pivot block's LU may start its own set-up
    if (st->code) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int M = nrows - npiv;
    for (int i = tid; i < nrows; i += FT_THREADS) sperm[i] = perm[i];
    __syncthreads();
    // columns [cb0, cb1) of the contribution block (cb0 a multiple of the tile width)
    const int64_t t0 = cb0 / TN, ntile = (cb1 + TN - 1) / TN;
    T pre[PER];
    auto fetch = [&](int64_t t) {
        const int64_t c0 = t * TN;
#pragma unroll
        for (int q = 0; q < PER; q++) {
            const int e = tid + q * FT_THREADS, r = e % FT_NR, c = e / FT_NR;
            pre[q] = (t < ntile && r < nrows && c0 + c < cb1) ? W[sperm[r] + (npiv + c0 + c) * ld] : VT<T>::zero();
        }
    };
    fetch(t0 + bid);                                          // in flight while L is staged
    for (int e0 = tid; e0 < npiv * nrows; e0 += 8 * FT_THREADS) {     // 8 loads in flight per thread
        T v[8];
#pragma unroll
        for (int q = 0; q < 8; q++) { const int e = e0 + q * FT_THREADS; v[q] = e < npiv * nrows ? Lb[e] : VT<T>::zero(); }
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const int e = e0 + q * FT_THREADS, m = e % nrows, k = e / nrows;
            if (e < npiv * nrows) {
                if constexpr (CP) { sLr[k * FT_LD + m] = v[q].x; sLi[k * FT_LD + m] = v[q].y; } else sLr[k * FT_LD + m] = v[q];
            }
        }
    }
    __syncthreads();
    const int half = lane >> 4, hl = lane & 15;
    for (int64_t t = t0 + bid; t < ntile; t += nbk) {
        const int64_t c0 = t * TN;
        const int tn = (int)(cb1 - c0 < TN ? cb1 - c0 : TN);
#pragma unroll
        for (int q = 0; q < PER; q++) {
            const int e = tid + q * FT_THREADS, r = e % FT_NR, c = e / FT_NR;
            if constexpr (CP) { sXr[c * FT_LD + r] = pre[q].x; sXi[c * FT_LD + r] = pre[q].y; } else sXr[c * FT_LD + r] = pre[q];
        }
        __syncthreads();
        fetch(t + nbk);                                       // in flight during this tile
        for (int kb = 0; kb < npiv; kb += 16) {
            const int w = npiv - kb < 16 ? npiv - kb : 16;
            if (2 * warp < TN) {   // the diagonal block: a half-warp per column, lane hl holds row kb + hl
                const int c = 2 * warp + half;
                double xr = hl < w ? sXr[c * FT_LD + kb + hl] : 0.0, xi = CP && hl < w ? sXi[c * FT_LD + kb + hl] : 0.0;
                for (int i = 0; i < w; i++) {
                    const double pr = __shfl_sync(0xffffffffu, xr, i, 16);
                    const double pi = CP ? __shfl_sync(0xffffffffu, xi, i, 16) : 0.0;
                    if (hl > i && hl < w) {
                        const double lr = sLr[(kb + i) * FT_LD + kb + hl];
                        if constexpr (CP) {
                            const double li = sLi[(kb + i) * FT_LD + kb + hl];
                            const T x = sub(T{xr, xi}, mul(T{lr, li}, T{pr, pi}));
                            xr = x.x; xi = x.y;
                        } else xr = xr - lr * pr;
                    }
                }
                if (hl < w) { sXr[c * FT_LD + kb + hl] = xr; if constexpr (CP) sXi[c * FT_LD + kb + hl] = xi; }
            }
            __syncthreads();
            const int rb = kb + w, R = nrows - rb;
            if (R > 0) {
                const int mt = (R + 7) >> 3, nt = (tn + 7) >> 3;
                for (int p = warp; p < mt * nt; p += FT_THREADS / 32) {
                    const int m0 = rb + 8 * (p % mt), n0 = 8 * (p / mt);
                    const int am = m0 + (lane >> 2), bn = n0 + (lane >> 2);
                    double a0 = 0.0, a1 = 0.0, b0 = 0.0, b1 = 0.0;         // re / im accumulators (two columns each)
                    for (int ks = 0; ks < w; ks += 4) {
                        const int k = kb + ks + (lane & 3);
                        const bool kin = ks + (lane & 3) < w;
                        const double ar = kin && am < nrows ? sLr[k * FT_LD + am] : 0.0;
                        const double br = kin ? sXr[bn * FT_LD + k] : 0.0;
                        dmma(a0, a1, ar, br);
                        if constexpr (CP) {
                            const double ai = kin && am < nrows ? sLi[k * FT_LD + am] : 0.0;
                            const double bi = kin ? sXi[bn * FT_LD + k] : 0.0;
                            dmma(a0, a1, ai, -bi);
                            dmma(b0, b1, ar, bi);
                            dmma(b0, b1, ai, br);
                        }
                    }
                    const int cr = m0 + (lane >> 2), cc = n0 + 2 * (lane & 3);
                    if (cr < nrows) {
                        sXr[cc * FT_LD + cr] -= a0;
                        sXr[(cc + 1) * FT_LD + cr] -= a1;
                        if constexpr (CP) { sXi[cc * FT_LD + cr] -= b0; sXi[(cc + 1) * FT_LD + cr] -= b1; }
                    }
                }
            }
            __syncthreads();
        }
        for (int e = tid; e < nrows * tn; e += FT_THREADS) {
            const int r = e % nrows, c = e / nrows;
            T v;
            if constexpr (CP) v = T{sXr[c * FT_LD + r], sXi[c * FT_LD + r]}; else v = sXr[c * FT_LD + r];
            if (r < npiv) U[r + (c0 + c) * (int64_t)npiv] = v;
            else CB[(r - npiv) + (c0 + c) * (int64_t)M] = v;
        }
        __syncthreads();
    }
}

template <typename T, int TN>
__global__ void __launch_bounds__(FT_THREADS) k_front_tail(const T *__restrict__ W, int64_t ld, const int *__restrict__ perm,
                                                           int npiv, int nrows, int64_t ncb, int64_t cb0, int64_t cb1,
                                                           const T *__restrict__ Lb, T *__restrict__ U, T *__restrict__ CB,
                                                           const DevStatus *st)
{
    front_tail_body<T, TN>(W, ld, perm, npiv, nrows, ncb, cb0, cb1, Lb, U, CB, st, (int)blockIdx.x, (int)gridDim.x);
}

// d += a b on the FP64 tensor cores (mma m8n8k4), free for the compiler to schedule
__device__ __forceinline__ void dmma_s(double &d0, double &d1, double a, double b)
{
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n" : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}

// The tail's multipliers with the diagonal blocks folded in, formed in shared memory from the front's L block (sL: L[m, k]
// at k * FT_LD + m): for each 16-column block b of the pivot columns (rows and columns [16b, 16b + w)), D_b = L_bb^-1
// (unit lower, zero above the diagonal) replaces the block's rows, and every row r below the block holds
// M[r, block b] = L[r, block b] D_b.  Then the blocked forward substitution X_b <- D_b X_b, X_r -= L[r, b] X_b becomes, per
// block, one product M[rows >= 16b, block b] X_b with no serial step: X_b = D_b X_b and X_r -= M[r, b] X_b.  Every thread of
// the CTA (FT_THREADS) takes part; ends with a block barrier.
template <bool CP>
__device__ __forceinline__ void tail_prep_m(double *__restrict__ sLr, double *__restrict__ sLi, int npiv, int nrows, int tid)
{
    const int lane = tid & 31, warp = tid >> 5, half = lane >> 4, hl = lane & 15;
    const int nbk = (npiv + 15) >> 4;
    // (1) the columns of every D_b: the half-warp (warp, half) solves L_bb x = e for columns 2 warp + half and that + 32
    // (both halves of a warp are in the same block, so the shuffles see the same trip count)
    double dr[2], di[2];
#pragma unroll
    for (int q = 0; q < 2; q++) {
        const int c = 2 * warp + half + 32 * q, k0 = c & ~15, cb = c & 15;
        const int w = npiv - k0 < 16 ? npiv - k0 : 16;
        double xr = hl == cb ? 1.0 : 0.0, xi = 0.0;
        for (int i = 0; i < w; i++) {
            const double pr = __shfl_sync(0xffffffffu, xr, i, 16);
            const double pi = CP ? __shfl_sync(0xffffffffu, xi, i, 16) : 0.0;
            if (hl > i && hl < w) {
                const double lr = sLr[(k0 + i) * FT_LD + k0 + hl];
                if constexpr (CP) {
                    const double li = sLi[(k0 + i) * FT_LD + k0 + hl];
                    const cplx x = sub(cplx{xr, xi}, mul(cplx{lr, li}, cplx{pr, pi}));
                    xr = x.x; xi = x.y;
                } else xr = xr - lr * pr;
            }
        }
        dr[q] = xr; di[q] = xi;
    }
    // (2) the products M[r, block b] = L[r, block b] D_b of the rows below each block (D_b read from the registers of
    // step 1 through shared memory after the barrier): items (b, 8-row fragment), two 8-column fragments each, at most
    // 14 + 12 + 10 + 8 = 44 items, three per warp
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 2; q++) {
        const int c = 2 * warp + half + 32 * q, k0 = c & ~15, cb = c & 15;
        const int w = npiv - k0 < 16 ? npiv - k0 : 16;
        if (cb < w && hl < w) { sLr[(k0 + cb) * FT_LD + k0 + hl] = dr[q]; if constexpr (CP) sLi[(k0 + cb) * FT_LD + k0 + hl] = di[q]; }
    }
    __syncthreads();
    int rs[4], nf[4], pre[5];
    pre[0] = 0;
#pragma unroll
    for (int b = 0; b < 4; b++) {
        const int k0 = 16 * b, w = b < nbk ? (npiv - k0 < 16 ? npiv - k0 : 16) : 0;
        rs[b] = (k0 + w) & ~7;
        nf[b] = b < nbk && nrows > k0 + w ? (nrows - rs[b] + 7) >> 3 : 0;
        pre[b + 1] = pre[b] + nf[b];
    }
    double res[3][2][4];
    int rb[3], rr0[3];
#pragma unroll
    for (int s = 0; s < 3; s++) {
        const int p = warp + 16 * s;
        rb[s] = -1;
        if (p >= pre[4]) continue;                                   // warp-uniform
        int b = 0, rsb = rs[0], preb = 0;
#pragma unroll
        for (int q = 1; q < 4; q++) if (p >= pre[q]) { b = q; rsb = rs[q]; preb = pre[q]; }
        const int k0 = 16 * b, w = npiv - k0 < 16 ? npiv - k0 : 16;
        const int r0 = rsb + 8 * (p - preb);
        rb[s] = b; rr0[s] = r0;
        const int am = r0 + (lane >> 2);
#pragma unroll
        for (int cf = 0; cf < 2; cf++) { res[s][cf][0] = res[s][cf][1] = res[s][cf][2] = res[s][cf][3] = 0.0; }
        for (int ks = 0; ks < w; ks += 4) {
            const int kk = ks + (lane & 3), k = k0 + kk;
            const bool kin = kk < w;
            const double ar = kin && am < nrows ? sLr[k * FT_LD + am] : 0.0;
            const double ai = CP && kin && am < nrows ? sLi[k * FT_LD + am] : 0.0;
#pragma unroll
            for (int cf = 0; cf < 2; cf++) {
                const int nn = 8 * cf + (lane >> 2);                    // column of D_b
                const bool bok = kin && nn < w;
                const double br = bok ? sLr[(k0 + nn) * FT_LD + k] : 0.0;
                dmma_s(res[s][cf][0], res[s][cf][1], ar, br);
                if constexpr (CP) {
                    const double bi = bok ? sLi[(k0 + nn) * FT_LD + k] : 0.0;
                    dmma_s(res[s][cf][0], res[s][cf][1], ai, -bi);
                    dmma_s(res[s][cf][2], res[s][cf][3], ar, bi);
                    dmma_s(res[s][cf][2], res[s][cf][3], ai, br);
                }
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < 3; s++) {
        if (rb[s] < 0) continue;
        const int k0 = 16 * rb[s], w = npiv - k0 < 16 ? npiv - k0 : 16;
        const int cr = rr0[s] + (lane >> 2);
        if (cr < k0 + w || cr >= nrows) continue;
#pragma unroll
        for (int cf = 0; cf < 2; cf++) {
            const int cc = 8 * cf + 2 * (lane & 3);
#pragma unroll
            for (int h = 0; h < 2; h++) {
                if (cc + h >= w) continue;
                sLr[(k0 + cc + h) * FT_LD + cr] = res[s][cf][h];
                if constexpr (CP) sLi[(k0 + cc + h) * FT_LD + cr] = res[s][cf][2 + h];
            }
        }
    }
    __syncthreads();
}

// Where a front's tail writes its contribution block: the stack (W null), or straight into its parent's working block W
// (leading dimension ld): CB row t to parent row slot + t (t < nslot) or tau_base + t - nslot, CB column c to parent column
// relcol[c]; the parent's first `slot` rows (its entering rows) of those columns are written as zeros.
struct TailOut {
    void *W;
    int64_t ld, nslot, slot, tau_base;
    const int64_t *relcol;
};

// The tail of a front with npiv <= 64 and nrows <= 128 (the successor of front_tail_body): the same U12 and contribution
// block, X = [L11; L21]-forward-substitution of the gathered columns A[perm, npiv + c], with the multipliers M of
// tail_prep_m (formed once per CTA): per tile of TN columns and per 16-column block b of the pivots, one FP64 tensor-core
// product over the rows at and below the block (warp w takes rows 16b + 8w .. + 7 and every column of the tile, so the
// M fragment is loaded once for all of them): rows below the block leave as X_r -= M[r, b] X_b at once, the block's own
// rows as X_b = D_b X_b after the block barrier (no later block reads them).  One barrier per pivot block, no serial
// diagonal solve.
template <typename T, int TN>
__device__ __forceinline__ void front_tail2_body(const T *__restrict__ W, int64_t ld, const int *__restrict__ perm, int npiv,
                                                 int nrows, int64_t ncb, int64_t cb0, int64_t cb1, const T *__restrict__ Lb,
                                                 T *__restrict__ U, T *__restrict__ CB, const DevStatus *st, int bid, int nbk,
                                                 const TailOut &to)
{
    constexpr bool CP = VT<T>::cplx_;
    constexpr int PER = FT_NR * TN / FT_THREADS;                   // tile values per thread
    constexpr int NCF = TN / 8;                                     // 8-column fragments per tile
    extern __shared__ __align__(16) double ft_smem[];
    double *sLr = ft_smem;                                          // M[m, k] at k * FT_LD + m
    double *sLi = sLr + (CP ? FT_NP * FT_LD : 0);
    double *sXr = sLr + (CP ? 2 : 1) * FT_NP * FT_LD;               // X[r, c] at c * FT_LD + r
    double *sXi = sXr + (CP ? TN * FT_LD : 0);
    __shared__ int sperm[FT_NR];
    pdl_trigger();                                   // the next pivot block's LU may start its own set-up
    if (st->code) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int M = nrows - npiv;
    for (int i = tid; i < nrows; i += FT_THREADS) sperm[i] = perm[i];
    __syncthreads();
    const int64_t t0 = cb0 / TN, ntile = (cb1 + TN - 1) / TN;
    T pre[PER];
    auto fetch = [&](int64_t t) {
        const int64_t c0 = t * TN;
#pragma unroll
        for (int q = 0; q < PER; q++) {
            const int e = tid + q * FT_THREADS, r = e % FT_NR, c = e / FT_NR;
            pre[q] = (t < ntile && r < nrows && c0 + c < cb1) ? W[sperm[r] + (npiv + c0 + c) * ld] : VT<T>::zero();
        }
    };
    if (t0 + bid < ntile) fetch(t0 + bid);                          // in flight while M is formed
    for (int e0 = tid; e0 < npiv * nrows; e0 += 8 * FT_THREADS) {     // 8 loads in flight per thread
        T v[8];
#pragma unroll
        for (int q = 0; q < 8; q++) { const int e = e0 + q * FT_THREADS; v[q] = e < npiv * nrows ? Lb[e] : VT<T>::zero(); }
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const int e = e0 + q * FT_THREADS, m = e % nrows, k = e / nrows;
            if (e < npiv * nrows) {
                if constexpr (CP) { sLr[k * FT_LD + m] = v[q].x; sLi[k * FT_LD + m] = v[q].y; } else sLr[k * FT_LD + m] = v[q];
            }
        }
    }
    __syncthreads();
    tail_prep_m<CP>(sLr, sLi, npiv, nrows, tid);
    const int nb16 = (npiv + 15) >> 4;
    for (int64_t t = t0 + bid; t < ntile; t += nbk) {
        const int64_t c0 = t * TN;
        const int tn = (int)(cb1 - c0 < TN ? cb1 - c0 : TN);
#pragma unroll
        for (int q = 0; q < PER; q++) {
            const int e = tid + q * FT_THREADS, r = e % FT_NR, c = e / FT_NR;
            if constexpr (CP) { sXr[c * FT_LD + r] = pre[q].x; sXi[c * FT_LD + r] = pre[q].y; } else sXr[c * FT_LD + r] = pre[q];
        }
        __syncthreads();
        fetch(t + nbk);                                       // in flight during this tile
        for (int b = 0; b < nb16; b++) {
            const int k0 = 16 * b, w = npiv - k0 < 16 ? npiv - k0 : 16;
            const int r0 = k0 + 8 * warp;                            // this warp's 8 rows
            const bool act = r0 < nrows;                             // warp-uniform
            double acc[NCF][4];
#pragma unroll
            for (int cf = 0; cf < NCF; cf++) acc[cf][0] = acc[cf][1] = acc[cf][2] = acc[cf][3] = 0.0;
            const int am = r0 + (lane >> 2);
            if (act) {
                for (int ks = 0; ks < w; ks += 4) {
                    const int kk = ks + (lane & 3), k = k0 + kk;
                    const bool kin = kk < w;
                    const double ar = kin && am < nrows ? sLr[k * FT_LD + am] : 0.0;
                    const double ai = CP && kin && am < nrows ? sLi[k * FT_LD + am] : 0.0;
                    double br[NCF], bi[NCF];
#pragma unroll
                    for (int cf = 0; cf < NCF; cf++) {
                        const int bn = 8 * cf + (lane >> 2);
                        br[cf] = kin ? sXr[bn * FT_LD + k] : 0.0;
                        bi[cf] = CP && kin ? sXi[bn * FT_LD + k] : 0.0;
                    }
                    // the products grouped so that consecutive tensor-core instructions are independent (2 NCF - 1
                    // others between two on the same accumulator)
#pragma unroll
                    for (int cf = 0; cf < NCF; cf++) dmma_s(acc[cf][0], acc[cf][1], ar, br[cf]);
                    if constexpr (CP) {
#pragma unroll
                        for (int cf = 0; cf < NCF; cf++) dmma_s(acc[cf][2], acc[cf][3], ar, bi[cf]);
#pragma unroll
                        for (int cf = 0; cf < NCF; cf++) dmma_s(acc[cf][0], acc[cf][1], ai, -bi[cf]);
#pragma unroll
                        for (int cf = 0; cf < NCF; cf++) dmma_s(acc[cf][2], acc[cf][3], ai, br[cf]);
                    }
                }
            }
            // the output fragment: row cr, columns cc and cc + 1 of each 8-column fragment
            const int cr = r0 + (lane >> 2);
            const bool yrow = cr < k0 + w;                           // a row of block b: X_b = D_b X_b after the barrier
            if (act && !yrow && cr < nrows) {
#pragma unroll
                for (int cf = 0; cf < NCF; cf++) {
                    const int cc = 8 * cf + 2 * (lane & 3);
                    sXr[cc * FT_LD + cr] -= acc[cf][0];
                    sXr[(cc + 1) * FT_LD + cr] -= acc[cf][1];
                    if constexpr (CP) { sXi[cc * FT_LD + cr] -= acc[cf][2]; sXi[(cc + 1) * FT_LD + cr] -= acc[cf][3]; }
                }
            }
            __syncthreads();
            if (act && yrow && cr < nrows) {
#pragma unroll
                for (int cf = 0; cf < NCF; cf++) {
                    const int cc = 8 * cf + 2 * (lane & 3);
                    sXr[cc * FT_LD + cr] = acc[cf][0];
                    sXr[(cc + 1) * FT_LD + cr] = acc[cf][1];
                    if constexpr (CP) { sXi[cc * FT_LD + cr] = acc[cf][2]; sXi[(cc + 1) * FT_LD + cr] = acc[cf][3]; }
                }
            }
        }
        __syncthreads();
        T *Wo = reinterpret_cast<T *>(to.W);
        for (int e = tid; e < nrows * tn; e += FT_THREADS) {
            const int r = e % nrows, c = e / nrows;
            T v;
            if constexpr (CP) v = T{sXr[c * FT_LD + r], sXi[c * FT_LD + r]}; else v = sXr[c * FT_LD + r];
            if (r < npiv) U[r + (c0 + c) * (int64_t)npiv] = v;
            else if (!Wo) CB[(r - npiv) + (c0 + c) * (int64_t)M] = v;
            else {
                const int64_t t = r - npiv, pr = t < to.nslot ? to.slot + t : to.tau_base + (t - to.nslot);
                Wo[pr + to.relcol[c0 + c] * to.ld] = v;
            }
        }
        if (Wo) {
            const int sl = (int)to.slot;
            for (int e = tid; e < sl * tn; e += FT_THREADS) {
                const int r = e % sl, c = e / sl;
                Wo[r + to.relcol[c0 + c] * to.ld] = VT<T>::zero();
            }
        }
        __syncthreads();
    }
}

template <typename T, int TN>
__global__ void __launch_bounds__(FT_THREADS) k_front_tail2(const T *__restrict__ W, int64_t ld, const int *__restrict__ perm,
                                                            int npiv, int nrows, int64_t ncb, int64_t cb0, int64_t cb1,
                                                            const T *__restrict__ Lb, T *__restrict__ U, T *__restrict__ CB,
                                                            const DevStatus *st, TailOut to)
{
    front_tail2_body<T, TN>(W, ld, perm, npiv, nrows, ncb, cb0, cb1, Lb, U, CB, st, (int)blockIdx.x, (int)gridDim.x, to);
}

// X <- L^-1 X for a unit lower w x w block (w <= 32 RPL) and every column of X (rows [0, w) of each column, ld ldx):
// a warp per column, RPL rows per lane, the solved entries broadcast by shuffles
template <typename T, int RPL>
__global__ void __launch_bounds__(256) k_trsm_warp(T *__restrict__ X, int64_t ldx, int w, int64_t ncols,
                                                   const T *__restrict__ Lb, int64_t ldl, const DevStatus *st)
{
    constexpr int CPW = 4;                            // columns per warp at once (independent chains through one loop)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *sL = reinterpret_cast<T *>(smem_raw);          // w x w, column-major, ld w
    if (st->code) return;
    for (int e0 = threadIdx.x; e0 < w * w; e0 += 8 * blockDim.x) {       // eight loads in flight per thread
        T v[8];
#pragma unroll
        for (int q = 0; q < 8; q++) { const int e = e0 + q * blockDim.x; v[q] = e < w * w ? Lb[(e % w) + (int64_t)(e / w) * ldl] : VT<T>::zero(); }
#pragma unroll
        for (int q = 0; q < 8; q++) { const int e = e0 + q * blockDim.x; if (e < w * w) sL[e] = v[q]; }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t wid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5, nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c0 = wid * CPW; c0 < ncols; c0 += nwarp * CPW) {
        T x[CPW][RPL];
#pragma unroll
        for (int j = 0; j < CPW; j++)
#pragma unroll
            for (int q = 0; q < RPL; q++) {
                const int r = lane + 32 * q;
                x[j][q] = (r < w && c0 + j < ncols) ? X[r + (c0 + j) * ldx] : VT<T>::zero();
            }
        for (int i = 0; i < w; i++) {
            T xi[CPW];
#pragma unroll
            for (int j = 0; j < CPW; j++) xi[j] = shfl_v<T>(RPL > 1 && i >= 32 ? x[j][RPL > 1 ? 1 : 0] : x[j][0], i & 31);
#pragma unroll
            for (int q = 0; q < RPL; q++) {
                const int r = lane + 32 * q;
                if (r > i && r < w) {
                    const T l = sL[r + i * w];
#pragma unroll
                    for (int j = 0; j < CPW; j++) x[j][q] = sub(x[j][q], mul(l, xi[j]));
                }
            }
        }
#pragma unroll
        for (int j = 0; j < CPW; j++)
#pragma unroll
            for (int q = 0; q < RPL; q++) {
                const int r = lane + 32 * q;
                if (r < w && c0 + j < ncols) X[r + (c0 + j) * ldx] = x[j][q];
            }
    }
}

// =====================================================================================================================
// solves (x column-major n x nrhs; row space: rows of B; column / pivot space: columns of B = pivot steps)
// =====================================================================================================================

// Wr[r] = Drp[r] * b[row_perm[r]] (trans 0), or Wc[k] = Dcp[k] * b[col_perm[k]] (trans 1, 2); a null perm is the
// identity and a null scale is 1 (the low-level solve on the factors of the permuted matrix)
template <typename T>
__global__ void k_rhs_in(T *__restrict__ out, const T *__restrict__ b, int64_t ldb, const int64_t *__restrict__ perm,
                         const double *__restrict__ scale, int64_t n, int64_t nrhs)
{
    const int64_t total = n * nrhs;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        int64_t k = e % n, r = e / n;
        const T v = b[(perm ? perm[k] : k) + r * ldb];
        out[e] = scale ? scal(v, scale[k]) : v;
    }
}

// x[perm[k]] = scale[sidx[k]] * v[k]  (trans 0: perm = col_perm, sidx = identity; trans 1/2: perm = row_perm o p_lu);
// a null perm is the identity and a null scale is 1
template <typename T>
__global__ void k_rhs_out(T *__restrict__ x, int64_t ldx, const T *__restrict__ v, const int64_t *__restrict__ perm,
                          const int64_t *__restrict__ inner, const double *__restrict__ scale, int64_t n, int64_t nrhs)
{
    const int64_t total = n * nrhs;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        int64_t k = e % n, r = e / n;
        int64_t s = inner ? inner[k] : k;
        x[(perm ? perm[s] : s) + r * ldx] = scale ? scal(v[e], scale[s]) : v[e];
    }
}

// Y[k] = Wr[p_lu[k]]: the forward result in pivot order
template <typename T>
__global__ void k_gather_rows(T *__restrict__ Y, const T *__restrict__ Wr, const int64_t *__restrict__ p_lu, int64_t n, int64_t nrhs)
{
    const int64_t total = n * nrhs;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        int64_t k = e % n, r = e / n;
        Y[e] = Wr[p_lu[k] + r * n];
    }
}

// forward sweep with L through one front in shared memory (one CTA): gather the front's rows of the right-hand sides;
// the unit lower L11 solve by a warp per right-hand side (shared-memory column sweep, __syncwarp per step); the L21
// update by the whole CTA; scatter back
template <typename T>
__global__ void __launch_bounds__(256) k_fwdL2(const T *__restrict__ L, int64_t nrows, int64_t npiv,
                                               const int64_t *__restrict__ rowid, T *__restrict__ Wr, int64_t n, int64_t nrhs)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *v = reinterpret_cast<T *>(smem_raw);           // nrows x nrhs
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int64_t e = threadIdx.x; e < nrows * nrhs; e += blockDim.x) v[e] = Wr[rowid[e % nrows] + (e / nrows) * n];
    __syncthreads();
    const int64_t np = npiv < nrows ? npiv : nrows;
    for (int64_t r = warp; r < nrhs; r += nw) {
        T *vr = v + r * nrows;
        for (int64_t i = 0; i < np; i++) {
            const T xi = vr[i];
            if (!is_zero(xi))
                for (int64_t rr = i + 1 + lane; rr < np; rr += 32) vr[rr] = sub(vr[rr], mul(L[rr + i * nrows], xi));
            __syncwarp();
        }
    }
    __syncthreads();
    for (int64_t e = threadIdx.x; e < (nrows - np) * nrhs; e += blockDim.x) {
        const int64_t rr = np + e % (nrows - np), r = e / (nrows - np);
        T acc = VT<T>::zero();
        for (int64_t i = 0; i < np; i++) acc = add(acc, mul(L[rr + i * nrows], v[i + r * nrows]));
        v[rr + r * nrows] = sub(v[rr + r * nrows], acc);
    }
    __syncthreads();
    for (int64_t e = threadIdx.x; e < nrows * nrhs; e += blockDim.x) Wr[rowid[e % nrows] + (e / nrows) * n] = v[e];
}

// forward sweep with L through one front (one CTA, npiv <= 64): copy the front's L block into shared memory (cp.async,
// all copies in flight at once: the whole nrows x npiv block when `whole`, else the L11 block) while gathering the front's
// rows of the right-hand sides; the L11 solve by a warp per right-hand side with the vector in registers (rows lane and
// lane + 32; the pivot value broadcast by shuffle); the L21 update by the whole CTA; scatter back
template <typename T>
__global__ void __launch_bounds__(512) k_fwdL3(const T *__restrict__ L, int64_t nrows, int64_t npiv,
                                               const int64_t *__restrict__ rowid, T *__restrict__ Wr, int64_t n, int64_t nrhs,
                                               int whole)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *v = reinterpret_cast<T *>(smem_raw);           // nrows x nrhs
    T *sL = v + nrows * nrhs;                         // whole: nrows x np (ld nrows), else np x np (ld np)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int np = (int)(npiv < nrows ? npiv : nrows);
    const int64_t ld = whole ? nrows : np;
    if (whole)
        for (int64_t e = threadIdx.x; e < nrows * np; e += blockDim.x) cp_async_el(sL + e, L + e);
    else
        for (int e = threadIdx.x; e < np * np; e += blockDim.x) cp_async_el(sL + e, L + (e % np) + (int64_t)(e / np) * nrows);
    pdl_wait();                                       // the previous front's sweep has written Wr (the L copy runs on)
    pdl_trigger();
    for (int64_t e = threadIdx.x; e < nrows * nrhs; e += blockDim.x) v[e] = Wr[rowid[e % nrows] + (e / nrows) * n];
    cp_async_wait_all();
    __syncthreads();
    for (int64_t r = warp; r < nrhs; r += nw) {
        T *vr = v + r * nrows;
        T a = lane < np ? vr[lane] : VT<T>::zero();
        T b = lane + 32 < np ? vr[lane + 32] : VT<T>::zero();
        for (int i = 0; i < np; i++) {
            const T xi = shfl_v<T>(i < 32 ? a : b, i & 31);
            const T *col = sL + i * ld;
            if (lane > i && lane < np) a = sub(a, mul(col[lane], xi));
            if (lane + 32 > i && lane + 32 < np) b = sub(b, mul(col[lane + 32], xi));
        }
        if (lane < np) vr[lane] = a;
        if (lane + 32 < np) vr[lane + 32] = b;
    }
    __syncthreads();
    for (int64_t e = threadIdx.x; e < (nrows - np) * nrhs; e += blockDim.x) {
        const int64_t rr = np + e % (nrows - np), r = e / (nrows - np);
        T acc = VT<T>::zero();
        if (whole)
            for (int i = 0; i < np; i++) acc = add(acc, mul(sL[rr + i * nrows], v[i + r * nrows]));
        else
            for (int64_t i = 0; i < np; i++) acc = add(acc, mul(L[rr + i * nrows], v[i + r * nrows]));
        v[rr + r * nrows] = sub(v[rr + r * nrows], acc);
    }
    __syncthreads();
    for (int64_t e = threadIdx.x; e < nrows * nrhs; e += blockDim.x) Wr[rowid[e % nrows] + (e / nrows) * n] = v[e];
}


// forward sweep with L through one front (one CTA), in row space: for each pivot column i, the rows below it lose
// L[row, i] times the pivot row's value
// The forward sweep through a large front in two launches.  k_fwdL11 (one CTA): the pivot rows' values are gathered
// (rowid), solved with the unit-lower L11 (a warp per right-hand side, the rows of a step spread over the lanes),
// written back and copied to xs (np x nrhs, ld np).  k_fwdL21 (many CTAs, a thread per row below the pivots): the rows
// rr >= np take y[rr] -= sum_i L[rr, i] xs[i] with L read down its columns (coalesced) and xs staged in shared memory
// (np * nrhs values).  The same operations as one front's forward substitution, the L21 product spread over the GPU.
// A triangular solve of a large front's pivot block on the vector x (np x nrhs, ld np, shared memory) by blocks of 64:
// each diagonal block staged in shared memory (sT, 64 x 64) and solved with the block's rows in two registers per lane (a
// warp per right-hand side), then the other rows updated by the block's solved values (L read down its columns).
// Lower (UPPER false): the unit-lower L11, forward.  Upper: U11 with its diagonal, backward (a zero diagonal entry is
// reported as ST_SOLVE_ZERO).  The block is L[r + c * ld] (the front's L block: U11 on and above the diagonal).
template <typename T, bool UPPER>
__device__ void blk_trisolve(const T *__restrict__ L, int64_t ld, int np, T *x, int64_t nrhs, T *sT, T *dinv, DevStatus *st,
                             int64_t f, int *zflag = nullptr)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    const int nb = (np + 63) / 64;
    for (int bb = 0; bb < nb; bb++) {
        const int bi = UPPER ? nb - 1 - bb : bb;
        const int r0 = bi * 64, w = np - r0 < 64 ? np - r0 : 64;
        // the diagonal block into shared memory, eight loads in flight per thread
        for (int e0 = tid; e0 < w * w; e0 += 8 * blockDim.x) {
            T lv[8];
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const int e = e0 + q * blockDim.x;
                lv[q] = e < w * w ? L[(r0 + e % w) + (int64_t)(r0 + e / w) * ld] : VT<T>::zero();
            }
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const int e = e0 + q * blockDim.x;
                if (e < w * w) sT[e % w + (e / w) * 64] = lv[q];
            }
        }
        if (UPPER)
            for (int i = tid; i < w; i += blockDim.x) {
                const T d = L[(r0 + i) + (int64_t)(r0 + i) * ld];
                if (is_zero(d)) { set_status(st, ST_SOLVE_ZERO, f + r0 + i, 0, 0); if (zflag) *zflag = 1; }
                dinv[i] = is_zero(d) ? VT<T>::zero() : recip(d);
            }
        __syncthreads();
        // zflag (shared, cleared by the caller): this front's own zero diagonal, the same answer for every thread while
        // other CTAs may be writing the status word
        if (UPPER && (zflag ? *zflag != 0 : st->code == ST_SOLVE_ZERO)) return;
        for (int64_t r = warp; r < nrhs; r += nw) {
            T *xr = x + r * np + r0;
            T a = lane < w ? xr[lane] : VT<T>::zero(), b = lane + 32 < w ? xr[lane + 32] : VT<T>::zero();
            if (!UPPER) {
                for (int i = 0; i < w; i++) {
                    const T xi = shfl_v<T>(i < 32 ? a : b, i & 31);
                    if (lane > i && lane < w) a = sub(a, mul(sT[lane + i * 64], xi));
                    if (lane + 32 > i && lane + 32 < w) b = sub(b, mul(sT[lane + 32 + i * 64], xi));
                }
            } else {
                for (int i = w - 1; i >= 0; i--) {
                    const T xi = mul(shfl_v<T>(i < 32 ? a : b, i & 31), dinv[i]);
                    if (lane == (i & 31)) { if (i < 32) a = xi; else b = xi; }
                    if (lane < i) a = sub(a, mul(sT[lane + i * 64], xi));
                    if (lane + 32 < i) b = sub(b, mul(sT[lane + 32 + i * 64], xi));
                }
            }
            if (lane < w) xr[lane] = a;
            if (lane + 32 < w) xr[lane + 32] = b;
        }
        __syncthreads();
        const int o0 = UPPER ? 0 : r0 + w, o1 = UPPER ? r0 : np;
        if (o1 > o0) {
            // a thread per (row, block of 8 right-hand sides): L's row loaded once for the 8, sixteen loads in flight;
            // each sum in k order
            const int nrb = (int)((nrhs + 7) / 8);
            for (int e = tid; e < (o1 - o0) * nrb; e += blockDim.x) {
                const int row = o0 + e % (o1 - o0), rb0 = 8 * (e / (o1 - o0));
                const int rb = nrhs - rb0 < 8 ? (int)(nrhs - rb0) : 8;
                const T *Lr = L + row + (int64_t)r0 * ld;
                T acc[8];
#pragma unroll
                for (int r = 0; r < 8; r++) acc[r] = VT<T>::zero();
                for (int k0 = 0; k0 < w; k0 += 16) {
                    T lv[16];
#pragma unroll
                    for (int q = 0; q < 16; q++) lv[q] = k0 + q < w ? Lr[(int64_t)(k0 + q) * ld] : VT<T>::zero();
#pragma unroll
                    for (int q = 0; q < 16; q++)
                        if (k0 + q < w)
#pragma unroll
                            for (int r = 0; r < 8; r++)
                                if (r < rb) acc[r] = add(acc[r], mul(lv[q], x[(int64_t)(rb0 + r) * np + r0 + k0 + q]));
                }
#pragma unroll
                for (int r = 0; r < 8; r++)
                    if (r < rb) x[(int64_t)(rb0 + r) * np + row] = sub(x[(int64_t)(rb0 + r) * np + row], acc[r]);
            }
        }
        __syncthreads();
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_fwdL11(const T *__restrict__ L, int64_t nrows, int64_t np,
                                                const int64_t *__restrict__ rowid, T *__restrict__ Wr, int64_t n, int64_t nrhs,
                                                T *__restrict__ xs)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *v = reinterpret_cast<T *>(smem_raw);           // np x nrhs
    T *sT = v + np * nrhs;                            // 64 x 64
    for (int64_t e = threadIdx.x; e < np * nrhs; e += blockDim.x) v[e] = Wr[rowid[e % np] + (e / np) * n];
    __syncthreads();
    blk_trisolve<T, false>(L, nrows, (int)np, v, nrhs, sT, nullptr, nullptr, 0);
    for (int64_t e = threadIdx.x; e < np * nrhs; e += blockDim.x) {
        Wr[rowid[e % np] + (e / np) * n] = v[e];
        xs[e] = v[e];
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_fwdL21(const T *__restrict__ L, int64_t nrows, int64_t np,
                                                const int64_t *__restrict__ rowid, T *__restrict__ Wr, int64_t n, int64_t nrhs,
                                                const T *__restrict__ xs)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *x = reinterpret_cast<T *>(smem_raw);           // np x nrhs
    for (int64_t e = threadIdx.x; e < np * nrhs; e += blockDim.x) x[e] = xs[e];
    __syncthreads();
    const int64_t rr = np + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (rr >= nrows) return;
    const int64_t o = rowid[rr];
    for (int64_t r = 0; r < nrhs; r++) {
        const T *xr = x + r * np;
        T acc = VT<T>::zero();
        for (int64_t i = 0; i < np; i++) acc = add(acc, mul(L[rr + i * nrows], xr[i]));
        Wr[o + r * n] = sub(Wr[o + r * n], acc);
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_fwdL(const T *__restrict__ L, int64_t nrows, int64_t npiv,
                                              const int64_t *__restrict__ rowid, T *__restrict__ Wr, int64_t n, int64_t nrhs)
{
    for (int64_t i = 0; i < npiv && i < nrows; i++) {
        for (int64_t e = threadIdx.x; e < (nrows - i - 1) * nrhs; e += blockDim.x) {
            const int64_t rr = i + 1 + e % (nrows - i - 1), r = e / (nrows - i - 1);
            const T xi = Wr[rowid[i] + r * n];
            if (is_zero(xi)) continue;
            T *y = Wr + rowid[rr] + r * n;
            *y = sub(*y, mul(L[rr + i * nrows], xi));
        }
        __syncthreads();
    }
}

// backward sweep with U, step 1: partial sums of U12 x_cb over column chunks, part[chunk][i + r * npiv]; lanes over the
// pivot rows (coalesced reads of each U12 column), warps over the chunk's columns, a shared-memory reduction per chunk
template <typename T>
__global__ void __launch_bounds__(256) k_u12_gemv(const T *__restrict__ U12, int64_t npiv, int64_t ncb,
                                                  const int64_t *__restrict__ cbcols, const T *__restrict__ X, int64_t n,
                                                  int64_t nrhs, int64_t chunk, T *__restrict__ part)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *red = reinterpret_cast<T *>(smem_raw);         // (blockDim / 32) x npiv
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int64_t c0 = blockIdx.x * chunk, c1 = c0 + chunk < ncb ? c0 + chunk : ncb;
    for (int64_t r = 0; r < nrhs; r++) {
        for (int64_t i0 = 0; i0 < npiv; i0 += 32) {
            const int64_t i = i0 + lane;
            T acc = VT<T>::zero();
            if (i < npiv)
                for (int64_t c = c0 + warp; c < c1; c += nw) acc = add(acc, mul(U12[i + c * npiv], X[cbcols[c] + r * n]));
            if (i < npiv) red[warp * npiv + i] = acc;
        }
        __syncthreads();
        for (int64_t i = threadIdx.x; i < npiv; i += blockDim.x) {
            T s = VT<T>::zero();
            for (int q = 0; q < nw; q++) s = add(s, red[q * npiv + i]);
            part[blockIdx.x * npiv * nrhs + i + r * npiv] = s;
        }
        __syncthreads();
    }
}

// backward sweep with U, step 2 (one CTA): s = y - the partial sums (all threads), then x = U11^-1 s by a warp per
// right-hand side (column sweep from the last pivot, __syncwarp per step)
template <typename T>
__global__ void __launch_bounds__(256) k_bwdU(const T *__restrict__ L, int64_t nrows, int64_t npiv, int64_t f,
                                              const T *__restrict__ part, int64_t nchunk, const T *__restrict__ Y,
                                              T *__restrict__ X, int64_t n, int64_t nrhs, DevStatus *st)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *s = reinterpret_cast<T *>(smem_raw);           // npiv * nrhs
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int64_t e = threadIdx.x; e < npiv * nrhs; e += blockDim.x) {
        const int64_t i = e % npiv, r = e / npiv;
        T v = Y[f + i + r * n];
        for (int64_t q = 0; q < nchunk; q++) v = sub(v, part[q * npiv * nrhs + e]);
        s[e] = v;
    }
    T *dinv = s + npiv * nrhs;                        // 1 / U[i, i], computed in parallel
    for (int64_t i = threadIdx.x; i < npiv; i += blockDim.x) {
        const T d = L[i + i * nrows];
        if (is_zero(d)) set_status(st, ST_SOLVE_ZERO, f + i, 0, 0);
        dinv[i] = is_zero(d) ? VT<T>::zero() : recip(d);
    }
    __syncthreads();
    if (st->code == ST_SOLVE_ZERO) return;
    for (int64_t r = warp; r < nrhs; r += nw) {
        T *sr = s + r * npiv;
        for (int64_t i = npiv - 1; i >= 0; i--) {
            const T xi = mul(sr[i], dinv[i]);
            __syncwarp();
            if (lane == 0) sr[i] = xi;
            for (int64_t j = lane; j < i; j += 32) sr[j] = sub(sr[j], mul(L[j + i * nrows], xi));
            __syncwarp();
        }
    }
    __syncthreads();
    for (int64_t e = threadIdx.x; e < npiv * nrhs; e += blockDim.x) {
        const int64_t i = e % npiv, r = e / npiv;
        X[f + i + r * n] = s[e];
    }
}

// backward sweep with U through one front, in one launch.  Every CTA forms the partial products U12[:, chunk] x_cb of its
// chunk of contribution-block columns, for blocks of up to 8 right-hand sides: thread (row i = tid % 64, column group
// tid / 64) reads U12 in double-buffered batches of 16 columns (32 loads in flight per thread; each U12 entry read once
// per block of right-hand sides), the x values of a 256-column tile staged in shared memory.  The last CTA to finish (the
// status word's ticket, after a fence) copies U11 into shared memory (cp.async) while it sums the partials in chunk order,
// subtracts them from y and solves with U11: a warp per right-hand side with the vector in registers (npiv <= 64), else
// in shared memory.  The ticket is returned to 0 for the next launch.
// The backward sweep through a large front (npiv > 64): y = Y[f ..] minus the U12 partial sums of k_u12_gemv (in chunk
// order), then U11 by 64-row blocks (blk_trisolve)
template <typename T>
__global__ void __launch_bounds__(256) k_bwdU_blk(const T *__restrict__ L, int64_t nrows, int64_t npiv, int64_t f,
                                                  const T *__restrict__ part, int64_t nchunk, const T *__restrict__ Y,
                                                  T *__restrict__ X, int64_t n, int64_t nrhs, DevStatus *st)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *s = reinterpret_cast<T *>(smem_raw);           // npiv * nrhs
    T *sT = s + npiv * nrhs;                          // 64 x 64
    T *dinv = sT + 64 * 64;                           // 64
    for (int64_t e = threadIdx.x; e < npiv * nrhs; e += blockDim.x) {
        T v = Y[f + e % npiv + (e / npiv) * n];
        for (int64_t q = 0; q < nchunk; q++) v = sub(v, part[q * npiv * nrhs + e]);
        s[e] = v;
    }
    __syncthreads();
    blk_trisolve<T, true>(L, nrows, (int)npiv, s, nrhs, sT, dinv, st, f);
    if (st->code == ST_SOLVE_ZERO) return;
    for (int64_t e = threadIdx.x; e < npiv * nrhs; e += blockDim.x) X[f + e % npiv + (e / npiv) * n] = s[e];
}

template <typename T>
__global__ void __launch_bounds__(256) k_bwdU_fused(const T *__restrict__ L, int64_t nrows, int64_t npiv, int64_t f,
                                                    const T *__restrict__ U12, int64_t ncb, const int64_t *__restrict__ cbcols,
                                                    int64_t chunk, T *__restrict__ part, const T *__restrict__ Y,
                                                    T *__restrict__ X, int64_t n, int64_t nrhs, DevStatus *st)
{
    constexpr int RB = 8, CT = 256, UB = 16;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int last;
    const int tid = threadIdx.x, ri = tid & 63, cg = tid >> 6;
    const int lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    const int64_t G = gridDim.x;
    const int64_t c0 = blockIdx.x * chunk, c1 = c0 + chunk < ncb ? c0 + chunk : ncb;
    T *xs = reinterpret_cast<T *>(smem_raw);          // CT x RB
    T *red = xs + CT * RB;                            // 4 x 64 x RB
    for (int64_t r0 = 0; r0 < nrhs; r0 += RB) {
        const int rb = nrhs - r0 < RB ? (int)(nrhs - r0) : RB;
        for (int64_t i0 = 0; i0 < npiv; i0 += 64) {
            const int64_t i = i0 + ri;
            const bool row_ok = i < npiv;
            T acc[RB];
#pragma unroll
            for (int r = 0; r < RB; r++) acc[r] = VT<T>::zero();
            for (int64_t t0 = c0; t0 < c1; t0 += CT) {
                const int ct = c1 - t0 < CT ? (int)(c1 - t0) : CT;
                const T *u = U12 + i + t0 * npiv;
                T ucur[UB], unext[UB];
#pragma unroll
                for (int k = 0; k < UB; k++) {
                    const int cc = cg + 4 * k;
                    ucur[k] = row_ok && cc < ct ? u[(int64_t)cc * npiv] : VT<T>::zero();
                }
                __syncthreads();
                for (int e = tid; e < ct * rb; e += blockDim.x) {
                    const int cc = e % ct, r = e / ct;
                    xs[cc + r * CT] = X[cbcols[t0 + cc] + (r0 + r) * n];
                }
                __syncthreads();
                for (int kb = 0; kb < ct; kb += 4 * UB) {
                    const bool more = kb + 4 * UB < ct;
                    if (more) {
#pragma unroll
                        for (int k = 0; k < UB; k++) {
                            const int cc = kb + 4 * UB + cg + 4 * k;
                            unext[k] = row_ok && cc < ct ? u[(int64_t)cc * npiv] : VT<T>::zero();
                        }
                    }
#pragma unroll
                    for (int k = 0; k < UB; k++) {
                        const int cc = kb + cg + 4 * k;
                        if (cc < ct) {
#pragma unroll
                            for (int r = 0; r < RB; r++)
                                if (r < rb) acc[r] = add(acc[r], mul(ucur[k], xs[cc + r * CT]));
                        }
                    }
                    if (more) {
#pragma unroll
                        for (int k = 0; k < UB; k++) ucur[k] = unext[k];
                    }
                }
            }
            __syncthreads();
#pragma unroll
            for (int r = 0; r < RB; r++)
                if (r < rb) red[(cg * 64 + ri) * RB + r] = acc[r];
            __syncthreads();
            for (int e = tid; e < 64 * rb; e += blockDim.x) {
                const int rr = e & 63, r = e >> 6;
                if (i0 + rr < npiv) {
                    T sm = red[rr * RB + r];
                    sm = add(sm, red[(64 + rr) * RB + r]);
                    sm = add(sm, red[(128 + rr) * RB + r]);
                    sm = add(sm, red[(192 + rr) * RB + r]);
                    part[blockIdx.x * npiv * nrhs + (i0 + rr) + (r0 + r) * npiv] = sm;
                }
            }
        }
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) last = atomicAdd(&st->ticket, 1u) == (unsigned)(G - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the last CTA
    const int np = (int)npiv;
    const bool reg = npiv <= 64;
    const int64_t E = npiv * nrhs;
    T *s = reinterpret_cast<T *>(smem_raw);           // npiv * nrhs
    T *dinv = s + E;                                  // npiv
    T *ps = dinv + npiv;                              // 4 x 64 partial sums
    T *sU = ps + 256;                                 // U11 (npiv <= 64): sU[j + i * np] = U[j, i]
    if (reg)
        for (int e = tid; e < np * np; e += blockDim.x) cp_async_el(sU + e, L + (e % np) + (int64_t)(e / np) * nrows);
    for (int64_t e0 = 0; e0 < E; e0 += 64) {
        const int64_t e = e0 + ri;
        T v = VT<T>::zero();
        if (e < E) {
            const T *pp = part + e;
            for (int64_t q0 = cg; q0 < G; q0 += 4 * UB) {
                T pv[UB];
#pragma unroll
                for (int k = 0; k < UB; k++) {
                    const int64_t q = q0 + 4 * k;
                    pv[k] = q < G ? ldcg_v(pp + q * E) : VT<T>::zero();
                }
#pragma unroll
                for (int k = 0; k < UB; k++) v = add(v, pv[k]);
            }
        }
        ps[cg * 64 + ri] = v;
        __syncthreads();
        if (tid < 64 && e < E) {
            const int64_t ii = e % npiv, r = e / npiv;
            T t = add(add(ps[tid], ps[64 + tid]), add(ps[128 + tid], ps[192 + tid]));
            s[e] = sub(Y[f + ii + r * n], t);
        }
        __syncthreads();
    }
    for (int64_t ii = tid; ii < npiv; ii += blockDim.x) {
        const T d = L[ii + ii * nrows];
        if (is_zero(d)) set_status(st, ST_SOLVE_ZERO, f + ii, 0, 0);
        dinv[ii] = is_zero(d) ? VT<T>::zero() : recip(d);
    }
    if (tid == 0) st->ticket = 0u;
    cp_async_wait_all();
    __syncthreads();
    if (st->code == ST_SOLVE_ZERO) return;
    if (reg) {
        // U11's columns scaled by the reciprocal diagonal (off the sweep's chain): s_j -= (U_ji / u_ii) s_i, x = s / u
        for (int e = tid; e < np * np; e += blockDim.x) sU[e] = mul(sU[e], dinv[e / np]);
        __syncthreads();
        for (int64_t r = warp; r < nrhs; r += nw) {
            T a = lane < np ? s[lane + r * npiv] : VT<T>::zero();
            T b = lane + 32 < np ? s[lane + 32 + r * npiv] : VT<T>::zero();
            for (int ii = np - 1; ii >= 0; ii--) {
                const T *col = sU + ii * np;
                const T si = shfl_v<T>(ii < 32 ? a : b, ii & 31);
                if (ii >= 32) {
                    if (lane < ii - 32) b = sub(b, mul(col[lane + 32], si));
                    a = sub(a, mul(col[lane], si));
                } else if (lane < ii) a = sub(a, mul(col[lane], si));
            }
            if (lane < np) X[f + lane + r * n] = mul(a, dinv[lane]);
            if (lane + 32 < np) X[f + lane + 32 + r * n] = mul(b, dinv[lane + 32]);
        }
        return;
    }
    for (int64_t r = warp; r < nrhs; r += nw) {
        T *sr = s + r * npiv;
        for (int64_t ii = npiv - 1; ii >= 0; ii--) {
            const T xi = mul(sr[ii], dinv[ii]);
            __syncwarp();
            if (lane == 0) sr[ii] = xi;
            for (int64_t j = lane; j < ii; j += 32) sr[j] = sub(sr[j], mul(L[j + ii * nrows], xi));
            __syncwarp();
        }
    }
    __syncthreads();
    for (int64_t e = tid; e < npiv * nrhs; e += blockDim.x) {
        const int64_t ii = e % npiv, r = e / npiv;
        X[f + ii + r * n] = s[e];
    }
}

// Backward sweep through the dense chain (fronts of nb pivots from column f0, each with all columns to its right), one
// launch per front k, column-oriented: every CTA subtracts U[:, the nb columns of front k + 1] x_{k+1} from its rows of
// the chain above front k + 1 (each row's U12 entries read once for all right-hand sides; no cross-CTA sums), then the
// last CTA to finish (the status word's ticket) solves front k's U11 with its now complete rows, the columns of U11
// scaled by the reciprocal diagonal as in k_bwdU_fused.  jk1 < 0: front k is the last one (no update).
template <typename T>
__global__ void __launch_bounds__(512) k_chain_bwd(const T *__restrict__ Ua, const int64_t *__restrict__ cU_off, int64_t f0,
                                                   int64_t nb, int64_t jk1, int npk1, const T *__restrict__ Lk, int64_t nrowsk,
                                                   int64_t fk, int npk, T *__restrict__ Y, T *__restrict__ X, int64_t n,
                                                   int64_t nrhs, DevStatus *st)
{
    constexpr int RB = 8;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int last;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    T *xs = reinterpret_cast<T *>(smem_raw);          // x of front k + 1: column cc of rhs t at XS(cc, t)
    // each 16-column group padded by one element, so that the four lanes of a row (16 columns apart) hit different banks
    const int xld = npk1 + (npk1 + 15) / 16;
    auto XS = [&](int cc, int64_t t) -> int64_t { return cc + (cc >> 4) + t * xld; };
    const int q = lane & 3;
    const int64_t fk1 = jk1 >= 0 ? f0 + jk1 * nb : 0, R = jk1 >= 0 ? fk1 - f0 : 0;
    const int64_t nwarp_all = (int64_t)gridDim.x * nw;
    // four lanes per row, sixteen of front k + 1's columns each (all their loads in flight at once); the lanes' sums
    // are combined by shuffles in a fixed order.  The first rows' U12 entries are loaded before waiting for the previous
    // front's launch (U does not change during the solve).
    T uv[16];
    auto load_u = [&](int64_t base) {
        const int64_t r = base + (lane >> 2);
        const bool on = r < R;
        const int64_t j = on ? r / nb : 0, i = on ? r % nb : 0;
        const T *u = Ua + cU_off[j] + i + (fk1 - (f0 + j * nb) - nb) * nb;      // U12_j[i, column fk1]
#pragma unroll
        for (int c = 0; c < 16; c++) {
            const int cc = q * 16 + c;
            uv[c] = on && cc < npk1 ? u[(int64_t)cc * nb] : VT<T>::zero();
        }
    };
    const int64_t base0 = (blockIdx.x * (int64_t)nw + warp) * 8;
    if (jk1 >= 0 && base0 < R) load_u(base0);
    pdl_wait();                                       // the previous front's x is written
    pdl_trigger();
    if (jk1 >= 0) {
        for (int64_t e = tid; e < npk1 * nrhs; e += blockDim.x) xs[XS((int)(e % npk1), e / npk1)] = X[fk1 + e % npk1 + (e / npk1) * n];
        __syncthreads();
        for (int64_t base = base0; base < R; base += nwarp_all * 8) {
            if (base != base0) load_u(base);
            const int64_t r = base + (lane >> 2);
            const bool on = r < R;
            for (int64_t r0 = 0; r0 < nrhs; r0 += RB) {
                const int rb = nrhs - r0 < RB ? (int)(nrhs - r0) : RB;
                T acc[RB];
#pragma unroll
                for (int t = 0; t < RB; t++) acc[t] = VT<T>::zero();
#pragma unroll
                for (int c = 0; c < 16; c++) {
                    const int cc = q * 16 + c;
                    if (cc < npk1) {
#pragma unroll
                        for (int t = 0; t < RB; t++)
                            if (t < rb) acc[t] = add(acc[t], mul(uv[c], xs[XS(cc, r0 + t)]));
                    }
                }
#pragma unroll
                for (int t = 0; t < RB; t++) {
                    acc[t] = add(acc[t], shfl_xor_v<T>(acc[t], 1));
                    acc[t] = add(acc[t], shfl_xor_v<T>(acc[t], 2));
                }
                if (on && q == 0) {
#pragma unroll
                    for (int t = 0; t < RB; t++)
                        if (t < rb) { T *y = Y + f0 + r + (r0 + t) * n; *y = sub(*y, acc[t]); }
                }
            }
        }
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) last = atomicAdd(&st->ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the last CTA: front k's rows of Y are complete; x_k = U11^-1 y_k
    T *s = reinterpret_cast<T *>(smem_raw);           // npk x nrhs
    T *dinv = s + npk * nrhs;                         // npk
    T *sU = dinv + npk;                               // npk x npk: sU[j + i * npk] = U[j, i] / U[i, i]
    for (int e = tid; e < npk * npk; e += blockDim.x) cp_async_el(sU + e, Lk + (e % npk) + (int64_t)(e / npk) * nrowsk);
    for (int64_t e = tid; e < npk * nrhs; e += blockDim.x) s[e] = ldcg_v(Y + fk + e % npk + (e / npk) * n);
    for (int i = tid; i < npk; i += blockDim.x) {
        const T d = Lk[i + (int64_t)i * nrowsk];
        if (is_zero(d)) set_status(st, ST_SOLVE_ZERO, fk + i, 0, 0);
        dinv[i] = is_zero(d) ? VT<T>::zero() : recip(d);
    }
    if (tid == 0) st->ticket = 0u;
    cp_async_wait_all();
    __syncthreads();
    if (st->code == ST_SOLVE_ZERO) return;
    for (int e = tid; e < npk * npk; e += blockDim.x) sU[e] = mul(sU[e], dinv[e / npk]);
    __syncthreads();
    for (int64_t r = warp; r < nrhs; r += nw) {
        T a = lane < npk ? s[lane + r * npk] : VT<T>::zero();
        T b = lane + 32 < npk ? s[lane + 32 + r * npk] : VT<T>::zero();
        for (int ii = npk - 1; ii >= 0; ii--) {
            const T *col = sU + ii * npk;
            const T si = shfl_v<T>(ii < 32 ? a : b, ii & 31);
            if (ii >= 32) {
                if (lane < ii - 32) b = sub(b, mul(col[lane + 32], si));
                a = sub(a, mul(col[lane], si));
            } else if (lane < ii) a = sub(a, mul(col[lane], si));
        }
        if (lane < npk) X[fk + lane + r * n] = mul(a, dinv[lane]);
        if (lane + 32 < npk) X[fk + lane + 32 + r * n] = mul(b, dinv[lane + 32]);
    }
}

// the sum over a warp by a fixed butterfly (every lane gets the same result)
template <typename T> __device__ __forceinline__ T shfl_sum(T v)
{
    for (int m = 16; m > 0; m >>= 1) v = add(v, shfl_xor_v<T>(v, m));
    return v;
}

// The L21^T product of a large front's transposed backward sweep over many CTAs: CTA c sums its chunk of rows,
// part[c][r][i] = sum over rows rr of its chunk of L[rr, i] (conjugated for CJ) v[pinv[rowid[rr]], r], a warp per pivot
// column with its lanes down the rows (coalesced) and a fixed butterfly; k_bwdLt adds the chunks in order.
template <typename T, bool CJ>
__global__ void __launch_bounds__(256) k_ltdot(const T *__restrict__ L, int64_t nrows, int64_t npiv,
                                               const int64_t *__restrict__ rowid, const int64_t *__restrict__ pinv,
                                               const T *__restrict__ V, int64_t n, int64_t nrhs, int64_t chunk,
                                               T *__restrict__ part)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int64_t r0 = npiv + blockIdx.x * chunk, r1 = r0 + chunk < nrows ? r0 + chunk : nrows;
    T *pc = part + (int64_t)blockIdx.x * npiv * nrhs;
    for (int64_t e = warp; e < npiv * nrhs; e += nw) {
        const int64_t i = e % npiv, r = e / npiv;
        T acc = VT<T>::zero();
        for (int64_t rr = r0 + lane; rr < r1; rr += 32) {
            T l = L[rr + i * nrows];
            if (CJ) l = conjv(l);
            acc = add(acc, mul(l, V[pinv[rowid[rr]] + r * n]));
        }
        acc = shfl_sum(acc);
        if (lane == 0) pc[e] = acc;
    }
}

// transposed solves: forward with U^T (U^H when conj) through one front, step 1 (one CTA): z = U11^-T w[f ..] by a warp
// per right-hand side
template <typename T, bool CJ>
__global__ void __launch_bounds__(256) k_fwdUt2(const T *__restrict__ L, int64_t nrows, int64_t npiv, int64_t f,
                                                T *__restrict__ Wc, int64_t n, int64_t nrhs, DevStatus *st)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *dinv = reinterpret_cast<T *>(smem_raw);         // 1 / U[i, i] (conjugated for U^H), computed in parallel
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int64_t i = threadIdx.x; i < npiv; i += blockDim.x) {
        T d = L[i + i * nrows];
        if (CJ) d = conjv(d);
        if (is_zero(d)) set_status(st, ST_SOLVE_ZERO, f + i, 0, 0);
        dinv[i] = is_zero(d) ? VT<T>::zero() : recip(d);
    }
    __syncthreads();
    if (st->code == ST_SOLVE_ZERO) return;
    for (int64_t r = warp; r < nrhs; r += nw) {
        T *w = Wc + f + r * n;
        for (int64_t i = 0; i < npiv; i++) {
            const T zi = mul(w[i], dinv[i]);
            __syncwarp();
            if (lane == 0) w[i] = zi;
            for (int64_t j = i + 1 + lane; j < npiv; j += 32) {
                T u = L[i + j * nrows];
                if (CJ) u = conjv(u);
                w[j] = sub(w[j], mul(u, zi));
            }
            __syncwarp();
        }
    }
}


// step 2 (many CTAs, a warp per CB column): w[cbcol[c]] -= U12[:, c]^T z
template <typename T, bool CJ>
__global__ void k_ut_scatter(const T *__restrict__ U12, int64_t npiv, int64_t ncb, const int64_t *__restrict__ cbcols,
                             int64_t f, T *__restrict__ Wc, int64_t n, int64_t nrhs)
{
    const int lane = threadIdx.x & 31;
    for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < ncb; c += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        for (int64_t r = 0; r < nrhs; r++) {
            T s = VT<T>::zero();
            for (int64_t i = lane; i < npiv; i += 32) {
                T u = U12[i + c * npiv];
                if (CJ) u = conjv(u);
                s = add(s, mul(u, Wc[f + i + r * n]));
            }
            for (int o = 16; o > 0; o >>= 1) {
                if constexpr (VT<T>::cplx_) {
                    cplx t; t.x = __shfl_xor_sync(0xffffffffu, ((cplx &)s).x, o); t.y = __shfl_xor_sync(0xffffffffu, ((cplx &)s).y, o);
                    s = add(s, *(T *)&t);
                } else s = add(s, __shfl_xor_sync(0xffffffffu, s, o));
            }
            if (lane == 0) { T *w = Wc + cbcols[c] + r * n; *w = sub(*w, s); }
        }
    }
}

// backward with L^T (L^H) through one front (one CTA): V[f + i] = z_i - sum over the rows below of L[row, i] V[row's step]
template <typename T, bool CJ>
__global__ void __launch_bounds__(256) k_bwdLt(const T *__restrict__ L, int64_t nrows, int64_t npiv, int64_t f,
                                               const int64_t *__restrict__ rowid, const int64_t *__restrict__ pinv,
                                               const T *__restrict__ Z, T *__restrict__ V, int64_t n, int64_t nrhs,
                                               const T *__restrict__ part = nullptr, int nch = 0)
{
    extern __shared__ unsigned char smem_raw[];
    T *s = reinterpret_cast<T *>(smem_raw);           // npiv * nrhs
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    // s = z - L21^T v_cb: summed here from the partial sums of k_ltdot (in chunk order), or a warp per pivot column
    if (part) {
        for (int64_t e = threadIdx.x; e < npiv * nrhs; e += blockDim.x) {
            T acc = VT<T>::zero();
            for (int c = 0; c < nch; c++) acc = add(acc, part[(int64_t)c * npiv * nrhs + e]);
            s[e] = sub(Z[f + e % npiv + (e / npiv) * n], acc);
        }
    }
    for (int64_t e = warp; !part && e < npiv * nrhs; e += nw) {
        const int64_t i = e % npiv, r = e / npiv;
        T acc = VT<T>::zero();
        for (int64_t rr = npiv + lane; rr < nrows; rr += 32) {
            T l = L[rr + i * nrows];
            if (CJ) l = conjv(l);
            acc = add(acc, mul(l, V[pinv[rowid[rr]] + r * n]));
        }
        for (int o = 16; o > 0; o >>= 1) {
            if constexpr (VT<T>::cplx_) {
                cplx t; t.x = __shfl_xor_sync(0xffffffffu, ((cplx &)acc).x, o); t.y = __shfl_xor_sync(0xffffffffu, ((cplx &)acc).y, o);
                acc = add(acc, *(T *)&t);
            } else acc = add(acc, __shfl_xor_sync(0xffffffffu, acc, o));
        }
        if (lane == 0) s[e] = sub(Z[f + i + r * n], acc);
    }
    __syncthreads();
    for (int64_t r = warp; r < nrhs; r += nw) {
        T *sr = s + r * npiv;
        for (int64_t i = npiv - 1; i >= 0; i--) {
            // s[i] final; s[j] -= L[i, j] s[i] for j < i
            const T vi = sr[i];
            for (int64_t j = lane; j < i; j += 32) {
                T l = L[i + j * nrows];
                if (CJ) l = conjv(l);
                sr[j] = sub(sr[j], mul(l, vi));
            }
            __syncwarp();
        }
    }
    __syncthreads();
    for (int64_t e = threadIdx.x; e < npiv * nrhs; e += blockDim.x) {
        const int64_t i = e % npiv, r = e / npiv;
        V[f + i + r * n] = s[e];
    }
}

// transposed solves, npiv <= 64 (one CTA): the front's U11 (or L11) block copied transposed into shared memory (ld
// npiv + 1, so that the transposing stores and the sweep's row reads are free of bank conflicts), then a warp per
// right-hand side with the vector in registers (rows lane and lane + 32)
template <typename T, bool CJ>
__device__ __forceinline__ void stage_transposed(const T *__restrict__ L, int64_t nrows, int np, T *sT)
{
    const int ld = np + 1;
    for (int e = threadIdx.x; e < np * np; e += blockDim.x) {
        const int row = e % np, col = e / np;
        T v = L[row + (int64_t)col * nrows];
        if (CJ) v = conjv(v);
        sT[col + row * ld] = v;                        // sT[j + i * ld] = block[i, j]
    }
}

// forward with U^T (U^H when conj): z_i = w_i / u_ii, then w_j -= u_ij z_i for j > i
template <typename T, bool CJ>
__global__ void __launch_bounds__(256) k_fwdUt3(const T *__restrict__ L, int64_t nrows, int64_t npiv, int64_t f,
                                                T *__restrict__ Wc, int64_t n, int64_t nrhs, DevStatus *st)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int np = (int)npiv, ld = np + 1;
    T *sT = reinterpret_cast<T *>(smem_raw);           // np x ld
    T *dinv = sT + np * ld;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    stage_transposed<T, CJ>(L, nrows, np, sT);
    for (int i = threadIdx.x; i < np; i += blockDim.x) {
        T d = L[i + (int64_t)i * nrows];
        if (CJ) d = conjv(d);
        if (is_zero(d)) set_status(st, ST_SOLVE_ZERO, f + i, 0, 0);
        dinv[i] = is_zero(d) ? VT<T>::zero() : recip(d);
    }
    __syncthreads();
    if (st->code == ST_SOLVE_ZERO) return;
    for (int64_t r = warp; r < nrhs; r += nw) {
        T *w = Wc + f + r * n;
        T a = lane < np ? w[lane] : VT<T>::zero();
        T b = lane + 32 < np ? w[lane + 32] : VT<T>::zero();
        for (int i = 0; i < np; i++) {
            const T zi = mul(shfl_v<T>(i < 32 ? a : b, i & 31), dinv[i]);
            const T *row = sT + i * ld;                 // row[j] = u_ij
            if (lane == i) a = zi;
            else if (lane > i && lane < np) a = sub(a, mul(row[lane], zi));
            if (lane + 32 == i) b = zi;
            else if (lane + 32 > i && lane + 32 < np) b = sub(b, mul(row[lane + 32], zi));
        }
        if (lane < np) w[lane] = a;
        if (lane + 32 < np) w[lane + 32] = b;
    }
}

// w[cbcol[c]] -= U12[:, c]^T z (a warp per CB column; the column's U12 entries loaded once for all right-hand sides)
template <typename T, bool CJ>
__global__ void k_ut_scatter2(const T *__restrict__ U12, int64_t npiv, int64_t ncb, const int64_t *__restrict__ cbcols,
                              int64_t f, T *__restrict__ Wc, int64_t n, int64_t nrhs)
{
    const int lane = threadIdx.x & 31;
    for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < ncb; c += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        T u0 = lane < npiv ? U12[lane + c * npiv] : VT<T>::zero();
        T u1 = lane + 32 < npiv ? U12[lane + 32 + c * npiv] : VT<T>::zero();
        if (CJ) { u0 = conjv(u0); u1 = conjv(u1); }
        for (int64_t r = 0; r < nrhs; r++) {
            const T *z = Wc + f + r * n;
            T s = lane < npiv ? mul(u0, z[lane]) : VT<T>::zero();
            if (lane + 32 < npiv) s = add(s, mul(u1, z[lane + 32]));
            for (int o = 16; o > 0; o >>= 1) s = add(s, shfl_xor_v<T>(s, o));
            if (lane == 0) { T *w = Wc + cbcols[c] + r * n; *w = sub(*w, s); }
        }
    }
}

// backward with L^T (L^H): s = z - L21^T v_cb (a warp per pivot column and right-hand side), then the unit upper
// L11^T solve from the last pivot
template <typename T, bool CJ>
__global__ void __launch_bounds__(256) k_bwdLt3(const T *__restrict__ L, int64_t nrows, int64_t npiv, int64_t f,
                                                const int64_t *__restrict__ rowid, const int64_t *__restrict__ pinv,
                                                const T *__restrict__ Z, T *__restrict__ V, int64_t n, int64_t nrhs)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int np = (int)npiv, ld = np + 1;
    T *sT = reinterpret_cast<T *>(smem_raw);           // np x ld: sT[j + i * ld] = L11[i, j]
    T *s = sT + np * ld;                               // np * nrhs
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    stage_transposed<T, CJ>(L, nrows, np, sT);
    for (int64_t e = warp; e < npiv * nrhs; e += nw) {
        const int64_t i = e % npiv, r = e / npiv;
        T acc = VT<T>::zero();
        for (int64_t rr = npiv + lane; rr < nrows; rr += 32) {
            T l = L[rr + i * nrows];
            if (CJ) l = conjv(l);
            acc = add(acc, mul(l, V[pinv[rowid[rr]] + r * n]));
        }
        for (int o = 16; o > 0; o >>= 1) acc = add(acc, shfl_xor_v<T>(acc, o));
        if (lane == 0) s[e] = sub(Z[f + i + r * n], acc);
    }
    __syncthreads();
    for (int64_t r = warp; r < nrhs; r += nw) {
        T *sr = s + r * npiv;
        T a = lane < np ? sr[lane] : VT<T>::zero();
        T b = lane + 32 < np ? sr[lane + 32] : VT<T>::zero();
        for (int i = np - 1; i >= 0; i--) {
            const T vi = shfl_v<T>(i < 32 ? a : b, i & 31);
            const T *row = sT + i * ld;                 // row[j] = L11[i, j], j < i
            if (lane < i) a = sub(a, mul(row[lane], vi));
            if (lane + 32 < i) b = sub(b, mul(row[lane + 32], vi));
        }
        if (lane < np) V[f + lane + r * n] = a;
        if (lane + 32 < np) V[f + lane + 32 + r * n] = b;
    }
}

// every value finite: the first non-finite double (by index) is reported
__global__ void k_check_finite(const double *__restrict__ d, int64_t m, DevStatus *st)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < m; q += (int64_t)gridDim.x * blockDim.x)
        if (!isfinite(d[q])) {
            atomicCAS(&st->code, 0, ST_BAD_VALUE);
            atomicMin((unsigned long long *)&st->idx, (unsigned long long)q);
        }
}

// a front with fewer rows than pivot columns: no pivot for step `step` (unless an earlier failure is recorded)
__global__ void k_set_singular(DevStatus *st, int64_t step)
{
    set_status(st, ST_SINGULAR, step, 0.0, 0.0);
}

// the inverse pivot order; nothing when the factorization stopped (p_lu is then incomplete), and indices outside [0, n)
// are never written
__global__ void k_pinv(const int64_t *__restrict__ p_lu, int64_t *__restrict__ pinv, int64_t n, const DevStatus *st)
{
    if (st->code) return;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = p_lu[k];
        if (r >= 0 && r < n) pinv[r] = k;
    }
}

// =====================================================================================================================
// iterative refinement: the residual r = b - op(A) x and the componentwise backward error, in the original coordinates
// =====================================================================================================================


// One warp per line of B = A[row_perm, :][:, col_perm]: trans 0 the rows of B (CSR: idx = B's column, the x entry
// col_perm[idx], the output row row_perm[k]), trans 1 / 2 the columns of B (CSC: idx = B's row, x entry row_perm[idx],
// the output col_perm[k]; conjugated for 2).  Entry e has the value Ax[src[e]].  The partial sums over the line are
// added by a fixed butterfly.  r = b - op(A) x; the backward error of right-hand side c, max over lines of
// |r| / (|op(A)| |x| + |b|) (moduli), goes to bits[c] by atomicMax on its bits (non-negative doubles order as their bits;
// a zero denominator with a non-zero residual counts as infinity).
template <typename T, bool CJ>
__global__ void __launch_bounds__(256) k_resid(const int64_t *__restrict__ ptr, const int64_t *__restrict__ idx,
                                               const int64_t *__restrict__ src, const T *__restrict__ Ax,
                                               const int64_t *__restrict__ outmap, const int64_t *__restrict__ inmap,
                                               const T *__restrict__ x, const T *__restrict__ b, T *__restrict__ r,
                                               int64_t n, int64_t nrhs, unsigned long long *__restrict__ bits)
{
    const int lane = threadIdx.x & 31;
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t k = w; k < n; k += nw) {
        const int64_t e0 = ptr[k], e1 = ptr[k + 1], o = outmap[k];
        for (int64_t c = 0; c < nrhs; c++) {
            const T *xc = x + c * n;
            T s = VT<T>::zero();
            double a = 0.0;
            for (int64_t e = e0 + lane; e < e1; e += 32) {
                T v = Ax[src[e]];
                if (CJ) v = conjv(v);
                const T xv = xc[inmap[idx[e]]];
                s = add(s, mul(v, xv));
                a += vabs(v) * vabs(xv);
            }
            s = shfl_sum(s);
            for (int m = 16; m > 0; m >>= 1) a += __shfl_xor_sync(0xffffffffu, a, m);
            if (lane == 0) {
                const T rr = sub(b[o + c * n], s);
                r[o + c * n] = rr;
                const double den = a + vabs(b[o + c * n]), num = vabs(rr);
                const double be = den > 0.0 ? num / den : (num > 0.0 ? __longlong_as_double(0x7ff0000000000000ll) : 0.0);
                atomicMax(bits + c, dbits(be));
            }
        }
    }
}

// ---- the captured (graph) form of the factorization: set-up done on the device instead of by host copies
// the status word cleared (idx: the largest index, so that the smallest failing one wins)
__global__ void k_clear_status(DevStatus *st, int range_guard)
{
    DevStatus h{};
    h.idx = INT64_MAX;
    if (range_guard) h.amin_bits = 0x7ff0000000000000ull;
    *st = h;
}
__global__ void k_fill(double *a, int64_t m, double v)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < m; q += (int64_t)gridDim.x * blockDim.x) a[q] = v;
}
// after k_abs_range: values whose range the host-side guard would rescale (FPLUS src/equil.c:197-241) cannot take the
// captured path, which has no host decision; they are reported (ST_RANGE) and the caller factors them the usual way
__global__ void k_range_flag(DevStatus *st)
{
    const double amax = bitsd(st->amax_bits), amin = bitsd(st->amin_bits);
    if (amax > 0.0 && (amax > 0x1p500 || amin < 0x1p-500)) atomicCAS(&st->code, 0, ST_RANGE);
}

// x += d, or x -= d (undo), over m contiguous entries
template <typename T>
__global__ void k_axpy1(T *__restrict__ x, const T *__restrict__ d, int64_t m, int undo)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x)
        x[e] = undo ? sub(x[e], d[e]) : add(x[e], d[e]);
}

// ---------------------------------------------------------------------------------------------------------------------
// Frobenius norms of the factors straight from the arenas, in two passes so that no square overflows or underflows:
// PASS 0 the largest modulus of each factor (integer maxima of the bits), PASS 1 the sum of (|x| / max)^2.  In a front's
// nrows x npiv block of the L arena (rows in the final order) an entry below the diagonal (row > column) belongs to L,
// one on or above it to U (U11); every entry of the U arena belongs to U (U12).  L's unit diagonal is added on the host.
// acc: [0] bits of max |L| (starts at 1.0: the unit diagonal), [1] bits of max |U|, [2] sum for L, [3] sum for U.
// fr: (L_off, nrows, npiv) per front; one CTA per front.
template <typename T, int PASS>
__global__ void k_lblock_norm(const T *__restrict__ La, const int64_t *__restrict__ fr, unsigned long long *acc)
{
    const int64_t off = fr[3 * blockIdx.x], nr = fr[3 * blockIdx.x + 1], np = fr[3 * blockIdx.x + 2];
    const double sl = PASS ? 1.0 / bitsd(acc[0]) : 0.0;
    const double mu = PASS ? bitsd(acc[1]) : 0.0, su = PASS ? (mu > 0.0 ? 1.0 / mu : 1.0) : 0.0;
    double a0 = 0.0, a1 = 0.0;
    for (int64_t e = threadIdx.x; e < nr * np; e += blockDim.x) {
        const int64_t i = e % nr, c = e / nr;
        const double v = vabs(La[off + e]);
        if (i > c) { if (PASS) { const double t = v * sl; a0 += t * t; } else a0 = fmax(a0, v); }
        else if (i < np) { if (PASS) { const double t = v * su; a1 += t * t; } else a1 = fmax(a1, v); }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double b0 = __shfl_xor_sync(0xffffffffu, a0, o), b1 = __shfl_xor_sync(0xffffffffu, a1, o);
        a0 = PASS ? a0 + b0 : fmax(a0, b0);
        a1 = PASS ? a1 + b1 : fmax(a1, b1);
    }
    if ((threadIdx.x & 31) == 0) {
        if (PASS) { atomicAdd((double *)&acc[2], a0); atomicAdd((double *)&acc[3], a1); }
        else { atomicMax(&acc[0], dbits(a0)); atomicMax(&acc[1], dbits(a1)); }
    }
}

template <typename T, int PASS>
__global__ void k_flat_norm(const T *__restrict__ U, int64_t m, unsigned long long *acc)
{
    const double mu = PASS ? bitsd(acc[1]) : 0.0, su = PASS ? (mu > 0.0 ? 1.0 / mu : 1.0) : 0.0;
    double a = 0.0;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x) {
        const double v = vabs(U[e]);
        if (PASS) { const double t = v * su; a += t * t; } else a = fmax(a, v);
    }
    for (int o = 16; o > 0; o >>= 1) { const double b = __shfl_xor_sync(0xffffffffu, a, o); a = PASS ? a + b : fmax(a, b); }
    if ((threadIdx.x & 31) == 0) { if (PASS) atomicAdd((double *)&acc[3], a); else atomicMax(&acc[1], dbits(a)); }
}

// ---------------------------------------------------------------------------------------------------------------------
// GMRES-IR helpers (one right-hand side at a time).  part[v * gridDim.x + chunk] = the sum over the chunk of
// conj(V_v) w (V column-major n x nv); a fixed-order tree in shared memory, the chunks summed in order on the host, so the
// products do not depend on scheduling.  Block 256.
template <typename T>
__global__ void __launch_bounds__(256) k_vdots(const T *__restrict__ V, int64_t n, const T *__restrict__ w, T *__restrict__ part)
{
    __shared__ T red[256];
    const int v = blockIdx.y;
    const T *Vv = V + (int64_t)v * n;
    T s = VT<T>::zero();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        s = add(s, mul(conjv(Vv[i]), w[i]));
    red[threadIdx.x] = s;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] = add(red[threadIdx.x], red[threadIdx.x + h]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[(int64_t)v * gridDim.x + blockIdx.x] = red[0];
}

// w -= sum_v V_v h[v] (nv columns of V, h in device memory); with scale: then w *= scale
template <typename T>
__global__ void k_vupdate(const T *__restrict__ V, int64_t n, int nv, const T *__restrict__ h, T *__restrict__ w, double scale)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        T s = w[i];
        for (int v = 0; v < nv; v++) s = sub(s, mul(V[(int64_t)v * n + i], h[v]));
        w[i] = scal(s, scale);
    }
}

// =====================================================================================================================
// the level-scheduled solve
// =====================================================================================================================
// The fronts of one level of the tree (the same height above the leaves) are independent in every sweep, so each sweep
// runs level by level: one launch for the level's small fronts (a CTA each), the others front by front.  The two
// forward sweeps pass contribution vectors up the tree instead of scattering into a global vector, so no two fronts of a
// level write the same entry and every sum is taken in a fixed order: front f's vector occupies the entries [row_off,
// row_off + nrows) (the L sweep: its rows in their final order) or [col_off, col_off + ncols) (the U^T sweep: its
// columns) of a buffer VB laid out one right-hand side after another (stride: the plan's total front rows, or its total
// front columns).  A front's vector entry gathers the right-hand side where the row (column) enters the tree, then, in
// the children's order, the children's contribution entries that land on it (the lists rsp/rsi over the plan's rows,
// csp/csi over its columns).
constexpr int SV_RC = 8;              // right-hand sides per pass of the one-CTA sweep kernels
constexpr int SVB_RC = 16;            // right-hand sides per pass over a larger front's L21 or U12
constexpr int SV_THREADS = 256;

// L sweep (trans 0) of a level's small fronts, a CTA each: the front's vector in its final row order (position k holds
// initial row perm[k]: the entering row's right-hand side, then the children's entries that land on it), x = L11^-1 v
// (the pivot rows, into Y in pivot order), then the contribution u = v[np:] - L21 x into VB
template <typename T>
__global__ void __launch_bounds__(SV_THREADS) k_sv_fwdL(const SvFront *__restrict__ fr, const int *__restrict__ list,
                                                        const T *__restrict__ La, const int64_t *__restrict__ rowinit,
                                                        const int *__restrict__ permall, const int64_t *__restrict__ rsp,
                                                        const int64_t *__restrict__ rsi, const T *__restrict__ R,
                                                        T *__restrict__ Y, T *__restrict__ VB, int64_t vstride, int64_t n,
                                                        int nrhs)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const SvFront F = fr[list[blockIdx.x]];
    const int nr = (int)F.nr, np = (int)(F.np < F.nr ? F.np : F.nr), nri = (int)F.nri, tid = threadIdx.x;
    T *v = reinterpret_cast<T *>(smem_raw);          // nr x SV_RC (ld nr)
    T *x = v + nr * SV_RC;                           // np x SV_RC (ld np)
    T *sT = x + np * SV_RC;                          // 64 x np
    const T *L = La + F.L_off;
    const int *perm = permall + F.row_off;
    pdl_wait();
    pdl_trigger();
    for (int r0 = 0; r0 < nrhs; r0 += SV_RC) {
        const int rc = nrhs - r0 < SV_RC ? nrhs - r0 : SV_RC;
        for (int e = tid; e < nr * rc; e += SV_THREADS) {
            const int k = e % nr, r = e / nr, i = F.np > 0 ? perm[k] : k;     // (a front without pivots keeps its order)
            const int64_t g = F.row_off + i, ri = rowinit[g];
            T val = (i < nri && ri >= 0) ? R[ri + (int64_t)(r0 + r) * n] : VT<T>::zero();
            for (int64_t q = rsp[g]; q < rsp[g + 1]; q++) val = add(val, VB[rsi[q] + (int64_t)(r0 + r) * vstride]);
            v[k + r * nr] = val;
        }
        __syncthreads();
        for (int e = tid; e < np * rc; e += SV_THREADS) x[e] = v[e % np + (e / np) * nr];
        __syncthreads();
        blk_trisolve<T, false>(L, nr, np, x, rc, sT, nullptr, nullptr, 0);
        for (int e = tid; e < np * rc; e += SV_THREADS) Y[F.f + e % np + (int64_t)(r0 + e / np) * n] = x[e];
        const int m = nr - np;
        for (int e = tid; e < m * rc; e += SV_THREADS) {
            const int t = e % m, r = e / m;
            T acc = VT<T>::zero();
            for (int k0 = 0; k0 < np; k0 += 8) {
                T lv[8];
#pragma unroll
                for (int q = 0; q < 8; q++) lv[q] = k0 + q < np ? L[np + t + (int64_t)(k0 + q) * nr] : VT<T>::zero();
#pragma unroll
                for (int q = 0; q < 8; q++)
                    if (k0 + q < np) acc = add(acc, mul(lv[q], x[k0 + q + r * np]));
            }
            VB[F.row_off + np + t + (int64_t)(r0 + r) * vstride] = sub(v[np + t + r * nr], acc);
        }
        __syncthreads();
    }
}

// a larger front's vector (the L sweep), in its final row order, into its own entries of VB
template <typename T>
__global__ void k_sv_gatherL(int64_t row_off, int64_t nr, int64_t nri, const int64_t *__restrict__ rowinit,
                             const int *__restrict__ perm, const int64_t *__restrict__ rsp, const int64_t *__restrict__ rsi,
                             const T *__restrict__ R, T *__restrict__ VB, int64_t vstride, int64_t n, int64_t nrhs)
{
    // perm == nullptr: a front without pivots, in its initial order
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nr * nrhs; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = e % nr, r = e / nr, i = perm ? perm[k] : k, g = row_off + i, ri = rowinit[g];
        T val = (i < nri && ri >= 0) ? R[ri + r * n] : VT<T>::zero();
        for (int64_t q = rsp[g]; q < rsp[g + 1]; q++) val = add(val, VB[rsi[q] + r * vstride]);
        VB[row_off + k + r * vstride] = val;
    }
}

// R[rowid[k]] = the front's vector entry k (its rows in their final order): a front's gathered vector into the row-space
// vector, for the sequential sweep that takes over from it
template <typename T>
__global__ void k_sv_toR(const T *__restrict__ Vf, int64_t vstride, int64_t nr, const int64_t *__restrict__ rowid,
                         T *__restrict__ R, int64_t n, int64_t nrhs)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nr * nrhs; e += (int64_t)gridDim.x * blockDim.x)
        R[rowid[e % nr] + (e / nr) * n] = Vf[e % nr + (e / nr) * vstride];
}

// Y[j] = R[p_lu[j]] for the pivots j in [j0, n)
template <typename T>
__global__ void k_gather_range(T *__restrict__ Y, const T *__restrict__ R, const int64_t *__restrict__ p_lu, int64_t j0,
                               int64_t n, int64_t nrhs)
{
    const int64_t m = n - j0;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < m * nrhs; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = j0 + e % m, r = e / m;
        Y[j + r * n] = R[p_lu[j] + r * n];
    }
}

// Y[f + k] = the front's solved pivot entries (rows [0, np) of its VB vector)
template <typename T>
__global__ void k_sv_put(const T *__restrict__ Vf, int64_t vstride, int64_t np, T *__restrict__ Y, int64_t f, int64_t n,
                         int64_t nrhs)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < np * nrhs; e += (int64_t)gridDim.x * blockDim.x)
        Y[f + e % np + (e / np) * n] = Vf[e % np + (e / np) * vstride];
}

// U sweep (trans 0) of a level's small fronts, a CTA each: x = U11^-1 (y - U12 x[CB columns]) (the CB columns' x from
// the fronts above, already solved)
template <typename T>
__global__ void __launch_bounds__(SV_THREADS) k_sv_bwdU(const SvFront *__restrict__ fr, const int *__restrict__ list,
                                                        const T *__restrict__ La, const T *__restrict__ Ua,
                                                        const int64_t *__restrict__ cols, const T *__restrict__ Y,
                                                        T *__restrict__ X, int64_t n, int nrhs, DevStatus *st)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_zero;
    const SvFront F = fr[list[blockIdx.x]];
    const int np = (int)F.np, ncb = (int)(F.nc - F.np), tid = threadIdx.x;
    T *x = reinterpret_cast<T *>(smem_raw);          // np x SV_RC
    T *sT = x + np * SV_RC;                          // 64 x np
    T *dinv = sT + 64 * np;                          // 64
    const T *U12 = Ua + F.U_off;
    const int64_t *cb = cols + F.col_off + np;
    pdl_wait();
    pdl_trigger();
    for (int r0 = 0; r0 < nrhs; r0 += SV_RC) {
        const int rc = nrhs - r0 < SV_RC ? nrhs - r0 : SV_RC;
        for (int e = tid; e < np * rc; e += SV_THREADS) {
            const int i = e % np, r = e / np;
            const T *xr = X + (int64_t)(r0 + r) * n;
            T acc = VT<T>::zero();
            for (int t = 0; t < ncb; t++) acc = add(acc, mul(U12[i + (int64_t)t * np], xr[cb[t]]));
            x[e] = sub(Y[F.f + i + (int64_t)(r0 + r) * n], acc);
        }
        if (tid == 0) s_zero = 0;
        __syncthreads();
        blk_trisolve<T, true>(La + F.L_off, F.nr, np, x, rc, sT, dinv, st, F.f, &s_zero);
        if (s_zero) return;
        for (int e = tid; e < np * rc; e += SV_THREADS) X[F.f + e % np + (int64_t)(r0 + e / np) * n] = x[e];
        __syncthreads();
    }
}

// U^T sweep (trans 1; 2 with conj) of a level's small fronts (npiv <= 64), a CTA each: the front's column vector (the
// pivot columns' right-hand side, then the children's entries that land on each column), y = U11^-T w[:np] (into R),
// then the contribution u = w[np:] - U12^T y into VB
template <typename T, bool CJ>
__global__ void __launch_bounds__(SV_THREADS) k_sv_fwdUt(const SvFront *__restrict__ fr, const int *__restrict__ list,
                                                         const T *__restrict__ La, const T *__restrict__ Ua,
                                                         const int64_t *__restrict__ csp, const int64_t *__restrict__ csi,
                                                         T *__restrict__ R, T *__restrict__ VB, int64_t vstride, int64_t n,
                                                         int nrhs, DevStatus *st)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_zero;
    const SvFront F = fr[list[blockIdx.x]];
    const int np = (int)F.np, nc = (int)F.nc, ncb = nc - np, ld = np + 1, tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5, nw = SV_THREADS / 32;
    T *w = reinterpret_cast<T *>(smem_raw);          // nc x SV_RC (ld nc)
    T *sT = w + nc * SV_RC;                          // np x ld: sT[j + i * ld] = U11[i, j] (conj)
    T *dinv = sT + np * ld;
    const T *L = La + F.L_off, *U12 = Ua + F.U_off;
    if (tid == 0) s_zero = 0;
    stage_transposed<T, CJ>(L, F.nr, np, sT);
    __syncthreads();
    for (int i = tid; i < np; i += SV_THREADS) {
        T d = L[i + (int64_t)i * F.nr];
        if (CJ) d = conjv(d);
        if (is_zero(d)) { set_status(st, ST_SOLVE_ZERO, F.f + i, 0, 0); s_zero = 1; }
        dinv[i] = is_zero(d) ? VT<T>::zero() : recip(d);
    }
    pdl_wait();
    pdl_trigger();
    __syncthreads();
    if (s_zero) return;
    for (int r0 = 0; r0 < nrhs; r0 += SV_RC) {
        const int rc = nrhs - r0 < SV_RC ? nrhs - r0 : SV_RC;
        for (int e = tid; e < nc * rc; e += SV_THREADS) {
            const int c = e % nc, r = e / nc;
            const int64_t g = F.col_off + c;
            T val = c < np ? R[F.f + c + (int64_t)(r0 + r) * n] : VT<T>::zero();
            for (int64_t q = csp[g]; q < csp[g + 1]; q++) val = add(val, VB[csi[q] + (int64_t)(r0 + r) * vstride]);
            w[c + r * nc] = val;
        }
        __syncthreads();
        for (int r = warp; r < rc; r += nw) {
            T *wr = w + r * nc;
            T a = lane < np ? wr[lane] : VT<T>::zero();
            T b = lane + 32 < np ? wr[lane + 32] : VT<T>::zero();
            for (int i = 0; i < np; i++) {
                const T zi = mul(shfl_v<T>(i < 32 ? a : b, i & 31), dinv[i]);
                const T *row = sT + i * ld;             // row[j] = u_ij
                if (lane == i) a = zi;
                else if (lane > i && lane < np) a = sub(a, mul(row[lane], zi));
                if (lane + 32 == i) b = zi;
                else if (lane + 32 > i && lane + 32 < np) b = sub(b, mul(row[lane + 32], zi));
            }
            if (lane < np) wr[lane] = a;
            if (lane + 32 < np) wr[lane + 32] = b;
        }
        __syncthreads();
        for (int e = tid; e < np * rc; e += SV_THREADS) R[F.f + e % np + (int64_t)(r0 + e / np) * n] = w[e % np + (e / np) * nc];
        for (int t = warp; t < ncb; t += nw) {
            T u0 = lane < np ? U12[lane + (int64_t)t * np] : VT<T>::zero();
            T u1 = lane + 32 < np ? U12[lane + 32 + (int64_t)t * np] : VT<T>::zero();
            if (CJ) { u0 = conjv(u0); u1 = conjv(u1); }
            for (int r = 0; r < rc; r++) {
                const T *z = w + r * nc;
                T s = lane < np ? mul(u0, z[lane]) : VT<T>::zero();
                if (lane + 32 < np) s = add(s, mul(u1, z[lane + 32]));
                for (int o = 16; o > 0; o >>= 1) s = add(s, shfl_xor_v<T>(s, o));
                if (lane == 0) VB[F.col_off + np + t + (int64_t)(r0 + r) * vstride] = sub(z[np + t], s);
            }
        }
        __syncthreads();
    }
}

// a larger front's column vector (the U^T sweep): the pivot columns' entries into R[f ..], the others into its own
// entries of VB
template <typename T>
__global__ void k_sv_gatherU(int64_t f, int64_t np, int64_t nc, int64_t col_off, const int64_t *__restrict__ csp,
                             const int64_t *__restrict__ csi, T *__restrict__ R, T *__restrict__ VB, int64_t vstride, int64_t n,
                             int64_t nrhs)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nc * nrhs; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = e % nc, r = e / nc, g = col_off + c;
        T val = c < np ? R[f + c + r * n] : VT<T>::zero();
        for (int64_t q = csp[g]; q < csp[g + 1]; q++) val = add(val, VB[csi[q] + r * vstride]);
        if (c < np) R[f + c + r * n] = val;
        else VB[col_off + c + r * vstride] = val;
    }
}

// a larger front's contribution (the U^T sweep): u[t] = w[np + t] - sum_k U12[k, t] y[k] (conj), a warp per column
template <typename T, bool CJ>
__global__ void k_sv_utcb(const T *__restrict__ U12, int64_t npiv, int64_t ncb, int64_t f, const T *__restrict__ R,
                          T *__restrict__ VBc, int64_t vstride, int64_t n, int64_t nrhs)
{
    const int lane = threadIdx.x & 31;
    for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < ncb; c += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        for (int64_t r = 0; r < nrhs; r++) {
            const T *z = R + f + r * n;
            T s = VT<T>::zero();
            for (int64_t k = lane; k < npiv; k += 32) {
                T u = U12[k + c * npiv];
                if (CJ) u = conjv(u);
                s = k < 32 ? mul(u, z[k]) : add(s, mul(u, z[k]));
            }
            for (int o = 16; o > 0; o >>= 1) s = add(s, shfl_xor_v<T>(s, o));
            if (lane == 0) VBc[c + r * vstride] = sub(VBc[c + r * vstride], s);
        }
    }
}

// L^T sweep (trans 1; 2 with conj) of a level's small fronts (npiv <= 64), a CTA each: x = L11^-T (y - L21^T x[CB rows])
// (the CB rows' x, in pivot order through pinv, from the fronts above, already solved)
template <typename T, bool CJ>
__global__ void __launch_bounds__(SV_THREADS) k_sv_bwdLt(const SvFront *__restrict__ fr, const int *__restrict__ list,
                                                         const T *__restrict__ La, const int64_t *__restrict__ rowid_all,
                                                         const int64_t *__restrict__ pinv, const T *__restrict__ Z,
                                                         T *__restrict__ V, int64_t n, int nrhs)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const SvFront F = fr[list[blockIdx.x]];
    const int np = (int)F.np, nr = (int)F.nr, ld = np + 1, tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5, nw = SV_THREADS / 32;
    T *sT = reinterpret_cast<T *>(smem_raw);          // np x ld: sT[j + i * ld] = L11[i, j] (conj)
    T *s = sT + np * ld;                              // np x SV_RC
    const T *L = La + F.L_off;
    const int64_t *rowid = rowid_all + F.row_off;
    stage_transposed<T, CJ>(L, nr, np, sT);
    pdl_wait();
    pdl_trigger();
    __syncthreads();
    for (int r0 = 0; r0 < nrhs; r0 += SV_RC) {
        const int rc = nrhs - r0 < SV_RC ? nrhs - r0 : SV_RC;
        for (int e = warp; e < np * rc; e += nw) {
            const int i = e % np, r = e / np;
            T acc = VT<T>::zero();
            for (int rr = np + lane; rr < nr; rr += 32) {
                T l = L[rr + (int64_t)i * nr];
                if (CJ) l = conjv(l);
                acc = add(acc, mul(l, V[pinv[rowid[rr]] + (int64_t)(r0 + r) * n]));
            }
            for (int o = 16; o > 0; o >>= 1) acc = add(acc, shfl_xor_v<T>(acc, o));
            if (lane == 0) s[e] = sub(Z[F.f + i + (int64_t)(r0 + r) * n], acc);
        }
        __syncthreads();
        for (int r = warp; r < rc; r += nw) {
            T *sr = s + r * np;
            T a = lane < np ? sr[lane] : VT<T>::zero();
            T b = lane + 32 < np ? sr[lane + 32] : VT<T>::zero();
            for (int i = np - 1; i >= 0; i--) {
                const T vi = shfl_v<T>(i < 32 ? a : b, i & 31);
                const T *row = sT + i * ld;             // row[j] = L11[i, j], j < i
                if (lane < i) a = sub(a, mul(row[lane], vi));
                if (lane + 32 < i) b = sub(b, mul(row[lane + 32], vi));
            }
            if (lane < np) V[F.f + lane + (int64_t)(r0 + r) * n] = a;
            if (lane + 32 < np) V[F.f + lane + 32 + (int64_t)(r0 + r) * n] = b;
        }
        __syncthreads();
    }
}

// The larger fronts of a level in the trans-0 sweeps, all in each launch (blockIdx.y: the front in the level's list).
// L sweep, 1: the fronts' vectors in their final row order into VB
template <typename T>
__global__ void k_svb_gatherL(const SvFront *__restrict__ fr, const int *__restrict__ list, const int64_t *__restrict__ rowinit,
                              const int *__restrict__ permall, const int64_t *__restrict__ rsp, const int64_t *__restrict__ rsi,
                              const T *__restrict__ R, T *__restrict__ VB, int64_t vstride, int64_t n, int64_t nrhs)
{
    const SvFront F = fr[list[blockIdx.y]];
    const int *perm = permall + F.row_off;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < F.nr * nrhs; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = e % F.nr, r = e / F.nr, i = F.np > 0 ? perm[k] : k, g = F.row_off + i, ri = rowinit[g];
        T val = (i < F.nri && ri >= 0) ? R[ri + r * n] : VT<T>::zero();
        for (int64_t q = rsp[g]; q < rsp[g + 1]; q++) val = add(val, VB[rsi[q] + r * vstride]);
        VB[F.row_off + k + r * vstride] = val;
    }
}

// L sweep, 2: x = L11^-1 v[:np], a CTA per front, rcb right-hand sides per pass; x into VB (in place) and into Y in
// pivot order
template <typename T>
__global__ void __launch_bounds__(256) k_svb_L11(const SvFront *__restrict__ fr, const int *__restrict__ list,
                                                 const T *__restrict__ La, T *__restrict__ VB, int64_t vstride,
                                                 T *__restrict__ Y, int64_t n, int nrhs, int rcb)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const SvFront F = fr[list[blockIdx.x]];
    const int np = (int)(F.np < F.nr ? F.np : F.nr), tid = threadIdx.x;
    if (np == 0) return;
    T *x = reinterpret_cast<T *>(smem_raw);          // np x rcb
    T *sT = x + (int64_t)np * rcb;                   // 64 x 64
    // blockIdx.y: the group of right-hand sides [y * rcb, y * rcb + rcb) (the groups are independent)
    for (int r0 = blockIdx.y * rcb; r0 < nrhs && r0 < (int)(blockIdx.y + 1) * rcb; r0 += rcb) {
        const int rc = nrhs - r0 < rcb ? nrhs - r0 : rcb;
        for (int e = tid; e < np * rc; e += blockDim.x) x[e] = VB[F.row_off + e % np + (int64_t)(r0 + e / np) * vstride];
        __syncthreads();
        blk_trisolve<T, false>(La + F.L_off, F.nr, np, x, rc, sT, nullptr, nullptr, 0);
        for (int e = tid; e < np * rc; e += blockDim.x) {
            const int k = e % np;
            const int64_t r = r0 + e / np;
            VB[F.row_off + k + r * vstride] = x[e];
            Y[F.f + k + r * n] = x[e];
        }
        __syncthreads();
    }
}

// L sweep, 3: u = v[np:] - L21 x on 256 rows per CTA (x from VB), rc2 right-hand sides per pass over L
template <typename T>
__global__ void __launch_bounds__(256) k_svb_L21(const SvFront *__restrict__ fr, const int *__restrict__ list,
                                                 const T *__restrict__ La, T *__restrict__ VB, int64_t vstride, int nrhs, int rc2)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const SvFront F = fr[list[blockIdx.y]];
    const int np = (int)(F.np < F.nr ? F.np : F.nr), tid = threadIdx.x;
    const int64_t rows = F.nr - np, row0 = (int64_t)blockIdx.x * 256;
    if (np == 0 || row0 >= rows) return;
    T *xs = reinterpret_cast<T *>(smem_raw);         // np x rc2
    const T *L = La + F.L_off;
    const int64_t rr = np + row0 + tid;
    for (int r0 = 0; r0 < nrhs; r0 += rc2) {
        const int rc = nrhs - r0 < rc2 ? nrhs - r0 : rc2;
        for (int e = tid; e < np * rc; e += blockDim.x) xs[e] = VB[F.row_off + e % np + (int64_t)(r0 + e / np) * vstride];
        __syncthreads();
        if (rr < F.nr) {
            T acc[SVB_RC];
#pragma unroll
            for (int r = 0; r < SVB_RC; r++) acc[r] = VT<T>::zero();
            for (int k0 = 0; k0 < np; k0 += 8) {
                T lv[8];
#pragma unroll
                for (int q = 0; q < 8; q++) lv[q] = k0 + q < np ? L[rr + (int64_t)(k0 + q) * F.nr] : VT<T>::zero();
#pragma unroll
                for (int q = 0; q < 8; q++)
                    if (k0 + q < np)
#pragma unroll
                        for (int r = 0; r < SVB_RC; r++)
                            if (r < rc) acc[r] = add(acc[r], mul(lv[q], xs[k0 + q + r * np]));
            }
#pragma unroll
            for (int r = 0; r < SVB_RC; r++)
                if (r < rc) {
                    T *o = VB + F.row_off + rr + (int64_t)(r0 + r) * vstride;
                    *o = sub(*o, acc[r]);
                }
        }
        __syncthreads();
    }
}

// U sweep, 1: the partial products U12 x[CB columns] of chunk blockIdx.x of a front's CB columns (F.nch chunks), a
// thread per row of U12, into part (the front's partial sums start at F.poff * nrhs); the chunk's x values staged in
// shared memory, SVB_RC right-hand sides per pass over U12
template <typename T>
__global__ void __launch_bounds__(256) k_svb_u12(const SvFront *__restrict__ fr, const int *__restrict__ list,
                                                 const T *__restrict__ Ua, const int64_t *__restrict__ cols,
                                                 const T *__restrict__ X, int64_t n, int nrhs, T *__restrict__ part)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *Xs = reinterpret_cast<T *>(smem_raw);         // chunk x SVB_RC: Xs[k * SVB_RC + r]
    const SvFront F = fr[list[blockIdx.y]];
    if (blockIdx.x >= F.nch || F.np == 0) return;
    const int64_t np = F.np, ncb = F.nc - F.np, chunk = (ncb + F.nch - 1) / F.nch;
    const int64_t c0 = blockIdx.x * chunk, c1 = c0 + chunk < ncb ? c0 + chunk : ncb;
    const int cc = (int)(c1 - c0);
    const T *U12 = Ua + F.U_off;
    const int64_t *cb = cols + F.col_off + np;
    T *pp = part + F.poff * nrhs + (int64_t)blockIdx.x * np * nrhs;
    for (int r0 = 0; r0 < nrhs; r0 += SVB_RC) {
        const int rc = nrhs - r0 < SVB_RC ? nrhs - r0 : SVB_RC;
        for (int e = threadIdx.x; e < cc * rc; e += blockDim.x) {
            const int k = e / rc, r = e - k * rc;
            Xs[k * SVB_RC + r] = X[cb[c0 + k] + (int64_t)(r0 + r) * n];
        }
        __syncthreads();
        for (int64_t i = threadIdx.x; i < np; i += blockDim.x) {
            T acc[SVB_RC];
#pragma unroll
            for (int r = 0; r < SVB_RC; r++) acc[r] = VT<T>::zero();
            for (int k0 = 0; k0 < cc; k0 += 8) {
                T uv[8];
#pragma unroll
                for (int q = 0; q < 8; q++) uv[q] = k0 + q < cc ? U12[i + (c0 + k0 + q) * np] : VT<T>::zero();
#pragma unroll
                for (int q = 0; q < 8; q++)
                    if (k0 + q < cc)
#pragma unroll
                        for (int r = 0; r < SVB_RC; r++)
                            if (r < rc) acc[r] = add(acc[r], mul(uv[q], Xs[(k0 + q) * SVB_RC + r]));
            }
#pragma unroll
            for (int r = 0; r < SVB_RC; r++)
                if (r < rc) pp[i + (int64_t)(r0 + r) * np] = acc[r];
        }
        __syncthreads();
    }
}

// U sweep, 2: y - the partial products (in chunk order) for every front of the level, over many CTAs, into the front's
// first partial sum
template <typename T>
__global__ void k_svb_psum(const SvFront *__restrict__ fr, const int *__restrict__ list, T *__restrict__ part,
                           const T *__restrict__ Y, int64_t n, int nrhs)
{
    const SvFront F = fr[list[blockIdx.y]];
    if (F.np == 0 || F.nch == 0) return;              // (no partial sums: k_svb_bwdU reads y itself)
    const int64_t np = F.np, E = np * nrhs;
    T *pp = part + F.poff * nrhs;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
        T v = Y[F.f + e % np + (e / np) * n];
        for (int64_t q0 = 0; q0 < F.nch; q0 += 8) {          // eight loads in flight
            T pv[8];
#pragma unroll
            for (int q = 0; q < 8; q++) pv[q] = q0 + q < F.nch ? pp[(q0 + q) * E + e] : VT<T>::zero();
#pragma unroll
            for (int q = 0; q < 8; q++)
                if (q0 + q < F.nch) v = sub(v, pv[q]);
        }
        pp[e] = v;
    }
}

// U sweep, 3: x = U11^-1 (y - the partial products, in chunk order), a CTA per front, rcb right-hand sides per pass
// (presummed: k_svb_psum left y - the products in the front's first partial sum)
template <typename T>
__global__ void __launch_bounds__(256) k_svb_bwdU(const SvFront *__restrict__ fr, const int *__restrict__ list,
                                                  const T *__restrict__ La, const T *__restrict__ part, const T *__restrict__ Y,
                                                  T *__restrict__ X, int64_t n, int nrhs, int rcb, DevStatus *st, int presummed)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_zero;
    const SvFront F = fr[list[blockIdx.x]];
    const int np = (int)F.np, tid = threadIdx.x;
    if (np == 0) return;
    T *x = reinterpret_cast<T *>(smem_raw);          // np x rcb
    T *sT = x + (int64_t)np * rcb;                   // 64 x 64
    T *dinv = sT + 64 * 64;                          // 64
    const T *pp = part + F.poff * nrhs;
    // blockIdx.y: the group of right-hand sides [y * rcb, y * rcb + rcb) (the groups are independent)
    for (int r0 = blockIdx.y * rcb; r0 < nrhs && r0 < (int)(blockIdx.y + 1) * rcb; r0 += rcb) {
        const int rc = nrhs - r0 < rcb ? nrhs - r0 : rcb;
        for (int e = tid; e < np * rc; e += blockDim.x) {
            const int i = e % np;
            const int64_t r = r0 + e / np;
            T v;
            if (presummed && F.nch > 0) v = pp[i + r * np];
            else {
                v = Y[F.f + i + r * n];
                for (int64_t q0 = 0; q0 < F.nch; q0 += 8) {      // eight loads in flight, the sum in chunk order
                    T pv[8];
#pragma unroll
                    for (int q = 0; q < 8; q++) pv[q] = q0 + q < F.nch ? pp[(q0 + q) * np * nrhs + i + r * np] : VT<T>::zero();
#pragma unroll
                    for (int q = 0; q < 8; q++)
                        if (q0 + q < F.nch) v = sub(v, pv[q]);
                }
            }
            x[e] = v;
        }
        if (tid == 0) s_zero = 0;
        __syncthreads();
        blk_trisolve<T, true>(La + F.L_off, F.nr, np, x, rc, sT, dinv, st, F.f, &s_zero);
        if (s_zero) return;
        for (int e = tid; e < np * rc; e += blockDim.x) X[F.f + e % np + (int64_t)(r0 + e / np) * n] = x[e];
        __syncthreads();
    }
}

// =====================================================================================================================
// the batched fronts of the factorization: one launch per level for each of assembly, pivot-block LU and tail
// =====================================================================================================================
// Assembly of a level's batched fronts, a CTA each, into their own working blocks (zeroed beforehand): the original
// entries and the entering rows' ids, then the children's contribution blocks one child after another (the order of the
// front-by-front assembly) with the children's CB row ids into their slots
template <typename T>
__global__ void __launch_bounds__(256) k_bat_assemble(const FcFront *__restrict__ fc, const int *__restrict__ list,
                                                      const int64_t *__restrict__ children, T *__restrict__ Wbase,
                                                      const T *__restrict__ Bx, const int64_t *__restrict__ asm_src,
                                                      const int64_t *__restrict__ asm_dst, const int64_t *__restrict__ rowinit,
                                                      int64_t *__restrict__ rowid_all, const int64_t *__restrict__ relcol,
                                                      const T *__restrict__ CBA, const DevStatus *st)
{
    if (st->code) return;
    const FcFront F = fc[list[blockIdx.x]];
    T *W = Wbase + F.wofs;
    const int tid = threadIdx.x, nr = (int)F.nr;
    int64_t *rowid = rowid_all + F.row_off;
    for (int64_t e = F.asm_begin + tid; e < F.asm_end; e += blockDim.x) W[asm_dst[e]] = Bx[asm_src[e]];
    for (int i = tid; i < nr; i += blockDim.x) if (rowinit[F.row_off + i] >= 0) rowid[i] = rowinit[F.row_off + i];
    __syncthreads();
    for (int64_t k = F.child_begin; k < F.child_end; k++) {
        const FcFront G = fc[children[k]];
        const int cbr = (int)(G.nr - G.np), cbc = (int)(G.nc - G.np), nslot = (int)(G.nri - G.np > 0 ? G.nri - G.np : 0);
        const T *cb = CBA + G.cbofs;
        const int64_t *rc = relcol + G.relcol_off;
        for (int e = tid; e < cbr * cbc; e += blockDim.x) {
            const int c = e / cbr, t = e - c * cbr;
            const int64_t pr = t < nslot ? G.slot + t : F.tau_base + (t - nslot);
            T *w = W + pr + rc[c] * nr;
            *w = add(*w, cb[e]);
        }
        for (int t = tid; t < nslot; t += blockDim.x) rowid[G.slot + t] = rowid_all[G.row_off + G.np + t];
        __syncthreads();
    }
}

// the pivot-block LU of a level's batched fronts, a CTA each (the body of k_front_lu2)
template <typename T>
__global__ void __launch_bounds__(640) k_bat_lu2(const FcFront *__restrict__ fc, const int *__restrict__ list,
                                                 const T *__restrict__ Wbase, const double *__restrict__ colmax, double pivot_rel,
                                                 int64_t *__restrict__ rowid_all, T *__restrict__ La, int *__restrict__ permall,
                                                 int64_t *__restrict__ p_lu, DevStatus *st)
{
    const int fi = list[blockIdx.x];
    const FcFront F = fc[fi];
    PivotAsm pa;
    pa.on = 0;
    front_lu2_body<T>(Wbase + F.wofs, F.nr, (int)F.nr, (int)F.np, (int)F.nri, F.f, colmax, pivot_rel, rowid_all + F.row_off,
                      La + F.L_off, permall + F.row_off, p_lu, st, fi, pa);
}

// the same with the blocked pivot-block LU (the body of k_front_lu5)
template <typename T>
__global__ void __launch_bounds__(LU5_THREADS) k_bat_lu5(const FcFront *__restrict__ fc, const int *__restrict__ list,
                                                          const T *__restrict__ Wbase, const double *__restrict__ colmax,
                                                          double pivot_rel, int64_t *__restrict__ rowid_all, T *__restrict__ La,
                                                          int *__restrict__ permall, int64_t *__restrict__ p_lu, DevStatus *st)
{
    const int fi = list[blockIdx.x];
    const FcFront F = fc[fi];
    PivotAsm pa;
    pa.on = 0;
    front_lu5_body<T>(Wbase + F.wofs, F.nr, (int)F.nr, (int)F.np, (int)F.nri, F.f, colmax, pivot_rel, rowid_all + F.row_off,
                      La + F.L_off, permall + F.row_off, p_lu, st, fi, pa);
}

// U12 and the contribution block of a level's batched fronts (blockIdx.y: the front; blockIdx.x: its CTAs over the
// 32-column tiles; the body of k_front_tail)
template <typename T, int TN>
__global__ void __launch_bounds__(FT_THREADS) k_bat_tail(const FcFront *__restrict__ fc, const int *__restrict__ list,
                                                         const T *__restrict__ Wbase, const int *__restrict__ permall,
                                                         const T *__restrict__ La, T *__restrict__ Ua, T *__restrict__ CBA,
                                                         const DevStatus *st)
{
    const FcFront F = fc[list[blockIdx.y]];
    const int64_t ncb = F.nc - F.np;
    const int64_t ntile = (ncb + TN - 1) / TN;
    if (ncb <= 0 || blockIdx.x >= ntile) return;
    const int nbk = (int)(gridDim.x < ntile ? gridDim.x : ntile);
    front_tail_body<T, TN>(Wbase + F.wofs, F.nr, permall + F.row_off, (int)F.np, (int)F.nr, ncb, 0, ncb, La + F.L_off,
                           Ua + F.U_off, CBA + F.cbofs, st, (int)blockIdx.x, nbk);
}

// the same with the tail of k_front_tail2 (blockIdx.y: the front; blockIdx.x: its CTAs over the
// 32-column tiles; the body of k_front_tail2)
template <typename T, int TN>
__global__ void __launch_bounds__(FT_THREADS) k_bat_tail2(const FcFront *__restrict__ fc, const int *__restrict__ list,
                                                         const T *__restrict__ Wbase, const int *__restrict__ permall,
                                                         const T *__restrict__ La, T *__restrict__ Ua, T *__restrict__ CBA,
                                                         const DevStatus *st)
{
    const FcFront F = fc[list[blockIdx.y]];
    const int64_t ncb = F.nc - F.np;
    const int64_t ntile = (ncb + TN - 1) / TN;
    if (ncb <= 0 || blockIdx.x >= ntile) return;
    const int nbk = (int)(gridDim.x < ntile ? gridDim.x : ntile);
    front_tail2_body<T, TN>(Wbase + F.wofs, F.nr, permall + F.row_off, (int)F.np, (int)F.nr, ncb, 0, ncb, La + F.L_off,
                            Ua + F.U_off, CBA + F.cbofs, st, (int)blockIdx.x, nbk, TailOut{});
}

}  // namespace fpl
