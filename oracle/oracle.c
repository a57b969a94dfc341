/* oracle.c -- TEST INFRASTRUCTURE ONLY: a CPU restatement of the FPLUS numeric path, the checker of the CUDA path.
 *
 * Follows, function by function (file:line in the FPLUS sources):
 *   orc_permute_csc  src/pipeline.c:14-82       B = A[row_perm,:][:,col_perm], canonical (counting sort: rows ascending)
 *   orc_ruiz         src/equil.c:60-183,186-441 Ruiz on CSC: range guard, squared-modulus row / column maxima, the
 *                                               1/sqrt(sqrt(max)) scales, residual max |log|/2, fold of the 2^k guard
 *   lu_partial       src/factor_sn.c:246-451    left-looking column LU, x = L^-1 B[:,j] by a depth-first reach, the pivot
 *                                               = largest modulus among the rows not yet pivotal, singular test
 *                                               best < pivot_rel * max|B(:,j)|, L column divided by the pivot
 *   (L, U layout)    src/factor_sn.c:741-808    L in pivot-order rows, unit diagonal first; U with its diagonal
 *   orc_factor       src/numeric.c:39-83        p = row_perm[p_lu], q = col_perm[q_lu], Dr[row_perm[k]] = Drp[k], ...
 *   tri_solve        src/solve.c:11-60          the plain column sweeps for trans 0 / 1 / 2
 *   orc_solve        src/numeric.c:88-131       scale and permute in, sweeps, unscale and permute out
 *
 * The reference's supernodes, relaxed joins and panels change how the LU is computed, not what it computes: P B = L U
 * with the same pivots (the reference's own tests pin panel > 1 to panel 1's pivots, test_sparse_lu_full_pivot.py:
 * 775-782).  This restatement therefore factors column by column without supernodes.  Ties between equal moduli go to
 * the smallest row index (the reference takes the first in its search order); the two differ only on exact ties.
 * Compiled as ISO C99 without floating-point contraction, like the reference (CMakeLists.txt:19-21, 97-102).
 */
#include "oracle.h"
#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef double complex zc;

struct orc_numeric {
    int64_t n;
    int is_complex;
    int64_t *Lp, *Li, *Up, *Ui, *p_lu;
    void *Lx, *Ux;
    int64_t *p, *q;
    double *Dr, *Dc, *Drp, *Dcp;
    int ruiz_iters;
    int64_t *Bp, *Bi;
    void *Bx;
};

static void errf(char *err, size_t errlen, const char *msg, long a)
{
    if (err && errlen) snprintf(err, errlen, msg, a);
}

/* ------------------------------------------------------------------ permute (src/pipeline.c:14-82) */
int orc_permute_csc(int64_t n, const int64_t *Ap, const int64_t *Ai, const void *Ax, int is_complex,
                    const int64_t *row_perm, const int64_t *col_perm, int64_t *Bp, int64_t *Bi, void *Bx)
{
    const size_t vs = is_complex ? sizeof(zc) : sizeof(double);
    const int64_t nnz = Ap[n];
    int64_t *inv = malloc((size_t)(n + 1) * sizeof(int64_t));
    int64_t *rc = calloc((size_t)(n + 1), sizeof(int64_t));
    int64_t *tj = malloc((size_t)(nnz + 1) * sizeof(int64_t)), *ts = malloc((size_t)(nnz + 1) * sizeof(int64_t));
    int64_t *fill = malloc((size_t)(n + 1) * sizeof(int64_t));
    if (!inv || !rc || !tj || !ts || !fill) { free(inv); free(rc); free(tj); free(ts); free(fill); return -1; }
    for (int64_t i = 0; i < n; i++) inv[row_perm[i]] = i;
    Bp[0] = 0;
    for (int64_t jj = 0; jj < n; jj++) { int64_t c = col_perm[jj]; Bp[jj + 1] = Bp[jj] + Ap[c + 1] - Ap[c]; }
    /* rows of the permuted matrix: a counting sort by new row, columns visited in new order, then back to columns */
    for (int64_t q = 0; q < nnz; q++) rc[inv[Ai[q]] + 1]++;
    for (int64_t i = 0; i < n; i++) rc[i + 1] += rc[i];
    memcpy(fill, rc, (size_t)(n + 1) * sizeof(int64_t));
    for (int64_t jj = 0; jj < n; jj++) {
        int64_t c = col_perm[jj];
        for (int64_t q = Ap[c]; q < Ap[c + 1]; q++) { int64_t t = fill[inv[Ai[q]]]++; tj[t] = jj; ts[t] = q; }
    }
    memcpy(fill, Bp, (size_t)(n + 1) * sizeof(int64_t));
    for (int64_t r = 0; r < n; r++)
        for (int64_t t = rc[r]; t < rc[r + 1]; t++) {
            int64_t o = fill[tj[t]]++;
            Bi[o] = r;
            memcpy((char *)Bx + (size_t)o * vs, (const char *)Ax + (size_t)ts[t] * vs, vs);
        }
    free(inv); free(rc); free(tj); free(ts); free(fill);
    return 0;
}

/* ------------------------------------------------------------------ Ruiz (src/equil.c) */
/* one iteration on CSC (src/equil.c:60-183): 0, 1 + i for an all-zero row i, -(1 + j) for an all-zero column j */
static int64_t ruiz_iter(int64_t n, const int64_t *Bp, const int64_t *Bi, double *d, int cplx, double *Dr, double *Dc,
                         double *rmax, double *cmax, double *res_out)
{
    for (int64_t i = 0; i < n; i++) rmax[i] = 0.0;
    for (int64_t j = 0; j < n; j++)
        for (int64_t p = Bp[j]; p < Bp[j + 1]; p++) {
            double av;
            if (cplx) { double re = d[2 * p], im = d[2 * p + 1]; av = re * re + im * im; }
            else av = d[p] * d[p];
            if (av > rmax[Bi[p]]) rmax[Bi[p]] = av;
        }
    for (int64_t i = 0; i < n; i++) if (rmax[i] == 0.0) return 1 + i;
    double res = 0.0;
    for (int64_t i = 0; i < n; i++) { double v = 0.5 * fabs(log(rmax[i])); if (v > res) res = v; }
    for (int64_t i = 0; i < n; i++) { double dr = 1.0 / sqrt(sqrt(rmax[i])); Dr[i] *= dr; rmax[i] = dr; }
    for (int64_t j = 0; j < n; j++) {
        double cm = 0.0;
        for (int64_t p = Bp[j]; p < Bp[j + 1]; p++) {
            double av, s = rmax[Bi[p]];
            if (cplx) { d[2 * p] *= s; d[2 * p + 1] *= s; double re = d[2 * p], im = d[2 * p + 1]; av = re * re + im * im; }
            else { d[p] *= s; av = d[p] * d[p]; }
            if (av > cm) cm = av;
        }
        cmax[j] = cm;
    }
    for (int64_t j = 0; j < n; j++) if (cmax[j] == 0.0) return -(1 + j);
    for (int64_t j = 0; j < n; j++) {
        double v = 0.5 * fabs(log(cmax[j]));
        if (v > res) res = v;
        cmax[j] = 1.0 / sqrt(sqrt(cmax[j]));
        Dc[j] *= cmax[j];
    }
    for (int64_t j = 0; j < n; j++)
        for (int64_t p = Bp[j]; p < Bp[j + 1]; p++) {
            if (cplx) { d[2 * p] *= cmax[j]; d[2 * p + 1] *= cmax[j]; }
            else d[p] *= cmax[j];
        }
    *res_out = res;
    return 0;
}

int orc_ruiz(int64_t n, const int64_t *Bp, const int64_t *Bi, void *Bx, int is_complex, int max_iter, double tol,
             double *Dr, double *Dc, int *iters, char *err, size_t errlen)
{
    const int64_t nnz = Bp[n];
    double *d = (double *)Bx;
    int k4 = 0;
    /* range guard (src/equil.c:197-241) */
    {
        const int64_t m = is_complex ? 2 * nnz : nnz;
        double amax = 0.0, amin = INFINITY;
        for (int64_t q = 0; q < m; q++) { double a = fabs(d[q]); if (a > amax) amax = a; if (a > 0.0 && a < amin) amin = a; }
        if (amax > 0.0 && (amax > 0x1p500 || amin < 0x1p-500)) {
            int emax = ilogb(amax), emin = ilogb(amin);
            if (emax - emin > 990) {
                double *lmax = calloc((size_t)(2 * (n > 0 ? n : 1)), sizeof(double));
                if (!lmax) return -1;
                for (int64_t j = 0; j < n; j++)
                    for (int64_t p = Bp[j]; p < Bp[j + 1]; p++) {
                        double a = is_complex ? fmax(fabs(d[2 * p]), fabs(d[2 * p + 1])) : fabs(d[p]);
                        if (a > lmax[Bi[p]]) lmax[Bi[p]] = a;
                        if (a > lmax[n + j]) lmax[n + j] = a;
                    }
                double lmin = INFINITY;
                for (int64_t q = 0; q < 2 * n; q++) if (lmax[q] > 0.0 && lmax[q] < lmin) lmin = lmax[q];
                free(lmax);
                int elmin = ilogb(lmin);
                if (emax - elmin > 990) { errf(err, errlen, "line maxima span too wide for Ruiz (%ld)", (long)(emax - elmin)); return -3; }
                emin = elmin;
            }
            k4 = -((emax + emin) / 2 / 4) * 4;
            const double sc = ldexp(1.0, k4);
            for (int64_t q = 0; q < m; q++) d[q] *= sc;
        }
    }
    double *rmax = malloc((size_t)(n > 0 ? n : 1) * sizeof(double)), *cmax = malloc((size_t)(n > 0 ? n : 1) * sizeof(double));
    if (!rmax || !cmax) { free(rmax); free(cmax); return -1; }
    for (int64_t i = 0; i < n; i++) { Dr[i] = 1.0; Dc[i] = 1.0; }
    int used = 0;
    for (int it = 0; it < max_iter; it++) {
        double res = 0.0;
        int64_t bad = ruiz_iter(n, Bp, Bi, d, is_complex, Dr, Dc, rmax, cmax, &res);
        if (bad != 0) {
            free(rmax); free(cmax);
            if (bad > 0) errf(err, errlen, "Row %ld of the matrix is entirely zero", (long)(bad - 1));
            else errf(err, errlen, "Column %ld of the matrix is entirely zero", (long)(-bad - 1));
            return -2;
        }
        used = it + 1;
        if (res < tol) break;
    }
    free(rmax); free(cmax);
    if (k4 != 0) { const double h = ldexp(1.0, k4 / 2); for (int64_t i = 0; i < n; i++) { Dr[i] *= h; Dc[i] *= h; } }
    if (iters) *iters = used;
    return 0;
}

/* ------------------------------------------------------------------ LU (src/factor_sn.c:246-451, 741-808) */
typedef struct { int64_t *i; void *x; int64_t n, cap; } Vec;

static int vec_push(Vec *v, int64_t i, const void *x, size_t vs)
{
    if (v->n == v->cap) {
        int64_t nc = v->cap ? 2 * v->cap : 1024;
        int64_t *ni = realloc(v->i, (size_t)nc * sizeof(int64_t));
        if (!ni) return -1;
        v->i = ni;
        void *nx = realloc(v->x, (size_t)nc * vs);
        if (!nx) return -1;
        v->x = nx; v->cap = nc;
    }
    v->i[v->n] = i;
    memcpy((char *)v->x + (size_t)v->n * vs, x, vs);
    v->n++;
    return 0;
}

typedef struct { int64_t key; int64_t pos; } KP;
static int kp_cmp(const void *a, const void *b)
{
    int64_t x = ((const KP *)a)->key, y = ((const KP *)b)->key;
    return (x > y) - (x < y);
}

/* sort entries [a, b) of (idx, val) by idx */
static int sort_seg(int64_t *idx, void *val, int64_t a, int64_t b, size_t vs, KP *kp, char *tmp)
{
    int64_t m = b - a;
    if (m <= 1) return 0;
    for (int64_t t = 0; t < m; t++) { kp[t].key = idx[a + t]; kp[t].pos = a + t; }
    qsort(kp, (size_t)m, sizeof(KP), kp_cmp);
    for (int64_t t = 0; t < m; t++) memcpy(tmp + (size_t)t * vs, (char *)val + (size_t)kp[t].pos * vs, vs);
    for (int64_t t = 0; t < m; t++) { idx[a + t] = kp[t].key; memcpy((char *)val + (size_t)(a + t) * vs, tmp + (size_t)t * vs, vs); }
    return 0;
}

static double vabs(const double *x, int cplx) { return cplx ? cabs(*(const zc *)x) : fabs(*x); }

static int lu_partial(int64_t n, const int64_t *Bp, const int64_t *Bi, const void *Bx, int cplx, double pivot_rel,
                      orc_numeric *num, char *err, size_t errlen)
{
    const size_t vs = cplx ? sizeof(zc) : sizeof(double);
    const size_t nn = (size_t)(n > 0 ? n : 1);
    double *x = calloc(nn, vs);                  /* dense accumulator over rows (2 doubles per entry when complex) */
    int64_t *pinv = malloc(nn * sizeof(int64_t)), *mark = calloc(nn, sizeof(int64_t));
    int64_t *xi = malloc(nn * sizeof(int64_t)), *stk = malloc(nn * sizeof(int64_t)), *hd = malloc(nn * sizeof(int64_t));
    int64_t *Lp = malloc((nn + 1) * sizeof(int64_t)), *Up = malloc((nn + 1) * sizeof(int64_t));
    int64_t *p_lu = malloc(nn * sizeof(int64_t));
    Vec L = {0}, U = {0};
    int rc = -1;
    if (!x || !pinv || !mark || !xi || !stk || !hd || !Lp || !Up || !p_lu) goto out;
    for (int64_t i = 0; i < n; i++) pinv[i] = -1;
    Lp[0] = Up[0] = 0;
    for (int64_t j = 0; j < n; j++) {
        const int64_t stamp = j + 1;
        /* reach of B[:, j] in the graph of L: rows in topological order at xi[top..n) */
        int64_t top = n;
        for (int64_t q = Bp[j]; q < Bp[j + 1]; q++) {
            int64_t r0 = Bi[q];
            if (mark[r0] == stamp) continue;
            int64_t sp = 0;
            stk[0] = r0; mark[r0] = stamp;
            hd[0] = pinv[r0] >= 0 ? Lp[pinv[r0]] + 1 : 0;
            while (sp >= 0) {
                int64_t r = stk[sp], k = pinv[r];
                int done = 1;
                if (k >= 0) {
                    for (int64_t t = hd[sp]; t < Lp[k + 1]; t++) {
                        int64_t c = L.i[t];
                        if (mark[c] == stamp) continue;
                        hd[sp] = t + 1;
                        mark[c] = stamp;
                        stk[++sp] = c;
                        hd[sp] = pinv[c] >= 0 ? Lp[pinv[c]] + 1 : 0;
                        done = 0;
                        break;
                    }
                }
                if (done) { sp--; xi[--top] = r; }
            }
        }
        /* scatter B[:, j], its largest modulus */
        double colmax = 0.0;
        for (int64_t q = Bp[j]; q < Bp[j + 1]; q++) {
            const double *v = (const double *)Bx + (cplx ? 2 * q : q);
            if (cplx) ((zc *)x)[Bi[q]] += *(const zc *)v; else x[Bi[q]] += *v;
            double a = vabs(v, cplx);
            if (a > colmax) colmax = a;
        }
        /* x = L^-1 x over the reach, in topological order */
        for (int64_t t = top; t < n; t++) {
            int64_t r = xi[t], k = pinv[r];
            if (k < 0) continue;
            if (cplx) {
                zc xk = ((zc *)x)[r];
                if (xk == 0) continue;
                for (int64_t s = Lp[k] + 1; s < Lp[k + 1]; s++) ((zc *)x)[L.i[s]] -= xk * ((zc *)L.x)[s];
            } else {
                double xk = x[r];
                if (xk == 0) continue;
                for (int64_t s = Lp[k] + 1; s < Lp[k + 1]; s++) x[L.i[s]] -= xk * ((double *)L.x)[s];
            }
        }
        /* pivot: the largest modulus among the rows not yet pivotal (ties: smallest row) */
        int64_t piv = -1; double best = -1.0;
        for (int64_t t = top; t < n; t++) {
            int64_t r = xi[t];
            if (pinv[r] >= 0) continue;
            double a = cplx ? cabs(((zc *)x)[r]) : fabs(x[r]);
            if (a > best || (a == best && piv >= 0 && r < piv)) { best = a; piv = r; }
        }
        double thr = pivot_rel * colmax;
        if (piv < 0 || best <= 0.0 || best < thr) {
            if (err && errlen) snprintf(err, errlen, "Near-zero or zero pivot %.6e at step %ld (threshold %.6e). Matrix is singular.",
                                        best > 0 ? best : 0.0, (long)j, thr);
            rc = -2; goto out;
        }
        /* U[:, j]: the pivotal rows of the reach (pivot step), then the diagonal */
        for (int64_t t = top; t < n; t++) {
            int64_t r = xi[t];
            if (pinv[r] < 0) continue;
            if (vec_push(&U, pinv[r], (char *)x + (size_t)r * vs, vs)) goto out;
        }
        if (vec_push(&U, j, (char *)x + (size_t)piv * vs, vs)) goto out;
        Up[j + 1] = U.n;
        /* L[:, j]: the unit diagonal (the pivot row), then x / pivot on the other non-pivotal rows */
        {
            double one[2] = {1.0, 0.0};
            if (vec_push(&L, piv, one, vs)) goto out;
            for (int64_t t = top; t < n; t++) {
                int64_t r = xi[t];
                if (pinv[r] >= 0 || r == piv) continue;
                if (cplx) { zc v = ((zc *)x)[r] / ((zc *)x)[piv]; if (vec_push(&L, r, &v, vs)) goto out; }
                else { double v = x[r] / x[piv]; if (vec_push(&L, r, &v, vs)) goto out; }
            }
        }
        Lp[j + 1] = L.n;
        pinv[piv] = j; p_lu[j] = piv;
        for (int64_t t = top; t < n; t++) memset((char *)x + (size_t)xi[t] * vs, 0, vs);
    }
    /* renumber L's rows to pivot order and sort: the diagonal first, the rest ascending; U ascending (diagonal last) */
    {
        int64_t mx = 1;
        for (int64_t j = 0; j < n; j++) { if (Lp[j + 1] - Lp[j] > mx) mx = Lp[j + 1] - Lp[j]; if (Up[j + 1] - Up[j] > mx) mx = Up[j + 1] - Up[j]; }
        KP *kp = malloc((size_t)mx * sizeof(KP));
        char *tmp = malloc((size_t)mx * vs);
        if (!kp || !tmp) { free(kp); free(tmp); goto out; }
        for (int64_t t = 0; t < L.n; t++) L.i[t] = pinv[L.i[t]];
        for (int64_t j = 0; j < n; j++) { sort_seg(L.i, L.x, Lp[j] + 1, Lp[j + 1], vs, kp, tmp); sort_seg(U.i, U.x, Up[j], Up[j + 1] - 1, vs, kp, tmp); }
        free(kp); free(tmp);
    }
    num->Lp = Lp; num->Li = L.i; num->Lx = L.x; num->Up = Up; num->Ui = U.i; num->Ux = U.x; num->p_lu = p_lu;
    Lp = Up = p_lu = NULL; L.i = U.i = NULL; L.x = U.x = NULL;
    rc = 0;
out:
    if (rc == -1) errf(err, errlen, "out of memory", 0);
    free(x); free(pinv); free(mark); free(xi); free(stk); free(hd); free(Lp); free(Up); free(p_lu);
    free(L.i); free(L.x); free(U.i); free(U.x);
    return rc;
}

/* ------------------------------------------------------------------ composition (src/numeric.c:39-83) */
int orc_factor(int64_t n, const int64_t *Ap, const int64_t *Ai, const void *Ax, int is_complex,
               const int64_t *row_perm, const int64_t *col_perm, int equilibrate, int ruiz_max_iter, double ruiz_tol,
               double pivot_rel, orc_numeric **out, char *err, size_t errlen)
{
    *out = NULL;
    const size_t vs = is_complex ? sizeof(zc) : sizeof(double);
    const size_t nn = (size_t)(n > 0 ? n : 1), nz = (size_t)(Ap[n] > 0 ? Ap[n] : 1);
    orc_numeric *num = calloc(1, sizeof(*num));
    if (!num) return -1;
    num->n = n; num->is_complex = is_complex;
    num->Bp = malloc((nn + 1) * sizeof(int64_t)); num->Bi = malloc(nz * sizeof(int64_t)); num->Bx = malloc(nz * vs);
    num->Drp = malloc(nn * sizeof(double)); num->Dcp = malloc(nn * sizeof(double));
    num->Dr = malloc(nn * sizeof(double)); num->Dc = malloc(nn * sizeof(double));
    num->p = malloc(nn * sizeof(int64_t)); num->q = malloc(nn * sizeof(int64_t));
    if (!num->Bp || !num->Bi || !num->Bx || !num->Drp || !num->Dcp || !num->Dr || !num->Dc || !num->p || !num->q) { orc_free(num); return -1; }
    if (orc_permute_csc(n, Ap, Ai, Ax, is_complex, row_perm, col_perm, num->Bp, num->Bi, num->Bx)) { orc_free(num); return -1; }
    int rc = 0;
    if (equilibrate) rc = orc_ruiz(n, num->Bp, num->Bi, num->Bx, is_complex, ruiz_max_iter, ruiz_tol, num->Drp, num->Dcp,
                                   &num->ruiz_iters, err, errlen);
    else for (int64_t i = 0; i < n; i++) { num->Drp[i] = 1.0; num->Dcp[i] = 1.0; }
    if (rc == 0) rc = lu_partial(n, num->Bp, num->Bi, num->Bx, is_complex, pivot_rel, num, err, errlen);
    if (rc != 0) { orc_free(num); return rc; }
    for (int64_t k = 0; k < n; k++) {
        num->p[k] = row_perm[num->p_lu[k]];
        num->q[k] = col_perm[k];
        num->Dr[row_perm[k]] = num->Drp[k];
        num->Dc[col_perm[k]] = num->Dcp[k];
    }
    *out = num;
    return 0;
}

/* ------------------------------------------------------------------ solves (src/solve.c:11-60, src/numeric.c:88-131) */
static int tri_solve(const orc_numeric *f, void *xv, int trans)
{
    const int64_t n = f->n;
    const int64_t *Lp = f->Lp, *Li = f->Li, *Up = f->Up, *Ui = f->Ui;
    if (f->is_complex) {
        zc *x = xv; const zc *Lx = f->Lx, *Ux = f->Ux;
        if (trans == 0) {
            for (int64_t j = 0; j < n; j++) { zc xj = x[j]; if (xj == 0) continue;
                for (int64_t q = Lp[j]; q < Lp[j + 1]; q++) if (Li[q] != j) x[Li[q]] -= xj * Lx[q]; }
            for (int64_t j = n - 1; j >= 0; j--) {
                zc d = 0; int have = 0;
                for (int64_t q = Up[j]; q < Up[j + 1]; q++) if (Ui[q] == j) { d = Ux[q]; have = 1; break; }
                if (!have || d == 0) return -1;
                zc xj = x[j] / d; x[j] = xj; if (xj == 0) continue;
                for (int64_t q = Up[j]; q < Up[j + 1]; q++) if (Ui[q] < j) x[Ui[q]] -= xj * Ux[q];
            }
            return 0;
        }
        int cj = trans == 2;
        for (int64_t j = 0; j < n; j++) {
            zc s = x[j], d = 0; int have = 0;
            for (int64_t q = Up[j]; q < Up[j + 1]; q++) { zc v = cj ? conj(Ux[q]) : Ux[q];
                if (Ui[q] < j) s -= v * x[Ui[q]]; else if (Ui[q] == j) { d = v; have = 1; } }
            if (!have || d == 0) return -1;
            x[j] = s / d;
        }
        for (int64_t j = n - 1; j >= 0; j--) {
            zc s = x[j];
            for (int64_t q = Lp[j]; q < Lp[j + 1]; q++) if (Li[q] > j) s -= (cj ? conj(Lx[q]) : Lx[q]) * x[Li[q]];
            x[j] = s;
        }
        return 0;
    }
    double *x = xv; const double *Lx = f->Lx, *Ux = f->Ux;
    if (trans == 0) {
        for (int64_t j = 0; j < n; j++) { double xj = x[j]; if (xj == 0) continue;
            for (int64_t q = Lp[j]; q < Lp[j + 1]; q++) if (Li[q] != j) x[Li[q]] -= xj * Lx[q]; }
        for (int64_t j = n - 1; j >= 0; j--) {
            double d = 0; int have = 0;
            for (int64_t q = Up[j]; q < Up[j + 1]; q++) if (Ui[q] == j) { d = Ux[q]; have = 1; break; }
            if (!have || d == 0) return -1;
            double xj = x[j] / d; x[j] = xj; if (xj == 0) continue;
            for (int64_t q = Up[j]; q < Up[j + 1]; q++) if (Ui[q] < j) x[Ui[q]] -= xj * Ux[q];
        }
        return 0;
    }
    for (int64_t j = 0; j < n; j++) {
        double s = x[j], d = 0; int have = 0;
        for (int64_t q = Up[j]; q < Up[j + 1]; q++) { if (Ui[q] < j) s -= Ux[q] * x[Ui[q]]; else if (Ui[q] == j) { d = Ux[q]; have = 1; } }
        if (!have || d == 0) return -1;
        x[j] = s / d;
    }
    for (int64_t j = n - 1; j >= 0; j--) {
        double s = x[j];
        for (int64_t q = Lp[j]; q < Lp[j + 1]; q++) if (Li[q] > j) s -= Lx[q] * x[Li[q]];
        x[j] = s;
    }
    return 0;
}

int orc_solve(const orc_numeric *num, void *b, int64_t nrhs, int64_t ldb, int trans)
{
    const int64_t n = num->n;
    if (trans < 0 || trans > 2 || nrhs < 0 || ldb < n) return -3;
    const int64_t *p = num->p, *q = num->q;
    const double *Dr = num->Dr, *Dc = num->Dc;
    const size_t vs = num->is_complex ? sizeof(zc) : sizeof(double);
    void *w = malloc((size_t)(n > 0 ? n : 1) * vs);
    if (!w) return -1;
    for (int64_t r = 0; r < nrhs; r++) {
        if (num->is_complex) {
            zc *x = (zc *)b + r * ldb, *ww = w;
            if (trans == 0) for (int64_t k = 0; k < n; k++) ww[k] = Dr[p[k]] * x[p[k]];
            else            for (int64_t k = 0; k < n; k++) ww[k] = Dc[q[k]] * x[q[k]];
            if (tri_solve(num, w, trans)) { free(w); return -2; }
            if (trans == 0) for (int64_t k = 0; k < n; k++) x[q[k]] = Dc[q[k]] * ww[k];
            else            for (int64_t k = 0; k < n; k++) x[p[k]] = Dr[p[k]] * ww[k];
        } else {
            double *x = (double *)b + r * ldb, *ww = w;
            if (trans == 0) for (int64_t k = 0; k < n; k++) ww[k] = Dr[p[k]] * x[p[k]];
            else            for (int64_t k = 0; k < n; k++) ww[k] = Dc[q[k]] * x[q[k]];
            if (tri_solve(num, w, trans)) { free(w); return -2; }
            if (trans == 0) for (int64_t k = 0; k < n; k++) x[q[k]] = Dc[q[k]] * ww[k];
            else            for (int64_t k = 0; k < n; k++) x[p[k]] = Dr[p[k]] * ww[k];
        }
    }
    free(w);
    return 0;
}

void orc_free(orc_numeric *num)
{
    if (!num) return;
    free(num->Lp); free(num->Li); free(num->Lx); free(num->Up); free(num->Ui); free(num->Ux); free(num->p_lu);
    free(num->p); free(num->q); free(num->Dr); free(num->Dc); free(num->Drp); free(num->Dcp);
    free(num->Bp); free(num->Bi); free(num->Bx); free(num);
}

int64_t orc_n(const orc_numeric *f) { return f->n; }
const int64_t *orc_Lp(const orc_numeric *f) { return f->Lp; }
const int64_t *orc_Li(const orc_numeric *f) { return f->Li; }
const void *orc_Lx(const orc_numeric *f) { return f->Lx; }
const int64_t *orc_Up(const orc_numeric *f) { return f->Up; }
const int64_t *orc_Ui(const orc_numeric *f) { return f->Ui; }
const void *orc_Ux(const orc_numeric *f) { return f->Ux; }
const int64_t *orc_p_lu(const orc_numeric *f) { return f->p_lu; }
const int64_t *orc_p(const orc_numeric *f) { return f->p; }
const int64_t *orc_q(const orc_numeric *f) { return f->q; }
const double *orc_Dr(const orc_numeric *f) { return f->Dr; }
const double *orc_Dc(const orc_numeric *f) { return f->Dc; }
const double *orc_Drp(const orc_numeric *f) { return f->Drp; }
const double *orc_Dcp(const orc_numeric *f) { return f->Dcp; }
int orc_ruiz_iters(const orc_numeric *f) { return f->ruiz_iters; }
const int64_t *orc_Bp(const orc_numeric *f) { return f->Bp; }
const int64_t *orc_Bi(const orc_numeric *f) { return f->Bi; }
const void *orc_Bx(const orc_numeric *f) { return f->Bx; }
