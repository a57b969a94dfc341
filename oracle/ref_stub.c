/* ref_stub.c -- test infrastructure only (never shipped).
 *
 * The reference's src/order.c calls SuiteSparse COLAMD / AMD, which this image lacks.  These stand-ins let the
 * unmodified order.c compile and run: the test injects the column order (fplusref_inject_order) and the next
 * colamd_l / amd_l_order call returns it.  Everything else order.c does -- dense-line pinning, the row order, the
 * column-etree postorder, the composition of the orders -- is the reference's own code, so the product's analysis can be
 * checked against it with the same injected fill-reducing order. */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "colamd.h"
#include "amd.h"

static int64_t *inj = NULL, inj_n = -1;

void fplusref_inject_order(const int64_t *perm, int64_t n)
{
    free(inj); inj = NULL; inj_n = -1;
    if (!perm || n < 0) return;
    inj = (int64_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int64_t));
    if (!inj) return;
    memcpy(inj, perm, (size_t)n * sizeof(int64_t));
    inj_n = n;
}

size_t colamd_l_recommended(int64_t nnz, int64_t n_row, int64_t n_col)
{
    (void)n_row;
    return (size_t)(nnz + n_col + 1);
}

void colamd_l_set_defaults(double knobs[COLAMD_KNOBS]) { for (int k = 0; k < COLAMD_KNOBS; k++) knobs[k] = 0; }

int64_t colamd_l(int64_t n_row, int64_t n_col, int64_t Alen, int64_t *A, int64_t *p, double knobs[COLAMD_KNOBS],
                 int64_t stats[COLAMD_STATS])
{
    (void)n_row; (void)Alen; (void)A; (void)knobs;
    for (int k = 0; k < COLAMD_STATS; k++) stats[k] = 0;
    if (inj_n != n_col) { stats[COLAMD_STATUS] = -999; return 0; }
    memcpy(p, inj, (size_t)n_col * sizeof(int64_t));
    return 1;
}

void amd_l_defaults(double Control[AMD_CONTROL]) { for (int k = 0; k < AMD_CONTROL; k++) Control[k] = 0; }

int amd_l_order(int64_t n, const int64_t *Ap, const int64_t *Ai, int64_t *P, double Control[AMD_CONTROL], double Info[AMD_INFO])
{
    (void)Ap; (void)Ai; (void)Control; (void)Info;
    if (inj_n != n) return -2;
    memcpy(P, inj, (size_t)n * sizeof(int64_t));
    return AMD_OK;
}
