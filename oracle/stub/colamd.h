/* colamd.h -- test infrastructure: the declarations the reference's src/order.c compiles against (SuiteSparse COLAMD's
 * names and calling convention), served by oracle/ref_stub.c, which returns an order injected by the test instead of
 * running COLAMD (SuiteSparse is not installed here). */
#ifndef ORACLE_STUB_COLAMD_H
#define ORACLE_STUB_COLAMD_H
#include <stddef.h>
#include <stdint.h>
#define COLAMD_KNOBS 20
#define COLAMD_STATS 20
#define COLAMD_STATUS 3
size_t colamd_l_recommended(int64_t nnz, int64_t n_row, int64_t n_col);
void colamd_l_set_defaults(double knobs[COLAMD_KNOBS]);
int64_t colamd_l(int64_t n_row, int64_t n_col, int64_t Alen, int64_t *A, int64_t *p, double knobs[COLAMD_KNOBS],
                 int64_t stats[COLAMD_STATS]);
#endif
