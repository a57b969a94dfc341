/* amd.h -- test infrastructure: SuiteSparse AMD's names as the reference's src/order.c uses them, served by
 * oracle/ref_stub.c (an injected order; no minimum-degree code). */
#ifndef ORACLE_STUB_AMD_H
#define ORACLE_STUB_AMD_H
#include <stdint.h>
#define AMD_CONTROL 5
#define AMD_INFO 20
#define AMD_OK 0
#define AMD_OK_BUT_JUMBLED 1
void amd_l_defaults(double Control[AMD_CONTROL]);
int amd_l_order(int64_t n, const int64_t *Ap, const int64_t *Ai, int64_t *P, double Control[AMD_CONTROL], double Info[AMD_INFO]);
#endif
