/* ref_callers.c -- test infrastructure: the reference's own C caller, tests/c/test_fplus.c, built against this
 * repository's include/fplus.h and linked with fplus_b200/libfplus.so (oracle/Makefile, target `callers`).
 *
 * The reference file is compiled into this translation unit with its main renamed, so that this main can run the cases
 * that exercise partial pivoting, the production path, in the reference's order: the high-level analyze / factor /
 * solve round trips on its random matrices with dense lines (complex unscaled, complex and real with row scales over 12
 * decades; every solve direction, 3 right-hand sides, backward error < 1e-12), the Ruiz range guard and the input
 * validation of fplus_factor_sn / fplus_analyze.  Its rook / full pivoting and incomplete-LU cases need the row kernel,
 * which this library does not build, and are not called.  Exit status 0 when every check passes. */
#define main fplus_reference_test_main
#include "test_fplus.c"
#undef main

int main(void)
{
    test_high_level(1, 0.0, FPLUS_PIVOT_PARTIAL);
    test_high_level(1, 6.0, FPLUS_PIVOT_PARTIAL);
    test_high_level(0, 6.0, FPLUS_PIVOT_PARTIAL);
    test_ruiz_range_guard();
    test_validation();
    if (failures) { printf("%d check(s) failed\n", failures); return 1; }
    printf("partial-pivoting checks of the reference's C test passed\n");
    return 0;
}
