// schur_tc.hpp -- the precision form's Schur-complement update on the tensor cores (schur_tc.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>
#include "plan.hpp"

namespace fpl {

// The arithmetic of the Schur-complement GEMMs (the rest of the factorization is FP64 in every form)
enum SchurPrec : int {
    PREC_FP64 = 0,      // FP64 tensor cores (DMMA), the plain form
    PREC_FP32 = 1,      // FP32-accurate: operands split into two TF32 parts, three tcgen05 kind::tf32 products
    PREC_BF16X3 = 2,    // operands split into two BF16 parts, three tcgen05 kind::f16 products
    PREC_TF32 = 3,      // one TF32 part, one tcgen05 kind::tf32 product
};

// Bytes of workspace schur_tc needs for an M x K times K x N update (the split, K-major operand copies).
size_t schur_tc_workspace(int prec, int64_t M, int64_t N, int64_t K, int cplx);
// Whether the tensor-core path takes this shape (32-bit tile indices; the driver's tensor-map encoder present).
bool schur_tc_supported(int64_t M, int64_t N, int64_t K, int cplx);
// Cout[i, j] = Cin[rmap ? rmap[i] : i, j] - (A B)[i, j] on stream s (asynchronous): A M x K (lda), B K x N (ldb), Cin
// (ldci), Cout (ldco), all FP64 column-major device arrays (complex: interleaved pairs, cplx = 1).  prec is PREC_FP32,
// PREC_BF16X3 or PREC_TF32.  ws: at least schur_tc_workspace() bytes of device memory.  A wait in the kernel that runs
// out of time sets bit 0 (or 1) of *err (device memory).  Returns 0, or a negative value when the launch could not be
// made (workspace too small, no tensor-map encoder, a launch error).
// om: where each output element goes (OutMap; identity when om.col is null).
int schur_tc(int prec, int cplx, int64_t M, int64_t N, int64_t K, const double *A, int64_t lda, const double *B, int64_t ldb,
             const double *Cin, int64_t ldci, const int *rmap, double *Cout, int64_t ldco, void *ws, size_t ws_bytes,
             unsigned *err, cudaStream_t s, OutMap om = OutMap{});

}  // namespace fpl
