// dev_common.cuh -- value types and small helpers shared by the CUDA kernels of libfplus (sm_100a).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace fpl {

struct __align__(16) cplx { double x, y; };

template <typename T> struct VT;
template <> struct VT<double> {
    static constexpr int cplx_ = 0;
    __device__ __forceinline__ static double zero() { return 0.0; }
    __device__ __forceinline__ static double one() { return 1.0; }
};
template <> struct VT<cplx> {
    static constexpr int cplx_ = 1;
    __device__ __forceinline__ static cplx zero() { return cplx{0.0, 0.0}; }
    __device__ __forceinline__ static cplx one() { return cplx{1.0, 0.0}; }
};

__device__ __forceinline__ double vabs(double a) { return fabs(a); }
__device__ __forceinline__ double vabs(cplx a) { return hypot(a.x, a.y); }
__device__ __forceinline__ double add(double a, double b) { return a + b; }
__device__ __forceinline__ cplx add(cplx a, cplx b) { return cplx{a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ double sub(double a, double b) { return a - b; }
__device__ __forceinline__ cplx sub(cplx a, cplx b) { return cplx{a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ double mul(double a, double b) { return a * b; }
__device__ __forceinline__ cplx mul(cplx a, cplx b) { return cplx{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
__device__ __forceinline__ double conjv(double a) { return a; }
__device__ __forceinline__ cplx conjv(cplx a) { return cplx{a.x, -a.y}; }
__device__ __forceinline__ double scal(double a, double s) { return a * s; }
__device__ __forceinline__ cplx scal(cplx a, double s) { return cplx{a.x * s, a.y * s}; }
__device__ __forceinline__ bool is_zero(double a) { return a == 0.0; }
__device__ __forceinline__ bool is_zero(cplx a) { return a.x == 0.0 && a.y == 0.0; }
// a / b; complex: Smith's scaled division (R. L. Smith, CACM 5(8), 1962)
__device__ __forceinline__ double divv(double a, double b) { return a / b; }
__device__ __forceinline__ cplx divv(cplx a, cplx b)
{
    if (fabs(b.y) <= fabs(b.x)) {
        double r = b.y / b.x, d = b.x + b.y * r;
        return cplx{(a.x + a.y * r) / d, (a.y - a.x * r) / d};
    }
    double r = b.x / b.y, d = b.y + b.x * r;
    return cplx{(a.x * r + a.y) / d, (a.y * r - a.x) / d};
}

// device status word: the first failure wins (code, then the smallest step / index)
enum : int {
    ST_OK = 0,
    ST_SINGULAR = 1,       // no admissible pivot at step `idx` (best, thr)
    ST_BORDER = 2,         // a border (dense) row chosen as pivot in front `idx`
    ST_ZERO_ROW = 3,       // Ruiz: row idx entirely zero
    ST_ZERO_COL = 4,       // Ruiz: column idx entirely zero
    ST_SOLVE_ZERO = 5,     // a zero diagonal of U in a solve
    ST_BAD_VALUE = 6,      // a non-finite input value at idx
};
struct DevStatus {
    int code;
    int pad;
    long long idx;
    double best, thr;
    // Ruiz
    unsigned long long res_bits;   // max |log| residual of the running iteration (bits of a non-negative double)
    int done, iters;
    unsigned long long amax_bits, amin_bits;
    unsigned int ticket;           // CTAs of the running fused backward-sweep launch that have finished (0 between launches)
    int pad2;
};

__device__ __forceinline__ void set_status(DevStatus *st, int code, long long idx, double best, double thr)
{
    // one winner: the first to move the code from 0
    if (atomicCAS(&st->code, 0, code) == 0) { st->idx = idx; st->best = best; st->thr = thr; }
}

__device__ __forceinline__ unsigned long long dbits(double v) { return (unsigned long long)__double_as_longlong(v); }
__device__ __forceinline__ double bitsd(unsigned long long b) { return __longlong_as_double((long long)b); }

}  // namespace fpl
