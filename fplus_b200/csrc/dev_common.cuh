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
// a - l p in fused multiply-adds (complex: four)
__device__ __forceinline__ double msub(double a, double l, double p) { return fma(-l, p, a); }
__device__ __forceinline__ cplx msub(cplx a, cplx l, cplx p)
{
    return cplx{fma(l.y, p.y, fma(-l.x, p.x, a.x)), fma(-l.y, p.x, fma(-l.x, p.y, a.y))};
}
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

// ---------------------------------------------------------------------------------------------------------------------
// Pivot keys.  Partial pivoting picks the largest modulus (FPLUS src/factor_sn_panel.inc:225-231 compares fabs / cabs).
// The key of a value is an unsigned integer that orders values as their moduli do, with no overflow or underflow:
//   real     the bits of |x| (non-negative doubles order as their bit patterns); exact
//   complex  |x|^2 = m * 2^E (m in [1, 2)) packed as (E + 1023 + PIVKEY_OFF) << 50 | the top 50 fraction bits of m.
//            Where |x|^2 is a normal double in [2^-1000, 2^1000] that is the double's own bits shifted right by two
//            (plus the offset); elsewhere the components are first scaled by a power of two (exact), so both routes
//            give the same key.  E ranges over [-2148, 2048], so the packed exponent fits 13 bits.
// Zero and NaN have key 0; an infinite modulus the largest key.
constexpr unsigned long long PIVKEY_OFF = 1200ull;
constexpr unsigned long long PIVKEY_INF = 8191ull << 50;

__device__ __forceinline__ unsigned long long pivkey(double a)
{
    const double m = fabs(a);
    return m == m ? (unsigned long long)__double_as_longlong(m) : 0ull;
}
static __device__ __noinline__ unsigned long long pivkey_wide(double re, double im)
{
    const double ax = fabs(re), ay = fabs(im);
    if (!(ax == ax) || !(ay == ay)) return 0ull;
    const double s = fmax(ax, ay);
    if (s == 0.0) return 0ull;
    if (isinf(s)) return PIVKEY_INF;
    int e = 0, f = 0;
    frexp(s, &e);                                                  // s = (0.5 .. 1) * 2^e
    const double xs = ldexp(ax, -e), ys = ldexp(ay, -e);           // exact (a component far below the other may round)
    const double q = __dadd_rn(__dmul_rn(xs, xs), __dmul_rn(ys, ys));   // |x|^2 * 2^(-2e), in [0.25, 2)
    const double m = frexp(q, &f);                                 // q = m * 2^f, m in [0.5, 1)
    const long long E = (long long)f + 2LL * e - 1;                // |x|^2 = (2m) * 2^E
    const unsigned long long frac = (unsigned long long)__double_as_longlong(2.0 * m) & ((1ull << 52) - 1);
    return ((unsigned long long)(E + 1023 + (long long)PIVKEY_OFF) << 50) | (frac >> 2);
}
__device__ __forceinline__ unsigned long long pivkey(cplx a)
{
    const double q = __dadd_rn(__dmul_rn(a.x, a.x), __dmul_rn(a.y, a.y));
    if (q >= 0x1p-1000 && q <= 0x1p1000) return ((unsigned long long)__double_as_longlong(q) >> 2) + (PIVKEY_OFF << 50);
    if (a.x == 0.0 && a.y == 0.0) return 0ull;                     // exact zeros (common in a front) stay off the slow path
    return pivkey_wide(a.x, a.y);
}
// the key of a value of modulus t >= 0
template <typename T> __device__ __forceinline__ unsigned long long pivkey_of_modulus(double t);
template <> __device__ __forceinline__ unsigned long long pivkey_of_modulus<double>(double t) { return pivkey(t); }
template <> __device__ __forceinline__ unsigned long long pivkey_of_modulus<cplx>(double t) { return pivkey(cplx{t, 0.0}); }

// the largest 64-bit key over the warp: two 32-bit reductions (the high word, then the low word among the lanes that hold
// the high word)
__device__ __forceinline__ unsigned long long warp_max_key(unsigned long long key)
{
    const unsigned khi = (unsigned)(key >> 32);
    const unsigned hi = __reduce_max_sync(0xffffffffu, khi);
    const unsigned lo = __reduce_max_sync(0xffffffffu, khi == hi ? (unsigned)key : 0u);
    return ((unsigned long long)hi << 32) | lo;
}

// the smallest 64-bit value over the warp (two 32-bit reductions)
__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v)
{
    const unsigned vhi = (unsigned)(v >> 32);
    const unsigned hi = __reduce_min_sync(0xffffffffu, vhi);
    const unsigned lo = __reduce_min_sync(0xffffffffu, vhi == hi ? (unsigned)v : 0xffffffffu);
    return ((unsigned long long)hi << 32) | lo;
}
// the lane holding the best candidate of the warp: the largest key (>= 0; -1: no candidate), ties to the smaller row id
// (ids are distinct and >= 0); -1 when no lane holds one
__device__ __forceinline__ int warp_argbest(long long key, long long rid)
{
    const unsigned long long k = key >= 0 ? (unsigned long long)key + 1ull : 0ull;
    const unsigned long long m = warp_max_key(k);
    if (m == 0ull) return -1;
    const unsigned long long rmin = warp_min_u64(k == m ? (unsigned long long)rid : ~0ull);
    const unsigned bal = __ballot_sync(0xffffffffu, k == m && (unsigned long long)rid == rmin);
    return __ffs(bal) - 1;
}

// 1 / p for the pivot: conj(p) / |p|^2 with the components scaled by max(|re|, |im|) first (no overflow or underflow of the
// squares); real: 1 / p
// (__drcp_rn: the correctly rounded reciprocal, the same value as the IEEE quotient 1.0 / q)
__device__ __forceinline__ double recip(double p) { return __drcp_rn(p); }
__device__ __forceinline__ cplx recip(cplx p)
{
    const double q = p.x * p.x + p.y * p.y;
    if (q > 1e-300 && q < 1e300) { const double d = __drcp_rn(q); return cplx{p.x * d, -p.y * d}; }
    const double s = fmax(fabs(p.x), fabs(p.y)), is = __drcp_rn(s);     // scaled: no overflow or underflow
    const double a = p.x * is, b = p.y * is, d = __drcp_rn(a * a + b * b);
    return cplx{a * d * is, -b * d * is};
}

// a load that bypasses L1 (values another CTA wrote during this launch)
__device__ __forceinline__ double ldcg_v(const double *p) { return __ldcg(p); }
__device__ __forceinline__ cplx ldcg_v(const cplx *p)
{
    const double2 v = __ldcg(reinterpret_cast<const double2 *>(p));
    return cplx{v.x, v.y};
}
// a counter read with acquire semantics, and an increment with release semantics (GPU scope): the writes the
// incrementing thread made, or saw through a barrier, before the increment are visible to a thread whose acquire reads it
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_add_u32(unsigned *p, unsigned v)
{
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
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
    ST_RANGE = 7,          // a captured factorization met values beyond 2^+-500 (the range guard needs the host path)
    ST_WAIT = 8,           // a wait of a multi-CTA pivot search for the other CTAs' candidates ran out of time
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
    unsigned int tc_err;           // a tensor-core Schur update whose wait ran out of time (bits, see schur_tc.hpp)
};

__device__ __forceinline__ void set_status(DevStatus *st, int code, long long idx, double best, double thr)
{
    // one winner: the first to move the code from 0
    if (atomicCAS(&st->code, 0, code) == 0) { st->idx = idx; st->best = best; st->thr = thr; }
}

__device__ __forceinline__ unsigned long long dbits(double v) { return (unsigned long long)__double_as_longlong(v); }
__device__ __forceinline__ double bitsd(unsigned long long b) { return __longlong_as_double((long long)b); }

}  // namespace fpl
