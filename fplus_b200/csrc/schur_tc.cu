// schur_tc.cu -- the Schur-complement update of the precision form on the 5th-generation tensor cores (sm_100a).
//
//   Cout[i, j] = Cin[rmap[i], j] - sum_k A[i, k] B[k, j]        (i < M, j < N; A = L21, B = U12, C = the front's CB)
//
// A (M x K) and B (K x N) are FP64 (real or complex), column-major, as the factorization keeps them; Cin and Cout are
// FP64.  The product runs on tcgen05.mma with FP32 accumulation in tensor memory, in one of three precisions:
//
//   PREC_FP32    each FP64 operand split into two TF32 parts (x = hi + lo, ~22 significant bits), three products
//                hi*hi + hi*lo + lo*hi (kind::tf32): the accuracy of an FP32 GEMM
//   PREC_BF16X3  the same split into two BF16 parts (~16 bits), three products (kind::f16, BF16 inputs)
//   PREC_TF32    one TF32 part, one product (kind::tf32)
//
// The splits are folded into the K dimension: a pre-pass writes A_ext = [A_hi | A_hi | A_lo] (M x 3K) and
// B_ext = [B_hi ; B_lo ; B_hi] (3K x N), both K-major, so that one GEMM over K' = 3K forms the three products.  A complex
// product is folded the same way: with A2 = [Ar | -Ai] (M x 2K), column 2c of B2 = [Br(:, c) ; Bi(:, c)] and column 2c + 1
// = [Bi(:, c) ; -Br(:, c)], the real GEMM A2 B2 (M x 2N) holds Re(A B)(:, c) in column 2c and Im(A B)(:, c) in 2c + 1.
//
// The GEMM is persistent and warp-specialised: warp 0 issues TMA loads (128-byte swizzled K-major tiles, 4-stage ring),
// warp 1 issues the MMAs (one elected thread; 128 x 256 tiles, the accumulator double-buffered in tensor memory: 2 x 256
// of the 512 columns), warps 2..9 drain the accumulators (tcgen05.ld) and write Cout = Cin - D in FP64 while the next tile
// is multiplied.  Every wait is bounded in time: a wait that runs out sets the error word and the kernel winds down.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <cstring>
#include <mutex>
#include "schur_tc.hpp"

namespace fpl {

namespace {

constexpr int BM = 128, BN = 256, STAGES = 4, ROWB = 128;       // tile rows / columns, ring stages, bytes of K per row
constexpr int A_BYTES = BM * ROWB, B_BYTES = BN * ROWB, STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int EPI_WARPS = 8, THREADS = 32 * (2 + EPI_WARPS);
constexpr size_t SMEM_BYTES = (size_t)STAGES * STAGE_BYTES + 1024 /* alignment */ + 256 /* barriers, TMEM address */;
constexpr long long WAIT_CYCLES = 4000000000LL;                   // about 2 s at 1.9 GHz

struct cplx_t { double x, y; };

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    return ok != 0;
}
// wait for the phase of parity `parity` to complete; false (and the error word set) when it has not within the limit
// or another role has given up already
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *abort, unsigned *err)
{
    if (mbar_try(bar, parity)) return true;
    const long long t0 = clock64();
    for (;;) {
        if (mbar_try(bar, parity)) return true;
        if (*abort) return false;
        if (clock64() - t0 > WAIT_CYCLES) { *abort = 1; atomicOr(err, 1u); return false; }
    }
}
// the same wait, bounded in time only (the wind-down of a role after an abort)
__device__ __forceinline__ void mbar_wait_drain(uint32_t bar, uint32_t parity, unsigned *err)
{
    const long long t0 = clock64();
    while (!mbar_try(bar, parity))
        if (clock64() - t0 > WAIT_CYCLES) { atomicOr(err, 2u); return; }
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                 ::"r"(dst), "l"((uint64_t)map), "r"(x), "r"(y), "r"(bar) : "memory");
}
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// shared-memory matrix descriptor of a K-major tile with 128-byte rows, 128-byte swizzle: 8-row groups 1024 bytes apart
__device__ __forceinline__ uint64_t sdesc(uint32_t addr)
{
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) | ((uint64_t)1 << 46) |
           ((uint64_t)2 << 61);
}

template <bool BF16>
__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accum)
{
    if constexpr (BF16)
        asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                     "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                     ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accum) : "memory");
    else
        asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                     "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
                     ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accum) : "memory");
}

// 32 consecutive accumulator columns of this warp's 32 lanes (one row per lane)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v)
{
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                 "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
                   "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
                   "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; j++) v[j] = __uint_as_float(r[j]);
}

// ---------------------------------------------------------------------------------------------------------------------
// The GEMM.  D (M x Nd, FP32) = A_ext (M x Kp) B_ext^T (Nd x Kp), both K-major in global memory behind the tensor maps;
// kb128 = Kp * element size / 128 stages per tile.  The epilogue writes Cout (real: column d of D is column d of C;
// complex: columns 2c, 2c + 1 of D are the real and imaginary parts of column c).
template <bool BF16, bool CPLX>
__global__ void __launch_bounds__(THREADS, 1) k_schur_tc(const __grid_constant__ CUtensorMap tmA,
                                                        const __grid_constant__ CUtensorMap tmB, int M, int Nd, int kb128,
                                                        const double *Cin, int64_t ldci, const int *__restrict__ rmap,
                                                        double *Cout, int64_t ldco, unsigned *err, OutMap om)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    unsigned char *sm = (unsigned char *)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);   // 1024-byte aligned ring
    uint64_t *bars = (uint64_t *)(sm + (size_t)STAGES * STAGE_BYTES);
    // bars: full[STAGES], empty[STAGES], tfull[2], tempty[2], done; then the TMEM base address and the abort flag
    uint32_t *tmem_slot = (uint32_t *)(bars + 2 * STAGES + 5);
    volatile int *abort = (volatile int *)(tmem_slot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t full0 = smem_u32(bars), empty0 = full0 + 8 * STAGES, tfull0 = empty0 + 8 * STAGES, tempty0 = tfull0 + 16,
                   done0 = tempty0 + 16;
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) { mbar_init(full0 + 8 * s, 1); mbar_init(empty0 + 8 * s, 1); }
        for (int b = 0; b < 2; b++) { mbar_init(tfull0 + 8 * b, 1); mbar_init(tempty0 + 8 * b, EPI_WARPS); }
        mbar_init(done0, 1);
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {       // the whole warp allocates the 512 tensor-memory columns (one CTA per SM)
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(tmem_slot)) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const int mt = (M + BM - 1) / BM, nt = (Nd + BN - 1) / BN, ntiles = mt * nt;
    constexpr int KSTEP = BF16 ? 16 : 8;                          // K of one MMA
    constexpr int MMAS = (ROWB / (BF16 ? 2 : 4)) / KSTEP;         // MMAs per 128-byte row: 4
    const uint32_t idesc = (1u << 4) | ((BF16 ? 1u : 2u) << 7) | ((BF16 ? 1u : 2u) << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);
    const uint32_t ring = smem_u32(sm);

    if (warp == 0) {
        if (lane == 0) {
            int s = 0; uint32_t ph = 0;
            long long issued = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                const int m0 = (t % mt) * BM, n0 = (t / mt) * BN;
                for (int kb = 0; kb < kb128 && ok; kb++) {
                    if (!(ok = mbar_wait(empty0 + 8 * s, ph ^ 1, abort, err))) break;
                    const uint32_t st = ring + (uint32_t)s * STAGE_BYTES;
                    mbar_expect_tx(full0 + 8 * s, STAGE_BYTES);
                    const int x = kb * (ROWB / (BF16 ? 2 : 4));
                    tma_load_2d(st, &tmA, x, m0, full0 + 8 * s);
                    tma_load_2d(st + A_BYTES, &tmB, x, n0, full0 + 8 * s);
                    issued++;
                    if (++s == STAGES) { s = 0; ph ^= 1; }
                }
            }
            // before the CTA may leave, the last loads have landed (their full barriers complete whatever the MMA
            // thread does): the fills issued - 1, issued - 2, ... of the ring
            for (long long f = issued - 1; f >= 0 && f >= issued - STAGES; f--)
                mbar_wait_drain(full0 + 8 * (uint32_t)(f % STAGES), (uint32_t)((f / STAGES) & 1), err);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int s = 0; uint32_t ph = 0, acc = 0, aph = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                if (!(ok = mbar_wait(tempty0 + 8 * acc, aph ^ 1, abort, err))) break;
                tc_fence_after();
                const uint32_t td = tmem + acc * BN;
                for (int kb = 0; kb < kb128; kb++) {
                    if (!(ok = mbar_wait(full0 + 8 * s, ph, abort, err))) break;
                    tc_fence_after();
                    const uint32_t st = ring + (uint32_t)s * STAGE_BYTES;
#pragma unroll
                    for (int k = 0; k < MMAS; k++)
                        mma<BF16>(td, sdesc(st + 32 * k), sdesc(st + A_BYTES + 32 * k), idesc, (kb | k) != 0);
                    tc_commit(empty0 + 8 * s);                    // the stage is free once these MMAs have read it
                    if (++s == STAGES) { s = 0; ph ^= 1; }
                }
                if (!ok) break;
                tc_commit(tfull0 + 8 * acc);                      // the accumulator is complete
                acc ^= 1; if (acc == 0) aph ^= 1;
            }
            // every MMA issued has completed before the tensor memory is released
            tc_commit(done0);
            mbar_wait_drain(done0, 0, err);
        }
    } else {
        const int e = warp - 2, q = warp & 3, half = e >> 2;     // lane quarter q (rows 32q..), column half
        uint32_t acc = 0, aph = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
            const int m0 = (t % mt) * BM, n0 = (t / mt) * BN;
            bool ok = true;
            if (lane == 0) ok = mbar_wait(tfull0 + 8 * acc, aph, abort, err);
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) break;
            tc_fence_after();
            const int row = m0 + q * 32 + lane;
            const bool live = row < M;
            const int64_t src = live ? (int64_t)(rmap ? rmap[row] : row) : 0;
            const int64_t orow = om.col ? (row < om.nslot ? om.slot + row : om.tau + (row - om.nslot)) : row;
            for (int c0 = half * (BN / 2); c0 < (half + 1) * (BN / 2); c0 += 32) {
                float v[32];
                __syncwarp();
                tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + acc * BN + c0, v);
                const int d0 = n0 + c0;
                if (!live || d0 >= Nd) continue;
                if constexpr (!CPLX) {
                    double cin[32];
#pragma unroll
                    for (int j = 0; j < 32; j++) cin[j] = d0 + j < Nd ? Cin[src + (int64_t)(d0 + j) * ldci] : 0.0;
#pragma unroll
                    for (int j = 0; j < 32; j++)
                        if (d0 + j < Nd) Cout[orow + (om.col ? om.col[d0 + j] : (int64_t)(d0 + j)) * ldco] = cin[j] - (double)v[j];
                } else {
                    const cplx_t *ci = (const cplx_t *)Cin;
                    cplx_t *co = (cplx_t *)Cout;
                    const int c = d0 >> 1;                        // d0 is even: 32 D columns = 16 complex columns
                    cplx_t cin[16];
#pragma unroll
                    for (int j = 0; j < 16; j++) cin[j] = d0 + 2 * j < Nd ? ci[src + (int64_t)(c + j) * ldci] : cplx_t{0.0, 0.0};
#pragma unroll
                    for (int j = 0; j < 16; j++)
                        if (d0 + 2 * j < Nd)
                            co[orow + (om.col ? om.col[c + j] : (int64_t)(c + j)) * ldco] =
                                cplx_t{cin[j].x - (double)v[2 * j], cin[j].y - (double)v[2 * j + 1]};
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(tempty0 + 8 * acc);
            acc ^= 1; if (acc == 0) aph ^= 1;
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
    }
}

// ---------------------------------------------------------------------------------------------------------------------
// The pre-pass: the split, K-major operands.  One part of x: TF32 (round to nearest, ties away: cvt.rna.tf32.f32, kept
// in an FP32 container) or BF16 (round to nearest even).  The second part is the same rounding of the remainder.
__device__ __forceinline__ float tf32_rn(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}
template <bool BF16> struct SplitT;
template <> struct SplitT<false> {
    using E = float;
    __device__ static void split(double x, float &hi, float &lo)
    {
        hi = tf32_rn((float)x);
        lo = tf32_rn((float)(x - (double)hi));
    }
};
template <> struct SplitT<true> {
    using E = __nv_bfloat16;
    __device__ static void split(double x, __nv_bfloat16 &hi, __nv_bfloat16 &lo)
    {
        hi = __double2bfloat16(x);
        lo = __double2bfloat16(x - (double)__bfloat162float(hi));
    }
};

// A_ext row m (Kp entries): the base row of A2 (real: A(m, :); complex: [Re A(m, :) | -Im A(m, :)]) as parts
// [hi | hi | lo] (P = 3) or [hi] (P = 1), zero-padded to Kp.  One warp per row, the row's source entries strided by lda.
template <bool BF16, bool CPLX>
__global__ void k_split_a(const double *__restrict__ A, int64_t lda, int M, int K, int P, int Kp,
                          typename SplitT<BF16>::E *__restrict__ out)
{
    using E = typename SplitT<BF16>::E;
    const int K2 = CPLX ? 2 * K : K;
    for (int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; w < M; w += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int lane = threadIdx.x & 31;
        E *o = out + w * (int64_t)Kp;
        for (int k = lane; k < Kp; k += 32) {
            E v = E(0.0f);
            const int part = k / K2, kk = k - part * K2;
            if (part < P) {
                double x;
                if (CPLX) { const int kc = kk < K ? kk : kk - K; x = A[2 * (w + (int64_t)kc * lda) + (kk < K ? 0 : 1)]; if (kk >= K) x = -x; }
                else x = A[w + (int64_t)kk * lda];
                E hi, lo;
                SplitT<BF16>::split(x, hi, lo);
                v = (P == 3 && part == 2) ? lo : hi;
            }
            o[k] = v;
        }
    }
}

// B_ext row d (the d-th column of B2): real: B(:, d); complex: d = 2c: [Re B(:, c) ; Im B(:, c)], d = 2c + 1:
// [Im B(:, c) ; -Re B(:, c)]; as parts [hi | lo | hi] (P = 3) or [hi] (P = 1), zero-padded to Kp
template <bool BF16, bool CPLX>
__global__ void k_split_b(const double *__restrict__ B, int64_t ldb, int Nd, int K, int P, int Kp,
                          typename SplitT<BF16>::E *__restrict__ out)
{
    using E = typename SplitT<BF16>::E;
    const int K2 = CPLX ? 2 * K : K;
    for (int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; w < Nd; w += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int lane = threadIdx.x & 31;
        E *o = out + w * (int64_t)Kp;
        const int64_t col = CPLX ? (w >> 1) : w;
        for (int k = lane; k < Kp; k += 32) {
            E v = E(0.0f);
            const int part = k / K2, kk = k - part * K2;
            if (part < P) {
                double x;
                if (CPLX) {
                    const bool top = kk < K, imcol = (w & 1) != 0;
                    const int kc = top ? kk : kk - K;
                    const double *z = B + 2 * (kc + col * ldb);
                    // d = 2c: [Re ; Im]; d = 2c + 1: [Im ; -Re]
                    x = !imcol ? (top ? z[0] : z[1]) : (top ? z[1] : -z[0]);
                } else x = B[kk + col * ldb];
                E hi, lo;
                SplitT<BF16>::split(x, hi, lo);
                v = (P == 3 && part == 1) ? lo : hi;
            }
            o[k] = v;
        }
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    return fn;
}

// a 2D K-major tensor map: rows x Kp elements of esize bytes, boxes of box_rows x 128 bytes, 128-byte swizzle
bool make_map(CUtensorMap *m, const void *base, int64_t rows, int64_t Kp, int esize, int box_rows, bool bf16)
{
    auto enc = encode_fn();
    if (!enc) return false;
    cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)Kp * (cuuint64_t)esize};
    cuuint32_t box[2] = {(cuuint32_t)(ROWB / esize), (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    return enc(m, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(base), dims,
               strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <bool BF16, bool CPLX>
int run(int P, int64_t M, int64_t N, int64_t K, const double *A, int64_t lda, const double *B, int64_t ldb, const double *Cin,
        int64_t ldci, const int *rmap, double *Cout, int64_t ldco, void *ws, size_t ws_bytes, unsigned *err, cudaStream_t s,
        int nsm, OutMap om)
{
    using E = typename SplitT<BF16>::E;
    const int64_t esz = sizeof(E), per = ROWB / esz;
    const int64_t Nd = CPLX ? 2 * N : N, K2 = CPLX ? 2 * K : K;
    if (!schur_tc_supported(M, N, K, CPLX)) return -5;
    const int64_t Kp = (P * K2 + per - 1) / per * per;
    const size_t abytes = ((size_t)M * Kp * esz + 1023) & ~(size_t)1023, bbytes = (size_t)Nd * Kp * esz;
    if (abytes + bbytes > ws_bytes) return -1;
    E *Ae = (E *)ws, *Be = (E *)((char *)ws + abytes);
    k_split_a<BF16, CPLX><<<(unsigned)std::min<int64_t>((M + 7) / 8, 4096), 256, 0, s>>>(A, lda, (int)M, (int)K, P, (int)Kp, Ae);
    k_split_b<BF16, CPLX><<<(unsigned)std::min<int64_t>((Nd + 7) / 8, 4096), 256, 0, s>>>(B, ldb, (int)Nd, (int)K, P, (int)Kp, Be);
    CUtensorMap ma, mb;
    if (!make_map(&ma, Ae, M, Kp, (int)esz, BM, BF16) || !make_map(&mb, Be, Nd, Kp, (int)esz, BN, BF16)) return -2;
    static thread_local int attr = 0;
    if (!(attr & (1 << ((BF16 ? 2 : 0) + (CPLX ? 1 : 0))))) {
        if (cudaFuncSetAttribute(k_schur_tc<BF16, CPLX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES) != cudaSuccess)
            return -3;
        attr |= 1 << ((BF16 ? 2 : 0) + (CPLX ? 1 : 0));
    }
    const int64_t tiles = ((M + BM - 1) / BM) * ((Nd + BN - 1) / BN);
    const int grid = (int)std::min<int64_t>(tiles, nsm);
    k_schur_tc<BF16, CPLX><<<grid, THREADS, SMEM_BYTES, s>>>(ma, mb, (int)M, (int)Nd, (int)(Kp * esz / ROWB), Cin, ldci, rmap,
                                                             Cout, ldco, err, om);
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

}  // namespace

size_t schur_tc_workspace(int prec, int64_t M, int64_t N, int64_t K, int cplx)
{
    const int64_t esz = prec == PREC_BF16X3 ? 2 : 4, per = ROWB / esz, P = prec == PREC_TF32 ? 1 : 3;
    const int64_t Nd = cplx ? 2 * N : N, K2 = cplx ? 2 * K : K;
    const int64_t Kp = (P * K2 + per - 1) / per * per;
    return (((size_t)M * Kp * esz + 1023) & ~(size_t)1023) + (size_t)Nd * Kp * esz;
}

bool schur_tc_supported(int64_t M, int64_t N, int64_t K, int cplx)
{
    // 32-bit tile coordinates and row indices; at least one whole tile (the TMA boxes are 128 and 256 rows)
    const int64_t Nd = cplx ? 2 * N : N;
    return M >= BM && Nd >= BN && K > 0 && M < (1LL << 31) && Nd < (1LL << 31) && K < (1LL << 24) && encode_fn() != nullptr;
}

int schur_tc(int prec, int cplx, int64_t M, int64_t N, int64_t K, const double *A, int64_t lda, const double *B, int64_t ldb,
             const double *Cin, int64_t ldci, const int *rmap, double *Cout, int64_t ldco, void *ws, size_t ws_bytes,
             unsigned *err, cudaStream_t s, OutMap om)
{
    static int nsm = 0;
    if (!nsm) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (nsm <= 0) nsm = 148;
    }
    const int P = prec == PREC_TF32 ? 1 : 3;
    if (prec == PREC_BF16X3)
        return cplx ? run<true, true>(P, M, N, K, A, lda, B, ldb, Cin, ldci, rmap, Cout, ldco, ws, ws_bytes, err, s, nsm, om)
                    : run<true, false>(P, M, N, K, A, lda, B, ldb, Cin, ldci, rmap, Cout, ldco, ws, ws_bytes, err, s, nsm, om);
    return cplx ? run<false, true>(P, M, N, K, A, lda, B, ldb, Cin, ldci, rmap, Cout, ldco, ws, ws_bytes, err, s, nsm, om)
                : run<false, false>(P, M, N, K, A, lda, B, ldb, Cin, ldci, rmap, Cout, ldco, ws, ws_bytes, err, s, nsm, om);
}

}  // namespace fpl
