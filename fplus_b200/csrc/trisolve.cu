// trisolve.cu -- level-scheduled triangular sweeps on caller-supplied CSC factors (see trisolve.hpp).
//
// FPLUS solves such factors column by column on the CPU (src/solve.c:11-74, src/solve_plan.c:568-659).  Here each sweep
// is row-oriented: row r of the sweep gathers its entries (one warp per row, summed by a fixed butterfly, so the result
// does not depend on scheduling) and the rows are taken in levels of the dependency DAG.  The transposed solves read the
// CSC columns directly as rows; the untransposed ones read a row list built once on the host.
#include "trisolve.hpp"
#include "numeric.hpp"
#include "dev_common.cuh"
#include <algorithm>
#include <cstring>

namespace fpl {

// ---------------------------------------------------------------------------------------------------------------------
// device

template <typename T> __device__ __forceinline__ T wsum(T v);
template <> __device__ __forceinline__ double wsum<double>(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
template <> __device__ __forceinline__ cplx wsum<cplx>(cplx v)
{
    for (int o = 16; o > 0; o >>= 1) { v.x += __shfl_xor_sync(0xffffffffu, v.x, o); v.y += __shfl_xor_sync(0xffffffffu, v.y, o); }
    return v;
}

template <typename T, bool CJ> __device__ __forceinline__ T ldv(const T *__restrict__ val, int64_t q)
{
    const T v = val[q];
    return CJ ? conjv(v) : v;
}

// the partial sum of row r's entries e0 + k * step (k = 0, 1, ...) for right-hand side c, lane-strided
template <typename T, bool CJ>
__device__ __forceinline__ T row_part(int64_t e0, int64_t e1, int64_t step, const int64_t *__restrict__ idx,
                                      const int64_t *__restrict__ src, const T *__restrict__ val, const T *x)
{
    T s = VT<T>::zero();
    for (int64_t e = e0; e < e1; e += step) s = add(s, mul(ldv<T, CJ>(val, src[e]), x[idx[e]]));
    return s;
}

template <typename T, bool CJ>
__device__ __forceinline__ void row_finish(int64_t r, T s, const int64_t *__restrict__ diag, const T *__restrict__ val, T *x)
{
    T y = sub(x[r], s);
    const int64_t q = diag[r];
    if (q >= 0) y = divv(y, ldv<T, CJ>(val, q));
    x[r] = y;
}

// One wide level: rows order[t0 .. t1), a warp per row.
template <typename T, bool CJ>
__global__ void __launch_bounds__(256) k_tri_rows(const int64_t *__restrict__ order, int64_t t0, int64_t t1,
                                                  const int64_t *__restrict__ ptr, const int64_t *__restrict__ idx,
                                                  const int64_t *__restrict__ src, const int64_t *__restrict__ diag,
                                                  const T *__restrict__ val, T *x, int64_t n, int64_t nrhs)
{
    const int lane = threadIdx.x & 31;
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t t = t0 + w; t < t1; t += nw) {
        const int64_t r = order[t];
        for (int64_t c = 0; c < nrhs; c++) {
            T *xc = x + c * n;
            const T s = wsum(row_part<T, CJ>(ptr[r] + lane, ptr[r + 1], 32, idx, src, val, xc));
            if (lane == 0) row_finish<T, CJ>(r, s, diag, val, xc);
        }
    }
}

// A run of thin levels [l0, l1) in one CTA of 1024 threads.  A level of nr rows gives each row wpr warps (a power of
// two, nr * wpr <= 32), whose partial sums are added in warp order; a block barrier separates the levels.
template <typename T, bool CJ>
__global__ void __launch_bounds__(1024) k_tri_levels(const int64_t *__restrict__ order, const int64_t *__restrict__ lev_ptr,
                                                     int64_t l0, int64_t l1, const int64_t *__restrict__ ptr,
                                                     const int64_t *__restrict__ idx, const int64_t *__restrict__ src,
                                                     const int64_t *__restrict__ diag, const T *__restrict__ val, T *x,
                                                     int64_t n, int64_t nrhs)
{
    __shared__ T part[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int64_t l = l0; l < l1; l++) {
        const int64_t t0 = lev_ptr[l], nr = lev_ptr[l + 1] - t0;
        int wpr = 1;
        while ((int64_t)wpr * 2 * nr <= nw && wpr < 32) wpr *= 2;
        for (int64_t c = 0; c < nrhs; c++) {
            T *xc = x + c * n;
            if (wpr == 1) {
                for (int64_t t = warp; t < nr; t += nw) {
                    const int64_t r = order[t0 + t];
                    const T s = wsum(row_part<T, CJ>(ptr[r] + lane, ptr[r + 1], 32, idx, src, val, xc));
                    if (lane == 0) row_finish<T, CJ>(r, s, diag, val, xc);
                }
            } else {
                const int64_t t = warp / wpr;
                const int sub = warp % wpr;
                T s = VT<T>::zero();
                int64_t r = -1;
                if (t < nr) {
                    r = order[t0 + t];
                    s = row_part<T, CJ>(ptr[r] + (int64_t)sub * 32 + lane, ptr[r + 1], (int64_t)wpr * 32, idx, src, val, xc);
                }
                s = wsum(s);
                if (lane == 0) part[warp] = s;
                __syncthreads();
                if (t < nr && sub == 0 && lane == 0) {
                    T tot = part[warp];
                    for (int k = 1; k < wpr; k++) tot = add(tot, part[warp + k]);
                    row_finish<T, CJ>(r, tot, diag, val, xc);
                }
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------------------------------------------------
// host: the sweeps from the patterns

// levels of the rows (forward: every entry reads an earlier row; backward: a later one), their order and the launch runs
static void make_levels(TriSweep &S, int64_t n, bool forward)
{
    std::vector<int64_t> lev((size_t)(n > 0 ? n : 1), 0);
    int64_t maxl = -1;
    for (int64_t k = 0; k < n; k++) {
        const int64_t r = forward ? k : n - 1 - k;
        int64_t l = 0;
        for (int64_t e = S.ptr[r]; e < S.ptr[r + 1]; e++) l = std::max(l, lev[S.idx[e]] + 1);
        lev[r] = l;
        maxl = std::max(maxl, l);
    }
    const int64_t nl = maxl + 1;
    S.lev_ptr.assign((size_t)nl + 1, 0);
    for (int64_t r = 0; r < n; r++) S.lev_ptr[lev[r] + 1]++;
    for (int64_t l = 0; l < nl; l++) S.lev_ptr[l + 1] += S.lev_ptr[l];
    S.order.assign((size_t)(n > 0 ? n : 1), 0);
    std::vector<int64_t> fill(S.lev_ptr.begin(), S.lev_ptr.end() - 1);
    for (int64_t r = 0; r < n; r++) S.order[fill[lev[r]]++] = r;
    S.runs.clear();
    for (int64_t l = 0; l < nl; l++) {
        const bool thin = S.lev_ptr[l + 1] - S.lev_ptr[l] <= TRI_THIN;
        if (thin && !S.runs.empty() && S.runs.back().cta && S.runs.back().l1 == l) S.runs.back().l1 = l + 1;
        else S.runs.push_back({l, l + 1, thin});
    }
}

// rows = the CSC columns themselves: column r's entries with row index on the wanted side (below: i > r)
static void from_columns(TriSweep &S, int64_t n, const int64_t *p, const int64_t *ix, bool below, const int64_t *dpos)
{
    S.ptr.assign((size_t)n + 1, 0);
    S.idx.clear(); S.src.clear();
    for (int64_t r = 0; r < n; r++) {
        for (int64_t q = p[r]; q < p[r + 1]; q++) {
            const int64_t i = ix[q];
            if (below ? i > r : i < r) { S.idx.push_back(i); S.src.push_back(q); }
        }
        S.ptr[r + 1] = (int64_t)S.idx.size();
    }
    S.diag.assign((size_t)(n > 0 ? n : 1), -1);
    if (dpos) for (int64_t r = 0; r < n; r++) S.diag[r] = dpos[r];
}

// rows = the rows of the CSC matrix (a transpose): row i's entries (column j, position q) on the wanted side
static void from_rows(TriSweep &S, int64_t n, const int64_t *p, const int64_t *ix, bool below, const int64_t *dpos)
{
    S.ptr.assign((size_t)n + 1, 0);
    for (int64_t j = 0; j < n; j++)
        for (int64_t q = p[j]; q < p[j + 1]; q++) { const int64_t i = ix[q]; if (below ? i > j : i < j) S.ptr[i + 1]++; }
    for (int64_t i = 0; i < n; i++) S.ptr[i + 1] += S.ptr[i];
    S.idx.assign((size_t)S.ptr[n], 0);
    S.src.assign((size_t)S.ptr[n], 0);
    std::vector<int64_t> fill(S.ptr.begin(), S.ptr.end() - 1);
    for (int64_t j = 0; j < n; j++)
        for (int64_t q = p[j]; q < p[j + 1]; q++) {
            const int64_t i = ix[q];
            if (below ? i > j : i < j) { const int64_t o = fill[i]++; S.idx[o] = j; S.src[o] = q; }
        }
    S.diag.assign((size_t)(n > 0 ? n : 1), -1);
    if (dpos) for (int64_t r = 0; r < n; r++) S.diag[r] = dpos[r];
}

void tri_plan_build(TriPlan &P, int64_t n, const int64_t *Lp, const int64_t *Li, const int64_t *Up, const int64_t *Ui)
{
    P.n = n; P.nnzL = Lp[n]; P.nnzU = Up[n];
    P.udiag.assign((size_t)(n > 0 ? n : 1), -1);
    for (int64_t j = 0; j < n; j++)
        for (int64_t q = Up[j]; q < Up[j + 1]; q++) if (Ui[q] == j) { P.udiag[j] = q; break; }
    from_rows(P.lf, n, Lp, Li, true, nullptr);                 // L x = b: row i of L, entries j < i
    make_levels(P.lf, n, true);
    from_rows(P.ub, n, Up, Ui, false, P.udiag.data());        // U x = b: row i of U, entries j > i
    make_levels(P.ub, n, false);
    from_columns(P.utf, n, Up, Ui, false, P.udiag.data());    // U^T x = b: column r of U, entries i < r
    make_levels(P.utf, n, true);
    from_columns(P.ltb, n, Lp, Li, true, nullptr);            // L^T x = b: column r of L, entries i > r
    make_levels(P.ltb, n, false);
}

// ---------------------------------------------------------------------------------------------------------------------
// host: device copies and the solve

#define CKT(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) { errf(err, errlen, "CUDA: %s", cudaGetErrorString(e_)); return FPLUS_ERR_GPU; } } while (0)

// (a buffer left from an earlier, failed upload is freed first, so a retry does not leak it)
template <typename I>
static int upload(I **d, const std::vector<I> &h, char *err, size_t errlen)
{
    const size_t b = std::max<size_t>(h.size(), 1) * sizeof(I);
    if (*d) { cudaFree(*d); *d = nullptr; }
    CKT(cudaMalloc((void **)d, b));
    if (!h.empty()) CKT(cudaMemcpy(*d, h.data(), h.size() * sizeof(I), cudaMemcpyHostToDevice));
    return FPLUS_OK;
}

static int upload_sweep(TriSweep &S, char *err, size_t errlen)
{
    int rc;
    if ((rc = upload(&S.d_ptr, S.ptr, err, errlen)) || (rc = upload(&S.d_idx, S.idx, err, errlen)) ||
        (rc = upload(&S.d_src, S.src, err, errlen)) || (rc = upload(&S.d_diag, S.diag, err, errlen)) ||
        (rc = upload(&S.d_order, S.order, err, errlen)) || (rc = upload(&S.d_lev, S.lev_ptr, err, errlen)))
        return rc;
    return FPLUS_OK;
}

static void free_sweep(TriSweep &S)
{
    cudaFree(S.d_ptr); cudaFree(S.d_idx); cudaFree(S.d_src); cudaFree(S.d_diag); cudaFree(S.d_order); cudaFree(S.d_lev);
    S.d_ptr = S.d_idx = S.d_src = S.d_diag = S.d_order = S.d_lev = nullptr;
}

TriPlan::~TriPlan()
{
    if (device < 0) return;
    int cur = -1;
    cudaGetDevice(&cur);
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    free_sweep(lf); free_sweep(ub); free_sweep(utf); free_sweep(ltb);
    cudaFree(d_Lx); cudaFree(d_Ux); cudaFree(d_x);
    if (stream) cudaStreamDestroy(stream);
    if (cur >= 0) cudaSetDevice(cur);
}

static int grow(void **p, size_t *cap, size_t bytes, char *err, size_t errlen)
{
    if (*cap >= bytes && *p) return FPLUS_OK;
    cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    CKT(cudaMalloc(p, bytes > 0 ? bytes : 1));
    *cap = bytes;
    return FPLUS_OK;
}

template <typename T, bool CJ>
static long long run_sweep(const TriSweep &S, const T *val, T *x, int64_t n, int64_t nrhs, cudaStream_t st)
{
    long long launches = 0;
    for (const TriSweep::Run &R : S.runs) {
        if (R.cta) {
            k_tri_levels<T, CJ><<<1, 1024, 0, st>>>(S.d_order, S.d_lev, R.l0, R.l1, S.d_ptr, S.d_idx, S.d_src, S.d_diag, val, x,
                                                    n, nrhs);
        } else {
            const int64_t t0 = S.lev_ptr[R.l0], t1 = S.lev_ptr[R.l1];
            const int64_t blocks = std::min<int64_t>((t1 - t0 + 7) / 8, 148 * 16);
            k_tri_rows<T, CJ><<<(unsigned)blocks, 256, 0, st>>>(S.d_order, t0, t1, S.d_ptr, S.d_idx, S.d_src, S.d_diag, val, x,
                                                                n, nrhs);
        }
        launches++;
    }
    return launches;
}

template <typename T>
static long long run_solve_t(TriPlan &P, int64_t nrhs, int trans, cudaStream_t st)
{
    const T *Lx = (const T *)P.d_Lx, *Ux = (const T *)P.d_Ux;
    T *x = (T *)P.d_x;
    long long k = 0;
    if (trans == 0) {
        k += run_sweep<T, false>(P.lf, Lx, x, P.n, nrhs, st);
        k += run_sweep<T, false>(P.ub, Ux, x, P.n, nrhs, st);
    } else if (trans == 1) {
        k += run_sweep<T, false>(P.utf, Ux, x, P.n, nrhs, st);
        k += run_sweep<T, false>(P.ltb, Lx, x, P.n, nrhs, st);
    } else {
        k += run_sweep<T, true>(P.utf, Ux, x, P.n, nrhs, st);
        k += run_sweep<T, true>(P.ltb, Lx, x, P.n, nrhs, st);
    }
    return k;
}

int tri_plan_solve(TriPlan &P, const void *Lx, const void *Ux, void *x, int64_t nrhs, int64_t ldx, int trans,
                   int is_complex, cudaStream_t user_stream, char *err, size_t errlen)
{
    std::lock_guard<std::mutex> lk(P.mu);
    const int64_t n = P.n;
    if (n == 0 || nrhs == 0) return FPLUS_OK;
    int dev = 0;
    CKT(cudaGetDevice(&dev));
    struct Restore {            // the caller's current device again on every return
        int d;
        ~Restore() { cudaSetDevice(d); }
    } restore{dev};
    if (P.device >= 0 && P.device != dev) CKT(cudaSetDevice(P.device));
    if (!P.uploaded) {
        if (P.device < 0) P.device = dev;
        if (!P.stream) CKT(cudaStreamCreateWithFlags(&P.stream, cudaStreamNonBlocking));
        int rc;
        if ((rc = upload_sweep(P.lf, err, errlen)) || (rc = upload_sweep(P.ub, err, errlen)) ||
            (rc = upload_sweep(P.utf, err, errlen)) || (rc = upload_sweep(P.ltb, err, errlen)))
            return rc;
        P.uploaded = true;
    }
    const size_t vs = is_complex ? 16 : 8;
    int rc;
    if ((rc = grow(&P.d_Lx, &P.cap_Lx, (size_t)P.nnzL * vs, err, errlen)) ||
        (rc = grow(&P.d_Ux, &P.cap_Ux, (size_t)P.nnzU * vs, err, errlen)) ||
        (rc = grow(&P.d_x, &P.cap_x, (size_t)n * (size_t)nrhs * vs, err, errlen)))
        return rc;
    cudaStream_t st = user_stream ? user_stream : P.stream;
    if (P.nnzL) CKT(cudaMemcpyAsync(P.d_Lx, Lx, (size_t)P.nnzL * vs, cudaMemcpyHostToDevice, st));
    if (P.nnzU) CKT(cudaMemcpyAsync(P.d_Ux, Ux, (size_t)P.nnzU * vs, cudaMemcpyHostToDevice, st));
    CKT(cudaMemcpy2DAsync(P.d_x, (size_t)n * vs, x, (size_t)ldx * vs, (size_t)n * vs, (size_t)nrhs, cudaMemcpyHostToDevice, st));
    const long long k = is_complex ? run_solve_t<cplx>(P, nrhs, trans, st) : run_solve_t<double>(P, nrhs, trans, st);
    add_launches(k);
    CKT(cudaGetLastError());
    CKT(cudaMemcpy2DAsync(x, (size_t)ldx * vs, P.d_x, (size_t)n * vs, (size_t)n * vs, (size_t)nrhs, cudaMemcpyDeviceToHost, st));
    CKT(cudaStreamSynchronize(st));
    return FPLUS_OK;
}

}  // namespace fpl
