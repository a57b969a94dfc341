// numeric.cu -- the device side of fplus_factor / fplus_solve: device copies of the multifrontal plan, the numeric
// state of one factorization, and the launch sequences.
#include "numeric.hpp"
#include "kernels.cuh"
#include "schur_tc.hpp"
#include <algorithm>
#include <cstring>
#include <cmath>
#include <mutex>
#include <atomic>
#include <complex>

namespace fpl {

static std::atomic<long long> g_launches{0};
static inline void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(); }
void add_launches(long long k) { g_launches.fetch_add(k, std::memory_order_relaxed); }

// optional per-class device timing of the factorization's kernels (CUDA events around each launch of a class)
static std::atomic<int> g_prof{0};
static std::mutex g_prof_mu;
static ProfClass g_pc[PROF_NCLASS];
void prof_enable(int on) { g_prof = on; std::lock_guard<std::mutex> lk(g_prof_mu); for (auto &c : g_pc) c = ProfClass(); }
ProfClass prof_read(int cls) { std::lock_guard<std::mutex> lk(g_prof_mu); return (cls >= 0 && cls < PROF_NCLASS) ? g_pc[cls] : ProfClass(); }

struct ProfRec { int cls; cudaEvent_t a, b; double flops, bytes; };
struct Prof {
    std::vector<ProfRec> recs;
    bool on = g_prof.load() != 0;
    void begin(cudaStream_t s, int cls, double flops, double bytes) {
        if (!on) return;
        ProfRec r{cls, nullptr, nullptr, flops, bytes};
        cudaEventCreate(&r.a); cudaEventCreate(&r.b);
        cudaEventRecord(r.a, s);
        recs.push_back(r);
    }
    void end(cudaStream_t s) { if (on && !recs.empty()) cudaEventRecord(recs.back().b, s); }
    void flush() {
        if (!on) return;
        std::lock_guard<std::mutex> lk(g_prof_mu);
        for (auto &r : recs) {
            float ms = 0;
            if (cudaEventSynchronize(r.b) == cudaSuccess && cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
                ProfClass &c = g_pc[r.cls];
                c.ms += ms; c.count++; c.flops += r.flops; c.bytes += r.bytes;
            }
            cudaEventDestroy(r.a); cudaEventDestroy(r.b);
        }
        recs.clear();
    }
};

// a launch that may begin before the kernel ahead of it in the stream has finished (programmatic dependent launch); the
// kernel waits (pdl_wait) before it reads that kernel's results
template <typename... KArgs, typename... Args>
static cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid; cfg.blockDim = block; cfg.dynamicSmemBytes = smem; cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at; cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

#define CK(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) { errf(err, errlen, "CUDA: %s (%s:%d)", cudaGetErrorString(e_), __FILE__, __LINE__); return FPLUS_ERR_GPU; } } while (0)

static inline int nblk(int64_t work, int per = 256, int cap = 148 * 16)
{
    int64_t b = (work + per - 1) / per;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (int)b;
}

template <typename T> static int upload(const std::vector<T> &h, T **d, char *err, size_t errlen)
{
    *d = nullptr;
    size_t bytes = (h.empty() ? 1 : h.size()) * sizeof(T);
    CK(cudaMalloc((void **)d, bytes));
    if (!h.empty()) CK(cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return FPLUS_OK;
}

DevPlan::~DevPlan()
{
    for (void *p : {(void *)cols, (void *)relcol, (void *)rowinit, (void *)asm_src, (void *)asm_dst, (void *)Bp, (void *)Bi,
                    (void *)Bsrc, (void *)row_perm, (void *)col_perm, (void *)seg, (void *)chain_uoff, (void *)sv, (void *)sv_rows, (void *)sv_cols, (void *)rsp, (void *)rsi, (void *)csp,
                    (void *)csi, (void *)iota, (void *)sv_brows, (void *)sv_bcols, (void *)fc, (void *)children, (void *)bs_list})
        if (p) cudaFree(p);
}

// B's columns cut into segments of at most COL_SEG entries (column, first entry, end), for the column passes
static int upload_segments(int64_t n, const std::vector<int64_t> &Bp, DevPlan &D, char *err, size_t errlen)
{
    std::vector<int64_t> seg;
    for (int64_t j = 0; j < n; j++)
        for (int64_t p0 = Bp[j]; p0 < Bp[j + 1]; p0 += COL_SEG) {
            seg.push_back(j); seg.push_back(p0); seg.push_back(std::min<int64_t>(p0 + COL_SEG, Bp[j + 1]));
        }
    D.nseg = (int64_t)seg.size() / 3;
    return upload(seg, &D.seg, err, errlen);
}

// The level-scheduled solve's structures.  A front is small for the row sweeps (L, L^T) when one CTA holds its vector
// for SV_RC right-hand sides and its pivot block is at most 64 wide and 512 KB (complex), and small for the column sweeps
// (U, U^T) likewise with its columns and U12; the dense chain's fronts, which the U sweep takes by its own kernels, go
// with the larger fronts in the column sweeps.
static const int64_t SV_MAXDIM = 768, SV_MAXNP = 64, SV_MAXBLK = 32768;
static int upload_solve_levels(const FrontPlan &P, DevPlan &D, char *err, size_t errlen)
{
    const int64_t nf = (int64_t)P.fronts.size(), nlev = P.nlevels > 0 ? P.nlevels : 1;
    std::vector<SvFront> sv((size_t)(nf > 0 ? nf : 1));
    std::vector<std::vector<int64_t>> lr((size_t)nlev), lc((size_t)nlev);
    D.big_rows.assign((size_t)nlev, {});
    D.big_cols.assign((size_t)nlev, {});
    D.sv_rows_maxnr.assign((size_t)nlev, 0); D.sv_rows_maxnp.assign((size_t)nlev, 0);
    D.sv_cols_maxnc.assign((size_t)nlev, 0); D.sv_cols_maxnp.assign((size_t)nlev, 0);
    for (int64_t fi = 0; fi < nf; fi++) {
        const Front &F = P.fronts[fi];
        sv[(size_t)fi] = SvFront{F.f, F.npiv, F.nrows, F.nri, F.ncols, F.L_off, F.U_off, F.row_off, F.col_off, 0, 0};
        const size_t L = (size_t)F.level;
        const int64_t ncb = F.ncols - F.npiv;
        const bool base = F.npiv <= SV_MAXNP && F.npiv <= F.nrows;
        const bool rsmall = base && F.nrows <= SV_MAXDIM && F.nrows * F.npiv <= SV_MAXBLK;
        const bool csmall = base && F.ncols <= SV_MAXDIM && F.npiv * ncb <= SV_MAXBLK && !(D.chain_begin >= 0 && fi >= D.chain_begin);
        if (rsmall) {
            lr[L].push_back(fi);
            D.sv_rows_maxnr[L] = std::max(D.sv_rows_maxnr[L], F.nrows);
            D.sv_rows_maxnp[L] = std::max(D.sv_rows_maxnp[L], F.npiv);
        } else D.big_rows[L].push_back(fi);
        if (csmall) {
            lc[L].push_back(fi);
            D.sv_cols_maxnc[L] = std::max(D.sv_cols_maxnc[L], F.ncols);
            D.sv_cols_maxnp[L] = std::max(D.sv_cols_maxnp[L], F.npiv);
        } else D.big_cols[L].push_back(fi);
    }
    // the larger fronts of the trans-0 sweeps: device lists by level; the U sweep's CB-column chunks (at most 296, at least
    // 32 columns each) and each front's first partial sum within its level
    std::vector<int> brows_list, bcols_list;
    D.sv_brows_ptr.assign(1, 0); D.sv_bcols_ptr.assign(1, 0);
    D.brows_maxnr.assign((size_t)nlev, 0); D.brows_maxnp.assign((size_t)nlev, 0); D.brows_maxm.assign((size_t)nlev, 0);
    D.bcols_maxnp.assign((size_t)nlev, 0); D.bcols_maxnch.assign((size_t)nlev, 0); D.bcols_maxchunk.assign((size_t)nlev, 0);
    D.part_need = 1;
    for (int64_t L = 0; L < nlev; L++) {
        for (int64_t fi : D.big_rows[(size_t)L]) {
            const Front &F = P.fronts[(size_t)fi];
            if (F.nrows == 0) continue;
            const int64_t np = std::min(F.npiv, F.nrows);
            brows_list.push_back((int)fi);
            D.brows_maxnr[(size_t)L] = std::max(D.brows_maxnr[(size_t)L], F.nrows);
            D.brows_maxnp[(size_t)L] = std::max(D.brows_maxnp[(size_t)L], np);
            D.brows_maxm[(size_t)L] = std::max(D.brows_maxm[(size_t)L], F.nrows - np);
        }
        int64_t poff = 0;
        for (int64_t fi : D.big_cols[(size_t)L]) {
            const Front &F = P.fronts[(size_t)fi];
            if (F.npiv == 0 || (D.chain_begin >= 0 && fi >= D.chain_begin)) continue;
            const int64_t ncb = F.ncols - F.npiv;
            const int64_t chunk = ncb > 0 ? std::max<int64_t>(32, (ncb + 295) / 296) : 1;
            const int64_t nch = ncb > 0 ? (ncb + chunk - 1) / chunk : 0;
            sv[(size_t)fi].nch = nch;
            sv[(size_t)fi].poff = poff;
            poff += nch * F.npiv;
            bcols_list.push_back((int)fi);
            D.bcols_maxnp[(size_t)L] = std::max(D.bcols_maxnp[(size_t)L], F.npiv);
            D.bcols_maxnch[(size_t)L] = std::max(D.bcols_maxnch[(size_t)L], nch);
            if (nch > 0) D.bcols_maxchunk[(size_t)L] = std::max(D.bcols_maxchunk[(size_t)L], (ncb + nch - 1) / nch);
        }
        D.part_need = std::max(D.part_need, poff);
        D.sv_brows_ptr.push_back((int64_t)brows_list.size());
        D.sv_bcols_ptr.push_back((int64_t)bcols_list.size());
    }
    if (brows_list.empty()) brows_list.push_back(0);
    if (bcols_list.empty()) bcols_list.push_back(0);
    D.sv_brows_host.assign(brows_list.begin(), brows_list.end());
    std::vector<int> rows_list, cols_list;
    D.sv_rows_ptr.assign(1, 0); D.sv_cols_ptr.assign(1, 0);
    for (int64_t L = 0; L < nlev; L++) {
        for (int64_t fi : lr[(size_t)L]) rows_list.push_back((int)fi);
        for (int64_t fi : lc[(size_t)L]) cols_list.push_back((int)fi);
        D.sv_rows_ptr.push_back((int64_t)rows_list.size());
        D.sv_cols_ptr.push_back((int64_t)cols_list.size());
    }
    if (rows_list.empty()) rows_list.push_back(0);
    if (cols_list.empty()) cols_list.push_back(0);
    // the children's contribution entries on each plan row and column, in the children's order
    D.vrow = P.rows_total;
    D.vcol = (int64_t)P.cols.size();
    std::vector<int64_t> rsp((size_t)D.vrow + 1, 0), csp((size_t)D.vcol + 1, 0);
    auto each_entry = [&](auto fn) {
        for (int64_t fi = 0; fi < nf; fi++) {
            const Front &F = P.fronts[fi];
            for (int64_t k = F.child_begin; k < F.child_end; k++) {
                const Front &G = P.fronts[(size_t)P.children[(size_t)k]];
                const int64_t cbr = std::max<int64_t>(0, G.nrows - G.npiv), nslot = std::max<int64_t>(0, G.nri - G.npiv);
                for (int64_t t = 0; t < cbr; t++) {
                    const int64_t i = t < nslot ? G.slot + t : F.tau_base + (t - nslot);
                    fn(0, F.row_off + i, G.row_off + G.npiv + t);
                }
                for (int64_t t = 0; t < G.ncols - G.npiv; t++) fn(1, F.col_off + P.relcol[(size_t)(G.relcol_off + t)], G.col_off + G.npiv + t);
            }
        }
    };
    each_entry([&](int kind, int64_t at, int64_t) { (kind ? csp : rsp)[(size_t)at + 1]++; });
    for (size_t i = 1; i < rsp.size(); i++) rsp[i] += rsp[i - 1];
    for (size_t i = 1; i < csp.size(); i++) csp[i] += csp[i - 1];
    std::vector<int64_t> rsi((size_t)std::max<int64_t>(1, rsp.back())), csi((size_t)std::max<int64_t>(1, csp.back()));
    std::vector<int64_t> rfill(rsp.begin(), rsp.end() - 1), cfill(csp.begin(), csp.end() - 1);
    each_entry([&](int kind, int64_t at, int64_t src) {
        if (kind) csi[(size_t)cfill[(size_t)at]++] = src;
        else rsi[(size_t)rfill[(size_t)at]++] = src;
    });
    std::vector<int64_t> iota((size_t)std::max<int64_t>(1, P.max_nrows));
    for (size_t i = 0; i < iota.size(); i++) iota[i] = (int64_t)i;
    int rc;
    if ((rc = upload(sv, &D.sv, err, errlen))) return rc;
    if ((rc = upload(rows_list, &D.sv_rows, err, errlen))) return rc;
    if ((rc = upload(brows_list, &D.sv_brows, err, errlen))) return rc;
    if ((rc = upload(bcols_list, &D.sv_bcols, err, errlen))) return rc;
    if ((rc = upload(cols_list, &D.sv_cols, err, errlen))) return rc;
    if ((rc = upload(rsp, &D.rsp, err, errlen))) return rc;
    if ((rc = upload(rsi, &D.rsi, err, errlen))) return rc;
    if ((rc = upload(csp, &D.csp, err, errlen))) return rc;
    if ((rc = upload(csi, &D.csi, err, errlen))) return rc;
    if ((rc = upload(iota, &D.iota, err, errlen))) return rc;
    return FPLUS_OK;
}

// The factorization's batched fronts (DevPlan): an interior front with 1..64 pivots, at most 128 rows and no more pivots
// than rows, whose children are all batched.
static const int64_t BS_MAXNR = 128, BS_MAXNP = 64;
static int upload_batched_fronts(const FrontPlan &P, DevPlan &D, char *err, size_t errlen)
{
    const int64_t nf = (int64_t)P.fronts.size(), nlev = P.nlevels > 0 ? P.nlevels : 1;
    D.is_bs.assign((size_t)nf, 0);
    D.bs_cbofs.assign((size_t)nf, 0);
    std::vector<FcFront> fc((size_t)(nf > 0 ? nf : 1));
    std::vector<std::vector<int64_t>> lists((size_t)nlev);
    D.bs_maxnr.assign((size_t)nlev, 0); D.bs_maxnp.assign((size_t)nlev, 0); D.bs_maxtiles.assign((size_t)nlev, 0);
    D.bs_wsz.assign((size_t)nlev, 0);
    D.bs_lu_flops.assign((size_t)nlev, 0); D.bs_tail_flops.assign((size_t)nlev, 0);
    D.bs_asm_bytes.assign((size_t)nlev, 0); D.bs_lu_bytes.assign((size_t)nlev, 0); D.bs_tail_bytes.assign((size_t)nlev, 0);
    int64_t cbo = 0;
    for (int64_t fi = 0; fi < nf; fi++) {
        const Front &F = P.fronts[(size_t)fi];
        bool ok = !F.dense && F.npiv >= 1 && F.npiv <= BS_MAXNP && F.nrows <= BS_MAXNR && F.npiv <= F.nrows;
        for (int64_t k = F.child_begin; ok && k < F.child_end; k++) ok = D.is_bs[(size_t)P.children[(size_t)k]] != 0;
        const int64_t ncb = F.ncols - F.npiv, M = F.nrows - F.npiv;
        FcFront &c = fc[(size_t)fi];
        c = FcFront{F.f, F.npiv, F.nrows, F.nri, F.ncols, F.L_off, F.U_off, F.row_off, F.relcol_off, F.asm_begin, F.asm_end,
                    F.child_begin, F.child_end, F.slot, F.tau_base, 0, 0};
        if (!ok) continue;
        D.is_bs[(size_t)fi] = 1;
        const size_t L = (size_t)F.level;
        lists[L].push_back(fi);
        c.wofs = D.bs_wsz[L];
        D.bs_wsz[L] += F.nrows * F.ncols;
        c.cbofs = cbo;
        D.bs_cbofs[(size_t)fi] = cbo;
        cbo += M * ncb;
        D.bs_maxnr[L] = std::max(D.bs_maxnr[L], F.nrows);
        D.bs_maxnp[L] = std::max(D.bs_maxnp[L], F.npiv);
        D.bs_maxtiles[L] = std::max<int64_t>(D.bs_maxtiles[L], (ncb + 31) / 32);
        double fl = 0;
        for (int64_t k = 0; k < F.npiv; k++) fl += (double)(F.nrows - k - 1) * (double)(F.npiv - k);
        D.bs_lu_flops[L] += fl;
        D.bs_tail_flops[L] += ((double)F.npiv * (double)F.npiv / 2.0 + (double)M * (double)F.npiv) * (double)ncb;
        D.bs_asm_bytes[L] += (double)(F.nrows * F.ncols + 2 * (F.asm_end - F.asm_begin));
        D.bs_lu_bytes[L] += 2.0 * (double)(F.nrows * F.npiv);
        D.bs_tail_bytes[L] += (double)(2 * F.nrows * ncb + F.nrows * F.npiv);
    }
    D.bs_cb = cbo;
    D.bs_ws = 0;
    std::vector<int> list;
    D.bs_ptr.assign(1, 0);
    for (int64_t L = 0; L < nlev; L++) {
        for (int64_t fi : lists[(size_t)L]) list.push_back((int)fi);
        D.bs_ptr.push_back((int64_t)list.size());
        D.bs_ws = std::max(D.bs_ws, D.bs_wsz[(size_t)L]);
    }
    if (list.empty()) list.push_back(0);
    std::vector<int64_t> ch(P.children.begin(), P.children.end());
    if (ch.empty()) ch.push_back(0);
    int rc;
    if ((rc = upload(fc, &D.fc, err, errlen))) return rc;
    if ((rc = upload(ch, &D.children, err, errlen))) return rc;
    if ((rc = upload(list, &D.bs_list, err, errlen))) return rc;
    return FPLUS_OK;
}

int dev_upload_plan(const fplus_symbolic *S, const FrontPlan &P, DevPlan &D, char *err, size_t errlen)
{
    CK(cudaGetDevice(&D.device));
    int rc;
    if ((rc = upload(P.cols, &D.cols, err, errlen))) return rc;
    if ((rc = upload(P.relcol, &D.relcol, err, errlen))) return rc;
    if ((rc = upload(P.rowinit, &D.rowinit, err, errlen))) return rc;
    if ((rc = upload(P.asm_src, &D.asm_src, err, errlen))) return rc;
    if ((rc = upload(P.asm_dst, &D.asm_dst, err, errlen))) return rc;
    if ((rc = upload(S->Bp, &D.Bp, err, errlen))) return rc;
    if ((rc = upload(S->Bi, &D.Bi, err, errlen))) return rc;
    if ((rc = upload(S->Bsrc, &D.Bsrc, err, errlen))) return rc;
    if ((rc = upload(S->row_perm, &D.row_perm, err, errlen))) return rc;
    if ((rc = upload(S->col_perm, &D.col_perm, err, errlen))) return rc;
    if ((rc = upload_segments(S->n, S->Bp, D, err, errlen))) return rc;
    {
        // the dense chain: trailing dense fronts, nb_chain pivots each (the last at most), columns [f, n), no gaps
        const int64_t nf = (int64_t)P.fronts.size(), nb = P.nb_chain;
        int64_t c0 = nf;
        while (c0 > 0 && P.fronts[c0 - 1].dense) c0--;
        bool ok = nf - c0 >= 2 && nb > 0 && nb <= 64;
        std::vector<int64_t> uoff;
        for (int64_t j = c0; ok && j < nf; j++) {
            const Front &F = P.fronts[j];
            const bool lastf = j == nf - 1;
            ok = F.f == P.fronts[c0].f + (j - c0) * nb && (lastf ? F.npiv <= nb : F.npiv == nb) && F.npiv <= F.nrows &&
                 F.ncols == S->n - F.f;
            uoff.push_back(F.U_off);
        }
        if (ok) {
            D.chain_begin = c0; D.chain_nb = nb; D.chain_f0 = P.fronts[c0].f;
            if ((rc = upload(uoff, &D.chain_uoff, err, errlen))) return rc;
        }
    }
    if ((rc = upload_solve_levels(P, D, err, errlen))) return rc;
    if ((rc = upload_batched_fronts(P, D, err, errlen))) return rc;
    return FPLUS_OK;
}

DevNum::~DevNum()
{
    if (device >= 0) cudaSetDevice(device);
    for (void *p : {(void *)Ax, (void *)Bx, (void *)Drp, (void *)Dcp, (void *)colmax, (void *)Larena, (void *)Uarena,
                    (void *)cbstack, (void *)work, (void *)rowid, (void *)p_lu, (void *)pinv, (void *)ipiv, (void *)perm,
                    (void *)st, (void *)scratch, (void *)rbuf, (void *)sbuf, (void *)xbuf, (void *)part, (void *)work2,
                    (void *)perm2, (void *)rr_p, (void *)rr_l, (void *)rr_s, (void *)ir_b, (void *)ir_x, (void *)ir_r,
                    (void *)ir_d, (void *)ir_bits, scratch_norm, tcws, gm_buf, coopbuf, (void *)permall, vbuf, bsw, bscb})
        if (p) cudaFreeAsync(p, stream);
    if (stream) cudaStreamSynchronize(stream);
    if (crit) cudaStreamSynchronize(crit);
    if (ev_begin) cudaEventDestroy(ev_begin);
    if (ev_done) cudaEventDestroy(ev_done);
    if (ev_lu) cudaEventDestroy(ev_lu);
    if (ev_head) cudaEventDestroy(ev_head);
    if (crit) cudaStreamDestroy(crit);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream && stream_owned) cudaStreamDestroy(stream);
}

// stream-ordered allocation from the device's default pool, which keeps freed memory for reuse (release threshold: no
// limit), so a refactorization of the same size allocates nothing new
static int pool_init(int dev, char *err, size_t errlen)
{
    static std::mutex mu;
    static int done[64] = {0};
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 0 || dev >= 64 || done[dev]) return FPLUS_OK;
    cudaMemPool_t pool;
    CK(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t thr = UINT64_MAX;
    CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    done[dev] = 1;
    return FPLUS_OK;
}

int ensure_async(DevNum &N, void **p, size_t *cap, size_t bytes, char *err, size_t errlen)
{
    if (N.capture) {                      // a captured sequence must not allocate: the buffers are sized beforehand
        if ((*p && *cap >= bytes) || bytes == 0) return FPLUS_OK;
        errf(err, errlen, "a captured factorization or solve needs a larger buffer (%zu > %zu bytes)", bytes, *cap);
        return FPLUS_ERR_INTERNAL;
    }
    if (*cap >= bytes && *p) return FPLUS_OK;
    if (*p) { CK(cudaFreeAsync(*p, N.stream)); *p = nullptr; *cap = 0; }
    CK(cudaMallocAsync(p, bytes > 0 ? bytes : 16, N.stream));
    *cap = bytes;
    return FPLUS_OK;
}

static int ensure(void **p, size_t *cap, size_t bytes, char *err, size_t errlen)
{
    if (*cap >= bytes && *p) return FPLUS_OK;
    if (*p) { cudaFree(*p); *p = nullptr; *cap = 0; }
    CK(cudaMalloc(p, bytes > 0 ? bytes : 16));
    *cap = bytes;
    return FPLUS_OK;
}

int dev_num_init(DevNum &N, int64_t n, int64_t nnz, int cplx, char *err, size_t errlen)
{
    N.n = n; N.nnz = nnz; N.cplx = cplx;
    N.vs = cplx ? 16 : 8;
    CK(cudaGetDevice(&N.device));
    int rc = pool_init(N.device, err, errlen);
    if (rc) return rc;
    if (!N.stream) { CK(cudaStreamCreateWithFlags(&N.stream, cudaStreamNonBlocking)); N.stream_owned = true; }
    CK(cudaEventCreate(&N.ev0));
    CK(cudaEventCreate(&N.ev1));
    CK(cudaEventCreate(&N.ev_begin));
    CK(cudaEventCreate(&N.ev_done));
    const size_t nn = (size_t)(n > 0 ? n : 1), nz = (size_t)(nnz > 0 ? nnz : 1);
    cudaStream_t s = N.stream;
    CK(cudaMallocAsync((void **)&N.Ax, nz * N.vs, s));
    CK(cudaMallocAsync((void **)&N.Bx, nz * N.vs, s));
    CK(cudaMallocAsync((void **)&N.Drp, nn * 8, s));
    CK(cudaMallocAsync((void **)&N.Dcp, nn * 8, s));
    CK(cudaMallocAsync((void **)&N.colmax, nn * 8, s));
    CK(cudaMallocAsync((void **)&N.p_lu, nn * 8, s));
    CK(cudaMallocAsync((void **)&N.pinv, nn * 8, s));
    CK(cudaMallocAsync((void **)&N.st, sizeof(DevStatus), s));
    CK(cudaMallocAsync((void **)&N.scratch, 2 * nn * 8, s));
    return FPLUS_OK;
}

// ---------------------------------------------------------------------------------------------------------------------
// permutation + Ruiz: Bx = the scaled permuted values, Drp / Dcp, colmax; returns FPLUS_OK or an error
template <typename T>
static int run_equil(const DevPlan &D, DevNum &N, int equilibrate, int max_iter, double tol, char *err, size_t errlen)
{
    cudaStream_t s = N.stream;
    const int64_t n = N.n, nnz = N.nnz;
    T *Bx = (T *)N.Bx;
    k_gather<T><<<nblk(nnz), 256, 0, s>>>(Bx, (const T *)N.Ax, D.Bsrc, nnz), note_launch();
    if (N.capture) {
        // the same steps without host copies or decisions: the set-up on the device, every Ruiz iteration launched (the
        // kernels do nothing once the iteration has converged), values the range guard would rescale reported
        k_clear_status<<<1, 1, 0, s>>>(N.st, 1), note_launch();
        k_fill<<<nblk(n), 256, 0, s>>>(N.Drp, n, 1.0), note_launch();
        k_fill<<<nblk(n), 256, 0, s>>>(N.Dcp, n, 1.0), note_launch();
        if (equilibrate) {
            const int64_t m = (N.cplx ? 2 : 1) * nnz;
            k_abs_range<<<nblk(m), 256, 0, s>>>((const double *)Bx, m, N.st), note_launch();
            k_range_flag<<<1, 1, 0, s>>>(N.st), note_launch();
            unsigned long long *rmax = (unsigned long long *)N.scratch, *cmax = rmax + n;
            for (int it = 0; it < max_iter; it++) {
                CK(cudaMemsetAsync(rmax, 0, (size_t)n * 8, s));
                k_ruiz_rowmax<T><<<nblk(nnz), 256, 0, s>>>(D.Bi, Bx, nnz, rmax, N.st), note_launch();
                k_ruiz_rowscale<<<nblk(n), 256, 0, s>>>(n, rmax, N.Drp, cmax, N.st), note_launch();
                k_first_zero<<<nblk(n), 256, 0, s>>>(n, rmax, N.st, ST_ZERO_ROW), note_launch();
                k_ruiz_colpass<T><<<nblk(32 * D.nseg), 256, 0, s>>>(D.seg, D.nseg, D.Bi, Bx, rmax, cmax, N.st), note_launch();
                k_ruiz_colscale<<<nblk(n), 256, 0, s>>>(n, cmax, N.Dcp, N.st), note_launch();
                k_first_zero<<<nblk(n), 256, 0, s>>>(n, cmax, N.st, ST_ZERO_COL), note_launch();
                k_ruiz_colapply<T><<<nblk(32 * D.nseg), 256, 0, s>>>(D.seg, D.nseg, Bx, cmax, N.st), note_launch();
                k_ruiz_check<<<1, 1, 0, s>>>(N.st, tol), note_launch();
            }
        }
        CK(cudaMemsetAsync(N.colmax, 0, (size_t)n * 8, s));
        k_colmax<T><<<nblk(32 * D.nseg), 256, 0, s>>>(D.seg, D.nseg, Bx, (unsigned long long *)N.colmax), note_launch();
        CK(cudaGetLastError());
        return FPLUS_OK;
    }
    // the status (the smallest failing index wins; the range's minimum starts at +inf) and the unit scalings, set on the
    // device (no pageable host copies)
    k_clear_status<<<1, 1, 0, s>>>(N.st, 1), note_launch();
    k_fill<<<nblk(n), 256, 0, s>>>(N.Drp, n, 1.0), note_launch();
    k_fill<<<nblk(n), 256, 0, s>>>(N.Dcp, n, 1.0), note_launch();
    if (equilibrate) {
        // range guard (FPLUS src/equil.c:197-241)
        const int64_t m = (N.cplx ? 2 : 1) * nnz;
        k_abs_range<<<nblk(m), 256, 0, s>>>((const double *)Bx, m, N.st), note_launch();
        DevStatus h;
        CK(cudaMemcpyAsync(&h, N.st, sizeof(h), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        double amax = bitsd_h(h.amax_bits), amin = bitsd_h(h.amin_bits);
        int k4 = 0;
        if (amax > 0.0 && (amax > 0x1p500 || amin < 0x1p-500)) {
            int emax = std::ilogb(amax), emin = std::ilogb(amin);
            if (emax - emin > 990) {
                unsigned long long *lmax = (unsigned long long *)N.scratch;
                CK(cudaMemsetAsync(lmax, 0, (size_t)(2 * n) * 8, s));
                if (N.cplx) k_line_max<true><<<nblk(n), 256, 0, s>>>(D.Bp, D.Bi, (const double *)Bx, n, lmax), note_launch();
                else k_line_max<false><<<nblk(n), 256, 0, s>>>(D.Bp, D.Bi, (const double *)Bx, n, lmax), note_launch();
                unsigned long long inf = 0x7ff0000000000000ull;
                CK(cudaMemcpyAsync(&N.st->amin_bits, &inf, 8, cudaMemcpyHostToDevice, s));
                k_min_pos<<<nblk(2 * n), 256, 0, s>>>(lmax, 2 * n, N.st), note_launch();
                CK(cudaMemcpyAsync(&h, N.st, sizeof(h), cudaMemcpyDeviceToHost, s));
                CK(cudaStreamSynchronize(s));
                double lmin = bitsd_h(h.amin_bits);
                int elmin = std::ilogb(lmin);
                if (emax - elmin > 990) {
                    errf(err, errlen, "line maxima span 2^%d .. 2^%d (entries 2^%d ..): wider than Ruiz equilibration can handle "
                         "in double precision; factor without equilibration (equilibrate=False)", elmin, emax, emin);
                    return FPLUS_ERR_BADARG;
                }
                emin = elmin;
            }
            k4 = -((emax + emin) / 2 / 4) * 4;
            k_scale_raw<<<nblk(m), 256, 0, s>>>((double *)Bx, m, std::ldexp(1.0, k4)), note_launch();
        }
        unsigned long long *rmax = (unsigned long long *)N.scratch, *cmax = rmax + n;
        for (int it = 0; it < max_iter; it++) {
            CK(cudaMemsetAsync(rmax, 0, (size_t)n * 8, s));
            k_ruiz_rowmax<T><<<nblk(nnz), 256, 0, s>>>(D.Bi, Bx, nnz, rmax, N.st), note_launch();
            k_ruiz_rowscale<<<nblk(n), 256, 0, s>>>(n, rmax, N.Drp, cmax, N.st), note_launch();
            k_first_zero<<<nblk(n), 256, 0, s>>>(n, rmax, N.st, ST_ZERO_ROW), note_launch();
            k_ruiz_colpass<T><<<nblk(32 * D.nseg), 256, 0, s>>>(D.seg, D.nseg, D.Bi, Bx, rmax, cmax, N.st), note_launch();
            k_ruiz_colscale<<<nblk(n), 256, 0, s>>>(n, cmax, N.Dcp, N.st), note_launch();
            k_first_zero<<<nblk(n), 256, 0, s>>>(n, cmax, N.st, ST_ZERO_COL), note_launch();
            k_ruiz_colapply<T><<<nblk(32 * D.nseg), 256, 0, s>>>(D.seg, D.nseg, Bx, cmax, N.st), note_launch();
            k_ruiz_check<<<1, 1, 0, s>>>(N.st, tol), note_launch();
        }
        if (k4 != 0) k_fold<<<nblk(n), 256, 0, s>>>(N.Drp, N.Dcp, n, std::ldexp(1.0, k4 / 2)), note_launch();
    }
    CK(cudaMemsetAsync(N.colmax, 0, (size_t)n * 8, s));
    k_colmax<T><<<nblk(32 * D.nseg), 256, 0, s>>>(D.seg, D.nseg, Bx, (unsigned long long *)N.colmax), note_launch();
    CK(cudaGetLastError());
    DevStatus h;
    CK(cudaMemcpyAsync(&h, N.st, sizeof(h), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    N.ruiz_iters = h.iters;
    if (h.code == ST_ZERO_ROW) {
        errf(err, errlen, "Row %ld of the matrix is entirely zero (structural singularity detected during equilibration).", (long)h.idx);
        return FPLUS_ERR_SINGULAR;
    }
    if (h.code == ST_ZERO_COL) {
        errf(err, errlen, "Column %ld of the matrix is entirely zero (structural singularity detected during equilibration).", (long)h.idx);
        return FPLUS_ERR_SINGULAR;
    }
    return FPLUS_OK;
}

// ---------------------------------------------------------------------------------------------------------------------
// the fronts, in order.  Returns FPLUS_OK, or ST_BORDER through *border_front (>= 0) for a restart with a dense chain.
static size_t front_lu_smem(int64_t nrows, int64_t npiv, int64_t vs) { return (size_t)(nrows * npiv * vs + nrows * (2 * vs + 16) + npiv * 16); }
// k_front_lu3: the block, two panels of masked multipliers, row ids, tags, positions, thresholds and pivot rows
static size_t front_lu3_smem(int64_t nrows, int64_t npiv, int64_t vs)
{
    return (size_t)(nrows * npiv * vs + 2 * LU3_PB * nrows * vs + nrows * 16 + npiv * 12);
}
static bool use_lu3(int64_t nrows, int64_t npiv, int64_t vs)
{
    return nrows <= 128 && npiv <= 64 && npiv <= nrows && front_lu3_smem(nrows, npiv, vs) <= 220 * 1024;
}
static const size_t SMEM_MAX = 220 * 1024;   // dynamic shared memory opt-in, below the 227 KB per-block limit (static smem on top)
// the precision form takes a Schur update to the tensor cores from this size on (smaller ones stay FP64: they are cheap,
// and a 128 x 256 tile would be mostly padding)
static const int64_t TC_MIN_ROWS = 128, TC_MIN_COLS = 256;
static const double TC_MIN_MADDS = 1 << 24;

template <typename T>
static int run_fronts(const FrontPlan &P, const DevPlan &D, DevNum &N, double pivot_rel, int64_t *border_front,
                      char *err, size_t errlen, bool batch = true)
{
    cudaStream_t s = N.stream;
    const int64_t vs = N.vs;
    int rc;
    *border_front = -1;
    if ((rc = ensure_async(N, (void **)&N.Larena, &N.cap_L, (size_t)P.L_size * vs, err, errlen))) return rc;
    if ((rc = ensure_async(N, (void **)&N.Uarena, &N.cap_U, (size_t)P.U_size * vs, err, errlen))) return rc;
    if ((rc = ensure_async(N, (void **)&N.cbstack, &N.cap_cb, (size_t)P.cb_size * vs, err, errlen))) return rc;
    if ((rc = ensure_async(N, (void **)&N.work, &N.cap_work, (size_t)P.work_size * vs, err, errlen))) return rc;
    if ((rc = ensure_async(N, (void **)&N.rowid, &N.cap_rowid, (size_t)P.rows_total * 8, err, errlen))) return rc;
    if ((rc = ensure_async(N, (void **)&N.ipiv, &N.cap_ipiv, (size_t)(N.n > 0 ? N.n : 1) * 4, err, errlen))) return rc;
    if ((rc = ensure_async(N, (void **)&N.permall, &N.cap_permall, (size_t)(P.rows_total > 0 ? P.rows_total : 1) * 4, err, errlen))) return rc;
    static thread_local int attr_set = 0;
    if (!attr_set) {
        CK(cudaFuncSetAttribute(k_front_lu2<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX));
        CK(cudaFuncSetAttribute(k_front_lu5<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)front_lu5_smem(128, 64, sizeof(T))));
        CK(cudaFuncSetAttribute(k_bat_lu5<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)front_lu5_smem(128, 64, sizeof(T))));
        CK(cudaFuncSetAttribute(k_front_lu3<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX));
        CK(cudaFuncSetAttribute(k_trsm_warp<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX));
        CK(cudaFuncSetAttribute(k_trsm_warp<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX));
        CK(cudaFuncSetAttribute(k_u12_blk<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX));
        CK(cudaFuncSetAttribute(k_front_tail<T, FT_TN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX));
        CK(cudaFuncSetAttribute(k_front_tail<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX));
        CK(cudaFuncSetAttribute(k_bat_lu2<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX));
        CK(cudaFuncSetAttribute(k_bat_tail<T, FT_TN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX));
        CK(cudaFuncSetAttribute(k_front_tail2<T, FT_TN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX));
        CK(cudaFuncSetAttribute(k_bat_tail2<T, FT_TN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX));
        attr_set = 1;
    }
    // (captured: the status was cleared where the captured equilibration began, and must keep what it reported)
    if (!N.capture && (rc = dev_clear_status(N, err, errlen))) return rc;
    N.tc_updates = 0; N.tc_flops = 0;
    T *La = (T *)N.Larena, *Ua = (T *)N.Uarena, *CB = (T *)N.cbstack;
    const T *Bx = (const T *)N.Bx;
    constexpr int PW = 32;       // panel width of the blocked path
    // the multi-CTA pivot-block LU (k_block_lu_mc): one cluster of up to mc_cl CTAs, or a cooperative launch of up to one
    // CTA per SM (mc_sms); its buffer: the grid form's posts (two per CTA), its ticket and counter, the choices, U12 of
    // the pivot rows, and two row scratches
    const int per_max = VT<T>::cplx_ ? 256 : 512;
    static thread_local int mc_sms = -1, mc_cl = 0;
    if (mc_sms < 0) {
        int dev = 0, sms = 0, k = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (cudaFuncSetAttribute(k_block_lu_mc<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&k, k_block_lu_mc<T, false>, MC_THREADS, mc_smem<T>(per_max, false)) != cudaSuccess)
            k = 0;
        (void)cudaGetLastError();
        mc_sms = k >= 1 ? sms : 0;
        // the largest cluster the device places with the cluster form's largest shared memory
        // (the opt-in is the largest request of the cluster form: with the 220 KB cap its static posts would pass the 227 KB
        // limit for complex values)
        if (cudaFuncSetAttribute(k_block_lu_mc<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mc_smem<T>(per_max, true)) == cudaSuccess &&
            cudaFuncSetAttribute(k_block_lu_mc<T, true>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
            for (int csz = MC_CMAX; csz >= 4 && mc_cl == 0; csz /= 2) {
                cudaLaunchConfig_t oc = {};
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeClusterDimension;
                at[0].val.clusterDim.x = (unsigned)csz; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
                oc.gridDim = dim3((unsigned)csz); oc.blockDim = dim3(MC_THREADS); oc.dynamicSmemBytes = mc_smem<T>(per_max, true);
                oc.attrs = at; oc.numAttrs = 1;
                int ncl = 0;
                if (cudaOccupancyMaxActiveClusters(&ncl, (const void *)k_block_lu_mc<T, true>, &oc) == cudaSuccess && ncl >= 1) mc_cl = csz;
            }
        }
        (void)cudaGetLastError();
    }
    auto r256 = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t mc_slots = r256((size_t)2 * (mc_sms > 0 ? mc_sms : 1) * sizeof(McSlot<T>)), mc_tk = 256,
                 mc_ch = r256((size_t)(P.max_npiv > 0 ? P.max_npiv : 1) * 8),
                 mc_ub = r256((size_t)(P.max_npiv > 0 ? P.max_npiv : 1) * (P.max_npiv > 0 ? P.max_npiv : 1) * vs),
                 mc_mark = r256((size_t)(P.max_nrows > 0 ? P.max_nrows : 1) * 4), mc_rid = r256((size_t)(P.max_nrows > 0 ? P.max_nrows : 1) * 8);
    bool any_mc = false;
    for (const Front &F : P.fronts)
        if (front_lu_smem(F.nrows, F.npiv, vs) > SMEM_MAX) { any_mc = true; break; }
    any_mc = any_mc && (mc_sms > 0 || mc_cl > 0);
    if (any_mc) {
        if ((rc = ensure_async(N, &N.coopbuf, &N.cap_coop, mc_slots + mc_tk + mc_ch + mc_ub + mc_mark + mc_rid, err, errlen))) return rc;
        CK(cudaMemsetAsync((char *)N.coopbuf + mc_slots, 0, mc_tk, s));      // the ticket and the counter start at zero
    }
    McSlot<T> *mc_slot = (McSlot<T> *)N.coopbuf;
    unsigned int *mc_sync = (unsigned int *)((char *)N.coopbuf + mc_slots);
    int64_t *mc_chosen = (int64_t *)((char *)N.coopbuf + mc_slots + mc_tk);
    T *mc_U = (T *)((char *)N.coopbuf + mc_slots + mc_tk + mc_ch);
    int *mc_markp = (int *)((char *)N.coopbuf + mc_slots + mc_tk + mc_ch + mc_ub);
    int64_t *mc_ridp = (int64_t *)((char *)N.coopbuf + mc_slots + mc_tk + mc_ch + mc_ub + mc_mark);
    const int TB = VT<T>::cplx_ ? 32 : 64;    // rows per TRSM block of U12
    const int64_t nf = (int64_t)P.fronts.size();
    const double fm = VT<T>::cplx_ ? 8.0 : 2.0;     // flops per multiply-add
    Prof prof;

    // Chain fronts whose CB goes to the next front run with a one-front look-ahead on two streams.  The critical stream
    // (high priority) assembles a front's pivot columns and factors its pivot block; the bulk stream (the caller's)
    // assembles the front's other columns, then, once the pivot block is factored, forms U12 and the CB for the CB
    // columns that are the parent's pivot columns (the head), signals the critical stream, and forms the rest of the
    // front's tail while the critical stream moves on to the parent.  Consecutive such fronts alternate between two
    // working blocks and two row orders.
    const std::vector<int64_t> &hc = P.head_cols;
    std::vector<char> pipe((size_t)nf, 0);
    bool any_pipe = false;
    for (int64_t fi = 0; fi < nf; fi++) {
        const Front &F = P.fronts[fi];
        const int64_t nr = F.nrows, np = F.npiv, ncb = F.ncols - F.npiv;
        bool ok = F.dense && np > 0 && np <= nr && np <= FT_NP && nr <= FT_NR && front_lu_smem(nr, np, vs) <= SMEM_MAX;
        ok = ok && (ncb == 0 || (F.parent == fi + 1 && hc[fi] >= 0));
        for (int64_t k = F.child_begin; ok && k < F.child_end; k++) ok = hc[P.children[k]] >= 0;
        pipe[fi] = ok;
        any_pipe = any_pipe || ok;
    }
    if (any_pipe) {
        const size_t wbytes = (size_t)P.work_size * vs;
        if ((rc = ensure_async(N, (void **)&N.work2, &N.cap_work2, wbytes, err, errlen))) return rc;
        if (!N.crit) {
            int lo = 0, hi = 0;
            CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
            CK(cudaStreamCreateWithPriority(&N.crit, cudaStreamNonBlocking, hi));
            CK(cudaEventCreateWithFlags(&N.ev_lu, cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&N.ev_head, cudaEventDisableTiming));
        }
    }
    cudaStream_t A = N.crit;
    // A pipelined front whose parent is the next pipelined front, takes no other child, and whose contribution block has
    // the parent's every column and every row but its entering rows: the bulk of its tail (the columns after the ones
    // the parent's pivot block takes from the stack) writes straight into the parent's working block, the other of the
    // two, entering rows as zeros; the parent then adds only its original entries to those columns (part 4).
    std::vector<char> pdirect((size_t)nf, 0);
    if (any_pipe && !(N.lu_variant & 48)) {
        for (int64_t fi = 0; fi + 1 < nf; fi++) {
            const Front &F = P.fronts[(size_t)fi], &Q = P.fronts[(size_t)fi + 1];
            if (!pipe[(size_t)fi] || !pipe[(size_t)fi + 1] || F.parent != fi + 1 || Q.child_end - Q.child_begin != 1) continue;
            const int64_t np = F.npiv, M = F.nrows - np, ncb = F.ncols - np, nslot = std::max<int64_t>(0, F.nri - np);
            const int64_t h = std::min<int64_t>(ncb, (hc[(size_t)fi] + FT_TN - 1) / FT_TN * FT_TN);
            if (M <= 0 || h != hc[(size_t)fi] || h >= ncb || ncb != Q.ncols || hc[(size_t)fi] != Q.npiv) continue;
            if (F.slot + nslot != Q.tau_base || M - nslot != Q.nrows - Q.tau_base) continue;
            pdirect[(size_t)fi] = 1;
        }
    }

    // the batched fronts (variant + 8 or the blocked small-front LU turn them off): their contribution blocks live in
    // their own arena
    const bool bs_on = batch && D.bs_ptr.size() > 1 && D.bs_ptr.back() > 0 && !(N.lu_variant & 8) && (N.lu_variant & 3) != 3;
    T *CBA = nullptr;
    if (bs_on) {
        if ((rc = ensure_async(N, &N.bsw, &N.cap_bsw, (size_t)std::max<int64_t>(1, D.bs_ws) * vs, err, errlen))) return rc;
        if ((rc = ensure_async(N, &N.bscb, &N.cap_bscb, (size_t)std::max<int64_t>(1, D.bs_cb) * vs, err, errlen))) return rc;
        CBA = (T *)N.bscb;
    }
    auto cb_of = [&](int64_t gi) -> T * { return bs_on && D.is_bs[(size_t)gi] ? CBA + D.bs_cbofs[(size_t)gi] : CB + P.fronts[(size_t)gi].cb_off; };

    // the assembly of columns [0, npiv) (part 1), the others (part 2), or all (part 0)
    // (part 3: every column, with the single child's contribution block already written into W by its Schur update and
    // the entering rows zeroed: the original entries add to it, the child gives its row ids only; part 4: the same for
    // the columns of part 2, written by the child's tail)
    auto assemble = [&](int64_t fi, T *W, cudaStream_t st, int part) {
        const Front &F = P.fronts[fi];
        const int64_t nr = F.nrows, nc = F.ncols, np = F.npiv, ld = nr;
        const bool pre = part == 3 || part == 4;
        if (part == 4) {
            const int64_t e0 = F.asm_mid, cnt = F.asm_end - F.asm_mid;
            prof.begin(st, PROF_ASM, 0.0, (double)(2 * cnt) * vs);
            if (cnt > 0)
                k_assemble<T><<<nblk(cnt), 256, 0, st>>>(W, Bx, D.asm_src + e0, D.asm_dst + e0, cnt, N.rowid + F.row_off,
                                                         D.rowinit + F.row_off, 0, N.st, 1), note_launch();
            prof.end(st);
            return FPLUS_OK;
        }
        const int64_t e0 = part == 2 ? F.asm_mid : F.asm_begin, e1 = part == 1 ? F.asm_mid : F.asm_end;
        const int64_t z0 = part == 2 ? nr * np : 0, z1 = pre ? 0 : part == 1 ? nr * np : nr * nc;
        prof.begin(st, PROF_ASM, 0.0, (double)((z1 - z0) + 2 * (e1 - e0)) * vs);
        if (z1 > z0) CK(cudaMemsetAsync(W + z0, 0, (size_t)(z1 - z0) * vs, st));
        const int64_t cnt = e1 - e0, nri = part == 2 ? 0 : nr;
        if (cnt > 0 || nri > 0)
            k_assemble<T><<<nblk(std::max(cnt, nri)), 256, 0, st>>>(W, Bx, D.asm_src + e0, D.asm_dst + e0, cnt,
                                                                    N.rowid + F.row_off, D.rowinit + F.row_off, nri, N.st,
                                                                    pre ? 1 : 0), note_launch();
        for (int64_t k = F.child_begin; k < F.child_end; k++) {
            const int64_t gi = P.children[k];
            const Front &G = P.fronts[gi];
            const int64_t cbr = std::max<int64_t>(0, G.nrows - G.npiv), cbc = G.ncols - G.npiv;
            const int64_t nslot = std::max<int64_t>(0, G.nri - G.npiv);
            if (cbr == 0) continue;
            const int64_t c0 = part == 2 ? hc[gi] : 0, c1 = pre ? 0 : part == 1 ? hc[gi] : cbc;
            const int rowids = part != 2;
            if (c1 <= c0 && !rowids) continue;
            k_extend_add<T><<<nblk(std::max(cbr * std::max<int64_t>(c1 - c0, 0), nslot)), 256, 0, st>>>(
                W, ld, cb_of(gi), cbr, c0, std::max(c0, c1), nslot, G.slot, F.tau_base, D.relcol + G.relcol_off,
                N.rowid + F.row_off, N.rowid + G.row_off + G.npiv, rowids, N.st), note_launch();
        }
        prof.end(st);
        return FPLUS_OK;
    };
    // the pivot block: partial-pivot LU, L\U into the arena in the final row order, the order into perm
    auto factor_block = [&](int64_t fi, T *W, int *perm, cudaStream_t st, const PivotAsm &pa) {
        const Front &F = P.fronts[fi];
        const int64_t nr = F.nrows, np = F.npiv, ld = nr;
        T *Lf = La + F.L_off;
        const size_t sm = front_lu_smem(nr, np, vs);
        {
            double fl = 0;
            for (int64_t k = 0; k < std::min(np, nr); k++) fl += (double)(nr - k - 1) * (double)(np - k);
            prof.begin(st, sm <= SMEM_MAX ? PROF_LU : PROF_LU_TALL, fm * fl, 2.0 * (double)(nr * np) * vs);
        }
        if ((N.lu_variant & 3) == 3 && use_lu3(nr, np, vs)) {
            const size_t sm3 = front_lu3_smem(nr, np, vs);
            if (pa.on) {
                CK(launch_pdl(k_front_lu3<T>, 1, LU3_THREADS, sm3, st, (const T *)W, ld, (int)nr, (int)np, (int)F.nri, F.f,
                              (const double *)N.colmax, pivot_rel, N.rowid + F.row_off, Lf, perm, N.p_lu, N.st, fi, pa));
                note_launch();
            } else
                k_front_lu3<T><<<1, LU3_THREADS, sm3, st>>>(W, ld, (int)nr, (int)np, (int)F.nri, F.f, N.colmax, pivot_rel,
                                                            N.rowid + F.row_off, Lf, perm, N.p_lu, N.st, fi, pa), note_launch();
        } else if ((N.lu_variant & 3) == 1 && nr <= 128 && np <= 64) {
            const size_t sm5 = front_lu5_smem(nr, np, vs);
            if (pa.on) {      // right after the child's tail head on the critical stream: overlap the launch
                CK(launch_pdl(k_front_lu5<T>, 1, LU5_THREADS, sm5, st, (const T *)W, ld, (int)nr, (int)np, (int)F.nri, F.f,
                              (const double *)N.colmax, pivot_rel, N.rowid + F.row_off, Lf, perm, N.p_lu, N.st, fi, pa));
                note_launch();
            } else
                k_front_lu5<T><<<1, LU5_THREADS, sm5, st>>>(W, ld, (int)nr, (int)np, (int)F.nri, F.f, N.colmax, pivot_rel,
                                                            N.rowid + F.row_off, Lf, perm, N.p_lu, N.st, fi, pa), note_launch();
        } else if (sm <= SMEM_MAX) {
            const int R = (int)((nr + 31) & ~31);
            int nt = 32 + (R <= 128 ? 4 * R : R);   // the pivot warp + the update warps
            if (nt > 640) nt = 640;
            if (pa.on) {      // right after the child's tail head on the critical stream: overlap the launch
                CK(launch_pdl(k_front_lu2<T>, 1, nt, sm, st, (const T *)W, ld, (int)nr, (int)np, (int)F.nri, F.f,
                              (const double *)N.colmax, pivot_rel, N.rowid + F.row_off, Lf, perm, N.p_lu, N.st, fi, pa));
                note_launch();
            } else
                k_front_lu2<T><<<1, nt, sm, st>>>(W, ld, (int)nr, (int)np, (int)F.nri, F.f, N.colmax, pivot_rel, N.rowid + F.row_off,
                                                Lf, perm, N.p_lu, N.st, fi, pa), note_launch();
        } else {
            const int64_t npr = std::min(np, nr);
            // the multi-CTA pivoting in one launch, when the rows fit the CTAs (at most per_max rows each): one cluster
            // when it holds them, else a cooperative launch
            bool done = false;
            if (any_mc && !(N.lu_variant & 4)) {
                // (measured on B200: the cluster form is the faster up to about 3,000 rows, with as many CTAs as the
                // cluster takes; above, the grid form over the SMs)
                const bool cl = mc_cl > 0 && nr <= std::min<int64_t>((int64_t)mc_cl * per_max, 3072);
                int G = cl ? (int)std::min<int64_t>(mc_cl, std::max<int64_t>(2, (nr + 31) / 32))
                           : (int)std::min<int64_t>(mc_sms, std::max<int64_t>(1, (nr + 63) / 64));
                if ((nr + G - 1) / G > per_max) G = (int)((nr + per_max - 1) / per_max);
                const int per = (int)((nr + G - 1) / G);
                const int64_t *rid = N.rowid + F.row_off;
                cudaError_t le = cudaErrorInvalidValue;
                if (cl && G <= mc_cl) {
                    cudaLaunchConfig_t cfg = {};
                    cudaLaunchAttribute at[1];
                    at[0].id = cudaLaunchAttributeClusterDimension;
                    at[0].val.clusterDim.x = (unsigned)G; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
                    cfg.gridDim = dim3((unsigned)G); cfg.blockDim = dim3(MC_THREADS); cfg.dynamicSmemBytes = mc_smem<T>(per, true);
                    cfg.stream = st; cfg.attrs = at; cfg.numAttrs = 1;
                    le = cudaLaunchKernelEx(&cfg, k_block_lu_mc<T, true>, W, ld, (int)nr, (int)np, (int)F.nri, per, F.f,
                                            (const double *)N.colmax, pivot_rel, rid, mc_chosen, mc_U, mc_slot, mc_sync, N.st, fi);
                } else if (!cl && mc_sms > 0 && G <= mc_sms) {
                    T *Wp = W;
                    int64_t ldl = ld, fcol = F.f, frow = fi;
                    int nri_ = (int)nr, npi = (int)np, nrii = (int)F.nri, peri = per;
                    const double *cm = N.colmax;
                    double prel = pivot_rel;
                    int64_t *chs = mc_chosen;
                    T *ub = mc_U;
                    McSlot<T> *sl = mc_slot;
                    unsigned int *sy = mc_sync;
                    DevStatus *stp = N.st;
                    void *args[] = {&Wp, &ldl, &nri_, &npi, &nrii, &peri, &fcol, &cm, &prel, &rid, &chs, &ub, &sl, &sy, &stp, &frow};
                    le = cudaLaunchCooperativeKernel((const void *)k_block_lu_mc<T, false>, G, MC_THREADS, args,
                                                     mc_smem<T>(per, false), st);
                }
                if (le == cudaSuccess) {
                    note_launch();
                    k_mc_order<T><<<1, 1024, 0, st>>>((int)nr, (int)npr, mc_chosen, N.rowid + F.row_off, perm, F.f, N.p_lu,
                                                      mc_markp, mc_ridp, N.st), note_launch();
                    k_mc_lout<T><<<nblk(nr * np), 256, 0, st>>>(W, ld, nr, np, npr, perm, mc_U, Lf, N.st), note_launch();
                    done = true;
                } else (void)cudaGetLastError();
            }
            if (!done) {
                // one CTA per 32-column panel, then the swaps, the unit-lower solve and the update of the block's later
                // columns
                for (int64_t k0 = 0; k0 < npr; k0 += PW) {
                    const int w = (int)std::min<int64_t>(PW, npr - k0);
                    k_panel<T><<<1, 512, 0, st>>>(W, ld, nr, F.nri, (int)k0, w, F.f, N.colmax, pivot_rel, N.rowid + F.row_off,
                                                 N.ipiv + F.f, N.st, fi), note_launch();
                    if (k0 > 0) k_laswp<T><<<nblk(k0, 128), 128, 0, st>>>(W, ld, N.ipiv + F.f, (int)k0, w, 0, k0, N.st), note_launch();
                    if (k0 + w < np) {
                        k_laswp<T><<<nblk(np - k0 - w, 128), 128, 0, st>>>(W, ld, N.ipiv + F.f, (int)k0, w, k0 + w, np, N.st), note_launch();
                        k_trsm_unit<T><<<nblk(np - k0 - w, 128), 128, 0, st>>>(W, ld, (int)k0, w, k0 + w, np, N.st), note_launch();
                        const int64_t M = nr - k0 - w, Nn = np - k0 - w;
                        if (M > 0) {
                            dim3 g((unsigned)((M + GBM - 1) / GBM), (unsigned)((Nn + GBN - 1) / GBN));
                            T *C = W + (k0 + w) + (k0 + w) * ld;
                            k_gemm_sub<T><<<g, 256, 0, st>>>(M, Nn, w, W + (k0 + w) + k0 * ld, ld, W + k0 + (k0 + w) * ld, ld,
                                                             C, ld, nullptr, C, ld, N.st, OutMap{}), note_launch();
                        }
                    }
                }
                k_left_finish<T><<<nblk(nr * np), 256, 0, st>>>(W, ld, nr, np, N.ipiv + F.f, perm, N.rowid + F.row_off, F.f, N.p_lu,
                                                               Lf, N.st), note_launch();
            }
        }
        prof.end(st);
        if (nr < np) { k_set_singular<<<1, 1, 0, st>>>(N.st, F.f + nr), note_launch(); }
        return FPLUS_OK;
    };
    // U12 and the CB for CB columns [c0, c1) by the fused tail kernel (at most `cap` CTAs)
    auto tail = [&](int64_t fi, T *W, const int *perm, cudaStream_t st, int64_t c0, int64_t c1, int cap, bool narrow,
                    const TailOut &to = TailOut{}) {
        const Front &F = P.fronts[fi];
        const int64_t nr = F.nrows, np = F.npiv, ncb = F.ncols - F.npiv, M = nr - np;
        if (c1 <= c0) return FPLUS_OK;
        prof.begin(st, PROF_SCHUR, fm * ((double)np * (double)np / 2.0 + (double)M * (double)np) * (double)(c1 - c0),
                   (double)(2 * nr * (c1 - c0) + nr * np) * vs);
        const int tn = narrow ? 8 : FT_TN;
        const size_t fsm = (size_t)(VT<T>::cplx_ ? 2 : 1) * (FT_NP + tn) * FT_LD * sizeof(double);
        const int blocks = (int)std::min<int64_t>((c1 - c0 + tn - 1) / tn, cap);
        // (the narrow tiles of a pipelined front's head, which the next pivot block waits for, by forward substitution:
        // eight CTAs, each forming the block-inverse multipliers first, would take longer)
        if (!(N.lu_variant & 16) && !narrow)
            k_front_tail2<T, FT_TN><<<blocks, FT_THREADS, fsm, st>>>(W, nr, perm, (int)np, (int)nr, ncb, c0, c1, La + F.L_off,
                                                                    Ua + F.U_off, CB + F.cb_off, N.st, to), note_launch();
        else if (narrow)
            k_front_tail<T, 8><<<blocks, FT_THREADS, fsm, st>>>(W, nr, perm, (int)np, (int)nr, ncb, c0, c1, La + F.L_off,
                                                               Ua + F.U_off, CB + F.cb_off, N.st), note_launch();
        else
            k_front_tail<T, FT_TN><<<blocks, FT_THREADS, fsm, st>>>(W, nr, perm, (int)np, (int)nr, ncb, c0, c1, La + F.L_off,
                                                                   Ua + F.U_off, CB + F.cb_off, N.st), note_launch();
        prof.end(st);
        return FPLUS_OK;
    };

    // the batched fronts first, level by level: the working blocks zeroed, then one launch each for the assembly, the
    // pivot-block LU and the tail of every batched front of the level (their children are batched and done)
    if (bs_on) {
        T *Wb = (T *)N.bsw;
        const int64_t nlev = (int64_t)D.bs_ptr.size() - 1;
        const size_t fsm = (size_t)(VT<T>::cplx_ ? 2 : 1) * (FT_NP + FT_TN) * FT_LD * sizeof(double);
        for (int64_t lv = 0; lv < nlev; lv++) {
            const int64_t a0 = D.bs_ptr[(size_t)lv], a1 = D.bs_ptr[(size_t)lv + 1];
            if (a1 <= a0) continue;
            const unsigned cnt = (unsigned)(a1 - a0);
            const int *bl = D.bs_list + a0;
            prof.begin(s, PROF_ASM, 0.0, D.bs_asm_bytes[(size_t)lv] * (double)vs);
            CK(cudaMemsetAsync(Wb, 0, (size_t)D.bs_wsz[(size_t)lv] * vs, s));
            k_bat_assemble<T><<<cnt, 256, 0, s>>>(D.fc, bl, D.children, Wb, Bx, D.asm_src, D.asm_dst, D.rowinit, N.rowid, D.relcol,
                                                  CBA, N.st), note_launch();
            prof.end(s);
            const int R = (int)((D.bs_maxnr[(size_t)lv] + 31) & ~31);
            int nt = 32 + (R <= 128 ? 4 * R : R);
            if (nt > 640) nt = 640;
            prof.begin(s, PROF_LU, fm * D.bs_lu_flops[(size_t)lv], D.bs_lu_bytes[(size_t)lv] * (double)vs);
            if ((N.lu_variant & 3) == 1)
                k_bat_lu5<T><<<cnt, LU5_THREADS, front_lu5_smem(D.bs_maxnr[(size_t)lv], D.bs_maxnp[(size_t)lv], vs), s>>>(
                    D.fc, bl, Wb, N.colmax, pivot_rel, N.rowid, La, N.permall, N.p_lu, N.st), note_launch();
            else
                k_bat_lu2<T><<<cnt, nt, front_lu_smem(D.bs_maxnr[(size_t)lv], D.bs_maxnp[(size_t)lv], vs), s>>>(
                    D.fc, bl, Wb, N.colmax, pivot_rel, N.rowid, La, N.permall, N.p_lu, N.st), note_launch();
            prof.end(s);
            if (D.bs_maxtiles[(size_t)lv] > 0) {
                prof.begin(s, PROF_SCHUR, fm * D.bs_tail_flops[(size_t)lv], D.bs_tail_bytes[(size_t)lv] * (double)vs);
                const dim3 tg((unsigned)std::min<int64_t>(D.bs_maxtiles[(size_t)lv], 148), cnt);
                if (!(N.lu_variant & 16))
                    k_bat_tail2<T, FT_TN><<<tg, FT_THREADS, fsm, s>>>(D.fc, bl, Wb, N.permall, La, Ua, CBA, N.st), note_launch();
                else
                    k_bat_tail<T, FT_TN><<<tg, FT_THREADS, fsm, s>>>(D.fc, bl, Wb, N.permall, La, Ua, CBA, N.st), note_launch();
                prof.end(s);
            }
        }
    }

    // A front whose parent is the next front, takes no other child, and whose contribution block covers every row of the
    // parent's working block but its entering rows, and every column: its Schur update writes straight into the
    // parent's working block (through the extend-add maps; the two working blocks alternate), whose entering rows are
    // zeroed first and whose original entries are added after.  The contribution block never goes through the stack.
    std::vector<char> direct((size_t)nf, 0);
    bool any_direct = false;
    for (int64_t fi = 0; fi + 1 < nf; fi++) {
        const Front &F = P.fronts[(size_t)fi], &Q = P.fronts[(size_t)fi + 1];
        if (pipe[(size_t)fi] || pipe[(size_t)fi + 1] || F.parent != fi + 1 || Q.child_end - Q.child_begin != 1) continue;
        if (bs_on && (D.is_bs[(size_t)fi] || D.is_bs[(size_t)fi + 1])) continue;
        const int64_t np = F.npiv, nr = F.nrows, ncb = F.ncols - np, M = nr - np;
        if (np == 0 || np > nr || M <= 0 || ncb <= 0 || (np <= FT_NP && nr <= FT_NR)) continue;
        const int64_t nslot = std::max<int64_t>(0, F.nri - np);
        if (ncb != Q.ncols || F.slot + nslot != Q.tau_base || M - nslot != Q.nrows - Q.tau_base) continue;
        direct[(size_t)fi] = 1;
        any_direct = true;
    }
    // the second working block only where it fits a quarter of the free device memory (a pattern whose largest front is
    // a sizable share of HBM keeps the contribution blocks on the stack)
    if (any_direct && N.cap_work2 < (size_t)P.work_size * vs) {
        size_t fr = 0, tot = 0;
        const bool big = (size_t)P.work_size * vs > ((size_t)1 << 30);        // (small blocks: no device query)
        if (N.capture || (big && (cudaMemGetInfo(&fr, &tot) != cudaSuccess || (size_t)P.work_size * vs > fr / 4))) {
            (void)cudaGetLastError();
            std::fill(direct.begin(), direct.end(), 0);
            any_direct = false;
        }
    }
    if (any_direct && (rc = ensure_async(N, (void **)&N.work2, &N.cap_work2, (size_t)P.work_size * vs, err, errlen))) return rc;
    T *next_W = nullptr;                 // the working block a direct child has written into, for the next front

    bool in_pipe = false;
    int wsel = 0;
    for (int64_t fi = 0; fi < nf; fi++) {
        const Front &F = P.fronts[fi];
        const int64_t nr = F.nrows, nc = F.ncols, np = F.npiv, ncb = nc - np;
        if (bs_on && D.is_bs[(size_t)fi]) continue;
        if (pipe[fi]) {
            // critical stream: [pivot-column assembly], LU, then (once the bulk stream has assembled the other
            // columns) the tail on the CB columns that are the parent's pivot columns; bulk stream: the assembly of the
            // other columns, then (after the LU) the rest of the tail
            if (!in_pipe) { CK(cudaEventRecord(N.ev_head, s)); CK(cudaStreamWaitEvent(A, N.ev_head, 0)); in_pipe = true; }
            T *W = (T *)(wsel ? N.work2 : N.work);
            int *perm = N.permall + F.row_off;
            wsel ^= 1;
            PivotAsm pa{};
            if (F.child_end - F.child_begin <= 1) {
                // the LU kernel assembles the pivot block itself (from at most one child)
                pa.on = 1;
                pa.asrc = D.asm_src + F.asm_begin; pa.adst = D.asm_dst + F.asm_begin;
                pa.acnt = (ncb > 0 ? F.asm_mid : F.asm_end) - F.asm_begin;
                pa.Bx = Bx; pa.rowinit = D.rowinit + F.row_off; pa.tau_base = F.tau_base;
                if (F.child_end > F.child_begin) {
                    const int64_t gi = P.children[F.child_begin];
                    const Front &G = P.fronts[gi];
                    pa.cbr = std::max<int64_t>(0, G.nrows - G.npiv);
                    pa.h = pa.cbr > 0 ? hc[gi] : 0;
                    pa.nslot = std::max<int64_t>(0, G.nri - G.npiv);
                    pa.slot = G.slot;
                    pa.cb = cb_of(gi); pa.relcol = D.relcol + G.relcol_off; pa.child_rowid = N.rowid + G.row_off + G.npiv;
                }
            } else if ((rc = assemble(fi, W, A, ncb > 0 ? 1 : 0))) return rc;
            if ((rc = factor_block(fi, W, perm, A, pa))) return rc;
            CK(cudaEventRecord(N.ev_lu, A));
            if (ncb > 0) {
                if ((rc = assemble(fi, W, s, fi > 0 && pdirect[(size_t)fi - 1] ? 4 : 2))) return rc;
                CK(cudaEventRecord(N.ev_head, s));
                CK(cudaStreamWaitEvent(s, N.ev_lu, 0));
                const int64_t h = std::min<int64_t>(ncb, (hc[fi] + FT_TN - 1) / FT_TN * FT_TN);
                TailOut to{};
                if (pdirect[(size_t)fi]) {
                    const Front &Q = P.fronts[(size_t)fi + 1];
                    to.W = wsel ? N.work2 : N.work;                    // the parent's working block (the next in turn)
                    to.ld = Q.nrows;
                    to.nslot = std::max<int64_t>(0, F.nri - np);
                    to.slot = F.slot;
                    to.tau_base = Q.tau_base;
                    to.relcol = D.relcol + F.relcol_off;
                }
                // at most 139 CTAs: one SM stays free for the next LU and eight for the next tail head
                if ((rc = tail(fi, W, perm, s, h, ncb, 139, false, to))) return rc;
                CK(cudaStreamWaitEvent(A, N.ev_head, 0));
                if ((rc = tail(fi, W, perm, A, 0, h, 148, true))) return rc;
            }
            if ((fi & 255) == 255) CK(cudaGetLastError());
            continue;
        }
        if (in_pipe) { CK(cudaEventRecord(N.ev_lu, A)); CK(cudaStreamWaitEvent(s, N.ev_lu, 0)); in_pipe = false; }
        T *W = next_W ? next_W : (T *)N.work;
        const bool pre = next_W != nullptr;
        next_W = nullptr;
        T *Lf = La + F.L_off;
        const int64_t ld = nr;
        if ((rc = assemble(fi, W, s, pre ? 3 : 0))) return rc;
        if (np == 0) continue;
        if (nr == 0) { k_set_singular<<<1, 1, 0, s>>>(N.st, F.f), note_launch(); continue; }     // no row can take pivot step f
        if ((rc = factor_block(fi, W, N.permall + F.row_off, s, PivotAsm{}))) return rc;
        if (ncb == 0) continue;
        T *Uf = Ua + F.U_off;
        if (std::min(np, nr) == np && np <= FT_NP && nr <= FT_NR) {
            if ((rc = tail(fi, W, N.permall + F.row_off, s, 0, ncb, 148, false))) return rc;
            if ((fi & 255) == 255) CK(cudaGetLastError());
            continue;
        }
        // U12 = L11^-1 A12[perm]: gather the pivot rows into the arena, then blocked TRSM in place
        prof.begin(s, PROF_U12, fm * (double)np * (double)np / 2.0 * (double)ncb, 3.0 * (double)(np * ncb) * vs);
        const int64_t npr = std::min(np, nr);
        if (npr == np && np <= U12_NP) {
            // gather + blocked TRSM of 32-column tiles in shared memory; persistent CTAs (L11 staged once per CTA)
            const size_t tsm = (size_t)(U12_NP * U12_NP + U12_NP * U12_TN) * vs;
            const int blocks = (int)std::min<int64_t>((ncb + U12_TN - 1) / U12_TN, 2 * 148);
            k_u12_blk<T><<<blocks, 256, tsm, s>>>(W, ld, N.permall + F.row_off, (int)np, ncb, Lf, ld, Uf, N.st), note_launch();
        } else {
        k_u12_gather<T><<<nblk(np * ncb), 256, 0, s>>>(W, ld, np, ncb, N.permall + F.row_off, Uf, N.st), note_launch();
        for (int64_t k0 = 0; k0 < npr; k0 += TB) {
            const int w = (int)std::min<int64_t>(TB, npr - k0);
            const size_t tsm = (size_t)w * w * vs;
            const int nwarps = (int)std::min<int64_t>((ncb + 3) / 4, 148 * 32);     // four columns per warp at once
            const int blocks = (nwarps + 7) / 8;
            if (w <= 32) k_trsm_warp<T, 1><<<blocks, 256, tsm, s>>>(Uf + k0, np, w, ncb, Lf + k0 + k0 * ld, ld, N.st), note_launch();
            else k_trsm_warp<T, 2><<<blocks, 256, tsm, s>>>(Uf + k0, np, w, ncb, Lf + k0 + k0 * ld, ld, N.st), note_launch();
            const int64_t M = npr - k0 - w;
            if (M > 0) {
                dim3 g((unsigned)((M + GBM - 1) / GBM), (unsigned)((ncb + GBN - 1) / GBN));
                T *C = Uf + k0 + w;
                k_gemm_sub<T><<<g, 256, 0, s>>>(M, ncb, w, Lf + (k0 + w) + k0 * ld, ld, Uf + k0, np, C, np, nullptr, C, np, N.st, OutMap{}), note_launch();
            }
        }
        }
        prof.end(s);
        // the Schur complement into the CB stack: CB = A22[perm] - L21 U12 (the precision form: on the tcgen05 tensor
        // cores in reduced precision for the large updates; FP64 DMMA otherwise)
        const int64_t M = nr - np;
        if (M > 0) {
            // the output: the stack, or (direct) the parent's working block, the other of the two, its entering rows zeroed
            T *Cout = CB + F.cb_off;
            int64_t ldco = M;
            OutMap om{};
            if (direct[(size_t)fi]) {
                const Front &Q = P.fronts[(size_t)fi + 1];
                T *Wq = W == (T *)N.work ? (T *)N.work2 : (T *)N.work;
                if (F.slot > 0)
                    CK(cudaMemset2DAsync(Wq, (size_t)Q.nrows * vs, 0, (size_t)F.slot * vs, (size_t)Q.ncols, s));
                Cout = Wq;
                ldco = Q.nrows;
                om = OutMap{D.relcol + F.relcol_off, std::max<int64_t>(0, F.nri - np), F.slot, Q.tau_base};
                next_W = Wq;
            }
            prof.begin(s, PROF_SCHUR, fm * (double)M * (double)ncb * (double)np, (double)(2 * M * ncb + M * np + np * ncb) * vs);
            const bool tc = N.prec != PREC_FP64 && M >= TC_MIN_ROWS && ncb >= TC_MIN_COLS &&
                            (double)M * (double)ncb * (double)np >= TC_MIN_MADDS && schur_tc_supported(M, ncb, np, VT<T>::cplx_);
            int trc = 1;
            if (tc) {
                const size_t wsb = schur_tc_workspace(N.prec, M, ncb, np, VT<T>::cplx_);
                if ((rc = ensure_async(N, &N.tcws, &N.cap_tcws, wsb, err, errlen))) return rc;
                trc = schur_tc(N.prec, VT<T>::cplx_, M, ncb, np, (const double *)(Lf + np), ld, (const double *)Uf, np,
                               (const double *)(W + np * ld), ld, N.permall + F.row_off + np, (double *)Cout, ldco, N.tcws, N.cap_tcws,
                               &N.st->tc_err, s, om);
                if (trc == 0) { note_launch(); add_launches(2); N.tc_updates++; N.tc_flops += fm * (double)M * (double)ncb * (double)np; }
            }
            if (trc != 0) {
                dim3 g((unsigned)((M + GBM - 1) / GBM), (unsigned)((ncb + GBN - 1) / GBN));
                k_gemm_sub<T><<<g, 256, 0, s>>>(M, ncb, np, Lf + np, ld, Uf, np, W + np * ld, ld, N.permall + F.row_off + np, Cout,
                                                ldco, N.st, om), note_launch();
            }
            prof.end(s);
        }
        if ((fi & 255) == 255) CK(cudaGetLastError());
    }
    if (in_pipe) { CK(cudaEventRecord(N.ev_lu, A)); CK(cudaStreamWaitEvent(s, N.ev_lu, 0)); }    // the bulk stream joins
    CK(cudaGetLastError());
    k_pinv<<<nblk(N.n), 256, 0, s>>>(N.p_lu, N.pinv, N.n, N.st), note_launch();
    if (N.capture) return FPLUS_OK;              // the status is read after the graph has run
    DevStatus h;
    CK(cudaMemcpyAsync(&h, N.st, sizeof(h), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    prof.flush();
    // A pivot event (a dense-row pivot, no admissible pivot) must be the first in the fronts' order, as the reference
    // meets it column by column; the batched levels run the lower fronts of later subtrees first.  Redo it front by
    // front: this happens on a pattern's first factorization (before its dense-chain start is known) or on failure.
    if (bs_on && (h.code == ST_BORDER || h.code == ST_SINGULAR) && !h.tc_err)
        return run_fronts<T>(P, D, N, pivot_rel, border_front, err, errlen, false);
    if (h.tc_err) { errf(err, errlen, "factorization: a tensor-core Schur update timed out (status %u)", h.tc_err); return FPLUS_ERR_GPU; }
    if (h.code == ST_WAIT) { errf(err, errlen, "factorization: a multi-CTA pivot search in front %ld timed out", (long)h.idx); return FPLUS_ERR_GPU; }
    if (h.code == ST_BORDER) { *border_front = h.idx; return FPLUS_OK; }
    if (h.code == ST_SINGULAR) {
        errf(err, errlen, "Near-zero or zero pivot %.6e at step %ld (threshold %.6e). Matrix is singular.", h.best, (long)h.idx, h.thr);
        return FPLUS_ERR_SINGULAR;
    }
    if (h.code != ST_OK) { errf(err, errlen, "factorization: device status %d", h.code); return FPLUS_ERR_INTERNAL; }
    return FPLUS_OK;
}

int dev_equilibrate(const DevPlan &D, DevNum &N, int equilibrate, int max_iter, double tol, char *err, size_t errlen)
{
    return N.cplx ? run_equil<cplx>(D, N, equilibrate, max_iter, tol, err, errlen)
                  : run_equil<double>(D, N, equilibrate, max_iter, tol, err, errlen);
}

int dev_ruiz_matrix(int64_t n, const std::vector<int64_t> &Cp, const std::vector<int64_t> &Ci, const std::vector<int64_t> &src,
                    const void *x_in, void *x_out, int cplx, int max_iter, double tol, double *Dr, double *Dc, int *iters,
                    cudaStream_t stream, char *err, size_t errlen)
{
    const int64_t nnz = Cp[n];
    DevPlan D;
    CK(cudaGetDevice(&D.device));
    int rc;
    if ((rc = upload(Cp, &D.Bp, err, errlen)) || (rc = upload(Ci, &D.Bi, err, errlen)) || (rc = upload(src, &D.Bsrc, err, errlen)) ||
        (rc = upload_segments(n, Cp, D, err, errlen)))
        return rc;
    DevNum N;
    if (stream) N.stream = stream;
    if ((rc = dev_num_init(N, n, nnz, cplx, err, errlen))) return rc;
    const size_t bytes = (size_t)nnz * (size_t)N.vs;
    if (bytes) CK(cudaMemcpyAsync(N.Ax, x_in, bytes, cudaMemcpyHostToDevice, N.stream));
    if ((rc = dev_equilibrate(D, N, 1, max_iter, tol, err, errlen))) { cudaStreamSynchronize(N.stream); return rc; }
    if (bytes) CK(cudaMemcpyAsync(x_out, N.Bx, bytes, cudaMemcpyDeviceToHost, N.stream));
    CK(cudaMemcpyAsync(Dr, N.Drp, (size_t)n * 8, cudaMemcpyDeviceToHost, N.stream));
    CK(cudaMemcpyAsync(Dc, N.Dcp, (size_t)n * 8, cudaMemcpyDeviceToHost, N.stream));
    CK(cudaStreamSynchronize(N.stream));
    *iters = N.ruiz_iters;
    return FPLUS_OK;
}

int dev_factor_fronts(const FrontPlan &P, const DevPlan &D, DevNum &N, double pivot_rel, int64_t *border_front,
                      char *err, size_t errlen)
{
    return N.cplx ? run_fronts<cplx>(P, D, N, pivot_rel, border_front, err, errlen)
                  : run_fronts<double>(P, D, N, pivot_rel, border_front, err, errlen);
}

// ---------------------------------------------------------------------------------------------------------------------
// solves on device buffers: x (n x nrhs, ld = n) in, solution out, through the plan's fronts
template <typename T>
static int run_solve_block(const FrontPlan &P, const DevPlan &D, DevNum &N, T *xb, int64_t nrhs, int trans, int raw,
                           char *err, size_t errlen)
{
    cudaStream_t s = N.stream;
    const int64_t n = N.n;
    int rc;
    const size_t nb = (size_t)(n > 0 ? n : 1) * (size_t)nrhs * sizeof(T);
    if ((rc = ensure_async(N, (void **)&N.rbuf, &N.cap_r, nb, err, errlen))) return rc;
    if ((rc = ensure_async(N, (void **)&N.sbuf, &N.cap_s, nb, err, errlen))) return rc;
    // fused backward sweep: one CTA per SM at most, each over >= 128 contribution-block columns
    auto bwd_chunk = [](int64_t ncb) { int64_t c = (ncb + 147) / 148; return c < 128 ? (int64_t)128 : c; };
    auto bwd_grid = [&](int64_t ncb) { return ncb > 0 ? (ncb + bwd_chunk(ncb) - 1) / bwd_chunk(ncb) : (int64_t)1; };
    auto chunk_of = [](int64_t ncb) { int64_t c = (ncb + 295) / 296; return c < 32 ? (int64_t)32 : c; };
    int64_t maxpart = 1;
    // the L21^T partial sums of a large front's transposed sweep: at most LT_CH chunks of rows
    constexpr int64_t LT_CH = 148;
    auto lt_chunk = [](int64_t rows) { int64_t c = (rows + LT_CH - 1) / LT_CH; return c < 256 ? (int64_t)256 : c; };
    for (const Front &F : P.fronts) {
        const int64_t ncb = F.ncols - F.npiv;
        maxpart = std::max(maxpart, bwd_grid(ncb) * F.npiv);
        if (ncb > 0) maxpart = std::max(maxpart, ((ncb + chunk_of(ncb) - 1) / chunk_of(ncb)) * F.npiv);
        if (F.nrows > F.npiv) maxpart = std::max(maxpart, ((F.nrows - F.npiv + lt_chunk(F.nrows - F.npiv) - 1) / lt_chunk(F.nrows - F.npiv)) * F.npiv);
    }
    maxpart = std::max(maxpart, D.part_need);
    if ((rc = ensure_async(N, (void **)&N.part, &N.cap_part, (size_t)maxpart * (size_t)nrhs * sizeof(T), err, errlen))) return rc;
    // the contribution vectors of the level-scheduled forward sweeps (rows or columns of every front, per right-hand side)
    const size_t vbytes = (size_t)std::max<int64_t>(1, std::max(D.vrow, D.vcol)) * (size_t)nrhs * sizeof(T);
    if ((rc = ensure_async(N, &N.vbuf, &N.cap_vb, vbytes, err, errlen))) return rc;
    T *R = (T *)N.rbuf, *S2 = (T *)N.sbuf, *part = (T *)N.part, *VB = (T *)N.vbuf;
    const T *La = (const T *)N.Larena, *Ua = (const T *)N.Uarena;
    const int64_t nf = (int64_t)P.fronts.size();
    const int64_t nlev = (int64_t)D.sv_rows_ptr.size() - 1;
    {
        static thread_local bool sv_attr = false;
        if (!sv_attr) {
            CK(cudaFuncSetAttribute(k_sv_fwdL<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX));
            CK(cudaFuncSetAttribute(k_sv_bwdU<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX));
            CK(cudaFuncSetAttribute(k_sv_fwdUt<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX));
            CK(cudaFuncSetAttribute(k_sv_fwdUt<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX));
            CK(cudaFuncSetAttribute(k_sv_bwdLt<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX));
            CK(cudaFuncSetAttribute(k_sv_bwdLt<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX));
            CK(cudaFuncSetAttribute(k_svb_L11<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX));
            CK(cudaFuncSetAttribute(k_svb_L21<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX));
            CK(cudaFuncSetAttribute(k_svb_bwdU<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX));
            CK(cudaFuncSetAttribute(k_svb_u12<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX));
            sv_attr = true;
        }
    }
    const size_t smem = (size_t)P.max_npiv * (size_t)(nrhs + 1) * sizeof(T);
    const size_t fsmem = std::max((size_t)(256 * 8 + 64 * 4 * 8), (size_t)(P.max_npiv * (nrhs + 1) + 256 + 64 * 64)) * sizeof(T);
    constexpr size_t FWD_SMEM = 200 * 1024;
    CK(cudaFuncSetAttribute(k_fwdL2<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
    CK(cudaFuncSetAttribute(k_fwdL3<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FWD_SMEM));
    CK(cudaFuncSetAttribute(k_fwdL11<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FWD_SMEM));
    CK(cudaFuncSetAttribute(k_fwdL21<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FWD_SMEM));
    CK(cudaFuncSetAttribute(k_u12_gemv<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
    if (fsmem > 48 * 1024) CK(cudaFuncSetAttribute(k_bwdU_fused<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fsmem));
    {
        const int t3 = (int)((64 * 65 + 64) * sizeof(T)), b3 = (int)((64 * 65 + 64 * nrhs) * sizeof(T));
        CK(cudaFuncSetAttribute(k_fwdUt3<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, t3));
        CK(cudaFuncSetAttribute(k_fwdUt3<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, t3));
        CK(cudaFuncSetAttribute(k_bwdLt3<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, b3));
        CK(cudaFuncSetAttribute(k_bwdLt3<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, b3));
    }
    if (smem > 48 * 1024) {
        CK(cudaFuncSetAttribute(k_bwdU<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        CK(cudaFuncSetAttribute(k_bwdLt<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        CK(cudaFuncSetAttribute(k_bwdLt<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    if (trans == 0) {
        // R (row space) = Dr * b[row_perm]; forward with L; S2 = R[p_lu] (pivot order); backward with U into R.  raw:
        // b is in pivot order (R[i] = b[pinv[i]]), without scaling
        if (raw) k_rhs_in<T><<<nblk(n * nrhs), 256, 0, s>>>(R, xb, n, N.pinv, nullptr, n, nrhs), note_launch();
        else k_rhs_in<T><<<nblk(n * nrhs), 256, 0, s>>>(R, xb, n, D.row_perm, N.Drp, n, nrhs), note_launch();
        // the L sweep by levels (leaves first): the level's small fronts in one launch (a CTA each), then its larger
        // fronts together (their vectors gathered into VB, then the L11 solves and the L21 products there); y into S2 in
        // pivot order.  The dense chain (the levels above the tree, a front each) sequentially in the row-space vector:
        // its first front's gathered vector into R, then front after front (the next launch overlapping the previous).
        const int64_t chain_lv = D.chain_begin >= 0 ? (int64_t)P.fronts[(size_t)D.chain_begin].level : nlev;
        for (int64_t lv = 0; lv < chain_lv; lv++) {
            const int64_t a0 = D.sv_rows_ptr[(size_t)lv], a1 = D.sv_rows_ptr[(size_t)lv + 1];
            if (a1 > a0) {
                const int64_t mnr = D.sv_rows_maxnr[(size_t)lv], mnp = D.sv_rows_maxnp[(size_t)lv];
                const size_t sm = (size_t)(mnr * SV_RC + mnp * SV_RC + 64 * mnp) * sizeof(T);
                CK(launch_pdl(k_sv_fwdL<T>, (int)(a1 - a0), SV_THREADS, sm, s, (const SvFront *)D.sv, (const int *)(D.sv_rows + a0),
                              La, (const int64_t *)D.rowinit, (const int *)N.permall, (const int64_t *)D.rsp,
                              (const int64_t *)D.rsi, (const T *)R, S2, VB, D.vrow, n, (int)nrhs));
                note_launch();
            }
            // the level's larger fronts together: their vectors, the L11 solves (a CTA each), the L21 products
            const int64_t b0 = D.sv_brows_ptr[(size_t)lv], b1 = D.sv_brows_ptr[(size_t)lv + 1];
            if (b1 > b0) {
                const unsigned nb = (unsigned)(b1 - b0);
                const int *bl = D.sv_brows + b0;
                const int64_t mnr = D.brows_maxnr[(size_t)lv], mnp = D.brows_maxnp[(size_t)lv], mm = D.brows_maxm[(size_t)lv];
                const unsigned gx = (unsigned)std::max<int64_t>(1, std::min<int64_t>((mnr * nrhs + 255) / 256,
                                                                                     std::max<int64_t>(1, 2368 / (int64_t)nb)));
                k_svb_gatherL<T><<<dim3(gx, nb), 256, 0, s>>>(D.sv, bl, D.rowinit, N.permall, D.rsp, D.rsi, R, VB, D.vrow, n,
                                                              nrhs), note_launch();
                if (mnp > 0) {
                    // the L11 solves: at most 8 right-hand sides per CTA (the groups in parallel)
                    const int rcb = (int)std::max<int64_t>(1, std::min<int64_t>(std::min<int64_t>(nrhs, 8),
                        (int64_t)((SMEM_MAX - 64 * 64 * sizeof(T)) / ((size_t)mnp * sizeof(T)))));
                    k_svb_L11<T><<<dim3(nb, (unsigned)((nrhs + rcb - 1) / rcb)), 256, ((size_t)mnp * rcb + 64 * 64) * sizeof(T), s>>>(
                        D.sv, bl, La, VB, D.vrow, S2, n, (int)nrhs, rcb), note_launch();
                    if (mm > 0 && nrhs >= 8 && nb == 1) {
                        // one front and several right-hand sides: u = v[np:] - L21 x as an FP64 tensor-core GEMM, in place
                        const Front &F1 = P.fronts[(size_t)D.sv_brows_host[(size_t)b0]];
                        const int64_t np1 = std::min(F1.npiv, F1.nrows), M1 = F1.nrows - np1;
                        if (M1 > 0) {
                            T *C = VB + F1.row_off + np1;
                            dim3 g((unsigned)((M1 + GBM - 1) / GBM), (unsigned)((nrhs + GBN - 1) / GBN));
                            k_gemm_sub<T><<<g, 256, 0, s>>>(M1, nrhs, np1, La + F1.L_off + np1, F1.nrows, VB + F1.row_off, D.vrow, C,
                                                            D.vrow, nullptr, C, D.vrow, N.st, OutMap{}), note_launch();
                        }
                    } else if (mm > 0) {
                        const int rc2 = (int)std::max<int64_t>(1, std::min<int64_t>(SVB_RC, (int64_t)(SMEM_MAX / ((size_t)mnp * sizeof(T)))));
                        k_svb_L21<T><<<dim3((unsigned)((mm + 255) / 256), nb), 256, (size_t)mnp * rc2 * sizeof(T), s>>>(
                            D.sv, bl, La, VB, D.vrow, (int)nrhs, rc2), note_launch();
                    }
                }
            }
        }
        if (D.chain_begin >= 0) {
            const Front &C = P.fronts[(size_t)D.chain_begin];
            k_sv_gatherL<T><<<nblk(C.nrows * nrhs), 256, 0, s>>>(C.row_off, C.nrows, C.nri, D.rowinit,
                                                                 C.npiv > 0 ? N.permall + C.row_off : nullptr, D.rsp, D.rsi, R, VB,
                                                                 D.vrow, n, nrhs), note_launch();
            k_sv_toR<T><<<nblk(C.nrows * nrhs), 256, 0, s>>>(VB + C.row_off, D.vrow, C.nrows, N.rowid + C.row_off, R, n, nrhs),
                note_launch();
            for (int64_t fi = D.chain_begin; fi < nf; fi++) {
                const Front &F = P.fronts[(size_t)fi];
                if (F.npiv == 0 || F.nrows == 0) continue;
                const size_t fsm = (size_t)F.nrows * nrhs * sizeof(T);
                const int64_t np = std::min(F.npiv, F.nrows);
                const size_t whole_sm = fsm + (size_t)F.nrows * np * sizeof(T), l11_sm = fsm + (size_t)np * np * sizeof(T);
                const int swt = nrhs > 8 ? 512 : 256;        // a warp per right-hand side in the sweeps
                if (F.npiv <= 64 && whole_sm <= FWD_SMEM) {
                    CK(launch_pdl(k_fwdL3<T>, 1, swt, whole_sm, s, La + F.L_off, F.nrows, F.npiv, N.rowid + F.row_off, R, n, nrhs, 1));
                    note_launch();
                } else if (F.npiv <= 64 && l11_sm <= FWD_SMEM) {
                    CK(launch_pdl(k_fwdL3<T>, 1, swt, l11_sm, s, La + F.L_off, F.nrows, F.npiv, N.rowid + F.row_off, R, n, nrhs, 0));
                    note_launch();
                } else if ((size_t)(np * nrhs + 64 * 64) * sizeof(T) <= FWD_SMEM) {
                    const size_t xsm = (size_t)np * nrhs * sizeof(T);
                    k_fwdL11<T><<<1, 256, xsm + 64 * 64 * sizeof(T), s>>>(La + F.L_off, F.nrows, np, N.rowid + F.row_off, R, n, nrhs,
                                                                           part), note_launch();
                    if (F.nrows > np)
                        k_fwdL21<T><<<(unsigned)((F.nrows - np + 255) / 256), 256, xsm, s>>>(La + F.L_off, F.nrows, np,
                                                                                          N.rowid + F.row_off, R, n, nrhs, part), note_launch();
                } else
                    k_fwdL<T><<<1, 256, 0, s>>>(La + F.L_off, F.nrows, F.npiv, N.rowid + F.row_off, R, n, nrhs), note_launch();
            }
            k_gather_range<T><<<nblk((n - C.f) * nrhs), 256, 0, s>>>(S2, R, N.p_lu, C.f, n, nrhs), note_launch();
        }
        int64_t fi_end = nf;                   // fronts below the chain: the row-oriented kernel
        if (D.chain_begin >= 0) {
            // the dense chain, column-oriented: front k's launch first applies front k + 1's solution to the rows above
            const int64_t cb = D.chain_begin, nb = D.chain_nb;
            const size_t csm = std::max((size_t)(nb + (nb + 15) / 16) * nrhs, (size_t)(nb * (nrhs + 1) + nb * nb)) * sizeof(T);
            if (csm > 48 * 1024) CK(cudaFuncSetAttribute(k_chain_bwd<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csm));
            // front by front from the last: each launch subtracts front k + 1's solution from every chain row above it
            // (U read once for all right-hand sides), and its last CTA solves front k's U11 block
            for (int64_t fi = nf - 1; fi >= cb; fi--) {
                const Front &F = P.fronts[fi];
                const int64_t jk1 = fi + 1 < nf ? fi + 1 - cb : -1;
                const int npk1 = jk1 >= 0 ? (int)P.fronts[fi + 1].npiv : 0;
                const int64_t rows = jk1 >= 0 ? jk1 * nb : 0;
                const int cbt = nrhs > 8 ? 512 : 256;      // a warp per right-hand side in the U11 sweep
                const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((rows + cbt / 4 - 1) / (cbt / 4), 296));
                CK(launch_pdl(k_chain_bwd<T>, grid, cbt, csm, s, (const T *)Ua, (const int64_t *)D.chain_uoff, D.chain_f0, nb,
                              jk1, npk1, (const T *)(La + F.L_off), F.nrows, F.f, (int)F.npiv, S2, R, n, nrhs, N.st));
                note_launch();
            }
            fi_end = cb;
        }
        CK(cudaFuncSetAttribute(k_bwdU_blk<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FWD_SMEM));
        // the U sweep below the chain by levels (roots first): the level's small fronts in one launch (a CTA each), then
        // its larger fronts together
        for (int64_t lv = nlev - 1; lv >= 0; lv--) {
            const int64_t a0 = D.sv_cols_ptr[(size_t)lv], a1 = D.sv_cols_ptr[(size_t)lv + 1];
            if (a1 > a0) {
                const int64_t mnp = D.sv_cols_maxnp[(size_t)lv];
                const size_t sm = (size_t)(mnp * SV_RC + 64 * mnp + 64) * sizeof(T);
                CK(launch_pdl(k_sv_bwdU<T>, (int)(a1 - a0), SV_THREADS, sm, s, (const SvFront *)D.sv, (const int *)(D.sv_cols + a0),
                              La, Ua, (const int64_t *)D.cols, (const T *)S2, R, n, (int)nrhs, N.st));
                note_launch();
            }
            // the level's larger fronts together: the U12 partial products, then the U11 solves (a CTA each)
            const int64_t b0 = D.sv_bcols_ptr[(size_t)lv], b1 = D.sv_bcols_ptr[(size_t)lv + 1];
            if (b1 > b0) {
                const unsigned nb = (unsigned)(b1 - b0);
                const int *bl = D.sv_bcols + b0;
                const int64_t mnp = D.bcols_maxnp[(size_t)lv], mch = D.bcols_maxnch[(size_t)lv];
                if (mch > 0) {
                    const size_t xsm = (size_t)D.bcols_maxchunk[(size_t)lv] * SVB_RC * sizeof(T);
                    k_svb_u12<T><<<dim3((unsigned)mch, nb), 256, xsm, s>>>(D.sv, bl, Ua, D.cols, R, n, (int)nrhs, part), note_launch();
                    // the partial sums over many CTAs when a front's right-hand sides are more than its CTA's threads
                    if (mnp * nrhs > 256) {
                        const unsigned gx = (unsigned)std::max<int64_t>(1, std::min<int64_t>((mnp * nrhs + 255) / 256, 148));
                        k_svb_psum<T><<<dim3(gx, nb), 256, 0, s>>>(D.sv, bl, part, S2, n, (int)nrhs), note_launch();
                    }
                }
                const int rcb = (int)std::max<int64_t>(1, std::min<int64_t>(std::min<int64_t>(nrhs, 8),
                    (int64_t)((SMEM_MAX - (64 * 64 + 64) * sizeof(T)) / ((size_t)mnp * sizeof(T)))));
                k_svb_bwdU<T><<<dim3(nb, (unsigned)((nrhs + rcb - 1) / rcb)), 256, ((size_t)mnp * rcb + 64 * 64 + 64) * sizeof(T), s>>>(
                    D.sv, bl, La, part, S2, R, n,
                                                                                               (int)nrhs, rcb, N.st,
                                                                                               mch > 0 && mnp * nrhs > 256 ? 1 : 0),
                    note_launch();
            }
        }
        // x[col_perm[k]] = Dcp[k] * R[k]  (raw: x[k] = R[k])
        k_rhs_out<T><<<nblk(n * nrhs), 256, 0, s>>>(xb, n, R, raw ? nullptr : D.col_perm, nullptr, raw ? nullptr : N.Dcp, n, nrhs),
            note_launch();
    } else {
        // R (column space) = Dc * b[col_perm]; forward with U^T; backward with L^T into S2 (pivot order).  raw: R = b
        k_rhs_in<T><<<nblk(n * nrhs), 256, 0, s>>>(R, xb, n, raw ? nullptr : D.col_perm, raw ? nullptr : N.Dcp, n, nrhs),
            note_launch();
        const bool cj = trans == 2;
        // the U^T sweep by levels (leaves first): the level's small fronts in one launch, the others front by front (their
        // column vector gathered: the pivot columns into R, the others into VB; the U11^T solve in R; the contribution)
        for (int64_t lv = 0; lv < nlev; lv++) {
            const int64_t a0 = D.sv_cols_ptr[(size_t)lv], a1 = D.sv_cols_ptr[(size_t)lv + 1];
            if (a1 > a0) {
                const int64_t mnc = D.sv_cols_maxnc[(size_t)lv], mnp = D.sv_cols_maxnp[(size_t)lv];
                const size_t sm = (size_t)(mnc * SV_RC + mnp * (mnp + 1) + mnp) * sizeof(T);
                if (cj)
                    CK(launch_pdl(k_sv_fwdUt<T, true>, (int)(a1 - a0), SV_THREADS, sm, s, (const SvFront *)D.sv,
                                  (const int *)(D.sv_cols + a0), La, Ua, (const int64_t *)D.csp, (const int64_t *)D.csi, R, VB,
                                  D.vcol, n, (int)nrhs, N.st));
                else
                    CK(launch_pdl(k_sv_fwdUt<T, false>, (int)(a1 - a0), SV_THREADS, sm, s, (const SvFront *)D.sv,
                                  (const int *)(D.sv_cols + a0), La, Ua, (const int64_t *)D.csp, (const int64_t *)D.csi, R, VB,
                                  D.vcol, n, (int)nrhs, N.st));
                note_launch();
            }
            for (int64_t fi : D.big_cols[(size_t)lv]) {
                const Front &F = P.fronts[(size_t)fi];
                const int64_t ncb = F.ncols - F.npiv;
                k_sv_gatherU<T><<<nblk(F.ncols * nrhs), 256, 0, s>>>(F.f, F.npiv, F.ncols, F.col_off, D.csp, D.csi, R, VB, D.vcol,
                                                                     n, nrhs), note_launch();
                if (F.npiv == 0) continue;
                const bool small = F.npiv <= 64 && F.npiv <= F.nrows;
                const size_t tsm = (size_t)(F.npiv * (F.npiv + 1) + F.npiv) * sizeof(T);
                if (small && cj) k_fwdUt3<T, true><<<1, 256, tsm, s>>>(La + F.L_off, F.nrows, F.npiv, F.f, R, n, nrhs, N.st), note_launch();
                else if (small) k_fwdUt3<T, false><<<1, 256, tsm, s>>>(La + F.L_off, F.nrows, F.npiv, F.f, R, n, nrhs, N.st), note_launch();
                else if (cj) k_fwdUt2<T, true><<<1, 256, (size_t)F.npiv * sizeof(T), s>>>(La + F.L_off, F.nrows, F.npiv, F.f, R, n, nrhs, N.st), note_launch();
                else k_fwdUt2<T, false><<<1, 256, (size_t)F.npiv * sizeof(T), s>>>(La + F.L_off, F.nrows, F.npiv, F.f, R, n, nrhs, N.st), note_launch();
                if (ncb > 0) {
                    T *Vc = VB + F.col_off + F.npiv;
                    if (cj) k_sv_utcb<T, true><<<nblk(32 * ncb), 256, 0, s>>>(Ua + F.U_off, F.npiv, ncb, F.f, R, Vc, D.vcol, n, nrhs), note_launch();
                    else k_sv_utcb<T, false><<<nblk(32 * ncb), 256, 0, s>>>(Ua + F.U_off, F.npiv, ncb, F.f, R, Vc, D.vcol, n, nrhs), note_launch();
                }
            }
        }
        // the L^T sweep by levels (roots first): the level's small fronts in one launch, the others front by front
        for (int64_t lv = nlev - 1; lv >= 0; lv--) {
            const int64_t a0 = D.sv_rows_ptr[(size_t)lv], a1 = D.sv_rows_ptr[(size_t)lv + 1];
            if (a1 > a0) {
                const int64_t mnp = D.sv_rows_maxnp[(size_t)lv];
                const size_t sm = (size_t)(mnp * (mnp + 1) + mnp * SV_RC) * sizeof(T);
                if (cj)
                    CK(launch_pdl(k_sv_bwdLt<T, true>, (int)(a1 - a0), SV_THREADS, sm, s, (const SvFront *)D.sv,
                                  (const int *)(D.sv_rows + a0), La, (const int64_t *)N.rowid, (const int64_t *)N.pinv, (const T *)R,
                                  S2, n, (int)nrhs));
                else
                    CK(launch_pdl(k_sv_bwdLt<T, false>, (int)(a1 - a0), SV_THREADS, sm, s, (const SvFront *)D.sv,
                                  (const int *)(D.sv_rows + a0), La, (const int64_t *)N.rowid, (const int64_t *)N.pinv, (const T *)R,
                                  S2, n, (int)nrhs));
                note_launch();
            }
            for (int64_t fi : D.big_rows[(size_t)lv]) {
                const Front &F = P.fronts[(size_t)fi];
                if (F.npiv == 0) continue;
                const size_t sm = (size_t)F.npiv * nrhs * sizeof(T);
                const bool small = F.npiv <= 64 && F.npiv <= F.nrows;
                const size_t tsm = sm + (size_t)F.npiv * (F.npiv + 1) * sizeof(T);
                const int64_t *rid = N.rowid + F.row_off;
                const int64_t rows21 = F.nrows - F.npiv;
                if (small && cj) k_bwdLt3<T, true><<<1, 256, tsm, s>>>(La + F.L_off, F.nrows, F.npiv, F.f, rid, N.pinv, R, S2, n, nrhs), note_launch();
                else if (small) k_bwdLt3<T, false><<<1, 256, tsm, s>>>(La + F.L_off, F.nrows, F.npiv, F.f, rid, N.pinv, R, S2, n, nrhs), note_launch();
                else if (rows21 > 1024) {
                    // a large front: the L21^T product over many CTAs, then the sum and the L11^T solve on one
                    const int64_t ch = lt_chunk(rows21), nch = (rows21 + ch - 1) / ch;
                    if (cj) k_ltdot<T, true><<<(unsigned)nch, 256, 0, s>>>(La + F.L_off, F.nrows, F.npiv, rid, N.pinv, S2, n, nrhs, ch, part), note_launch();
                    else k_ltdot<T, false><<<(unsigned)nch, 256, 0, s>>>(La + F.L_off, F.nrows, F.npiv, rid, N.pinv, S2, n, nrhs, ch, part), note_launch();
                    if (cj) k_bwdLt<T, true><<<1, 256, sm, s>>>(La + F.L_off, F.nrows, F.npiv, F.f, rid, N.pinv, R, S2, n, nrhs, part, (int)nch), note_launch();
                    else k_bwdLt<T, false><<<1, 256, sm, s>>>(La + F.L_off, F.nrows, F.npiv, F.f, rid, N.pinv, R, S2, n, nrhs, part, (int)nch), note_launch();
                }
                else if (cj) k_bwdLt<T, true><<<1, 256, sm, s>>>(La + F.L_off, F.nrows, F.npiv, F.f, rid, N.pinv, R, S2, n, nrhs), note_launch();
                else k_bwdLt<T, false><<<1, 256, sm, s>>>(La + F.L_off, F.nrows, F.npiv, F.f, rid, N.pinv, R, S2, n, nrhs), note_launch();
            }
        }
        // x[row_perm[p_lu[k]]] = Drp[p_lu[k]] * S2[k]  (raw: x[k] = S2[k], pivot order)
        if (raw) k_rhs_out<T><<<nblk(n * nrhs), 256, 0, s>>>(xb, n, S2, nullptr, nullptr, nullptr, n, nrhs), note_launch();
        else k_rhs_out<T><<<nblk(n * nrhs), 256, 0, s>>>(xb, n, S2, D.row_perm, N.p_lu, N.Drp, n, nrhs), note_launch();
    }
    CK(cudaGetLastError());
    return FPLUS_OK;
}

// at most SOLVE_BLOCK right-hand sides per pass (the sweeps' buffers grow with the count)
static constexpr int64_t SOLVE_BLOCK = 32;
template <typename T>
static int run_solve(const FrontPlan &P, const DevPlan &D, DevNum &N, T *xb, int64_t nrhs, int trans, int raw, char *err,
                     size_t errlen)
{
    for (int64_t r0 = 0; r0 < nrhs; r0 += SOLVE_BLOCK) {
        const int rc = run_solve_block(P, D, N, xb + r0 * N.n, std::min(SOLVE_BLOCK, nrhs - r0), trans, raw, err, errlen);
        if (rc) return rc;
    }
    return FPLUS_OK;
}

int dev_solve(const FrontPlan &P, const DevPlan &D, DevNum &N, void *x_dev, int64_t nrhs, int trans, char *err, size_t errlen,
              int raw)
{
    return N.cplx ? run_solve<cplx>(P, D, N, (cplx *)x_dev, nrhs, trans, raw, err, errlen)
                  : run_solve<double>(P, D, N, (double *)x_dev, nrhs, trans, raw, err, errlen);
}

// ---------------------------------------------------------------------------------------------------------------------
// The allocation-free solve (fplus_b200_solve_dev_noalloc), in place on the caller's right-hand sides (leading dimension
// ldx), with the scratch vectors carved from one file-scope device array instead of allocations.  It runs the unfused
// sweep kernels (k_fwdL / k_fwdL2, k_u12_gemv + k_bwdU, k_fwdUt2, k_ut_scatter, k_bwdLt), whose scratch is two vectors
// and the U12 partial sums, not run_solve's fused and chain kernels; its results agree with run_solve's to rounding
// (the sums run in another order), not bit for bit, and it is slower on the dense chain.  Host code cannot use g_noalloc_scratch's name as a device address (it is a host-side stand-in):
// the address comes from cudaGetSymbolAddress, once per device, with that device current.  The array keeps the last
// call's contents; every scratch vector is written before it is read, so nothing needs clearing.  Calls share the array:
// calls that overlap on the GPU (other streams, other host threads) race.
static constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)16 << 20;       // 16 MiB per device, held until exit
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

static int noalloc_scratch(void **ptr, char *err, size_t errlen)
{
    static std::mutex mu;
    static void *addr[64] = {nullptr};
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) { errf(err, errlen, "device %d out of range", dev); return FPLUS_ERR_GPU; }
    std::lock_guard<std::mutex> lk(mu);
    if (!addr[dev]) {
        void *p = nullptr;
        CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        addr[dev] = p;
    }
    *ptr = addr[dev];
    return FPLUS_OK;
}

static inline size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

static constexpr int64_t NOALLOC_GROUP = 32;                          // right-hand sides per pass (the solve kernels' width)

template <typename T>
static int run_solve_noalloc_group(const FrontPlan &P, const DevPlan &D, DevNum &N, T *xb, int64_t ldx, int64_t nrhs,
                                   int trans, cudaStream_t s, char *err, size_t errlen)
{
    const int64_t n = N.n;
    auto chunk_of = [](int64_t ncb) { int64_t c = (ncb + 295) / 296; return c < 32 ? (int64_t)32 : c; };
    int64_t maxpart = 1;
    for (const Front &F : P.fronts) {
        const int64_t ncb = F.ncols - F.npiv;
        if (ncb > 0) maxpart = std::max(maxpart, ((ncb + chunk_of(ncb) - 1) / chunk_of(ncb)) * F.npiv);
    }
    const size_t vb = round256((size_t)(n > 0 ? n : 1) * (size_t)nrhs * sizeof(T));
    const size_t pb = round256((size_t)maxpart * (size_t)nrhs * sizeof(T));
    const size_t need = 2 * vb + pb;
    if (need > NOALLOC_SCRATCH_BYTES) {
        errf(err, errlen, "fplus_b200_solve_dev_noalloc: %zu bytes of scratch needed (n = %ld, %ld right-hand sides per "
             "pass), the fixed maximum is %zu", need, (long)n, (long)nrhs, NOALLOC_SCRATCH_BYTES);
        return FPLUS_ERR_BADARG;
    }
    void *base = nullptr;
    int rc = noalloc_scratch(&base, err, errlen);
    if (rc) return rc;
    T *R = (T *)base, *S2 = (T *)((char *)base + vb), *part = (T *)((char *)base + 2 * vb);
    const T *La = (const T *)N.Larena, *Ua = (const T *)N.Uarena;
    const int64_t nf = (int64_t)P.fronts.size();
    const size_t smem = (size_t)P.max_npiv * (size_t)(nrhs + 1) * sizeof(T);
    CK(cudaFuncSetAttribute(k_fwdL2<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
    CK(cudaFuncSetAttribute(k_u12_gemv<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
    if (smem > 48 * 1024) {
        CK(cudaFuncSetAttribute(k_bwdU<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        CK(cudaFuncSetAttribute(k_bwdLt<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        CK(cudaFuncSetAttribute(k_bwdLt<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    if (trans == 0) {
        k_rhs_in<T><<<nblk(n * nrhs), 256, 0, s>>>(R, xb, ldx, D.row_perm, N.Drp, n, nrhs), note_launch();
        for (int64_t fi = 0; fi < nf; fi++) {
            const Front &F = P.fronts[fi];
            if (F.npiv == 0 || F.nrows == 0) continue;
            const size_t fsm = (size_t)F.nrows * nrhs * sizeof(T);
            if (fsm <= 96 * 1024)
                k_fwdL2<T><<<1, 256, fsm, s>>>(La + F.L_off, F.nrows, F.npiv, N.rowid + F.row_off, R, n, nrhs), note_launch();
            else
                k_fwdL<T><<<1, 256, 0, s>>>(La + F.L_off, F.nrows, F.npiv, N.rowid + F.row_off, R, n, nrhs), note_launch();
        }
        k_gather_rows<T><<<nblk(n * nrhs), 256, 0, s>>>(S2, R, N.p_lu, n, nrhs), note_launch();
        for (int64_t fi = nf - 1; fi >= 0; fi--) {
            const Front &F = P.fronts[fi];
            const int64_t ncb = F.ncols - F.npiv;
            if (F.npiv == 0) continue;
            int64_t nchunk = 0;
            if (ncb > 0) {
                const int64_t chunk = chunk_of(ncb);
                nchunk = (ncb + chunk - 1) / chunk;
                k_u12_gemv<T><<<(unsigned)nchunk, 256, (size_t)8 * F.npiv * sizeof(T), s>>>(
                    Ua + F.U_off, F.npiv, ncb, D.cols + F.col_off + F.npiv, R, n, nrhs, chunk, part), note_launch();
            }
            k_bwdU<T><<<1, 256, (size_t)F.npiv * (nrhs + 1) * sizeof(T), s>>>(La + F.L_off, F.nrows, F.npiv, F.f, part, nchunk, S2, R,
                                                                         n, nrhs, N.st), note_launch();
        }
        k_rhs_out<T><<<nblk(n * nrhs), 256, 0, s>>>(xb, ldx, R, D.col_perm, nullptr, N.Dcp, n, nrhs), note_launch();
    } else {
        k_rhs_in<T><<<nblk(n * nrhs), 256, 0, s>>>(R, xb, ldx, D.col_perm, N.Dcp, n, nrhs), note_launch();
        const bool cj = trans == 2;
        for (int64_t fi = 0; fi < nf; fi++) {
            const Front &F = P.fronts[fi];
            const int64_t ncb = F.ncols - F.npiv;
            if (F.npiv == 0) continue;
            if (cj) k_fwdUt2<T, true><<<1, 256, (size_t)F.npiv * sizeof(T), s>>>(La + F.L_off, F.nrows, F.npiv, F.f, R, n, nrhs, N.st), note_launch();
            else k_fwdUt2<T, false><<<1, 256, (size_t)F.npiv * sizeof(T), s>>>(La + F.L_off, F.nrows, F.npiv, F.f, R, n, nrhs, N.st), note_launch();
            if (ncb > 0) {
                if (cj) k_ut_scatter<T, true><<<nblk(32 * ncb), 256, 0, s>>>(Ua + F.U_off, F.npiv, ncb, D.cols + F.col_off + F.npiv, F.f, R, n, nrhs), note_launch();
                else k_ut_scatter<T, false><<<nblk(32 * ncb), 256, 0, s>>>(Ua + F.U_off, F.npiv, ncb, D.cols + F.col_off + F.npiv, F.f, R, n, nrhs), note_launch();
            }
        }
        for (int64_t fi = nf - 1; fi >= 0; fi--) {
            const Front &F = P.fronts[fi];
            if (F.npiv == 0) continue;
            const size_t sm = (size_t)F.npiv * nrhs * sizeof(T);
            if (cj) k_bwdLt<T, true><<<1, 256, sm, s>>>(La + F.L_off, F.nrows, F.npiv, F.f, N.rowid + F.row_off, N.pinv, R, S2, n, nrhs), note_launch();
            else k_bwdLt<T, false><<<1, 256, sm, s>>>(La + F.L_off, F.nrows, F.npiv, F.f, N.rowid + F.row_off, N.pinv, R, S2, n, nrhs), note_launch();
        }
        k_rhs_out<T><<<nblk(n * nrhs), 256, 0, s>>>(xb, ldx, S2, D.row_perm, N.p_lu, N.Drp, n, nrhs), note_launch();
    }
    CK(cudaGetLastError());
    return FPLUS_OK;
}

int dev_solve_noalloc(const FrontPlan &P, const DevPlan &D, DevNum &N, void *b_dev, int64_t ldb, int64_t nrhs, int trans,
                      cudaStream_t s, char *err, size_t errlen)
{
    const int64_t g = nrhs < NOALLOC_GROUP ? nrhs : NOALLOC_GROUP;
    int rc = FPLUS_OK;
    for (int64_t r0 = 0; r0 < nrhs && rc == FPLUS_OK; r0 += g) {
        const int64_t m = nrhs - r0 < g ? nrhs - r0 : g;
        char *bb = (char *)b_dev + (size_t)r0 * (size_t)ldb * (size_t)N.vs;
        rc = N.cplx ? run_solve_noalloc_group<cplx>(P, D, N, (cplx *)bb, ldb, m, trans, s, err, errlen)
                    : run_solve_noalloc_group<double>(P, D, N, (double *)bb, ldb, m, trans, s, err, errlen);
    }
    return rc;
}

// ||L||_F and ||U||_F of the device factors (the unit diagonal of L included)
template <typename T>
static int run_factor_norms(const FrontPlan &P, DevNum &N, double *lfro, double *ufro, char *err, size_t errlen)
{
    cudaStream_t s = N.stream;
    const int64_t nf = (int64_t)P.fronts.size();
    std::vector<int64_t> fr((size_t)std::max<int64_t>(nf, 1) * 3, 0);
    for (int64_t k = 0; k < nf; k++) {
        fr[3 * k] = P.fronts[k].L_off; fr[3 * k + 1] = P.fronts[k].nrows; fr[3 * k + 2] = P.fronts[k].npiv;
    }
    int rc;
    if ((rc = ensure_async(N, &N.scratch_norm, &N.cap_norm, fr.size() * 8 + 64, err, errlen))) return rc;
    unsigned long long *acc = (unsigned long long *)N.scratch_norm;
    int64_t *dfr = (int64_t *)((char *)N.scratch_norm + 64);
    const unsigned long long init[4] = {0x3ff0000000000000ull, 0ull, 0ull, 0ull};    // 1.0, 0, 0.0, 0.0
    CK(cudaMemcpyAsync(acc, init, sizeof init, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dfr, fr.data(), fr.size() * 8, cudaMemcpyHostToDevice, s));
    const T *La = (const T *)N.Larena, *Ua = (const T *)N.Uarena;
    if (nf > 0) k_lblock_norm<T, 0><<<(unsigned)nf, 256, 0, s>>>(La, dfr, acc), note_launch();
    if (P.U_size > 0) k_flat_norm<T, 0><<<nblk(P.U_size), 256, 0, s>>>(Ua, P.U_size, acc), note_launch();
    if (nf > 0) k_lblock_norm<T, 1><<<(unsigned)nf, 256, 0, s>>>(La, dfr, acc), note_launch();
    if (P.U_size > 0) k_flat_norm<T, 1><<<nblk(P.U_size), 256, 0, s>>>(Ua, P.U_size, acc), note_launch();
    unsigned long long h[4];
    CK(cudaMemcpyAsync(h, acc, sizeof h, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const double ml = bitsd_h(h[0]), mu = bitsd_h(h[1]), sl = bitsd_h(h[2]), su = bitsd_h(h[3]);
    *lfro = ml * std::sqrt(sl + (double)N.n / (ml * ml));
    *ufro = mu * std::sqrt(su);
    return FPLUS_OK;
}

int dev_factor_norms(const FrontPlan &P, DevNum &N, double *lfro, double *ufro, char *err, size_t errlen)
{
    return N.cplx ? run_factor_norms<cplx>(P, N, lfro, ufro, err, errlen) : run_factor_norms<double>(P, N, lfro, ufro, err, errlen);
}

int dev_status(DevNum &N, int *code, int64_t *idx, char *err, size_t errlen)
{
    DevStatus h;
    CK(cudaMemcpyAsync(&h, N.st, sizeof(h), cudaMemcpyDeviceToHost, N.stream));
    CK(cudaStreamSynchronize(N.stream));
    *code = h.code; *idx = h.idx;
    return FPLUS_OK;
}

int dev_status_rc(DevNum &N, int *rc, char *err, size_t errlen)
{
    DevStatus h;
    CK(cudaMemcpy(&h, N.st, sizeof h, cudaMemcpyDeviceToHost));
    if (h.tc_err || h.code == ST_WAIT) *rc = FPLUS_ERR_GPU;
    else if (h.code == ST_SINGULAR || h.code == ST_ZERO_ROW || h.code == ST_ZERO_COL || h.code == ST_SOLVE_ZERO) *rc = FPLUS_ERR_SINGULAR;
    else if (h.code != ST_OK) *rc = FPLUS_ERR_BADARG;
    else *rc = FPLUS_OK;
    return FPLUS_OK;
}

int dev_clear_status(DevNum &N, char *err, size_t errlen)
{
    if (N.capture) { k_clear_status<<<1, 1, 0, N.stream>>>(N.st, 0), note_launch(); return FPLUS_OK; }
    DevStatus h0;
    std::memset(&h0, 0, sizeof(h0));
    h0.idx = INT64_MAX;
    CK(cudaMemcpyAsync(N.st, &h0, sizeof(h0), cudaMemcpyHostToDevice, N.stream));
    return FPLUS_OK;
}

int dev_ensure_x(DevNum &N, size_t bytes, char *err, size_t errlen)
{
    return ensure_async(N, (void **)&N.xbuf, &N.cap_x, bytes, err, errlen);
}

int dev_check_finite(DevNum &N, char *err, size_t errlen)
{
    const int64_t m = (N.cplx ? 2 : 1) * N.nnz;
    if (dev_clear_status(N, err, errlen) != FPLUS_OK) return FPLUS_ERR_GPU;
    k_check_finite<<<nblk(m), 256, 0, N.stream>>>((const double *)N.Ax, m, N.st), note_launch();
    DevStatus h;
    CK(cudaMemcpyAsync(&h, N.st, sizeof(h), cudaMemcpyDeviceToHost, N.stream));
    CK(cudaStreamSynchronize(N.stream));
    if (h.code != 0) {
        errf(err, errlen, "non-finite value in entry %ld", (long)(N.cplx ? h.idx / 2 : h.idx));
        return FPLUS_ERR_BADARG;
    }
    return FPLUS_OK;
}

}  // namespace fpl

// ---------------------------------------------------------------------------------------------------------------------
// iterative refinement (the precision form's driver; here on the FP64 factors)
namespace fpl {

using Hc = std::complex<double>;
static inline Hc toH(double v) { return Hc(v, 0.0); }
static inline Hc toH(const cplx &v) { return Hc(v.x, v.y); }
template <typename T> static inline T fromH(Hc h);
template <> inline double fromH<double>(Hc h) { return h.real(); }
template <> inline cplx fromH<cplx>(Hc h) { return cplx{h.real(), h.imag()}; }

// GMRES-IR (Carson and Higham, SIAM J. Sci. Comput. 40(2), 2018) for one right-hand side, when classic refinement has
// stalled: x is corrected by x += d, d from GMRES (restart GM_RESTART) on the preconditioned correction equation
// M^-1 op(A) d = M^-1 r, where M = the factorization's own LU (whatever the precision of its updates) and the residual
// r = b - op(A) x, the matrix products, the Arnoldi process (classical Gram-Schmidt applied twice) and the update are
// FP64.  A cycle ends when the preconditioned residual has dropped by GM_INNER_TOL.  Stops when the componentwise
// backward error is at most tol, after max_solves applications of M^-1, or when a cycle does not lower the error (that
// cycle is undone).  On return *be is the backward error of x and *solves the applications of M^-1 made.
constexpr int GM_RESTART = 30, GM_CHUNKS = 64;
constexpr double GM_INNER_TOL = 1e-12;

template <typename T>
static int gmres_ir_column(const FrontPlan &P, const DevPlan &D, DevNum &N, T *x, const T *b, int trans, int max_solves,
                           double tol, double *be, int *solves, char *err, size_t errlen)
{
    cudaStream_t s = N.stream;
    const int64_t n = N.n;
    constexpr int RS = GM_RESTART;
    const size_t need = sizeof(T) * ((size_t)n * (RS + 1) + 3 * (size_t)n + (RS + 1) + (size_t)(RS + 1) * GM_CHUNKS);
    int rc;
    if ((rc = ensure_async(N, &N.gm_buf, &N.cap_gm, need, err, errlen))) return rc;
    T *V = (T *)N.gm_buf, *w = V + (size_t)n * (RS + 1), *r = w + n, *zero = r + n, *hd = zero + n, *part = hd + (RS + 1);
    CK(cudaMemsetAsync(zero, 0, (size_t)n * sizeof(T), s));
    const bool t0 = trans == 0;
    const int64_t *ptr = t0 ? N.rr_p : D.Bp, *ix = t0 ? N.rr_l : D.Bi, *src = t0 ? N.rr_s : D.Bsrc;
    const int64_t *outm = t0 ? D.row_perm : D.col_perm, *inm = t0 ? D.col_perm : D.row_perm;
    const int grid = nblk(n * 32);
    // out = bv - op(A) xv, with the componentwise backward error of xv when err_out
    auto resid = [&](const T *xv, const T *bv, T *out, double *err_out) -> int {
        CK(cudaMemsetAsync(N.ir_bits, 0, 8, s));
        if (trans == 2) k_resid<T, true><<<grid, 256, 0, s>>>(ptr, ix, src, (const T *)N.Ax, outm, inm, xv, bv, out, n, 1, N.ir_bits);
        else k_resid<T, false><<<grid, 256, 0, s>>>(ptr, ix, src, (const T *)N.Ax, outm, inm, xv, bv, out, n, 1, N.ir_bits);
        note_launch();
        if (err_out) {
            unsigned long long bits = 0;
            CK(cudaMemcpyAsync(&bits, N.ir_bits, 8, cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            *err_out = bitsd_h(bits);
        }
        return FPLUS_OK;
    };
    // h[v] = conj(V_v) . wv for v < nv
    std::vector<T> hp((size_t)(RS + 1) * GM_CHUNKS);
    auto dots = [&](const T *Vb, int nv, const T *wv, std::vector<Hc> &h) -> int {
        k_vdots<T><<<dim3(GM_CHUNKS, (unsigned)nv), 256, 0, s>>>(Vb, n, wv, part), note_launch();
        CK(cudaMemcpyAsync(hp.data(), part, (size_t)nv * GM_CHUNKS * sizeof(T), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        h.assign((size_t)nv, Hc(0.0, 0.0));
        for (int v = 0; v < nv; v++)
            for (int c = 0; c < GM_CHUNKS; c++) h[(size_t)v] += toH(hp[(size_t)v * GM_CHUNKS + c]);
        return FPLUS_OK;
    };
    std::vector<T> hu((size_t)RS + 1);
    // wv = (wv - sum_v V_v h[v]) * scale
    auto update = [&](const T *Vb, int nv, const std::vector<Hc> &h, T *wv, double scale) -> int {
        for (int v = 0; v < nv; v++) hu[(size_t)v] = fromH<T>(h[(size_t)v]);
        if (nv > 0) CK(cudaMemcpyAsync(hd, hu.data(), (size_t)nv * sizeof(T), cudaMemcpyHostToDevice, s));
        k_vupdate<T><<<nblk(n), 256, 0, s>>>(Vb, n, nv, hd, wv, scale), note_launch();
        if (nv > 0) CK(cudaStreamSynchronize(s));        // hu is reused by the next call
        return FPLUS_OK;
    };
    const std::vector<Hc> none;
    double e = 0.0;
    if ((rc = resid(x, b, r, &e))) return rc;
    int used = 0;
    while (e > tol && used < max_solves) {
        // v0 = M^-1 r / beta
        CK(cudaMemcpyAsync(V, r, (size_t)n * sizeof(T), cudaMemcpyDeviceToDevice, s));
        if ((rc = dev_solve(P, D, N, V, 1, trans, err, errlen))) return rc;
        used++;
        std::vector<Hc> hh, h2;
        if ((rc = dots(V, 1, V, hh))) return rc;
        const double beta = std::sqrt(hh[0].real());
        if (!(beta > 0.0) || !std::isfinite(beta)) break;
        if ((rc = update(V, 0, none, V, 1.0 / beta))) return rc;
        std::vector<std::vector<Hc>> H((size_t)RS, std::vector<Hc>((size_t)RS + 1, Hc(0.0, 0.0)));   // H[j] = column j
        std::vector<double> cs((size_t)RS, 0.0);
        std::vector<Hc> sn((size_t)RS), g((size_t)RS + 1, Hc(0.0, 0.0));
        g[0] = Hc(beta, 0.0);
        int k = 0;          // the basis vectors in use
        for (int j = 0; j < RS && used < max_solves; j++) {
            T *vn = V + (size_t)(j + 1) * n;
            if ((rc = resid(V + (size_t)j * n, zero, vn, nullptr))) return rc;      // vn = -op(A) v_j
            if ((rc = dev_solve(P, D, N, vn, 1, trans, err, errlen))) return rc;
            used++;
            if ((rc = update(V, 0, none, vn, -1.0))) return rc;                  // vn = M^-1 op(A) v_j
            if ((rc = dots(V, j + 1, vn, hh)) || (rc = update(V, j + 1, hh, vn, 1.0))) return rc;
            if ((rc = dots(V, j + 1, vn, h2)) || (rc = update(V, j + 1, h2, vn, 1.0))) return rc;
            std::vector<Hc> &Hj = H[(size_t)j];
            for (int i = 0; i <= j; i++) Hj[(size_t)i] = hh[(size_t)i] + h2[(size_t)i];
            std::vector<Hc> nn;
            if ((rc = dots(vn, 1, vn, nn))) return rc;
            const double hn = std::sqrt(std::max(nn[0].real(), 0.0));
            Hj[(size_t)j + 1] = Hc(hn, 0.0);
            if (hn > 0.0 && (rc = update(V, 0, none, vn, 1.0 / hn))) return rc;
            for (int i = 0; i < j; i++) {      // the earlier rotations
                const Hc a = Hj[(size_t)i], bb = Hj[(size_t)i + 1];
                Hj[(size_t)i] = cs[(size_t)i] * a + sn[(size_t)i] * bb;
                Hj[(size_t)i + 1] = -std::conj(sn[(size_t)i]) * a + cs[(size_t)i] * bb;
            }
            // the rotation that zeroes H(j + 1, j)
            const Hc a = Hj[(size_t)j], bb = Hj[(size_t)j + 1];
            const double aa = std::abs(a), rr = std::hypot(aa, std::abs(bb));
            if (rr == 0.0) { cs[(size_t)j] = 1.0; sn[(size_t)j] = 0.0; }
            else if (aa == 0.0) { cs[(size_t)j] = 0.0; sn[(size_t)j] = std::conj(bb) / std::abs(bb); }
            else { cs[(size_t)j] = aa / rr; sn[(size_t)j] = (a / aa) * std::conj(bb) / rr; }
            Hj[(size_t)j] = cs[(size_t)j] * a + sn[(size_t)j] * bb;
            Hj[(size_t)j + 1] = 0.0;
            g[(size_t)j + 1] = -std::conj(sn[(size_t)j]) * g[(size_t)j];
            g[(size_t)j] = cs[(size_t)j] * g[(size_t)j];
            k = j + 1;
            if (std::abs(g[(size_t)j + 1]) <= GM_INNER_TOL * beta || hn == 0.0) break;
        }
        if (k == 0) break;
        // y = H(0:k, 0:k) \ g(0:k); w = V y; x += w
        std::vector<Hc> y((size_t)k);
        for (int i = k - 1; i >= 0; i--) {
            Hc t = g[(size_t)i];
            for (int c = i + 1; c < k; c++) t -= H[(size_t)c][(size_t)i] * y[(size_t)c];
            y[(size_t)i] = t / H[(size_t)i][(size_t)i];
        }
        for (auto &v : y) v = -v;
        CK(cudaMemsetAsync(w, 0, (size_t)n * sizeof(T), s));
        if ((rc = update(V, k, y, w, 1.0))) return rc;
        k_axpy1<T><<<nblk(n), 256, 0, s>>>(x, w, n, 0), note_launch();
        double e2 = 0.0;
        if ((rc = resid(x, b, r, &e2))) return rc;
        if (!(e2 < e)) {                          // no progress: undo the cycle and stop
            k_axpy1<T><<<nblk(n), 256, 0, s>>>(x, w, n, 1), note_launch();
            if ((rc = resid(x, b, r, nullptr))) return rc;
            break;
        }
        e = e2;
    }
    *be = e;
    *solves = used;
    return FPLUS_OK;
}

template <typename T>
static int run_refine(const FrontPlan &P, const DevPlan &D, DevNum &N, void *bh, int64_t ldb, int64_t nrhs, int trans,
                      int max_iter, double tol, double *berr, int *iters, char *err, size_t errlen)
{
    cudaStream_t s = N.stream;
    const int64_t n = N.n, nnz = N.nnz;
    int rc;
    if (!N.rr_p) {
        // B's rows from its columns: row k lists (column l, position of the entry in A's values)
        std::vector<int64_t> Bp((size_t)n + 1), Bi((size_t)(nnz > 0 ? nnz : 1)), Bs((size_t)(nnz > 0 ? nnz : 1));
        CK(cudaMemcpyAsync(Bp.data(), D.Bp, (size_t)(n + 1) * 8, cudaMemcpyDeviceToHost, s));
        if (nnz) {
            CK(cudaMemcpyAsync(Bi.data(), D.Bi, (size_t)nnz * 8, cudaMemcpyDeviceToHost, s));
            CK(cudaMemcpyAsync(Bs.data(), D.Bsrc, (size_t)nnz * 8, cudaMemcpyDeviceToHost, s));
        }
        CK(cudaStreamSynchronize(s));
        std::vector<int64_t> rp((size_t)n + 1, 0), rl(Bi.size()), rs(Bi.size());
        for (int64_t e = 0; e < nnz; e++) rp[Bi[e] + 1]++;
        for (int64_t k = 0; k < n; k++) rp[k + 1] += rp[k];
        std::vector<int64_t> fill(rp.begin(), rp.end() - 1);
        for (int64_t l = 0; l < n; l++)
            for (int64_t e = Bp[l]; e < Bp[l + 1]; e++) { const int64_t o = fill[Bi[e]]++; rl[o] = l; rs[o] = Bs[e]; }
        if ((rc = ensure_async(N, (void **)&N.rr_p, &N.cap_rrp, rp.size() * 8, err, errlen)) ||
            (rc = ensure_async(N, (void **)&N.rr_l, &N.cap_rrl, rl.size() * 8, err, errlen)) ||
            (rc = ensure_async(N, (void **)&N.rr_s, &N.cap_rrs, rs.size() * 8, err, errlen)))
            return rc;
        CK(cudaMemcpyAsync(N.rr_p, rp.data(), rp.size() * 8, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(N.rr_l, rl.data(), rl.size() * 8, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(N.rr_s, rs.data(), rs.size() * 8, cudaMemcpyHostToDevice, s));
        CK(cudaStreamSynchronize(s));
    }
    const int64_t g = nrhs < 32 ? nrhs : 32;
    const size_t vb = (size_t)n * (size_t)g * sizeof(T);
    if ((rc = ensure_async(N, &N.ir_b, &N.cap_irb, vb, err, errlen)) || (rc = ensure_async(N, &N.ir_x, &N.cap_irx, vb, err, errlen)) ||
        (rc = ensure_async(N, &N.ir_r, &N.cap_irr, vb, err, errlen)) || (rc = ensure_async(N, &N.ir_d, &N.cap_ird, vb, err, errlen)) ||
        (rc = ensure_async(N, (void **)&N.ir_bits, &N.cap_bits, (size_t)g * 8, err, errlen)))
        return rc;
    T *Bd = (T *)N.ir_b, *X = (T *)N.ir_x, *R = (T *)N.ir_r, *Dd = (T *)N.ir_d;
    const bool t0 = trans == 0;
    const int64_t *ptr = t0 ? N.rr_p : D.Bp, *ix = t0 ? N.rr_l : D.Bi, *src = t0 ? N.rr_s : D.Bsrc;
    const int64_t *outm = t0 ? D.row_perm : D.col_perm, *inm = t0 ? D.col_perm : D.row_perm;
    std::vector<double> cur((size_t)g), prev((size_t)g);
    std::vector<char> want((size_t)g), stopped((size_t)g);
    const int grid = nblk(n * 32);
    for (int64_t r0 = 0; r0 < nrhs; r0 += g) {
        const int64_t m = nrhs - r0 < g ? nrhs - r0 : g;
        char *bb = (char *)bh + (size_t)r0 * (size_t)ldb * sizeof(T);
        CK(cudaMemcpy2DAsync(Bd, (size_t)n * sizeof(T), bb, (size_t)ldb * sizeof(T), (size_t)n * sizeof(T), (size_t)m,
                             cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(X, Bd, (size_t)n * (size_t)m * sizeof(T), cudaMemcpyDeviceToDevice, s));
        if ((rc = dev_solve(P, D, N, X, m, trans, err, errlen))) return rc;
        for (int64_t c = 0; c < m; c++) { iters[r0 + c] = 0; stopped[c] = 0; want[c] = 0; }
        for (int it = 0;; it++) {
            CK(cudaMemsetAsync(N.ir_bits, 0, (size_t)m * 8, s));
            if (trans == 2) k_resid<T, true><<<grid, 256, 0, s>>>(ptr, ix, src, (const T *)N.Ax, outm, inm, X, Bd, R, n, m, N.ir_bits);
            else k_resid<T, false><<<grid, 256, 0, s>>>(ptr, ix, src, (const T *)N.Ax, outm, inm, X, Bd, R, n, m, N.ir_bits);
            note_launch();
            CK(cudaMemcpyAsync(cur.data(), N.ir_bits, (size_t)m * 8, cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            bool any = false;
            for (int64_t c = 0; c < m; c++) {
                if (it > 0 && want[c] && cur[c] > prev[c]) {      // the last correction made it worse: undo it
                    k_axpy1<T><<<nblk(n), 256, 0, s>>>(X + c * n, Dd + c * n, n, 1), note_launch();
                    cur[c] = prev[c];
                    iters[r0 + c]--;
                    stopped[c] = 1;
                }
                // LAPACK's rule (xGERFS): refine while the error is above the target and at least halves
                want[c] = !stopped[c] && it < max_iter && cur[c] > tol && (it == 0 || 2.0 * cur[c] <= prev[c]);
                any = any || want[c];
            }
            for (int64_t c = 0; c < m; c++) berr[r0 + c] = cur[c];
            if (!any) break;
            CK(cudaMemcpyAsync(Dd, R, (size_t)n * (size_t)m * sizeof(T), cudaMemcpyDeviceToDevice, s));
            for (int64_t c = 0; c < m; c++)
                if (!want[c]) CK(cudaMemsetAsync(Dd + c * n, 0, (size_t)n * sizeof(T), s));
                else iters[r0 + c]++;
            if ((rc = dev_solve(P, D, N, Dd, m, trans, err, errlen))) return rc;
            k_axpy1<T><<<nblk(n * m), 256, 0, s>>>(X, Dd, n * m, 0), note_launch();
            prev = cur;
        }
        // classic refinement stalled above the target: GMRES-IR for those right-hand sides, within the same budget of
        // max_iter solves per right-hand side (at least 2 GMRES cycles' worth)
        for (int64_t c = 0; c < m; c++) {
            if (!(berr[r0 + c] > tol) || !std::isfinite(berr[r0 + c])) continue;
            const int budget = max_iter > 0 ? std::max(max_iter, 2 * GM_RESTART + 2) - iters[r0 + c] : 0;
            if (budget <= 0) continue;
            double be = berr[r0 + c];
            int used = 0;
            if ((rc = gmres_ir_column<T>(P, D, N, X + c * n, Bd + c * n, trans, budget, tol, &be, &used, err, errlen))) return rc;
            berr[r0 + c] = be;
            iters[r0 + c] += used;
        }
        CK(cudaMemcpy2DAsync(bb, (size_t)ldb * sizeof(T), X, (size_t)n * sizeof(T), (size_t)n * sizeof(T), (size_t)m,
                             cudaMemcpyDeviceToHost, s));
    }
    CK(cudaStreamSynchronize(s));
    return FPLUS_OK;
}

int dev_solve_refine(const FrontPlan &P, const DevPlan &D, DevNum &N, void *b, int64_t ldb, int64_t nrhs, int trans,
                     int max_iter, double tol, double *berr, int *iters, char *err, size_t errlen)
{
    return N.cplx ? run_refine<cplx>(P, D, N, b, ldb, nrhs, trans, max_iter, tol, berr, iters, err, errlen)
                  : run_refine<double>(P, D, N, b, ldb, nrhs, trans, max_iter, tol, berr, iters, err, errlen);
}

}  // namespace fpl
