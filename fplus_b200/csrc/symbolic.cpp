// symbolic.cpp -- the multifrontal structure (plan.hpp) of the permuted pattern B: column elimination tree, column
// counts of the Cholesky factor of B^T B (the George-Ng bound on the LU structure under any partial pivoting), the
// supernode partition (fundamental, relaxed, width-capped), the front row / column sets, the assembly map of each
// entry of B, the extend-add maps, and the arena / stack offsets.  Everything here depends on the pattern only (and on
// the start of the dense chain), so it is built once per pattern and reused for every set of values.
#include "internal.hpp"
#include "plan.hpp"
#include <algorithm>
#include <cstring>
#include <new>

namespace fpl {

namespace {

// Column counts of the Cholesky factor of C^T C (C: m x n CSC, parent[j] > j) without forming C^T C: the row-subtree
// counting of Gilbert, Ng and Peyton (SIAM J. Matrix Anal. Appl. 15(4), 1994), each row of C assigned to the first of its
// columns in postorder (the "A^T A" form).  cc[j] = entries of column j of the factor, the diagonal included.
void ata_colcounts(int64_t m, int64_t n, const int64_t *Cp, const int64_t *Ci, const int64_t *parent, const int64_t *post,
                   int64_t *cc)
{
    std::vector<int64_t> ipost((size_t)n), first((size_t)n, -1), maxfirst((size_t)n, -1), prevleaf((size_t)n, -1),
        ancestor((size_t)n), delta((size_t)n, 0);
    for (int64_t k = 0; k < n; k++) ipost[post[k]] = k;
    for (int64_t k = 0; k < n; k++) {
        int64_t j = post[k];
        delta[j] = first[j] == -1 ? 1 : 0;
        for (; j != -1 && first[j] == -1; j = parent[j]) first[j] = k;
    }
    // rows of C, each listed under the earliest (in postorder) of its columns
    std::vector<int64_t> Rp((size_t)m + 1, 0), Rj((size_t)Cp[n]);
    for (int64_t q = 0; q < Cp[n]; q++) Rp[Ci[q] + 1]++;
    for (int64_t r = 0; r < m; r++) Rp[r + 1] += Rp[r];
    {
        std::vector<int64_t> fill(Rp.begin(), Rp.end() - 1);
        for (int64_t c = 0; c < n; c++) for (int64_t q = Cp[c]; q < Cp[c + 1]; q++) Rj[fill[Ci[q]]++] = c;
    }
    std::vector<int64_t> head((size_t)n + 1, -1), next((size_t)(m > 0 ? m : 1), -1);
    for (int64_t r = 0; r < m; r++) {
        int64_t k = n;
        for (int64_t q = Rp[r]; q < Rp[r + 1]; q++) k = std::min(k, ipost[Rj[q]]);
        if (k < n) { next[r] = head[k]; head[k] = r; }
    }
    for (int64_t j = 0; j < n; j++) ancestor[j] = j;
    for (int64_t k = 0; k < n; k++) {
        const int64_t j = post[k];
        if (parent[j] != -1) delta[parent[j]]--;
        for (int64_t r = head[k]; r != -1; r = next[r]) {
            for (int64_t q = Rp[r]; q < Rp[r + 1]; q++) {
                const int64_t i = Rj[q];
                // is j a leaf of the row subtree of i?
                if (i <= j || first[j] <= maxfirst[i]) continue;
                maxfirst[i] = first[j];
                const int64_t jprev = prevleaf[i];
                prevleaf[i] = j;
                delta[j]++;
                if (jprev != -1) {
                    int64_t a = jprev;
                    while (a != ancestor[a]) a = ancestor[a];
                    for (int64_t s = jprev; s != a;) { int64_t nx = ancestor[s]; ancestor[s] = a; s = nx; }
                    delta[a]--;       // the least common ancestor of jprev and j
                }
            }
        }
        if (parent[j] != -1) ancestor[j] = parent[j];
    }
    for (int64_t j = 0; j < n; j++) cc[j] = delta[j];
    for (int64_t k = 0; k < n; k++) { int64_t j = post[k]; if (parent[j] != -1) cc[parent[j]] += cc[j]; }
}

struct SN { int64_t first, last, parent; int64_t w, ccf; double tnz; bool alive; };

}  // namespace

int build_plan(const fplus_symbolic_view &S, int64_t f_tail, int64_t nb_chain, int64_t max_width, FrontPlan &P)
{
    try {
    const int64_t n = S.n, ntr = S.ntr, ntc = S.ntc, mi = n - ntr, ni = n - ntc;
    const int64_t *Bp = S.Bp, *Bi = S.Bi;
    P = FrontPlan();
    P.n = n; P.mi = mi; P.ni = ni; P.ntr = ntr; P.ntc = ntc;
    P.nb_chain = nb_chain > 0 ? nb_chain : 64;
    P.max_width = max_width > 0 ? max_width : 256;
    int64_t f_dense = (f_tail >= 0 && f_tail < ni) ? f_tail : ni;
    P.col_front.assign((size_t)n, -1);
    if (n == 0) { P.f_dense = 0; return 0; }

    // the interior pattern C = B[0:mi, 0:ni] (rows ascending in each column of B, so a prefix of each column)
    std::vector<int64_t> Cp((size_t)ni + 1, 0), Ci;
    Ci.reserve((size_t)Bp[ni]);
    for (int64_t j = 0; j < ni; j++) {
        for (int64_t q = Bp[j]; q < Bp[j + 1] && Bi[q] < mi; q++) Ci.push_back(Bi[q]);
        Cp[j + 1] = (int64_t)Ci.size();
    }
    std::vector<int64_t> parent((size_t)(ni > 0 ? ni : 1)), post((size_t)(ni > 0 ? ni : 1)), cc((size_t)(ni > 0 ? ni : 1));
    coletree(mi, ni, Cp.data(), Ci.data(), parent.data());
    tree_postorder(ni, parent.data(), post.data());
    ata_colcounts(mi, ni, Cp.data(), Ci.data(), parent.data(), post.data(), cc.data());

    // first column of each row of B (interior columns first; n for an empty row)
    std::vector<int64_t> firstcol((size_t)n, n);
    for (int64_t j = 0; j < n; j++)
        for (int64_t q = Bp[j]; q < Bp[j + 1]; q++) if (j < firstcol[Bi[q]]) firstcol[Bi[q]] = j;
    // rows of B (CSR): entry index per (row, column)
    std::vector<int64_t> Rp((size_t)n + 1, 0), Rc((size_t)Bp[n]), Rq((size_t)Bp[n]);
    for (int64_t q = 0; q < Bp[n]; q++) Rp[Bi[q] + 1]++;
    for (int64_t r = 0; r < n; r++) Rp[r + 1] += Rp[r];
    {
        std::vector<int64_t> fill(Rp.begin(), Rp.end() - 1);
        for (int64_t j = 0; j < n; j++) for (int64_t q = Bp[j]; q < Bp[j + 1]; q++) { int64_t o = fill[Bi[q]]++; Rc[o] = j; Rq[o] = q; }
    }

    // ---- supernodes of the interior columns [0, f_dense): fundamental, then relaxed (CHOLMOD-style amalgamation
    // bounds: width <= 4 always, <= 16 with < 80% zeros, <= 48 with < 10%, any width with < 5%), width-capped
    std::vector<int64_t> nchild((size_t)(ni > 0 ? ni : 1), 0);
    for (int64_t j = 0; j < ni; j++) if (parent[j] >= 0) nchild[parent[j]]++;
    std::vector<SN> sn;
    std::vector<int64_t> col2sn((size_t)(ni > 0 ? ni : 1), -1);
    for (int64_t j = 0; j < f_dense; j++) {
        bool cont = j > 0 && !sn.empty() && parent[j - 1] == j && nchild[j] == 1 && cc[j - 1] == cc[j] + 1 &&
                    (j - sn.back().first) < P.max_width;
        if (!cont) sn.push_back(SN{j, j, -1, 0, cc[j], 0.0, true});
        SN &s = sn.back();
        s.last = j; s.w = j - s.first + 1; s.tnz += (double)cc[j];
        col2sn[j] = (int64_t)sn.size() - 1;
    }
    const int64_t ns0 = (int64_t)sn.size();
    for (int64_t s = 0; s < ns0; s++) {
        int64_t pc = parent[sn[s].last];
        sn[s].parent = (pc >= 0 && pc < f_dense) ? col2sn[pc] : -1;
    }
    // relaxed merges: a supernode absorbs its last child (the one ending just before it) while the rule holds
    std::vector<int64_t> rep((size_t)(ns0 > 0 ? ns0 : 1));
    for (int64_t s = 0; s < ns0; s++) rep[s] = s;
    auto find = [&](int64_t x) { while (rep[x] != x) { rep[x] = rep[rep[x]]; x = rep[x]; } return x; };
    for (int64_t p = 0; p < ns0; p++) {
        for (;;) {
            SN &Pn = sn[p];
            if (Pn.first == 0) break;
            int64_t s = find(col2sn[Pn.first - 1]);
            if (s == p || !sn[s].alive) break;
            int64_t sp = sn[s].parent >= 0 ? find(sn[s].parent) : -1;
            if (sp != p) break;
            const int64_t w = sn[s].w + Pn.w;
            if (w > P.max_width) break;
            const int64_t ccf = sn[s].w + Pn.ccf;
            const double stored = (double)w * (double)ccf - (double)w * (double)(w - 1) / 2.0;
            const double tnz = sn[s].tnz + Pn.tnz;
            const double z = stored > 0 ? (stored - tnz) / stored : 0.0;
            const bool ok = w <= 4 || (w <= 16 && z < 0.8) || (w <= 48 && z < 0.1) || z < 0.05;
            if (!ok) break;
            Pn.first = sn[s].first; Pn.w = w; Pn.ccf = ccf; Pn.tnz = tnz;
            sn[s].alive = false;
            rep[s] = p;
        }
    }
    std::vector<int64_t> snmap((size_t)(ns0 > 0 ? ns0 : 1), -1);
    std::vector<SN> sup;
    for (int64_t s = 0; s < ns0; s++) if (sn[s].alive) { snmap[s] = (int64_t)sup.size(); sup.push_back(sn[s]); }
    for (auto &s : sup) s.parent = s.parent >= 0 ? snmap[find(s.parent)] : -1;
    const int64_t nsup = (int64_t)sup.size();

    // ---- the dense chain
    const int64_t nb = P.nb_chain;
    const int64_t nchain = f_dense < n ? (n - f_dense + nb - 1) / nb : 0;
    P.f_dense = f_dense;
    const int64_t nfront = nsup + nchain;
    P.fronts.resize((size_t)nfront);
    // rows entering each front
    std::vector<std::vector<int64_t>> enter((size_t)nfront);
    std::vector<int64_t> colfront((size_t)n, -1);
    for (int64_t s = 0; s < nsup; s++) for (int64_t j = sup[s].first; j <= sup[s].last; j++) colfront[j] = s;
    for (int64_t b = 0; b < nchain; b++) {
        const int64_t s0 = f_dense + b * nb, e0 = std::min(s0 + nb, n);
        for (int64_t j = s0; j < e0; j++) colfront[j] = nsup + b;
    }
    for (int64_t r = 0; r < mi; r++) if (firstcol[r] < n) enter[colfront[firstcol[r]]].push_back(r);
    P.col_front = colfront;

    // parents and children
    for (int64_t s = 0; s < nsup; s++) {
        Front &F = P.fronts[s];
        F.f = sup[s].first; F.npiv = sup[s].w;
        // the etree parent's front, or (a root, or a parent in the chain) the first chain front
        F.parent = sup[s].parent >= 0 ? sup[s].parent : (nchain > 0 ? nsup : -1);
    }
    for (int64_t b = 0; b < nchain; b++) {
        Front &F = P.fronts[nsup + b];
        F.f = f_dense + b * nb; F.npiv = std::min(nb, n - F.f); F.dense = 1;
        F.parent = b + 1 < nchain ? nsup + b + 1 : -1;
    }
    std::vector<std::vector<int64_t>> kids((size_t)nfront);
    for (int64_t s = 0; s < nfront; s++) if (P.fronts[s].parent >= 0) kids[P.fronts[s].parent].push_back(s);

    // ---- column sets, row counts, local row layout, assembly map
    std::vector<int64_t> mark((size_t)n, -1), pos((size_t)n, -1);
    std::vector<int64_t> tmp;
    for (int64_t s = 0; s < nfront; s++) {
        Front &F = P.fronts[s];
        const int64_t fl = F.f + F.npiv;     // one past the last pivot column
        // columns
        F.col_off = (int64_t)P.cols.size();
        if (F.dense) {
            for (int64_t c = F.f; c < n; c++) P.cols.push_back(c);
        } else {
            tmp.clear();
            for (int64_t c = F.f; c < fl; c++) mark[c] = s;
            for (int64_t r : enter[s])
                for (int64_t t = Rp[r]; t < Rp[r + 1]; t++) { int64_t c = Rc[t]; if (c < ni && mark[c] != s) { mark[c] = s; tmp.push_back(c); } }
            for (int64_t g : kids[s]) {
                const Front &G = P.fronts[g];
                for (int64_t t = G.npiv; t < G.ncols; t++) { int64_t c = P.cols[G.col_off + t]; if (c < ni && mark[c] != s) { mark[c] = s; tmp.push_back(c); } }
            }
            std::sort(tmp.begin(), tmp.end());
            for (int64_t c = F.f; c < fl; c++) P.cols.push_back(c);
            for (int64_t c : tmp) P.cols.push_back(c);
            for (int64_t c = ni; c < n; c++) P.cols.push_back(c);
        }
        F.ncols = (int64_t)P.cols.size() - F.col_off;
        for (int64_t t = 0; t < F.ncols; t++) pos[P.cols[F.col_off + t]] = t;
        // rows: entering rows | each child's interior CB rows | dense rows (border rows of an interior front; ordinary
        // rows of the first chain front)
        const bool tau_here = F.dense ? (s == nsup) : true;
        int64_t nr = (int64_t)enter[s].size();
        for (int64_t g : kids[s]) { Front &G = P.fronts[g]; G.slot = nr; nr += std::max<int64_t>(0, G.nri - G.npiv); }
        const int64_t tau_base = nr;
        F.tau_base = tau_base;
        if (tau_here) nr += ntr;
        F.nrows = nr;
        F.nbord = F.dense ? 0 : ntr;
        F.nri = F.nrows - F.nbord;
        F.row_off = (int64_t)P.rowinit.size();
        for (int64_t r : enter[s]) P.rowinit.push_back(r);
        for (int64_t g : kids[s]) { const Front &G = P.fronts[g]; for (int64_t t = 0; t < G.nri - G.npiv; t++) P.rowinit.push_back(-1); }
        F.nbord = std::min(F.nbord, F.nrows);
        if (tau_here) for (int64_t t = 0; t < ntr; t++) P.rowinit.push_back(mi + t);
        // extend-add column maps of the children
        F.child_begin = (int64_t)P.children.size();
        for (int64_t g : kids[s]) {
            Front &G = P.fronts[g];
            P.children.push_back(g);
            G.relcol_off = (int64_t)P.relcol.size();
            for (int64_t t = G.npiv; t < G.ncols; t++) P.relcol.push_back(pos[P.cols[G.col_off + t]]);
        }
        F.child_end = (int64_t)P.children.size();
        // assembly: entering rows whole; dense rows in this front's pivot columns (interior front) or in all its
        // columns (first chain front)
        F.asm_begin = (int64_t)P.asm_src.size();
        for (size_t k = 0; k < enter[s].size(); k++) {
            const int64_t r = enter[s][k];
            for (int64_t t = Rp[r]; t < Rp[r + 1]; t++) {
                P.asm_src.push_back(Rq[t]);
                P.asm_dst.push_back(pos[Rc[t]] * F.nrows + (int64_t)k);
            }
        }
        if (ntr > 0 && tau_here) {
            const int64_t c1 = F.dense ? n : fl;
            for (int64_t c = F.f; c < c1; c++)
                for (int64_t q = Bp[c + 1] - 1; q >= Bp[c] && Bi[q] >= mi; q--) {
                    P.asm_src.push_back(q);
                    P.asm_dst.push_back(pos[c] * F.nrows + tau_base + (Bi[q] - mi));
                }
        }
        F.asm_end = (int64_t)P.asm_src.size();
        {   // the pivot-column entries first (a stable partition), so that the pivot block can be assembled on its own
            std::vector<std::pair<int64_t, int64_t>> head, tail;
            for (int64_t q = F.asm_begin; q < F.asm_end; q++) {
                auto e = std::make_pair(P.asm_src[q], P.asm_dst[q]);
                (P.asm_dst[q] / F.nrows < F.npiv ? head : tail).push_back(e);
            }
            int64_t q = F.asm_begin;
            for (auto &e : head) { P.asm_src[q] = e.first; P.asm_dst[q] = e.second; q++; }
            F.asm_mid = q;
            for (auto &e : tail) { P.asm_src[q] = e.first; P.asm_dst[q] = e.second; q++; }
        }
        for (int64_t t = 0; t < F.ncols; t++) pos[P.cols[F.col_off + t]] = -1;
        // levels
        int lv = 0;
        for (int64_t g : kids[s]) lv = std::max(lv, P.fronts[g].level + 1);
        F.level = lv;
        P.nlevels = std::max(P.nlevels, lv + 1);
        // sizes
        P.max_nrows = std::max(P.max_nrows, F.nrows);
        P.max_ncols = std::max(P.max_ncols, F.ncols);
        P.max_npiv = std::max(P.max_npiv, F.npiv);
        P.work_size = std::max(P.work_size, F.nrows * F.ncols);
        for (int64_t k = 0; k < F.npiv; k++) {
            const double a = (double)(F.nrows - k - 1), b = (double)(F.ncols - k - 1);
            if (a > 0) P.flops_real += a * (b > 0 ? b : 0) + a;
        }
    }
    P.rows_total = (int64_t)P.rowinit.size();
    P.head_cols.assign(P.fronts.size(), 0);
    for (size_t g = 0; g < P.fronts.size(); g++) {
        const Front &G = P.fronts[g];
        if (G.parent < 0) continue;
        const int64_t ncb = G.ncols - G.npiv, pnp = P.fronts[(size_t)G.parent].npiv;
        int64_t h = 0;
        while (h < ncb && P.relcol[G.relcol_off + h] < pnp) h++;
        for (int64_t c = h; c < ncb && h >= 0; c++) if (P.relcol[G.relcol_off + c] < pnp) h = -1;
        P.head_cols[g] = h;
    }

    // ---- factor arena and the CB stack (children's CBs are popped by the parent, in processing order)
    int64_t lo = 0, uo = 0;
    for (auto &F : P.fronts) { F.L_off = lo; F.U_off = uo; lo += F.nrows * F.npiv; uo += F.npiv * (F.ncols - F.npiv); }
    P.L_size = lo; P.U_size = uo;
    {
        std::vector<int64_t> stk;       // front ids
        int64_t top = 0, peak = 0;
        bool ok = true;
        for (int64_t s = 0; s < nfront && ok; s++) {
            Front &F = P.fronts[s];
            for (int64_t k = F.child_end - 1; k >= F.child_begin; k--) {
                int64_t g = P.children[k];
                if (stk.empty() || stk.back() != g) { ok = false; break; }
                stk.pop_back();
                top = P.fronts[g].cb_off;
            }
            if (!ok) break;
            const int64_t cbs = std::max<int64_t>(0, F.nrows - F.npiv) * (F.ncols - F.npiv);
            F.cb_off = top;
            if (F.parent >= 0) { stk.push_back(s); top += cbs; peak = std::max(peak, top); }
        }
        if (!ok) {      // not a postorder: every CB in its own place
            int64_t o = 0;
            for (auto &F : P.fronts) { F.cb_off = o; o += std::max<int64_t>(0, F.nrows - F.npiv) * (F.ncols - F.npiv); }
            peak = o;
        }
        P.cb_size = peak;
    }
    } catch (const std::bad_alloc &) {
        return -1;
    }
    return 0;
}

}  // namespace fpl
