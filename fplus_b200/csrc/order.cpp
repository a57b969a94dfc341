// order.cpp -- the symbolic analysis on the host: dense-line pinning, the fill-reducing column order, the column-etree
// postorder (FPLUS src/order.c:259-399), and the input checks (FPLUS src/fplus_internal.h:147-182).
#include "internal.hpp"
#include <algorithm>
#include <cstring>
#include <cmath>
#include <thread>
#include <vector>

namespace fpl {

void errf(char *err, size_t errlen, const char *fmt, ...)
{
    if (!err || errlen == 0) return;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, errlen, fmt, ap);
    va_end(ap);
}

int check_compressed(int64_t n, const int64_t *ptr, const int64_t *idx, int canonical, char *err, size_t errlen)
{
    if (n < 0) { errf(err, errlen, "n must be >= 0 (got %ld)", (long)n); return FPLUS_ERR_BADARG; }
    if (!ptr || (n > 0 && !idx && ptr[n] > 0)) { errf(err, errlen, "NULL index array"); return FPLUS_ERR_BADARG; }
    if (ptr[0] != 0) { errf(err, errlen, "indptr[0] must be 0 (got %ld)", (long)ptr[0]); return FPLUS_ERR_BADARG; }
    for (int64_t j = 0; j < n; j++) {
        if (ptr[j + 1] < ptr[j]) { errf(err, errlen, "indptr decreases at %ld", (long)j); return FPLUS_ERR_BADARG; }
        for (int64_t q = ptr[j]; q < ptr[j + 1]; q++) {
            if (idx[q] < 0 || idx[q] >= n) {
                errf(err, errlen, "index %ld out of range [0, %ld) in line %ld", (long)idx[q], (long)n, (long)j);
                return FPLUS_ERR_BADARG;
            }
            if (canonical && q > ptr[j] && idx[q] <= idx[q - 1]) {
                errf(err, errlen, "indices not strictly increasing in line %ld (canonical form required: sorted, no duplicates)", (long)j);
                return FPLUS_ERR_BADARG;
            }
        }
    }
    return FPLUS_OK;
}

// whether any of d[0 .. m) is infinite or NaN (its exponent bits all ones), without an early exit
static bool any_nonfinite(const double *d, int64_t m)
{
    const uint64_t E = 0x7ff0000000000000ull;
    uint64_t f0 = 0, f1 = 0, f2 = 0, f3 = 0;
    int64_t k = 0;
    for (; k + 4 <= m; k += 4) {
        uint64_t b[4];
        std::memcpy(b, d + k, sizeof b);
        f0 |= (uint64_t)((b[0] & E) == E); f1 |= (uint64_t)((b[1] & E) == E);
        f2 |= (uint64_t)((b[2] & E) == E); f3 |= (uint64_t)((b[3] & E) == E);
    }
    for (; k < m; k++) { uint64_t b; std::memcpy(&b, d + k, 8); f0 |= (uint64_t)((b & E) == E); }
    return (f0 | f1 | f2 | f3) != 0;
}

// Every value finite, else the first entry that is not (the error names it).  Large arrays are first scanned for any
// non-finite value by up to 8 host threads; only then is the first one located, serially.
int check_finite(int64_t nnz, const void *x, int is_complex, char *err, size_t errlen)
{
    const double *d = (const double *)x;
    const int64_t m = is_complex ? 2 * nnz : nnz;
    if (m > 0 && !d) { errf(err, errlen, "NULL value array"); return FPLUS_ERR_BADARG; }
    bool bad = false;
    const unsigned hc = std::thread::hardware_concurrency();
    const int nt = m >= (int64_t)1 << 20 ? (int)std::min<unsigned>(8u, hc > 1 ? hc : 1u) : 1;
    if (nt > 1) {
        std::vector<char> r((size_t)nt, 0);
        std::vector<std::thread> th;
        bool all = true;                                   // every chunk has its thread
        try {
            for (int t = 1; t < nt; t++)
                th.emplace_back([&r, d, m, nt, t]() { const int64_t a = m * t / nt, b = m * (t + 1) / nt; r[(size_t)t] = any_nonfinite(d + a, b - a); });
        } catch (...) {
            all = false;
        }
        r[0] = any_nonfinite(d, m / nt);                   // chunk 0 on this thread
        for (std::thread &x : th) x.join();
        if (!all) bad = any_nonfinite(d, m);               // (threads could not be had: one pass over everything)
        else for (char v : r) bad = bad || v;
    } else
        bad = any_nonfinite(d, m);
    if (!bad) return FPLUS_OK;
    for (int64_t k = 0; k < m; k++)
        if (!std::isfinite(d[k])) { errf(err, errlen, "non-finite value in entry %ld", (long)(is_complex ? k / 2 : k)); return FPLUS_ERR_BADARG; }
    return FPLUS_OK;
}

int check_perm(int64_t n, const int64_t *p, const char *name, char *err, size_t errlen)
{
    std::vector<unsigned char> seen((size_t)(n > 0 ? n : 1), 0);
    for (int64_t i = 0; i < n; i++) {
        if (p[i] < 0 || p[i] >= n || seen[(size_t)p[i]]) {
            errf(err, errlen, "%s is not a permutation of 0..n-1 (entry %ld)", name, (long)i);
            return FPLUS_ERR_BADARG;
        }
        seen[(size_t)p[i]] = 1;
    }
    return FPLUS_OK;
}

// ---------------------------------------------------------------------------------------------------------------------
// Column elimination tree: the elimination tree of C^T C without forming it (Liu's algorithm on the row-merged graph, each
// row represented by its first column; disjoint sets with path compression).  The tree is unique, so is its postorder with
// children in increasing order: the same output as FPLUS src/order.c:21-62.
void coletree(int64_t m, int64_t n, const int64_t *Cp, const int64_t *Ci, int64_t *parent)
{
    std::vector<int64_t> firstcol((size_t)(m > 0 ? m : 1), n), set((size_t)(n > 0 ? n : 1)), top((size_t)(n > 0 ? n : 1));
    for (int64_t c = 0; c < n; c++)
        for (int64_t q = Cp[c]; q < Cp[c + 1]; q++) { int64_t r = Ci[q]; if (r >= 0 && r < m && c < firstcol[r]) firstcol[r] = c; }
    auto find = [&](int64_t x) {
        int64_t r = x;
        while (set[r] != r) r = set[r];
        while (set[x] != r) { int64_t nx = set[x]; set[x] = r; x = nx; }
        return r;
    };
    for (int64_t c = 0; c < n; c++) {
        set[c] = c; top[c] = c; parent[c] = -1;
        for (int64_t q = Cp[c]; q < Cp[c + 1]; q++) {
            int64_t r = Ci[q];
            if (r < 0 || r >= m) continue;
            int64_t f = firstcol[r];
            if (f >= c) continue;
            int64_t s = find(f), t = top[s];
            if (t != c) { parent[t] = c; set[s] = c; top[c] = c; }
        }
    }
}

void tree_postorder(int64_t n, const int64_t *parent, int64_t *post)
{
    std::vector<int64_t> head((size_t)n + 1, -1), next((size_t)(n > 0 ? n : 1), -1), stack((size_t)n + 1);
    for (int64_t v = n - 1; v >= 0; v--) { int64_t p = parent[v] < 0 ? n : parent[v]; next[v] = head[p]; head[p] = v; }
    int64_t k = 0, sp = 0;
    stack[0] = n;
    while (sp >= 0) {
        int64_t v = stack[sp], c = head[v];
        if (c >= 0) { head[v] = next[c]; stack[++sp] = c; }
        else { sp--; if (v < n) post[k++] = v; }
    }
}

// ---------------------------------------------------------------------------------------------------------------------
// Minimum degree on the column intersection graph (COLAMD's setting: Davis, Gilbert, Larimore, Ng, ACM TOMS 30(3), 2004;
// approximate degrees as in AMD: Amestoy, Davis, Duff, SIAM J. Matrix Anal. Appl. 17(4), 1996).  Variables are the
// columns; the initial elements are the rows (each row is a clique of C^T C).  Eliminating a variable p merges the elements
// adjacent to p into a new element L_p; the degree of each variable of L_p is updated with AMD's approximate external
// degree; variables with identical adjacency (supervariables) are merged and eliminated together; elements contained in
// L_p are absorbed.
namespace {
struct MinDeg {
    int64_t n;
    std::vector<std::vector<int64_t>> elems;   // per variable: adjacent elements (element ids; may hold stale ids)
    std::vector<std::vector<int64_t>> evars;   // per element: its variables (may hold eliminated / merged variables)
    std::vector<int64_t> nv;                   // supervariable size (0: merged into another or eliminated)
    std::vector<int64_t> deg;                  // approximate external degree
    std::vector<char> is_elim;                 // variable eliminated
    std::vector<char> e_dead;                  // element absorbed
    std::vector<int64_t> w;                    // |L_e \ L_p| workspace (AMD's w), stamped
    std::vector<int64_t> wstamp;
    std::vector<int64_t> mark;                 // variable marker
    std::vector<int64_t> head, nxt, prv;       // degree buckets
    std::vector<std::vector<int64_t>> members; // variables merged into a supervariable (eliminated with it)
    int64_t mindeg = 0, stamp = 0;

    void bucket_insert(int64_t i) {
        int64_t d = deg[i];
        prv[i] = -1; nxt[i] = head[d]; if (head[d] >= 0) prv[head[d]] = i; head[d] = i;
        if (d < mindeg) mindeg = d;
    }
    void bucket_remove(int64_t i) {
        int64_t d = deg[i];
        if (prv[i] >= 0) nxt[prv[i]] = nxt[i]; else head[d] = nxt[i];
        if (nxt[i] >= 0) prv[nxt[i]] = prv[i];
        prv[i] = nxt[i] = -1;
    }
};
}  // namespace

void colamd_order(int64_t m, int64_t ncol, const int64_t *Cp, const int64_t *Ci, int64_t *perm)
{
    const int64_t n = ncol;
    MinDeg G;
    G.n = n;
    G.elems.assign((size_t)n, {});
    G.nv.assign((size_t)n, 1);
    G.deg.assign((size_t)n, 0);
    G.is_elim.assign((size_t)n, 0);
    G.mark.assign((size_t)n, 0);
    G.head.assign((size_t)n + 1, -1);
    G.nxt.assign((size_t)n, -1);
    G.prv.assign((size_t)n, -1);
    G.members.assign((size_t)n, {});
    // rows of C -> elements (rows with fewer than two entries add no edge and are dropped)
    std::vector<int64_t> rcnt((size_t)(m > 0 ? m : 1), 0);
    for (int64_t q = 0; q < Cp[n]; q++) rcnt[Ci[q]]++;
    std::vector<int64_t> eid((size_t)(m > 0 ? m : 1), -1);
    int64_t ne = 0;
    for (int64_t r = 0; r < m; r++) if (rcnt[r] >= 2) eid[r] = ne++;
    G.evars.assign((size_t)(ne + n), {});       // row elements, then one element per eliminated pivot
    for (int64_t r = 0; r < m; r++) if (eid[r] >= 0) G.evars[eid[r]].reserve(rcnt[r]);
    for (int64_t c = 0; c < n; c++)
        for (int64_t q = Cp[c]; q < Cp[c + 1]; q++) {
            int64_t e = eid[Ci[q]];
            if (e < 0) continue;
            G.evars[e].push_back(c);
            G.elems[c].push_back(e);
        }
    G.e_dead.assign((size_t)(ne + n), 0);
    G.w.assign((size_t)(ne + n), 0);
    G.wstamp.assign((size_t)(ne + n), -1);
    // initial degrees: |union of the rows of c| - 1
    std::vector<char> empty((size_t)n, 0);
    int64_t nempty = 0;
    for (int64_t c = 0; c < n; c++) {
        if (G.elems[c].empty() && Cp[c + 1] == Cp[c]) { empty[c] = 1; nempty++; }
    }
    {
        int64_t st = 0;
        for (int64_t c = 0; c < n; c++) {
            if (empty[c]) continue;
            st++;
            int64_t d = 0;
            G.mark[c] = -st;
            for (int64_t e : G.elems[c])
                for (int64_t v : G.evars[e]) if (G.mark[v] != -st) { G.mark[v] = -st; d++; }
            G.deg[c] = std::min<int64_t>(d, n - 1);
        }
        std::fill(G.mark.begin(), G.mark.end(), 0);
    }
    for (int64_t c = n - 1; c >= 0; c--) if (!empty[c]) G.bucket_insert(c);
    G.mindeg = 0;
    int64_t k = 0;                  // variables ordered so far
    const int64_t nlive = n - nempty;
    std::vector<int64_t> Lp;        // the new element's variables
    std::vector<int64_t> hashv;
    std::vector<int64_t> order;
    order.reserve((size_t)n);
    int64_t tagbase = 1;
    int64_t next_elem = ne;
    while (k < nlive) {
        // select the variable of minimum approximate degree
        while (G.mindeg <= n && (G.mindeg >= (int64_t)G.head.size() || G.head[G.mindeg] < 0)) G.mindeg++;
        if (G.mindeg > n) break;
        const int64_t p = G.head[G.mindeg];
        G.bucket_remove(p);
        const int64_t pe = next_elem++;        // p becomes element pe
        // L_p = union of the variables of p's elements, minus p
        tagbase++;
        const int64_t tag = tagbase;
        Lp.clear();
        G.mark[p] = tag;
        for (int64_t e : G.elems[p]) {
            if (G.e_dead[e]) continue;
            for (int64_t v : G.evars[e]) {
                if (G.is_elim[v] || G.nv[v] == 0 || G.mark[v] == tag) continue;
                G.mark[v] = tag;
                Lp.push_back(v);
            }
            G.e_dead[e] = 1;                   // absorbed into pe
            std::vector<int64_t>().swap(G.evars[e]);
        }
        G.is_elim[p] = 1;
        order.push_back(p);
        k += G.nv[p];
        for (int64_t v : G.members[p]) order.push_back(v);
        std::vector<int64_t>().swap(G.members[p]);
        std::vector<int64_t>().swap(G.elems[p]);
        int64_t lp_weight = 0;
        for (int64_t v : Lp) lp_weight += G.nv[v];
        G.evars[pe] = Lp;
        // |L_e \ L_p| for the elements adjacent to L_p (AMD's w)
        for (int64_t v : Lp) {
            for (int64_t e : G.elems[v]) {
                if (G.e_dead[e]) continue;
                if (G.wstamp[e] != tag) {
                    G.wstamp[e] = tag;
                    int64_t sz = 0;
                    for (int64_t u : G.evars[e]) if (!G.is_elim[u] && G.nv[u] > 0) sz += G.nv[u];
                    G.w[e] = sz;
                }
                G.w[e] -= G.nv[v];
            }
        }
        // update each variable of L_p: drop absorbed elements, add pe, approximate degree, hash
        hashv.assign(Lp.size(), 0);
        for (size_t t = 0; t < Lp.size(); t++) {
            const int64_t v = Lp[t];
            G.bucket_remove(v);
            auto &E = G.elems[v];
            size_t o = 0;
            int64_t ext = 0;
            int64_t h = 0;
            for (size_t s = 0; s < E.size(); s++) {
                int64_t e = E[s];
                if (G.e_dead[e]) continue;
                if (G.w[e] <= 0) { G.e_dead[e] = 1; std::vector<int64_t>().swap(G.evars[e]); continue; }  // e inside L_p
                E[o++] = e;
                ext += G.w[e];
                h += e;
            }
            E.resize(o);
            E.push_back(pe);
            h += pe;
            const int64_t dold = G.deg[v];
            int64_t d = std::min<int64_t>({(int64_t)(n - k), dold + lp_weight - G.nv[v], lp_weight - G.nv[v] + ext});
            G.deg[v] = d < 0 ? 0 : d;
            hashv[t] = h;
        }
        // supervariables: variables of L_p with identical element lists
        {
            std::vector<size_t> idx(Lp.size());
            for (size_t t = 0; t < idx.size(); t++) idx[t] = t;
            std::sort(idx.begin(), idx.end(), [&](size_t a, size_t b) {
                if (hashv[a] != hashv[b]) return hashv[a] < hashv[b];
                return Lp[a] < Lp[b];
            });
            for (size_t s = 0; s < idx.size();) {
                size_t e = s + 1;
                while (e < idx.size() && hashv[idx[e]] == hashv[idx[s]]) e++;
                for (size_t a = s; a < e; a++) {
                    int64_t va = Lp[idx[a]];
                    if (G.nv[va] == 0) continue;
                    auto &Ea = G.elems[va];
                    std::sort(Ea.begin(), Ea.end());
                    for (size_t b = a + 1; b < e; b++) {
                        int64_t vb = Lp[idx[b]];
                        if (G.nv[vb] == 0) continue;
                        auto &Eb = G.elems[vb];
                        if (Eb.size() != Ea.size()) continue;
                        std::sort(Eb.begin(), Eb.end());
                        if (Eb != Ea) continue;
                        // merge vb into va: vb is no longer external to va
                        const int64_t wb = G.nv[vb];
                        G.nv[va] += wb;
                        G.members[va].push_back(vb);
                        for (int64_t u : G.members[vb]) G.members[va].push_back(u);
                        std::vector<int64_t>().swap(G.members[vb]);
                        G.nv[vb] = 0;
                        std::vector<int64_t>().swap(Eb);
                        G.deg[va] = std::max<int64_t>(0, G.deg[va] - wb);
                    }
                }
                s = e;
            }
        }
        // compact L_p and reinsert
        {
            size_t o = 0;
            for (int64_t v : Lp) if (G.nv[v] > 0) Lp[o++] = v;
            Lp.resize(o);
            G.evars[pe] = Lp;
            for (int64_t v : Lp) {
                int64_t d = G.deg[v];
                int64_t lim = n - k - G.nv[v];
                if (d > lim) d = lim;
                if (d < 0) d = 0;
                G.deg[v] = d;
                G.bucket_insert(v);
            }
            if (Lp.empty()) G.e_dead[pe] = 1;
        }
    }
    // any variable left (should not happen), then the empty columns
    for (int64_t c = 0; c < n; c++) if (!empty[c] && !G.is_elim[c] && G.nv[c] > 0) {
        order.push_back(c);
        for (int64_t v : G.members[c]) order.push_back(v);
    }
    for (int64_t c = 0; c < n; c++) if (empty[c]) order.push_back(c);
    // guard: a permutation of 0..n-1
    std::vector<char> seen((size_t)n, 0);
    int64_t o = 0;
    for (int64_t v : order) if (v >= 0 && v < n && !seen[v]) { seen[v] = 1; perm[o++] = v; }
    for (int64_t c = 0; c < n; c++) if (!seen[c]) perm[o++] = c;
}

}  // namespace fpl

// ---------------------------------------------------------------------------------------------------------------------
// public entry points of the analysis

using namespace fpl;

extern "C" int fplus_coletree_postorder(int64_t m, int64_t n, const int64_t *Ap, const int64_t *Ai, int64_t *post)
{
    if (m < 0 || n < 0 || !Ap || !post) return FPLUS_ERR_BADARG;
    std::vector<int64_t> parent((size_t)(n > 0 ? n : 1));
    coletree(m, n, Ap, Ai, parent.data());
    tree_postorder(n, parent.data(), post);
    return FPLUS_OK;
}

extern "C" void fplus_symbolic_free(fplus_symbolic *sym) { delete sym; }
extern "C" int64_t fplus_symbolic_n(const fplus_symbolic *sym) { return sym->n; }
extern "C" int64_t fplus_symbolic_nnz(const fplus_symbolic *sym) { return sym->nnz; }
extern "C" const int64_t *fplus_symbolic_row_perm(const fplus_symbolic *sym) { return sym->row_perm.data(); }
extern "C" const int64_t *fplus_symbolic_col_perm(const fplus_symbolic *sym) { return sym->col_perm.data(); }
extern "C" int64_t fplus_symbolic_n_dense_rows(const fplus_symbolic *sym) { return sym->n_tau_rows; }
extern "C" int64_t fplus_symbolic_n_dense_cols(const fplus_symbolic *sym) { return sym->n_tau_cols; }

// The interior pattern (dense rows' entries and dense columns dropped, the dimensions kept) and the fill-reducing order
// of its columns (empty ones, the dense columns among them, last).  Exported for the tests (fplus_b200.h).
extern "C" int fplus_b200_interior_order(int64_t n, const int64_t *Ap, const int64_t *Ai, const unsigned char *trow,
                                         const unsigned char *tcol, int64_t *perm)
{
    std::vector<int64_t> pin((size_t)n + 1), ain;
    ain.reserve((size_t)Ap[n]);
    pin[0] = 0;
    for (int64_t j = 0; j < n; j++) {
        if (!(tcol && tcol[j]))
            for (int64_t q = Ap[j]; q < Ap[j + 1]; q++) if (!(trow && trow[Ai[q]])) ain.push_back(Ai[q]);
        pin[j + 1] = (int64_t)ain.size();
    }
    colamd_order(n, n, pin.data(), ain.data(), perm);
    return FPLUS_OK;
}

namespace fpl {

// The permuted pattern B = A[row_perm, :][:, col_perm] (rows ascending in each column) and its gather map, and the
// analysed pattern itself; row_perm and col_perm are set.
static void build_permuted(fplus_symbolic *sym, const int64_t *Ap, const int64_t *Ai)
{
    const int64_t n = sym->n, nnz = Ap[n];
    std::vector<int64_t> inv((size_t)(n > 0 ? n : 1));
    for (int64_t i = 0; i < n; i++) inv[sym->row_perm[i]] = i;
    sym->Ap0.assign(Ap, Ap + n + 1);
    sym->Ai0.assign(Ai, Ai + nnz);
    sym->Bp.assign((size_t)n + 1, 0);
    sym->Bi.resize((size_t)nnz);
    sym->Bsrc.resize((size_t)nnz);
    for (int64_t jj = 0; jj < n; jj++) { int64_t c = sym->col_perm[jj]; sym->Bp[jj + 1] = sym->Bp[jj] + Ap[c + 1] - Ap[c]; }
    std::vector<std::pair<int64_t, int64_t>> tmp;
    for (int64_t jj = 0; jj < n; jj++) {
        int64_t c = sym->col_perm[jj];
        tmp.clear();
        for (int64_t q = Ap[c]; q < Ap[c + 1]; q++) tmp.emplace_back(inv[Ai[q]], q);
        std::sort(tmp.begin(), tmp.end());
        int64_t o = sym->Bp[jj];
        for (auto &t : tmp) { sym->Bi[o] = t.first; sym->Bsrc[o] = t.second; o++; }
    }
}

// A symbolic object for static orders the caller chose (FPLUS src/pipeline.c:84-111 factors A[row_perm, :][:, col_perm]
// as given).  The trailing rows of B with more than max(n / 2, 10) entries, and likewise its trailing columns, become
// the dense (border) lines of the front structure: where the orders come from fplus_analyze these are its dense lines.
// A dense line elsewhere in the order is an ordinary row or column: correct, but its fronts are wide.
int symbolic_from_orders(int64_t n, const int64_t *Ap, const int64_t *Ai, const int64_t *row_perm, const int64_t *col_perm,
                         fplus_symbolic **out, char *err, size_t errlen)
{
    *out = nullptr;
    fplus_symbolic *sym = new (std::nothrow) fplus_symbolic;
    if (!sym) { errf(err, errlen, "out of memory"); return FPLUS_ERR_NOMEM; }
    try {
        const int64_t nnz = Ap[n];
        sym->n = n; sym->nnz = nnz;
        sym->row_perm.assign(row_perm, row_perm + n);
        sym->col_perm.assign(col_perm, col_perm + n);
        const double thr = std::max(0.5 * (double)n, 10.0);
        std::vector<int64_t> cnt((size_t)(n > 0 ? n : 1), 0);
        for (int64_t q = 0; q < nnz; q++) cnt[Ai[q]]++;
        int64_t ntr = 0, ntc = 0;
        while (ntr < n && (double)cnt[row_perm[n - 1 - ntr]] > thr) ntr++;
        while (ntc < n && (double)(Ap[col_perm[n - 1 - ntc] + 1] - Ap[col_perm[n - 1 - ntc]]) > thr) ntc++;
        sym->n_tau_rows = ntr; sym->n_tau_cols = ntc;
        build_permuted(sym, Ap, Ai);
    } catch (const std::bad_alloc &) {
        delete sym;
        errf(err, errlen, "out of memory");
        return FPLUS_ERR_NOMEM;
    }
    *out = sym;
    return FPLUS_OK;
}

}  // namespace fpl

// FPLUS src/order.c:267-399, with this library's minimum-degree order in place of SuiteSparse's COLAMD / AMD (every
// `ordering` value runs it: minimum degree on the graph of A^T A is what both orders compute).
extern "C" int fplus_analyze_ord(int64_t n, const int64_t *Ap, const int64_t *Ai, int pin_dense, double tau_density,
                                 int64_t tau_min_nnz, const unsigned char *tau_row_mask, const unsigned char *tau_col_mask,
                                 int postorder, int ordering, fplus_symbolic **sym_out, char *err, size_t errlen)
{
    if (!sym_out) { errf(err, errlen, "sym is NULL"); return FPLUS_ERR_BADARG; }
    *sym_out = nullptr;
    if (ordering < FPLUS_ORDER_COLAMD || ordering > FPLUS_ORDER_AUTO) { errf(err, errlen, "unknown ordering %d", ordering); return FPLUS_ERR_BADARG; }
    int vrc = check_compressed(n, Ap, Ai, 1, err, errlen);
    if (vrc != FPLUS_OK) return vrc;
    const int64_t nnz = Ap[n];
    fplus_symbolic *sym = new (std::nothrow) fplus_symbolic;
    if (!sym) { errf(err, errlen, "out of memory"); return FPLUS_ERR_NOMEM; }
    try {
        sym->n = n; sym->nnz = nnz;
        std::vector<unsigned char> trow((size_t)(n > 0 ? n : 1), 0), tcol((size_t)(n > 0 ? n : 1), 0);
        // dense lines: more than max(tau_density n, tau_min_nnz) entries, or the masks (FPLUS src/order.c:286-296)
        if (pin_dense) {
            const double thr = tau_density * (double)n > (double)tau_min_nnz ? tau_density * (double)n : (double)tau_min_nnz;
            if (tau_row_mask) std::memcpy(trow.data(), tau_row_mask, (size_t)n);
            else {
                std::vector<int64_t> cnt((size_t)(n > 0 ? n : 1), 0);
                for (int64_t q = 0; q < nnz; q++) cnt[Ai[q]]++;
                for (int64_t i = 0; i < n; i++) trow[i] = (double)cnt[i] > thr;
            }
            if (tau_col_mask) std::memcpy(tcol.data(), tau_col_mask, (size_t)n);
            else for (int64_t j = 0; j < n; j++) tcol[j] = (double)(Ap[j + 1] - Ap[j]) > thr;
        }
        int64_t ntr = 0, ntc = 0;
        for (int64_t i = 0; i < n; i++) { ntr += trow[i] != 0; ntc += tcol[i] != 0; }
        sym->n_tau_rows = ntr; sym->n_tau_cols = ntc;
        // row order: interior rows, then dense rows, each ascending (FPLUS src/order.c:303-304)
        sym->row_perm.resize((size_t)n);
        { int64_t k = 0; for (int64_t i = 0; i < n; i++) if (!trow[i]) sym->row_perm[k++] = i;
          for (int64_t i = 0; i < n; i++) if (trow[i]) sym->row_perm[k++] = i; }
        // fill-reducing order of the pattern without the dense lines
        std::vector<int64_t> perm((size_t)(n > 0 ? n : 1));
        fplus_b200_interior_order(n, Ap, Ai, trow.data(), tcol.data(), perm.data());
        sym->col_perm.resize((size_t)n);
        if (postorder) {
            // postorder of the column etree of the interior pattern (interior rows renumbered ascending, columns in the
            // fill-reducing order), then the dense columns in that order (FPLUS src/order.c:361-386)
            std::vector<int64_t> icols, rmap((size_t)(n > 0 ? n : 1));
            int64_t mi = 0;
            for (int64_t k = 0; k < n; k++) if (!tcol[perm[k]]) icols.push_back(perm[k]);
            for (int64_t i = 0; i < n; i++) rmap[i] = trow[i] ? -1 : mi++;
            const int64_t ni = (int64_t)icols.size();
            std::vector<int64_t> Cp((size_t)ni + 1), Ci, post((size_t)(ni > 0 ? ni : 1));
            Cp[0] = 0;
            for (int64_t jj = 0; jj < ni; jj++) {
                int64_t c = icols[jj];
                for (int64_t q = Ap[c]; q < Ap[c + 1]; q++) if (rmap[Ai[q]] >= 0) Ci.push_back(rmap[Ai[q]]);
                Cp[jj + 1] = (int64_t)Ci.size();
            }
            fplus_coletree_postorder(mi, ni, Cp.data(), Ci.data(), post.data());
            int64_t k = 0;
            for (int64_t jj = 0; jj < ni; jj++) sym->col_perm[k++] = icols[post[jj]];
            for (int64_t q = 0; q < n; q++) if (tcol[perm[q]]) sym->col_perm[k++] = perm[q];
        } else {
            int64_t k = 0;
            for (int64_t q = 0; q < n; q++) if (!tcol[perm[q]]) sym->col_perm[k++] = perm[q];
            for (int64_t q = 0; q < n; q++) if (tcol[perm[q]]) sym->col_perm[k++] = perm[q];
        }
        build_permuted(sym, Ap, Ai);
    } catch (const std::bad_alloc &) {
        delete sym;
        errf(err, errlen, "out of memory");
        return FPLUS_ERR_NOMEM;
    }
    *sym_out = sym;
    return FPLUS_OK;
}

extern "C" int fplus_analyze(int64_t n, const int64_t *Ap, const int64_t *Ai, int pin_dense, double tau_density,
                             int64_t tau_min_nnz, const unsigned char *tau_row_mask, const unsigned char *tau_col_mask,
                             int postorder, fplus_symbolic **sym, char *err, size_t errlen)
{
    return fplus_analyze_ord(n, Ap, Ai, pin_dense, tau_density, tau_min_nnz, tau_row_mask, tau_col_mask, postorder,
                             FPLUS_ORDER_COLAMD, sym, err, errlen);
}

// FPLUS src/numeric.c:15-22
extern "C" void fplus_default_options(fplus_options *o)
{
    o->pin_dense = 1; o->tau_density = 0.5; o->tau_min_nnz = 10; o->postorder = 1;
    o->equilibrate = 1; o->ruiz_max_iter = 20; o->ruiz_tol = 1e-2;
    o->pivot_rel = FPLUS_PIVOT_REL_DEFAULT; o->pivot_strategy = FPLUS_PIVOT_PARTIAL; o->drop_tol = 0.0;
    o->relax_rows = 32; o->panel = 512;
    o->use_gpu = 0; o->gpu_min_flops = 5e7; o->verbose = 0;
}

// FPLUS src/numeric.c:24-29
extern "C" int fplus_analyze_opts(int64_t n, const int64_t *Ap, const int64_t *Ai, const fplus_options *opt,
                                  fplus_symbolic **sym, char *err, size_t errlen)
{
    fplus_options d;
    if (!opt) { fplus_default_options(&d); opt = &d; }
    return fplus_analyze(n, Ap, Ai, opt->pin_dense, opt->tau_density, opt->tau_min_nnz, nullptr, nullptr, opt->postorder,
                         sym, err, errlen);
}
