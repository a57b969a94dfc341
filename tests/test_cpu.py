"""CPU tests (no GPU): the oracle against the reference and the golden fixtures, the host-side analysis against the
reference's own ordering code, the multifrontal structure against the oracle's factors, the C-ABI library's exports,
and the host-side argument checks of the boundary."""
import ctypes
import os
import re

import numpy as np
import pytest
import scipy.sparse as sp

import fplus_b200 as F
import oracle as O
from fplus_b200 import workloads as W
from tests.cases import CASES

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
needs_ref = pytest.mark.skipif(not O.have_reference(), reason="oracle/_ref (the reference build) is not present")


def _rel(A, B):
    return sp.linalg.norm(A - B) / max(sp.linalg.norm(B), 1e-300)


def _masks(n, S):
    tr = np.zeros(n, np.uint8); tr[S.row_perm[n - S.n_dense_rows:]] = 1
    tc = np.zeros(n, np.uint8); tc[S.col_perm[n - S.n_dense_cols:]] = 1
    return tr, tc


# ------------------------------------------------------------------------------------------------ the library boundary
def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fplus_\w+)\s*\(", text)) - {"fplus_symbolic", "fplus_numeric"})


def test_library_exports_every_declared_symbol():
    L = F.lib()
    declared = _declared("fplus.h") + _declared("fplus_b200.h")
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, f"declared but not exported: {missing}"
    assert set(F.FPLUS_H_SYMBOLS) <= set(declared) and set(F.FPLUS_B200_H_SYMBOLS) <= set(declared)


def test_options_defaults_match_reference():
    o = F.default_options()
    # FPLUS src/numeric.c:15-22
    assert (o.pin_dense, o.tau_density, o.tau_min_nnz, o.postorder) == (1, 0.5, 10, 1)
    assert (o.equilibrate, o.ruiz_max_iter, o.ruiz_tol) == (1, 20, 1e-2)
    assert o.pivot_rel == F.FPLUS_PIVOT_REL_DEFAULT and o.pivot_strategy == F.FPLUS_PIVOT_PARTIAL and o.drop_tol == 0.0
    assert (o.relax_rows, o.panel, o.use_gpu, o.gpu_min_flops, o.verbose) == (32, 512, 0, 5e7, 0)
    assert ctypes.sizeof(F.Options) == 112


def _factor_rc(S, Ax, cplx, opt=None, Ap=None, Ai=None):
    err = ctypes.create_string_buffer(256)
    h = ctypes.c_void_p()
    Ap = S.Ap if Ap is None else np.ascontiguousarray(Ap, np.int64)
    Ai = S.Ai if Ai is None else np.ascontiguousarray(Ai, np.int64)
    Ax = np.ascontiguousarray(Ax)
    rc = F.lib().fplus_factor(S._h, F._p64(Ap), F._p64(Ai), Ax.ctypes.data_as(ctypes.c_void_p), int(cplx),
                              ctypes.byref(opt if opt is not None else S.options), ctypes.byref(h), err, 256)
    return rc, err.value.decode()


def test_factor_argument_checks_on_host():
    n, Ap, Ai, Ax = W.convdiff2d(8, 1)
    S = F.analyze(n, Ap, Ai)
    assert _factor_rc(S, Ax, 0, F.default_options(pivot_strategy=7))[0] == F.FPLUS_ERR_BADARG
    assert _factor_rc(S, Ax, 0, F.default_options(drop_tol=-1.0))[0] == F.FPLUS_ERR_BADARG
    rc, msg = _factor_rc(S, Ax, 0, F.default_options(pivot_strategy=F.FPLUS_PIVOT_ROOK))
    assert rc == F.FPLUS_ERR_BADARG and "partial pivoting" in msg
    assert _factor_rc(S, Ax, 0, F.default_options(drop_tol=1e-3))[0] == F.FPLUS_ERR_BADARG
    assert _factor_rc(S, Ax, 0, F.default_options(pivot_rel=-1.0))[0] == F.FPLUS_ERR_BADARG
    bad = Ax.copy(); bad[5] = np.nan
    rc, msg = _factor_rc(S, bad, 0)
    assert rc == F.FPLUS_ERR_BADARG and "non-finite" in msg
    # a different pattern with the same number of entries
    Ai2 = Ai.copy(); Ai2[Ap[3]] = (Ai2[Ap[3]] + 1) % n
    A2 = sp.csc_matrix((Ax, Ai2, Ap), shape=(n, n)); A2.sort_indices()
    if A2.nnz == len(Ax):
        rc, msg = _factor_rc(S, A2.data, 0, None, A2.indptr, A2.indices)
        assert rc == F.FPLUS_ERR_BADARG
    rc, msg = _factor_rc(S, Ax[:-1], 0, None, np.r_[Ap[:-1], Ap[-1] - 1], Ai[:-1])
    assert rc == F.FPLUS_ERR_BADARG and "nonzeros" in msg


def test_non_finite_values_found_in_large_arrays():
    """The host check of the values (several threads over arrays of a million values or more): the first non-finite
    entry is named, real and complex, wherever it lies; finite values pass."""
    n, Ap, Ai, Ax = W.convdiff2d(1100, 1)                  # 6 million entries
    assert Ax.size >= 1 << 20
    S = F.analyze(n, Ap, Ai)
    for pos in (3, Ax.size // 2 + 7, Ax.size - 1):
        for val in (np.nan, np.inf, -np.inf):
            bad = Ax.copy(); bad[pos] = val; bad[-1 if pos != Ax.size - 1 else 0] = np.nan
            first = min(pos, Ax.size - 1 if pos != Ax.size - 1 else 0)
            rc, msg = _factor_rc(S, bad, 0)
            assert rc == F.FPLUS_ERR_BADARG and f"non-finite value in entry {first}" in msg, (pos, val, msg)
    cx = Ax.astype(np.complex128); cx[11] = complex(1.0, np.nan)
    rc, msg = _factor_rc(S, cx, 1)
    assert rc == F.FPLUS_ERR_BADARG and "non-finite value in entry 11" in msg


def test_analyze_argument_checks():
    with pytest.raises(F.FplusError) as e:
        F.analyze(2, np.array([0, 2, 3]), np.array([1, 0, 1]))       # unsorted: not canonical
    assert e.value.code == F.FPLUS_ERR_BADARG
    with pytest.raises(F.FplusError) as e:
        F.analyze(2, np.array([0, 2, 3]), np.array([0, 5, 1]))       # index out of range
    assert e.value.code == F.FPLUS_ERR_BADARG


# ------------------------------------------------------------------------------------------------ the analysis
@needs_ref
@pytest.mark.parametrize("name", ["convdiff2d_g20", "pencil_1x64", "hard_real_300", "hard_cplx_300", "banded_cplx_1200"])
def test_analysis_matches_reference_order_code(name):
    """Dense-line pinning, the row order and the column-etree postorder against the reference's src/order.c, given the
    same fill-reducing order (SuiteSparse COLAMD is absent: the order is injected into the reference's code)."""
    n, Ap, Ai, Ax = CASES[name]()
    S = F.analyze(n, Ap, Ai)
    cnt = np.bincount(Ai, minlength=n)
    thr = max(0.5 * n, 10)
    tr, tc = (cnt > thr).astype(np.uint8), (np.diff(Ap) > thr).astype(np.uint8)
    assert S.n_dense_rows == tr.sum() and S.n_dense_cols == tc.sum()
    perm = F.interior_order(n, Ap, Ai, tr, tc)
    R = O.RefLU(n, Ap, Ai, None, perm, None, None, postorder=1)
    assert np.array_equal(R.row_perm, S.row_perm)
    assert np.array_equal(R.col_perm, S.col_perm)


@needs_ref
def test_coletree_postorder_matches_reference():
    rng = np.random.default_rng(4)
    for m, n in ((40, 30), (200, 200), (150, 170)):
        A = sp.random(m, n, density=0.04, random_state=rng, format="csc")
        A.sort_indices()
        Ap, Ai = A.indptr.astype(np.int64), A.indices.astype(np.int64)
        p1, p2 = np.zeros(n, np.int64), np.zeros(n, np.int64)
        assert F.lib().fplus_coletree_postorder(m, n, F._p64(Ap), F._p64(Ai), F._p64(p1)) == 0
        assert O.reference().fplus_coletree_postorder(m, n, F._p64(Ap), F._p64(Ai), F._p64(p2)) == 0
        assert np.array_equal(p1, p2)


def test_interior_order_is_a_fill_reducing_permutation():
    n, Ap, Ai, Ax = W.convdiff2d(30, 1)
    perm = F.interior_order(n, Ap, Ai)
    assert np.array_equal(np.sort(perm), np.arange(n))
    S = F.analyze(n, Ap, Ai)
    A = sp.csc_matrix((np.ones(len(Ai)), Ai, Ap), shape=(n, n))
    fill = lambda cp: O.OracleLU(n, Ap, Ai, Ax, np.arange(n), cp).L.nnz
    assert fill(S.col_perm) < 0.7 * fill(np.arange(n))            # less fill than the natural (banded) order


# ------------------------------------------------------------------------------------------------ the oracle
@needs_ref
@pytest.mark.parametrize("name", ["convdiff2d_g20", "convdiff2d_g100", "pencil_1x64", "hard_real_300", "hard_cplx_300",
                                  "hard_cplx_300_s0", "banded_cplx_1200", "convdiff3d_g12"])
def test_oracle_matches_reference(name):
    n, Ap, Ai, Ax = CASES[name]()
    S = F.analyze(n, Ap, Ai)
    tr, tc = _masks(n, S)
    R = O.RefLU(n, Ap, Ai, Ax, S.col_perm, tr, tc, postorder=0)
    orc = O.OracleLU(n, Ap, Ai, Ax, S.row_perm, S.col_perm)
    assert np.array_equal(R.p, orc.p)
    assert np.array_equal(R.Dr, orc.Dr) and np.array_equal(R.Dc, orc.Dc)
    L, U, p_lu, _ = R.factors()
    assert np.array_equal(p_lu, orc.p_lu)
    assert _rel(orc.L, L) < 1e-12 and _rel(orc.U, U) < 1e-12
    b = np.random.default_rng(3).standard_normal(n) + (1j if np.iscomplexobj(Ax) else 0)
    for t in ((0, 1, 2) if np.iscomplexobj(Ax) else (0, 1)):
        x, xr = orc.solve(b, t), R.solve(b, t)
        assert np.linalg.norm(x - xr) <= 1e-10 * np.linalg.norm(xr)


@pytest.mark.parametrize("name", ["relaxed_panel_case50", "relaxed_panel_case3"])
def test_oracle_against_golden_regression_matrices(name):
    """The reference's regression matrices (identity orders): the reference keeps the same pivots for every relax /
    panel combination, and the oracle reproduces them, the scalings bit for bit, and the solution."""
    z = np.load(os.path.join(GOLD, name + ".npz"))
    assert bool(z["p_all_equal"])
    n = int(z["n"])
    orc = O.OracleLU(n, z["Ap"], z["Ai"], z["Ax"], z["row_perm"], z["col_perm"])
    assert np.array_equal(orc.p, z["p"])
    assert np.array_equal(orc.Dr, z["Dr"]) and np.array_equal(orc.Dc, z["Dc"])
    assert abs(sp.linalg.norm(orc.L) - float(z["L_fro"])) <= 1e-12 * float(z["L_fro"])
    assert abs(sp.linalg.norm(orc.U) - float(z["U_fro"])) <= 1e-12 * float(z["U_fro"])
    x = orc.solve(z["b"], 0)
    assert np.linalg.norm(x - z["x"]) <= 1e-10 * np.linalg.norm(z["x"])
    assert O.backward_error(n, z["Ap"], z["Ai"], z["Ax"], x, z["b"]) < 1e-13


def _golden_generated():
    z = np.load(os.path.join(GOLD, "generated_cases.npz"))
    return z, [str(s) for s in z["names"]]


@pytest.mark.parametrize("name", ["convdiff2d_g20", "pencil_1x64", "hard_real_300", "hard_cplx_300", "banded_cplx_600"])
def test_oracle_against_golden_generated(name):
    z, names = _golden_generated()
    g = lambda k: z[f"{name}__{k}"]
    n = int(g("n"))
    orc = O.OracleLU(n, g("Ap"), g("Ai"), g("Ax"), g("row_perm"), g("col_perm"))
    assert np.array_equal(orc.p, g("p"))
    assert np.array_equal(orc.Dr, g("Dr")) and np.array_equal(orc.Dc, g("Dc"))
    assert abs(sp.linalg.norm(orc.L) - float(g("L_fro"))) <= 1e-12 * float(g("L_fro"))
    assert abs(sp.linalg.norm(orc.U) - float(g("U_fro"))) <= 1e-12 * float(g("U_fro"))
    B = g("B")
    for t in ((0, 1, 2) if np.iscomplexobj(g("Ax")) else (0, 1)):
        X = orc.solve(B, t)
        assert np.linalg.norm(X - g(f"X{t}")) <= 1e-10 * np.linalg.norm(g(f"X{t}"))
    # the analysis of this build reproduces the committed orders
    S = F.analyze(n, g("Ap"), g("Ai"))
    assert np.array_equal(S.row_perm, g("row_perm")) and np.array_equal(S.col_perm, g("col_perm"))


def test_ruiz_range_guard_known_answers():
    """tests/c/test_fplus.c:249-266: entries near 1e200 are rescaled by a power of two (scaled to 1 within e^0.01, and
    Dr A Dc reproduces them); a 1e300 / 1e-300 span is refused."""
    L = O.restatement()
    n = 3
    p = np.array([0, 1, 2, 3], np.int64); i = np.array([0, 1, 2], np.int64)
    x = np.array([1e200, 1e100, 1e150]); x0 = x.copy()
    Dr, Dc = np.zeros(3), np.zeros(3)
    it = ctypes.c_int()
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    rc = L.orc_ruiz(n, F._p64(p), F._p64(i), x.ctypes.data_as(ctypes.c_void_p), 0, 20, 1e-2, dp(Dr), dp(Dc), ctypes.byref(it), None, 0)
    assert rc == 0
    assert np.all(np.abs(np.log(np.abs(x))) < 1e-2)
    assert np.all(np.abs(Dr * x0 * Dc - x) < 1e-14 * np.abs(x))
    y = np.array([1e300, 1e-300, 1.0])
    rc = L.orc_ruiz(n, F._p64(p), F._p64(i), y.ctypes.data_as(ctypes.c_void_p), 0, 20, 1e-2, dp(Dr), dp(Dc), ctypes.byref(it), None, 0)
    assert rc == -3
    if O.have_reference():
        R = O.reference()
        x = x0.copy()
        Dr2, Dc2 = np.zeros(3), np.zeros(3)
        assert R.fplus_ruiz(n, F._p64(p), F._p64(i), x.ctypes.data_as(ctypes.c_void_p), 0, 1, 20, 1e-2, 0, dp(Dr2), dp(Dc2), None, 0) == 0
        x1 = x0.copy()
        L.orc_ruiz(n, F._p64(p), F._p64(i), x1.ctypes.data_as(ctypes.c_void_p), 0, 20, 1e-2, dp(Dr), dp(Dc), ctypes.byref(it), None, 0)
        assert np.array_equal(x, x1) and np.array_equal(Dr, Dr2) and np.array_equal(Dc, Dc2)


def test_oracle_several_rhs_equal_one_at_a_time():
    n, Ap, Ai, Ax = CASES["banded_cplx_1200"]()
    S = F.analyze(n, Ap, Ai)
    orc = O.OracleLU(n, Ap, Ai, Ax, S.row_perm, S.col_perm)
    B = np.random.default_rng(1).standard_normal((n, 5)) + 1j
    X = orc.solve(B, 2)
    assert np.array_equal(X, np.column_stack([orc.solve(B[:, k], 2) for k in range(5)]))


# ------------------------------------------------------------------------------------------------ the front structure
@pytest.mark.parametrize("name", ["convdiff2d_g20", "convdiff2d_g100", "convdiff3d_g12", "pencil_1x64", "hard_real_300",
                                  "hard_cplx_300", "banded_cplx_1200"])
def test_front_structure_contains_the_factors(name):
    """Every nonzero of the oracle's L and U (same orders, same pivots) lies inside the multifrontal structure: U[k, c]
    in the columns of the front of k, and each L[row, k]'s row (by its first column) in the subtree of that front.  A
    dense row pivoted inside a front with border rows needs the dense chain: with the chain started at that front's first
    column, the containment holds."""
    n, Ap, Ai, Ax = CASES[name]()
    S = F.analyze(n, Ap, Ai)
    orc = O.OracleLU(n, Ap, Ai, Ax, S.row_perm, S.col_perm)
    mi = n - S.n_dense_rows
    Bc = orc.B.tocoo()
    firstcol = np.full(n, n)
    np.minimum.at(firstcol, Bc.row, Bc.col)
    p_lu = orc.p_lu
    Lc, Uc = orc.L.tocoo(), orc.U.tocoo()

    def check(tail):
        """containment for the pivot steps before the first dense-row pivot in a front with border rows (all steps when
        there is none); returns that step or None"""
        P = S.plan(tail)
        cf, par, cptr, cols, nbord = P["col_front"], P["parent"], P["col_ptr"], P["cols"], P["nbord"]
        nf = len(par)
        border = np.nonzero((p_lu >= mi) & (nbord[cf] > 0))[0]
        kmax = border[0] if len(border) else n
        first = np.arange(nf)
        for s in range(nf):
            if par[s] >= 0:
                first[par[s]] = min(first[par[s]], first[s])
        member = sp.csr_matrix((np.ones(len(cols), bool), cols, cptr), shape=(nf, n))
        u = Uc.row < kmax
        assert np.all(np.asarray(member[cf[Uc.row[u]], Uc.col[u]]).ravel()), "U entry outside its front's columns"
        off = (Lc.row != Lc.col) & (Lc.col < kmax)
        rows = p_lu[Lc.row[off]]
        ks = Lc.col[off]
        interior = rows < mi
        fb = cf[firstcol[rows[interior]]]
        fk = cf[ks[interior]]
        assert np.all((first[fk] <= fb) & (fb <= fk)), "L row outside its front's subtree"
        return border[0] if len(border) else None

    b = check(-1)
    if b is not None:
        P = S.plan(-1)
        s = P["col_front"][b]
        f0 = int(np.nonzero(P["col_front"] == s)[0][0])
        assert check(f0) is None


# ------------------------------------------------------------------------------------------------ multi-process (gloo)
def _replica_worker(rank, world, port, out):
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out[rank] = bench.allreduce_max(float(10 + rank), "cpu")
    finally:
        dist.destroy_process_group()


def test_replica_timing_is_the_max_over_ranks():
    """bench.py --gpus N runs N independent replicas (one factorization does not shard); the reported time is the
    slowest rank's, reduced the same way on every rank (two gloo ranks on CPU)."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_replica_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    assert dict(out) == {0: 11.0, 1: 11.0}


def test_batch_argument_checks_on_host():
    """The batch entry points: an empty batch succeeds; NULL arrays are refused before any GPU work."""
    L = F.lib()
    err = ctypes.create_string_buffer(256)
    assert L.fplus_b200_factor_batch(0, None, None, None, None, 0, None, 2, None, None, err, 256) == F.FPLUS_OK
    assert L.fplus_b200_factor_batch(3, None, None, None, None, 0, None, 2, None, None, err, 256) == F.FPLUS_ERR_BADARG
    assert L.fplus_b200_solve_batch(0, None, None, None, None, 0, 2, None, err, 256) == F.FPLUS_OK
    assert L.fplus_b200_solve_batch(2, None, None, None, None, 0, 2, None, err, 256) == F.FPLUS_ERR_BADARG


def test_front_shape_checks_on_host():
    """fplus_b200_set_front_shape (host only): the pivot-block LU kernel 1, 2 or 3, plus 4 (tall blocks by panels), 8 (no
    batched levels), 16 (forward-substitution tails) and 32 (no direct write of the chain's contribution blocks); widths
    16 .. 4096 and chain fronts of 8 .. 64 pivots; anything else is refused and leaves the shape as it was."""
    n, Ap, Ai, _ = W.convdiff2d(12, 1)
    S = F.analyze(n, Ap, Ai)
    L = F.lib()
    for v in (1, 2, 3, 5, 10, 18, 33, 63):
        assert L.fplus_b200_set_front_shape(S._h, 256, 64, v) == F.FPLUS_OK, v
    for v in (0, 4, 8, 64, 66, -1):
        assert L.fplus_b200_set_front_shape(S._h, 256, 64, v) == F.FPLUS_ERR_BADARG, v
    assert L.fplus_b200_set_front_shape(S._h, 8, 64, 2) == F.FPLUS_ERR_BADARG
    assert L.fplus_b200_set_front_shape(S._h, 256, 65, 2) == F.FPLUS_ERR_BADARG
    assert L.fplus_b200_set_front_shape(None, 256, 64, 2) == F.FPLUS_ERR_BADARG


def test_lowlevel_argument_checks_on_host():
    """The low-level entry points refuse bad arguments, and a zero or missing diagonal of U, on the host before any
    GPU work (FPLUS src/pipeline.c:91-99, src/solve_plan.c:664-673, src/solve.c:62-66); a plan on factors this library
    did not return is host-only until its first solve and reports -1 supernodes."""
    n, Ap, Ai, Ax = CASES["convdiff2d_g20"]()
    rp = np.arange(n)
    bad = rp.copy(); bad[3] = bad[4]
    with pytest.raises(F.FplusError) as e:
        F.factor_sn_perm(Ax, Ai, Ap, n, bad, rp, False)
    assert e.value.code == F.FPLUS_ERR_BADARG
    with pytest.raises(F.FplusError) as e:
        F.factor_sn_perm(Ax, Ai[::-1].copy(), Ap, n, rp, rp, False)       # rows not ascending
    assert e.value.code == F.FPLUS_ERR_BADARG
    # unit lower L and upper U, one zero on U's diagonal
    m = 6
    Lm = sp.csc_matrix(np.tril(np.ones((m, m))))
    Um = sp.csc_matrix(np.triu(np.ones((m, m)) * 2.0))
    Lp, Li, Up, Ui = (a.astype(np.int64) for a in (Lm.indptr, Lm.indices, Um.indptr, Um.indices))
    pl = F.solve_plan(Lp, Li, Up, Ui)
    assert pl.nsupernodes == -1
    Ux = Um.data.copy(); Ux[Up[3 + 1] - 1] = 0.0                           # U(3, 3) = 0
    b = np.arange(1.0, m + 1)
    with pytest.raises(F.FplusError) as e:
        F.lu_solve_plan(pl, Lp, Li, Lm.data, Up, Ui, Ux, b, 0, False)
    assert e.value.code == F.FPLUS_ERR_SINGULAR
    L = F.lib()
    x = b.copy()
    assert L.fplus_tri_solve(m, F._p64(Lp), F._p64(Li), Lm.data.ctypes.data_as(ctypes.c_void_p), F._p64(Up), F._p64(Ui),
                             Ux.ctypes.data_as(ctypes.c_void_p), x.ctypes.data_as(ctypes.c_void_p), 0, 0) == F.FPLUS_ERR_SINGULAR
    assert np.array_equal(x, b), "x changed before the singular diagonal was reported"
    for trans, nrhs, ldx, nn in ((3, 1, m, m), (0, -1, m, m), (0, 1, m - 1, m), (0, 1, m + 1, m + 1)):
        assert L.fplus_tri_solve_plan(pl._h, nn, F._p64(Lp), F._p64(Li), Lm.data.ctypes.data_as(ctypes.c_void_p), F._p64(Up),
                                      F._p64(Ui), Um.data.ctypes.data_as(ctypes.c_void_p), x.ctypes.data_as(ctypes.c_void_p),
                                      nrhs, ldx, trans, 0) == F.FPLUS_ERR_BADARG
    assert L.fplus_tri_solve(m, F._p64(Lp), F._p64(Li), Lm.data.ctypes.data_as(ctypes.c_void_p), F._p64(Up), F._p64(Ui),
                             Um.data.ctypes.data_as(ctypes.c_void_p), x.ctypes.data_as(ctypes.c_void_p), 3, 0) == F.FPLUS_ERR_BADARG
    # nrhs 0 on a plan: nothing to do, no GPU needed
    assert L.fplus_tri_solve_plan(pl._h, m, F._p64(Lp), F._p64(Li), Lm.data.ctypes.data_as(ctypes.c_void_p), F._p64(Up),
                                  F._p64(Ui), Um.data.ctypes.data_as(ctypes.c_void_p), x.ctypes.data_as(ctypes.c_void_p),
                                  0, m, 0, 0) == F.FPLUS_OK


def test_solve_refine_argument_checks_on_host():
    """fplus_b200_solve_refine refuses a NULL factorization before any GPU work."""
    L = F.lib()
    err = ctypes.create_string_buffer(256)
    x = np.zeros(4)
    assert L.fplus_b200_solve_refine(None, x.ctypes.data_as(ctypes.c_void_p), 1, 4, 0, 5, 0.0, None, None, err, 256) \
        == F.FPLUS_ERR_BADARG


def test_sparse_lu_and_orders_checks_on_host():
    """SparseLU refuses what this build does not compute (incomplete LU, rook / full pivoting) before any GPU work, and
    fplus_b200_symbolic_from_orders refuses a non-permutation; a valid call analyses on the host only."""
    n, Ap, Ai, Ax = CASES["convdiff2d_g20"]()
    A = sp.csc_matrix((Ax, Ai, Ap), shape=(n, n))
    for kw in (dict(drop_tol=1e-3), dict(pivot_strategy="rook"), dict(pivot_strategy="full"), dict(ordering="nd")):
        with pytest.raises(ValueError):
            F.SparseLU(A, **kw)
    bad = np.arange(n); bad[0] = 1
    with pytest.raises(F.FplusError) as e:
        F.Symbolic.from_orders(n, Ap, Ai, bad, np.arange(n))
    assert e.value.code == F.FPLUS_ERR_BADARG
    S = F.Symbolic.from_orders(n, Ap, Ai, np.arange(n)[::-1], np.arange(n))
    assert np.array_equal(S.row_perm, np.arange(n)[::-1]) and S.n_dense_rows == 0
    assert S.plan()["col_front"].shape == (n,)


@pytest.mark.parametrize("name", ["pencil_1x64", "pencil_2x256", "hard_real_300", "convdiff3d_g12"])
def test_symbolic_from_orders_matches_analysis(name):
    """Given the analysis' own orders, the symbolic object for caller-given orders (fplus_factor_sn_perm, SparseLU without
    colamd) finds the same dense lines and builds the same front structure, so both paths factor alike (host only)."""
    n, Ap, Ai, Ax = CASES[name]()
    S = F.analyze(n, Ap, Ai)
    T = F.Symbolic.from_orders(n, Ap, Ai, S.row_perm, S.col_perm)
    assert (T.n_dense_rows, T.n_dense_cols) == (S.n_dense_rows, S.n_dense_cols)
    P, Q = S.plan(), T.plan()
    for k in ("col_front", "parent", "col_ptr", "cols", "nrows", "nbord"):
        assert np.array_equal(P[k], Q[k]), k
    assert P["f_dense"] == Q["f_dense"]


def test_ruiz_and_factor_sn_sym_checks_on_host():
    """fplus_ruiz refuses non-finite values and a row index out of range, and fplus_factor_sn_sym a matrix whose entry count
    differs from the analysis, before any GPU work (FPLUS src/equil.c:189-192, src/pipeline.c:118-122)."""
    n, Ap, Ai, Ax = CASES["convdiff2d_g20"]()
    bad = Ax.copy(); bad[5] = np.nan
    oob = Ai.copy(); oob[3] = n + 5                     # unsorted rows are accepted (FPLUS checks ranges only)
    for data, idx in ((bad, Ai), (Ax, oob)):
        with pytest.raises(F.FplusError) as e:
            F.ruiz_equilibrate(data, idx, Ap, n, 20, 1e-2, False, 0, 1)
        assert e.value.code == F.FPLUS_ERR_BADARG
    out = F.ruiz_equilibrate(np.zeros(0), np.zeros(0, np.int64), np.zeros(1, np.int64), 0, 20, 1e-2, False)
    assert out["Dr"].shape == (0,)
    S = F.analyze(n, Ap, Ai)
    Ap2 = Ap.copy(); Ap2[-1] -= 1
    with pytest.raises(F.FplusError) as e:
        F.factor_sn_sym(S, Ax[:-1], Ai[:-1], Ap2, False)
    assert e.value.code == F.FPLUS_ERR_BADARG and "nonzeros" in str(e.value)


# ------------------------------------------------------------------------------------ fixtures the GPU tests rely on
@pytest.mark.parametrize("name", ["pencil_m1", "pencil_m8", "convdiff2d_g100"])
def test_committed_orders_are_the_analysis(name):
    """tests/golden/orders.npz (the static orders the benchmark's reference arm injects) equals this build's analysis."""
    gens = {"pencil_m1": lambda: W.pencil(modes=1), "pencil_m8": lambda: W.pencil(), "convdiff2d_g100": lambda: W.convdiff2d(100, 1)}
    z = np.load(os.path.join(GOLD, "orders.npz"))
    n, Ap, Ai, _ = gens[name]()
    S = F.analyze(n, Ap, Ai)
    tr, tc = _masks(n, S)
    assert np.array_equal(S.row_perm, z[name + "__row_perm"]) and np.array_equal(S.col_perm, z[name + "__col_perm"])
    assert np.array_equal(tr, z[name + "__trow"]) and np.array_equal(tc, z[name + "__tcol"])


@pytest.mark.parametrize("name", ["pencil_n32768", "convdiff3d_g32"])
def test_big_fixtures_orders_and_generator(name):
    """The full-size fixtures of the GPU tests: the generator still makes the stored matrix and the analysis still gives
    the stored orders (the oracle's outputs in them were computed on those orders)."""
    z = np.load(os.path.join(GOLD, name + ".npz"))
    n, Ap, Ai, Ax = W.pencil() if name.startswith("pencil") else W.convdiff3d(32, 3)
    a = np.asarray(Ax)
    cs = np.array([a.real.sum(), (a.imag.sum() if np.iscomplexobj(a) else 0.0), np.abs(a).max(), float(a.size)])
    assert np.allclose(cs, z["checksum"], rtol=1e-13, atol=0)
    S = F.analyze(n, Ap, Ai)
    assert np.array_equal(S.row_perm, z["row_perm"]) and np.array_equal(S.col_perm, z["col_perm"])
    assert z["berr"] <= 1e-14


@needs_ref
@pytest.mark.parametrize("scale", [1e-170, 1e160])
def test_oracle_matches_reference_at_extreme_magnitudes(scale):
    """Without equilibration, values whose squared moduli underflow or overflow: the oracle picks the reference's pivots
    (both compare cabs), which pins the GPU test of the same matrices."""
    from tests.cases import hard_matrix
    n, Ap, Ai, Ax = hard_matrix(300, True, 0.0, 13)
    Ax = Ax * scale
    S = F.analyze(n, Ap, Ai, equilibrate=0)
    tr, tc = _masks(n, S)
    R = O.RefLU(n, Ap, Ai, Ax, S.col_perm, tr, tc, postorder=0, equilibrate=0)
    orc = O.OracleLU(n, Ap, Ai, Ax, S.row_perm, S.col_perm, equilibrate=0)
    assert np.array_equal(R.p, orc.p)


# -------------------------------------------------------------------------------- the batch form across GPUs (gloo, CPU)
def _lpt_worker(rank, world, port, costs, out):
    import torch.distributed as dist
    from fplus_b200 import shard
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        parts = shard.lpt_partition(costs, world)
        mine = parts[rank]
        # each rank "processes" its share (the sum of its costs stands for its device time) and the results are gathered
        res = shard.gather_results({"rank": rank, "jobs": mine, "load": float(sum(costs[k] for k in mine))})
        out[rank] = res
    finally:
        dist.destroy_process_group()


def test_lpt_partition_properties():
    from fplus_b200 import shard
    rng = np.random.default_rng(4)
    n = np.exp(rng.uniform(np.log(500), np.log(8000), 512)).astype(int)
    costs = [shard.pencil_cost(int(k), 20 * int(k)) for k in n]
    for parts in (1, 2, 3, 8):
        p = shard.lpt_partition(costs, parts)
        flat = sorted(k for q in p for k in q)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[k] for k in q) for q in p]
        assert max(loads) <= 4.0 / 3.0 * max(sum(costs) / parts, max(costs)) + 1e-6      # Graham's bound
        for q in p:
            assert all(costs[q[i]] >= costs[q[i + 1]] for i in range(len(q) - 1))    # largest first within a rank


def test_lpt_sharding_over_two_gloo_ranks():
    """The pencils of the batch form split across two ranks with no data exchange: both ranks compute the same
    partition, the shares are disjoint and complete, and the gathered loads are balanced."""
    import socket
    import torch.multiprocessing as mp
    from fplus_b200 import shard
    rng = np.random.default_rng(5)
    costs = [float(c) for c in rng.uniform(1.0, 100.0, 64)]
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_lpt_worker, args=(2, port, costs, out), nprocs=2, join=True, start_method="spawn")
    r0, r1 = out[0], out[1]
    assert r0 == r1                                                       # every rank holds every rank's result
    jobs = sorted(r0[0]["jobs"] + r0[1]["jobs"])
    assert jobs == list(range(64))
    assert set(r0[0]["jobs"]).isdisjoint(r0[1]["jobs"])
    assert abs(r0[0]["load"] - r0[1]["load"]) <= max(costs)
    assert shard.lpt_partition(costs, 2) == [r0[0]["jobs"], r0[1]["jobs"]]


@pytest.mark.skipif(not O.have_reference(), reason="the reference build (oracle/_ref) is not present")
def test_reference_arm_json_line():
    """bench.py --impl reference on the CPU-runnable stencil: one JSON line with the arm's metric, a measured value, a
    cpu_baseline of kind "reference" and an e2e with no host-device bytes; libfplus.so is not loaded by that arm."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    # the arm run as __main__, then whether the process mapped libfplus.so (printed after the arm's own line)
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'convdiff2d', '--steps', '1', "
            "'--warmup', '1']; runpy.run_path('bench.py', run_name='__main__'); "
            "print('LIBFPLUS_MAPPED', any('libfplus.so' in l for l in open('/proc/self/maps')))")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=root)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = out.stdout.strip().splitlines()
    assert lines[-1] == "LIBFPLUS_MAPPED False", lines[-1]
    line = json.loads(lines[-2])
    assert line["impl"] == "reference" and line["unit"] == "ms" and line["higher_is_better"] is False
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["config"]["n"] == 10000
