"""Parity of the low-level interface (the calls of FPLUS's Python extension, FPLUS include/fplus.h:73-88, 125-134)
through the C-ABI.

- fplus_factor_sn_perm / fplus_factor_sn_sym against the oracle with the same static orders: identical pivots, Dr and
  Dc (permuted order) bit-identical, L and U within 1e-12 normwise: the bar of fplus_factor.
- fplus_tri_solve_plan / fplus_tri_solve in the coordinates of the permuted matrix: on the arrays fplus_factor_sn_perm
  returned (the factorization's device copy) and on any other CSC factors (level-scheduled sweeps), each checked by its
  normwise backward error against the CSC factors themselves, at most 1e-13.
"""
import ctypes
import re

import numpy as np
import pytest
import scipy.sparse as sp

import fplus_b200 as F
import oracle as O
from tests.cases import CASES

pytestmark = pytest.mark.gpu

FACTOR_TOL = 1e-12
SOLVE_BERR = 1e-13


@pytest.fixture(scope="module")
def gpu():
    import torch
    assert torch.cuda.is_available(), "the GPU tests need a CUDA device"
    torch.cuda.init()
    return torch.device("cuda:0")


def _rel(A, B):
    nb = sp.linalg.norm(B)
    return sp.linalg.norm(A - B) / (nb if nb > 0 else 1.0)


def _LU(d, n):
    L = sp.csc_matrix((np.array(d["L_data"]), np.array(d["L_indices"]), np.array(d["L_indptr"])), shape=(n, n))
    U = sp.csc_matrix((np.array(d["U_data"]), np.array(d["U_indices"]), np.array(d["U_indptr"])), shape=(n, n))
    return L, U


def _berr(L, U, X, B, trans):
    """max over columns of ||b - M x|| / (||L|| ||U|| ||x|| + ||b||), M = L U, (L U)^T or (L U)^H, L with a unit diagonal."""
    n = L.shape[0]
    Lu = sp.tril(L, -1, format="csc") + sp.identity(n, format="csc")
    M = Lu @ U
    if trans == 1:
        M = M.T
    elif trans == 2:
        M = M.conj().T
    X = X.reshape(n, -1)
    B = B.reshape(n, -1)
    nl, nu = sp.linalg.norm(Lu), sp.linalg.norm(U)
    return max(np.linalg.norm(B[:, r] - M @ X[:, r]) / (nl * nu * np.linalg.norm(X[:, r]) + np.linalg.norm(B[:, r]))
               for r in range(X.shape[1]))


def _rhs(n, nrhs, cplx, seed):
    rng = np.random.default_rng(seed)
    B = rng.standard_normal((n, nrhs))
    return B + 1j * rng.standard_normal((n, nrhs)) if cplx else B


@pytest.mark.parametrize("name", sorted(CASES))
def test_factor_sn_perm_matches_oracle(gpu, name):
    n, Ap, Ai, Ax = CASES[name]()
    cplx = np.iscomplexobj(Ax)
    S = F.analyze(n, Ap, Ai)
    d = F.factor_sn_perm(Ax, Ai, Ap, n, S.row_perm, S.col_perm, cplx)
    orc = O.OracleLU(n, Ap, Ai, Ax, S.row_perm, S.col_perm)
    assert np.array_equal(d["p"], orc.p_lu), "pivot order differs from the oracle"
    assert np.array_equal(d["q"], np.arange(n))
    assert np.array_equal(d["Dr"], orc.Drp) and np.array_equal(d["Dc"], orc.Dcp), "Ruiz scalings are not bit-identical"
    L, U = _LU(d, n)
    assert _rel(L, orc.L) <= FACTOR_TOL, f"L differs by {_rel(L, orc.L):.2e}"
    assert _rel(U, orc.U) <= FACTOR_TOL, f"U differs by {_rel(U, orc.U):.2e}"


@pytest.mark.parametrize("name", ["convdiff2d_g20", "hard_real_300", "hard_cplx_300_s0"])
def test_factor_sn_perm_with_caller_orders(gpu, name):
    """Orders the analysis did not make (random permutations; the dense lines of the hard matrices land anywhere).
    Where the oracle finds no admissible pivot (hard_real_300 without equilibration, step 199), the GPU path reports the
    same error at the same step."""
    n, Ap, Ai, Ax = CASES[name]()
    cplx = np.iscomplexobj(Ax)
    rng = np.random.default_rng(5)
    rp, cp = rng.permutation(n), rng.permutation(n)
    for equilibrate in (1, 0):
        try:
            orc = O.OracleLU(n, Ap, Ai, Ax, rp, cp, equilibrate=equilibrate)
        except RuntimeError as e:
            step = re.search(r"at step (\d+)", str(e)).group(1)
            with pytest.raises(F.FplusError) as g:
                F.factor_sn_perm(Ax, Ai, Ap, n, rp, cp, cplx, equilibrate=equilibrate)
            assert g.value.code == F.FPLUS_ERR_SINGULAR and f"at step {step} " in str(g.value)
            continue
        d = F.factor_sn_perm(Ax, Ai, Ap, n, rp, cp, cplx, equilibrate=equilibrate)
        assert np.array_equal(d["p"], orc.p_lu)
        assert np.array_equal(d["Dr"], orc.Drp) and np.array_equal(d["Dc"], orc.Dcp)
        if not equilibrate:
            assert np.all(d["Dr"] == 1.0) and np.all(d["Dc"] == 1.0)
        L, U = _LU(d, n)
        assert _rel(L, orc.L) <= FACTOR_TOL and _rel(U, orc.U) <= FACTOR_TOL


def test_factor_sn_sym_and_factor_agree_bitwise(gpu):
    n, Ap, Ai, Ax = CASES["pencil_1x64"]()
    S = F.analyze(n, Ap, Ai)
    d1 = F.factor_sn_sym(S, Ax, Ai, Ap, True)
    d2 = F.factor_sn_perm(Ax, Ai, Ap, n, S.row_perm, S.col_perm, True)
    L, U, p_lu = S.factor(Ax).factors()
    for d in (d1, d2):
        Ld, Ud = _LU(d, n)
        assert np.array_equal(d["p"], p_lu)
        assert (Ld != L).nnz == 0 and (Ud != U).nnz == 0
    assert np.array_equal(d1["Dr"], d2["Dr"]) and np.array_equal(d1["Dc"], d2["Dc"])


@pytest.mark.parametrize("name", ["convdiff2d_g20", "pencil_1x64", "hard_cplx_300", "banded_cplx_1200"])
def test_plan_solve_on_returned_factors(gpu, name):
    """The arrays fplus_factor_sn_perm returned: the plan finds the device copy (nsupernodes > 0); a plan on copies of
    the same arrays takes the sweeps (nsupernodes -1); both solve to backward error <= 1e-13, also two calls in a row."""
    n, Ap, Ai, Ax = CASES[name]()
    cplx = np.iscomplexobj(Ax)
    S = F.analyze(n, Ap, Ai)
    d = F.factor_sn_perm(Ax, Ai, Ap, n, S.row_perm, S.col_perm, cplx)
    arrays = [d[k] for k in ("L_indptr", "L_indices", "L_data", "U_indptr", "U_indices", "U_data")]
    Lp, Li, Lx, Up, Ui, Ux = arrays
    L, U = _LU(d, n)
    pl = F.solve_plan(Lp, Li, Up, Ui)
    assert pl.nsupernodes > 0
    copies = [np.array(a, copy=True) for a in arrays]
    pl2 = F.solve_plan(copies[0], copies[1], copies[3], copies[4])
    assert pl2.nsupernodes == -1
    B = _rhs(n, 3, cplx, 2)
    for trans in ((0, 1, 2) if cplx else (0, 1)):
        X = F.lu_solve_plan(pl, Lp, Li, Lx, Up, Ui, Ux, B, trans, cplx)
        assert _berr(L, U, X, B, trans) <= SOLVE_BERR, f"device path, trans {trans}"
        X1 = F.lu_solve_plan(pl, Lp, Li, Lx, Up, Ui, Ux, B, trans, cplx)
        assert np.array_equal(X, X1)
        X2 = F.lu_solve_plan(pl2, *copies, B, trans, cplx)
        assert _berr(L, U, X2, B, trans) <= SOLVE_BERR, f"sweeps, trans {trans}"
        assert np.linalg.norm(X2 - X) <= 1e-8 * np.linalg.norm(X)
    x1 = F.lu_solve(Lp, Li, Lx, Up, Ui, Ux, B[:, 0], 0, cplx)
    assert _berr(L, U, x1, B[:, 0], 0) <= SOLVE_BERR


def test_plan_solve_after_values_change(gpu):
    """Values of the returned arrays scaled in place: the solve uses the arrays as they are now."""
    n, Ap, Ai, Ax = CASES["convdiff2d_g20"]()
    S = F.analyze(n, Ap, Ai)
    d = F.factor_sn_perm(Ax, Ai, Ap, n, S.row_perm, S.col_perm, False)
    pl = F.solve_plan(d["L_indptr"], d["L_indices"], d["U_indptr"], d["U_indices"])
    assert pl.nsupernodes > 0
    d["U_data"][:] *= 2.0
    L, U = _LU(d, n)
    B = _rhs(n, 2, False, 4)
    X = F.lu_solve_plan(pl, d["L_indptr"], d["L_indices"], d["L_data"], d["U_indptr"], d["U_indices"], d["U_data"], B, 0, False)
    assert _berr(L, U, X, B, 0) <= SOLVE_BERR


def _random_factors(n, cplx, seed, density, dense_row=True):
    """Unit lower L (its diagonal stored first in every column) and upper U with a dominant diagonal, random patterns."""
    rng = np.random.default_rng(seed)

    def vals(k):
        v = rng.standard_normal(k) * 0.3
        return v + 1j * rng.standard_normal(k) * 0.3 if cplx else v

    Ls = sp.random(n, n, density=density, random_state=rng, format="csc")
    Ls = sp.tril(Ls, -1, format="csc")
    if dense_row:                      # the last row reads every column: one deep level
        Ls = Ls + sp.csc_matrix((np.ones(n - 1), (np.full(n - 1, n - 1), np.arange(n - 1))), shape=(n, n))
    Ls = sp.csc_matrix((vals(Ls.nnz), Ls.indices, Ls.indptr), shape=(n, n))
    L = (Ls + sp.identity(n, format="csc")).tocsc()
    L.sort_indices()
    Us = sp.triu(sp.random(n, n, density=density, random_state=rng, format="csc"), 1, format="csc")
    Us = sp.csc_matrix((vals(Us.nnz), Us.indices, Us.indptr), shape=(n, n))
    d = 2.0 + rng.random(n)
    U = (Us + sp.diags(d + (1j * rng.random(n) if cplx else 0), format="csc")).tocsc()
    U.sort_indices()
    return L, U


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("n,density", [(1500, 0.003), (20000, 0.00005)])
def test_sweeps_on_other_factors(gpu, cplx, n, density):
    """Level-scheduled sweeps on CSC factors from elsewhere: a few deep levels (the dense last row) and, at n = 20000,
    levels wider than one CTA's run; nrhs 1 and 4; lu_solve (fplus_tri_solve) too."""
    L, U = _random_factors(n, cplx, 21 + n, density)
    args = (L.indptr.astype(np.int64), L.indices.astype(np.int64), L.data, U.indptr.astype(np.int64),
            U.indices.astype(np.int64), U.data)
    pl = F.solve_plan(args[0], args[1], args[3], args[4])
    assert pl.nsupernodes == -1
    for nrhs in (1, 4):
        B = _rhs(n, nrhs, cplx, 9)
        for trans in ((0, 1, 2) if cplx else (0, 1)):
            X = F.lu_solve_plan(pl, *args, B, trans, cplx)
            assert _berr(L, U, X, B, trans) <= SOLVE_BERR, f"nrhs {nrhs} trans {trans}"
    b = _rhs(n, 1, cplx, 10)[:, 0]
    x = F.lu_solve(*args, b, 2 if cplx else 1, cplx)
    assert _berr(L, U, x, b, 2 if cplx else 1) <= SOLVE_BERR


def test_lu_solve_perm_solves_the_original_system(gpu):
    """The low-level chain as FPLUS's Python SparseLU runs it: analyze, factor_sn_perm, solve_plan, then lu_solve_perm
    with p = row_perm[p_lu], q = col_perm, Dr, Dc in original coordinates; the result solves A x = b like fplus_solve."""
    n, Ap, Ai, Ax = CASES["pencil_1x64"]()
    S = F.analyze(n, Ap, Ai)
    rp, cp = S.row_perm, S.col_perm
    d = F.factor_sn_perm(Ax, Ai, Ap, n, rp, cp, True)
    pl = F.solve_plan(d["L_indptr"], d["L_indices"], d["U_indptr"], d["U_indices"])
    p = rp[d["p"]]
    q = cp[d["q"]]
    Dr = np.empty(n); Dr[rp] = d["Dr"]
    Dc = np.empty(n); Dc[cp] = d["Dc"]
    B = _rhs(n, 2, True, 3)
    for trans in (0, 1, 2):
        X = F.lu_solve_perm(pl, d["L_indptr"], d["L_indices"], d["L_data"], d["U_indptr"], d["U_indices"], d["U_data"],
                            B, trans, True, p, q, Dr, Dc)
        Xr = S.factor(Ax).solve(B, trans)
        assert np.linalg.norm(X - Xr) <= 1e-10 * np.linalg.norm(Xr), f"trans {trans}"


@pytest.mark.parametrize("name", ["convdiff2d_g20", "hard_real_300", "hard_cplx_300", "pencil_1x64"])
@pytest.mark.parametrize("is_csc", [1, 0])
def test_ruiz_matches_reference_bitwise(gpu, name, is_csc):
    """fplus_ruiz on the GPU against the reference's own fplus_ruiz (oracle/_ref), CSC and CSR routes: Dr, Dc and the
    scaled values bit-identical."""
    if not O.have_reference():
        pytest.skip("oracle/_ref (the reference build) is not present")
    n, Ap, Ai, Ax = CASES[name]()
    cplx = np.iscomplexobj(Ax)
    A = sp.csc_matrix((Ax, Ai, Ap), shape=(n, n))
    M = A if is_csc else A.tocsr()
    M.sort_indices()
    ptr, idx = M.indptr.astype(np.int64), M.indices.astype(np.int64)
    got = F.ruiz_equilibrate(M.data, idx, ptr, n, 20, 1e-2, cplx, 0, is_csc)
    R = O.reference()
    x = np.array(M.data, dtype=np.complex128 if cplx else np.float64, copy=True)
    Dr, Dc = np.empty(n), np.empty(n)
    err = ctypes.create_string_buffer(256)
    assert R.fplus_ruiz(n, F._p64(ptr), F._p64(idx), x.ctypes.data_as(ctypes.c_void_p), int(cplx), is_csc, 20, 1e-2, 0,
                        Dr.ctypes.data_as(F._dp), Dc.ctypes.data_as(F._dp), err, 256) == 0
    assert np.array_equal(got["Dr"], Dr) and np.array_equal(got["Dc"], Dc)
    assert np.array_equal(got["data"].view(np.float64), x.view(np.float64))


def test_ruiz_range_guard_matches_reference(gpu):
    """Entries above 2^500: the reference's power-of-two pre-scaling, folded back into Dr and Dc."""
    if not O.have_reference():
        pytest.skip("oracle/_ref (the reference build) is not present")
    n, Ap, Ai, Ax = CASES["convdiff2d_g20"]()
    Ax = Ax * np.where(np.arange(Ax.shape[0]) % 2, 2.0 ** 510, 2.0 ** -5)
    got = F.ruiz_equilibrate(Ax, Ai, Ap, n, 20, 1e-2, False, 0, 1)
    R = O.reference()
    x = Ax.copy()
    Dr, Dc = np.empty(n), np.empty(n)
    err = ctypes.create_string_buffer(256)
    rc = R.fplus_ruiz(n, F._p64(Ap.astype(np.int64)), F._p64(Ai.astype(np.int64)), x.ctypes.data_as(ctypes.c_void_p), 0, 1, 20,
                      1e-2, 0, Dr.ctypes.data_as(F._dp), Dc.ctypes.data_as(F._dp), err, 256)
    assert rc == 0
    assert np.array_equal(got["Dr"], Dr) and np.array_equal(got["Dc"], Dc) and np.array_equal(got["data"], x)


@pytest.mark.parametrize("name", ["convdiff2d_g20", "pencil_1x64", "hard_cplx_300"])
@pytest.mark.parametrize("colamd", [True, False])
def test_sparse_lu(gpu, name, colamd):
    """FPLUS's SparseLU interface: with colamd (the analysis' orders) and without (the identity orders, FPLUS's default),
    perm_r / perm_c and L, U as the oracle's with the same orders, and solves for 'N', 'T', 'H'."""
    n, Ap, Ai, Ax = CASES[name]()
    cplx = np.iscomplexobj(Ax)
    A = sp.csc_matrix((Ax, Ai, Ap), shape=(n, n))
    lu = F.SparseLU(A, colamd=colamd, pin_dense_rows=True)
    if colamd:
        S = F.analyze(n, Ap, Ai)
        rp, cp = S.row_perm, S.col_perm
    else:
        rp = cp = np.arange(n)
    orc = O.OracleLU(n, Ap, Ai, Ax, rp, cp)
    assert np.array_equal(lu.perm_r, orc.p) and np.array_equal(lu.perm_c, orc.q)
    assert _rel(lu.L, orc.L) <= FACTOR_TOL and _rel(lu.U, orc.U) <= FACTOR_TOL
    assert lu.shape == (n, n) and lu.nnz >= lu.L.nnz
    B = _rhs(n, 2, cplx, 6)
    for trans in ("N", "T", "H"):
        X = lu.solve(B, trans)
        M = A if trans == "N" else (A.T if trans == "T" else A.conj().T)
        be = max(np.linalg.norm(B[:, r] - M @ X[:, r]) / (sp.linalg.norm(A) * np.linalg.norm(X[:, r]) + np.linalg.norm(B[:, r]))
                 for r in range(2))
        assert be <= 1e-13, f"trans {trans}: backward error {be:.2e}"
