"""Parity of the CUDA path (libfplus.so, through the fplus.h C-ABI) with the oracle on the same inputs and orders.

The bar (factor+solve contract): identical pivots; Ruiz scalings Dr, Dc bit-identical; L and U within 1e-12 normwise of
the oracle's; backward error of the solves at most 1e-14 (1e-13 for the 12-decade-scaled test matrices, whose
conditioning the reference's own tests grant 1e-12).
"""
import numpy as np
import pytest
import scipy.sparse as sp

import fplus_b200 as F
from fplus_b200 import workloads as W
import oracle as O
from tests.cases import CASES

pytestmark = pytest.mark.gpu

FACTOR_TOL = 1e-12


def _rel(A, B):
    nb = sp.linalg.norm(B)
    return sp.linalg.norm(A - B) / (nb if nb > 0 else 1.0)


@pytest.fixture(scope="module")
def gpu():
    import torch
    assert torch.cuda.is_available(), "the GPU tests need a CUDA device"
    torch.cuda.init()
    return torch.device("cuda:0")


@pytest.mark.parametrize("name", sorted(CASES))
def test_factor_matches_oracle(gpu, name):
    n, Ap, Ai, Ax = CASES[name]()
    S = F.analyze(n, Ap, Ai)
    N = S.factor(Ax)
    orc = O.OracleLU(n, Ap, Ai, Ax, S.row_perm, S.col_perm)
    assert np.array_equal(N.p, orc.p), "pivot order differs from the oracle"
    assert np.array_equal(N.q, orc.q)
    assert np.array_equal(N.Dr, orc.Dr) and np.array_equal(N.Dc, orc.Dc), "Ruiz scalings are not bit-identical"
    L, U, p_lu = N.factors()
    assert np.array_equal(p_lu, orc.p_lu)
    assert _rel(L, orc.L) <= FACTOR_TOL, f"L differs by {_rel(L, orc.L):.2e}"
    assert _rel(U, orc.U) <= FACTOR_TOL, f"U differs by {_rel(U, orc.U):.2e}"


@pytest.mark.parametrize("name", sorted(CASES))
def test_solve_backward_error(gpu, name):
    n, Ap, Ai, Ax = CASES[name]()
    cplx = np.iscomplexobj(Ax)
    S = F.analyze(n, Ap, Ai)
    N = S.factor(Ax)
    orc = O.OracleLU(n, Ap, Ai, Ax, S.row_perm, S.col_perm)
    rng = np.random.default_rng(7)
    nrhs = 3
    B = rng.standard_normal((n, nrhs)) + (1j * rng.standard_normal((n, nrhs)) if cplx else 0)
    tol = 1e-13 if name.startswith("hard") else 1e-14
    for trans in ((0, 1, 2) if cplx else (0, 1)):
        X = N.solve(B, trans)
        Xo = orc.solve(B, trans)
        for r in range(nrhs):
            be = O.backward_error(n, Ap, Ai, Ax, X[:, r], B[:, r], trans)
            assert be <= tol, f"trans {trans} rhs {r}: backward error {be:.2e}"
        d = np.linalg.norm(X - Xo) / np.linalg.norm(Xo)
        assert d < 1e-8, f"trans {trans}: differs from the oracle's solve by {d:.1e}"


def test_dense_row_pivot_restarts_with_chain(gpu):
    """A dense row chosen as pivot inside the interior fronts: the factorization is redone with the dense chain from that
    front and the pivots still match the oracle."""
    n, Ap, Ai, Ax = CASES["pencil_1x64"]()
    S = F.analyze(n, Ap, Ai)
    N = S.factor(Ax)
    info = N.info
    assert info["attempts"] == 2 and info["f_dense"] < n - S.n_dense_cols
    N2 = S.factor(Ax * (1 + 0.25j))          # the same pattern again: the chain start is remembered
    assert N2.info["attempts"] == 1
    orc = O.OracleLU(n, Ap, Ai, Ax * (1 + 0.25j), S.row_perm, S.col_perm)
    assert np.array_equal(N2.p, orc.p)


def test_several_rhs_and_leading_dimension(gpu):
    n, Ap, Ai, Ax = CASES["banded_cplx_1200"]()
    S = F.analyze(n, Ap, Ai)
    N = S.factor(Ax)
    rng = np.random.default_rng(3)
    nrhs, ldb = 37, n + 5                      # more than one group of 32, padded leading dimension
    Bfull = rng.standard_normal((ldb, nrhs)) + 1j * rng.standard_normal((ldb, nrhs))
    B = np.asfortranarray(Bfull.copy())
    import ctypes
    err = ctypes.create_string_buffer(256)
    rc = F.lib().fplus_solve(N._h, B.ctypes.data_as(ctypes.c_void_p), nrhs, ldb, 0, err, 256)
    assert rc == 0, err.value
    X1 = N.solve(Bfull[:n, :], 0)
    assert np.array_equal(B[:n, :], X1), "solving with ldb > n changed the result"
    assert np.array_equal(B[n:, :], Bfull[n:, :]), "rows beyond n were written"
    cols = np.column_stack([N.solve(Bfull[:n, k], 0) for k in range(nrhs)])
    assert np.allclose(cols, X1, rtol=0, atol=1e-12 * np.abs(X1).max())


def test_singular_matrix_reports_singular(gpu):
    # [[1, 1], [1, 1]]: an exact LU fails (tests/c/test_fplus.c:226-228)
    Ap = np.array([0, 2, 4]); Ai = np.array([0, 1, 0, 1]); Ax = np.array([1.0, 1.0, 1.0, 1.0])
    S = F.analyze(2, Ap, Ai, pin_dense=0, equilibrate=0)
    with pytest.raises(F.FplusError) as e:
        S.factor(Ax)
    assert e.value.code == F.FPLUS_ERR_SINGULAR


def test_zero_row_reported_by_equilibration(gpu):
    # a structurally present but numerically zero row: Ruiz reports it (FPLUS src/equil.c:276-284)
    Ap = np.array([0, 2, 4]); Ai = np.array([0, 1, 0, 1]); Ax = np.array([1.0, 0.0, 2.0, 0.0])
    S = F.analyze(2, Ap, Ai)
    with pytest.raises(F.FplusError) as e:
        S.factor(Ax)
    assert e.value.code == F.FPLUS_ERR_SINGULAR and "Row 1" in str(e.value)


def test_example_program_values(gpu):
    """The reference's example (examples/solve.c): x = (1, 1, 1) for A and A^H."""
    Ap = np.array([0, 2, 5, 7]); Ai = np.array([0, 1, 0, 1, 2, 1, 2])
    Ax = np.array([4, 1j, 1, 3, 2, 1, 5], dtype=complex)
    S = F.analyze(3, Ap, Ai)
    N = S.factor(Ax)
    assert np.allclose(N.solve(np.array([5, 4 + 1j, 7]), 0), 1.0, atol=1e-14)
    assert np.allclose(N.solve(np.array([4 - 1j, 6, 6]), 2), 1.0, atol=1e-14)


def test_device_resident_entry_points(gpu):
    import torch
    n, Ap, Ai, Ax = CASES["convdiff2d_g20"]()
    S = F.analyze(n, Ap, Ai)
    Ad = torch.from_numpy(Ax).to(gpu)
    Nd = S.factor(Ad, device=True)
    Nh = S.factor(Ax)
    assert np.array_equal(Nd.p, Nh.p)
    b = np.random.default_rng(5).standard_normal(n)
    bd = torch.from_numpy(b.copy()).to(gpu)
    Nd.solve_device(bd, 0)
    assert np.array_equal(bd.cpu().numpy(), Nh.solve(b, 0))


def test_batch_factor_and_solve_match_single(gpu):
    """fplus_b200_factor_batch / solve_batch: shifts A - sigma_k B of one analysed pattern and a second pattern in the same
    batch, factored and solved concurrently, give exactly the results of the one-by-one calls."""
    mats = [W.pencil(modes=1, nc=64, sigma=0.3 + 1.7j + 0.1 * k) for k in range(4)]
    mats.append(W.pencil(modes=2, nc=64, sigma=0.5 + 1.0j))
    S0 = F.analyze(*mats[0][:3])
    S1 = F.analyze(*mats[4][:3])
    syms = [S0, S0, S0, S0, S1]
    Ns = F.factor_batch(syms, [m[3] for m in mats], nworkers=3)
    rng = np.random.default_rng(3)
    bs = [rng.standard_normal((m[0], 2)) + 1j * rng.standard_normal((m[0], 2)) for m in mats]
    Xs = F.solve_batch(Ns, bs, trans=0, nworkers=3)
    for k, (m, S) in enumerate(zip(mats, syms)):
        N1 = S.factor(m[3])
        assert np.array_equal(Ns[k].p, N1.p), f"matrix {k}: pivots differ"
        Lb, Ub, _ = Ns[k].factors()
        L1, U1, _ = N1.factors()
        assert np.array_equal(Lb.data, L1.data) and np.array_equal(Ub.data, U1.data), f"matrix {k}: factors differ"
        X1 = N1.solve(bs[k])
        assert np.array_equal(Xs[k], X1), f"matrix {k}: solutions differ"
        for r in range(2):
            assert O.backward_error(m[0], m[1], m[2], m[3], Xs[k][:, r], bs[k][:, r]) <= 1e-14


def test_chain_solve_many_rhs(gpu):
    """A pencil (dense chain: the column-oriented backward sweep) with 20 right-hand sides (more than one warp's worth per
    sweep CTA): every column at backward error <= 1e-14, and each equal within rounding to its own one-column solve."""
    n, Ap, Ai, Ax = CASES["pencil_2x256"]()
    S = F.analyze(n, Ap, Ai)
    N = S.factor(Ax)
    assert N.info["f_dense"] < n, "the case should factor with a dense chain"
    rng = np.random.default_rng(9)
    B = rng.standard_normal((n, 20)) + 1j * rng.standard_normal((n, 20))
    for trans in (0, 1, 2):
        X = N.solve(B, trans)
        for r in range(20):
            assert O.backward_error(n, Ap, Ai, Ax, X[:, r], B[:, r], trans) <= 1e-14
        x3 = N.solve(B[:, 3], trans)
        assert np.allclose(X[:, 3], x3, rtol=0, atol=1e-12 * np.abs(x3).max())


def _cw_berr(A, x, b):
    """componentwise backward error max_i |b - A x|_i / (|A| |x| + |b|)_i, in numpy"""
    r = b - A @ x
    den = abs(A) @ np.abs(x) + np.abs(b)
    with np.errstate(divide="ignore", invalid="ignore"):
        q = np.where(den > 0, np.abs(r) / den, np.where(np.abs(r) > 0, np.inf, 0.0))
    return q.max()


@pytest.mark.parametrize("name", ["hard_real_300", "hard_cplx_300", "convdiff2d_g100", "pencil_1x64", "banded_cplx_1200"])
def test_solve_refine(gpu, name):
    """fplus_b200_solve_refine: with max_iter 0 it returns fplus_solve's solution and its backward error; refinement
    brings the componentwise backward error, measured here, to the FP64 floor and never above the unrefined one."""
    n, Ap, Ai, Ax = CASES[name]()
    cplx = np.iscomplexobj(Ax)
    S = F.analyze(n, Ap, Ai)
    N = S.factor(Ax)
    A = sp.csc_matrix((Ax, Ai, Ap), shape=(n, n))
    rng = np.random.default_rng(17)
    B = rng.standard_normal((n, 3)) + (1j * rng.standard_normal((n, 3)) if cplx else 0)
    for trans in ((0, 1, 2) if cplx else (0, 1)):
        M = A if trans == 0 else (A.T if trans == 1 else A.conj().T)
        X0 = N.solve(B, trans)
        Xz, bz, iz = N.solve_refine(B, trans, max_iter=0)
        assert np.array_equal(Xz, X0) and np.all(iz == 0)
        Xr, br, ir = N.solve_refine(B, trans)
        assert np.all(br <= bz) and np.all(ir >= 0) and np.all(ir <= 10)
        for r in range(3):
            c0, cr = _cw_berr(M, X0[:, r], B[:, r]), _cw_berr(M, Xr[:, r], B[:, r])
            assert bz[r] <= max(2 * c0, 1e-15) and c0 <= max(2 * bz[r], 1e-15), f"device {bz[r]:.2e} vs numpy {c0:.2e}"
            assert cr <= max(1e-15, 2 * c0), f"trans {trans} rhs {r}: refined {cr:.2e}, unrefined {c0:.2e}"


@pytest.mark.parametrize("cplx", [False, True])
def test_large_fronts_all_solve_directions(gpu, cplx):
    """A 32^3 stencil (fronts of up to 256 pivots and thousands of rows: the multi-CTA forward and transposed sweeps):
    every direction solves to a backward error <= 1e-14 and agrees with the oracle's solve."""
    n, Ap, Ai, Ax = W.convdiff3d(32, 3)
    if cplx:
        Ax = Ax + 0.25j * np.random.default_rng(9).uniform(-1, 1, Ax.size)
    S = F.analyze(n, Ap, Ai)
    N = S.factor(Ax)
    B = W.rhs(n, 2, cplx, 8).T.copy(order="F")
    for trans in ((0, 1, 2) if cplx else (0, 1)):
        X = N.solve(B, trans)
        for r in range(2):
            be = O.backward_error(n, Ap, Ai, Ax, X[:, r], B[:, r], trans)
            assert be <= 1e-14, f"trans {trans} rhs {r}: backward error {be:.2e}"


@pytest.mark.parametrize("variant", [1, 3])
@pytest.mark.parametrize("name", ["pencil_1x64", "pencil_2x256", "banded_cplx_1200", "convdiff3d_g12", "hard_cplx_300"])
def test_other_pivot_block_lus_match_oracle(gpu, name, variant):
    """The other pivot-block LU kernels of the small fronts (k_front_lu5: 8-column panels with the later columns' rank-8
    updates on the FP64 tensor cores, the autotuner's other choice; k_front_lu3: blocked panels in FP64 lanes) give the
    oracle's pivots and factors."""
    n, Ap, Ai, Ax = CASES[name]()
    S = F.analyze(n, Ap, Ai)
    S.set_front_shape(256, 64, variant)
    N = S.factor(Ax)
    orc = O.OracleLU(n, Ap, Ai, Ax, S.row_perm, S.col_perm)
    assert np.array_equal(N.p, orc.p)
    L, U, _ = N.factors()
    assert _rel(L, orc.L) <= FACTOR_TOL and _rel(U, orc.U) <= FACTOR_TOL


@pytest.mark.parametrize("variant", [1, 5])
@pytest.mark.parametrize("cplx", [False, True])
def test_tall_pivot_blocks_match_oracle(gpu, cplx, variant):
    """Pivot blocks too large for one CTA (a 20^3 / 16^3 stencil: 256 pivots, hundreds to thousands of rows), pivoted by
    all SMs in one launch (k_block_lu_mc, variant 1) and by one CTA per 32-column panel (variant 5): the oracle's pivots,
    and L and U within 1e-12."""
    g = 16 if cplx else 20
    n, Ap, Ai, Ax = W.convdiff3d(g, 3)
    if cplx:
        Ax = Ax + 0.25j * np.random.default_rng(21).uniform(-1, 1, Ax.size)
    S = F.analyze(n, Ap, Ai)
    S.set_front_shape(256, 64, variant)
    N = S.factor(Ax)
    orc = O.OracleLU(n, Ap, Ai, Ax, S.row_perm, S.col_perm)
    assert np.array_equal(N.p, orc.p), "pivot order differs from the oracle"
    lo, uo = orc.fro_norms()
    lf, uf = N.factor_norms()
    assert abs(lf - lo) <= 1e-12 * lo and abs(uf - uo) <= 1e-12 * uo
    b = W.rhs(n, 1, cplx, 4)[0]
    x = N.solve(b)
    assert O.backward_error(n, Ap, Ai, Ax, x, b) <= 1e-14


@pytest.mark.parametrize("lu", [1, 2])
@pytest.mark.parametrize("cplx", [False, True])
def test_batched_small_fronts_match_front_by_front(gpu, cplx, lu):
    """The small fronts at the bottom of the tree factored level by level (one launch per level for assembly, LU and
    tail) give bit for bit the factors of the front-by-front path (set_front_shape variant + 8), and the oracle's pivots,
    with either pivot-block LU kernel (1: blocked with tensor-core updates, 2: the block in shared memory)."""
    g = 14 if cplx else 18
    n, Ap, Ai, Ax = W.convdiff3d(g, 3)
    if cplx:
        Ax = Ax + 0.25j * np.random.default_rng(23).uniform(-1, 1, Ax.size)
    Ns = []
    for variant in (lu, lu + 8):
        S = F.analyze(n, Ap, Ai)
        S.set_front_shape(256, 64, variant)
        Ns.append((S, S.factor(Ax)))
    (S1, N1), (S2, N2) = Ns
    assert np.array_equal(N1.p, N2.p)
    L1, U1, _ = N1.factors()
    L2, U2, _ = N2.factors()
    assert np.array_equal(L1.data, L2.data) and np.array_equal(U1.data, U2.data), "batched factors differ from front by front"
    orc = O.OracleLU(n, Ap, Ai, Ax, S1.row_perm, S1.col_perm)
    assert np.array_equal(N1.p, orc.p)
    b = W.rhs(n, 2, cplx, 6).T.copy(order="F")
    for trans in ((0, 1, 2) if cplx else (0, 1)):
        X = N1.solve(b, trans)
        for r in range(2):
            assert O.backward_error(n, Ap, Ai, Ax, X[:, r], b[:, r], trans) <= 1e-14


@pytest.mark.parametrize("name", ["pencil_1x64", "pencil_2x256", "banded_cplx_1200"])
def test_chain_tail_forms(gpu, name):
    """The dense chain's tails: the block-inverse products writing the contribution blocks straight into the next
    front's working block (the default), the same through the stack and the extend-add (variant + 32: bit for bit the
    same factors, as the sums are the same), and the 16-row forward substitution (variant + 16): the oracle's pivots and
    L and U within 1e-12 for each."""
    n, Ap, Ai, Ax = CASES[name]()
    S0 = F.analyze(n, Ap, Ai)
    orc = O.OracleLU(n, Ap, Ai, Ax, S0.row_perm, S0.col_perm)
    got = {}
    for variant in (1, 33, 17):
        S = F.analyze(n, Ap, Ai)
        S.set_front_shape(256, 64, variant)
        N = S.factor(Ax)
        assert np.array_equal(N.p, orc.p), f"variant {variant}: pivots differ from the oracle"
        L, U, _ = N.factors()
        assert _rel(L, orc.L) <= FACTOR_TOL and _rel(U, orc.U) <= FACTOR_TOL, f"variant {variant}"
        got[variant] = (L, U)
    assert np.array_equal(got[1][0].data, got[33][0].data) and np.array_equal(got[1][1].data, got[33][1].data), \
        "the direct write changed the factors"
