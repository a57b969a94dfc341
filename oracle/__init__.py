"""TEST INFRASTRUCTURE ONLY -- the CPU checkers of the CUDA path.

* :func:`restatement` -- ``liboracle.so``, this repository's CPU restatement of the FPLUS numeric path (oracle.c).
* :func:`reference`   -- ``_ref/libfplusref.so``, the FPLUS sources themselves compiled by ``oracle/Makefile`` (present
  where the sources were available at build time, or copied along with the repository).

Only the tests, ``__graft_entry__.smoke()`` and the benchmark's CPU-baseline arm import this package.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(_HERE, "liboracle.so")
REF_LIB = os.path.join(_HERE, "_ref", "libfplusref.so")
_i64p = ctypes.POINTER(ctypes.c_int64)
_dp = ctypes.POINTER(ctypes.c_double)


def _arr(p, n, cplx=False):
    if cplx:
        return np.ctypeslib.as_array(ctypes.cast(p, _dp), (2 * n,)).copy().view(np.complex128)
    return np.ctypeslib.as_array(ctypes.cast(p, _dp) if not isinstance(p, ctypes.POINTER(ctypes.c_int64)) else p, (n,)).copy()


class _Orc:
    def __init__(self):
        L = ctypes.CDLL(ORACLE_LIB)
        for f in ("orc_Lp", "orc_Li", "orc_Up", "orc_Ui", "orc_p_lu", "orc_p", "orc_q", "orc_Bp", "orc_Bi"):
            getattr(L, f).restype = _i64p
            getattr(L, f).argtypes = [ctypes.c_void_p]
        for f in ("orc_Lx", "orc_Ux", "orc_Bx"):
            getattr(L, f).restype = ctypes.c_void_p
            getattr(L, f).argtypes = [ctypes.c_void_p]
        for f in ("orc_Dr", "orc_Dc", "orc_Drp", "orc_Dcp"):
            getattr(L, f).restype = _dp
            getattr(L, f).argtypes = [ctypes.c_void_p]
        L.orc_factor.argtypes = [ctypes.c_int64, _i64p, _i64p, ctypes.c_void_p, ctypes.c_int, _i64p, _i64p, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_void_p),
                                 ctypes.c_char_p, ctypes.c_size_t]
        L.orc_solve.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int]
        L.orc_free.argtypes = [ctypes.c_void_p]
        L.orc_ruiz_iters.argtypes = [ctypes.c_void_p]
        L.orc_ruiz.argtypes = [ctypes.c_int64, _i64p, _i64p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                               _dp, _dp, ctypes.POINTER(ctypes.c_int), ctypes.c_char_p, ctypes.c_size_t]
        self.L = L


_orc = None


def restatement():
    global _orc
    if _orc is None:
        _orc = _Orc()
    return _orc.L


class OracleLU:
    """orc_factor / orc_solve on one matrix with given static orders."""

    def __init__(self, n, Ap, Ai, Ax, row_perm, col_perm, equilibrate=1, ruiz_max_iter=20, ruiz_tol=1e-2,
                 pivot_rel=1.4901161193847656e-08):
        L = restatement()
        self.n = n
        self.cplx = np.iscomplexobj(Ax)
        self._keep = [np.ascontiguousarray(a) for a in (Ap, Ai, Ax, row_perm, col_perm)]
        Ap, Ai, Ax, rp, cp = self._keep
        self._h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        rc = L.orc_factor(n, Ap.ctypes.data_as(_i64p), Ai.ctypes.data_as(_i64p), Ax.ctypes.data_as(ctypes.c_void_p),
                          int(self.cplx), rp.ctypes.data_as(_i64p), cp.ctypes.data_as(_i64p), int(equilibrate), int(ruiz_max_iter),
                          float(ruiz_tol), float(pivot_rel), ctypes.byref(self._h), err, 512)
        self.rc, self.err = rc, err.value.decode(errors="replace")
        if rc != 0:
            raise RuntimeError(f"oracle factor failed ({rc}): {self.err}")

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value:
            restatement().orc_free(self._h)

    def _csc(self, fp, fi, fx):
        import scipy.sparse as sp
        L = restatement()
        n = self.n
        p = np.ctypeslib.as_array(getattr(L, fp)(self._h), (n + 1,)).copy()
        nnz = int(p[-1])
        i = np.ctypeslib.as_array(getattr(L, fi)(self._h), (max(nnz, 1),))[:nnz].copy()
        raw = np.ctypeslib.as_array(ctypes.cast(getattr(L, fx)(self._h), _dp), (max(nnz, 1) * (2 if self.cplx else 1),))
        x = raw[: nnz * (2 if self.cplx else 1)].copy()
        if self.cplx:
            x = x.view(np.complex128)
        return sp.csc_matrix((x, i, p), shape=(n, n))

    def _fro(self, fp, fx):
        L = restatement()
        nnz = int(np.ctypeslib.as_array(getattr(L, fp)(self._h), (self.n + 1,))[-1])
        raw = np.ctypeslib.as_array(ctypes.cast(getattr(L, fx)(self._h), _dp), (max(nnz, 1) * (2 if self.cplx else 1),))
        v = raw[: nnz * (2 if self.cplx else 1)]
        m = float(np.abs(v).max()) if v.size else 0.0
        return m * float(np.linalg.norm(v / m)) if m > 0 else 0.0        # scaled: the squares neither overflow nor underflow

    def fro_norms(self):
        """(||L||_F, ||U||_F) straight from the factor arrays (no copies: for factors too large to convert)."""
        return self._fro("orc_Lp", "orc_Lx"), self._fro("orc_Up", "orc_Ux")

    @property
    def L(self):
        return self._csc("orc_Lp", "orc_Li", "orc_Lx")

    @property
    def U(self):
        return self._csc("orc_Up", "orc_Ui", "orc_Ux")

    @property
    def B(self):
        return self._csc("orc_Bp", "orc_Bi", "orc_Bx")

    def _v(self, f, dt=np.int64):
        L = restatement()
        return np.ctypeslib.as_array(getattr(L, f)(self._h), (self.n,)).copy()

    @property
    def p_lu(self):
        return self._v("orc_p_lu")

    @property
    def p(self):
        return self._v("orc_p")

    @property
    def q(self):
        return self._v("orc_q")

    @property
    def Dr(self):
        return self._v("orc_Dr")

    @property
    def Dc(self):
        return self._v("orc_Dc")

    @property
    def Drp(self):
        return self._v("orc_Drp")

    @property
    def Dcp(self):
        return self._v("orc_Dcp")

    @property
    def ruiz_iters(self):
        return int(restatement().orc_ruiz_iters(self._h))

    def solve(self, b, trans=0):
        b = np.asarray(b)
        one = b.ndim == 1
        X = np.array(b.reshape(self.n, -1), dtype=np.complex128 if self.cplx else np.float64, order="F", copy=True)
        rc = restatement().orc_solve(self._h, X.ctypes.data_as(ctypes.c_void_p), X.shape[1], self.n, trans)
        if rc != 0:
            raise RuntimeError(f"oracle solve failed ({rc})")
        return X[:, 0] if one else X


# ---------------------------------------------------------------------------------------------------------------- reference
class _RefOpt(ctypes.Structure):
    _fields_ = [("pin_dense", ctypes.c_int), ("tau_density", ctypes.c_double), ("tau_min_nnz", ctypes.c_int64),
                ("postorder", ctypes.c_int), ("equilibrate", ctypes.c_int), ("ruiz_max_iter", ctypes.c_int),
                ("ruiz_tol", ctypes.c_double), ("pivot_rel", ctypes.c_double), ("pivot_strategy", ctypes.c_int),
                ("drop_tol", ctypes.c_double), ("relax_rows", ctypes.c_int64), ("panel", ctypes.c_int64),
                ("use_gpu", ctypes.c_int), ("gpu_min_flops", ctypes.c_double), ("verbose", ctypes.c_int)]


class _RefFactors(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("is_complex", ctypes.c_int), ("csc", ctypes.c_int),
                ("Lp", _i64p), ("Li", _i64p), ("Lx", ctypes.c_void_p), ("Up", _i64p), ("Ui", _i64p), ("Ux", ctypes.c_void_p),
                ("p", _i64p), ("q", _i64p), ("nsupernodes", ctypes.c_int64), ("n_pivots_replaced", ctypes.c_int64)]


_ref = None


def have_reference():
    return os.path.exists(REF_LIB)


def reference():
    """The FPLUS sources compiled as oracle/_ref/libfplusref.so (raises when absent)."""
    global _ref
    if _ref is None:
        L = ctypes.CDLL(REF_LIB)
        L.fplusref_inject_order.argtypes = [_i64p, ctypes.c_int64]
        L.fplus_default_options.argtypes = [ctypes.POINTER(_RefOpt)]
        L.fplus_analyze.argtypes = [ctypes.c_int64, _i64p, _i64p, ctypes.c_int, ctypes.c_double, ctypes.c_int64,
                                    ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                    ctypes.c_char_p, ctypes.c_size_t]
        L.fplus_factor.argtypes = [ctypes.c_void_p, _i64p, _i64p, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(_RefOpt),
                                   ctypes.POINTER(ctypes.c_void_p), ctypes.c_char_p, ctypes.c_size_t]
        L.fplus_solve.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                  ctypes.c_char_p, ctypes.c_size_t]
        L.fplus_numeric_factors.argtypes = [ctypes.c_void_p]
        L.fplus_numeric_factors.restype = ctypes.POINTER(_RefFactors)
        for f in ("fplus_numeric_p", "fplus_numeric_q", "fplus_symbolic_row_perm", "fplus_symbolic_col_perm"):
            getattr(L, f).argtypes = [ctypes.c_void_p]
            getattr(L, f).restype = _i64p
        for f in ("fplus_numeric_Dr", "fplus_numeric_Dc"):
            getattr(L, f).argtypes = [ctypes.c_void_p]
            getattr(L, f).restype = _dp
        L.fplus_numeric_free.argtypes = [ctypes.c_void_p]
        L.fplus_symbolic_free.argtypes = [ctypes.c_void_p]
        L.fplus_coletree_postorder.argtypes = [ctypes.c_int64, ctypes.c_int64, _i64p, _i64p, _i64p]
        L.fplus_ruiz.argtypes = [ctypes.c_int64, _i64p, _i64p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_double, ctypes.c_int, _dp, _dp, ctypes.c_char_p, ctypes.c_size_t]
        _ref = L
    return _ref


class RefLU:
    """The reference's own fplus_analyze (with an injected fill-reducing order) + fplus_factor + fplus_solve."""

    def __init__(self, n, Ap, Ai, Ax, inject_order, tau_row_mask=None, tau_col_mask=None, postorder=1, pin_dense=1,
                 **opts):
        L = reference()
        self.n, self.cplx = n, np.iscomplexobj(Ax)
        self._keep = [None if a is None else np.ascontiguousarray(a) for a in (Ap, Ai, Ax)]
        Ap, Ai, Ax = self._keep
        inj = np.ascontiguousarray(inject_order, dtype=np.int64)
        L.fplusref_inject_order(inj.ctypes.data_as(_i64p), n)
        tr = None if tau_row_mask is None else np.ascontiguousarray(tau_row_mask, np.uint8)
        tc = None if tau_col_mask is None else np.ascontiguousarray(tau_col_mask, np.uint8)
        self._keep += [tr, tc]
        self._sym = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        rc = L.fplus_analyze(n, Ap.ctypes.data_as(_i64p), Ai.ctypes.data_as(_i64p), pin_dense, 0.5, 10,
                             None if tr is None else tr.ctypes.data_as(ctypes.c_char_p),
                             None if tc is None else tc.ctypes.data_as(ctypes.c_char_p), postorder, ctypes.byref(self._sym), err, 512)
        if rc != 0:
            raise RuntimeError(f"reference analyze failed ({rc}): {err.value}")
        self.row_perm = np.ctypeslib.as_array(L.fplus_symbolic_row_perm(self._sym), (n,)).copy()
        self.col_perm = np.ctypeslib.as_array(L.fplus_symbolic_col_perm(self._sym), (n,)).copy()
        self._num = ctypes.c_void_p()
        o = _RefOpt()
        L.fplus_default_options(ctypes.byref(o))
        for k, v in opts.items():
            setattr(o, k, v)
        self.opt = o
        if Ax is not None:
            rc = L.fplus_factor(self._sym, Ap.ctypes.data_as(_i64p), Ai.ctypes.data_as(_i64p), Ax.ctypes.data_as(ctypes.c_void_p),
                                int(self.cplx), ctypes.byref(o), ctypes.byref(self._num), err, 512)
            self.rc, self.err = rc, err.value.decode(errors="replace")
            if rc != 0:
                raise RuntimeError(f"reference factor failed ({rc}): {self.err}")

    def refactor(self, Ax):
        """fplus_factor of new values on this analysis (the previous factorization is freed first)."""
        L = reference()
        if self._num.value:
            L.fplus_numeric_free(self._num)
            self._num = ctypes.c_void_p()
        Ap, Ai = self._keep[0], self._keep[1]
        self.cplx = np.iscomplexobj(Ax)
        Ax = np.ascontiguousarray(Ax)
        self._keep[2] = Ax
        err = ctypes.create_string_buffer(512)
        rc = L.fplus_factor(self._sym, Ap.ctypes.data_as(_i64p), Ai.ctypes.data_as(_i64p), Ax.ctypes.data_as(ctypes.c_void_p),
                            int(self.cplx), ctypes.byref(self.opt), ctypes.byref(self._num), err, 512)
        if rc != 0:
            raise RuntimeError(f"reference factor failed ({rc}): {err.value}")

    def __del__(self):
        L = _ref
        if L is None:
            return
        if getattr(self, "_num", None) and self._num.value:
            L.fplus_numeric_free(self._num)
        if getattr(self, "_sym", None) and self._sym.value:
            L.fplus_symbolic_free(self._sym)

    def factors(self):
        import scipy.sparse as sp
        f = reference().fplus_numeric_factors(self._num).contents
        n = f.n

        def csc(Pp, Pi, Px):
            p = np.ctypeslib.as_array(Pp, (n + 1,)).copy()
            nnz = int(p[-1])
            i = np.ctypeslib.as_array(Pi, (max(nnz, 1),))[:nnz].copy()
            x = np.ctypeslib.as_array(ctypes.cast(Px, _dp), (max(nnz, 1) * (2 if self.cplx else 1),))[: nnz * (2 if self.cplx else 1)].copy()
            if self.cplx:
                x = x.view(np.complex128)
            return sp.csc_matrix((x, i, p), shape=(n, n))
        return csc(f.Lp, f.Li, f.Lx), csc(f.Up, f.Ui, f.Ux), np.ctypeslib.as_array(f.p, (n,)).copy(), int(f.nsupernodes)

    @property
    def p(self):
        return np.ctypeslib.as_array(reference().fplus_numeric_p(self._num), (self.n,)).copy()

    @property
    def Dr(self):
        return np.ctypeslib.as_array(reference().fplus_numeric_Dr(self._num), (self.n,)).copy()

    @property
    def Dc(self):
        return np.ctypeslib.as_array(reference().fplus_numeric_Dc(self._num), (self.n,)).copy()

    def solve(self, b, trans=0):
        b = np.asarray(b)
        one = b.ndim == 1
        X = np.array(b.reshape(self.n, -1), dtype=np.complex128 if self.cplx else np.float64, order="F", copy=True)
        err = ctypes.create_string_buffer(512)
        rc = reference().fplus_solve(self._num, X.ctypes.data_as(ctypes.c_void_p), X.shape[1], self.n, trans, err, 512)
        if rc != 0:
            raise RuntimeError(f"reference solve failed ({rc}): {err.value}")
        return X[:, 0] if one else X


def backward_error(n, Ap, Ai, Ax, x, b, trans=0):
    """||op(A) x - b||_2 / (||A||_1 ||x||_2 + ||b||_2), the reference's definition (tests/c/test_fplus.c:75-89)."""
    import scipy.sparse as sp
    A = sp.csc_matrix((Ax, Ai, Ap), shape=(n, n))
    op = {0: A, 1: A.T, 2: A.conj().T}[trans]
    nA = abs(A).sum(axis=0).max()
    r = op @ x - b
    return float(np.linalg.norm(r) / (nA * np.linalg.norm(x) + np.linalg.norm(b)))
