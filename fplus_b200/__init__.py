"""fplus_b200 -- the FPLUS C interface on B200, for Python callers (ctypes over libfplus.so).

``libfplus.so`` (built by ``__graft_entry__.build()`` / ``make -C fplus_b200/csrc``) serves the unchanged fplus.h
interface (analyze / factor / solve) with every numeric step on the GPU.  This module binds it for the tests and the
benchmark: ``analyze`` -> :class:`Symbolic`, ``Symbolic.factor`` -> :class:`Numeric`, ``Numeric.solve``.  Errors raise
:class:`FplusError` with the library's code and message.  There is no fallback: a missing library or a failing CUDA call
raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfplus.so")

FPLUS_OK, FPLUS_ERR_NOMEM, FPLUS_ERR_SINGULAR, FPLUS_ERR_BADARG, FPLUS_ERR_GPU, FPLUS_ERR_INTERNAL = 0, -1, -2, -3, -4, -5
# the precision form's Schur-update arithmetic (fplus_b200_factor_prec)
PREC_FP64, PREC_FP32, PREC_BF16X3, PREC_TF32 = 0, 1, 2, 3
FPLUS_PIVOT_FULL, FPLUS_PIVOT_PARTIAL, FPLUS_PIVOT_ROOK = 0, 1, 2
FPLUS_PIVOT_REL_DEFAULT = 1.4901161193847656e-08

_i64p = ctypes.POINTER(ctypes.c_int64)
_dp = ctypes.POINTER(ctypes.c_double)


class Options(ctypes.Structure):
    """fplus_options (include/fplus.h), field for field."""
    _fields_ = [("pin_dense", ctypes.c_int), ("tau_density", ctypes.c_double), ("tau_min_nnz", ctypes.c_int64),
                ("postorder", ctypes.c_int), ("equilibrate", ctypes.c_int), ("ruiz_max_iter", ctypes.c_int),
                ("ruiz_tol", ctypes.c_double), ("pivot_rel", ctypes.c_double), ("pivot_strategy", ctypes.c_int),
                ("drop_tol", ctypes.c_double), ("relax_rows", ctypes.c_int64), ("panel", ctypes.c_int64),
                ("use_gpu", ctypes.c_int), ("gpu_min_flops", ctypes.c_double), ("verbose", ctypes.c_int)]


class Factors(ctypes.Structure):
    """fplus_factors (include/fplus.h)."""
    _fields_ = [("n", ctypes.c_int64), ("is_complex", ctypes.c_int), ("csc", ctypes.c_int),
                ("Lp", _i64p), ("Li", _i64p), ("Lx", ctypes.c_void_p), ("Up", _i64p), ("Ui", _i64p), ("Ux", ctypes.c_void_p),
                ("p", _i64p), ("q", _i64p), ("nsupernodes", ctypes.c_int64), ("n_pivots_replaced", ctypes.c_int64)]


class Info(ctypes.Structure):
    """fplus_b200_info (include/fplus_b200.h)."""
    _fields_ = [("n", ctypes.c_int64), ("nfronts", ctypes.c_int64), ("f_dense", ctypes.c_int64), ("attempts", ctypes.c_int),
                ("ruiz_iters", ctypes.c_int), ("nnz_L", ctypes.c_int64), ("nnz_U", ctypes.c_int64),
                ("front_flops", ctypes.c_double), ("ms_equil", ctypes.c_double), ("ms_fronts", ctypes.c_double),
                ("device_bytes", ctypes.c_int64), ("precision", ctypes.c_int), ("reserved", ctypes.c_int),
                ("tc_updates", ctypes.c_int64), ("tc_flops", ctypes.c_double)]


# every entry point of include/fplus.h and include/fplus_b200.h (the tests check that each is exported)
FPLUS_H_SYMBOLS = [
    "fplus_factors_free", "fplus_analyze", "fplus_analyze_ord", "fplus_symbolic_free", "fplus_symbolic_n",
    "fplus_symbolic_nnz", "fplus_symbolic_row_perm", "fplus_symbolic_col_perm", "fplus_symbolic_n_dense_rows",
    "fplus_symbolic_n_dense_cols", "fplus_coletree_postorder", "fplus_default_options", "fplus_analyze_opts",
    "fplus_factor", "fplus_solve", "fplus_numeric_factors", "fplus_numeric_p", "fplus_numeric_q", "fplus_numeric_Dr",
    "fplus_numeric_Dc", "fplus_numeric_free", "fplus_tri_solve", "fplus_solve_plan_create", "fplus_tri_solve_plan",
    "fplus_solve_plan_nsupernodes", "fplus_solve_plan_free", "fplus_factor_sn_perm", "fplus_factor_sn_sym", "fplus_ruiz",
    "fplus_factor_sn", "fplus_factor_row", "fplus_factor_row_perm", "fplus_factor_row_sym",
]
FPLUS_B200_H_SYMBOLS = [
    "fplus_b200_numeric_info", "fplus_b200_use_stream", "fplus_b200_factor_dev", "fplus_b200_solve_dev",
    "fplus_b200_interior_order", "fplus_b200_plan_size", "fplus_b200_plan_export", "fplus_b200_launch_count",
    "fplus_b200_profile", "fplus_b200_profile_read", "fplus_b200_solve_dev_noalloc", "fplus_b200_factor_batch",
    "fplus_b200_solve_batch", "fplus_b200_solve_refine", "fplus_b200_symbolic_from_orders", "fplus_b200_factor_norms",
    "fplus_b200_factor_prec", "fplus_b200_schur_update", "fplus_b200_batch_span_ms", "fplus_b200_graph_create",
    "fplus_b200_graph_values", "fplus_b200_graph_rhs", "fplus_b200_graph_launch", "fplus_b200_graph_status",
    "fplus_b200_graph_free", "fplus_b200_graph_upload", "fplus_b200_graph_download", "fplus_b200_autotune",
    "fplus_b200_set_front_shape",
]

_lib = None


def lib():
    """The loaded libfplus.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FplusError(FPLUS_ERR_INTERNAL, f"{LIB_PATH} is missing: build it with __graft_entry__.build()")
    L = ctypes.CDLL(LIB_PATH)
    L.fplus_default_options.argtypes = [ctypes.POINTER(Options)]
    L.fplus_analyze_opts.argtypes = [ctypes.c_int64, _i64p, _i64p, ctypes.POINTER(Options), ctypes.POINTER(ctypes.c_void_p),
                                     ctypes.c_char_p, ctypes.c_size_t]
    L.fplus_analyze.argtypes = [ctypes.c_int64, _i64p, _i64p, ctypes.c_int, ctypes.c_double, ctypes.c_int64, ctypes.c_char_p,
                                ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), ctypes.c_char_p, ctypes.c_size_t]
    L.fplus_analyze_ord.argtypes = [ctypes.c_int64, _i64p, _i64p, ctypes.c_int, ctypes.c_double, ctypes.c_int64,
                                    ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_void_p), ctypes.c_char_p, ctypes.c_size_t]
    L.fplus_symbolic_free.argtypes = [ctypes.c_void_p]
    for f in ("fplus_symbolic_n", "fplus_symbolic_nnz", "fplus_symbolic_n_dense_rows", "fplus_symbolic_n_dense_cols"):
        getattr(L, f).argtypes = [ctypes.c_void_p]
        getattr(L, f).restype = ctypes.c_int64
    for f in ("fplus_symbolic_row_perm", "fplus_symbolic_col_perm"):
        getattr(L, f).argtypes = [ctypes.c_void_p]
        getattr(L, f).restype = _i64p
    L.fplus_coletree_postorder.argtypes = [ctypes.c_int64, ctypes.c_int64, _i64p, _i64p, _i64p]
    L.fplus_factor.argtypes = [ctypes.c_void_p, _i64p, _i64p, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(Options),
                               ctypes.POINTER(ctypes.c_void_p), ctypes.c_char_p, ctypes.c_size_t]
    L.fplus_b200_factor_dev.argtypes = L.fplus_factor.argtypes
    L.fplus_b200_factor_prec.argtypes = [ctypes.c_void_p, _i64p, _i64p, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(Options),
                                         ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), ctypes.c_char_p,
                                         ctypes.c_size_t]
    L.fplus_solve.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.c_char_p,
                              ctypes.c_size_t]
    L.fplus_b200_solve_dev.argtypes = L.fplus_solve.argtypes
    L.fplus_b200_solve_dev_noalloc.argtypes = L.fplus_solve.argtypes
    L.fplus_b200_factor_batch.argtypes = [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_int, ctypes.POINTER(Options), ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_char_p, ctypes.c_size_t]
    L.fplus_b200_solve_batch.argtypes = [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    L.fplus_numeric_factors.argtypes = [ctypes.c_void_p]
    L.fplus_numeric_factors.restype = ctypes.POINTER(Factors)
    for f in ("fplus_numeric_p", "fplus_numeric_q"):
        getattr(L, f).argtypes = [ctypes.c_void_p]
        getattr(L, f).restype = _i64p
    for f in ("fplus_numeric_Dr", "fplus_numeric_Dc"):
        getattr(L, f).argtypes = [ctypes.c_void_p]
        getattr(L, f).restype = _dp
    L.fplus_numeric_free.argtypes = [ctypes.c_void_p]
    L.fplus_b200_numeric_info.argtypes = [ctypes.c_void_p, ctypes.POINTER(Info)]
    L.fplus_b200_use_stream.argtypes = [ctypes.c_void_p]
    L.fplus_b200_interior_order.argtypes = [ctypes.c_int64, _i64p, _i64p, ctypes.c_char_p, ctypes.c_char_p, _i64p]
    L.fplus_b200_plan_size.argtypes = [ctypes.c_void_p, ctypes.c_int64, _i64p, _i64p, _i64p]
    L.fplus_b200_plan_export.argtypes = [ctypes.c_void_p, ctypes.c_int64, _i64p, _i64p, _i64p, _i64p, _i64p, _i64p]
    L.fplus_b200_launch_count.restype = ctypes.c_longlong
    L.fplus_b200_profile.argtypes = [ctypes.c_int]
    L.fplus_b200_profile_read.argtypes = [ctypes.c_int, _dp, ctypes.POINTER(ctypes.c_longlong), _dp, _dp]
    L.fplus_factors_free.argtypes = [ctypes.POINTER(Factors)]
    L.fplus_b200_symbolic_from_orders.argtypes = [ctypes.c_int64, _i64p, _i64p, _i64p, _i64p, ctypes.POINTER(ctypes.c_void_p),
                                                  ctypes.c_char_p, ctypes.c_size_t]
    L.fplus_b200_schur_update.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                          ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                          ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                          ctypes.c_char_p, ctypes.c_size_t]
    L.fplus_b200_graph_create.argtypes = [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_void_p), ctypes.c_char_p, ctypes.c_size_t]
    for f in ("fplus_b200_graph_values", "fplus_b200_graph_rhs"):
        getattr(L, f).argtypes = [ctypes.c_void_p, ctypes.c_int64]
        getattr(L, f).restype = ctypes.c_void_p
    L.fplus_b200_graph_launch.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    L.fplus_b200_graph_status.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    L.fplus_b200_graph_free.argtypes = [ctypes.c_void_p]
    L.fplus_b200_graph_upload.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p,
                                          ctypes.c_size_t]
    L.fplus_b200_graph_download.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    L.fplus_b200_set_front_shape.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int]
    L.fplus_b200_autotune.argtypes = [ctypes.c_void_p, _i64p, _i64p, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(Options),
                                      ctypes.c_int, _i64p, _i64p, ctypes.POINTER(ctypes.c_int), _dp, ctypes.c_char_p,
                                      ctypes.c_size_t]
    L.fplus_b200_batch_span_ms.argtypes = [ctypes.c_int64, ctypes.c_void_p, _dp, ctypes.c_char_p, ctypes.c_size_t]
    L.fplus_b200_factor_norms.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_char_p, ctypes.c_size_t]
    L.fplus_b200_solve_refine.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_double, _dp, ctypes.POINTER(ctypes.c_int), ctypes.c_char_p,
                                          ctypes.c_size_t]
    _lo = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
           ctypes.c_double, ctypes.c_double, ctypes.POINTER(Factors), _dp, _dp, ctypes.c_char_p, ctypes.c_size_t]
    L.fplus_factor_sn_perm.argtypes = [ctypes.c_int64, _i64p, _i64p, ctypes.c_void_p, ctypes.c_int, _i64p, _i64p] + _lo
    L.fplus_factor_sn_sym.argtypes = [ctypes.c_void_p, _i64p, _i64p, ctypes.c_void_p, ctypes.c_int] + _lo
    L.fplus_factor_sn.argtypes = [ctypes.c_int64, _i64p, _i64p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int64,
                                  ctypes.c_int64, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.POINTER(Factors),
                                  ctypes.c_char_p, ctypes.c_size_t]
    L.fplus_solve_plan_create.argtypes = [ctypes.c_int64, _i64p, _i64p, _i64p, _i64p, ctypes.POINTER(ctypes.c_void_p),
                                          ctypes.c_char_p, ctypes.c_size_t]
    L.fplus_tri_solve_plan.argtypes = [ctypes.c_void_p, ctypes.c_int64, _i64p, _i64p, ctypes.c_void_p, _i64p, _i64p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.c_int]
    L.fplus_tri_solve.argtypes = [ctypes.c_int64, _i64p, _i64p, ctypes.c_void_p, _i64p, _i64p, ctypes.c_void_p,
                                  ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    L.fplus_solve_plan_nsupernodes.argtypes = [ctypes.c_void_p]
    L.fplus_solve_plan_nsupernodes.restype = ctypes.c_int64
    L.fplus_solve_plan_free.argtypes = [ctypes.c_void_p]
    L.fplus_ruiz.argtypes = [ctypes.c_int64, _i64p, _i64p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                             ctypes.c_double, ctypes.c_int, _dp, _dp, ctypes.c_char_p, ctypes.c_size_t]
    _lib = L
    return L


class FplusError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"FPLUS error {code}: {msg}")
        self.code = code


def _check(rc, err):
    if rc != FPLUS_OK:
        raise FplusError(rc, err.value.decode(errors="replace") if err is not None else "")


def _p64(a):
    return a.ctypes.data_as(_i64p)


def default_options(**kw):
    o = Options()
    lib().fplus_default_options(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def csc_arrays(n, Ap, Ai, Ax=None):
    Ap = np.ascontiguousarray(Ap, dtype=np.int64)
    Ai = np.ascontiguousarray(Ai, dtype=np.int64)
    if Ax is not None:
        Ax = np.ascontiguousarray(Ax, dtype=np.complex128 if np.iscomplexobj(Ax) else np.float64)
    return n, Ap, Ai, Ax


class Symbolic:
    """fplus_analyze_opts: the static orders of one pattern (reusable for any values on it)."""

    def __init__(self, n, Ap, Ai, options=None, **kw):
        n, Ap, Ai, _ = csc_arrays(n, Ap, Ai)
        self.n, self.Ap, self.Ai = n, Ap, Ai
        self.options = options if options is not None else default_options(**kw)
        self._h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        _check(lib().fplus_analyze_opts(n, _p64(Ap), _p64(Ai), ctypes.byref(self.options), ctypes.byref(self._h), err, 512), err)

    @classmethod
    def from_orders(cls, n, Ap, Ai, row_perm, col_perm):
        """fplus_b200_symbolic_from_orders: the caller's static orders instead of the analysis."""
        n, Ap, Ai, _ = csc_arrays(n, Ap, Ai)
        rp = np.ascontiguousarray(row_perm, dtype=np.int64)
        cp = np.ascontiguousarray(col_perm, dtype=np.int64)
        if rp.shape[0] != n or cp.shape[0] != n:
            raise ValueError("from_orders: the permutations must have length n")
        self = cls.__new__(cls)
        self.n, self.Ap, self.Ai = n, Ap, Ai
        self.options = default_options()
        self._h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        _check(lib().fplus_b200_symbolic_from_orders(n, _p64(Ap), _p64(Ai), _p64(rp), _p64(cp), ctypes.byref(self._h), err, 512),
               err)
        return self

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None and self._h.value:
            _lib.fplus_symbolic_free(self._h)
            self._h = ctypes.c_void_p()

    @property
    def row_perm(self):
        return np.ctypeslib.as_array(lib().fplus_symbolic_row_perm(self._h), (self.n,)).copy()

    @property
    def col_perm(self):
        return np.ctypeslib.as_array(lib().fplus_symbolic_col_perm(self._h), (self.n,)).copy()

    @property
    def n_dense_rows(self):
        return int(lib().fplus_symbolic_n_dense_rows(self._h))

    @property
    def n_dense_cols(self):
        return int(lib().fplus_symbolic_n_dense_cols(self._h))

    def plan(self, tail=-1):
        """The multifrontal structure (host only): dict of col_front, parent, col_ptr, cols, nrows, nbord, f_dense."""
        nf, nct, fd = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _check(lib().fplus_b200_plan_size(self._h, tail, ctypes.byref(nf), ctypes.byref(nct), ctypes.byref(fd)), None)
        nf, nct = nf.value, nct.value
        out = dict(col_front=np.zeros(self.n, np.int64), parent=np.zeros(nf, np.int64), col_ptr=np.zeros(nf + 1, np.int64),
                   cols=np.zeros(max(nct, 1), np.int64), nrows=np.zeros(nf, np.int64), nbord=np.zeros(nf, np.int64))
        _check(lib().fplus_b200_plan_export(self._h, tail, *(_p64(out[k]) for k in ("col_front", "parent", "col_ptr", "cols",
                                                                                   "nrows", "nbord"))), None)
        out["f_dense"] = fd.value
        return out

    def set_front_shape(self, max_width=256, nb_chain=64, lu_variant=2):
        """fplus_b200_set_front_shape."""
        _check(lib().fplus_b200_set_front_shape(self._h, int(max_width), int(nb_chain), int(lu_variant)), None)

    def autotune(self, Ax, precision=0, options=None):
        """fplus_b200_autotune: time each front shape on these values and keep the fastest; (width, nb, lu, ms)."""
        Ax = np.ascontiguousarray(Ax)
        cplx = np.iscomplexobj(Ax)
        Ax = Ax.astype(np.complex128 if cplx else np.float64, copy=False)
        w, nb, lu, ms = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int(), ctypes.c_double()
        err = ctypes.create_string_buffer(512)
        opts = options if options is not None else self.options
        _check(lib().fplus_b200_autotune(self._h, _p64(self.Ap), _p64(self.Ai), Ax.ctypes.data_as(ctypes.c_void_p), int(cplx),
                                         ctypes.byref(opts), int(precision), ctypes.byref(w), ctypes.byref(nb),
                                         ctypes.byref(lu), ctypes.byref(ms), err, 512), err)
        return w.value, nb.value, lu.value, ms.value

    def factor(self, Ax, options=None, device=False, precision=0):
        """fplus_factor (precision 0), or the precision form (PREC_FP32, PREC_BF16X3, PREC_TF32: fplus_b200_factor_prec)."""
        return Numeric(self, Ax, options, device, precision)


class Numeric:
    """fplus_factor: diag(Dr) A[p,:][:,q] diag(Dc) = L U, the factors in device memory."""

    def __init__(self, sym: Symbolic, Ax, options=None, device=False, precision=0):
        self.sym = sym
        self._h = ctypes.c_void_p()
        opts = options if options is not None else sym.options
        err = ctypes.create_string_buffer(512)
        if device:      # a torch CUDA tensor (float64, or complex128 viewed as float64 pairs)
            self.is_complex = bool(Ax.is_complex())
            ptr = ctypes.c_void_p(Ax.data_ptr())
        else:
            Ax = np.ascontiguousarray(Ax)
            self.is_complex = np.iscomplexobj(Ax)
            Ax = Ax.astype(np.complex128 if self.is_complex else np.float64, copy=False)
            ptr = Ax.ctypes.data_as(ctypes.c_void_p)
        if precision:
            rc = lib().fplus_b200_factor_prec(sym._h, _p64(sym.Ap), _p64(sym.Ai), ptr, int(self.is_complex), ctypes.byref(opts),
                                              int(precision), int(bool(device)), ctypes.byref(self._h), err, 512)
        elif device:
            rc = lib().fplus_b200_factor_dev(sym._h, _p64(sym.Ap), _p64(sym.Ai), ptr, int(self.is_complex), ctypes.byref(opts),
                                             ctypes.byref(self._h), err, 512)
        else:
            rc = lib().fplus_factor(sym._h, _p64(sym.Ap), _p64(sym.Ai), ptr, int(self.is_complex), ctypes.byref(opts),
                                    ctypes.byref(self._h), err, 512)
        _check(rc, err)
        self.n = sym.n

    @classmethod
    def _from_handle(cls, sym, h, is_complex):
        self = cls.__new__(cls)
        self.sym, self._h, self.is_complex, self.n = sym, ctypes.c_void_p(h), bool(is_complex), sym.n
        return self

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None and self._h.value:
            _lib.fplus_numeric_free(self._h)
            self._h = ctypes.c_void_p()

    def solve(self, b, trans=0):
        """x with op(A) x = b (trans 0: A, 1: A^T, 2: A^H); b of shape (n,) or (n, nrhs)."""
        b = np.asarray(b)
        dt = np.complex128 if self.is_complex else np.float64
        one = b.ndim == 1
        X = np.array(b.reshape(self.n, -1), dtype=dt, order="F", copy=True)
        err = ctypes.create_string_buffer(512)
        _check(lib().fplus_solve(self._h, X.ctypes.data_as(ctypes.c_void_p), X.shape[1], self.n, trans, err, 512), err)
        return X[:, 0] if one else X

    def solve_refine(self, b, trans=0, max_iter=10, tol=2.0 ** -52):
        """fplus_b200_solve_refine: (x, berr, iters), with the componentwise backward error and the corrections applied
        per right-hand side."""
        b = np.asarray(b)
        dt = np.complex128 if self.is_complex else np.float64
        one = b.ndim == 1
        X = np.array(b.reshape(self.n, -1), dtype=dt, order="F", copy=True)
        k = X.shape[1]
        berr = np.zeros(max(k, 1))
        iters = np.zeros(max(k, 1), dtype=np.int32)
        err = ctypes.create_string_buffer(512)
        _check(lib().fplus_b200_solve_refine(self._h, X.ctypes.data_as(ctypes.c_void_p), k, self.n, trans, int(max_iter),
                                             float(tol), berr.ctypes.data_as(_dp),
                                             iters.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), err, 512), err)
        return (X[:, 0] if one else X), berr[:k], iters[:k]

    def solve_device(self, B, trans=0):
        """In place on a torch CUDA tensor holding nrhs right-hand sides column-major (shape (nrhs, n), contiguous)."""
        err = ctypes.create_string_buffer(512)
        nrhs = 1 if B.dim() == 1 else B.shape[0]
        _check(lib().fplus_b200_solve_dev(self._h, ctypes.c_void_p(B.data_ptr()), nrhs, self.n, trans, err, 512), err)
        return B

    def factor_norms(self):
        """fplus_b200_factor_norms: (||L||_F, ||U||_F) computed on the GPU from the device factors."""
        lf, uf = ctypes.c_double(), ctypes.c_double()
        err = ctypes.create_string_buffer(512)
        _check(lib().fplus_b200_factor_norms(self._h, ctypes.byref(lf), ctypes.byref(uf), err, 512), err)
        return lf.value, uf.value

    @property
    def info(self):
        I = Info()
        _check(lib().fplus_b200_numeric_info(self._h, ctypes.byref(I)), None)
        return {k: getattr(I, k) for k, _ in Info._fields_}

    @property
    def p(self):
        return np.ctypeslib.as_array(lib().fplus_numeric_p(self._h), (self.n,)).copy()

    @property
    def q(self):
        return np.ctypeslib.as_array(lib().fplus_numeric_q(self._h), (self.n,)).copy()

    @property
    def Dr(self):
        return np.ctypeslib.as_array(lib().fplus_numeric_Dr(self._h), (self.n,)).copy()

    @property
    def Dc(self):
        return np.ctypeslib.as_array(lib().fplus_numeric_Dc(self._h), (self.n,)).copy()

    def factors(self):
        """(L, U, p_lu) of the scaled, permuted matrix as scipy CSC matrices (L unit lower in pivot order)."""
        import scipy.sparse as sp
        fp = lib().fplus_numeric_factors(self._h)
        if not fp:
            raise FplusError(FPLUS_ERR_GPU, "fplus_numeric_factors failed")
        f = fp.contents
        n = f.n
        return (_csc(f.Lp, f.Li, f.Lx, n, f.is_complex), _csc(f.Up, f.Ui, f.Ux, n, f.is_complex),
                np.ctypeslib.as_array(f.p, (n,)).copy())


def _csc(Pp, Pi, Px, n, cplx):
    import scipy.sparse as sp
    p = np.ctypeslib.as_array(Pp, (n + 1,)).copy()
    nnz = int(p[-1])
    i = np.ctypeslib.as_array(Pi, (max(nnz, 1),))[:nnz].copy()
    x = np.ctypeslib.as_array(ctypes.cast(Px, _dp), (max(nnz, 1) * (2 if cplx else 1),))[: nnz * (2 if cplx else 1)].copy()
    if cplx:
        x = x.view(np.complex128)
    return sp.csc_matrix((x, i, p), shape=(n, n))


PROFILE_CLASSES = {0: "schur_gemm", 1: "front_lu", 2: "u12_trsm", 3: "assemble", 4: "front_lu_tall"}


def launch_count() -> int:
    return int(lib().fplus_b200_launch_count())


def profile(on: bool):
    lib().fplus_b200_profile(1 if on else 0)


def profile_read(cls: int):
    ms, fl, by = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    cnt = ctypes.c_longlong()
    _check(lib().fplus_b200_profile_read(cls, ctypes.byref(ms), ctypes.byref(cnt), ctypes.byref(fl), ctypes.byref(by)), None)
    return dict(ms=ms.value, count=cnt.value, flops=fl.value, bytes=by.value)


def analyze(n, Ap, Ai, options=None, **kw) -> Symbolic:
    return Symbolic(n, Ap, Ai, options, **kw)


def factor_batch(syms, Axs, options=None, nworkers=8):
    """fplus_b200_factor_batch: factor matrix k (pattern syms[k], values Axs[k]) for every k, concurrently on the GPU.
    Returns the list of Numeric objects (raises FplusError with the first failure's code and message)."""
    count = len(syms)
    if count != len(Axs):
        raise FplusError(FPLUS_ERR_BADARG, "syms and Axs differ in length")
    cplx = any(np.iscomplexobj(a) for a in Axs)
    vals = [np.ascontiguousarray(a, dtype=np.complex128 if cplx else np.float64) for a in Axs]
    VP = ctypes.c_void_p * count
    P64 = _i64p * count
    hs = (ctypes.c_void_p * count)()
    rcs = (ctypes.c_int * count)()
    err = ctypes.create_string_buffer(512)
    opts = options if options is not None else (syms[0].options if count else Options())
    rc = lib().fplus_b200_factor_batch(count, VP(*[s._h for s in syms]), P64(*[_p64(s.Ap) for s in syms]),
                                       P64(*[_p64(s.Ai) for s in syms]), VP(*[v.ctypes.data for v in vals]), int(cplx),
                                       ctypes.byref(opts), nworkers, hs, rcs, err, 512)
    out = [Numeric._from_handle(syms[k], hs[k], cplx) if hs[k] else None for k in range(count)]
    _check(rc, err)
    return out


def solve_batch(nums, bs, trans=0, nworkers=8):
    """fplus_b200_solve_batch: x_k with op(A_k) x_k = b_k for every k, concurrently; returns the list of solutions."""
    count = len(nums)
    Xs = []
    for N, b in zip(nums, bs):
        b = np.asarray(b)
        Xs.append(np.array(b.reshape(N.n, -1), dtype=np.complex128 if N.is_complex else np.float64, order="F", copy=True))
    VP = ctypes.c_void_p * count
    I64 = ctypes.c_int64 * count
    rcs = (ctypes.c_int * count)()
    err = ctypes.create_string_buffer(512)
    rc = lib().fplus_b200_solve_batch(count, VP(*[N._h.value for N in nums]), VP(*[X.ctypes.data for X in Xs]),
                                      I64(*[X.shape[1] for X in Xs]), I64(*[N.n for N in nums]), trans, nworkers, rcs, err, 512)
    _check(rc, err)
    return [X[:, 0] if np.asarray(b).ndim == 1 else X for X, b in zip(Xs, bs)]


class BatchGraph:
    """fplus_b200_graph_*: the refactorization and solve of many factored matrices captured as one CUDA graph.  The
    Numeric objects must outlive the graph (it keeps references)."""

    def __init__(self, nums, nrhs, trans=0):
        self.nums = list(nums)
        self.nrhs = [int(r) for r in (nrhs if hasattr(nrhs, "__len__") else [nrhs] * len(self.nums))]
        self._h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        arr = (ctypes.c_void_p * len(self.nums))(*[N._h.value for N in self.nums])
        nr = (ctypes.c_int64 * len(self.nums))(*self.nrhs)
        _check(lib().fplus_b200_graph_create(len(self.nums), arr, nr, int(trans), ctypes.byref(self._h), err, 512), err)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None and self._h.value:
            _lib.fplus_b200_graph_free(self._h)
            self._h = ctypes.c_void_p()

    def upload(self, k, Ax=None, b=None):
        N = self.nums[k]
        dt = np.complex128 if N.is_complex else np.float64
        a = None if Ax is None else np.ascontiguousarray(Ax, dtype=dt)
        bb = None if b is None else np.asfortranarray(np.asarray(b, dtype=dt).reshape(N.n, -1))
        err = ctypes.create_string_buffer(512)
        _check(lib().fplus_b200_graph_upload(self._h, k, None if a is None else a.ctypes.data_as(ctypes.c_void_p),
                                             None if bb is None else bb.ctypes.data_as(ctypes.c_void_p), err, 512), err)

    def launch(self, stream=None):
        err = ctypes.create_string_buffer(512)
        _check(lib().fplus_b200_graph_launch(self._h, None if stream is None else ctypes.c_void_p(stream), err, 512), err)

    def status(self):
        """Waits for the graph; the per-matrix codes (0, FPLUS_ERR_SINGULAR, FPLUS_ERR_BADARG, FPLUS_ERR_GPU)."""
        rcs = (ctypes.c_int * len(self.nums))()
        err = ctypes.create_string_buffer(512)
        lib().fplus_b200_graph_status(self._h, rcs, err, 512)
        return list(rcs)

    def download(self, k):
        N = self.nums[k]
        X = np.zeros((N.n, self.nrhs[k]), dtype=np.complex128 if N.is_complex else np.float64, order="F")
        err = ctypes.create_string_buffer(512)
        _check(lib().fplus_b200_graph_download(self._h, k, X.ctypes.data_as(ctypes.c_void_p), err, 512), err)
        return X


def batch_span_ms(nums):
    """fplus_b200_batch_span_ms: the device time from the first factorization's start to the last solve's end."""
    arr = (ctypes.c_void_p * len(nums))(*[N._h.value for N in nums])
    ms = ctypes.c_double()
    err = ctypes.create_string_buffer(512)
    _check(lib().fplus_b200_batch_span_ms(len(nums), arr, ctypes.byref(ms), err, 512), err)
    return ms.value


def interior_order(n, Ap, Ai, trow=None, tcol=None):
    n, Ap, Ai, _ = csc_arrays(n, Ap, Ai)
    perm = np.zeros(n, np.int64)
    tr = None if trow is None else np.ascontiguousarray(trow, dtype=np.uint8).ctypes.data_as(ctypes.c_char_p)
    tc = None if tcol is None else np.ascontiguousarray(tcol, dtype=np.uint8).ctypes.data_as(ctypes.c_char_p)
    _check(lib().fplus_b200_interior_order(n, _p64(Ap), _p64(Ai), tr, tc, _p64(perm)), None)
    return perm


# ------------------------------------------------------------------------------------------------ the low-level interface
# The functions of FPLUS's Python extension (_sparse_lu_c.c:634-696) over the same C entry points: factor_sn_perm,
# solve_plan, lu_solve_plan, lu_solve.  The factor arrays returned by factor_sn_perm are views of the library's own
# memory (no copy), so that passing them back to solve_plan / lu_solve_plan keeps the pointers the library recognises
# and the solve runs with the factorization's device copy; the memory is released with the last array.


class _FactorsOwner:
    def __init__(self, f: Factors):
        self.f = f

    def __del__(self):
        if _lib is not None:
            _lib.fplus_factors_free(ctypes.byref(self.f))


class _Buf:
    """An __array_interface__ over library memory that keeps its owner alive while an array uses it."""

    def __init__(self, owner, addr, n, dtype):
        self._owner = owner
        self.__array_interface__ = {"data": (addr, False), "shape": (n,), "typestr": np.dtype(dtype).str, "version": 3}


def _view(owner, ptr, n, dtype):
    addr = ctypes.cast(ptr, ctypes.c_void_p).value
    if n == 0 or not addr:
        return np.zeros(n, dtype)
    return np.asarray(_Buf(owner, addr, n, dtype))


def _factors_dict(f: Factors):
    owner = _FactorsOwner(f)
    n = int(f.n)
    vt = np.complex128 if f.is_complex else np.float64
    Lp = _view(owner, f.Lp, n + 1, np.int64)
    Up = _view(owner, f.Up, n + 1, np.int64)
    nl, nu = int(Lp[n]) if n >= 0 else 0, int(Up[n]) if n >= 0 else 0
    return {"L_data": _view(owner, f.Lx, nl, vt), "L_indices": _view(owner, f.Li, nl, np.int64), "L_indptr": Lp,
            "U_data": _view(owner, f.Ux, nu, vt), "U_indices": _view(owner, f.Ui, nu, np.int64), "U_indptr": Up,
            "p": _view(owner, f.p, n, np.int64), "q": _view(owner, f.q, n, np.int64), "format": "csc"}


def factor_sn_perm(data, indices, indptr, n, row_perm, col_perm, is_complex, equilibrate=1, ruiz_max_iter=20,
                   ruiz_tol=1e-2, verbose=0, relax_rows=0, panel=1, use_gpu=0, gpu_min_flops=5e7,
                   pivot_rel=FPLUS_PIVOT_REL_DEFAULT):
    """fplus_factor_sn_perm: the factors of A[row_perm, :][:, col_perm] with Dr, Dc (permuted order), as a dict with the
    keys of FPLUS's extension (L_data, L_indices, L_indptr, U_data, U_indices, U_indptr, p, q, format, Dr, Dc)."""
    Ap = np.ascontiguousarray(indptr, dtype=np.int64)
    Ai = np.ascontiguousarray(indices, dtype=np.int64)
    Ax = np.ascontiguousarray(data, dtype=np.complex128 if is_complex else np.float64)
    rp = np.ascontiguousarray(row_perm, dtype=np.int64)
    cp = np.ascontiguousarray(col_perm, dtype=np.int64)
    if Ap.shape[0] != n + 1 or rp.shape[0] != n or cp.shape[0] != n:
        raise ValueError("factor_sn_perm: indptr must have length n + 1 and the permutations length n")
    Dr = np.empty(max(n, 1)); Dc = np.empty(max(n, 1))
    f = Factors()
    err = ctypes.create_string_buffer(512)
    rc = lib().fplus_factor_sn_perm(n, _p64(Ap), _p64(Ai), Ax.ctypes.data_as(ctypes.c_void_p), int(bool(is_complex)),
                                    _p64(rp), _p64(cp), int(equilibrate), int(ruiz_max_iter), float(ruiz_tol), int(verbose),
                                    int(relax_rows), int(panel), int(use_gpu), float(gpu_min_flops), float(pivot_rel),
                                    ctypes.byref(f), Dr.ctypes.data_as(_dp), Dc.ctypes.data_as(_dp), err, 512)
    _check(rc, err)
    d = _factors_dict(f)
    d["Dr"], d["Dc"] = Dr[:n], Dc[:n]
    return d


def factor_sn_sym(sym: "Symbolic", data, indices, indptr, is_complex, equilibrate=1, ruiz_max_iter=20, ruiz_tol=1e-2,
                  verbose=0, relax_rows=0, panel=1, use_gpu=0, gpu_min_flops=5e7, pivot_rel=FPLUS_PIVOT_REL_DEFAULT):
    """fplus_factor_sn_sym: factor_sn_perm with the orders of an analysis."""
    n = sym.n
    Ap = np.ascontiguousarray(indptr, dtype=np.int64)
    Ai = np.ascontiguousarray(indices, dtype=np.int64)
    Ax = np.ascontiguousarray(data, dtype=np.complex128 if is_complex else np.float64)
    Dr = np.empty(max(n, 1)); Dc = np.empty(max(n, 1))
    f = Factors()
    err = ctypes.create_string_buffer(512)
    rc = lib().fplus_factor_sn_sym(sym._h, _p64(Ap), _p64(Ai), Ax.ctypes.data_as(ctypes.c_void_p), int(bool(is_complex)),
                                   int(equilibrate), int(ruiz_max_iter), float(ruiz_tol), int(verbose), int(relax_rows),
                                   int(panel), int(use_gpu), float(gpu_min_flops), float(pivot_rel), ctypes.byref(f),
                                   Dr.ctypes.data_as(_dp), Dc.ctypes.data_as(_dp), err, 512)
    _check(rc, err)
    d = _factors_dict(f)
    d["Dr"], d["Dc"] = Dr[:n], Dc[:n]
    return d


class SolvePlan:
    """fplus_solve_plan_create on CSC factor patterns; freed with the object."""

    def __init__(self, Lp, Li, Up, Ui):
        self._keep = [np.ascontiguousarray(a, dtype=np.int64) for a in (Lp, Li, Up, Ui)]
        Lp, Li, Up, Ui = self._keep
        self.n = Lp.shape[0] - 1
        if Up.shape[0] != self.n + 1:
            raise ValueError("solve_plan: Lp and Up must both have length n + 1")
        self._h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        _check(lib().fplus_solve_plan_create(self.n, _p64(Lp), _p64(Li), _p64(Up), _p64(Ui), ctypes.byref(self._h), err, 512), err)

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value and _lib is not None:
            _lib.fplus_solve_plan_free(self._h)
            self._h = ctypes.c_void_p()

    @property
    def nsupernodes(self) -> int:
        return int(lib().fplus_solve_plan_nsupernodes(self._h))


def solve_plan(Lp, Li, Up, Ui) -> SolvePlan:
    return SolvePlan(Lp, Li, Up, Ui)


def _solve_x(b, n, is_complex, name):
    x = np.array(b, dtype=np.complex128 if is_complex else np.float64, order="F", copy=True)
    if x.ndim not in (1, 2) or x.shape[0] != n:
        raise ValueError(f"{name}: b must have shape (n,) or (n, nrhs)")
    return x


def _solve_rc(rc, name):
    if rc == FPLUS_ERR_SINGULAR:
        raise FplusError(rc, f"{name}: zero or missing diagonal in U")
    if rc == FPLUS_ERR_BADARG:
        raise FplusError(rc, f"{name}: the plan does not match these factors")
    if rc != FPLUS_OK:
        raise FplusError(rc, f"{name} failed")


def lu_solve_plan(plan: SolvePlan, Lp, Li, Lx, Up, Ui, Ux, b, trans, is_complex):
    """fplus_tri_solve_plan on a copy of b ((n,) or (n, nrhs)): trans 0 L U x = b, 1 (L U)^T x = b, 2 (L U)^H x = b."""
    vt = np.complex128 if is_complex else np.float64
    Lp, Li, Up, Ui = (np.ascontiguousarray(a, dtype=np.int64) for a in (Lp, Li, Up, Ui))
    Lx, Ux = np.ascontiguousarray(Lx, dtype=vt), np.ascontiguousarray(Ux, dtype=vt)
    n = Lp.shape[0] - 1
    x = _solve_x(b, n, is_complex, "lu_solve_plan")
    nrhs = 1 if x.ndim == 1 else x.shape[1]
    rc = lib().fplus_tri_solve_plan(plan._h, n, _p64(Lp), _p64(Li), Lx.ctypes.data_as(ctypes.c_void_p), _p64(Up), _p64(Ui),
                                    Ux.ctypes.data_as(ctypes.c_void_p), x.ctypes.data_as(ctypes.c_void_p), nrhs, n,
                                    int(trans), int(bool(is_complex)))
    _solve_rc(rc, "lu_solve_plan")
    return x


def lu_solve(Lp, Li, Lx, Up, Ui, Ux, b, trans, is_complex):
    """fplus_tri_solve, one right-hand side at a time, on a copy of b."""
    vt = np.complex128 if is_complex else np.float64
    Lp, Li, Up, Ui = (np.ascontiguousarray(a, dtype=np.int64) for a in (Lp, Li, Up, Ui))
    Lx, Ux = np.ascontiguousarray(Lx, dtype=vt), np.ascontiguousarray(Ux, dtype=vt)
    n = Lp.shape[0] - 1
    x = _solve_x(b, n, is_complex, "lu_solve")
    cols = [x] if x.ndim == 1 else [x[:, r] for r in range(x.shape[1])]
    for c in cols:
        rc = lib().fplus_tri_solve(n, _p64(Lp), _p64(Li), Lx.ctypes.data_as(ctypes.c_void_p), _p64(Up), _p64(Ui),
                                   Ux.ctypes.data_as(ctypes.c_void_p), c.ctypes.data_as(ctypes.c_void_p), int(trans),
                                   int(bool(is_complex)))
        _solve_rc(rc, "lu_solve")
    return x


def lu_solve_perm(plan: SolvePlan, Lp, Li, Lx, Up, Ui, Ux, b, trans, is_complex, p, q, Dr, Dc):
    """FPLUS's lu_solve_perm (_sparse_lu_c.c:551-633): the right-hand sides gathered through the row (trans 0) or column
    permutation with its scaling, the plan's solve, then scattered through the other one with the other scaling
    (trans 0: w = Dr[p] b[p], x[q] = Dc[q] z; else w = Dc[q] b[q], x[p] = Dr[p] z).  Dr / Dc None: no scaling.
    b: (n,) or (n, nrhs); returns a new array of b's shape."""
    vt = np.complex128 if is_complex else np.float64
    bin_ = np.asarray(b, dtype=vt)
    n = np.asarray(Lp).shape[0] - 1
    if trans not in (0, 1, 2):
        raise ValueError("lu_solve_perm: trans must be 0, 1 or 2")
    p = np.asarray(p, dtype=np.int64); q = np.asarray(q, dtype=np.int64)
    if bin_.ndim not in (1, 2) or bin_.shape[0] != n or p.shape[0] != n or q.shape[0] != n \
            or (Dr is not None and len(Dr) != n) or (Dc is not None and len(Dc) != n):
        raise ValueError("lu_solve_perm: b must have shape (n,) or (n, nrhs); p, q, Dr, Dc length n")
    if n and (p.min() < 0 or p.max() >= n or q.min() < 0 or q.max() >= n):
        raise ValueError("lu_solve_perm: p or q out of range")
    G, Sc = (p, q) if trans == 0 else (q, p)
    Dg, Ds = (Dr, Dc) if trans == 0 else (Dc, Dr)
    B2 = bin_.reshape(n, -1)
    w = B2[G, :] * (np.asarray(Dg)[G][:, None] if Dg is not None else 1.0)
    z = lu_solve_plan(plan, Lp, Li, Lx, Up, Ui, Ux, w, trans, is_complex)
    out = np.empty_like(B2)
    out[Sc, :] = z * (np.asarray(Ds)[Sc][:, None] if Ds is not None else 1.0)
    return out.reshape(bin_.shape)


def ruiz_equilibrate(data, indices, indptr, n, max_iter, tol, is_complex, verbose=0, is_csc=0):
    """fplus_ruiz on a copy of data (CSR, or CSC when is_csc), as FPLUS's ruiz_equilibrate: {"Dr", "Dc", "data"} with
    diag(Dr) A diag(Dc) in data (same indices and indptr)."""
    Ap = np.ascontiguousarray(indptr, dtype=np.int64)
    Ai = np.ascontiguousarray(indices, dtype=np.int64)
    x = np.array(data, dtype=np.complex128 if is_complex else np.float64, copy=True)
    if Ap.shape[0] != n + 1:
        raise ValueError("ruiz_equilibrate: indptr must have length n + 1")
    Dr = np.empty(max(n, 1)); Dc = np.empty(max(n, 1))
    err = ctypes.create_string_buffer(512)
    rc = lib().fplus_ruiz(n, _p64(Ap), _p64(Ai), x.ctypes.data_as(ctypes.c_void_p), int(bool(is_complex)), int(bool(is_csc)),
                          int(max_iter), float(tol), int(verbose), Dr.ctypes.data_as(_dp), Dc.ctypes.data_as(_dp), err, 512)
    _check(rc, err)
    return {"Dr": Dr[:n], "Dc": Dc[:n], "data": x}


class SparseLU:
    """FPLUS's SparseLU (sparse_lu_full_pivot.py:680-763) on the GPU: ``SparseLU(A, **kwargs).solve(b, trans)``.

    The keyword arguments are those of FPLUS's sparse_lu_full_pivot.  ``colamd`` (default False, as in FPLUS): the
    library's fill-reducing analysis with ``pin_dense_rows``, ``tau_density``, ``tau_min_nnz``, the masks, ``postorder``
    and ``ordering``; without it the identity orders.  ``equilibrate``: True (at most 20 Ruiz iterations), False / 0
    (none) or an iteration count.  ``pivot_rel`` (None: FPLUS's default).  This build factors exactly with partial
    pivoting: ``drop_tol`` must be 0 and ``pivot_strategy`` 'partial'.  ``relax_rows``, ``panel``, ``gpu``,
    ``gpu_min_flops``, ``cache_ordering`` and ``verbose`` are accepted.  The factors stay in device memory and the
    solves run there; ``L`` and ``U`` are read back on first use.
    """

    _ORDERINGS = {"colamd": 0, "amd": 1, "amd_ata": 1, "auto": 2}

    def __init__(self, A, *, drop_tol=0.0, equilibrate=True, colamd=False, pin_dense_rows=False, tau_density=0.5,
                 tau_min_nnz=10, tau_row_mask=None, tau_col_mask=None, pivot_strategy="partial", dtype=None, verbose=0,
                 relax_rows=0, panel=1, cache_ordering=True, gpu=False, gpu_min_flops=5e7, pivot_rel=None, postorder=True,
                 ordering="auto"):
        import scipy.sparse as sp
        if drop_tol != 0.0:
            raise ValueError("SparseLU: this build computes the exact factorization (drop_tol must be 0)")
        if pivot_strategy != "partial":
            raise ValueError("SparseLU: this build pivots by columns only (pivot_strategy 'partial')")
        if ordering not in self._ORDERINGS:
            raise ValueError(f"SparseLU: unknown ordering {ordering!r}")
        A = A if sp.issparse(A) else sp.csc_matrix(A)
        if A.shape[0] != A.shape[1]:
            raise ValueError("SparseLU: A must be square")
        cplx = np.iscomplexobj(A.data)
        if dtype is not None and np.dtype(dtype) not in (np.dtype(np.complex128), np.dtype(np.float64)):
            raise ValueError("SparseLU: this build works in float64 / complex128")
        if dtype is not None and np.dtype(dtype) == np.dtype(np.complex128):
            cplx = True
        A = sp.csc_matrix(A, dtype=np.complex128 if cplx else np.float64)
        A.sum_duplicates()
        A.sort_indices()
        n = A.shape[0]
        Ap, Ai = A.indptr.astype(np.int64), A.indices.astype(np.int64)
        if colamd:
            def mask(m):
                return None if m is None else np.ascontiguousarray(np.asarray(m, dtype=bool), dtype=np.uint8)
            sym = Symbolic.__new__(Symbolic)
            sym.n, sym.Ap, sym.Ai = n, Ap, Ai
            sym.options = default_options()
            sym._h = ctypes.c_void_p()
            err = ctypes.create_string_buffer(512)
            rm, cm = mask(tau_row_mask), mask(tau_col_mask)
            _check(lib().fplus_analyze_ord(n, _p64(Ap), _p64(Ai), int(bool(pin_dense_rows)), float(tau_density),
                                           int(tau_min_nnz), None if rm is None else rm.ctypes.data_as(ctypes.c_char_p),
                                           None if cm is None else cm.ctypes.data_as(ctypes.c_char_p), int(bool(postorder)),
                                           self._ORDERINGS[ordering], ctypes.byref(sym._h), err, 512), err)
        else:
            sym = Symbolic.from_orders(n, Ap, Ai, np.arange(n), np.arange(n))
        if equilibrate is True or (not isinstance(equilibrate, bool) and int(equilibrate) < 0):
            eq, iters = 1, 20
        elif equilibrate is False or int(equilibrate) == 0:
            eq, iters = 0, 20
        else:
            eq, iters = 1, int(equilibrate)
        opts = default_options(equilibrate=eq, ruiz_max_iter=iters, verbose=int(verbose), relax_rows=int(relax_rows),
                               panel=int(panel), use_gpu=int(bool(gpu)), gpu_min_flops=float(gpu_min_flops),
                               pivot_rel=FPLUS_PIVOT_REL_DEFAULT if pivot_rel is None else float(pivot_rel))
        self._sym = sym
        self._num = Numeric(sym, A.data, opts)
        self._n = n
        self._is_complex = cplx
        self._LU = None

    def _factors(self):
        if self._LU is None:
            L, U, _ = self._num.factors()
            self._LU = (L, U)
        return self._LU

    @property
    def L(self):
        """Unit lower-triangular factor (CSC), of diag(Dr) A[perm_r, :][:, perm_c] diag(Dc) = L U."""
        return self._factors()[0]

    @property
    def U(self):
        """Upper-triangular factor (CSC)."""
        return self._factors()[1]

    @property
    def perm_r(self):
        return self._num.p

    @property
    def perm_c(self):
        return self._num.q

    @property
    def Dr(self):
        return self._num.Dr

    @property
    def Dc(self):
        return self._num.Dc

    @property
    def shape(self):
        return (self._n, self._n)

    @property
    def nnz(self):
        """Stored entries of L and U (explicit zeros of the front structure included)."""
        info = self._num.info
        return int(info["nnz_L"] + info["nnz_U"])

    def solve(self, b, trans="N"):
        """x with A x = b ('N'), A^T x = b ('T') or A^H x = b ('H'); b of shape (n,) or (n, nrhs)."""
        if trans not in ("N", "T", "H"):
            raise ValueError("SparseLU.solve: trans must be 'N', 'T' or 'H'")
        tr = 0 if trans == "N" else (1 if trans == "T" or not self._is_complex else 2)
        b = np.asarray(b)
        if np.iscomplexobj(b) and not self._is_complex:
            return self._num.solve(b.real, tr) + 1j * self._num.solve(b.imag, tr)
        return self._num.solve(b, tr)
