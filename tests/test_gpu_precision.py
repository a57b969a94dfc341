"""The precision form: the Schur-complement update on the tcgen05 tensor cores in reduced precision, and factorizations
with it refined back to FP64 accuracy.

* The update kernel itself (fplus_b200_schur_update, through the C-ABI) against an FP64 torch reference of the same op,
  Cout = Cin[rmap] - A B, within error bounds stated per precision, relative to (|A| |B|)_ij; a plain torch FP32 GEMM is
  measured beside it, and the FP32 mode must be at least as accurate.
* Factorizations of 3D stencils (real and complex) in every precision: the large fronts' updates ran on the tensor
  cores, and iterative refinement in FP64 brings the solution to a backward error <= 1e-14.
"""
import ctypes

import numpy as np
import pytest

import fplus_b200 as F
from fplus_b200 import workloads as W
import oracle as O

pytestmark = pytest.mark.gpu

# |error| <= TOL * (|A| |B|)_ij: the split products' truncation (FP32: 2 x 11 bits, BF16X3: 2 x 8 bits, TF32: 11 bits) and
# FP32 accumulation over K' = 3K terms (K' = K for TF32), with margin
TOL = {F.PREC_FP32: 2e-5, F.PREC_BF16X3: 1e-4, F.PREC_TF32: 3e-3}


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "the GPU tests need a CUDA device"
    torch.cuda.init()
    return torch


def _update(torch, prec, cplx, M, N, K, R, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    dt = torch.complex128 if cplx else torch.float64

    def rnd(*shape):
        if cplx:
            return torch.complex(torch.randn(*shape, generator=g, device="cuda", dtype=torch.float64),
                                 torch.randn(*shape, generator=g, device="cuda", dtype=torch.float64))
        return torch.randn(*shape, generator=g, device="cuda", dtype=torch.float64)
    # column-major device arrays: a (cols, rows) row-major tensor
    At, Bt, Ct = rnd(K, M), rnd(N, K), rnd(N, R)
    rmap = torch.randperm(R, generator=g, device="cuda")[:M].to(torch.int32)
    Out = torch.full((N, M), float("nan"), dtype=dt, device="cuda")
    err = ctypes.create_string_buffer(512)
    rc = F.lib().fplus_b200_schur_update(prec, int(cplx), M, N, K, At.data_ptr(), M, Bt.data_ptr(), K, Ct.data_ptr(), R,
                                          rmap.data_ptr(), Out.data_ptr(), M, None, err, 512)
    assert rc == 0, err.value
    A, B = At.T, Bt.T                                  # M x K, K x N
    C = Ct.T[rmap.long(), :]                           # M x N
    ref = C - A @ B
    scale = A.abs() @ B.abs()
    got = Out.T
    e = ((got - ref).abs() / scale).max().item()
    ref32 = C - (A.to(torch.complex64 if cplx else torch.float32) @ B.to(torch.complex64 if cplx else torch.float32)).to(dt)
    e32 = ((ref32 - ref).abs() / scale).max().item()
    return e, e32, bool(torch.isfinite(got.abs()).all())


@pytest.mark.parametrize("prec", [F.PREC_FP32, F.PREC_BF16X3, F.PREC_TF32])
@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("shape", [(300, 700, 100), (128, 256, 256), (517, 1100, 64)])
def test_schur_update_against_fp64(torch_cuda, prec, cplx, shape):
    M, N, K = shape
    if cplx:
        N = N // 2          # the complex update is a real GEMM twice as wide
    e, e32, finite = _update(torch_cuda, prec, cplx, M, N, K, M + 37, 1000 * prec + 7 * K + int(cplx))
    assert finite, "non-finite or unwritten entries in the result"
    assert e <= TOL[prec], f"error {e:.2e} relative to |A||B| (plain torch FP32 GEMM: {e32:.2e})"
    if prec == F.PREC_FP32:
        # FP32-level accuracy: within a decade of a plain FP32 GEMM (the split adds 2^-22 per product, and the FP32
        # accumulation runs over 3K terms, 6K complex)
        assert e <= 10 * e32 + 1e-7, f"FP32 mode {e:.2e} vs torch FP32 {e32:.2e}"


def test_schur_update_rejects_small_shapes(torch_cuda):
    torch = torch_cuda
    A = torch.zeros(64 * 64, dtype=torch.float64, device="cuda")
    err = ctypes.create_string_buffer(512)
    rc = F.lib().fplus_b200_schur_update(F.PREC_FP32, 0, 64, 64, 64, A.data_ptr(), 64, A.data_ptr(), 64, A.data_ptr(), 64,
                                          None, A.data_ptr(), 64, None, err, 512)
    assert rc == F.FPLUS_ERR_BADARG


def _stencil(g, cplx):
    n, Ap, Ai, Ax = W.convdiff3d(g, 3)
    if cplx:
        rng = np.random.default_rng(9)
        Ax = Ax + 0.25j * rng.uniform(-1, 1, Ax.size)
    return n, Ap, Ai, Ax


@pytest.mark.parametrize("prec", [F.PREC_FP32, F.PREC_BF16X3, F.PREC_TF32])
@pytest.mark.parametrize("cplx", [False, True])
def test_precision_form_refines_to_fp64(torch_cuda, prec, cplx):
    n, Ap, Ai, Ax = _stencil(32, cplx)
    S = F.analyze(n, Ap, Ai)
    N = S.factor(Ax, precision=prec)
    info = N.info
    assert info["precision"] == prec
    assert info["tc_updates"] > 0 and info["tc_flops"] > 0.5 * info["front_flops"], "the large updates did not run on the tensor cores"
    b = W.rhs(n, 2, cplx, 3).T.copy(order="F")
    X, berr, iters = N.solve_refine(b, 0, max_iter=40, tol=1e-15)
    for r in range(2):
        be = O.backward_error(n, Ap, Ai, Ax, X[:, r], b[:, r])
        assert be <= 1e-14, f"rhs {r}: backward error {be:.2e} after {iters[r]} corrections (componentwise {berr[r]:.1e})"
    # the FP64 factorization of the same matrix: the refined solutions agree
    X64 = S.factor(Ax).solve(b)
    assert np.linalg.norm(X - X64) <= 1e-10 * np.linalg.norm(X64)
