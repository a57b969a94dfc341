"""fplus_b200_solve_dev_noalloc: the solve for callers that cannot allocate device memory at solve time.

Such callers are code that runs inside another runtime that owns the device memory and hands it only input and output
buffers, loops where the device synchronization an allocation implies is not acceptable, and processes held to a fixed
device-memory budget.  The entry point takes its scratch from one 16 MiB array that the library declares in device
memory, so it is checked here through the C-ABI against fplus_b200_solve_dev, the entry point that allocates its
scratch, on two calls in a row (the second call finds the first call's values left in the shared array), with a leading
dimension larger than n, more than one pass of 32 right-hand sides, and a request beyond the array's size.  Tolerances
are those of the parity tests: solutions within 1e-12 of each other (relative, Frobenius), backward error <= 1e-14.

The file is named to be collected last, and passes both alone in a fresh process and after the other GPU tests.
"""
import ctypes

import numpy as np
import pytest

import fplus_b200 as F
import oracle as O
from fplus_b200 import workloads as W
from tests.cases import CASES

pytestmark = pytest.mark.gpu

SOLVE_TOL = 1e-12
BERR_TOL = 1e-14


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "the GPU tests need a CUDA device"
    torch.cuda.init()
    return torch


def _device_rhs(torch, B, ldb):
    """B (n x nrhs) as a column-major device buffer of leading dimension ldb (rows n..ldb-1 padding), as a torch tensor
    of shape (nrhs, ldb)."""
    n, nrhs = B.shape
    host = np.full((nrhs, ldb), 7.0 + (7.0j if np.iscomplexobj(B) else 0), dtype=B.dtype)
    host[:, :n] = B.T
    return torch.from_numpy(host).cuda()


def _call(fn, N, buf, nrhs, ldb, trans):
    import torch
    torch.cuda.synchronize()
    err = ctypes.create_string_buffer(512)
    rc = fn(N._h, ctypes.c_void_p(buf.data_ptr()), nrhs, ldb, trans, err, 512)
    torch.cuda.synchronize()
    return rc, err.value.decode(errors="replace")


@pytest.mark.parametrize("name,nrhs", [("convdiff2d_g100", 5), ("pencil_2x256", 40), ("hard_cplx_300", 3)])
def test_noalloc_matches_solve_dev_on_two_calls(torch_cuda, name, nrhs):
    torch = torch_cuda
    n, Ap, Ai, Ax = CASES[name]()
    cplx = np.iscomplexobj(Ax)
    S = F.analyze(n, Ap, Ai)
    N = S.factor(Ax)
    L = F.lib()
    ldb = n + 3
    rng = np.random.default_rng(11)
    tol = 1e-13 if name.startswith("hard") else BERR_TOL
    for call in range(2):
        B = rng.standard_normal((n, nrhs)) + (1j * rng.standard_normal((n, nrhs)) if cplx else 0)
        for trans in ((0, 1, 2) if cplx else (0, 1)):
            x_ref = _device_rhs(torch, B, ldb)
            x_na = _device_rhs(torch, B, ldb)
            rc, msg = _call(L.fplus_b200_solve_dev, N, x_ref, nrhs, ldb, trans)
            assert rc == 0, msg
            rc, msg = _call(L.fplus_b200_solve_dev_noalloc, N, x_na, nrhs, ldb, trans)
            assert rc == 0, f"call {call} trans {trans}: {msg}"
            Xr = x_ref.cpu().numpy()
            Xn = x_na.cpu().numpy()
            assert np.all(Xn[:, n:] == Xr[:, n:]), "rows past n of the leading dimension were written"
            Xr, Xn = Xr[:, :n].T, Xn[:, :n].T
            d = np.linalg.norm(Xn - Xr) / np.linalg.norm(Xr)
            assert d <= SOLVE_TOL, f"call {call} trans {trans}: differs from fplus_b200_solve_dev by {d:.1e}"
            for r in range(nrhs):
                be = O.backward_error(n, Ap, Ai, Ax, Xn[:, r], B[:, r], trans)
                assert be <= tol, f"call {call} trans {trans} rhs {r}: backward error {be:.2e}"


def test_noalloc_rejects_beyond_scratch(torch_cuda):
    """n = 40,000 real: one pass of 32 right-hand sides needs about 20 MB of scratch, beyond the 16 MiB array, and is
    refused before any work with FPLUS_ERR_BADARG, leaving b untouched; 8 right-hand sides per call fit and solve."""
    torch = torch_cuda
    n, Ap, Ai, Ax = W.convdiff2d(200, 3)
    S = F.analyze(n, Ap, Ai)
    N = S.factor(Ax)
    L = F.lib()
    rng = np.random.default_rng(5)
    B = rng.standard_normal((n, 32))
    x = _device_rhs(torch, B, n)
    rc, msg = _call(L.fplus_b200_solve_dev_noalloc, N, x, 32, n, 0)
    assert rc == F.FPLUS_ERR_BADARG and "scratch" in msg, (rc, msg)
    assert np.array_equal(x.cpu().numpy()[:, :n].T, B)
    x8 = _device_rhs(torch, B[:, :8], n)
    rc, msg = _call(L.fplus_b200_solve_dev_noalloc, N, x8, 8, n, 0)
    assert rc == 0, msg
    X = x8.cpu().numpy().T
    for r in range(8):
        assert O.backward_error(n, Ap, Ai, Ax, X[:, r], B[:, r], 0) <= BERR_TOL
