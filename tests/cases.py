"""Seeded test matrices shared by the CPU and GPU tests (small enough for the oracle to finish in seconds)."""
import numpy as np
import scipy.sparse as sp

from fplus_b200 import workloads as W


def hard_matrix(n, cplx, scale, seed):
    """A band, 3 random entries per column, dense rows 1 and n/2, dense column n/3, row scales 10^[-s, s]: the random
    matrix family of the reference's C tests (tests/c/test_fplus.c:22-49), regenerated with numpy."""
    rng = np.random.default_rng(seed)
    mask = np.zeros((n, n), dtype=bool)
    for j in range(n):
        for d in range(-2, 3):
            if 0 <= j + d < n:
                mask[j + d, j] = True
        mask[rng.integers(0, n, 3), j] = True
    mask[1, :] = True
    mask[n // 2, :] = True
    mask[:, n // 3] = True
    rs = 10.0 ** (scale * (2 * rng.random(n) - 1))
    rows, cols = np.nonzero(mask)
    re = 2 * rng.random(len(rows)) - 1 + np.where(rows == cols, 0.5, 0.0)
    im = 2 * rng.random(len(rows)) - 1
    v = rs[rows] * (re + 1j * im if cplx else re)
    A = sp.csc_matrix((v, (rows, cols)), shape=(n, n))
    A.sort_indices()
    return n, A.indptr.astype(np.int64), A.indices.astype(np.int64), A.data


def banded_random_complex(n, seed, bw=6, density=0.004):
    """A complex band plus scattered entries (near-nesting patterns; not diagonally dominant)."""
    rng = np.random.default_rng(seed)
    offs = list(range(-bw, bw + 1))
    diags = [rng.standard_normal(n - abs(k)) + 1j * rng.standard_normal(n - abs(k)) for k in offs]
    B = sp.diags(diags, offs, shape=(n, n), format="csc", dtype=np.complex128)
    R = sp.random(n, n, density=density, format="csc", random_state=rng) * (1 + 1j)
    A = (B + R + 0.5 * sp.eye(n, dtype=np.complex128)).tocsc()
    A.sort_indices()
    return n, A.indptr.astype(np.int64), A.indices.astype(np.int64), A.data


CASES = {
    "convdiff2d_g20": lambda: W.convdiff2d(20, 1),
    "convdiff2d_g100": lambda: W.convdiff2d(100, 1),
    "convdiff3d_g12": lambda: W.convdiff3d(12, 3),
    "pencil_1x64": lambda: W.pencil(modes=1, nc=64),
    "pencil_2x256": lambda: W.pencil(modes=2, nc=256),
    "hard_real_300": lambda: hard_matrix(300, False, 6.0, 11),
    "hard_cplx_300": lambda: hard_matrix(300, True, 6.0, 12),
    "hard_cplx_300_s0": lambda: hard_matrix(300, True, 0.0, 13),
    "banded_cplx_1200": lambda: banded_random_complex(1200, 14),
}
