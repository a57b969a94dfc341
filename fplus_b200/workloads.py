"""Seeded synthetic matrices of the benchmark configurations (canonical int64 CSC, numpy only).

The shapes, sizes and value distributions follow the five workload descriptions of the factor+solve benchmark:

* ``convdiff2d``  -- 5-point nonsymmetric convection-diffusion on a g x g grid (g = 100: n = 10,000, 49,600 nnz), real.
* ``pencil``      -- a shift-invert pencil A - sigma B of a spectral solver: Fourier modes x fields x Chebyshev modes, each
  Fourier mode a fields x fields grid of banded blocks, plus dense tau rows / columns over all n (pinned by the analysis).
* ``convdiff3d``  -- 7-point convection-diffusion on a g^3 grid (g = 80: n = 512,000, 3,545,600 nnz), real.
* ``pencil_batch`` -- many small pencils of uneven size (batched form).
* ``random_scaled`` -- a well-conditioned random sparse base with row / column scales over 17 decades.

Every generator takes a seed (``numpy.random.default_rng(seed)``) and returns ``(n, Ap, Ai, Ax)``.
"""
from __future__ import annotations

import numpy as np


def _coo_to_csc(n, rows, cols, vals):
    """Canonical CSC (rows ascending in each column, duplicates summed) from COO triplets."""
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    key = cols * n + rows
    order = np.argsort(key, kind="stable")
    key = key[order]
    vals = np.asarray(vals)[order]
    uniq, start = np.unique(key, return_index=True)
    if len(uniq) != len(key):
        vals = np.add.reduceat(vals, start)
    Ai = (uniq % n).astype(np.int64)
    Ac = (uniq // n).astype(np.int64)
    Ap = np.zeros(n + 1, dtype=np.int64)
    np.add.at(Ap, Ac + 1, 1)
    Ap = np.cumsum(Ap)
    return n, Ap, Ai, np.ascontiguousarray(vals)


def convdiff2d(g: int = 100, seed: int = 1):
    """5-point stencil on a g x g grid: diagonal 4 + U(0, 0.1); the coupling of row i to its west / south neighbours is
    -1 + 0.3 c_i, to its east / north neighbours -1 - 0.3 c_i, c_i ~ U(-1, 1) per row."""
    rng = np.random.default_rng(seed)
    n = g * g
    idx = np.arange(n)
    gx, gy = idx % g, idx // g
    c = rng.uniform(-1.0, 1.0, n)
    diag = 4.0 + rng.uniform(0.0, 0.1, n)
    rows, cols, vals = [idx], [idx], [diag]
    for dx, dy, sgn in ((-1, 0, 1.0), (0, -1, 1.0), (1, 0, -1.0), (0, 1, -1.0)):
        ok = (gx + dx >= 0) & (gx + dx < g) & (gy + dy >= 0) & (gy + dy < g)
        i = idx[ok]
        rows.append(i)
        cols.append(i + dx + dy * g)
        vals.append(-1.0 + sgn * 0.3 * c[i])
    return _coo_to_csc(n, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals))


def convdiff3d(g: int = 80, seed: int = 3):
    """7-point stencil on a g^3 grid: diagonal 6 + U(0, 0.1); couplings -1 +/- 0.3 c_i (upwind side +), c_i ~ U(-2, 2)."""
    rng = np.random.default_rng(seed)
    n = g * g * g
    idx = np.arange(n, dtype=np.int64)
    gx, gy, gz = idx % g, (idx // g) % g, idx // (g * g)
    c = rng.uniform(-2.0, 2.0, n)
    diag = 6.0 + rng.uniform(0.0, 0.1, n)
    rows, cols, vals = [idx], [idx], [diag]
    for d, (dx, dy, dz) in enumerate(((-1, 0, 0), (0, -1, 0), (0, 0, -1), (1, 0, 0), (0, 1, 0), (0, 0, 1))):
        sgn = 1.0 if d < 3 else -1.0
        ok = ((gx + dx >= 0) & (gx + dx < g) & (gy + dy >= 0) & (gy + dy < g) & (gz + dz >= 0) & (gz + dz < g))
        i = idx[ok]
        rows.append(i)
        cols.append(i + dx + dy * g + dz * g * g)
        vals.append(-1.0 + sgn * 0.3 * c[i])
    return _coo_to_csc(n, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals))


def _logu_phase(rng, m, lo, hi):
    mag = 10.0 ** rng.uniform(np.log10(lo), np.log10(hi), m)
    return mag * np.exp(1j * rng.uniform(0.0, 2.0 * np.pi, m))


def pencil(modes: int = 8, fields: int = 4, nc: int = 1024, hbw: int = 6, bhbw: int = 2, tau_per_field: int = 2,
           sigma: complex = 0.3 + 1.7j, lo: float = 1e-6, hi: float = 1e6, seed: int = 2):
    """A - sigma B on modes x fields x nc unknowns (index = (mode * fields + field) * nc + k).  Within each Fourier mode a
    fields x fields grid of blocks banded with half-bandwidth hbw; B banded with half-bandwidth bhbw on the diagonal field
    blocks.  tau_per_field * fields tau rows and as many tau columns (the last Chebyshev rows / columns of each field of
    mode 0), each dense over all n; B is zero on the tau rows.  Magnitudes log-uniform in [lo, hi], phases U(0, 2 pi)."""
    rng = np.random.default_rng(seed)
    fb = fields * nc
    n = modes * fb
    tau_rows = np.array([f * nc + nc - 1 - t for f in range(fields) for t in range(tau_per_field)], dtype=np.int64)
    tau_cols = tau_rows.copy()
    is_tau_row = np.zeros(n, dtype=bool)
    is_tau_row[tau_rows] = True
    rows, cols = [], []
    k = np.arange(nc, dtype=np.int64)
    for m in range(modes):
        for fi in range(fields):
            for fj in range(fields):
                for d in range(-hbw, hbw + 1):
                    ok = (k + d >= 0) & (k + d < nc)
                    rows.append(m * fb + fi * nc + k[ok])
                    cols.append(m * fb + fj * nc + k[ok] + d)
    rows = np.concatenate(rows)
    cols = np.concatenate(cols)
    keep = ~is_tau_row[rows] & ~np.isin(cols, tau_cols)
    rows, cols = rows[keep], cols[keep]
    vals = _logu_phase(rng, len(rows), lo, hi)
    # B on the diagonal field blocks, half-bandwidth bhbw (inside A's pattern), not on tau rows
    same_field = (rows // nc) == (cols // nc)
    inb = same_field & (np.abs((rows % nc) - (cols % nc)) <= bhbw)
    bvals = _logu_phase(rng, int(inb.sum()), lo, hi)
    vals[inb] -= sigma * bvals
    # dense tau rows and columns
    all_idx = np.arange(n, dtype=np.int64)
    tr = [np.repeat(tau_rows, n), np.tile(all_idx, len(tau_rows))]
    tc_rows = np.tile(all_idx, len(tau_cols))
    tc_cols = np.repeat(tau_cols, n)
    tcm = ~is_tau_row[tc_rows]          # tau x tau entries come from the tau rows
    rows = np.concatenate([rows, tr[0], tc_rows[tcm]])
    cols = np.concatenate([cols, tr[1], tc_cols[tcm]])
    vals = np.concatenate([vals, _logu_phase(rng, len(tr[0]), lo, hi), _logu_phase(rng, int(tcm.sum()), lo, hi)])
    return _coo_to_csc(n, rows, cols, vals)


def pencil_batch(count: int = 512, nmin: int = 500, nmax: int = 8000, seed: int = 4):
    """count independent pencils, n log-uniform in [nmin, nmax], half-bandwidth U{4..8}, 2-4 dense tau rows / columns,
    entries log-uniform in [1e-4, 1e4] with phases.  Returns a list of (n, Ap, Ai, Ax)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(round(10.0 ** rng.uniform(np.log10(nmin), np.log10(nmax))))
        hbw = int(rng.integers(4, 9))
        ntau = int(rng.integers(2, 5))
        k = np.arange(n, dtype=np.int64)
        rows, cols = [], []
        for d in range(-hbw, hbw + 1):
            ok = (k + d >= 0) & (k + d < n)
            rows.append(k[ok])
            cols.append(k[ok] + d)
        rows, cols = np.concatenate(rows), np.concatenate(cols)
        taus = rng.choice(n, size=ntau, replace=False).astype(np.int64)
        tcol = rng.choice(n, size=ntau, replace=False).astype(np.int64)
        keep = ~np.isin(rows, taus) & ~np.isin(cols, tcol)
        rows, cols = rows[keep], cols[keep]
        rows = np.concatenate([rows, np.repeat(taus, n), np.tile(k, ntau)])
        cols = np.concatenate([cols, np.tile(k, ntau), np.repeat(tcol, n)])
        sub = np.random.default_rng(int(rng.integers(1 << 31)))
        vals = _logu_phase(sub, len(rows), 1e-4, 1e4)
        # a row and a column both dense meet once: drop the duplicate (keep the first occurrence)
        key = cols * n + rows
        _, first = np.unique(key, return_index=True)
        out.append(_coo_to_csc(n, rows[first], cols[first], vals[first]))
    return out


def random_scaled(n: int = 300_000, per_col: int = 12, seed: int = 5):
    """A random sparse base with per_col entries per column (the diagonal included), unit-magnitude complex values with a
    dominant diagonal, then row and column scales log-uniform over [1e-8, 1e9]."""
    rng = np.random.default_rng(seed)
    cols = np.repeat(np.arange(n, dtype=np.int64), per_col - 1)
    rows = rng.integers(0, n, size=len(cols), dtype=np.int64)
    rows = np.concatenate([rows, np.arange(n, dtype=np.int64)])
    cols = np.concatenate([cols, np.arange(n, dtype=np.int64)])
    vals = np.exp(1j * rng.uniform(0, 2 * np.pi, len(rows)))
    vals[-n:] *= per_col                      # structurally and numerically nonsingular diagonal
    dr = 10.0 ** rng.uniform(-8, 9, n)
    dc = 10.0 ** rng.uniform(-8, 9, n)
    vals = dr[rows] * vals * dc[cols]
    return _coo_to_csc(n, rows, cols, vals)


def rhs(n: int, nrhs: int, is_complex: bool, seed: int):
    """b ~ N(0, 1) (complex: independent real and imaginary parts), column-major n x nrhs."""
    rng = np.random.default_rng(seed + 1000)
    b = rng.standard_normal((nrhs, n))
    if is_complex:
        b = b + 1j * rng.standard_normal((nrhs, n))
    return np.ascontiguousarray(b)   # row r of this array is right-hand side r: column-major n x nrhs
