"""The static orders of the benchmark workloads, for the reference's arm of bench.py.

    python tests/golden/make_orders.py

The reference's own analysis cannot run here (its COLAMD/AMD come from SuiteSparse, which is absent), so the benchmark
injects this library's fill-reducing order into the reference's fplus_analyze and gives both libraries the same static
orders.  Storing them lets the reference's arm run without loading libfplus.so.  Each entry holds row_perm, col_perm, the
dense-row and dense-column masks and a checksum of the pattern (so a changed generator is caught); tests/test_cpu.py
checks that the analysis still produces them.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import fplus_b200 as F                  # noqa: E402  (the analysis)
from fplus_b200 import workloads as W   # noqa: E402

WORKLOADS = {
    "pencil_m1": lambda: W.pencil(modes=1),
    "pencil_m2": lambda: W.pencil(modes=2),
    "pencil_m8": lambda: W.pencil(modes=8),
    "convdiff2d_g100": lambda: W.convdiff2d(100, 1),
}


def pattern_checksum(Ap, Ai):
    return np.array([int(Ap[-1]), int(np.sum(Ap, dtype=np.int64)), int(np.sum(Ai * (np.arange(Ai.size) % 7 + 1), dtype=np.int64))])


def orders_for(name):
    n, Ap, Ai, _ = WORKLOADS[name]()
    S = F.analyze(n, Ap, Ai)
    trow = np.zeros(n, np.uint8); trow[S.row_perm[n - S.n_dense_rows:]] = 1
    tcol = np.zeros(n, np.uint8); tcol[S.col_perm[n - S.n_dense_cols:]] = 1
    return dict(row_perm=S.row_perm, col_perm=S.col_perm, trow=trow, tcol=tcol, pattern=pattern_checksum(Ap, Ai))


def main():
    flat = {}
    for name in WORKLOADS:
        for k, v in orders_for(name).items():
            flat[f"{name}__{k}"] = v
    np.savez_compressed(os.path.join(HERE, "orders.npz"), names=np.array(sorted(WORKLOADS)), **flat)
    print("orders:", sorted(WORKLOADS))


if __name__ == "__main__":
    main()
