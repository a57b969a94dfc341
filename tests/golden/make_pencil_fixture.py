"""Golden outputs of the oracle restatement on the full-size benchmark pencil and on a scaled 3D stencil.

    python tests/golden/make_pencil_fixture.py

The GPU parity tests check the CUDA path against these at sizes where the oracle takes minutes (too long to run inside a
test):

* ``pencil_n32768.npz``: A - sigma B with 8 Fourier modes x 4 fields x 1024 Chebyshev modes (n = 32,768, complex128,
  2,222,368 entries, 8 dense tau rows and 8 dense tau columns), the matrix the benchmark factors;
* ``convdiff3d_g32.npz``: the 7-point convection-diffusion stencil on a 32^3 grid (n = 32,768, real).

Each holds the static orders of the analysis, the oracle's composed pivot order p, the Ruiz scalings Dr and Dc, the
Frobenius norms of L and U, and the solution of one seeded right-hand side, with a checksum of the generated values so a
change of the generator is caught.  The matrices themselves are regenerated from their seeds (fplus_b200.workloads).
The oracle restatement is pinned to the reference itself by tests/test_cpu.py on the smaller golden cases.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import fplus_b200 as F          # noqa: E402  (host-only analysis: the orders)
import oracle as O              # noqa: E402
from fplus_b200 import workloads as W   # noqa: E402

RHS_SEED = 11


def checksum(Ax):
    a = np.asarray(Ax)
    return np.array([a.real.sum(), (a.imag.sum() if np.iscomplexobj(a) else 0.0), np.abs(a).max(), float(a.size)])


def make(name, gen):
    t0 = time.time()
    n, Ap, Ai, Ax = gen()
    S = F.analyze(n, Ap, Ai)
    orc = O.OracleLU(n, Ap, Ai, Ax, S.row_perm, S.col_perm)
    L_fro, U_fro = orc.fro_norms()
    b = W.rhs(n, 1, np.iscomplexobj(Ax), RHS_SEED)[0]
    x = orc.solve(b)
    berr = O.backward_error(n, Ap, Ai, Ax, x, b)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), n=n, nnz=Ap[-1], checksum=checksum(Ax), row_perm=S.row_perm,
                        col_perm=S.col_perm, p=orc.p, Dr=orc.Dr, Dc=orc.Dc, L_fro=L_fro, U_fro=U_fro, rhs_seed=RHS_SEED,
                        x=x, berr=berr)
    print(f"{name}: n={n} nnz={Ap[-1]} berr={berr:.2e} |L|={L_fro:.6e} |U|={U_fro:.6e} ({time.time() - t0:.0f} s)", flush=True)


def main():
    which = sys.argv[1:] or ["pencil_n32768", "convdiff3d_g32"]
    gens = {"pencil_n32768": lambda: W.pencil(), "convdiff3d_g32": lambda: W.convdiff3d(32, 3)}
    for name in which:
        make(name, gens[name])


if __name__ == "__main__":
    main()
