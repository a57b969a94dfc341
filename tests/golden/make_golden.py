"""Generate the golden fixtures of the parity tests from the reference itself.

Run where the FPLUS sources are available (their test matrices are read from the source tree) and after
``make -C oracle ref`` has built oracle/_ref/libfplusref.so from them:

    python tests/golden/make_golden.py [/path/to/FPLUS]

For every case the fixture holds the input (canonical CSC, right-hand side), the static orders used, and the reference's
own outputs through its fplus_factor / fplus_solve: the composed pivot order p, the Ruiz scalings Dr and Dc, the
Frobenius norms of L and U and their nonzero counts, and the solutions for trans 0/1(/2).  The matrices of
relaxed_panel_case{50,3} are the reference's regression inputs (test_data/, pre-ordered: identity column order); their
fixture records the pivots of every relax / panel combination the reference's test runs (test_sparse_lu_full_pivot.py:
787-815), which the reference requires to be identical.
"""
import os
import sys

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import fplus_b200 as F          # noqa: E402  (host-only analysis: the orders)
import oracle as O              # noqa: E402
from tests.cases import hard_matrix, banded_random_complex   # noqa: E402
from fplus_b200 import workloads as W                          # noqa: E402


def ref_case(n, Ap, Ai, Ax, row_perm, col_perm, ntr_mask, ntc_mask, relax=32, panel=512, nrhs=2, seed=0):
    R = O.RefLU(n, Ap, Ai, Ax, col_perm, ntr_mask, ntc_mask, postorder=0, relax_rows=relax, panel=panel)
    assert np.array_equal(R.row_perm, row_perm) and np.array_equal(R.col_perm, col_perm)
    L, U, p_lu, nsn = R.factors()
    cplx = np.iscomplexobj(Ax)
    rng = np.random.default_rng(seed)
    B = rng.standard_normal((n, nrhs)) + (1j * rng.standard_normal((n, nrhs)) if cplx else 0)
    X = {t: R.solve(B, t) for t in ((0, 1, 2) if cplx else (0, 1))}
    return dict(p=R.p, Dr=R.Dr, Dc=R.Dc, p_lu=p_lu, L_fro=sp.linalg.norm(L), U_fro=sp.linalg.norm(U),
                L_nnz_true=np.count_nonzero(L.data), U_nnz_true=np.count_nonzero(U.data), B=B,
                **{f"X{t}": X[t] for t in X})


def masks(n, S):
    tr = np.zeros(n, np.uint8); tr[S.row_perm[n - S.n_dense_rows:]] = 1
    tc = np.zeros(n, np.uint8); tc[S.col_perm[n - S.n_dense_cols:]] = 1
    return tr, tc


def generated_cases():
    cases = {
        "convdiff2d_g20": W.convdiff2d(20, 1),
        "pencil_1x64": W.pencil(modes=1, nc=64),
        "hard_real_300": hard_matrix(300, False, 6.0, 11),
        "hard_cplx_300": hard_matrix(300, True, 6.0, 12),
        "banded_cplx_600": banded_random_complex(600, 21),
    }
    out = {}
    for name, (n, Ap, Ai, Ax) in cases.items():
        S = F.analyze(n, Ap, Ai)
        tr, tc = masks(n, S)
        r = ref_case(n, Ap, Ai, Ax, S.row_perm, S.col_perm, tr, tc)
        out[name] = dict(n=n, Ap=Ap, Ai=Ai, Ax=Ax, row_perm=S.row_perm, col_perm=S.col_perm, **r)
    return out


def panel_cases(src):
    out = {}
    for name in ("relaxed_panel_case50", "relaxed_panel_case3"):
        z = np.load(os.path.join(src, "test_data", name + ".npz"))
        A = sp.csr_matrix((z["data"], z["indices"], z["indptr"]), shape=(1200, 1200)).tocsc()
        A.sort_indices()
        n = 1200
        Ap, Ai, Ax = A.indptr.astype(np.int64), A.indices.astype(np.int64), A.data.copy()
        ident = np.arange(n, dtype=np.int64)
        zero = np.zeros(n, np.uint8)
        rec = dict(n=n, Ap=Ap, Ai=Ai, Ax=Ax, b=z["b"], row_perm=ident, col_perm=ident)
        ps = []
        for relax in (2, 8):
            for panel in (1, 2, 4, 8, 16):
                R = O.RefLU(n, Ap, Ai, Ax, ident, zero, zero, postorder=0, pin_dense=0, relax_rows=relax, panel=panel)
                ps.append(R.p)
                if relax == 2 and panel == 1:
                    L, U, p_lu, _ = R.factors()
                    x = R.solve(z["b"], 0)
                    rec.update(p=R.p, Dr=R.Dr, Dc=R.Dc, L_fro=sp.linalg.norm(L), U_fro=sp.linalg.norm(U), x=x,
                               berr=O.backward_error(n, Ap, Ai, Ax, x, z["b"]))
        rec["p_all_equal"] = all(np.array_equal(ps[0], q) for q in ps)
        out[name] = rec
    return out


def main():
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FPLUS_REFERENCE", "/root/reference")
    if not O.have_reference():
        raise SystemExit("oracle/_ref/libfplusref.so is missing: make -C oracle ref")
    for name, rec in panel_cases(src).items():
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **rec)
        print(name, "pivots equal across relax/panel:", rec["p_all_equal"], "berr", rec["berr"])
    gen = generated_cases()
    flat = {}
    for name, rec in gen.items():
        for k, v in rec.items():
            flat[f"{name}__{k}"] = v
    np.savez_compressed(os.path.join(HERE, "generated_cases.npz"), names=np.array(sorted(gen)), **flat)
    print("generated:", sorted(gen))


if __name__ == "__main__":
    main()
