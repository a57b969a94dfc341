"""The batch form: many independent factorizations and solves (uneven pencils, shifts of one pattern), concurrently on
worker streams and captured as one CUDA graph, against the same calls made one by one."""
import numpy as np
import pytest

import fplus_b200 as F
from fplus_b200 import workloads as W
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    import torch
    assert torch.cuda.is_available(), "the GPU tests need a CUDA device"
    torch.cuda.init()
    return torch.device("cuda:0")


def _pencils(count, seed):
    return W.pencil_batch(count=count, nmin=500, nmax=2500, seed=seed)


def test_graph_refactor_and_solve_match_uncaptured(gpu):
    """Capture 12 uneven pencils' refactorization + solve (2 right-hand sides each) as one graph, replay it twice with
    new values: every solution equals the uncaptured factor + solve of the same values, bit for bit, and solves to a
    backward error <= 1e-14."""
    mats = _pencils(12, 31)
    syms = [F.analyze(n, Ap, Ai) for n, Ap, Ai, _ in mats]
    nums = [S.factor(m[3]) for S, m in zip(syms, mats)]
    G = F.BatchGraph(nums, 2)
    rng = np.random.default_rng(5)
    for rep in range(2):
        # new values with the same pivot order (a phase, and relative changes of 1e-9): the plans' dense-chain starts hold
        vals = [m[3] * (1.0 + 0.05 * (rep + 1) * 1j) * (1.0 + 1e-9 * rng.standard_normal(m[3].size)) for m in mats]
        rhs = [W.rhs(m[0], 2, True, 40 + 3 * k + rep).T.copy(order="F") for k, m in enumerate(mats)]
        for k in range(len(mats)):
            G.upload(k, vals[k], rhs[k])
        G.launch()
        assert G.status() == [0] * len(mats)
        for k, m in enumerate(mats):
            X = G.download(k)
            Xr = syms[k].factor(vals[k]).solve(rhs[k])
            assert np.array_equal(X, Xr), f"rep {rep} matrix {k}: the captured solve differs from the uncaptured one"
            for r in range(2):
                assert O.backward_error(m[0], m[1], m[2], vals[k], X[:, r], rhs[k][:, r]) <= 1e-14


def test_graph_reports_values_beyond_the_range_guard(gpu):
    """Values the Ruiz range guard would rescale on the host cannot take the captured path: that matrix reports
    FPLUS_ERR_BADARG, the others solve."""
    mats = _pencils(3, 32)
    syms = [F.analyze(n, Ap, Ai) for n, Ap, Ai, _ in mats]
    nums = [S.factor(m[3]) for S, m in zip(syms, mats)]
    G = F.BatchGraph(nums, 1)
    for k, m in enumerate(mats):
        G.upload(k, m[3] * (1e200 if k == 1 else 1.0), W.rhs(m[0], 1, True, k)[0])
    G.launch()
    st = G.status()
    assert st[1] == F.FPLUS_ERR_BADARG and st[0] == 0 and st[2] == 0


def test_worker_batch_matches_one_by_one(gpu):
    """fplus_b200_factor_batch / solve_batch on 16 uneven pencils: bit-identical to the one-by-one calls, and the device
    span of the batch is measured from the jobs' own events."""
    mats = _pencils(16, 33)
    syms = [F.analyze(n, Ap, Ai) for n, Ap, Ai, _ in mats]
    rhs = [W.rhs(m[0], 8, True, 7 + k).T.copy(order="F") for k, m in enumerate(mats)]
    Ns = F.factor_batch(syms, [m[3] for m in mats], nworkers=8)
    Xs = F.solve_batch(Ns, rhs, nworkers=8)
    assert F.batch_span_ms(Ns) > 0.0
    for S, m, b, X in zip(syms, mats, rhs, Xs):
        assert np.array_equal(X, S.factor(m[3]).solve(b))
