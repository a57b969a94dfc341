"""The front-shape autotuner (fplus_b200_autotune): it picks a shape from its candidates, the symbolic object keeps it,
and the factorization with it has the same pivots as with the default shape (the shape changes only how the work is
blocked)."""
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


@pytest.mark.parametrize("case", ["stencil3d", "pencil"])
def test_autotune_keeps_the_pivots(gpu, case):
    n, Ap, Ai, Ax = W.convdiff3d(20, 3) if case == "stencil3d" else W.pencil(modes=1, nc=512)
    S = F.analyze(n, Ap, Ai)
    p0 = S.factor(Ax).p
    w, nb, lu, ms = S.autotune(Ax)
    assert w in (128, 256, 512) and nb in (32, 64) and lu in (1, 2) and ms > 0
    N = S.factor(Ax)
    assert np.array_equal(N.p, p0)
    b = W.rhs(n, 1, np.iscomplexobj(Ax), 1)[0]
    assert O.backward_error(n, Ap, Ai, Ax, N.solve(b), b) <= 1e-14
