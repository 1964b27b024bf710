"""Several right-hand sides per solver (f3r_solver_solve_multi) and several
solvers at once (f3r_solve_batch): every column and every system must come
out exactly as its own single solve does."""
import numpy as np
import pytest
import torch

import f3r_b200 as F

pytestmark = pytest.mark.gpu


def single(S, b):
    x = np.zeros_like(b)
    r = S.solve(b, x)
    return x, r


def test_multi_rhs_equals_single_solves():
    ctx = F.Context(0)
    A = F.stencil27(14, 15, 16, 2, 0.5).scale()
    n = A.shape[0]
    S = F.Solver(ctx, A, rel_tol=1e-10, c=8)
    rng = np.random.default_rng(3)
    B = np.ascontiguousarray(rng.standard_normal((3, n)))
    B[1] = 0.0  # a zero right-hand side stops before the first step
    X = np.zeros_like(B)
    res = S.solve_multi(B, X)
    assert len(res) == 3
    for k in range(3):
        xk, rk = single(S, B[k].copy())
        assert np.array_equal(X[k], xk), k
        assert res[k].res_iter == rk.res_iter
    assert res[1].res_iter == 0 and not X[1].any()
    assert res[0].is_solved and res[0].expl_rel_res < 1e-10
    # the same on device memory
    Bd = torch.from_numpy(B).cuda()
    Xd = torch.zeros_like(Bd)
    S.solve_multi(Bd, Xd)
    assert np.array_equal(Xd.cpu().numpy(), X)
    with pytest.raises(ValueError):
        S.solve_multi(B[:, :-1].copy(), X[:, :-1].copy())


def test_batch_equals_single_solves():
    """five systems of different kinds and sizes, two of them sharing a
    context (they run one after the other), the others concurrently"""
    mats = [F.stencil27(12, 12, 12, 2, 0.5), F.diffusion7(16, 14, 12, 1.0, 3.0, 7), F.stencil27(20, 9, 10, 1, 0.5),
            F.diffusion7(10, 10, 30, 1.5, 2.0, 8), F.stencil27(8, 8, 8, 0, 0.5)]
    ctxs = [F.Context(0) for _ in range(4)]
    solvers = []
    for i, A in enumerate(mats):
        A.scale()
        solvers.append(F.Solver(ctxs[min(i, 3)], A, rel_tol=1e-10, c=8))  # systems 3 and 4 share a context
    rng = np.random.default_rng(5)
    systems = []
    for i, S in enumerate(solvers):
        B = np.ascontiguousarray(rng.standard_normal((1 + i % 3, S.n)))
        systems.append((S, B, np.zeros_like(B)))
    out = F.solve_batch(systems)
    for (S, B, X), res in zip(systems, out):
        assert len(res) == B.shape[0]
        for k in range(B.shape[0]):
            xk, rk = single(S, B[k].copy())
            assert np.array_equal(X[k], xk)
            assert res[k].is_solved and res[k].expl_rel_res < 1e-10 and res[k].res_iter == rk.res_iter
