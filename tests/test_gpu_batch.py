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


def _check_block(S, B, X0=None):
    """solve_multi of B's rows (K columns in lockstep) against one single solve
    per row: the same iterate bit for bit and the same step count"""
    X = np.zeros_like(B) if X0 is None else X0.copy()
    res = S.solve_multi(B, X)
    for k in range(B.shape[0]):
        xk = np.zeros(B.shape[1]) if X0 is None else X0[k].copy()
        rk = S.solve(B[k].copy(), xk)
        assert np.array_equal(X[k], xk), k
        assert res[k].res_iter == rk.res_iter and res[k].is_solved == rk.is_solved, (k, res[k], rk)
        assert res[k].restarts == rk.restarts and res[k].expl_rel_res == rk.expl_rel_res, k
    return res


@pytest.mark.parametrize("nrhs", [2, 5, 8, 16, 17, 19])
@pytest.mark.parametrize("layout", [dict(sell_align=1), dict(sell_align=0), dict(sell_sigma=256),
                                    dict(sell_align=1, sell_c=64)])
def test_block_solve_columns_bit_identical(nrhs, layout):
    """up to 16 right-hand sides per lockstep block (block SELL products over
    interleaved columns; padding columns inactive), 19 = 16 + 3 in two
    blocks, 17 = 16 + one column solved alone: every column is its single
    solve, bit for bit"""
    ctx = F.Context(0)
    A = F.stencil27(18, 17, 16, 2, 0.5).scale()
    S = F.Solver(ctx, A, rel_tol=1e-10, c=4, **layout)
    B = np.ascontiguousarray(np.random.default_rng(nrhs).standard_normal((nrhs, A.shape[0])))
    res = _check_block(S, B)
    assert all(r.is_solved and r.expl_rel_res < 1e-10 for r in res)


@pytest.mark.parametrize("layout", [dict(sell_align=0), dict(sell_align=1), dict(sell_align=1, sell_c=64)])
def test_block_solve_general_sdainv_and_uneven_convergence(layout):
    """non-diagonal SDAINV factors (block products of W^T and Z; aligned: the
    mixed offset-aligned form, or 64-row slices); columns that finish at
    different steps (an exact initial guess stops at step 0, a smooth
    right-hand side converges sooner than noise) leave the lockstep without
    disturbing the others"""
    ctx = F.Context(0)
    A = F.diffusion7(16, 15, 14, 1.5, 3.0, 4).scale()
    S = F.Solver(ctx, A, rel_tol=1e-10, c=4, **layout)
    assert not S.info()[1]
    n = A.shape[0]
    rng = np.random.default_rng(9)
    xs = F.random_uniform(2, -1.0, 1.0, n)
    B = np.ascontiguousarray(np.stack([rng.standard_normal(n), A.spmv(np.ones(n)), A.spmv(xs),
                                       rng.standard_normal(n) * 1e3]))
    X0 = np.zeros_like(B)
    X0[2] = xs  # already the solution
    res = _check_block(S, B, X0)
    assert res[2].res_iter == 0 and res[0].res_iter > 0


@pytest.mark.parametrize("scale", [0, 4])
def test_block_solve_with_scaled_richardson_input(scale):
    """with half_scale_log2 > 0 level 3 keeps an fp32 Z basis (R's output is
    hout x 2^-k), without it an fp16 one; either way every block column is
    its single solve bit for bit"""
    ctx = F.Context(0)
    A = F.stencil27(14, 13, 12, 2, 0.5).scale()
    S = F.Solver(ctx, A, rel_tol=1e-10, c=4, half_scale_log2=scale)
    B = np.ascontiguousarray(np.random.default_rng(5).standard_normal((6, A.shape[0])))
    res = _check_block(S, B)
    assert all(r.is_solved and r.expl_rel_res < 1e-10 for r in res)


def test_block_solve_restarts_in_lockstep():
    """a short outer restart length: every column restarts (its x += Z y, then
    a new residual) in the same step as its single solve"""
    ctx = F.Context(0)
    A = F.stencil27(16, 16, 16, 1, 0.5).scale()
    S = F.Solver(ctx, A, rel_tol=1e-10, c=4, m_outer=1, max_restarts=30)
    B = np.ascontiguousarray(np.random.default_rng(1).standard_normal((4, A.shape[0])))
    res = _check_block(S, B)
    assert all(r.restarts > 1 and r.is_solved for r in res)


def test_block_solve_multi_rhs_device_and_static_weight():
    """device blocks (torch), F3R-Static and m3 = 0 through the block engine"""
    ctx = F.Context(0)
    A = F.stencil27(14, 14, 14, 2, 0.5).scale()
    for kw in (dict(static_weight=1.1), dict(m3=0, m2=16), dict(m4=3, c=2)):
        S = F.Solver(ctx, A, rel_tol=1e-10, **kw)
        B = np.ascontiguousarray(np.random.default_rng(4).standard_normal((6, A.shape[0])))
        _check_block(S, B)
        Bd = torch.from_numpy(B).cuda()
        Xd = torch.zeros_like(Bd)
        S.solve_multi(Bd, Xd)
        Xh = np.zeros_like(B)
        S.solve_multi(B, Xh)
        assert np.array_equal(Xd.cpu().numpy(), Xh), kw


def _fields(kind, count, nx=14):
    """count systems of one pattern: log-normal diffusion fields (general
    SDAINV factors) or the 27-point stencil with different beta (diagonal)"""
    out = []
    for s in range(count):
        if kind == "diffusion":
            A = F.diffusion7(nx, nx - 1, nx + 1, 1.5, 3.0, 100 + s)
        else:
            A = F.stencil27(nx, nx - 1, nx + 1, 2, 0.1 + 0.1 * s)
        out.append(A.scale())
    return out


@pytest.mark.parametrize("kind,count,sigma", [("diffusion", 3, 1), ("diffusion", 8, 1), ("stencil", 5, 1),
                                              ("stencil", 2, 256), ("diffusion", 16, 256)])
def test_batch_of_one_pattern_equals_single_solves(kind, count, sigma):
    """systems of one pattern solved together (f3r_batch: every column of the
    block solve its own system, values interleaved, SDAINV factors on the
    union pattern): each system's iterate is its single solve's (packed SELL,
    the batch's layout), bit for bit"""
    ctx = F.Context(0)
    systems = _fields(kind, count)
    B = F.Batch(ctx, systems, rel_tol=1e-10, c=4, sell_sigma=sigma)
    c, k, diag = B.info()
    assert c == count and k >= count and diag == (kind == "stencil")
    n = systems[0].shape[0]
    rng = np.random.default_rng(count)
    bs = [rng.standard_normal(n) for _ in range(count)]
    xs = [np.zeros(n) for _ in range(count)]
    res = B.solve(bs, xs)
    for i, A in enumerate(systems):
        S = F.Solver(ctx, A, rel_tol=1e-10, c=4, sell_sigma=sigma, sell_align=0)
        x = np.zeros(n)
        r = S.solve(bs[i].copy(), x)
        assert np.array_equal(xs[i], x), i
        assert res[i].res_iter == r.res_iter and res[i].is_solved and res[i].expl_rel_res < 1e-10, i
        S.close()
    # device vectors, and the same solve again (graphs replayed)
    bd = [torch.from_numpy(b).cuda() for b in bs]
    xd = [torch.zeros_like(b) for b in bd]
    B.solve(bd, xd)
    for i in range(count):
        assert np.array_equal(xd[i].cpu().numpy(), xs[i])


def test_batch_with_given_factors_and_rejections():
    """given SDAINV factors per system (f3r_solver_create_factors' form), and
    the batch's checks: one pattern, at most 16 systems, SDAINV only"""
    ctx = F.Context(0)
    systems = _fields("diffusion", 4)
    fac = [A.sdainv() for A in systems]
    B = F.Batch(ctx, systems, factors=fac, rel_tol=1e-10, c=4)
    n = systems[0].shape[0]
    bs = [np.ones(n) * (i + 1) for i in range(4)]
    xs = [np.zeros(n) for _ in range(4)]
    res = B.solve(bs, xs)
    for i, A in enumerate(systems):
        S = F.Solver(ctx, A, factors=fac[i], rel_tol=1e-10, c=4, sell_align=0)
        x = np.zeros(n)
        S.solve(bs[i].copy(), x)
        assert np.array_equal(xs[i], x) and res[i].is_solved
    with pytest.raises(F.F3RError, match="pattern"):
        F.Batch(ctx, [systems[0], F.stencil27(14, 13, 15, 2, 0.5).scale()])
    with pytest.raises(F.F3RError):
        F.Batch(ctx, _fields("stencil", 17, nx=6))
    with pytest.raises(F.F3RError):
        F.Batch(ctx, systems, precond=F.PRECOND_ILU0_BJ, ilu_blocks=4)


@pytest.mark.parametrize("layout", ["aligned64", "packed"])
def test_block_solve_unit_diagonal_is_identical(layout):
    """the lockstep block solve (4 right-hand sides) and a full batch of 4
    stencil systems with unit fp16 diagonal factors: taking the constant gives
    the iterates of the solves that load the factors, bit for bit"""
    ctx = F.Context(0)
    kw = dict(sell_c=64) if layout == "aligned64" else dict(sell_align=0)
    A = F.stencil27(16, 15, 14, 2, 0.5).scale()
    n = A.shape[0]
    rng = np.random.default_rng(21)
    B = np.ascontiguousarray(rng.standard_normal((4, n)))
    outs = []
    for load in (0, 1):
        S = F.Solver(ctx, A, rel_tol=1e-10, c=4, diag_load=load, **kw)
        assert S.unit_diagonal == (load == 0)
        X = np.zeros_like(B)
        res = S.solve_multi(B, X)
        assert all(r.is_solved for r in res)
        outs.append((X, [r.res_iter for r in res]))
        S.close()
    assert outs[0][1] == outs[1][1] and np.array_equal(outs[0][0], outs[1][0])
    systems = _fields("stencil", 4)
    bs = [rng.standard_normal(systems[0].shape[0]) for _ in range(4)]
    got = []
    for load in (0, 1):
        Bt = F.Batch(ctx, systems, rel_tol=1e-10, c=4, diag_load=load)
        assert Bt.unit_diagonal == (load == 0)
        xs = [np.zeros_like(b) for b in bs]
        res = Bt.solve(bs, xs)
        assert all(r.is_solved for r in res)
        got.append(xs)
        Bt.close()
    for i in range(4):
        assert np.array_equal(got[0][i], got[1][i]), i
