"""Nested F3R solves on the GPU against the oracle's restatement and the
reference's own solve (compiled in place, run on the host)."""
import numpy as np
import pytest
import torch

import f3r_b200 as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return F.Context(0)


def system(nx, variant=2, seed=0):
    A = F.stencil27(nx, nx, nx, variant, 0.5).scale()
    n = A.shape[0]
    xs = F.random_uniform(seed, -1.0, 1.0, n)
    b = A.spmv(xs)
    return A, b, xs


def oracle_solve(A, b, precond=O.PRECOND_SDAINV, blocks=16, **kw):
    rptr, idx, val = A.arrays()
    M = O.Mat.from_csr(rptr, idx, val)
    if precond == O.PRECOND_SDAINV:
        Z, W = O.sdainv(M)
        P1, P2 = W, Z
    else:
        P1, P2 = O.ilu0_bj(M, blocks)
    p = O.params(precond=precond, **kw)
    return O.f3r_solve(M, P1, P2, b, p)


@pytest.mark.parametrize("nx,graphs,index16", [(16, 1, 0), (24, 0, 0), (32, 1, 0), (24, 1, 1)])
def test_solve_matches_oracle(ctx, nx, graphs, index16):
    A, b, xs = system(nx)
    S = F.Solver(ctx, A, rel_tol=1e-10, use_graphs=graphs, sell_index16=index16)
    assert S.info()[0].index_bits == (16 if index16 else 32)
    x = np.zeros_like(b)
    r = S.solve(b, x)
    o = oracle_solve(A, b, tol=1e-10)
    assert r.is_solved and o["solved"]
    assert r.expl_rel_res <= 1e-10
    assert abs(r.res_iter - o["iters"]) <= 1
    assert r.inner_applications == r.res_iter * 32
    assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-7


@pytest.mark.parametrize("scale", [3, 6])
def test_scaled_richardson_input_matches_oracle(ctx, scale):
    """half_scale_log2 = k scales R's fp16 input by 2^k and its output back by
    2^-k, so level 3 keeps its Z basis in fp32 (R's output is no longer an
    fp16 value): the solve converges as the oracle's with the same scaling"""
    A, b, xs = system(20)
    S = F.Solver(ctx, A, rel_tol=1e-10, half_scale_log2=scale)
    x = np.zeros_like(b)
    r = S.solve(b, x)
    o = oracle_solve(A, b, tol=1e-10, half_scale_log2=scale)
    assert r.is_solved and o["solved"]
    assert r.expl_rel_res <= 1e-10
    assert abs(r.res_iter - o["iters"]) <= 1
    assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-7


def test_solve_matches_reference(ctx):
    ref = O.Ref("golden")
    A, b, _ = system(24, variant=1)
    rptr, idx, val = A.arrays()
    rr = ref.f3r_solve(0, rptr, idx, val, b, tol=1e-10)
    S = F.Solver(ctx, A, rel_tol=1e-10)
    x = np.zeros_like(b)
    r = S.solve(b, x)
    assert rr["solved"] and r.is_solved
    assert abs(r.res_iter - rr["iters"]) <= 1
    assert r.expl_rel_res <= 1e-10


def test_history_and_cond(ctx):
    A, b, _ = system(20)
    seen = []

    def cond(i, e):
        seen.append((i, e))
        return e / np.linalg.norm(b) < 1e-9

    S = F.Solver(ctx, A)
    x = np.zeros_like(b)
    r = S.solve(b, x, cond)
    assert r.is_solved
    assert seen[0][0] == 0 and [s[0] for s in seen[1:]] == list(range(1, len(seen)))
    o = oracle_solve(A, b, tol=1e-9)
    got = np.array([e for _, e in seen[1:]]) / np.linalg.norm(b)
    assert len(got) == len(o["hist"]) or abs(len(got) - len(o["hist"])) <= 1
    k = min(len(got), len(o["hist"]))
    # first outer step: same residual reduction within fp16 noise
    assert abs(np.log10(got[0]) - np.log10(o["hist"][0])) < 0.5


def test_device_pointers_and_x0(ctx):
    A, b, xs = system(16)
    S = F.Solver(ctx, A, rel_tol=1e-10)
    bt = torch.from_numpy(b).cuda()
    xt = torch.zeros_like(bt)
    r = S.solve(bt, xt)
    assert r.is_solved and r.expl_rel_res <= 1e-10
    # warm start from the solution: converged at step 0
    r2 = S.solve(bt, xt)
    assert r2.is_solved and r2.res_iter == 0


@pytest.mark.parametrize("sigma", [1, 256])
def test_sigma_and_m4(ctx, sigma):
    A, b, xs = system(20)
    for m4 in (1, 2, 3):
        S = F.Solver(ctx, A, rel_tol=1e-10, sell_sigma=sigma, m4=m4, c=4)
        x = np.zeros_like(b)
        r = S.solve(b, x)
        o = oracle_solve(A, b, tol=1e-10, m4=m4, c=4)
        assert r.is_solved and r.expl_rel_res <= 1e-10, (sigma, m4)
        assert abs(r.res_iter - o["iters"]) <= 1, (sigma, m4, r.res_iter, o["iters"])


def test_general_sdainv(ctx):
    """non-diagonal SDAINV factors (log-normal diffusion) through SELL SpMVs"""
    A = F.diffusion7(16, 16, 16, 1.5, 3.0, 3).scale()
    n = A.shape[0]
    xs = F.random_uniform(1, -1, 1, n)
    b = A.spmv(xs)
    S = F.Solver(ctx, A, rel_tol=1e-10, c=8)
    _, diag = S.info()
    assert not diag
    x = np.zeros_like(b)
    r = S.solve(b, x)
    o = oracle_solve(A, b, tol=1e-10, c=8)
    assert r.is_solved and r.expl_rel_res <= 1e-10
    assert abs(r.res_iter - o["iters"]) <= max(1, 0.1 * o["iters"])


def test_ilu_bj(ctx):
    A, b, xs = system(16, variant=0)
    S = F.Solver(ctx, A, rel_tol=1e-10, precond=F.PRECOND_ILU0_BJ, ilu_blocks=16)
    x = np.zeros_like(b)
    r = S.solve(b, x)
    o = oracle_solve(A, b, precond=O.PRECOND_ILU0_BJ, blocks=16, tol=1e-10)
    assert r.is_solved and r.expl_rel_res <= 1e-10
    assert abs(r.res_iter - o["iters"]) <= 1


def test_invalid_params(ctx):
    A = F.stencil27(8, 8, 8).scale()
    for bad in (dict(m2=200), dict(m3=-1), dict(m3=128), dict(static_weight=-1.0), dict(m4=17)):
        with pytest.raises(F.F3RError):
            F.Solver(ctx, A, **bad)
    with pytest.raises(F.F3RError):
        F.Solver(ctx, A, precond=F.PRECOND_ILU0_BJ, ilu_blocks=112)


@pytest.mark.parametrize("kind", ["stencil27", "diffusion7"])
def test_csr_format_solve_is_identical(ctx, kind):
    """format CSR runs every product through the CSR kernel, in the packed
    SELL kernel's launch geometry and column order: the solve is the packed
    sigma = 1 layout's bit for bit (the diffusion matrix has non-diagonal
    SDAINV factors, so W^T and Z are CSR too)"""
    A = (F.stencil27(20, 20, 20, 2, 0.5) if kind == "stencil27" else F.diffusion7(18, 18, 18, 1.5, 6.0, 2)).scale()
    b = A.spmv(F.random_uniform(5, -1, 1, A.shape[0]))
    xs, its = [], []
    for fmt in (F.FORMAT_SELL, F.FORMAT_CSR):
        S = F.Solver(ctx, A, rel_tol=1e-10, c=8, format=fmt)
        info, diag = S.info()
        assert info.slice_height == (0 if fmt == F.FORMAT_CSR else 32)
        assert diag == (kind == "stencil27")
        x = np.zeros(len(b))
        r = S.solve(b, x)
        assert r.is_solved and r.expl_rel_res < 1e-10
        xs.append(x)
        its.append(r.res_iter)
    assert its[0] == its[1] and np.array_equal(xs[0], xs[1])
    with pytest.raises(F.F3RError, match="CSR"):
        F.Solver(ctx, A, format=F.FORMAT_CSR, sell_sigma=256)
    with pytest.raises(F.F3RError, match="format"):
        F.Solver(ctx, A, format=7)


@pytest.mark.parametrize("kind", ["stencil27", "ragged"])
def test_layout_autotuner(ctx, kind):
    """sell_autotune times every candidate layout's fp16 product at set-up and
    solves in the fastest: the solve is the one made with that layout given
    explicitly, bit for bit"""
    if kind == "stencil27":
        A = F.stencil27(24, 24, 24, 2, 0.5).scale()
    else:
        A = F.diffusion7(20, 17, 13, 1.0, 3.0, 9).scale()
    b = A.spmv(F.random_uniform(3, -1, 1, A.shape[0]))
    S = F.Solver(ctx, A, rel_tol=1e-10, c=8, sell_autotune=1)
    info, _ = S.info()
    fmt = F.FORMAT_CSR if info.slice_height == 0 else F.FORMAT_SELL
    assert info.sigma in (1, 256)
    x1 = np.zeros(len(b))
    r1 = S.solve(b, x1)
    assert r1.is_solved and r1.expl_rel_res < 1e-10
    kw = dict(format=fmt, sell_sigma=info.sigma, sell_align=1 if info.index_bits == 0 else 0,
              sell_c=info.slice_height if info.slice_height else 32,
              sell_index16=1 if info.index_bits == 16 else 0)
    S2 = F.Solver(ctx, A, rel_tol=1e-10, c=8, **kw)
    i2, _ = S2.info()
    assert (i2.sigma, i2.index_bits, i2.slice_height) == (info.sigma, info.index_bits, info.slice_height)
    x2 = np.zeros(len(b))
    r2 = S2.solve(b, x2)
    assert r2.res_iter == r1.res_iter and np.array_equal(x1, x2)


def test_aligned_sell_solve_is_identical(ctx):
    """the offset-aligned layout changes no sum: the solve's iterate is the
    packed layout's bit for bit (sigma 1, SDAINV factors aligned too)"""
    A = F.stencil27(20, 20, 20, 2, 0.5).scale()
    b = A.spmv(F.random_uniform(2, -1, 1, A.shape[0]))
    xs = []
    for align in (0, 1):
        S = F.Solver(ctx, A, rel_tol=1e-10, c=8, sell_align=align)
        x = np.zeros(len(b))
        r = S.solve(b, x)
        assert r.is_solved and r.expl_rel_res < 1e-10
        xs.append(x)
    assert np.array_equal(xs[0], xs[1])


@pytest.mark.parametrize("dims", [(24, 20, 18), (3, 3, 3), (5, 4, 7)])
def test_slice_height_64_solve_is_identical(ctx, dims):
    """the solver on 64-row slices (sell_c = 64) reproduces the 32-row
    aligned layout's solve bit for bit, the fused Richardson steps and the
    weight updates included; 27 and 140 rows: one partial slice, and a
    partial last slice"""
    A = F.stencil27(*dims, 2, 0.5).scale()
    b = A.spmv(F.random_uniform(7, -1, 1, A.shape[0]))
    xs = []
    for kw in (dict(sell_align=1), dict(sell_c=64)):
        S = F.Solver(ctx, A, rel_tol=1e-10, c=4, **kw)
        info, _ = S.info()
        assert info.slice_height == kw.get("sell_c", 32)
        x = np.zeros(len(b))
        r = S.solve(b, x)
        assert r.is_solved and r.expl_rel_res < 1e-10
        xs.append(x)
        S.close()
    assert np.array_equal(xs[0], xs[1])
    with pytest.raises(F.F3RError):
        F.Solver(ctx, A, sell_c=64, sell_sigma=256)


@pytest.mark.parametrize("kw", [dict(c=4), dict(sell_c=64, c=4), dict(m4=3, c=2), dict(sell_sigma=256, c=8)])
def test_unit_diagonal_solve_is_identical(ctx, kw):
    """the scaled stencil's SDAINV factors are diagonal and 1 in fp16: the
    Richardson kernels then take the constant 1 instead of loading it, and the
    solve is the one that loads the factors (diag_load = 1) bit for bit --
    plain steps, weight updates (c small), three Richardson steps, 64-row
    slices and sigma-sorted rows"""
    A = F.stencil27(20, 18, 16, 2, 0.5).scale()
    b = A.spmv(F.random_uniform(11, -1, 1, A.shape[0]))
    xs, its = [], []
    for load in (0, 1):
        S = F.Solver(ctx, A, rel_tol=1e-10, diag_load=load, **kw)
        assert S.info()[1] and S.unit_diagonal == (load == 0)
        x = np.zeros(len(b))
        r = S.solve(b, x)
        assert r.is_solved and r.expl_rel_res < 1e-10
        xs.append(x)
        its.append(r.res_iter)
        S.close()
    assert its[0] == its[1] and np.array_equal(xs[0], xs[1])


def test_non_unit_diagonal_loads_factors(ctx):
    """diagonal factors that are not all 1 in fp16 (an unscaled stencil) keep
    the loads; diag_load takes 0 or 1 only"""
    A = F.stencil27(12, 12, 12, 2, 0.5)
    S = F.Solver(ctx, A, rel_tol=1e-10, c=8)
    info, diag = S.info()
    if diag:
        assert not S.unit_diagonal
    b = A.spmv(F.random_uniform(4, -1, 1, A.shape[0]))
    x = np.zeros(len(b))
    r = S.solve(b, x)
    assert r.is_solved and r.expl_rel_res < 1e-10
    S.close()
    with pytest.raises(F.F3RError):
        F.Solver(ctx, A, diag_load=2)
