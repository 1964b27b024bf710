"""Jacobi-iteration triangular solves on the GPU (f3r_trsv, and the
PRECOND_ILU0_JACOBI / PRECOND_ILU0_BAJ solver options) against the oracle
(bit for bit in the product arithmetic) and the reference's own solves
(tests/golden/trsv.npz, recorded from trsv/jacobi.hpp and trsv/baj.hpp)."""
import numpy as np
import pytest
import torch

import f3r_b200 as F
from oracle import oracle as O
from test_oracle_pins import load, same, trsv_matrices

pytestmark = pytest.mark.gpu

FORMS = {O.FORM_LOWER: F.TRSV_LOWER, O.FORM_LOWER_D: F.TRSV_LOWER_D, O.FORM_D_UPPER: F.TRSV_D_UPPER}


@pytest.fixture(scope="module")
def ctx():
    return F.Context(0)


def gpu_trsv(ctx, csr, form, x, iters, omega=1.0, baj=False):
    T = F.Trsv(ctx, F.HostMatrix.from_csr(*csr), FORMS[form], F.TRSV_BAJ if baj else F.TRSV_JACOBI, iters, omega)
    xin = torch.from_numpy(np.ascontiguousarray(x, np.float16)).cuda()
    out = torch.empty_like(xin)
    torch.cuda.synchronize()
    T.solve(xin, out)
    ctx.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("name", ["L", "Tl", "U"])
def test_jacobi_bit_exact_against_oracle(ctx, name):
    x = load("setup.npz")["bj_in"]
    r, i, v, form = trsv_matrices()[name]
    M = O.Mat.from_csr(r, i, v)
    for iters in (0, 1, 2, 5):
        for om in (1.0, 0.7, 1.3):
            got = gpu_trsv(ctx, (r, i, v), form, x, iters, om)
            want = O.jacobi_trsv(M, form, x, iters, om, False, O.ARITH_PRODUCT)
            assert same(got, want), (name, iters, om)


def test_jacobi_close_to_reference(ctx):
    x = load("setup.npz")["bj_in"]
    mats = trsv_matrices()
    for key, want in load("trsv.npz").items():
        if key.startswith("tl_"):
            continue
        name, kind, iters, om = key.split("_")
        if not kind.startswith("jac"):
            continue
        r, i, v, form = mats[name]
        got = gpu_trsv(ctx, (r, i, v), form, x, int(iters), float(om)).astype(np.float64)
        w = want.astype(np.float64)
        assert np.max(np.abs(got - w)) <= 4 * 2.0 ** -11 * np.max(np.abs(w)), key


@pytest.mark.parametrize("name", ["L", "Tl", "U"])
def test_baj_first_step_and_fixed_point(ctx, name):
    """BAJ's sweeps race by design; its first step (the diagonal scaling) and
    its fixed point (reached once the sweeps outnumber the dependency chain)
    are deterministic and equal the oracle's, bit for bit, and the fixed
    point is the one synchronous Jacobi reaches too"""
    x = load("setup.npz")["bj_in"]
    r, i, v, form = trsv_matrices()[name]
    M = O.Mat.from_csr(r, i, v)
    got1 = gpu_trsv(ctx, (r, i, v), form, x, 1, baj=True)
    assert same(got1, O.jacobi_trsv(M, form, x, 1, 1.0, True, O.ARITH_PRODUCT))
    n = len(r) - 1
    fixed = O.jacobi_trsv(M, form, x, n + 1, 1.0, True, O.ARITH_PRODUCT)
    got = gpu_trsv(ctx, (r, i, v), form, x, n + 1, baj=True)
    assert same(got, fixed)
    # synchronous Jacobi (omega 1) lands on the same values (up to the sign of zeros)
    jac = gpu_trsv(ctx, (r, i, v), form, x, n, 1.0)
    assert np.array_equal(jac.astype(np.float32), fixed.astype(np.float32))


def test_jacobi_global_ilu_64(ctx):
    """one global ILU(0) (a single block) of the 64^3 27-point matrix:
    262144 rows, three sweeps per factor, bit exact"""
    r, i, v = O.stencil27(64, 64, 64, variant=1)
    v = O.scaling(r, i, v)
    L, U = O.ilu0_bj(O.Mat.from_csr(r, i, v), 1)
    x = np.random.default_rng(5).standard_normal(len(r) - 1).astype(np.float16)
    for Mt, form in ((L, O.FORM_LOWER), (U, O.FORM_D_UPPER)):
        csr = Mt.csr()
        got = gpu_trsv(ctx, csr, form, x, 3, 0.9)
        assert same(got, O.jacobi_trsv(Mt, form, x, 3, 0.9, False, O.ARITH_PRODUCT))


def test_trsv_rejects_bad_input(ctx):
    r, i, v, form = trsv_matrices()["U"]
    with pytest.raises(F.F3RError, match="diagonal"):  # an upper factor read as lower
        F.Trsv(ctx, F.HostMatrix.from_csr(r, i, v), F.TRSV_LOWER)
    with pytest.raises(F.F3RError):
        F.Trsv(ctx, F.HostMatrix.from_csr(r, i, v), F.TRSV_D_UPPER, F.TRSV_BAJ, 0)
    with pytest.raises(F.F3RError):
        F.Trsv(ctx, F.HostMatrix.from_csr(r, i, v), F.TRSV_D_UPPER, F.TRSV_JACOBI, 2, 2.5)
    T = F.Trsv(ctx, F.HostMatrix.from_csr(r, i, v), F.TRSV_D_UPPER)
    x = torch.zeros(len(r) - 1, dtype=torch.float16, device="cuda")
    with pytest.raises(F.F3RError, match="alias"):
        T.solve(x, x)


def _system(variant, nx, seed=0):
    r, i, v = O.stencil27(nx, nx, nx, variant=variant)
    v = O.scaling(r, i, v)
    xs = np.random.default_rng(seed).uniform(-1, 1, len(r) - 1)
    b = O.spmv(r, i, v, xs, O.DT_F64, O.DT_F64, O.DT_F64)
    return r, i, v, b


@pytest.mark.parametrize("blocks,iters,omega", [(16, 2, 1.0), (1, 3, 1.0), (1, 2, 0.8)])
def test_solver_with_jacobi_ilu(ctx, blocks, iters, omega):
    r, i, v, b = _system(2, 24)
    kw = dict(m2=4, m3=2, m4=1, c=8)
    o = O.f3r_solve(O.Mat.from_csr(r, i, v), *O.ilu0_bj(O.Mat.from_csr(r, i, v), blocks), b,
                    O.params(precond=O.PRECOND_ILU0_JACOBI, tol=1e-10, trsv_iters=iters, trsv_omega=omega, **kw))
    S = F.Solver(ctx, F.HostMatrix.from_csr(r, i, v), rel_tol=1e-10, precond=F.PRECOND_ILU0_JACOBI,
                 ilu_blocks=blocks, trsv_iters=iters, trsv_omega=omega, **kw)
    res = S.solve(b, np.zeros(len(b)))
    assert res.is_solved and res.expl_rel_res < 1e-10
    assert o["solved"] and abs(res.res_iter - o["iters"]) <= 1, (res.res_iter, o["iters"])


def test_solver_with_baj_ilu(ctx):
    r, i, v, b = _system(2, 24, 1)
    S = F.Solver(ctx, F.HostMatrix.from_csr(r, i, v), rel_tol=1e-10, precond=F.PRECOND_ILU0_BAJ, ilu_blocks=1,
                 trsv_iters=3, m2=4, m3=2, m4=1, c=8)
    res = S.solve(b, np.zeros(len(b)))
    assert res.is_solved and res.expl_rel_res < 1e-10


@pytest.mark.parametrize("kind,sigma", [("stencil27", 1), ("stencil27", 256), ("diffusion7", 1)])
def test_global_level_scheduled_ilu(ctx, kind, sigma):
    """PRECOND_ILU0_LEVEL: one global ILU(0), its triangular solves spread
    over the whole GPU (dependency flags, no grid barrier).  Every row is
    computed as the single-block block-Jacobi kernel computes it, so the
    solve is ILU0_BJ with one block bit for bit, and it matches the oracle's
    single-block ILU(0) solve"""
    if kind == "stencil27":
        A = F.stencil27(24, 24, 24, 2, 0.5).scale()
    else:
        A = F.diffusion7(24, 22, 20, 1.5, 6.0, 3).scale()
    b = A.spmv(F.random_uniform(7, -1, 1, A.shape[0]))
    kw = dict(rel_tol=1e-10, m2=4, m3=2, m4=1, c=8, sell_sigma=sigma)
    xs, its = [], []
    for prec, blocks in ((F.PRECOND_ILU0_LEVEL, 112), (F.PRECOND_ILU0_BJ, 1)):
        S = F.Solver(ctx, F.HostMatrix.from_csr(*A.arrays()), precond=prec, ilu_blocks=blocks, **kw)
        x = np.zeros(len(b))
        r = S.solve(b, x)
        assert r.is_solved and r.expl_rel_res < 1e-10
        xs.append(x)
        its.append(r.res_iter)
        S.close()
    assert its[0] == its[1] and np.array_equal(xs[0], xs[1])
    rptr, idx, val = A.arrays()
    M = O.Mat.from_csr(rptr, idx, val)
    o = O.f3r_solve(M, *O.ilu0_bj(M, 1), b, O.params(precond=O.PRECOND_ILU0_BJ, tol=1e-10, m2=4, m3=2, m4=1, c=8))
    assert o["solved"] and abs(its[0] - o["iters"]) <= 1, (its[0], o["iters"])


def test_global_level_ilu_many_levels(ctx):
    """a 64^3 27-point matrix: 262,144 rows in several hundred levels, warps
    far ahead of the frontier; repeated solves reuse the device-side
    generation counter (graph replays)"""
    A = F.stencil27(64, 64, 64, 1, 0.5).scale()
    b = A.spmv(F.random_uniform(8, -1, 1, A.shape[0]))
    kw = dict(rel_tol=1e-10, m2=4, m3=2, m4=1, c=8)
    S = F.Solver(ctx, A, precond=F.PRECOND_ILU0_LEVEL, **kw)
    x1 = np.zeros(len(b))
    r1 = S.solve(b, x1)
    x2 = np.zeros(len(b))
    r2 = S.solve(b, x2)
    assert r1.is_solved and r1.expl_rel_res < 1e-10 and np.array_equal(x1, x2) and r1.res_iter == r2.res_iter


def test_ilu_weight_scales_after_the_solve(ctx):
    """With a fixed Richardson weight (F3R-Static, omega 1.2 on every call)
    the result of the block-Jacobi ILU(0) solve is scaled by omega only after
    the whole triangular solve, as the reference does (hout *= ome[0],
    work/src/f3r.cpp:216, 229), so the GPU's first outer residuals follow
    the oracle's closely (measured within 0.2%; a solve whose later rows read
    omega-scaled values moves them by several percent)"""
    A = F.stencil27(16, 16, 16, 1, 0.5).scale()
    r, i, v = A.arrays()
    b = A.spmv(F.random_uniform(3, -1, 1, A.shape[0]))
    M = O.Mat.from_csr(r, i, v)
    kw = dict(m2=8, m3=4, m4=2, static_weight=1.2)
    o = O.f3r_solve(M, *O.ilu0_bj(M, 16), b, O.params(precond=O.PRECOND_ILU0_BJ, tol=1e-10, **kw))
    seen = []
    S = F.Solver(ctx, A, rel_tol=1e-10, precond=F.PRECOND_ILU0_BJ, ilu_blocks=16, **kw)
    S.solve(b, np.zeros(len(b)), cond=lambda it, e: (seen.append(e), e / np.linalg.norm(b) < 1e-10)[1])
    got = np.array(seen[1:3]) / np.linalg.norm(b)
    assert np.all(np.abs(got / o["hist"][:2] - 1.0) < 1e-2), (got, o["hist"][:2])
