"""F3R-Static and the depth ablations on the GPU against the reference's own
solves (static.cpp, depth.cpp, recorded in tests/golden/solves.npz), and the
F2 form's wide fp32 level (64 basis vectors, chunked dot pass)."""
import numpy as np
import pytest

import f3r_b200 as F
from test_oracle_pins import VARIANTS, golden_system

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return F.Context(0)


@pytest.mark.parametrize("name", sorted(VARIANTS))
def test_variant_matches_reference(ctx, name):
    r, i, v, b, xs, sol = golden_system(name)
    A = F.HostMatrix.from_csr(r, i, v)
    S = F.Solver(ctx, A, rel_tol=1e-10, precond=F.PRECOND_ILU0_BJ, ilu_blocks=int(sol[name + "_blocks"]), c=8,
                 **VARIANTS[name])
    x = np.zeros(len(b))
    res = S.solve(b, x)
    ref_iters = int(sol[name + "_iters"])
    assert res.is_solved and res.expl_rel_res < 1e-10
    assert abs(res.res_iter - ref_iters) <= max(1, round(0.1 * ref_iters)), (res.res_iter, ref_iters)
    calls_per_outer = VARIANTS[name]["m2"] * max(VARIANTS[name]["m3"], 1)
    assert res.inner_applications == res.res_iter * calls_per_outer


def test_static_weight_never_updates(ctx):
    """with a fixed weight the update kernels never run: the same solve with
    c = 1 (an update every call) and c = 64 is identical"""
    A = F.stencil27(12, 12, 12, 1, 0.5).scale()
    b = A.spmv(F.random_uniform(0, -1, 1, A.shape[0]))
    xs = []
    for c in (1, 64):
        S = F.Solver(ctx, A, rel_tol=1e-10, c=c, static_weight=1.0)
        x = np.zeros(len(b))
        S.solve(b, x)
        xs.append(x)
    assert np.array_equal(xs[0], xs[1])


@pytest.mark.parametrize("name", ["sstep1_hpgmp16", "sstep2_hpgmp16", "sstep3_hpgmp16"])
def test_sstep_matches_reference_and_oracle(ctx, name):
    """sFGMRES inner levels (solver/gmres2.hpp:137-221) against the
    reference's solve and the oracle's product arithmetic"""
    from oracle import oracle as O
    from test_oracle_pins import SSTEP
    r, i, v, b, xs, sol = golden_system(name)
    S = F.Solver(ctx, F.HostMatrix.from_csr(r, i, v), rel_tol=1e-10, c=8, inner_sstep=SSTEP[name])
    res = S.solve(b, np.zeros(len(b)))
    A = O.Mat.from_csr(r, i, v)
    Z, W = O.sdainv(A)
    o = O.f3r_solve(A, W, Z, b, O.params(c=8, tol=1e-10, sstep=SSTEP[name]))
    ref_iters = int(sol[name + "_iters"])
    assert res.is_solved and res.expl_rel_res < 1e-10
    assert abs(res.res_iter - ref_iters) <= 1, (res.res_iter, ref_iters)
    assert abs(res.res_iter - o["iters"]) <= 1, (res.res_iter, o["iters"])


def test_sstep_large_level_and_graphs(ctx):
    """both levels s-step with a wide level 2 (16 raw vectors, chunked dots),
    graphs on and off give the same iterate"""
    A = F.stencil27(20, 20, 20, 2, 0.5).scale()
    b = A.spmv(F.random_uniform(3, -1, 1, A.shape[0]))
    xs = []
    for graphs in (1, 0):
        S = F.Solver(ctx, A, rel_tol=1e-10, c=8, m2=16, m3=3, inner_sstep=3, use_graphs=graphs)
        x = np.zeros(len(b))
        res = S.solve(b, x)
        assert res.is_solved and res.expl_rel_res < 1e-10
        xs.append(x)
    assert np.array_equal(xs[0], xs[1])


HALF = {"f4_hpgmp16": (8, 4, 2), "f3h_hpgmp16": (8, 0, 8), "f2h_hpgmp16": (0, 0, 64)}


@pytest.mark.parametrize("name", sorted(HALF))
def test_half_level_variants(ctx, name):
    """F4 / F3H / F2H (depth.cpp:122-167): the fp16-vector FGMRES level below
    the fp32 levels (or directly below the outer level, m2 = 0) solves the
    golden system to 1e-10 with the expected count of preconditioner calls;
    graphs on and off give the same iterate (the history against the
    reference is checked in test_gpu_history.py)"""
    from history_band import CASES
    r, i, v, b, xs, sol = golden_system(name)
    m2, m3, mh = HALF[name]
    assert (CASES[name]["m2"], CASES[name]["m3"], CASES[name]["half_m"]) == (m2, m3, mh)
    xsol = []
    for graphs in (1, 0):
        S = F.Solver(ctx, F.HostMatrix.from_csr(r, i, v), rel_tol=1e-10, use_graphs=graphs, **CASES[name])
        x = np.zeros(len(b))
        res = S.solve(b, x)
        assert res.is_solved and res.expl_rel_res < 1e-10
        assert res.inner_applications == res.res_iter * max(m2, 1) * max(m3, 1) * mh
        xsol.append(x)
        S.close()
    assert np.array_equal(xsol[0], xsol[1])
    assert np.linalg.norm(xsol[0] - xs) / np.linalg.norm(xs) < 1e-7


def test_half_level_with_sdainv_richardson(ctx):
    """the fp16-vector level over the adaptive Richardson with diagonal SDAINV
    (m4 = 2, weights updated every c-th call): R runs on the level's fp16
    vectors in both the fused and the weight-update paths"""
    A = F.stencil27(20, 20, 20, 2, 0.5).scale()
    b = A.spmv(F.random_uniform(4, -1, 1, A.shape[0]))
    for m2, m3, mh in ((8, 0, 4), (4, 2, 2), (0, 0, 16)):
        S = F.Solver(ctx, A, rel_tol=1e-10, c=4, m2=m2, m3=m3, half_m=mh, m4=2)
        assert S.info()[1]  # diagonal SDAINV
        x = np.zeros(len(b))
        res = S.solve(b, x)
        assert res.is_solved and res.expl_rel_res < 1e-10, (m2, m3, mh)
        S.close()


def test_half_level_rejects_bad_nesting(ctx):
    A = F.stencil27(8, 8, 8).scale()
    for bad in (dict(m2=0), dict(m2=0, half_m=4, m3=2), dict(m2=0, half_m=4, inner_sstep=1), dict(half_m=128)):
        with pytest.raises(F.F3RError):
            F.Solver(ctx, A, **bad)
