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
