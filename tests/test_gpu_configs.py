"""The reference's two F3R configurations on the GPU against the reference's
own solves of the same systems (tests/golden/solves.npz, recorded from the
reference compiled in place):

  * BJ-ILU(0) + CSR (work/src/f3r.cpp:195-248) on the 64^3 27-point hpcg
    matrix with 112 blocks -- the CPU configuration, on the GPU;
  * SDAINV + SELL-C-sigma (work/src/f3r-gpu.cpp:210-265) on the 192^3
    nonsymmetric 27-point matrix with C = 32, sigma = 256 -- the benchmark.

Parity: outer iteration counts within one step of the reference, explicit
FP64 relative residual below 1e-10."""
import numpy as np
import pytest

import f3r_b200 as F
from oracle import oracle as O
from test_oracle_pins import golden_system

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return F.Context(0)


def _solve(ctx, name, **kw):
    r, i, v, b, xs, sol = golden_system(name)
    if name + "_iters" not in sol:
        pytest.skip(f"{name} not in the golden set (gen_golden.py --big)")
    A = F.HostMatrix.from_csr(r, i, v)
    S = F.Solver(ctx, A, rel_tol=1e-10, **kw)
    x = np.zeros(len(b))
    res = S.solve(b, x)
    S.close()
    return res, int(sol[name + "_iters"]), np.linalg.norm(x - xs) / np.linalg.norm(xs), sol[name + "_hist"]


def test_c1_bjilu_64(ctx):
    res, ref_iters, err, _ = _solve(ctx, "bjilu_hpcg64", precond=F.PRECOND_ILU0_BJ, ilu_blocks=112, c=64)
    assert res.is_solved and res.expl_rel_res < 1e-10
    assert abs(res.res_iter - ref_iters) <= 1, (res.res_iter, ref_iters)
    assert err < 1e-8


def test_c2_sdainv_sell_192(ctx):
    res, ref_iters, err, hist = _solve(ctx, "sdainv_half192", sell_sigma=256, c=64)
    assert res.is_solved and res.expl_rel_res < 1e-10
    assert abs(res.res_iter - ref_iters) <= 1, (res.res_iter, ref_iters)
    assert err < 1e-8
