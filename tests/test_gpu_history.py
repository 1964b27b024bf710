"""Outer residual histories on the GPU, step by step, against the reference's
own solves of the same systems (tests/golden/solves.npz).

Each golden solve is repeated with the matching configuration (history_band.
CASES); the implicit relative residual |e(j)| / ||b|| that cond() sees after
every outer step must stay inside the reference's envelope over five OpenMP
summation orders, widened by history_band.MARGIN decades (the band is
explained in tests/history_band.py).  The 64^3 and 192^3 configurations are
checked the same way in test_gpu_configs.py."""
import numpy as np
import pytest

import f3r_b200 as F
from history_band import CASES, violations
from test_oracle_pins import golden_system

pytestmark = pytest.mark.gpu

SMALL = [k for k in CASES if k not in ("bjilu_hpcg64", "sdainv_half192")]


@pytest.fixture(scope="module")
def ctx():
    return F.Context(0)


def gpu_history(ctx, name, **extra):
    """(history, result, solution error) of the golden system solved on the GPU to 1e-10"""
    r, i, v, b, xs, sol = golden_system(name)
    S = F.Solver(ctx, F.HostMatrix.from_csr(r, i, v), rel_tol=1e-10, **{**CASES[name], **extra})
    nb = np.linalg.norm(b)
    hist = []

    def cond(k, e):
        if k > 0:
            hist.append(e / nb)
        return e / nb < 1e-10

    x = np.zeros(len(b))
    res = S.solve(b, x, cond)
    S.close()
    return np.array(hist), res, np.linalg.norm(x - xs) / np.linalg.norm(xs), sol


@pytest.mark.parametrize("name", SMALL)
def test_history_in_reference_band(ctx, name):
    hist, res, err, sol = gpu_history(ctx, name)
    if name + "_env" not in sol:
        pytest.skip("no envelope recorded (gen_golden.py --envelope)")
    assert res.is_solved and res.expl_rel_res < 1e-10
    assert len(hist) == res.res_iter
    bad = violations(hist, sol, name)
    assert not bad, (name, bad, hist)
    assert err < 1e-7


@pytest.mark.parametrize("name", ["sdainv_hpgmp16", "sdainv_diffs25_48"])
def test_history_same_in_every_layout(ctx, name):
    """the layouts change no sum: the history is identical in packed, offset-
    aligned and CSR storage (sigma 1)"""
    hs = [gpu_history(ctx, name, **kw)[0] for kw in (dict(sell_align=0), dict(sell_align=1), dict(format=1))]
    assert all(np.array_equal(hs[0], h) for h in hs[1:]), hs
