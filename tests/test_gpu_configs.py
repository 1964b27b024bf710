"""The reference's two F3R configurations on the GPU against the reference's
own solves of the same systems (tests/golden/solves.npz, recorded from the
reference compiled in place):

  * BJ-ILU(0) + CSR (work/src/f3r.cpp:195-248) on the 64^3 27-point hpcg
    matrix with 112 blocks -- the CPU configuration, on the GPU;
  * SDAINV + SELL-C-sigma (work/src/f3r-gpu.cpp:210-265) on the 192^3
    nonsymmetric 27-point matrix with C = 32, sigma = 256 -- the benchmark.

Parity: the outer residual history, step by step, inside the reference's
envelope over five OpenMP summation orders widened by 0.3 decades
(tests/history_band.py), and an explicit FP64 relative residual below 1e-10."""
import numpy as np
import pytest

import f3r_b200 as F
from oracle import oracle as O
from history_band import CASES, violations
from test_gpu_history import gpu_history
from test_oracle_pins import golden_system

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return F.Context(0)


def _check(ctx, name):
    sol = golden_system(name)[-1]
    if name + "_env" not in sol:
        pytest.skip(f"{name} not in the golden set (gen_golden.py --big, --envelope --big)")
    hist, res, err, sol = gpu_history(ctx, name)
    assert res.is_solved and res.expl_rel_res < 1e-10
    bad = violations(hist, sol, name)
    assert not bad, (bad, hist)
    assert err < 1e-8


def test_c1_bjilu_64(ctx):
    """CSR, block-Jacobi ILU(0) over 112 blocks, c = 64 (f3r.cpp:195-248)"""
    assert CASES["bjilu_hpcg64"]["ilu_blocks"] == 112
    _check(ctx, "bjilu_hpcg64")


def test_c2_sdainv_sell_192(ctx):
    """SELL-C-sigma, C = 32, sigma = 256, SDAINV, c = 64 (f3r-gpu.cpp:210-265)"""
    assert CASES["sdainv_half192"]["sell_sigma"] == 256
    _check(ctx, "sdainv_half192")
