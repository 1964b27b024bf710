"""Precision stress (the C3 configuration at a small size): a 7-point
diffusion whose coefficients exp(g) span many orders of magnitude does not fit
fp16 as generated; after the diagonal scaling every level's product stays
within its precision of the fp64 product, and the nested solve still reaches
an fp64 relative residual of 1e-10."""
import numpy as np
import pytest
import torch

import f3r_b200 as F

pytestmark = pytest.mark.gpu


def test_precision_stress_levels():
    A = F.diffusion7(40, 40, 40, 2.5, 8.0, 3)
    raw = np.abs(A.arrays()[2])
    assert raw.max() / raw.min() > 1e5          # far outside what fp16's 2^-24..65504 can hold well
    A.scale()
    r, i, v = A.arrays()
    assert np.abs(v).max() <= 1.0 + 1e-12       # D^-1/2 A D^-1/2: the diagonal is 1
    n = A.shape[0]
    xs = F.random_uniform(0, -1.0, 1.0, n)
    b = A.spmv(xs)
    S = F.Solver(F.Context(0), A, rel_tol=1e-10, c=8, sell_align=1)
    z = torch.from_numpy(xs).cuda()
    ys = {}
    for name, vt, zt, yt in (("f64", F.F64, z, torch.float64), ("f32", F.F32, z.float(), torch.float32),
                             ("f16A_f32x", F.F16, z.float(), torch.float32),
                             ("f16A_f16x", F.F16, z.half(), torch.float16)):
        y = torch.empty(n, dtype=yt, device="cuda")
        S.operate(zt, y, val_t=vt)
        ys[name] = y.double().cpu().numpy()
    ref = ys["f64"]
    assert np.allclose(ref, b)
    rel = {k: np.linalg.norm(y - ref) / np.linalg.norm(ref) for k, y in ys.items()}
    # each level within its own precision (rounding of values and inputs, 7 terms per row)
    assert rel["f32"] < 1e-6
    assert rel["f16A_f32x"] < 5e-3
    assert rel["f16A_f16x"] < 1e-2
    x = np.zeros(n)
    res = S.solve(b, x)
    assert res.is_solved and res.expl_rel_res < 1e-10
    assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-6
