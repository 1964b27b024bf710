"""Host-side checks of the learned SDAINV correction: the block-diagonal
training stack, and the PyTorch fp64 reference (tests/learned_ref.py) the
GPU kernels are compared with, pinned by finite differences and by its
untrained form being plain SDAINV.  No GPU is needed."""
import numpy as np
import pytest
import torch

import f3r_b200 as F
from f3r_b200.learned import block_diag, LAYOUT, N_PARAMS
import learned_ref as R


def small_system(nt=4, seeds=(1, 2)):
    A = block_diag([F.diffusion7(nt, nt, nt, 1.5, 6.0, s).scale() for s in seeds])
    Z, Wt = A.sdainv()
    return A, Z, Wt


def test_layout_is_contiguous():
    off = 0
    for k, (o, s) in LAYOUT.items():
        assert o == off, k
        off += int(np.prod(s))
    assert off == N_PARAMS == 5192
    assert R.LAYOUT == LAYOUT


def test_block_diag_is_the_stack():
    mats = [F.stencil27(3, 3, 3), F.diffusion7(4, 3, 2, 1.0, 2.0, 7)]
    S = block_diag(mats)
    dense = np.zeros(S.shape)
    r, i, v = S.arrays()
    for row in range(len(r) - 1):
        dense[row, i[r[row]:r[row + 1]]] = v[r[row]:r[row + 1]]
    off = 0
    want = np.zeros_like(dense)
    for M in mats:
        mr, mi, mv = M.arrays()
        for row in range(len(mr) - 1):
            want[off + row, off + mi[mr[row]:mr[row + 1]]] = mv[mr[row]:mr[row + 1]]
        off += len(mr) - 1
    assert np.array_equal(dense, want)


def test_stacked_7point_pattern_has_the_sdainv_slots():
    """every factor entry of a stacked 7-point system sits in one of the four
    slots (so the network corrects all of them)"""
    A, Z, Wt = small_system(12, (3, 4))
    nx, sxy = 12, 144
    z = Z.arrays()
    w = Wt.arrays()
    assert (R.slots(z, R.Z_OFFS(nx, sxy)) >= 0).all()
    assert (R.slots(w, R.W_OFFS(nx, sxy)) >= 0).all()


def test_reference_untrained_is_plain_sdainv():
    A, Z, Wt = small_system()
    rng = np.random.default_rng(0)
    n = A.shape[0]
    e = rng.standard_normal((2, n))
    r = np.stack([A.spmv(x) for x in e])
    p = np.zeros(N_PARAMS)
    p[:448] = rng.standard_normal(448)
    loss, _ = R.loss(p, A.arrays(), 4, 4, Z.arrays(), Wt.arrays(), r, e)
    # plain M = Z W^T
    zr, zi, zv = Z.arrays()
    wr, wi, wv = Wt.arrays()
    Zd = np.zeros((n, n))
    Wd = np.zeros((n, n))
    for row in range(n):
        Zd[row, zi[zr[row]:zr[row + 1]]] = zv[zr[row]:zr[row + 1]]
        Wd[row, wi[wr[row]:wr[row + 1]]] = wv[wr[row]:wr[row + 1]]
    y = (Zd @ Wd @ r.T).T
    want = np.mean(((y - e) ** 2).sum(1) / (e ** 2).sum(1))
    assert abs(loss - want) <= 1e-12 * want


def test_reference_gradient_against_finite_differences():
    A, Z, Wt = small_system(3, (5,))
    rng = np.random.default_rng(1)
    n = A.shape[0]
    e = rng.standard_normal((2, n))
    r = np.stack([A.spmv(x) for x in e])
    p = rng.standard_normal(N_PARAMS) * 0.1
    args = (A.arrays(), 3, 3, Z.arrays(), Wt.arrays(), r, e)
    _, g = R.loss(p, *args)
    for k in (3, 450, 600, 4610, 4700, 5185):  # one weight or bias of each block
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (R.loss(pp, *args)[0] - R.loss(pm, *args)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k])), (k, fd, g[k])
