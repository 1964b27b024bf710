"""The learned SDAINV correction on the GPU (f3r_learned_*): the fp32
training kernels' loss and gradient against the PyTorch fp64 reference
(tests/learned_ref.py), the BF16 tensor-core inference against the fp32
forward pass, the untrained network as plain SDAINV, the solver built from
given factors, and what training gains on held-out systems."""
import numpy as np
import pytest

import f3r_b200 as F
from f3r_b200.learned import Learned, block_diag, training_set, solve_with_fallback, N_PARAMS
import learned_ref as R

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return F.Context(0)


def stacked(nt, seeds):
    A = block_diag([F.diffusion7(nt, nt, nt, 1.5, 6.0, s).scale() for s in seeds])
    Z, Wt = A.sdainv()
    return A, Z, Wt


def random_params(L, seed, scale=0.05):
    rng = np.random.default_rng(seed)
    p = L.params.astype(np.float64)
    p[4672:] = rng.standard_normal(N_PARAMS - 4672) * scale  # W3, b3 (zero at creation)
    p[448:512] = rng.standard_normal(64) * 0.1                # b1
    p[4608:4672] = rng.standard_normal(64) * 0.1              # b2
    return p.astype(np.float32)


def test_untrained_network_is_plain_sdainv(ctx):
    A, Z, Wt = stacked(8, (1, 2))
    L = Learned(ctx, seed=3)
    for bf16, engine in ((True, "tcgen05"), (True, "mma.sync"), (False, "tcgen05")):
        Zc, Wc = L.correct(A, 8, 8, Z, Wt, bf16=bf16, engine=engine)
        assert np.array_equal(Zc.arrays()[2], Z.arrays()[2])
        assert np.array_equal(Wc.arrays()[2], Wt.arrays()[2])


def test_loss_and_gradient_match_reference(ctx):
    nt = 5
    A, Z, Wt = stacked(nt, (4, 5, 6))
    n = A.shape[0]
    rng = np.random.default_rng(2)
    e = rng.standard_normal((3, n))
    r = np.stack([A.spmv(x) for x in e])
    L = Learned(ctx, seed=1)
    p = random_params(L, 7)
    L.params = p
    L.set_data(A, nt, nt, Z, Wt, r, e)
    loss, g = L.evaluate(grad=True)
    want_loss, want_g = R.loss(p.astype(np.float64), A.arrays(), nt, nt, Z.arrays(), Wt.arrays(), r, e)
    assert abs(loss - want_loss) <= 1e-5 * want_loss, (loss, want_loss)
    for name, (o, s) in R.LAYOUT.items():
        k = int(np.prod(s))
        got, want = g[o:o + k].astype(np.float64), want_g[o:o + k]
        assert np.linalg.norm(got - want) <= 1e-4 * np.linalg.norm(want) + 1e-7, name
    # evaluate leaves the parameters and the accumulated gradient untouched
    assert np.array_equal(L.params, p)
    assert L.evaluate() == pytest.approx(loss, rel=1e-12)


def test_forward_and_bf16_inference_match_reference(ctx):
    nt = 9
    A, Z, Wt = stacked(nt, (8,))
    L = Learned(ctx, seed=2)
    p = random_params(L, 9, scale=0.2)
    L.params = p
    want = R.delta(p.astype(np.float64), A.arrays(), nt, nt)
    scale = np.max(np.abs(want))
    Zc, Wc, d32 = L.correct(A, nt, nt, Z, Wt, bf16=False, want_delta=True)
    assert np.max(np.abs(d32 - want)) <= 1e-5 * scale
    Zb, Wb, d16 = L.correct(A, nt, nt, Z, Wt, bf16=True, want_delta=True)
    # bf16 weights and activations (8-bit mantissa), fp32 accumulation over 64 terms
    assert np.max(np.abs(d16 - want)) <= 3e-2 * scale
    _, _, dm = L.correct(A, nt, nt, Z, Wt, bf16=True, want_delta=True, engine="mma.sync")
    assert np.max(np.abs(dm - want)) <= 3e-2 * scale
    # corrected values v (1 + delta) on the fixed pattern
    zr, zi, zv = Z.arrays()
    rows = np.repeat(np.arange(len(zr) - 1), np.diff(zr))
    sl = R.slots((zr, zi, zv), R.Z_OFFS(nt, nt * nt))
    expect = np.where(sl >= 0, zv * (1 + d32[rows, np.maximum(sl, 0)].astype(np.float64)), zv)
    assert np.allclose(Zc.arrays()[2], expect, rtol=1e-15, atol=0)
    assert np.array_equal(Zb.arrays()[1], zi)


@pytest.mark.parametrize("nt", [9, 64, 71])
def test_tcgen05_inference_matches_mma_sync(ctx, nt):
    """The tcgen05 kernel (128-row tiles, TMEM accumulators) and the mma.sync
    kernel round the same operands to bf16 and accumulate in fp32.  They
    differ in the order of the fp32 sums and in the bias, which the tcgen05
    kernel adds inside the MMA as two bf16 parts (16 of its bits) where the
    mma.sync kernel adds it in fp32; either can move an activation by one
    bf16 step.  729 rows: one ragged tile per warpgroup; 64^3 and 71^3: more
    tiles than warpgroups (the persistent loop), 71^3 ragged."""
    A = F.diffusion7(nt, nt, nt, 1.5, 6.0, 5).scale()
    Z, Wt = A.sdainv()
    L = Learned(ctx, seed=4)
    p = random_params(L, 10, scale=0.2)
    L.params = p
    want = R.delta(p.astype(np.float64), A.arrays(), nt, nt)
    scale = np.max(np.abs(want))
    _, _, dt = L.correct(A, nt, nt, Z, Wt, bf16=True, want_delta=True, engine="tcgen05")
    _, _, dm = L.correct(A, nt, nt, Z, Wt, bf16=True, want_delta=True, engine="mma.sync")
    assert np.all(np.isfinite(dt))
    assert np.max(np.abs(dt - want)) <= 3e-2 * scale
    assert np.max(np.abs(dt - dm)) <= 1e-2 * scale
    # most rows see no activation rounding flip at all
    assert np.mean(np.all(np.abs(dt - dm) <= 1e-5 * scale, axis=1)) > 0.8
    us_t = L.time_inference(A, nt, nt, Z, Wt, engine="tcgen05", reps=5)
    us_m = L.time_inference(A, nt, nt, Z, Wt, engine="mma.sync", reps=5)
    assert us_t > 0 and us_m > 0


def test_inference_engine_is_checked(ctx):
    A, Z, Wt = stacked(8, (1,))
    L = Learned(ctx, seed=3)
    with pytest.raises(ValueError):
        L.correct(A, 8, 8, Z, Wt, engine="wmma")


def test_solver_from_given_factors_is_the_plain_solver(ctx):
    A = F.diffusion7(20, 20, 20, 1.5, 6.0, 11).scale()
    b = A.spmv(F.random_uniform(3, -1, 1, A.shape[0]))
    kw = dict(rel_tol=1e-10, m2=8, m3=4, m4=2, c=64)
    x1, x2 = np.zeros(len(b)), np.zeros(len(b))
    r1 = F.Solver(ctx, A, **kw).solve(b, x1)
    r2 = F.Solver(ctx, A, factors=A.sdainv(), **kw).solve(b, x2)
    assert r1.is_solved and r1.res_iter == r2.res_iter
    assert np.array_equal(x1, x2)


@pytest.fixture(scope="module")
def trained(ctx):
    """the network trained on the solver's residual / error pairs of 16
    seeded 12^3 fields (300 Adam steps), with its loss history"""
    ts = training_set(ctx, seeds=range(16), nt=12, rel_tol=1e-10)
    assert ts.r.shape == (7, 16 * 12 ** 3)
    L = Learned(ctx, seed=0)
    L.set_data(**ts.data())
    losses = L.train(300, lr=2e-3)
    return L, losses


def test_training_gains_on_held_out_systems(ctx, trained):
    """Trained on the solver's residual / error pairs of 16 seeded 12^3
    fields, the correction lowers the training loss; on held-out 32^3 fields
    the learned solve reaches 1e-10 without the plain fallback, and its
    residual after a fixed number of outer steps is compared with plain
    SDAINV's."""
    L, losses = trained
    assert np.all(np.isfinite(losses))
    final = L.evaluate()
    assert final < losses[0], (losses[0], final)
    ratios = []
    for seed in (1001, 1002):
        A = F.diffusion7(32, 32, 32, 1.5, 6.0, seed).scale()
        Z, Wt = A.sdainv()
        Zc, Wc = L.correct(A, 32, 32, Z, Wt)
        b = A.spmv(F.random_uniform(seed, -1, 1, A.shape[0]))
        x = np.zeros(len(b))
        res, fell_back = solve_with_fallback(ctx, A, b, x, (Zc, Wc), (Z, Wt), rel_tol=1e-10)
        assert res.is_solved and res.expl_rel_res < 1e-9 and not fell_back
        Sp = F.Solver(ctx, A, factors=(Z, Wt), rel_tol=1e-10)
        Sl = F.Solver(ctx, A, factors=(Zc, Wc), rel_tol=1e-10)
        k = max(1, Sp.solve(b, np.zeros(len(b))).res_iter - 1)
        rp = Sp.solve(b, np.zeros(len(b)), cond=lambda i, e: i >= k).expl_rel_res
        rl = Sl.solve(b, np.zeros(len(b)), cond=lambda i, e: i >= k).expl_rel_res
        ratios.append(rp / rl)
    print("residual gain at fixed outer steps", ratios)
    assert np.exp(np.mean(np.log(ratios))) > 1.0, ratios


def test_learned_batched_time_to_solution(ctx, trained):
    """Time to 1e-10 over 8 held-out 32^3 fields: the learned factors solved
    as one same-pattern batch (f3r_batch) against plain SDAINV solved one
    field after another, each solver built beforehand; host wall clock with
    the device synchronised on both sides, best of 3.  Every field reaches
    1e-10 in both, and the learned batch takes at most 1/1.5 of the time."""
    import time
    import torch
    L, _ = trained
    seeds = range(2001, 2009)
    fields = [F.diffusion7(32, 32, 32, 1.5, 6.0, s).scale() for s in seeds]
    plain = [A.sdainv() for A in fields]
    learned = [L.correct(A, 32, 32, Z, Wt) for A, (Z, Wt) in zip(fields, plain)]
    bs = [A.spmv(F.random_uniform(s, -1, 1, A.shape[0])) for A, s in zip(fields, seeds)]
    kw = dict(rel_tol=1e-10, m2=8, m3=4, m4=2, c=64)
    solvers = [F.Solver(ctx, A, factors=f, **kw) for A, f in zip(fields, plain)]
    batch = F.Batch(ctx, fields, factors=learned, **kw)

    def run_plain():
        xs = [np.zeros(len(b)) for b in bs]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = [S.solve(b, x) for S, b, x in zip(solvers, bs, xs)]
        torch.cuda.synchronize()
        return time.perf_counter() - t0, res

    def run_batch():
        xs = [np.zeros(len(b)) for b in bs]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = batch.solve(bs, xs)
        torch.cuda.synchronize()
        return time.perf_counter() - t0, res

    run_plain(), run_batch()  # warm-up: work buffers and graphs
    tp, rp = min((run_plain() for _ in range(3)), key=lambda t: t[0])
    tb, rb = min((run_batch() for _ in range(3)), key=lambda t: t[0])
    assert all(r.is_solved and r.expl_rel_res < 1e-9 for r in rp + rb)
    print(f"plain one after another {tp * 1e3:.2f} ms, learned batch {tb * 1e3:.2f} ms: {tp / tb:.2f}x")
    assert tb * 1.5 <= tp, (tp, tb)
    batch.close()
    for S in solvers:
        S.close()


def test_fallback_to_plain_sdainv(ctx):
    """factors whose values are noise (an untrustworthy correction) leave the
    solve short of 1e-10 within its 20 outer steps or break it down; the
    FP64 outer residual catches it and plain SDAINV finishes the solve"""
    A = F.diffusion7(16, 16, 16, 1.5, 6.0, 4).scale()
    Z, Wt = A.sdainv()
    zr, zi, zv = Z.arrays()
    wr, wi, wv = Wt.arrays()
    rng = np.random.default_rng(9)
    bad = (F.HostMatrix.from_csr(zr, zi, rng.standard_normal(len(zv))),
           F.HostMatrix.from_csr(wr, wi, rng.standard_normal(len(wv))))
    b = A.spmv(F.random_uniform(4, -1, 1, A.shape[0]))
    x = np.zeros(len(b))
    res, fell_back = solve_with_fallback(ctx, A, b, x, bad, (Z, Wt), rel_tol=1e-10, max_restarts=1, m_outer=20)
    assert fell_back and res.is_solved and res.expl_rel_res < 1e-9


def test_learned_rejects_bad_input(ctx):
    with pytest.raises(F.F3RError):
        Learned(ctx, hidden=32)
    L = Learned(ctx)
    with pytest.raises(F.F3RError, match="no training data"):
        L.evaluate()
    A, Z, Wt = stacked(4, (1,))
    n = A.shape[0]
    with pytest.raises(F.F3RError, match="zero"):
        L.set_data(A, 4, 4, Z, Wt, np.zeros((1, n)), np.zeros((1, n)))
    with pytest.raises(F.F3RError, match="strides"):
        L.correct(A, 100, 100, Z, Wt)
    with pytest.raises(ValueError):
        L.set_data(A, 4, 4, Z, Wt, np.zeros((1, n + 1)), np.zeros((1, n + 1)))
    bad = np.ones(N_PARAMS, np.float32)
    bad[7] = np.nan
    with pytest.raises(F.F3RError, match="non-finite"):
        L.params = bad
    with pytest.raises(F.F3RError, match="SDAINV"):
        F.Solver(ctx, A, factors=(Z, Wt), precond=F.PRECOND_ILU0_BJ)
