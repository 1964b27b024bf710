"""Failure paths on the GPU, none of which faults or hangs the device: a
bounded device wait that runs out (a flag that nothing sets) ends with a
TIMEOUT status and leaves the context usable; a non-finite right-hand side
is reported as a breakdown; the restart cap ends a solve as unsolved.  The
reference has no error statuses (it prints and exits, or divides unchecked,
solver/gmres.hpp:31-33)."""
import time

import numpy as np
import pytest

import f3r_b200 as F

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return F.Context(0)


def small_solve(ctx):
    A = F.stencil27(12, 12, 12, 2, 0.5).scale()
    b = A.spmv(F.random_uniform(1, -1, 1, A.shape[0]))
    x = np.zeros(len(b))
    return F.Solver(ctx, A, rel_tol=1e-10).solve(b, x)


def test_wait_runs_out_and_context_stays_usable(ctx):
    ctx.wait_probe(True, 200)  # a set flag: returns at once
    t0 = time.perf_counter()
    with pytest.raises(F.F3RError) as e:
        ctx.wait_probe(False, 200)  # nothing sets it: the bound ends the wait
    dt = time.perf_counter() - t0
    assert e.value.status == 7 and "bound" in str(e.value)
    assert 0.15 < dt < 5.0, dt
    ctx.wait_probe(True, 200)  # the error word is clear again
    r = small_solve(ctx)
    assert r.is_solved and r.expl_rel_res < 1e-10
    with pytest.raises(F.F3RError):
        ctx.wait_probe(False, 0)


def test_non_finite_rhs_is_a_breakdown(ctx):
    A = F.stencil27(12, 12, 12, 2, 0.5).scale()
    b = A.spmv(F.random_uniform(2, -1, 1, A.shape[0]))
    b[100] = np.nan
    S = F.Solver(ctx, A, rel_tol=1e-10)
    with pytest.raises(F.F3RError) as e:
        S.solve(b, np.zeros(len(b)))
    assert e.value.status == 5, e.value
    # the same solver and context solve a finite system afterwards
    b[100] = 0.0
    x = np.zeros(len(b))
    r = S.solve(b, x)
    assert r.is_solved and r.expl_rel_res < 1e-10


def test_restart_cap_ends_unsolved(ctx):
    A = F.stencil27(16, 16, 16, 2, 0.5).scale()
    b = A.spmv(F.random_uniform(3, -1, 1, A.shape[0]))
    x = np.zeros(len(b))
    r = F.Solver(ctx, A, rel_tol=1e-14, m_outer=2, max_restarts=1).solve(b, x)
    assert not r.is_solved and r.res_iter == 2 and r.restarts == 1
    assert np.isfinite(r.expl_rel_res) and r.expl_rel_res > 1e-14
