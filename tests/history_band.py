"""Step-by-step parity of outer residual histories with the reference.

The reference's own history is not reproducible to better than a fraction of
a decade: its fp16 inner levels round differently whenever the summation order
of a reduction changes, and OpenMP changes that order with the thread count.
tests/golden/gen_golden.py --envelope therefore records every golden solve at
1, 2, 3, 4 and 8 threads (<name>_env, one row per thread count; up to 64 for
the depth ablations whose fp16-vector level sums its dot products in fp16,
one partial sum per thread, so that their accuracy depends on the count).

This library computes the same algorithm in a deliberately different
arithmetic: fp16 storage with fp32 accumulation where the reference
accumulates in fp16 (and fp32 dot products where its fp16-vector levels use
fp16).  That makes its inner solves more accurate, and on some systems its
histories lie below every reference run (the 64^3 block-Jacobi ILU(0) solve
and F2H, for example).  gen_golden.py --oracle records the oracle's history
in that arithmetic (<name>_oracle, oracle/f3r_oracle.c, which restates the
reference's algorithm step by step), and the band spans it beside the
reference's runs.  A history is in band when

  * its length is within one step of the shortest and longest run;
  * at every step k that some run reaches, its implicit relative residual
    lies inside [min_k, max_k] of the runs, widened on each side by MARGIN
    decades, or by half the runs' own spread log10(max_k / min_k) where that
    is wider -- the lower side only while the runs are still above the stop
    tolerance: on the step that crosses it, how far below 1e-10 a solve lands
    is set by the noise floor of its fp16 levels.

The margin covers what the runs do not: the summation order of this library's
reductions (a fixed two-level tree) against the oracle's sequential sums.  A
step whose runs already disagree by a decade (the s-step variants, whose
monomial bases amplify rounding) is one where summation order moves the
history that much, hence the spread term.

The solver settings that reproduce each golden solve's configuration are in
CASES (keyword arguments of f3r_b200.Solver).
"""
import numpy as np

MARGIN = 0.3  # decades
TOL = 1e-10   # the stop tolerance of every golden solve

# the configuration of each golden solve (tests/golden/gen_golden.py: solve_cases)
CASES = {
    "sdainv_hpgmp16": dict(c=8),
    "sdainv_half16": dict(c=8),
    "sdainv_diff12": dict(c=8),
    "sdainv_diffs25_48": dict(c=64),
    "bjilu_hpcg16": dict(c=8, precond=1, ilu_blocks=16, format=1),
    "static_hpgmp16": dict(c=8, precond=1, ilu_blocks=16, format=1, m2=8, m3=4, m4=2, static_weight=1.2),
    "depth3_hpgmp16": dict(c=8, precond=1, ilu_blocks=16, format=1, m2=8, m3=8, m4=1, static_weight=1.0),
    "depth2_hpgmp16": dict(c=8, precond=1, ilu_blocks=16, format=1, m2=64, m3=0, m4=1, static_weight=1.0),
    "sstep1_hpgmp16": dict(c=8, inner_sstep=1),
    "sstep2_hpgmp16": dict(c=8, inner_sstep=2),
    "sstep3_hpgmp16": dict(c=8, inner_sstep=3),
    # the fp16-vector depth ablations (depth.cpp:122-167): block-Jacobi ILU(0) applied directly
    "f4_hpgmp16": dict(c=8, precond=1, ilu_blocks=16, format=1, m2=8, m3=4, half_m=2, m4=1, static_weight=1.0),
    "f3h_hpgmp16": dict(c=8, precond=1, ilu_blocks=16, format=1, m2=8, m3=0, half_m=8, m4=1, static_weight=1.0),
    "f2h_hpgmp16": dict(c=8, precond=1, ilu_blocks=16, format=1, m2=0, m3=0, half_m=64, m4=1, static_weight=1.0),
    "bjilu_hpcg64": dict(c=64, precond=1, ilu_blocks=112, format=1),
    "sdainv_half192": dict(c=64, sell_sigma=256),
}


def runs(sol, name, with_oracle=True):
    """the reference's runs of a golden solve and, when recorded and asked
    for, the oracle's run in the library's arithmetic: one row each, NaN past
    a run's last step"""
    env = np.asarray(sol[name + "_env"], np.float64)
    if with_oracle and name + "_oracle" in sol:
        o = np.asarray(sol[name + "_oracle"], np.float64)
        w = max(env.shape[1], len(o))
        rows = np.full((env.shape[0] + 1, w), np.nan)
        rows[:env.shape[0], :env.shape[1]] = env
        rows[-1, :len(o)] = o
        env = rows
    return env


def band(sol, name, with_oracle=True):
    """(lo, hi, shortest, longest) over the runs of a golden solve"""
    env = runs(sol, name, with_oracle)
    lens = (~np.isnan(env)).sum(axis=1)
    return np.nanmin(env, axis=0), np.nanmax(env, axis=0), int(lens.min()), int(lens.max())


def violations(hist, sol, name, margin=MARGIN, with_oracle=True):
    """the ways a history leaves the band (an empty list when it is in band);
    with_oracle = False: the reference's runs alone (for the oracle in the
    reference's own arithmetic)"""
    lo, hi, lmin, lmax = band(sol, name, with_oracle)
    hist = np.asarray(hist, np.float64)
    out = []
    if not (lmin - 1 <= len(hist) <= lmax + 1):
        out.append(f"{len(hist)} steps, the runs {lmin}..{lmax}")
    for k in range(min(len(hist), len(lo))):
        f = 10.0 ** max(margin, 0.5 * np.log10(hi[k] / lo[k]))
        if not ((lo[k] < TOL or lo[k] / f <= hist[k]) and hist[k] <= hi[k] * f):
            out.append(f"step {k + 1}: {hist[k]:.3e} outside [{lo[k] / f:.3e}, {hi[k] * f:.3e}]")
    return out


def spread(sol, name):
    """log10 width of the runs' band at each step"""
    lo, hi, _, _ = band(sol, name)
    return np.log10(hi) - np.log10(lo)
