"""Step-by-step parity of outer residual histories with the reference.

The reference's own history is not reproducible to better than a fraction of
a decade: its fp16 inner levels round differently whenever the summation order
of a reduction changes, and OpenMP changes that order with the thread count.
tests/golden/gen_golden.py --envelope therefore records every golden solve at
1, 2, 3, 4 and 8 threads (<name>_env, one row per thread count; up to 64 for
the depth ablations whose fp16-vector level sums its dot products in fp16,
one partial sum per thread, so that their accuracy depends on the count).  A history
from this library (or from the oracle) is in band when

  * its length is within one step of the shortest and longest reference run;
  * at every step k that some reference run reaches, its implicit relative
    residual lies inside [min_k, max_k] of the reference runs, widened by
    MARGIN decades on each side -- the lower side only while the reference's
    residual is still above the stop tolerance: on the step that crosses it,
    how far below 1e-10 a solve lands is set by the noise floor of its fp16
    levels, which fp32 accumulation lowers.

The margin covers what the reference's own five summation orders do not: this
library accumulates fp16 products in fp32 where the reference accumulates in
fp16 (its _Float16 / __half arithmetic), which moves each fp16 result by up to
one rounding, and sums its reductions in a fixed two-level tree.

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


# Golden solves whose reference arithmetic this library deliberately improves on, so that only the
# upper side of the band applies: F2H's 64-vector fp16 level, whose dot products and norms the
# reference sums in fp16 (its Gram-Schmidt loses orthogonality: 6 to 10 outer steps depending on
# the thread count), this library in fp32 (4 steps).  tests/test_oracle_pins.py shows that the
# restatement in the reference's fp16 arithmetic reproduces the reference's history.
ONE_SIDED = {"f2h_hpgmp16"}


def band(sol, name):
    """(lo, hi, shortest, longest) of the reference's runs of a golden solve"""
    env = np.asarray(sol[name + "_env"], np.float64)
    lens = (~np.isnan(env)).sum(axis=1)
    return np.nanmin(env, axis=0), np.nanmax(env, axis=0), int(lens.min()), int(lens.max())


def violations(hist, sol, name, margin=MARGIN):
    """the ways a history leaves the band (an empty list when it is in band)"""
    lo, hi, lmin, lmax = band(sol, name)
    hist = np.asarray(hist, np.float64)
    out = []
    one = name in ONE_SIDED
    if not ((one or lmin - 1 <= len(hist)) and len(hist) <= lmax + 1):
        out.append(f"{len(hist)} steps, the reference {lmin}..{lmax}")
    f = 10.0 ** margin
    for k in range(min(len(hist), len(lo))):
        if not ((one or lo[k] < TOL or lo[k] / f <= hist[k]) and hist[k] <= hi[k] * f):
            out.append(f"step {k + 1}: {hist[k]:.3e} outside [{lo[k] / f:.3e}, {hi[k] * f:.3e}]")
    return out


def spread(sol, name):
    """log10 width of the reference's own band at each step"""
    lo, hi, _, _ = band(sol, name)
    return np.log10(hi) - np.log10(lo)
